// Tensor-core multi-right-hand-side kernels for 16-bit stores (scaled FP16 /
// BF16 chunks), MR_RB = 8 right-hand sides per launch.
//
// With 8 right-hand sides a chunk product is a small dense contraction, run
// as mma.sync m16n8k16 tiles with FP32 accumulation.  The vector operand is
// split into two 16-bit terms, hi = round(s*v) and lo = round(s*v - hi), with
// a power-of-two scale s per chunk (N-form) or input tile (tile T-form) and
// right-hand side, so the product keeps about 22 significant bits of v
// (FP16) or 16 (BF16) and the storage rounding of the matrix stays the
// dominant error.  Chunk results are scaled back and accumulated in FP64,
// exactly where the CUDA-core kernels accumulate.
//
// Fragment placement.  The contraction index of an MMA may be mapped to
// storage rows or columns in any order, as long as both operands use the
// same map, and the output rows of a tile in any order the epilogue knows.
// The maps below make every lane's matrix load one 16-byte run of 8 rows
// of one column (column-major chunks, ld a multiple of 8):
//   tile T-form (t = V^T x): contraction = tile rows.  In k-tile kt = 2h + s,
//     lane (g, t) takes rows 32h + 8t + 4s + {0,1} as fragment k = 2t, 2t+1
//     and rows +{2,3} as k = 2t+8, 2t+9; output rows of the MMA are chunk
//     columns 16*mt + g and 16*mt + g + 8.
//   N-form (y = U t): contraction = chunk columns 16*kt + k; output rows of
//     m-tile i are tile rows 8g + 2i (fragment row g) and 8g + 2i + 1
//     (fragment row g + 8), so a lane's 16 bytes of column c hold its A
//     entries of all four m-tiles; a byte permute turns pairs of rows of one
//     column into the fragment's pairs of columns of one row.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "kernels_mr.cuh"
#include "kernels_q.cuh"
#include "layout.hpp"

namespace hlrc {

template <int FMT> struct TcOp;

template <> struct TcOp<FMT_F16> {
    static __device__ __forceinline__ float round16(float v) { return __half2float(__float2half_rn(v)); }
    static __device__ __forceinline__ uint32_t pack(float lo, float hi) {
        const __half2 h = __floats2half2_rn(lo, hi);
        uint32_t u;
        memcpy(&u, &h, 4);
        return u;
    }
    static __device__ __forceinline__ void mma(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                               uint32_t b0, uint32_t b1) {
        asm(
            "mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
            "{%0,%1,%2,%3};\n"
            : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
            : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
    }
};

template <> struct TcOp<FMT_BF16> {
    static __device__ __forceinline__ float round16(float v) { return __bfloat162float(__float2bfloat16_rn(v)); }
    static __device__ __forceinline__ uint32_t pack(float lo, float hi) {
        const __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
        uint32_t u;
        memcpy(&u, &h, 4);
        return u;
    }
    static __device__ __forceinline__ void mma(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                               uint32_t b0, uint32_t b1) {
        asm(
            "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
            "{%0,%1,%2,%3};\n"
            : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
            : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
    }
};

// Power-of-two scale bringing amax into [2^13, 2^14) (1 for amax == 0 or not
// finite); *inv receives its inverse.
__device__ __forceinline__ double tc_scale(double amax, double* inv) {
    if (!(amax > 0.0) || !(amax < 1e300) || amax < 1e-290) {
        *inv = 1.0;
        return 1.0;
    }
    int e;
    frexp(amax, &e);
    *inv = ldexp(1.0, e - 14);
    return ldexp(1.0, 14 - e);
}

// hi/lo 16-bit terms of the scaled pair (v0, v1), packed as MMA operands
template <int FMT>
__device__ __forceinline__ void tc_split(double v0, double v1, double s, uint32_t& hi, uint32_t& lo) {
    using O = TcOp<FMT>;
    const float f0 = float(v0 * s), f1 = float(v1 * s);
    const float h0 = O::round16(f0), h1 = O::round16(f1);
    hi = O::pack(h0, h1);
    lo = O::pack(f0 - h0, f1 - h1);
}

__device__ __forceinline__ uint4 ld_u4_stream(const uint8_t* p) { return __ldcs(reinterpret_cast<const uint4*>(p)); }

__device__ __forceinline__ uint32_t u4_word(const uint4& u, int i) {
    return i == 0 ? u.x : (i == 1 ? u.y : (i == 2 ? u.z : u.w));
}

// Tile T-form, 8 right-hand sides, 16-bit chunks on tensor cores.  One CTA
// per input tile; warps take packs round-robin; each chunk result is complete
// (the contraction covers the whole tile) and goes straight to its output or
// to its partial slot.
template <int W, int FMT>
__global__ void __launch_bounds__(W * 32)
k_ttform_tc(const TTSeg* __restrict__ segs, const QTTPack* __restrict__ packs, const uint8_t* __restrict__ A,
            const double* __restrict__ vin, OutMap om, double* __restrict__ part, double alpha, int add) {
    using O = TcOp<FMT>;
    const TTSeg sg = segs[blockIdx.x];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, t = lane & 3;
    // x entries of the lane: rows 32h + 8t + i (h = 0, 1; i < 8), right-hand side g
    double xv[16];
    double amax = 0.0;
#pragma unroll
    for (int h = 0; h < 2; ++h)
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int row = 32 * h + 8 * t + i;
            const double v = row < sg.rows ? __ldg(vin + size_t(sg.v_off + row) * MR_RB + g) : 0.0;
            xv[8 * h + i] = v;
            amax = fmax(amax, fabs(v));
        }
    amax = fmax(amax, __shfl_xor_sync(0xffffffffu, amax, 1));
    amax = fmax(amax, __shfl_xor_sync(0xffffffffu, amax, 2));
    double inv;
    const double s = tc_scale(amax, &inv);
    // dequantisation of the vector for right-hand sides 2t and 2t+1 (the
    // output columns of this lane's accumulator fragment)
    const double inv0 = __shfl_sync(0xffffffffu, inv, 8 * t);
    const double inv1 = __shfl_sync(0xffffffffu, inv, 8 * t + 4);
    uint32_t bh[4][2], bl[4][2];
#pragma unroll
    for (int kt = 0; kt < 4; ++kt) {
        const int base = 8 * (kt >> 1) + 4 * (kt & 1);
        tc_split<FMT>(xv[base], xv[base + 1], s, bh[kt][0], bl[kt][0]);
        tc_split<FMT>(xv[base + 2], xv[base + 3], s, bh[kt][1], bl[kt][1]);
    }
    const size_t colb = size_t(sg.ld) * 2;
    const int n0 = 2 * t, n1 = 2 * t + 1;
    for (uint32_t c = sg.cb + warp; c < sg.ce; c += W) {
        const QTTPack pk = ld_pack(packs + c);
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            const QTTChunk& ch = pk.p[q];
            if (ch.nc == 0) continue;
            const uint8_t* a = A + size_t(ch.a16) * 16;
            for (int mt = 0; mt * 16 < ch.nc; ++mt) {
                const int c0 = 16 * mt + g, c1 = c0 + 8;
                float d[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int row0 = 32 * h + 8 * t;
                    const uint4 z = make_uint4(0u, 0u, 0u, 0u);
                    const uint4 L0 = (row0 < sg.ld && c0 < ch.nc) ? ld_u4_stream(a + c0 * colb + 2 * row0) : z;
                    const uint4 L1 = (row0 < sg.ld && c1 < ch.nc) ? ld_u4_stream(a + c1 * colb + 2 * row0) : z;
                    O::mma(d, L0.x, L1.x, L0.y, L1.y, bh[2 * h][0], bh[2 * h][1]);
                    O::mma(d, L0.x, L1.x, L0.y, L1.y, bl[2 * h][0], bl[2 * h][1]);
                    O::mma(d, L0.z, L1.z, L0.w, L1.w, bh[2 * h + 1][0], bh[2 * h + 1][1]);
                    O::mma(d, L0.z, L1.z, L0.w, L1.w, bl[2 * h + 1][0], bl[2 * h + 1][1]);
                }
                const double f0 = double(ch.scale) * inv0, f1 = double(ch.scale) * inv1;
                const double val[4] = {double(d[0]) * f0, double(d[1]) * f1, double(d[2]) * f0, double(d[3]) * f1};
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    const int col = e < 2 ? c0 : c1;
                    const int n = (e & 1) ? n1 : n0;
                    if (col >= ch.nc || n >= om.nr) continue;
                    if (ch.flags & TT_DIRECT) {
                        double* o = om.base + int64_t(ch.out + col) * om.rs + int64_t(n) * om.cs;
                        if (add) *o += alpha * val[e];
                        else *o = val[e];
                    } else {
                        part[size_t(ch.out + col) * MR_RB + n] = val[e];
                    }
                }
            }
        }
    }
}

// N-form, 8 right-hand sides, 16-bit chunks on tensor cores.  One CTA per
// output tile; lane (g, t) accumulates tile rows 8g .. 8g+7 for right-hand
// sides 2t, 2t+1 in FP64; fixed-order cross-warp sum in shared memory.
template <int W, int FMT>
__global__ void __launch_bounds__(W * 32)
k_nform_tc(const NSeg* __restrict__ segs, const QNPack* __restrict__ packs, const uint8_t* __restrict__ A,
           const double* __restrict__ vx, const double* __restrict__ vt, OutMap om, double alpha, int add) {
    using O = TcOp<FMT>;
    __shared__ double red[W][TILE][MR_RB];
    const NSeg sg = segs[blockIdx.x];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, t = lane & 3;
    const bool rows_ok = 8 * g < sg.ld;
    const size_t colb = size_t(sg.ld) * 2;
    double acc[8][2];
#pragma unroll
    for (int r = 0; r < 8; ++r) acc[r][0] = acc[r][1] = 0.0;
    for (uint32_t c = sg.cb + warp; c < sg.ce; c += W) {
        const QNPack pk = ld_pack(packs + c);
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            const QNChunk& ch = pk.p[q];
            if (ch.nc == 0) continue;
            const double* v = (ch.v_off & VEC_T) ? vt + size_t(ch.v_off & ~VEC_T) * MR_RB
                                                 : vx + size_t(ch.v_off) * MR_RB;
            const int nkt = ch.nc > 16 ? 2 : 1;
            // vector operand: columns 16kt + 2t + {0, 1, 8, 9}, right-hand side g
            double bv[2][4];
            double amax = 0.0;
#pragma unroll
            for (int kt = 0; kt < 2; ++kt)
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int col = 16 * kt + 2 * t + (j & 1) + 8 * (j >> 1);
                    const double x = col < ch.nc ? __ldg(v + size_t(col) * MR_RB + g) : 0.0;
                    bv[kt][j] = x;
                    amax = fmax(amax, fabs(x));
                }
            amax = fmax(amax, __shfl_xor_sync(0xffffffffu, amax, 1));
            amax = fmax(amax, __shfl_xor_sync(0xffffffffu, amax, 2));
            double inv;
            const double s = tc_scale(amax, &inv);
            const double f0 = double(ch.scale) * __shfl_sync(0xffffffffu, inv, 8 * t);
            const double f1 = double(ch.scale) * __shfl_sync(0xffffffffu, inv, 8 * t + 4);
            const uint8_t* a = A + size_t(ch.a16) * 16;
            float d[4][4];
#pragma unroll
            for (int i = 0; i < 4; ++i) d[i][0] = d[i][1] = d[i][2] = d[i][3] = 0.f;
#pragma unroll
            for (int kt = 0; kt < 2; ++kt) {
                if (kt >= nkt) break;
                uint32_t bh0, bl0, bh1, bl1;
                tc_split<FMT>(bv[kt][0], bv[kt][1], s, bh0, bl0);
                tc_split<FMT>(bv[kt][2], bv[kt][3], s, bh1, bl1);
                uint4 L[4];
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int col = 16 * kt + 2 * t + (j & 1) + 8 * (j >> 1);
                    L[j] = (rows_ok && col < ch.nc) ? ld_u4_stream(a + col * colb + 16 * g)
                                                    : make_uint4(0u, 0u, 0u, 0u);
                }
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const uint32_t w0 = u4_word(L[0], i), w1 = u4_word(L[1], i);
                    const uint32_t w2 = u4_word(L[2], i), w3 = u4_word(L[3], i);
                    const uint32_t a0 = __byte_perm(w0, w1, 0x5410), a1 = __byte_perm(w0, w1, 0x7632);
                    const uint32_t a2 = __byte_perm(w2, w3, 0x5410), a3 = __byte_perm(w2, w3, 0x7632);
                    O::mma(d[i], a0, a1, a2, a3, bh0, bh1);
                    O::mma(d[i], a0, a1, a2, a3, bl0, bl1);
                }
            }
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                acc[2 * i][0] = fma(double(d[i][0]), f0, acc[2 * i][0]);
                acc[2 * i][1] = fma(double(d[i][1]), f1, acc[2 * i][1]);
                acc[2 * i + 1][0] = fma(double(d[i][2]), f0, acc[2 * i + 1][0]);
                acc[2 * i + 1][1] = fma(double(d[i][3]), f1, acc[2 * i + 1][1]);
            }
        }
    }
#pragma unroll
    for (int r = 0; r < 8; ++r) {
        red[warp][8 * g + r][2 * t] = acc[r][0];
        red[warp][8 * g + r][2 * t + 1] = acc[r][1];
    }
    __syncthreads();
    for (int i = threadIdx.x; i < TILE * MR_RB; i += W * 32) {
        const int row = i % TILE, k = i / TILE;
        if (row >= sg.rows || k >= om.nr) continue;
        double sum = 0.0;
#pragma unroll
        for (int w = 0; w < W; ++w) sum += red[w][row][k];
        double* o = om.base + int64_t(sg.out + row) * om.rs + int64_t(k) * om.cs;
        if (add) *o += alpha * sum;
        else *o = sum;
    }
}


// ------------------------------------------------------------- FP32 chunks
// FP32 chunks use m16n8k8 TF32 tiles with the usual three-term split
// (a_big b_big + a_big b_small + a_small b_big, each term rounded to TF32),
// which keeps about 21 significant bits of both operands; the vector gets
// the same per-right-hand-side power-of-two scale as on the 16-bit path.
// Fragment placement (ld a multiple of 4, a lane loads 4 rows of a column):
//   N-form: contraction = chunk columns 8*kt + {t, t+4}; lane (g, t) loads
//     rows 4g .. 4g+3 and 32+4g .. 32+4g+3, and m-tile i takes rows
//     4g + 2i, 4g + 2i + 1 (i < 2) or 32 + 4g + 2(i-2) + {0, 1} as its
//     fragment rows g and g + 8.
//   tile T-form: contraction = tile rows; in k-step s = 2j + u, fragment
//     k = t is row 16j + 4t + 2u and k = t + 4 is row 16j + 4t + 2u + 1.

__device__ __forceinline__ uint32_t to_tf32(float v) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;\n" : "=r"(r) : "f"(v));
    return r;
}

// big / small TF32 terms of a float
__device__ __forceinline__ void tf32_split(float v, uint32_t& big, uint32_t& small) {
    big = to_tf32(v);
    small = to_tf32(v - __uint_as_float(big));
}

__device__ __forceinline__ void mma_tf32(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3, uint32_t b0,
                                         uint32_t b1) {
    asm("mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// d += A B for the three-term split of A = (a0..a3 as floats) and B = (bb, bs)
__device__ __forceinline__ void mma_tf32x3(float (&d)[4], float a0, float a1, float a2, float a3, const uint32_t (&bb)[2],
                                           const uint32_t (&bs)[2]) {
    uint32_t ab[4], as[4];
    tf32_split(a0, ab[0], as[0]);
    tf32_split(a1, ab[1], as[1]);
    tf32_split(a2, ab[2], as[2]);
    tf32_split(a3, ab[3], as[3]);
    mma_tf32(d, as[0], as[1], as[2], as[3], bb[0], bb[1]);
    mma_tf32(d, ab[0], ab[1], ab[2], ab[3], bs[0], bs[1]);
    mma_tf32(d, ab[0], ab[1], ab[2], ab[3], bb[0], bb[1]);
}

__device__ __forceinline__ float u4_f(const uint4& u, int i) { return __uint_as_float(u4_word(u, i)); }

template <int W>
__global__ void __launch_bounds__(W * 32)
k_ttform_tc32(const TTSeg* __restrict__ segs, const QTTPack* __restrict__ packs, const uint8_t* __restrict__ A,
              const double* __restrict__ vin, OutMap om, double* __restrict__ part, double alpha, int add) {
    const TTSeg sg = segs[blockIdx.x];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, t = lane & 3;
    // x entries of the lane: rows 16j + 4t + i (j, i < 4), right-hand side g
    double xv[16];
    double amax = 0.0;
#pragma unroll
    for (int j = 0; j < 4; ++j)
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int row = 16 * j + 4 * t + i;
            const double v = row < sg.rows ? __ldg(vin + size_t(sg.v_off + row) * MR_RB + g) : 0.0;
            xv[4 * j + i] = v;
            amax = fmax(amax, fabs(v));
        }
    amax = fmax(amax, __shfl_xor_sync(0xffffffffu, amax, 1));
    amax = fmax(amax, __shfl_xor_sync(0xffffffffu, amax, 2));
    double inv;
    const double s = tc_scale(amax, &inv);
    const double inv0 = __shfl_sync(0xffffffffu, inv, 8 * t);
    const double inv1 = __shfl_sync(0xffffffffu, inv, 8 * t + 4);
    // k-step 2j + u: b0 = row 16j + 4t + 2u, b1 = the next row
    uint32_t bb[8][2], bs[8][2];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const int j = k >> 1, u = k & 1;
        tf32_split(float(xv[4 * j + 2 * u] * s), bb[k][0], bs[k][0]);
        tf32_split(float(xv[4 * j + 2 * u + 1] * s), bb[k][1], bs[k][1]);
    }
    const size_t colb = size_t(sg.ld) * 4;
    const int n0 = 2 * t, n1 = 2 * t + 1;
    for (uint32_t c = sg.cb + warp; c < sg.ce; c += W) {
        const QTTPack pk = ld_pack(packs + c);
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            const QTTChunk& ch = pk.p[q];
            if (ch.nc == 0) continue;
            const uint8_t* a = A + size_t(ch.a16) * 16;
            const int c0 = g, c1 = g + 8;   // an FP32 chunk has at most 16 columns: one m-tile
            float d[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int row0 = 16 * j + 4 * t;
                const uint4 z = make_uint4(0u, 0u, 0u, 0u);
                const uint4 L0 = (row0 < sg.ld && c0 < ch.nc) ? ld_u4_stream(a + c0 * colb + 4 * row0) : z;
                const uint4 L1 = (row0 < sg.ld && c1 < ch.nc) ? ld_u4_stream(a + c1 * colb + 4 * row0) : z;
                mma_tf32x3(d, u4_f(L0, 0), u4_f(L1, 0), u4_f(L0, 1), u4_f(L1, 1), bb[2 * j], bs[2 * j]);
                mma_tf32x3(d, u4_f(L0, 2), u4_f(L1, 2), u4_f(L0, 3), u4_f(L1, 3), bb[2 * j + 1], bs[2 * j + 1]);
            }
            const double f0 = double(ch.scale) * inv0, f1 = double(ch.scale) * inv1;
            const double val[4] = {double(d[0]) * f0, double(d[1]) * f1, double(d[2]) * f0, double(d[3]) * f1};
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                const int col = e < 2 ? c0 : c1;
                const int n = (e & 1) ? n1 : n0;
                if (col >= ch.nc || n >= om.nr) continue;
                if (ch.flags & TT_DIRECT) {
                    double* o = om.base + int64_t(ch.out + col) * om.rs + int64_t(n) * om.cs;
                    if (add) *o += alpha * val[e];
                    else *o = val[e];
                } else {
                    part[size_t(ch.out + col) * MR_RB + n] = val[e];
                }
            }
        }
    }
}

template <int W>
__global__ void __launch_bounds__(W * 32)
k_nform_tc32(const NSeg* __restrict__ segs, const QNPack* __restrict__ packs, const uint8_t* __restrict__ A,
             const double* __restrict__ vx, const double* __restrict__ vt, OutMap om, double alpha, int add) {
    __shared__ double red[W][TILE][MR_RB];
    const NSeg sg = segs[blockIdx.x];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, t = lane & 3;
    const bool lo_ok = 4 * g < sg.ld, hi_ok = 32 + 4 * g < sg.ld;
    const size_t colb = size_t(sg.ld) * 4;
    // accumulators: rows 4g + r and 32 + 4g + r (r < 4) -> acc[r] / acc[4 + r]
    double acc[8][2];
#pragma unroll
    for (int r = 0; r < 8; ++r) acc[r][0] = acc[r][1] = 0.0;
    for (uint32_t c = sg.cb + warp; c < sg.ce; c += W) {
        const QNPack pk = ld_pack(packs + c);
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            const QNChunk& ch = pk.p[q];
            if (ch.nc == 0) continue;
            const double* v = (ch.v_off & VEC_T) ? vt + size_t(ch.v_off & ~VEC_T) * MR_RB
                                                 : vx + size_t(ch.v_off) * MR_RB;
            const int nkt = ch.nc > 8 ? 2 : 1;
            // vector operand: columns 8kt + t and 8kt + t + 4, right-hand side g
            double bv[2][2];
            double amax = 0.0;
#pragma unroll
            for (int kt = 0; kt < 2; ++kt)
#pragma unroll
                for (int j = 0; j < 2; ++j) {
                    const int col = 8 * kt + t + 4 * j;
                    const double x = col < ch.nc ? __ldg(v + size_t(col) * MR_RB + g) : 0.0;
                    bv[kt][j] = x;
                    amax = fmax(amax, fabs(x));
                }
            amax = fmax(amax, __shfl_xor_sync(0xffffffffu, amax, 1));
            amax = fmax(amax, __shfl_xor_sync(0xffffffffu, amax, 2));
            double inv;
            const double s = tc_scale(amax, &inv);
            const double f0 = double(ch.scale) * __shfl_sync(0xffffffffu, inv, 8 * t);
            const double f1 = double(ch.scale) * __shfl_sync(0xffffffffu, inv, 8 * t + 4);
            const uint8_t* a = A + size_t(ch.a16) * 16;
            float d[4][4];
#pragma unroll
            for (int i = 0; i < 4; ++i) d[i][0] = d[i][1] = d[i][2] = d[i][3] = 0.f;
#pragma unroll
            for (int kt = 0; kt < 2; ++kt) {
                if (kt >= nkt) break;
                uint32_t bb[2], bs[2];
                tf32_split(float(bv[kt][0] * s), bb[0], bs[0]);
                tf32_split(float(bv[kt][1] * s), bb[1], bs[1]);
                const int ca = 8 * kt + t, cb = ca + 4;
                const uint4 z = make_uint4(0u, 0u, 0u, 0u);
                const bool oka = ca < ch.nc, okb = cb < ch.nc;
                const uint4 La0 = (lo_ok && oka) ? ld_u4_stream(a + ca * colb + 16 * g) : z;
                const uint4 Lb0 = (lo_ok && okb) ? ld_u4_stream(a + cb * colb + 16 * g) : z;
                const uint4 La1 = (hi_ok && oka) ? ld_u4_stream(a + ca * colb + 128 + 16 * g) : z;
                const uint4 Lb1 = (hi_ok && okb) ? ld_u4_stream(a + cb * colb + 128 + 16 * g) : z;
                mma_tf32x3(d[0], u4_f(La0, 0), u4_f(La0, 1), u4_f(Lb0, 0), u4_f(Lb0, 1), bb, bs);
                mma_tf32x3(d[1], u4_f(La0, 2), u4_f(La0, 3), u4_f(Lb0, 2), u4_f(Lb0, 3), bb, bs);
                mma_tf32x3(d[2], u4_f(La1, 0), u4_f(La1, 1), u4_f(Lb1, 0), u4_f(Lb1, 1), bb, bs);
                mma_tf32x3(d[3], u4_f(La1, 2), u4_f(La1, 3), u4_f(Lb1, 2), u4_f(Lb1, 3), bb, bs);
            }
            // m-tile i: fragment row g -> local row 2i, row g + 8 -> 2i + 1
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                acc[2 * i][0] = fma(double(d[i][0]), f0, acc[2 * i][0]);
                acc[2 * i][1] = fma(double(d[i][1]), f1, acc[2 * i][1]);
                acc[2 * i + 1][0] = fma(double(d[i][2]), f0, acc[2 * i + 1][0]);
                acc[2 * i + 1][1] = fma(double(d[i][3]), f1, acc[2 * i + 1][1]);
            }
        }
    }
    // local row l < 4 is tile row 4g + l, l >= 4 is 32 + 4g + (l - 4)
#pragma unroll
    for (int l = 0; l < 8; ++l) {
        const int row = (l < 4 ? 0 : 32) + 4 * g + (l & 3);
        red[warp][row][2 * t] = acc[l][0];
        red[warp][row][2 * t + 1] = acc[l][1];
    }
    __syncthreads();
    for (int i = threadIdx.x; i < TILE * MR_RB; i += W * 32) {
        const int row = i % TILE, k = i / TILE;
        if (row >= sg.rows || k >= om.nr) continue;
        double sum = 0.0;
#pragma unroll
        for (int w = 0; w < W; ++w) sum += red[w][row][k];
        double* o = om.base + int64_t(sg.out + row) * om.rs + int64_t(k) * om.cs;
        if (add) *o += alpha * sum;
        else *o = sum;
    }
}

}  // namespace hlrc
