// Multi-right-hand-side FP64 kernels: the matrix is streamed once per block
// of RB right-hand sides instead of once per vector.
//
// Vector operands are row-major blocks (entry (i, r) at i * RB + r), so the
// RB values that multiply one matrix column are contiguous: the caller's
// column-major X is transposed into that form first, and the coefficient
// workspaces (t, uy, partial sums) use it throughout.  Outputs go through
// (row stride, column stride) pairs, so the same kernel writes row-major
// coefficients or the caller's column-major Y.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "kernels_f64.cuh"
#include "layout.hpp"

namespace hlrc {

constexpr int MR_RB = 8;   // right-hand sides per block (N-form, finish, workspaces)
constexpr int MR_TB = 4;   // right-hand sides per tile T-form launch

// xr[i * RB + r] = X[i + (r0 + r) * ldx] for r < nr, 0 for nr <= r < RB
__global__ void k_rows_from_cols(const double* __restrict__ X, int64_t ldx, int64_t n, int r0, int nr,
                                 double* __restrict__ xr) {
    const int64_t idx = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (idx >= n * MR_RB) return;
    const int64_t i = idx / MR_RB;
    const int r = int(idx % MR_RB);
    xr[idx] = r < nr ? X[i + int64_t(r0 + r) * ldx] : 0.0;
}

struct OutMap {            // output element (i, r) lives at base[i * rs + r * cs]
    double* base;
    int64_t rs, cs;
    int nr;                // valid right-hand sides
};

// N-form, RB right-hand sides: one CTA per output tile, lane owns rows
// 2l, 2l+1 for all RB vectors; fixed-order cross-warp sum in shared memory.
template <int W>
__global__ void __launch_bounds__(W * 32)
k_nform_f64_mr(const NSeg* __restrict__ segs, const NChunk* __restrict__ chunks, const double* __restrict__ A,
               const double* __restrict__ vx, const double* __restrict__ vt, OutMap om, double alpha, int add) {
    constexpr int RB = MR_RB;
    __shared__ double red[W][TILE][RB];
    const NSeg sg = segs[blockIdx.x];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int r = 2 * lane;
    const bool active = r < sg.ld;
    double acc0[RB], acc1[RB];
#pragma unroll
    for (int k = 0; k < RB; ++k) acc0[k] = acc1[k] = 0.0;
    for (uint32_t c = sg.cb + warp; c < sg.ce; c += W) {
        const NChunk ch = chunks[c];
        const double* v = (ch.v_off & VEC_T) ? vt + size_t(ch.v_off & ~VEC_T) * RB : vx + size_t(ch.v_off) * RB;
        const double* a = A + ch.a_off + r;
        double2 m[NCHUNK];
#pragma unroll
        for (int j = 0; j < NCHUNK; ++j)
            m[j] = (active && j < ch.nc) ? ld_stream(a + size_t(j) * sg.ld) : make_double2(0.0, 0.0);
#pragma unroll
        for (int j = 0; j < NCHUNK; ++j) {
            if (j >= ch.nc) break;
            const double2* vj = reinterpret_cast<const double2*>(v + size_t(j) * RB);
#pragma unroll
            for (int k = 0; k < RB / 2; ++k) {
                const double2 w = __ldg(vj + k);
                acc0[2 * k] = fma(m[j].x, w.x, acc0[2 * k]);
                acc0[2 * k + 1] = fma(m[j].x, w.y, acc0[2 * k + 1]);
                acc1[2 * k] = fma(m[j].y, w.x, acc1[2 * k]);
                acc1[2 * k + 1] = fma(m[j].y, w.y, acc1[2 * k + 1]);
            }
        }
    }
#pragma unroll
    for (int k = 0; k < RB; ++k) {
        red[warp][r][k] = acc0[k];
        red[warp][r + 1][k] = acc1[k];
    }
    __syncthreads();
    for (int t = threadIdx.x; t < TILE * RB; t += W * 32) {
        const int row = t % TILE, k = t / TILE;
        if (row >= sg.rows || k >= om.nr) continue;
        double s = 0.0;
#pragma unroll
        for (int w = 0; w < W; ++w) s += red[w][row][k];
        double* o = om.base + int64_t(sg.out + row) * om.rs + int64_t(k) * om.cs;
        if (add) *o += alpha * s;
        else *o = s;
    }
}

// Tile T-form for MR_TB right-hand sides r0 .. r0+3 of the row-major input
// (stride MR_RB): 8 columns x 4 vectors = 32 partials per lane, one
// transpose-reduction, lane l then holds (column l / 4, vector l % 4).
template <int W>
__global__ void __launch_bounds__(W * 32)
k_ttform_f64_mr(const TTSeg* __restrict__ segs, const TTChunk* __restrict__ chunks, const double* __restrict__ A,
                const double* __restrict__ vin, int r0, OutMap om, double* __restrict__ part, double alpha,
                int add) {
    constexpr int TB = MR_TB;
    const TTSeg sg = segs[blockIdx.x];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int r = 2 * lane;
    const bool active = r < sg.ld;
    double x0[TB], x1[TB];
#pragma unroll
    for (int k = 0; k < TB; ++k) {
        x0[k] = r < sg.rows ? __ldg(vin + size_t(sg.v_off + r) * MR_RB + r0 + k) : 0.0;
        x1[k] = r + 1 < sg.rows ? __ldg(vin + size_t(sg.v_off + r + 1) * MR_RB + r0 + k) : 0.0;
    }
    for (uint32_t c = sg.cb + warp; c < sg.ce; c += W) {
        const TTChunk ch = chunks[c];
        const double* a = A + ch.a_off + r;
        double2 m[TCOLS];
#pragma unroll
        for (int j = 0; j < TCOLS; ++j)
            m[j] = (active && j < ch.nc) ? ld_stream(a + size_t(j) * sg.ld) : make_double2(0.0, 0.0);
        double p[TCOLS * TB];
#pragma unroll
        for (int j = 0; j < TCOLS; ++j)
#pragma unroll
            for (int k = 0; k < TB; ++k) p[j * TB + k] = fma(m[j].y, x1[k], m[j].x * x0[k]);
        TransposeReduce<TCOLS * TB, 16>::run(p, lane);
        const int j = lane / TB, k = lane % TB;
        if (j < ch.nc && r0 + k < om.nr) {
            if (ch.flags & TT_DIRECT) {
                double* o = om.base + int64_t(ch.out + j) * om.rs + int64_t(r0 + k) * om.cs;
                if (add) *o += alpha * p[0];
                else *o = p[0];
            } else {
                part[size_t(ch.out + j) * MR_RB + r0 + k] = p[0];
            }
        }
    }
}

// Sums per-tile partials (row-major, MR_RB vectors) of multi-tile outputs.
__global__ void __launch_bounds__(256)
k_ttfinish_f64_mr(const TGroup* __restrict__ groups, int ngroups, const double* __restrict__ part, OutMap om,
                  double alpha, int add) {
    const int gid = blockIdx.x * 8 + (threadIdx.x >> 5);
    if (gid >= ngroups) return;
    const int lane = threadIdx.x & 31;
    const TGroup g = groups[gid];
    const uint32_t n = g.nc * MR_RB;
    for (uint32_t q = lane; q < n; q += 32) {
        const uint32_t j = q / MR_RB, k = q % MR_RB;
        if (int(k) >= om.nr) continue;
        const double* p = part + size_t(g.slot0) * MR_RB + q;
        double s0 = 0.0, s1 = 0.0;
        uint32_t i = 0;
        for (; i + 2 <= g.nslots; i += 2) {
            s0 += p[size_t(i) * n];
            s1 += p[size_t(i + 1) * n];
        }
        for (; i < g.nslots; ++i) s0 += p[size_t(i) * n];
        const double s = s0 + s1;
        double* o = om.base + int64_t(g.out + j) * om.rs + int64_t(k) * om.cs;
        if (add) *o += alpha * s;
        else *o = s;
    }
}

// ------------------------------------------------- reduced-precision stores
// Multi-RHS kernels for FP32 / scaled 16-bit stores: lane owns rows 2l, 2l+1
// (a pair load of 8 or 4 bytes), products and sums inside a chunk in FP32,
// chunk results accumulated in FP64.  Work items are the stores' packs (up
// to two chunks each).

// rows r, r+1 of a column (r even: the pair is aligned to two elements)
template <int FMT>
__device__ __forceinline__ float2 ld_pair(const uint8_t* col, int r) {
    if constexpr (FMT == FMT_F32) {
        return __ldcs(reinterpret_cast<const float2*>(col) + (r >> 1));
    } else if constexpr (FMT == FMT_F16) {
        const unsigned u = __ldcs(reinterpret_cast<const unsigned*>(col) + (r >> 1));
        __half2 h;
        memcpy(&h, &u, 4);
        return __half22float2(h);
    } else {
        const unsigned u = __ldcs(reinterpret_cast<const unsigned*>(col) + (r >> 1));
        return make_float2(__uint_as_float(u << 16), __uint_as_float(u & 0xffff0000u));
    }
}

template <int W, int FMT>
__global__ void __launch_bounds__(W * 32)
k_nform_q_mr(const NSeg* __restrict__ segs, const QNPack* __restrict__ packs, const uint8_t* __restrict__ A,
             const double* __restrict__ vx, const double* __restrict__ vt, OutMap om, double alpha, int add) {
    constexpr int RB = MR_RB;
    __shared__ double red[W][TILE][RB];
    const NSeg sg = segs[blockIdx.x];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int r = 2 * lane;
    const bool active = r < sg.ld;
    const size_t colb = size_t(sg.ld) * fmt_bytes(FMT);
    double acc0[RB], acc1[RB];
#pragma unroll
    for (int k = 0; k < RB; ++k) acc0[k] = acc1[k] = 0.0;
    for (uint32_t c = sg.cb + warp; c < sg.ce; c += W) {
        const QNPack pk = packs[c];
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            const QNChunk& part = pk.p[q];
            if (part.nc == 0) continue;
            const uint8_t* a = A + size_t(part.a16) * 16;
            const double* v = (part.v_off & VEC_T) ? vt + size_t(part.v_off & ~VEC_T) * RB
                                                   : vx + size_t(part.v_off) * RB;
            float s0[RB], s1[RB];
#pragma unroll
            for (int k = 0; k < RB; ++k) s0[k] = s1[k] = 0.f;
            for (int j = 0; j < part.nc; ++j) {
                const float2 m = active ? ld_pair<FMT>(a + size_t(j) * colb, r) : make_float2(0.f, 0.f);
                const double2* vj = reinterpret_cast<const double2*>(v + size_t(j) * RB);
#pragma unroll
                for (int k = 0; k < RB / 2; ++k) {
                    const double2 w = __ldg(vj + k);
                    const float w0 = float(w.x), w1 = float(w.y);
                    s0[2 * k] = fmaf(m.x, w0, s0[2 * k]);
                    s0[2 * k + 1] = fmaf(m.x, w1, s0[2 * k + 1]);
                    s1[2 * k] = fmaf(m.y, w0, s1[2 * k]);
                    s1[2 * k + 1] = fmaf(m.y, w1, s1[2 * k + 1]);
                }
            }
            const double sc = part.scale;
#pragma unroll
            for (int k = 0; k < RB; ++k) {
                acc0[k] = fma(sc, double(s0[k]), acc0[k]);
                acc1[k] = fma(sc, double(s1[k]), acc1[k]);
            }
        }
    }
#pragma unroll
    for (int k = 0; k < RB; ++k) {
        red[warp][r][k] = acc0[k];
        red[warp][r + 1][k] = acc1[k];
    }
    __syncthreads();
    for (int t = threadIdx.x; t < TILE * RB; t += W * 32) {
        const int row = t % TILE, k = t / TILE;
        if (row >= sg.rows || k >= om.nr) continue;
        double s = 0.0;
#pragma unroll
        for (int w = 0; w < W; ++w) s += red[w][row][k];
        double* o = om.base + int64_t(sg.out + row) * om.rs + int64_t(k) * om.cs;
        if (add) *o += alpha * s;
        else *o = s;
    }
}

template <int W, int FMT>
__global__ void __launch_bounds__(W * 32)
k_ttform_q_mr(const TTSeg* __restrict__ segs, const QTTPack* __restrict__ packs, const uint8_t* __restrict__ A,
              const double* __restrict__ vin, int r0, OutMap om, double* __restrict__ part, double alpha, int add) {
    constexpr int TB = MR_TB;
    const TTSeg sg = segs[blockIdx.x];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int r = 2 * lane;
    const bool active = r < sg.ld;
    const size_t colb = size_t(sg.ld) * fmt_bytes(FMT);
    float x0[TB], x1[TB];
#pragma unroll
    for (int k = 0; k < TB; ++k) {
        x0[k] = r < sg.rows ? float(__ldg(vin + size_t(sg.v_off + r) * MR_RB + r0 + k)) : 0.f;
        x1[k] = r + 1 < sg.rows ? float(__ldg(vin + size_t(sg.v_off + r + 1) * MR_RB + r0 + k)) : 0.f;
    }
    for (uint32_t c = sg.cb + warp; c < sg.ce; c += W) {
        const QTTPack pk = packs[c];
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            const QTTChunk& ch = pk.p[q];
            for (int j0 = 0; j0 < ch.nc; j0 += TCOLS) {
                const uint8_t* a = A + size_t(ch.a16) * 16 + size_t(j0) * colb;
                float2 m[TCOLS];
#pragma unroll
                for (int j = 0; j < TCOLS; ++j)
                    m[j] = (active && j0 + j < ch.nc) ? ld_pair<FMT>(a + size_t(j) * colb, r) : make_float2(0.f, 0.f);
                float p[TCOLS * TB];
#pragma unroll
                for (int j = 0; j < TCOLS; ++j)
#pragma unroll
                    for (int k = 0; k < TB; ++k) p[j * TB + k] = fmaf(m[j].y, x1[k], m[j].x * x0[k]);
                TransposeReduce<TCOLS * TB, 16, float>::run(p, lane);
                const int j = j0 + lane / TB, k = lane % TB;
                if (j < ch.nc && r0 + k < om.nr) {
                    const double val = double(ch.scale) * double(p[0]);
                    if (ch.flags & TT_DIRECT) {
                        double* o = om.base + int64_t(ch.out + j) * om.rs + int64_t(r0 + k) * om.cs;
                        if (add) *o += alpha * val;
                        else *o = val;
                    } else {
                        part[size_t(ch.out + j) * MR_RB + r0 + k] = val;
                    }
                }
            }
        }
    }
}

}  // namespace hlrc
