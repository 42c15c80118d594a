// Reduced-precision (FP32 / scaled FP16 / scaled BF16 storage) versions of
// the N-form and tile T-form kernels.
//
// Every load is 16 bytes per lane whatever the format: a lane owns R = 16/e
// consecutive rows of a column (4 for FP32, 8 for 16-bit), G = 64/R lanes
// cover a 64-row tile column, and one warp instruction reads C = 32/G
// columns.  A work item is a pack of up to two chunks of one format with at
// most 8*C columns together (4 KB at full tile height), so a warp iteration
// moves as many bytes as the FP64 kernels'.  One launch handles one format.
// Products and the sums inside a pack are FP32; pack results are added to
// FP64 per-row accumulators, and y is accumulated in FP64 (HLR's compressed
// BLAS likewise decodes entries inside the GEMV loop: compress/fp32.hh:210-312,
// compress/bfp.hh:945-1100).
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "kernels_f64.cuh"
#include "layout.hpp"

namespace hlrc {

template <int FMT> struct QFmt;
template <> struct QFmt<FMT_F32> { static constexpr int R = 4, G = 16, C = 2, LOG_G = 4; };
template <> struct QFmt<FMT_F16> { static constexpr int R = 8, G = 8, C = 4, LOG_G = 3; };
template <> struct QFmt<FMT_BF16> { static constexpr int R = 8, G = 8, C = 4, LOG_G = 3; };
template <> struct QFmt<FMT_I16> { static constexpr int R = 8, G = 8, C = 4, LOG_G = 3; };
// 24-bit: a lane's 8 rows are 16 bytes of high parts plus 8 bytes of low parts
template <> struct QFmt<FMT_I24> { static constexpr int R = 8, G = 8, C = 4, LOG_G = 3; };

// Packed FP32 pairs (sm_100 fma / sub .f32x2: two FP32 operations per
// instruction) for the 16-bit integer format.
__device__ __forceinline__ uint64_t pk2(uint32_t lo, uint32_t hi) {
    uint64_t r;
    asm("mov.b64 %0, {%1, %2};\n" : "=l"(r) : "r"(lo), "r"(hi));
    return r;
}
__device__ __forceinline__ uint64_t pk2f(float lo, float hi) { return pk2(__float_as_uint(lo), __float_as_uint(hi)); }
__device__ __forceinline__ float2 upk2(uint64_t v) {
    float2 r;
    asm("mov.b64 {%0, %1}, %2;\n" : "=f"(r.x), "=f"(r.y) : "l"(v));
    return r;
}
__device__ __forceinline__ void fma2(uint64_t& d, uint64_t a, uint64_t b) {
    asm("fma.rn.f32x2 %0, %1, %2, %0;\n" : "+l"(d) : "l"(a), "l"(b));
}
__device__ __forceinline__ uint64_t sub2(uint64_t a, uint64_t b) {
    uint64_t d;
    asm("sub.rn.f32x2 %0, %1, %2;\n" : "=l"(d) : "l"(a), "l"(b));
    return d;
}


// 8 offset-binary 16-bit integers (16 loaded bytes) -> 4 exact packed float
// pairs: a value u = v + 2^15 becomes the low mantissa bits of 1.5 * 2^23,
// and one exact packed subtraction removes 1.5 * 2^23 + 2^15 (no integer
// conversion instruction).  Pair i holds rows 2i, 2i+1.
__device__ __forceinline__ void i16_pairs(const uint4& u, uint64_t (&p)[4]) {
    constexpr uint64_t BIAS = 0x4B4080004B408000ull;   // 1.5 * 2^23 + 2^15, twice
    const uint32_t w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
    for (int i = 0; i < 4; ++i)
        p[i] = sub2(pk2(__byte_perm(w[i], 0x4B400000u, 0x7610), __byte_perm(w[i], 0x4B400000u, 0x7632)), BIAS);
}

// 8 offset-binary 24-bit integers u = v + 2^22 < 2^23 (16 bytes of high
// parts h = u >> 8, 8 bytes of low parts l) -> 4 exact packed float pairs:
// the bytes l, h are placed under the exponent byte of 2^23 (u is the low 23
// mantissa bits of 2^23 + u) by two byte permutes per row pair plus one that
// interleaves the low parts with that exponent byte, and one packed
// subtraction removes 2^23 + 2^22.
__device__ __forceinline__ void i24_pairs(const uint4& hi, const uint2& lo, uint64_t (&p)[4]) {
    constexpr uint64_t BIAS = 0x4B4000004B400000ull;   // 2^23 + 2^22, twice
    const uint32_t h[4] = {hi.x, hi.y, hi.z, hi.w};
    const uint32_t w[2] = {lo.x, lo.y};
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        // [l(2i), 0x4B, l(2i+1), 0x4B]
        const uint32_t L = __byte_perm(w[i >> 1], 0x4B4B4B4Bu, (i & 1) ? 0x5342 : 0x5140);
        p[i] = sub2(pk2(__byte_perm(h[i], L, 0x5104), __byte_perm(h[i], L, 0x7326)), BIAS);
    }
}

// 16 loaded bytes -> R floats
template <int FMT>
__device__ __forceinline__ void unpack16(const uint4& u, float* f) {
    if constexpr (FMT == FMT_F32) {
        f[0] = __uint_as_float(u.x); f[1] = __uint_as_float(u.y);
        f[2] = __uint_as_float(u.z); f[3] = __uint_as_float(u.w);
    } else if constexpr (FMT == FMT_F16) {
        const unsigned w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            __half2 h;
            memcpy(&h, &w[i], 4);
            const float2 t = __half22float2(h);
            f[2 * i] = t.x;
            f[2 * i + 1] = t.y;
        }
    } else if constexpr (FMT == FMT_I16) {
        uint64_t p[4];
        i16_pairs(u, p);
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const float2 t = upk2(p[i]);
            f[2 * i] = t.x;
            f[2 * i + 1] = t.y;
        }
    } else {
        const unsigned w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            f[2 * i] = __uint_as_float(w[i] << 16);
            f[2 * i + 1] = __uint_as_float(w[i] & 0xffff0000u);
        }
    }
}

__device__ __forceinline__ QNPack ld_pack(const QNPack* p) {
    QNPack r;
    const uint4* s = reinterpret_cast<const uint4*>(p);
    const uint4 a = __ldg(s), b = __ldg(s + 1);
    memcpy(&r.p[0], &a, 16);
    memcpy(&r.p[1], &b, 16);
    return r;
}
__device__ __forceinline__ QTTPack ld_pack(const QTTPack* p) {
    QTTPack r;
    const uint4* s = reinterpret_cast<const uint4*>(p);
    const uint4 a = __ldg(s), b = __ldg(s + 1);
    memcpy(&r.p[0], &a, 16);
    memcpy(&r.p[1], &b, 16);
    return r;
}

// The lane's 8 loads of a pack: column j = g + C*i of the pack lies in part 0
// for j < n0, else in part 1.
// For 24-bit chunks ml gets the lane's 8 bytes of low parts (2*ld bytes into
// the column, 8 per lane).
template <int FMT>
__device__ __forceinline__ void load_pack(const uint8_t* A, uint32_t a0, uint32_t a1, int n0, int ntot, int ld,
                                          int lane, uint4* m, uint2* ml = nullptr) {
    using F = QFmt<FMT>;
    const int g = lane >> F::LOG_G, l = lane & (F::G - 1);
    const bool active = l * F::R < ld;
    const size_t colb = size_t(ld) * fmt_bytes(FMT);
    const size_t b0 = size_t(a0) * 16 + size_t(l) * 16, b1 = size_t(a1) * 16 + size_t(l) * 16;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int j = g + F::C * i;
        const size_t off = j < n0 ? b0 + size_t(j) * colb : b1 + size_t(j - n0) * colb;
        const bool ok = active && j < ntot;
        m[i] = ok ? __ldcs(reinterpret_cast<const uint4*>(A + off)) : make_uint4(0u, 0u, 0u, 0u);
        if constexpr (FMT == FMT_I24)
            ml[i] = ok ? __ldcs(reinterpret_cast<const uint2*>(A + off + (ptrdiff_t(2 * ld) - ptrdiff_t(8 * l))))
                       : make_uint2(0u, 0u);
    }
}

// ------------------------------------------------------------------ N-form
// acc[R] (this lane's rows) += A_pack(:, own columns) * v(own columns)
template <int FMT>
__device__ __forceinline__ void npack_q(const QNPack& pk, const uint8_t* A, const double* vx, const double* vt,
                                        int ld, int lane, double* acc) {
    using F = QFmt<FMT>;
    const int g = lane >> F::LOG_G;
    const int n0 = pk.p[0].nc, ntot = n0 + pk.p[1].nc;
    // vector entries of the pack, one per lane, pre-multiplied by the part's scale
    const bool second = lane >= n0;
    const uint32_t vo = second ? pk.p[1].v_off : pk.p[0].v_off;
    const float sc = second ? pk.p[1].scale : pk.p[0].scale;
    const double* v = (vo & VEC_T) ? vt + (vo & ~VEC_T) : vx + vo;
    const float vl = lane < ntot ? float(__ldg(v + (second ? lane - n0 : lane)) * double(sc)) : 0.f;
    uint4 m[8];
    uint2 ml[FMT == FMT_I24 ? 8 : 1];
    load_pack<FMT>(A, pk.p[0].a16, pk.p[1].a16, n0, ntot, ld, lane, m, ml);
    if constexpr (FMT == FMT_I16 || FMT == FMT_I24) {
        // row pairs: one packed FMA per two rows
        uint64_t s2[4] = {0ull, 0ull, 0ull, 0ull};
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const float vj = __shfl_sync(0xffffffffu, vl, (g + F::C * i) & 31);
            const uint64_t vv = pk2f(vj, vj);
            uint64_t pr[4];
            if constexpr (FMT == FMT_I24) i24_pairs(m[i], ml[i], pr);
            else i16_pairs(m[i], pr);
#pragma unroll
            for (int k = 0; k < 4; ++k) fma2(s2[k], pr[k], vv);
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const float2 t = upk2(s2[k]);
            acc[2 * k] += double(t.x);
            acc[2 * k + 1] += double(t.y);
        }
    } else {
        float s[F::R];
#pragma unroll
        for (int r = 0; r < F::R; ++r) s[r] = 0.f;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const float vj = __shfl_sync(0xffffffffu, vl, (g + F::C * i) & 31);
            float f[F::R];
            unpack16<FMT>(m[i], f);
#pragma unroll
            for (int r = 0; r < F::R; ++r) s[r] = fmaf(f[r], vj, s[r]);
        }
#pragma unroll
        for (int r = 0; r < F::R; ++r) acc[r] += double(s[r]);
    }
}

// sum the C column groups of the accumulators and store rows to red[]
template <int FMT>
__device__ __forceinline__ void nflush_q(double* acc, int lane, double* red_row) {
    using F = QFmt<FMT>;
#pragma unroll
    for (int o = F::G; o < 32; o <<= 1)
#pragma unroll
        for (int r = 0; r < F::R; ++r) acc[r] += __shfl_xor_sync(0xffffffffu, acc[r], o);
    if ((lane >> F::LOG_G) == 0)
#pragma unroll
        for (int r = 0; r < F::R; ++r) red_row[(lane & (F::G - 1)) * F::R + r] = acc[r];
}

// sum the C column groups of the accumulators and add rows to red[]
template <int FMT>
__device__ __forceinline__ void nflush_add_q(double* acc, int lane, double* red_row) {
    using F = QFmt<FMT>;
#pragma unroll
    for (int o = F::G; o < 32; o <<= 1)
#pragma unroll
        for (int r = 0; r < F::R; ++r) acc[r] += __shfl_xor_sync(0xffffffffu, acc[r], o);
    if ((lane >> F::LOG_G) == 0)
#pragma unroll
        for (int r = 0; r < F::R; ++r) red_row[(lane & (F::G - 1)) * F::R + r] += acc[r];
}

// a warp's share (packs cb + warp, cb + warp + W, ...) of one format's packs
// of a tile, with the next descriptor read ahead
template <int W, int FMT>
__device__ __forceinline__ void npacks_q(uint32_t cb, uint32_t ce, int ld, const QNPack* __restrict__ packs,
                                         const uint8_t* __restrict__ A, const double* __restrict__ vx,
                                         const double* __restrict__ vt, int warp, int lane, double* acc) {
    uint32_t c = cb + warp;
    QNPack nxt{};
    if (c < ce) nxt = ld_pack(packs + c);
    for (; c < ce; c += W) {
        const QNPack pk = nxt;
        if (c + W < ce) nxt = ld_pack(packs + c + W);
        npack_q<FMT>(pk, A, vx, vt, ld, lane, acc);
    }
}

// N-form of a reduced-precision store: a CTA takes one output tile, both its
// packs of the wide format WIDE (FP32, or 24-bit for block floating point)
// and its packs of the 16-bit format F16 (either may be empty), sums them in
// FP64 and updates y once.
template <int W, int WIDE, int F16>
__global__ void __launch_bounds__(W * 32, W >= 16 ? 1 : 3)
k_nform_q(const NSeg2* __restrict__ segs, const QNPack* __restrict__ packs, const uint8_t* __restrict__ A,
          const double* __restrict__ vx, const double* __restrict__ vt, double* __restrict__ out, double alpha,
          int add) {
    __shared__ double red[W][TILE];
    pdl_trigger();
    const NSeg2 sg = segs[blockIdx.x];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    pdl_wait();
    if constexpr (WIDE == FMT_I24) {
        // the wide packs flushed before the 16-bit ones start: fewer live
        // registers next to the 24-bit loads
        {
            double a32[QFmt<WIDE>::R];
#pragma unroll
            for (int r = 0; r < QFmt<WIDE>::R; ++r) a32[r] = 0.0;
            npacks_q<W, WIDE>(sg.cb32, sg.ce32, sg.ld32, packs, A, vx, vt, warp, lane, a32);
            nflush_q<WIDE>(a32, lane, red[warp]);
        }
        double a16[QFmt<F16>::R];
#pragma unroll
        for (int r = 0; r < QFmt<F16>::R; ++r) a16[r] = 0.0;
        npacks_q<W, F16>(sg.cb16, sg.ce16, sg.ld16, packs, A, vx, vt, warp, lane, a16);
        __syncwarp();
        nflush_add_q<F16>(a16, lane, red[warp]);
    } else {
        double a32[QFmt<WIDE>::R], a16[QFmt<F16>::R];
#pragma unroll
        for (int r = 0; r < QFmt<WIDE>::R; ++r) a32[r] = 0.0;
#pragma unroll
        for (int r = 0; r < QFmt<F16>::R; ++r) a16[r] = 0.0;
        npacks_q<W, WIDE>(sg.cb32, sg.ce32, sg.ld32, packs, A, vx, vt, warp, lane, a32);
        npacks_q<W, F16>(sg.cb16, sg.ce16, sg.ld16, packs, A, vx, vt, warp, lane, a16);
        nflush_q<WIDE>(a32, lane, red[warp]);
        __syncwarp();
        nflush_add_q<F16>(a16, lane, red[warp]);
    }
    __syncthreads();
    if (threadIdx.x < sg.rows) {
        double s = 0.0;
#pragma unroll
        for (int w = 0; w < W; ++w) s += red[w][threadIdx.x];
        double* o = out + sg.out + threadIdx.x;
        if (add) *o += alpha * s;
        else *o = s;
    }
}

// -------------------------------------------------------------- tile T-form
// x of the lane's R rows
// per-lane dot products of the 8 loaded column pieces with x
template <int FMT>
__device__ __forceinline__ void ttdots_q(const uint4* m, const uint2* ml, const float* xr, float* p) {
    using F = QFmt<FMT>;
    if constexpr (FMT == FMT_I16 || FMT == FMT_I24) {
        // packed: rows 2k, 2k+1 in one FMA, the two halves added at the end
        uint64_t x2[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) x2[k] = pk2f(xr[2 * k], xr[2 * k + 1]);
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            uint64_t pr[4];
            if constexpr (FMT == FMT_I24) i24_pairs(m[i], ml[i], pr);
            else i16_pairs(m[i], pr);
            uint64_t a = 0ull;
#pragma unroll
            for (int k = 0; k < 4; ++k) fma2(a, pr[k], x2[k]);
            const float2 t = upk2(a);
            p[i] = t.x + t.y;
        }
    } else {
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            float f[F::R];
            unpack16<FMT>(m[i], f);
            float s = 0.f;
#pragma unroll
            for (int r = 0; r < F::R; ++r) s = fmaf(f[r], xr[r], s);
            p[i] = s;
        }
    }
}

// ------------------------------------------------------- column streams
__device__ __forceinline__ MCol ld_mcol(const MCol* p) {
    const uint2 u = __ldg(reinterpret_cast<const uint2*>(p));
    return MCol{u.x, __uint_as_float(u.y)};
}

// Tile T-form on the tile's column stream (the chunks of one format that the
// tile visits, contiguous in the store; see MSeg).  Like k_ttform_q, but a
// warp iteration takes the next 8*C columns of the run whatever the chunk
// boundaries, so every iteration moves a full 4 KB even where the chunks
// are narrow; the output slot and scale of each column come from the
// per-column table.
template <int W, int FMT>
__device__ __forceinline__ void ttform_qs(const MSeg& sg, const MCol* __restrict__ cols, const uint8_t* __restrict__ A,
                                          const double* __restrict__ vin, double* __restrict__ out,
                                          double* __restrict__ part, double alpha, int add) {
    using F = QFmt<FMT>;
    constexpr int BC = 8 * F::C;   // columns per warp iteration
    constexpr int SH = F::LOG_G - 3;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> F::LOG_G, l = lane & (F::G - 1);
    float xr[F::R];
#pragma unroll
    for (int r = 0; r < F::R; ++r) {
        const int row = l * F::R + r;
        xr[r] = row < sg.rows ? float(__ldg(vin + sg.vo + row)) : 0.f;
    }
    const int ncols = int(sg.ncols);
    const size_t colb = size_t(sg.ld) * fmt_bytes(FMT);
    const uint8_t* base = A + size_t(sg.a16) * 16 + size_t(l) * 16;
    const bool active = l * F::R < sg.ld;
    const MCol* ctab = cols + sg.col0;
    // after the reduction the lane holds column jown of the iteration
    const int jown = g + F::C * (l >> SH);
    const bool writer = (l & ((1 << SH) - 1)) == 0;
    // 24-bit runs: the low parts of a lane's rows lie 2*ld - 8*l bytes after
    // its high parts
    const ptrdiff_t lo_off = 2 * ptrdiff_t(sg.ld) - 8 * ptrdiff_t(l);
    uint2 ml[FMT == FMT_I24 ? 8 : 1];
    auto load = [&](int c0, uint4 (&m)[8]) {
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const int j = c0 + g + F::C * i;
            const bool ok = active && j < ncols;
            m[i] = ok ? __ldcs(reinterpret_cast<const uint4*>(base + size_t(j) * colb)) : make_uint4(0u, 0u, 0u, 0u);
            if constexpr (FMT == FMT_I24)
                ml[i] = ok ? __ldcs(reinterpret_cast<const uint2*>(base + size_t(j) * colb + lo_off))
                           : make_uint2(0u, 0u);
        }
    };
    int c0 = warp * BC;
    if (c0 >= ncols) return;
    uint4 m[8];
    load(c0, m);
    MCol mc = (writer && c0 + jown < ncols) ? ld_mcol(ctab + c0 + jown) : MCol{0u, 0.f};
    for (; c0 < ncols; c0 += W * BC) {
        float p[8];
        ttdots_q<FMT>(m, ml, xr, p);
        const MCol done = mc;
        const int cd = c0;
        if (c0 + W * BC < ncols) {
            load(c0 + W * BC, m);
            mc = (writer && c0 + W * BC + jown < ncols) ? ld_mcol(ctab + c0 + W * BC + jown) : MCol{0u, 0.f};
        }
        TransposeReduce<8, F::G / 2, float>::run(p, lane);
        if (writer && cd + jown < ncols) {
            const double val = double(done.scale) * double(p[0]);
            if (done.idx & MC_DIRECT) {
                double* o = out + (done.idx & ~MC_DIRECT);
                if (add) *o += alpha * val;
                else *o = val;
            } else {
                part[done.idx] = val;
            }
        }
    }
}

// All stream segments of one tile T-form pass in one grid: the first n32
// CTAs take the runs of the wide format WIDE (FP32, or 24-bit for block
// floating point), the others the runs of the 16-bit format F16.
// The outputs of the two formats are disjoint, so their CTAs may run side
// by side, and the pass has a single tail.
template <int W, int WIDE, int F16>
__global__ void __launch_bounds__(W * 32, 24 / W)
k_ttform_qs(const MSeg* __restrict__ segs32, int n32, const MSeg* __restrict__ segs16, const MCol* __restrict__ cols,
            const uint8_t* __restrict__ A, const double* __restrict__ vin, double* __restrict__ out,
            double* __restrict__ part, double alpha, int add) {
    pdl_trigger();
    pdl_wait();
    if (int(blockIdx.x) < n32) ttform_qs<W, WIDE>(segs32[blockIdx.x], cols, A, vin, out, part, alpha, add);
    else ttform_qs<W, F16>(segs16[blockIdx.x - n32], cols, A, vin, out, part, alpha, add);
}

}  // namespace hlrc
