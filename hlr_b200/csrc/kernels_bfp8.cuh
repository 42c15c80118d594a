// 8-right-hand-side products of block-floating-point (BFP) stores on FP16
// tensor cores (mma.sync m16n8k16, FP32 accumulation), MR_RB = 8 vectors.
//
// A BFP column holds offset-binary integers: 16-bit u = v + 2^15, or 24-bit
// u = v + 2^22 split into a 16-bit high part (u >> 8) and a byte (u & 255),
// times a power-of-two chunk scale (compress/bfp.hh:945-1100 decodes such
// mantissas inside its GEMV loop).  Here the integers enter the MMA as exact
// FP16 byte planes, taken from the raw 16-bit words by byte permutes:
//   an FP16 with bits 0x64XX is 1024 + XX, so a byte b becomes the plane
//   value 1024 + b (offset plane), and the top byte becomes b - 128 (16-bit)
//   or b - 64 (24-bit) after one exact FP16 subtraction (signed plane).
//   16-bit: v = 256 (uh - 128) + (1024 + ul) - 1024
//   24-bit: v = 65536 (b2 - 64) + 256 (1024 + b1) + (1024 + b0) - 263168
// Each plane accumulates in its own FP32 MMA results; the plane weights and
// the constant offsets (offset x the sum of the vector operand over the
// contraction) are applied in FP64 once per 32-column stage (N-form) or per
// tile (tile T-form).  The vector operand is split into FP16 terms after a
// power-of-two scale per stage (or input tile) and right-hand side: two
// terms (about 22 bits) against 16-bit planes, three (about 33 bits) against
// the top plane of 24-bit columns, whose values carry 23 bits.  Data
// movement is that of kernels_tc.cuh: per-warp rings of cp.async stages of a
// segment's column run, ldmatrix fragments; the low bytes of 24-bit columns
// are staged raw and widened to an FP16 plane in shared memory per stage.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "kernels_tc.cuh"

namespace hlrc {

// One stage per warp and at least 3 CTAs per SM: on a 4-member batched
// problem (BFP store, 8 vectors) the N-form passes took 0.151 / 0.200 ms and
// the tile T-form 0.277 ms, against 0.184 / 0.200 / 0.309 ms with two
// stages and no register bound (the N-forms then held 164 and 204
// registers and 2 CTAs per SM).
#ifndef HLRC_BQ_STAGES
#define HLRC_BQ_STAGES 1
#endif
constexpr int BQ_STAGES = HLRC_BQ_STAGES;                         // ring depth per warp
#ifndef HLRC_BQ_MINB
#define HLRC_BQ_MINB 3
#endif
constexpr int BQ_LO_STRIDE = 80;                                  // raw low bytes of a 24-bit column (<= 64) + pad
constexpr int BQ_PLANE = 32 * TC_A16_STRIDE;                      // one widened low-byte plane of a stage
constexpr int BQ_STAGE_N16 = TC_STAGE_N16;                        // as FP16
constexpr int BQ_STAGE_N24 = 32 * TC_A16_STRIDE + 32 * BQ_LO_STRIDE + 32 * TC_V_STRIDE + 32 * 4;
constexpr int BQ_STAGE_T16 = TC_STAGE_T16;
constexpr int BQ_STAGE_T24 = 32 * TC_A16_STRIDE + 32 * BQ_LO_STRIDE + 32 * 8;

// dynamic shared memory of a launch: per warp a ring of stages, plus the
// widened low-byte plane for 24-bit columns
constexpr int bq_smem_n(bool i24) {
    return TC_WARPS * (BQ_STAGES * (i24 ? BQ_STAGE_N24 : BQ_STAGE_N16) + (i24 ? BQ_PLANE : 0));
}
constexpr int bq_smem_t(bool i24) {
    return TC_WARPS * (BQ_STAGES * (i24 ? BQ_STAGE_T24 : BQ_STAGE_T16) + (i24 ? BQ_PLANE : 0));
}

// FP16 pairs 1024 + byte of the two 16-bit words of r: high bytes, low bytes
__device__ __forceinline__ uint32_t plane_hi(uint32_t r) { return __byte_perm(r, 0x64646464u, 0x4341); }
__device__ __forceinline__ uint32_t plane_lo(uint32_t r) { return __byte_perm(r, 0x64646464u, 0x4240); }
__device__ __forceinline__ uint32_t hsub2_u(uint32_t a, uint32_t b) {
    uint32_t d;
    asm("sub.rn.f16x2 %0, %1, %2;\n" : "=r"(d) : "r"(a), "r"(b));
    return d;
}
constexpr uint32_t BQ_H1152 = 0x64806480u;   // (1152, 1152): 1024 + 128
constexpr uint32_t BQ_H1088 = 0x64406440u;   // (1088, 1088): 1024 + 64

// NT FP16 terms of the scaled pair (v0 * s, v1 * s), each the FP16 rounding
// of what the earlier terms leave (residuals in FP64); f0 + f1 of the pair
// rounded to FP32 is returned for the offset sums
template <int NT>
__device__ __forceinline__ float bq_split(double v0, double v1, double s, uint32_t (&t)[NT]) {
    using O = TcOp<FMT_F16>;
    double d0 = v0 * s, d1 = v1 * s;
    const float r = float(d0) + float(d1);
#pragma unroll
    for (int i = 0; i < NT; ++i) {
        t[i] = O::cvt2(float(d0), float(d1));
        const float2 h = O::unpack(t[i]);
        d0 -= double(h.x);
        d1 -= double(h.y);
    }
    return r;
}

// Copies units [0, units) (16 bytes each) of the COLS columns of a stage
// from base + column * colb into dst at `stride`; UPL units per column per
// lane round; the rest of each slot column, and columns past ncols, are
// zero-filled.
template <int UPL, int COLS>
__device__ __forceinline__ void stage_units(uint8_t* dst, int stride, const uint8_t* base, int c0, int ncols,
                                            int colb, int units, int lane) {
    const int u = lane % UPL;
    const uint8_t* src = base + size_t(c0 + lane / UPL) * colb + u * 16;
    uint8_t* d = dst + (lane / UPL) * stride + u * 16;
#pragma unroll
    for (int i = 0; i < COLS * UPL / 32; ++i) {
        const bool ok = c0 + lane / UPL + (32 / UPL) * i < ncols && u < units;
        cp16(d + (32 / UPL) * i * stride, ok ? src + size_t((32 / UPL) * i) * colb : base, ok);
    }
}

// The low-byte plane of a stage's 32 24-bit columns: lane j widens column
// j's 64 raw bytes (stride BQ_LO_STRIDE) to FP16 1024 + b at TC_A16_STRIDE.
__device__ __forceinline__ void widen_lo(const uint8_t* raw, uint8_t* plane, int lane) {
    const uint4* s = reinterpret_cast<const uint4*>(raw + lane * BQ_LO_STRIDE);
    uint4* d = reinterpret_cast<uint4*>(plane + lane * TC_A16_STRIDE);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const uint4 w = s[q];
        d[2 * q] = make_uint4(__byte_perm(w.x, 0x64646464u, 0x4140), __byte_perm(w.x, 0x64646464u, 0x4342),
                              __byte_perm(w.y, 0x64646464u, 0x4140), __byte_perm(w.y, 0x64646464u, 0x4342));
        d[2 * q + 1] = make_uint4(__byte_perm(w.z, 0x64646464u, 0x4140), __byte_perm(w.z, 0x64646464u, 0x4342),
                                  __byte_perm(w.w, 0x64646464u, 0x4140), __byte_perm(w.w, 0x64646464u, 0x4342));
    }
}

// Stages columns [c0, c0 + 32) of a BFP run: the 16-bit words (the whole
// column, or the high parts of 24-bit columns) at TC_A16_STRIDE, and for
// 24-bit columns the raw low bytes (2 ld bytes into the column) after them.
template <bool I24>
__device__ __forceinline__ void stage_bfp(uint8_t* sa, const uint8_t* base, int c0, int ncols, int ld, int lane) {
    const int colb = ld * (I24 ? 3 : 2);
    stage_units<8, 32>(sa, TC_A16_STRIDE, base, c0, ncols, colb, ld / 8, lane);
    if constexpr (I24) stage_units<4, 32>(sa + BQ_PLANE, BQ_LO_STRIDE, base + 2 * ld, c0, ncols, colb, ld / 16, lane);
}

// ------------------------------------------------------------------ N-form
// One CTA per output tile of one format (stream segment); the warps take
// the segment's 32-column stages round-robin.  Fragments as k_nform_tc:
// A[m][k] = tile row m, stream column k (ldmatrix.trans of the staged
// words); lane (g, t) accumulates rows 16i + g, 16i + g + 8 for right-hand
// sides 2t, 2t+1.  Launch: bq_smem_n(I24) bytes of dynamic shared memory.
template <bool I24>
__global__ void __launch_bounds__(TC_WARPS * 32, HLRC_BQ_MINB)
k_nform_bfp(const MSeg* __restrict__ segs, const MCol* __restrict__ cols, const uint8_t* __restrict__ A,
            const double* __restrict__ vx, const double* __restrict__ vt, OutMap om, double alpha, int add) {
    using O = TcOp<FMT_F16>;
    constexpr int STAGE = I24 ? BQ_STAGE_N24 : BQ_STAGE_N16;
    constexpr int VOFF = I24 ? BQ_PLANE + 32 * BQ_LO_STRIDE : BQ_PLANE;   // vector part of a stage
    constexpr int NT = I24 ? 3 : 2;                                        // FP16 terms of the vector operand
    extern __shared__ __align__(16) uint8_t smem[];
    const MSeg sg = segs[blockIdx.x];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, t = lane & 3;
    uint8_t* ring = smem + warp * (BQ_STAGES * STAGE + (I24 ? BQ_PLANE : 0));
    uint8_t* lo_plane = ring + BQ_STAGES * STAGE;                          // 24-bit: this warp's widened bytes
    const int ncols = int(sg.ncols);
    const uint8_t* base = A + size_t(sg.a16) * 16;
    const MCol* ctab = cols + sg.col0;
    const int nmt = (sg.rows + 15) / 16;
    // ldmatrix.trans row of this lane: column + 8 for lanes 16-31, rows + 8 for lanes 8-15 and 24-31
    const int lcol = (lane & 7) + ((lane >> 4) & 1) * 8, lrow = ((lane >> 3) & 1) * 8;
    double acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i) acc[i][0] = acc[i][1] = acc[i][2] = acc[i][3] = 0.0;
    MCol mc = warp * 32 + lane < ncols ? ld_mcol(ctab + warp * 32 + lane) : MCol{0u, 0.f};
    warp_stream<BQ_STAGES>(
        (ncols + 31) / 32, warp,
        [&](int slot, int st) {
            uint8_t* sa = ring + slot * STAGE;
            const int c0 = 32 * st;
            stage_bfp<I24>(sa, base, c0, ncols, sg.ld, lane);
            stage_vector<32>(sa + VOFF, mc.idx, c0, ncols, vx, vt, lane);
            reinterpret_cast<float*>(sa + VOFF + 32 * TC_V_STRIDE)[lane] = mc.scale;
            const int cn = c0 + 32 * TC_WARPS + lane;
            mc = cn < ncols ? ld_mcol(ctab + cn) : MCol{0u, 0.f};
        },
        [&](int slot, int st) {
            const uint8_t* sa = ring + slot * STAGE;
            if constexpr (I24) {
                widen_lo(sa + BQ_PLANE, lo_plane, lane);
                __syncwarp();
            }
            const double* sv = reinterpret_cast<const double*>(sa + VOFF);
            const float* ssc = reinterpret_cast<const float*>(sa + VOFF + 32 * TC_V_STRIDE);
            const int nkt = ncols - 32 * st > 16 ? 2 : 1;
            // vector operand: columns 16kt + 2t + {0, 1, 8, 9}, right-hand side g, times the column scale
            double bv[2][4];
            int E = 0;
#pragma unroll
            for (int kt = 0; kt < 2; ++kt)
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int col = 16 * kt + 2 * t + (j & 1) + 8 * (j >> 1);
                    const double x = sv[col * (TC_V_STRIDE / 8) + g] * double(ssc[col]);
                    bv[kt][j] = x;
                    E = max(E, dexp(x));
                }
            E = quad_max(E);
            const double s = exp_scale(E);
            const double f0 = exp_unscale(__shfl_sync(0xffffffffu, E, 8 * t));
            const double f1 = exp_unscale(__shfl_sync(0xffffffffu, E, 8 * t + 4));
            uint32_t b0[2][NT], b1[2][NT];
            float ssum = 0.f;
#pragma unroll
            for (int kt = 0; kt < 2; ++kt) {
                ssum += bq_split<NT>(bv[kt][0], bv[kt][1], s, b0[kt]);
                ssum += bq_split<NT>(bv[kt][2], bv[kt][3], s, b1[kt]);
            }
            // sum of the stage's (scaled) vector entries of right-hand side g,
            // then of this lane's output right-hand sides 2t, 2t+1
            ssum += __shfl_xor_sync(0xffffffffu, ssum, 1);
            ssum += __shfl_xor_sync(0xffffffffu, ssum, 2);
            const double S0 = double(__shfl_sync(0xffffffffu, ssum, 8 * t));
            const double S1 = double(__shfl_sync(0xffffffffu, ssum, 8 * t + 4));
            // plane results: [0] top (signed), [1] middle / low (offset), [2] 24-bit low byte
            float d[I24 ? 3 : 2][4][4];
#pragma unroll
            for (int p = 0; p < (I24 ? 3 : 2); ++p)
#pragma unroll
                for (int i = 0; i < 4; ++i) d[p][i][0] = d[p][i][1] = d[p][i][2] = d[p][i][3] = 0.f;
#pragma unroll
            for (int kt = 0; kt < 2; ++kt) {
                if (kt >= nkt) break;
                const uint8_t* row0 = sa + (16 * kt + lcol) * TC_A16_STRIDE + 2 * lrow;
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    if (i >= nmt) break;
                    uint32_t a[4], ph[4], pm[4];
                    ldsm_x4_t(a, row0 + 32 * i);
#pragma unroll
                    for (int r = 0; r < 4; ++r) {
                        ph[r] = hsub2_u(plane_hi(a[r]), I24 ? BQ_H1088 : BQ_H1152);
                        pm[r] = plane_lo(a[r]);
                    }
#pragma unroll
                    for (int q = 0; q < NT; ++q) O::mma(d[0][i], ph, b0[kt][q], b1[kt][q]);
                    O::mma(d[1][i], pm, b0[kt][0], b1[kt][0]);
                    O::mma(d[1][i], pm, b0[kt][1], b1[kt][1]);
                    if constexpr (I24) {
                        uint32_t pl[4];
                        ldsm_x4_t(pl, lo_plane + (row0 - sa) + 32 * i);
                        O::mma(d[2][i], pl, b0[kt][0], b1[kt][0]);
                    }
                }
            }
            // plane weights and offsets: 16-bit 256 top + low - 1024 S;
            // 24-bit 65536 top + 256 middle + low - 263168 S
            constexpr double WT = I24 ? 65536.0 : 256.0, WM = I24 ? 256.0 : 1.0;
            constexpr double OFS = I24 ? 263168.0 : 1024.0;
            const double o0 = OFS * S0, o1 = OFS * S1;
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                double v[4];
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    double low = 0.0;
                    if constexpr (I24) low = double(d[2][i][e]);
                    v[e] = fma(WT, double(d[0][i][e]), fma(WM, double(d[1][i][e]), low - ((e & 1) ? o1 : o0)));
                }
                acc[i][0] = fma(v[0], f0, acc[i][0]);
                acc[i][1] = fma(v[1], f1, acc[i][1]);
                acc[i][2] = fma(v[2], f0, acc[i][2]);
                acc[i][3] = fma(v[3], f1, acc[i][3]);
            }
        });
    // all warps are done with their rings: reuse the start of shared memory
    __syncthreads();
    double* red = reinterpret_cast<double*>(smem);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        double* r0 = red + (warp * TILE + 16 * i + g) * MR_RB + 2 * t;
        double* r1 = r0 + 8 * MR_RB;
        r0[0] = acc[i][0];
        r0[1] = acc[i][1];
        r1[0] = acc[i][2];
        r1[1] = acc[i][3];
    }
    __syncthreads();
    nform_store(red, int(sg.vo), sg.rows, om, alpha, add);
}

// -------------------------------------------------------------- tile T-form
// One CTA per input tile of one format; the warps take the segment's
// 32-column stages round-robin.  Fragments as ttform_tc: A[m][k] = stream
// column m, tile row k (plain ldmatrix), B[k][n] = x row k, right-hand
// side n, split once per tile.  Each column result is complete and goes to
// its output or FP32 partial slot through the column table.
template <bool I24>
__device__ __forceinline__ void ttform_bfp(const MSeg& sg, uint8_t* smem, const MCol* __restrict__ cols,
                                           const uint8_t* __restrict__ A, const double* __restrict__ vin,
                                           const OutMap& om, float* __restrict__ part, double alpha, int add) {
    using O = TcOp<FMT_F16>;
    constexpr int NT = I24 ? 3 : 2;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, t = lane & 3;
    constexpr int STAGE = I24 ? BQ_STAGE_T24 : BQ_STAGE_T16;
    uint8_t* ring = smem + warp * (BQ_STAGES * STAGE + (I24 ? BQ_PLANE : 0));
    uint8_t* lo_plane = ring + BQ_STAGES * STAGE;             // 24-bit: this warp's widened bytes
    constexpr int TABOFF = I24 ? BQ_PLANE + 32 * BQ_LO_STRIDE : BQ_PLANE;   // column table of a stage
    // x entries of the lane: rows 16kt + 2t + {0, 1, 8, 9} (kt < 4), right-hand side g
    double xv[4][4];
    int E = 0;
#pragma unroll
    for (int kt = 0; kt < 4; ++kt)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int row = 16 * kt + 2 * t + (j & 1) + 8 * (j >> 1);
            const double v = row < sg.rows ? __ldg(vin + size_t(sg.vo + row) * MR_RB + g) : 0.0;
            xv[kt][j] = v;
            E = max(E, dexp(v));
        }
    E = quad_max(E);
    const double s = exp_scale(E);
    const double inv0 = exp_unscale(__shfl_sync(0xffffffffu, E, 8 * t));
    const double inv1 = exp_unscale(__shfl_sync(0xffffffffu, E, 8 * t + 4));
    uint32_t b0[4][NT], b1[4][NT];
    float xsum = 0.f;
#pragma unroll
    for (int kt = 0; kt < 4; ++kt) {
        xsum += bq_split<NT>(xv[kt][0], xv[kt][1], s, b0[kt]);
        xsum += bq_split<NT>(xv[kt][2], xv[kt][3], s, b1[kt]);
    }
    xsum += __shfl_xor_sync(0xffffffffu, xsum, 1);
    xsum += __shfl_xor_sync(0xffffffffu, xsum, 2);
    constexpr double WT = I24 ? 65536.0 : 256.0, WM = I24 ? 256.0 : 1.0;
    constexpr double OFS = I24 ? 263168.0 : 1024.0;
    const double o0 = OFS * double(__shfl_sync(0xffffffffu, xsum, 8 * t));
    const double o1 = OFS * double(__shfl_sync(0xffffffffu, xsum, 8 * t + 4));
    const int ncols = int(sg.ncols);
    const uint8_t* base = A + size_t(sg.a16) * 16;
    const MCol* ctab = cols + sg.col0;
    const int nkt = (sg.rows + 15) / 16;
    // ldmatrix row of this lane: column + 8 for lanes 8-15 and 24-31, rows + 8 for lanes 16-31
    const int lcol = (lane & 7) + ((lane >> 3) & 1) * 8, lrow = ((lane >> 4) & 1) * 8;
    MCol mc = warp * 32 + lane < ncols ? ld_mcol(ctab + warp * 32 + lane) : MCol{0u, 0.f};
    warp_stream<BQ_STAGES>(
        (ncols + 31) / 32, warp,
        [&](int slot, int st) {
            uint8_t* sa = ring + slot * STAGE;
            const int c0 = 32 * st;
            stage_bfp<I24>(sa, base, c0, ncols, sg.ld, lane);
            reinterpret_cast<MCol*>(sa + TABOFF)[lane] = mc;
            const int cn = c0 + 32 * TC_WARPS + lane;
            mc = cn < ncols ? ld_mcol(ctab + cn) : MCol{0u, 0.f};
        },
        [&](int slot, int st) {
            const uint8_t* sa = ring + slot * STAGE;
            if constexpr (I24) {
                widen_lo(sa + BQ_PLANE, lo_plane, lane);
                __syncwarp();
            }
            const MCol* tab = reinterpret_cast<const MCol*>(sa + TABOFF);
            const int cnt = min(32, ncols - 32 * st);
            for (int mt = 0; 16 * mt < cnt; ++mt) {
                float d[I24 ? 3 : 2][4];
#pragma unroll
                for (int p = 0; p < (I24 ? 3 : 2); ++p) d[p][0] = d[p][1] = d[p][2] = d[p][3] = 0.f;
                const int roff = (16 * mt + lcol) * TC_A16_STRIDE + 2 * lrow;
#pragma unroll
                for (int kt = 0; kt < 4; ++kt) {
                    if (kt >= nkt) break;
                    uint32_t a[4], ph[4], pm[4];
                    ldsm_x4(a, sa + roff + 32 * kt);
#pragma unroll
                    for (int r = 0; r < 4; ++r) {
                        ph[r] = hsub2_u(plane_hi(a[r]), I24 ? BQ_H1088 : BQ_H1152);
                        pm[r] = plane_lo(a[r]);
                    }
#pragma unroll
                    for (int q = 0; q < NT; ++q) O::mma(d[0], ph, b0[kt][q], b1[kt][q]);
                    O::mma(d[1], pm, b0[kt][0], b1[kt][0]);
                    O::mma(d[1], pm, b0[kt][1], b1[kt][1]);
                    if constexpr (I24) {
                        uint32_t pl[4];
                        ldsm_x4(pl, lo_plane + roff + 32 * kt);
                        O::mma(d[2], pl, b0[kt][0], b1[kt][0]);
                    }
                }
                double v[4];
#pragma unroll
                for (int e = 0; e < 4; ++e) {
                    double low = 0.0;
                    if constexpr (I24) low = double(d[2][e]);
                    v[e] = fma(WT, double(d[0][e]), fma(WM, double(d[1][e]), low - ((e & 1) ? o1 : o0)));
                }
                const int c = 16 * mt + g;
                if (c < cnt) {
                    const MCol m = tab[c];
                    tt_out(m, 2 * t, v[0] * (double(m.scale) * inv0), om, part, alpha, add);
                    tt_out(m, 2 * t + 1, v[1] * (double(m.scale) * inv1), om, part, alpha, add);
                }
                if (c + 8 < cnt) {
                    const MCol m = tab[c + 8];
                    tt_out(m, 2 * t, v[2] * (double(m.scale) * inv0), om, part, alpha, add);
                    tt_out(m, 2 * t + 1, v[3] * (double(m.scale) * inv1), om, part, alpha, add);
                }
            }
        });
}

// Tile T-form of the runs of one BFP format (the 24-bit and the 16-bit runs
// write disjoint outputs and run as two grids, each with its own stage
// size).  Dynamic shared memory: bq_smem_t(I24).
template <bool I24>
__global__ void __launch_bounds__(TC_WARPS * 32, HLRC_BQ_MINB)
k_ttform_bfp(const MSeg* __restrict__ segs, const MCol* __restrict__ cols, const uint8_t* __restrict__ A,
             const double* __restrict__ vin, OutMap om, float* __restrict__ part, double alpha, int add) {
    extern __shared__ __align__(16) uint8_t smem[];
    ttform_bfp<I24>(segs[blockIdx.x], smem, cols, A, vin, om, part, alpha, add);
}

}  // namespace hlrc
