// Tensor-core multi-right-hand-side kernels for reduced-precision stores,
// MR_RB = 8 right-hand sides per launch.
//
// With 8 right-hand sides a chunk product is a small dense contraction.
// 16-bit columns (scaled FP16 / BF16) run as mma.sync m16n8k16 tiles with
// FP32 accumulation; the vector operand is split into two 16-bit terms,
// hi = round(s*v) and lo = round(s*v - hi), with a power-of-two scale per
// stage (N-form) or input tile (tile T-form) and right-hand side, so the
// product keeps about 22 significant bits of v (FP16) or 16 (BF16) and the
// storage rounding of the matrix stays the dominant error.  FP32 columns run
// on the FP64 tensor cores (m8n8k4): their values convert to FP64 exactly.
// Results are accumulated in FP64.
//
// Data movement.  The store is laid out so that the columns one segment
// (tile, format) visits form one contiguous run; a CTA owns a segment and its
// warps take 32-column stages (16 for FP32) of the run round-robin.  Each
// warp streams its stages through a ring of TC_STAGES shared-memory slots
// filled with cp.async 16-byte copies.  Columns land at a padded stride, so
// the fragment loads are free of bank conflicts, and the copies zero-fill
// everything past the run, so no slot ever holds stale data.  16-bit
// fragments come from ldmatrix: plain for the tile T-form (A = run^T, rows
// contiguous), .trans for the N-form (A = run, columns contiguous).  A
// per-column table gives each column's vector entry (N-form) or output
// (tile T-form) and its chunk scale; in the N-form the scale is folded into
// the vector operand, so a whole stage accumulates in one set of MMA results.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "kernels_mr.cuh"
#include "kernels_q.cuh"
#include "layout.hpp"

namespace hlrc {

constexpr int TC_WARPS = 4;    // warps per CTA
constexpr int TC_STAGES = 2;   // shared-memory stages per warp

// stage geometry: column strides in bytes
constexpr int TC_A16_STRIDE = 144;    // 16-bit chunk column (64 rows = 128 B) + 16 B pad
constexpr int TC_A32_STRIDE = 288;    // FP32 column (256 B) + 32 B pad (8-byte reads of row pairs)
constexpr int TC_V_STRIDE = 80;       // MR_RB doubles of one vector column + 16 B pad
constexpr int TC_STAGE_N16 = 32 * TC_A16_STRIDE + 32 * TC_V_STRIDE + 32 * 4;   // columns, vector, column scales
constexpr int TC_STAGE_T16 = 32 * TC_A16_STRIDE + 32 * 8;                        // columns, column table
constexpr int TC_STAGE_N32 = 16 * TC_A32_STRIDE + 16 * TC_V_STRIDE + 16 * 4;
constexpr int TC_STAGE_T32 = 16 * TC_A32_STRIDE + 16 * 8;

#ifndef HLRC_D32_STAGES
#define HLRC_D32_STAGES 2
#endif
constexpr int TC_STAGES_D32 = HLRC_D32_STAGES;   // ring depth of the FP32 N-form
#ifndef HLRC_N16_STAGES
#define HLRC_N16_STAGES 2
#endif
constexpr int TC_STAGES_N16 = HLRC_N16_STAGES;   // ring depth of the 16-bit N-form
#ifndef HLRC_N16_MINB
#define HLRC_N16_MINB 1
#endif
// The 8-vector tile T-form: one ring stage per warp and at least 6 CTAs per
// SM.  On a 4-member batched problem (mixed store) it took 0.193 ms against
// 0.206 ms with two stages; on one n = 32768 matrix the product time was the
// same (197 us) either way.  The ring depth changes no sum.
#ifndef HLRC_TT_STAGES
#define HLRC_TT_STAGES 1
#endif
constexpr int TC_STAGES_TT = HLRC_TT_STAGES;     // ring depth of the 8-vector tile T-form
#ifndef HLRC_TT_MINB
#define HLRC_TT_MINB 6
#endif

// dynamic shared memory of a launch: one ring of `nst` stages per warp
constexpr int tc_smem_bytes(int stage, int nst = TC_STAGES) { return TC_WARPS * nst * stage; }

template <int FMT> struct TcOp;

template <> struct TcOp<FMT_F16> {
    // two floats -> packed FP16 pair, lo in the low half (round to nearest even)
    static __device__ __forceinline__ uint32_t cvt2(float lo, float hi) {
        uint32_t r;
        asm("cvt.rn.f16x2.f32 %0, %1, %2;\n" : "=r"(r) : "f"(hi), "f"(lo));
        return r;
    }
    static __device__ __forceinline__ float2 unpack(uint32_t u) {
        __half2 h;
        memcpy(&h, &u, 4);
        return __half22float2(h);
    }
    static __device__ __forceinline__ void mma(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
        asm("mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
            "{%0,%1,%2,%3};\n"
            : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
            : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
    }
};

template <> struct TcOp<FMT_BF16> {
    static __device__ __forceinline__ uint32_t cvt2(float lo, float hi) {
        uint32_t r;
        asm("cvt.rn.bf16x2.f32 %0, %1, %2;\n" : "=r"(r) : "f"(hi), "f"(lo));
        return r;
    }
    static __device__ __forceinline__ float2 unpack(uint32_t u) {
        return make_float2(__uint_as_float(u << 16), __uint_as_float(u & 0xffff0000u));
    }
    static __device__ __forceinline__ void mma(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
        asm("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
            "{%0,%1,%2,%3};\n"
            : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
            : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
    }
};

// Power-of-two vector scales from exponent fields.  dexp(v) is the biased
// exponent of |v| (0 for zero and subnormals); for a block whose largest
// biased exponent is E the scale 2^(1036 - E) brings every entry below 2^14
// and the largest to at least 2^13.  Blocks with E < 14 (|v| < 2^-1009) are
// left unscaled.
__device__ __forceinline__ int dexp(double v) { return (__double2hiint(v) >> 20) & 0x7ff; }
__device__ __forceinline__ double exp_scale(int E) { return E < 14 ? 1.0 : __hiloint2double((2059 - E) << 20, 0); }
__device__ __forceinline__ double exp_unscale(int E) { return E < 14 ? 1.0 : __hiloint2double((E - 13) << 20, 0); }

// largest exponent over the 4 lanes of a quad (the lanes that share g)
__device__ __forceinline__ int quad_max(int e) {
    e = max(e, __shfl_xor_sync(0xffffffffu, e, 1));
    return max(e, __shfl_xor_sync(0xffffffffu, e, 2));
}

// hi/lo 16-bit terms of the scaled pair (v0, v1), packed as MMA operands
template <int FMT>
__device__ __forceinline__ void tc_split(double v0, double v1, double s, uint32_t& hi, uint32_t& lo) {
    using O = TcOp<FMT>;
    const float f0 = float(v0 * s), f1 = float(v1 * s);
    hi = O::cvt2(f0, f1);
    const float2 h = O::unpack(hi);
    lo = O::cvt2(f0 - h.x, f1 - h.y);
}

// ------------------------------------------------ shared-memory staging
__device__ __forceinline__ unsigned smem_addr(const void* p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

// 16-byte copy global -> shared; with ok == false the destination is
// zero-filled and nothing is read
__device__ __forceinline__ void cp16(void* dst, const void* src, bool ok) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_addr(dst)), "l"(src), "r"(ok ? 16 : 0)
                 : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

__device__ __forceinline__ void ldsm_x4(uint32_t (&r)[4], const void* row) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(smem_addr(row)));
}
__device__ __forceinline__ void ldsm_x4_t(uint32_t (&r)[4], const void* row) {
    asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(smem_addr(row)));
}

// One warp's pass over the stages s = warp, warp + W, ... < nst of a column
// stream through its ring: issue(slot, s) starts the copies of stage s into
// ring slot `slot`, and compute(slot, s) consumes the slot once its copies
// have landed.
template <int RING = TC_STAGES, typename Issue, typename Compute>
__device__ __forceinline__ void warp_stream(int nst, int warp, Issue&& issue, Compute&& compute) {
    const int n = nst > warp ? (nst - warp + TC_WARPS - 1) / TC_WARPS : 0;
    int issued = 0;
    auto issue_next = [&]() {
        if (issued < n) {
            issue(issued % RING, warp + issued * TC_WARPS);
            ++issued;
        }
        cp_commit();
    };
#pragma unroll
    for (int k = 0; k < RING - 1; ++k) issue_next();
    for (int k = 0; k < n; ++k) {
        issue_next();
        cp_wait<RING - 1>();
        __syncwarp();
        compute(k % RING, warp + k * TC_WARPS);
        __syncwarp();
    }
}

// Copies columns [c0, c0 + COLS) of a column stream (column j at
// base + j * colb, colb = ld * element bytes) into a stage at shared stride
// `stride`.  UPL 16-byte units make a 64-row column; lane l copies unit
// l % UPL of columns l / UPL + (32 / UPL) i.  Units below the column height
// of columns past ncols, and units past the column height, are zero-filled.
template <int UPL, int COLS>
__device__ __forceinline__ void stage_run(uint8_t* dst, int stride, const uint8_t* base, int c0, int ncols, int colb,
                                          int lane) {
    const int u = lane % UPL, units = colb / 16;
    const uint8_t* src = base + size_t(c0 + lane / UPL) * colb + u * 16;
    uint8_t* d = dst + (lane / UPL) * stride + u * 16;
#pragma unroll
    for (int i = 0; i < COLS * UPL / 32; ++i) {
        const bool ok = c0 + lane / UPL + (32 / UPL) * i < ncols && u < units;
        cp16(d + (32 / UPL) * i * stride, ok ? src + size_t((32 / UPL) * i) * colb : base, ok);
    }
}

// Copies the vector entries (MR_RB doubles = 4 units) of the COLS columns
// of an N-form stage, at shared stride TC_V_STRIDE.  Lane j holds the table
// entry of column j of the stage in `idx`.
template <int COLS>
__device__ __forceinline__ void stage_vector(uint8_t* dst, uint32_t idx, int c0, int ncols, const double* vx,
                                             const double* vt, int lane) {
    const int u = lane & 3;
#pragma unroll
    for (int i = 0; i < COLS / 8; ++i) {
        const int j = (lane >> 2) + 8 * i;
        const uint32_t e = __shfl_sync(0xffffffffu, idx, j);
        const bool ok = c0 + j < ncols;
        const double* v = ((e & VEC_T) ? vt : vx) + size_t(e & ~VEC_T) * MR_RB + 2 * u;
        cp16(dst + j * TC_V_STRIDE + u * 16, ok ? static_cast<const void*>(v) : vx, ok);
    }
}

// Epilogue of the tile T-forms: value val (already unscaled) of stream
// column entry m, right-hand side n, to its output (FP64) or to its partial
// slot.  Partials are stored in FP32: they are sums of FP32 MMA results of
// one tile, so nothing is lost, and the finish adds them up in FP64.
__device__ __forceinline__ void tt_out(const MCol& m, int n, double val, const OutMap& om, float* __restrict__ part,
                                       double alpha, int add) {
    if (n >= om.nr) return;
    if (m.idx & MC_DIRECT) {
        double* o = om.base + int64_t(m.idx & ~MC_DIRECT) * om.rs + int64_t(n) * om.cs;
        if (add) *o += alpha * val;
        else *o = val;
    } else {
        part[size_t(m.idx) * MR_RB + n] = float(val);
    }
}

// Fixed-order sum of the per-warp accumulators of an N-form tile
// (red[(w * TILE + row) * MR_RB + k]) and the update of the output rows.
__device__ __forceinline__ void nform_store(const double* red, int out, int rows, const OutMap& om, double alpha,
                                            int add) {
    for (int i = threadIdx.x; i < TILE * MR_RB; i += TC_WARPS * 32) {
        const int row = i % TILE, k = i / TILE;
        if (row >= rows || k >= om.nr) continue;
        double sum = 0.0;
#pragma unroll
        for (int w = 0; w < TC_WARPS; ++w) sum += red[(w * TILE + row) * MR_RB + k];
        double* o = om.base + int64_t(out + row) * om.rs + int64_t(k) * om.cs;
        if (add) *o += alpha * sum;
        else *o = sum;
    }
}

// ------------------------------------------------------- 16-bit chunks
// Tile T-form: one CTA per input tile (stream segment); the warps take the
// segment's 32-column stages round-robin.  Each column result is complete
// (the contraction covers the whole tile) and goes to its output or partial
// slot through the column table.  Fragments (natural placement): A[m][k] =
// stream column m, tile row k, read with ldmatrix from the staged columns;
// B[k][n] = x row k, right-hand side n.
template <int FMT>
__device__ __forceinline__ void ttform_tc(const MSeg& sg, uint8_t* smem, const MCol* __restrict__ cols,
                                          const uint8_t* __restrict__ A, const double* __restrict__ vin,
                                          const OutMap& om, float* __restrict__ part, double alpha, int add) {
    using O = TcOp<FMT>;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, t = lane & 3;
    uint8_t* ring = smem + warp * (TC_STAGES_TT * TC_STAGE_T16);
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
    // unscaling of the right-hand sides 2t and 2t+1 (the output columns of
    // this lane's accumulator fragment)
    const double inv0 = exp_unscale(__shfl_sync(0xffffffffu, E, 8 * t));
    const double inv1 = exp_unscale(__shfl_sync(0xffffffffu, E, 8 * t + 4));
    uint32_t bh[4][2], bl[4][2];
#pragma unroll
    for (int kt = 0; kt < 4; ++kt) {
        tc_split<FMT>(xv[kt][0], xv[kt][1], s, bh[kt][0], bl[kt][0]);
        tc_split<FMT>(xv[kt][2], xv[kt][3], s, bh[kt][1], bl[kt][1]);
    }
    const int colb = sg.ld * 2, ncols = int(sg.ncols);
    const uint8_t* base = A + size_t(sg.a16) * 16;
    const MCol* ctab = cols + sg.col0;
    const int nkt = (sg.rows + 15) / 16;
    // ldmatrix row of this lane: column + 8 for lanes 8-15 and 24-31, rows + 8 for lanes 16-31
    const int lcol = (lane & 7) + ((lane >> 3) & 1) * 8, lrow = ((lane >> 4) & 1) * 8;
    MCol mc = warp * 32 + lane < ncols ? ld_mcol(ctab + warp * 32 + lane) : MCol{0u, 0.f};
    warp_stream<TC_STAGES_TT>(
        (ncols + 31) / 32, warp,
        [&](int slot, int st) {
            uint8_t* sa = ring + slot * TC_STAGE_T16;
            const int c0 = 32 * st;
            stage_run<8, 32>(sa, TC_A16_STRIDE, base, c0, ncols, colb, lane);
            reinterpret_cast<MCol*>(sa + 32 * TC_A16_STRIDE)[lane] = mc;
            const int cn = c0 + 32 * TC_WARPS + lane;
            mc = cn < ncols ? ld_mcol(ctab + cn) : MCol{0u, 0.f};
        },
        [&](int slot, int st) {
            const uint8_t* sa = ring + slot * TC_STAGE_T16;
            const MCol* tab = reinterpret_cast<const MCol*>(sa + 32 * TC_A16_STRIDE);
            const int cnt = min(32, ncols - 32 * st);
            for (int mt = 0; 16 * mt < cnt; ++mt) {
                float d[4] = {0.f, 0.f, 0.f, 0.f};
                const uint8_t* row0 = sa + (16 * mt + lcol) * TC_A16_STRIDE + 2 * lrow;
#pragma unroll
                for (int kt = 0; kt < 4; ++kt) {
                    if (kt >= nkt) break;
                    uint32_t a[4];
                    ldsm_x4(a, row0 + 32 * kt);
                    O::mma(d, a, bh[kt][0], bh[kt][1]);
                    O::mma(d, a, bl[kt][0], bl[kt][1]);
                }
                const int c = 16 * mt + g;
                if (c < cnt) {
                    const MCol m = tab[c];
                    tt_out(m, 2 * t, double(d[0]) * (double(m.scale) * inv0), om, part, alpha, add);
                    tt_out(m, 2 * t + 1, double(d[1]) * (double(m.scale) * inv1), om, part, alpha, add);
                }
                if (c + 8 < cnt) {
                    const MCol m = tab[c + 8];
                    tt_out(m, 2 * t, double(d[2]) * (double(m.scale) * inv0), om, part, alpha, add);
                    tt_out(m, 2 * t + 1, double(d[3]) * (double(m.scale) * inv1), om, part, alpha, add);
                }
            }
        });
}

// N-form: one CTA per output tile (stream segment); the warps take the
// segment's 32-column stages round-robin.  The column scales are folded into
// the vector operand (B = scale * v, then one power-of-two scale per stage
// and right-hand side), so a whole stage accumulates in one set of MMA
// results and is added to FP64 once.  Fragments (natural placement):
// A[m][k] = tile row m, stream column k, read with ldmatrix.trans; lane
// (g, t) accumulates rows 16i + g, 16i + g + 8 (i < 4) for right-hand sides
// 2t, 2t+1; fixed-order cross-warp sum at the end.
template <int FMT>
__global__ void __launch_bounds__(TC_WARPS * 32, HLRC_N16_MINB)
k_nform_tc(const MSeg* __restrict__ segs, const MCol* __restrict__ cols, const uint8_t* __restrict__ A,
           const double* __restrict__ vx, const double* __restrict__ vt, OutMap om, double alpha, int add) {
    using O = TcOp<FMT>;
    extern __shared__ __align__(16) uint8_t smem[];
    const MSeg sg = segs[blockIdx.x];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, t = lane & 3;
    uint8_t* ring = smem + warp * (TC_STAGES_N16 * TC_STAGE_N16);
    const int colb = sg.ld * 2, ncols = int(sg.ncols);
    const uint8_t* base = A + size_t(sg.a16) * 16;
    const MCol* ctab = cols + sg.col0;
    const int nmt = (sg.rows + 15) / 16;
    // ldmatrix.trans row of this lane: column + 8 for lanes 16-31, rows + 8 for lanes 8-15 and 24-31
    const int lcol = (lane & 7) + ((lane >> 4) & 1) * 8, lrow = ((lane >> 3) & 1) * 8;
    double acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i) acc[i][0] = acc[i][1] = acc[i][2] = acc[i][3] = 0.0;
    MCol mc = warp * 32 + lane < ncols ? ld_mcol(ctab + warp * 32 + lane) : MCol{0u, 0.f};
    warp_stream<TC_STAGES_N16>(
        (ncols + 31) / 32, warp,
        [&](int slot, int st) {
            uint8_t* sa = ring + slot * TC_STAGE_N16;
            const int c0 = 32 * st;
            stage_run<8, 32>(sa, TC_A16_STRIDE, base, c0, ncols, colb, lane);
            stage_vector<32>(sa + 32 * TC_A16_STRIDE, mc.idx, c0, ncols, vx, vt, lane);
            reinterpret_cast<float*>(sa + 32 * (TC_A16_STRIDE + TC_V_STRIDE))[lane] = mc.scale;
            const int cn = c0 + 32 * TC_WARPS + lane;
            mc = cn < ncols ? ld_mcol(ctab + cn) : MCol{0u, 0.f};
        },
        [&](int slot, int st) {
            const uint8_t* sa = ring + slot * TC_STAGE_N16;
            const double* sv = reinterpret_cast<const double*>(sa + 32 * TC_A16_STRIDE);
            const float* ssc = reinterpret_cast<const float*>(sa + 32 * (TC_A16_STRIDE + TC_V_STRIDE));
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
            float d[4][4];
#pragma unroll
            for (int i = 0; i < 4; ++i) d[i][0] = d[i][1] = d[i][2] = d[i][3] = 0.f;
#pragma unroll
            for (int kt = 0; kt < 2; ++kt) {
                if (kt >= nkt) break;
                uint32_t bh0, bl0, bh1, bl1;
                tc_split<FMT>(bv[kt][0], bv[kt][1], s, bh0, bl0);
                tc_split<FMT>(bv[kt][2], bv[kt][3], s, bh1, bl1);
                const uint8_t* row0 = sa + (16 * kt + lcol) * TC_A16_STRIDE + 2 * lrow;
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    if (i >= nmt) break;
                    uint32_t a[4];
                    ldsm_x4_t(a, row0 + 32 * i);
                    O::mma(d[i], a, bh0, bh1);
                    O::mma(d[i], a, bl0, bl1);
                }
            }
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                acc[i][0] = fma(double(d[i][0]), f0, acc[i][0]);
                acc[i][1] = fma(double(d[i][1]), f1, acc[i][1]);
                acc[i][2] = fma(double(d[i][2]), f0, acc[i][2]);
                acc[i][3] = fma(double(d[i][3]), f1, acc[i][3]);
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

// --------------------------------------------------------- FP32 chunks
// FP32 columns run on the FP64 tensor cores (mma.sync m8n8k4 f64): FP32
// values convert to FP64 exactly, so the products are exact and the sums
// FP64, and no operand needs splitting.  Both forms read 8-byte pairs of
// rows from staged columns at a 288-byte stride (free of bank conflicts).
//   N-form: contraction = stream columns 4ks + t; m-tile 2p + b takes tile
//     row 16p + 2g + b as its fragment row g; the accumulators are the MMA
//     results themselves (FP64).
//   tile T-form: contraction = tile rows, k-step 2j + b maps fragment k = t to
//     row 8j + 2t + b; m-tiles are 8 stream columns.

// Tile T-form: one CTA per input tile; x in FP64 registers; 16-column stages.
__device__ __forceinline__ void ttform_d32(const MSeg& sg, uint8_t* smem, const MCol* __restrict__ cols,
                                           const uint8_t* __restrict__ A, const double* __restrict__ vin,
                                           const OutMap& om, float* __restrict__ part, double alpha, int add) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, t = lane & 3;
    uint8_t* ring = smem + warp * (TC_STAGES_TT * TC_STAGE_T32);
    // x of the lane: rows 8j + 2t + b (j < 8, b < 2), right-hand side g
    double xv[16];
#pragma unroll
    for (int jj = 0; jj < 8; ++jj)
#pragma unroll
        for (int b = 0; b < 2; ++b) {
            const int row = 8 * jj + 2 * t + b;
            xv[2 * jj + b] = row < sg.rows ? __ldg(vin + size_t(sg.vo + row) * MR_RB + g) : 0.0;
        }
    const int colb = sg.ld * 4, ncols = int(sg.ncols);
    const uint8_t* base = A + size_t(sg.a16) * 16;
    const MCol* ctab = cols + sg.col0;
    const int nj = (sg.rows + 7) / 8;
    MCol mc = (lane < 16 && warp * 16 + lane < ncols) ? ld_mcol(ctab + warp * 16 + lane) : MCol{0u, 0.f};
    warp_stream<TC_STAGES_TT>(
        (ncols + 15) / 16, warp,
        [&](int slot, int st) {
            uint8_t* sa = ring + slot * TC_STAGE_T32;
            const int c0 = 16 * st;
            stage_run<16, 16>(sa, TC_A32_STRIDE, base, c0, ncols, colb, lane);
            if (lane < 16) reinterpret_cast<MCol*>(sa + 16 * TC_A32_STRIDE)[lane] = mc;
            const int cn = c0 + 16 * TC_WARPS + lane;
            mc = (lane < 16 && cn < ncols) ? ld_mcol(ctab + cn) : MCol{0u, 0.f};
        },
        [&](int slot, int st) {
            const uint8_t* sa = ring + slot * TC_STAGE_T32;
            const MCol* tab = reinterpret_cast<const MCol*>(sa + 16 * TC_A32_STRIDE);
            const int cnt = min(16, ncols - 16 * st);
#pragma unroll
            for (int mt = 0; mt < 2; ++mt) {
                if (8 * mt >= cnt) break;
                const uint8_t* ca = sa + (8 * mt + g) * TC_A32_STRIDE + 8 * t;
                double d[2] = {0.0, 0.0};
                // all 8 row steps: rows past the tile hold zero-filled
                // columns and zero x entries
                (void)nj;
#pragma unroll
                for (int jj = 0; jj < 8; ++jj) {
                    const float2 a = *reinterpret_cast<const float2*>(ca + 32 * jj);
                    dmma(d, double(a.x), xv[2 * jj]);
                    dmma(d, double(a.y), xv[2 * jj + 1]);
                }
                const int c = 8 * mt + g;
                if (c < cnt) {
                    const MCol m = tab[c];
                    tt_out(m, 2 * t, d[0] * double(m.scale), om, part, alpha, add);
                    tt_out(m, 2 * t + 1, d[1] * double(m.scale), om, part, alpha, add);
                }
            }
        });
}

// N-form: one CTA per output tile; 16-column stages; the vector entries (times
// the column scale) are the B operand, and the MMA accumulates in FP64.
__global__ void __launch_bounds__(TC_WARPS * 32)
k_nform_d32(const MSeg* __restrict__ segs, const MCol* __restrict__ cols, const uint8_t* __restrict__ A,
            const double* __restrict__ vx, const double* __restrict__ vt, OutMap om, double alpha, int add) {
    extern __shared__ __align__(16) uint8_t smem[];
    const MSeg sg = segs[blockIdx.x];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, t = lane & 3;
    uint8_t* ring = smem + warp * (TC_STAGES_D32 * TC_STAGE_N32);
    const int colb = sg.ld * 4, ncols = int(sg.ncols);
    const uint8_t* base = A + size_t(sg.a16) * 16;
    const MCol* ctab = cols + sg.col0;
    const int np = (sg.rows + 15) / 16;
    // acc[2p + b]: tile row 16p + 2g + b, right-hand sides 2t, 2t+1
    double acc[8][2];
#pragma unroll
    for (int i = 0; i < 8; ++i) acc[i][0] = acc[i][1] = 0.0;
    MCol mc = (lane < 16 && warp * 16 + lane < ncols) ? ld_mcol(ctab + warp * 16 + lane) : MCol{0u, 0.f};
    warp_stream<TC_STAGES_D32>(
        (ncols + 15) / 16, warp,
        [&](int slot, int st) {
            uint8_t* sa = ring + slot * TC_STAGE_N32;
            const int c0 = 16 * st;
            stage_run<16, 16>(sa, TC_A32_STRIDE, base, c0, ncols, colb, lane);
            stage_vector<16>(sa + 16 * TC_A32_STRIDE, mc.idx, c0, ncols, vx, vt, lane);
            if (lane < 16) reinterpret_cast<float*>(sa + 16 * (TC_A32_STRIDE + TC_V_STRIDE))[lane] = mc.scale;
            const int cn = c0 + 16 * TC_WARPS + lane;
            mc = (lane < 16 && cn < ncols) ? ld_mcol(ctab + cn) : MCol{0u, 0.f};
        },
        [&](int slot, int st) {
            const uint8_t* sa = ring + slot * TC_STAGE_N32;
            const double* sv = reinterpret_cast<const double*>(sa + 16 * TC_A32_STRIDE);
            const float* ssc = reinterpret_cast<const float*>(sa + 16 * (TC_A32_STRIDE + TC_V_STRIDE));
            // every stage runs in full: the copies zero-fill the columns past
            // the run (and their vector entries and scales) and the rows past
            // the column height, so the extra products add zeros, and the
            // loads and conversions of a stage can all be issued up front
            (void)np;
#pragma unroll
            for (int ks = 0; ks < 4; ++ks) {
                const int col = 4 * ks + t;
                const double b = sv[col * (TC_V_STRIDE / 8) + g] * double(ssc[col]);
                const uint8_t* ca = sa + col * TC_A32_STRIDE + 8 * g;
#pragma unroll
                for (int p = 0; p < 4; ++p) {
                    const float2 a = *reinterpret_cast<const float2*>(ca + 64 * p);
                    dmma(acc[2 * p], double(a.x), b);
                    dmma(acc[2 * p + 1], double(a.y), b);
                }
            }
        });
    __syncthreads();
    double* red = reinterpret_cast<double*>(smem);
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int row = 16 * (i >> 1) + 2 * g + (i & 1);
        red[(warp * TILE + row) * MR_RB + 2 * t] = acc[i][0];
        red[(warp * TILE + row) * MR_RB + 2 * t + 1] = acc[i][1];
    }
    __syncthreads();
    nform_store(red, int(sg.vo), sg.rows, om, alpha, add);
}

// One tile T-form pass of a reduced-precision store in one grid: the first
// n32 CTAs take the FP32 runs (FP64 tensor cores), the others the runs of the
// 16-bit format F16.  The outputs of the two formats are disjoint.  Dynamic
// shared memory: tc_smem_bytes(TC_STAGE_TT, TC_STAGES_TT).
constexpr int TC_STAGE_TT = TC_STAGE_T16 > TC_STAGE_T32 ? TC_STAGE_T16 : TC_STAGE_T32;
template <int F16>
__global__ void __launch_bounds__(TC_WARPS * 32, HLRC_TT_MINB)
k_ttform_mr(const MSeg* __restrict__ segs32, int n32, const MSeg* __restrict__ segs16, const MCol* __restrict__ cols,
            const uint8_t* __restrict__ A, const double* __restrict__ vin, OutMap om, float* __restrict__ part,
            double alpha, int add) {
    extern __shared__ __align__(16) uint8_t smem[];
    if (int(blockIdx.x) < n32) ttform_d32(segs32[blockIdx.x], smem, cols, A, vin, om, part, alpha, add);
    else ttform_tc<F16>(segs16[blockIdx.x - n32], smem, cols, A, vin, om, part, alpha, add);
}

}  // namespace hlrc
