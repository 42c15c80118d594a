// Tensor-core multi-right-hand-side kernels for reduced-precision stores,
// MR_RB = 8 right-hand sides per launch.
//
// With 8 right-hand sides a chunk product is a small dense contraction:
// 16-bit chunks (scaled FP16 / BF16) run as mma.sync m16n8k16 tiles, FP32
// chunks as m16n8k8 TF32 tiles with the three-term split, all with FP32
// accumulation inside a chunk and FP64 accumulation across chunks.  The
// vector operand is split into two 16-bit terms, hi = round(s*v) and
// lo = round(s*v - hi), with a power-of-two scale s per chunk (N-form) or
// input tile (tile T-form) and right-hand side, so the product keeps about
// 22 significant bits of v (FP16) or 16 (BF16) and the storage rounding of
// the matrix stays the dominant error.
//
// Data movement.  Each warp streams its packs (work items of up to two
// chunks) through a ring of TC_STAGES shared-memory stages filled with
// cp.async 16-byte copies, so several chunks per warp are in flight without
// holding registers.  A stage holds the chunk columns at a padded stride
// (no bank conflicts for the fragment loads) and, for the N-form, the vector
// entries of those columns; units outside the chunk are zero-filled by the
// copies themselves, so no stage ever holds stale data.  Fragments come from
// ldmatrix: plain for the tile T-form (A = chunk^T, rows contiguous), .trans
// for the N-form (A = chunk, columns contiguous).  Fragment rows or columns
// that fall past the pack's columns read the stage's last column instead:
// their products either meet a zero vector entry or land in accumulator
// rows that are never stored.  FP32 N-form fragments are
// read as 16-byte runs of 4 rows with the row placement described at
// k_nform_tc32.
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
constexpr int TC_A32N_STRIDE = 288;   // FP32 column (256 B) + 32 B pad, N-form (16-byte reads)
constexpr int TC_A32T_STRIDE = 272;   // FP32 column + 16 B pad, tile T-form (ldmatrix reads)
constexpr int TC_V_STRIDE = 80;       // MR_RB doubles of one vector column + 16 B pad
constexpr int TC_STAGE_N16 = 32 * TC_A16_STRIDE + 32 * TC_V_STRIDE;
constexpr int TC_STAGE_T16 = 32 * TC_A16_STRIDE;
constexpr int TC_STAGE_N32 = 16 * TC_A32N_STRIDE + 16 * TC_V_STRIDE;
constexpr int TC_STAGE_T32 = 16 * TC_A32T_STRIDE;

// dynamic shared memory of a launch: the warps' rings, then per warp one
// 32-byte pack descriptor per stage
constexpr int tc_smem_bytes(int stage) { return TC_WARPS * TC_STAGES * (stage + 32); }

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

__device__ __forceinline__ void mma_tf32(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm("mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// d += A B for the three-term split of A (four FP32 values, as bits) and
// B = (bb, bs); the small products first
__device__ __forceinline__ void mma_tf32x3(float (&d)[4], const uint32_t (&a)[4], const uint32_t (&bb)[2],
                                           const uint32_t (&bs)[2]) {
    uint32_t ab[4], as[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) tf32_split(__uint_as_float(a[i]), ab[i], as[i]);
    mma_tf32(d, as, bb[0], bb[1]);
    mma_tf32(d, ab, bs[0], bs[1]);
    mma_tf32(d, ab, bb[0], bb[1]);
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

// One warp's pass over packs c0, c0 + step, ... < ce through its ring of
// TC_STAGES stages: issue(stage, pack) starts the copies of a pack, and
// compute(stage, pack) consumes a stage once its copies have landed.  Pack
// descriptors are read one pack ahead and kept beside their stage.
template <typename Pack, typename Issue, typename Compute>
__device__ __forceinline__ void warp_ring(const Pack* __restrict__ packs, uint32_t c0, uint32_t ce, uint32_t step,
                                          Pack* sdesc, int lane, Issue&& issue, Compute&& compute) {
    const int n = c0 < ce ? int((ce - c0 + step - 1) / step) : 0;
    Pack nxt;
    if (n > 0) nxt = ld_pack(packs + c0);
    int issued = 0;
    auto issue_next = [&]() {
        if (issued < n) {
            const Pack cur = nxt;
            if (issued + 1 < n) nxt = ld_pack(packs + c0 + uint32_t(issued + 1) * step);
            const int st = issued % TC_STAGES;
            if (lane == 0) sdesc[st] = cur;
            issue(st, cur);
            ++issued;
        }
        cp_commit();
    };
#pragma unroll
    for (int k = 0; k < TC_STAGES - 1; ++k) issue_next();
    for (int k = 0; k < n; ++k) {
        issue_next();
        cp_wait<TC_STAGES - 1>();
        __syncwarp();
        const int st = k % TC_STAGES;
        compute(st, sdesc[st]);
        __syncwarp();
    }
}

// Copies of the columns of a pack into a stage: columns [0, nc0) from part
// 0, [nc0, nc0 + nc1) from part 1, zero-filled up to COLS.  A column holds
// `units` 16-byte units (ld * element bytes / 16) at global stride `units`
// and shared stride `stride`; UPL units make a full 64-row column, and lane
// l copies unit l % UPL of columns l / UPL + (32 / UPL) i.  The parts are
// selected through two base pointers (no indexing into the descriptor).
template <int UPL, int COLS, typename Pack>
__device__ __forceinline__ void stage_columns(uint8_t* dst, int stride, const uint8_t* A, const Pack& pk, int units,
                                              int lane) {
    const int u = lane % UPL;
    const int n0 = pk.p[0].nc, ntot = n0 + pk.p[1].nc;
    const size_t cb = size_t(units) * 16;
    const uint8_t* b0 = A + size_t(pk.p[0].a16) * 16 + u * 16;
    const uint8_t* b1 = A + size_t(pk.p[1].a16) * 16 + u * 16 - size_t(n0) * cb;
    uint8_t* d = dst + (lane / UPL) * stride + u * 16;
#pragma unroll
    for (int i = 0; i < COLS * UPL / 32; ++i) {
        const int j = lane / UPL + (32 / UPL) * i;
        const bool ok = j < ntot && u < units;
        const uint8_t* src = (j < n0 ? b0 : b1) + size_t(j) * cb;
        cp16(d + (32 / UPL) * i * stride, ok ? src : A, ok);
    }
}

// Copies of the vector entries (MR_RB doubles = 4 units per column) of the
// columns of an N-form pack into a stage, at shared stride TC_V_STRIDE.
template <int COLS, typename Pack>
__device__ __forceinline__ void stage_vector(uint8_t* dst, const double* vx, const double* vt, const Pack& pk,
                                             int lane) {
    const int u = lane & 3;
    const int n0 = pk.p[0].nc, ntot = n0 + pk.p[1].nc;
    const uint32_t o0 = pk.p[0].v_off, o1 = pk.p[1].v_off;
    const double* v0 = ((o0 & VEC_T) ? vt + size_t(o0 & ~VEC_T) * MR_RB : vx + size_t(o0) * MR_RB) + 2 * u;
    const double* v1 = ((o1 & VEC_T) ? vt + size_t(o1 & ~VEC_T) * MR_RB : vx + size_t(o1) * MR_RB) + 2 * u -
                       size_t(n0) * MR_RB;
    uint8_t* d = dst + (lane >> 2) * TC_V_STRIDE + u * 16;
#pragma unroll
    for (int i = 0; i < COLS / 8; ++i) {
        const int j = (lane >> 2) + 8 * i;
        const bool ok = j < ntot;
        const double* src = (j < n0 ? v0 : v1) + size_t(j) * MR_RB;
        cp16(d + 8 * i * TC_V_STRIDE, ok ? static_cast<const void*>(src) : vx, ok);
    }
}

// Shared epilogue of the tile T-forms: value val of chunk column col,
// right-hand side n goes to its output or to its partial slot.
template <typename Chunk>
__device__ __forceinline__ void tt_store(const Chunk& ch, int col, int n, double val, const OutMap& om,
                                         double* __restrict__ part, double alpha, int add) {
    if (col >= ch.nc || n >= om.nr) return;
    if (ch.flags & TT_DIRECT) {
        double* o = om.base + int64_t(ch.out + col) * om.rs + int64_t(n) * om.cs;
        if (add) *o += alpha * val;
        else *o = val;
    } else {
        part[size_t(ch.out + col) * MR_RB + n] = val;
    }
}

// Fixed-order sum of the per-warp accumulators of an N-form tile
// (red[(w * TILE + row) * MR_RB + k]) and the update of the output rows.
__device__ __forceinline__ void nform_store(const double* red, const NSeg& sg, const OutMap& om, double alpha,
                                            int add) {
    for (int i = threadIdx.x; i < TILE * MR_RB; i += TC_WARPS * 32) {
        const int row = i % TILE, k = i / TILE;
        if (row >= sg.rows || k >= om.nr) continue;
        double sum = 0.0;
#pragma unroll
        for (int w = 0; w < TC_WARPS; ++w) sum += red[(w * TILE + row) * MR_RB + k];
        double* o = om.base + int64_t(sg.out + row) * om.rs + int64_t(k) * om.cs;
        if (add) *o += alpha * sum;
        else *o = sum;
    }
}

// ------------------------------------------------------- 16-bit chunks
// Tile T-form: one CTA per input tile; each chunk result is complete (the
// contraction covers the whole tile) and goes to its output or partial slot.
// Fragments (natural placement): A[m][k] = chunk column m, tile row k, read
// with ldmatrix from the staged columns; B[k][n] = x row k, right-hand side n.
template <int FMT>
__global__ void __launch_bounds__(TC_WARPS * 32)
k_ttform_tc(const TTSeg* __restrict__ segs, const QTTPack* __restrict__ packs, const uint8_t* __restrict__ A,
            const double* __restrict__ vin, OutMap om, double* __restrict__ part, double alpha, int add) {
    using O = TcOp<FMT>;
    extern __shared__ __align__(16) uint8_t smem[];
    const TTSeg sg = segs[blockIdx.x];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, t = lane & 3;
    uint8_t* ring = smem + warp * (TC_STAGES * TC_STAGE_T16);
    QTTPack* sdesc = reinterpret_cast<QTTPack*>(smem + TC_WARPS * TC_STAGES * TC_STAGE_T16) + warp * TC_STAGES;
    // x entries of the lane: rows 16kt + 2t + {0, 1, 8, 9} (kt < 4), right-hand side g
    double xv[4][4];
    int E = 0;
#pragma unroll
    for (int kt = 0; kt < 4; ++kt)
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int row = 16 * kt + 2 * t + (j & 1) + 8 * (j >> 1);
            const double v = row < sg.rows ? __ldg(vin + size_t(sg.v_off + row) * MR_RB + g) : 0.0;
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
    const int units = sg.ld / 8;
    const int nkt = (sg.rows + 15) / 16;
    // ldmatrix row of this lane: column + 8 for lanes 8-15 and 24-31, rows + 8 for lanes 16-31
    const int lcol = (lane & 7) + ((lane >> 3) & 1) * 8, lrow = ((lane >> 4) & 1) * 8;
    warp_ring(
        packs, sg.cb + warp, sg.ce, TC_WARPS, sdesc, lane,
        [&](int st, const QTTPack& pk) {
            stage_columns<8, 32>(ring + st * TC_STAGE_T16, TC_A16_STRIDE, A, pk, units, lane);
        },
        [&](int st, const QTTPack& pk) {
            const uint8_t* sa = ring + st * TC_STAGE_T16;
            int col0 = 0;
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const QTTChunk& ch = pk.p[q];
                const double f0 = double(ch.scale) * inv0, f1 = double(ch.scale) * inv1;
                for (int mt = 0; 16 * mt < ch.nc; ++mt) {
                    float d[4] = {0.f, 0.f, 0.f, 0.f};
                    const uint8_t* base = sa + min(col0 + 16 * mt + lcol, 31) * TC_A16_STRIDE + 2 * lrow;
#pragma unroll
                    for (int kt = 0; kt < 4; ++kt) {
                        if (kt >= nkt) break;
                        uint32_t a[4];
                        ldsm_x4(a, base + 32 * kt);
                        O::mma(d, a, bh[kt][0], bh[kt][1]);
                        O::mma(d, a, bl[kt][0], bl[kt][1]);
                    }
                    const int c = 16 * mt + g;
                    tt_store(ch, c, 2 * t, double(d[0]) * f0, om, part, alpha, add);
                    tt_store(ch, c, 2 * t + 1, double(d[1]) * f1, om, part, alpha, add);
                    tt_store(ch, c + 8, 2 * t, double(d[2]) * f0, om, part, alpha, add);
                    tt_store(ch, c + 8, 2 * t + 1, double(d[3]) * f1, om, part, alpha, add);
                }
                col0 += ch.nc;
            }
        });
}

// N-form: one CTA per output tile.  Fragments (natural placement): A[m][k] =
// tile row m, chunk column k, read with ldmatrix.trans from the staged
// columns; B[k][n] = vector entry of column k, right-hand side n, from the
// staged vector.  Lane (g, t) accumulates rows 16i + g, 16i + g + 8 (i < 4)
// for right-hand sides 2t, 2t+1 in FP64; fixed-order cross-warp sum.
template <int FMT>
__global__ void __launch_bounds__(TC_WARPS * 32)
k_nform_tc(const NSeg* __restrict__ segs, const QNPack* __restrict__ packs, const uint8_t* __restrict__ A,
           const double* __restrict__ vx, const double* __restrict__ vt, OutMap om, double alpha, int add) {
    using O = TcOp<FMT>;
    extern __shared__ __align__(16) uint8_t smem[];
    const NSeg sg = segs[blockIdx.x];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, t = lane & 3;
    uint8_t* ring = smem + warp * (TC_STAGES * TC_STAGE_N16);
    QNPack* sdesc = reinterpret_cast<QNPack*>(smem + TC_WARPS * TC_STAGES * TC_STAGE_N16) + warp * TC_STAGES;
    const int units = sg.ld / 8;
    const int nmt = (sg.rows + 15) / 16;
    // ldmatrix.trans row of this lane: column + 8 for lanes 16-31, rows + 8 for lanes 8-15 and 24-31
    const int lcol = (lane & 7) + ((lane >> 4) & 1) * 8, lrow = ((lane >> 3) & 1) * 8;
    double acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i) acc[i][0] = acc[i][1] = acc[i][2] = acc[i][3] = 0.0;
    warp_ring(
        packs, sg.cb + warp, sg.ce, TC_WARPS, sdesc, lane,
        [&](int st, const QNPack& pk) {
            uint8_t* sa = ring + st * TC_STAGE_N16;
            stage_columns<8, 32>(sa, TC_A16_STRIDE, A, pk, units, lane);
            stage_vector<32>(sa + 32 * TC_A16_STRIDE, vx, vt, pk, lane);
        },
        [&](int st, const QNPack& pk) {
            const uint8_t* sa = ring + st * TC_STAGE_N16;
            const double* sv = reinterpret_cast<const double*>(sa + 32 * TC_A16_STRIDE);
            int col0 = 0;
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const QNChunk& ch = pk.p[q];
                if (ch.nc == 0) continue;
                const int nkt = ch.nc > 16 ? 2 : 1;
                // vector operand: columns 16kt + 2t + {0, 1, 8, 9}, right-hand side g
                double bv[2][4];
                int E = 0;
#pragma unroll
                for (int kt = 0; kt < 2; ++kt)
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        const int col = 16 * kt + 2 * t + (j & 1) + 8 * (j >> 1);
                        const double x = col < ch.nc ? sv[(col0 + col) * (TC_V_STRIDE / 8) + g] : 0.0;
                        bv[kt][j] = x;
                        E = max(E, dexp(x));
                    }
                E = quad_max(E);
                const double s = exp_scale(E);
                const double f0 = double(ch.scale) * exp_unscale(__shfl_sync(0xffffffffu, E, 8 * t));
                const double f1 = double(ch.scale) * exp_unscale(__shfl_sync(0xffffffffu, E, 8 * t + 4));
                float d[4][4];
#pragma unroll
                for (int i = 0; i < 4; ++i) d[i][0] = d[i][1] = d[i][2] = d[i][3] = 0.f;
#pragma unroll
                for (int kt = 0; kt < 2; ++kt) {
                    if (kt >= nkt) break;
                    uint32_t bh0, bl0, bh1, bl1;
                    tc_split<FMT>(bv[kt][0], bv[kt][1], s, bh0, bl0);
                    tc_split<FMT>(bv[kt][2], bv[kt][3], s, bh1, bl1);
                    const uint8_t* base = sa + min(col0 + 16 * kt + lcol, 31) * TC_A16_STRIDE + 2 * lrow;
#pragma unroll
                    for (int i = 0; i < 4; ++i) {
                        if (i >= nmt) break;
                        uint32_t a[4];
                        ldsm_x4_t(a, base + 32 * i);
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
                col0 += ch.nc;
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
    nform_store(red, sg, om, alpha, add);
}

// --------------------------------------------------------- FP32 chunks
// Tile T-form on TF32 tiles.  ldmatrix (b16 granules) reads 32-bit A
// fragments directly: a 16-byte row of a staged column is 4 tile rows, and
// lane (g, t) receives granule pair (g, t) = chunk column g, tile row t of an
// 8 x 4 block, which is the m16n8k8 TF32 A layout.
__global__ void __launch_bounds__(TC_WARPS * 32)
k_ttform_tc32(const TTSeg* __restrict__ segs, const QTTPack* __restrict__ packs, const uint8_t* __restrict__ A,
              const double* __restrict__ vin, OutMap om, double* __restrict__ part, double alpha, int add) {
    extern __shared__ __align__(16) uint8_t smem[];
    const TTSeg sg = segs[blockIdx.x];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, t = lane & 3;
    uint8_t* ring = smem + warp * (TC_STAGES * TC_STAGE_T32);
    QTTPack* sdesc = reinterpret_cast<QTTPack*>(smem + TC_WARPS * TC_STAGES * TC_STAGE_T32) + warp * TC_STAGES;
    // x entries of the lane: rows 8ks + t and 8ks + t + 4 (ks < 8), right-hand side g
    double xv[8][2];
    int E = 0;
#pragma unroll
    for (int ks = 0; ks < 8; ++ks)
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const int row = 8 * ks + t + 4 * j;
            const double v = row < sg.rows ? __ldg(vin + size_t(sg.v_off + row) * MR_RB + g) : 0.0;
            xv[ks][j] = v;
            E = max(E, dexp(v));
        }
    E = quad_max(E);
    const double s = exp_scale(E);
    const double inv0 = exp_unscale(__shfl_sync(0xffffffffu, E, 8 * t));
    const double inv1 = exp_unscale(__shfl_sync(0xffffffffu, E, 8 * t + 4));
    uint32_t bb[8][2], bs[8][2];
#pragma unroll
    for (int ks = 0; ks < 8; ++ks)
#pragma unroll
        for (int j = 0; j < 2; ++j) tf32_split(float(xv[ks][j] * s), bb[ks][j], bs[ks][j]);
    const int units = sg.ld / 4;
    const int nks = (sg.rows + 7) / 8;
    // ldmatrix row of this lane: column + 8 for lanes 8-15 and 24-31, rows + 4 for lanes 16-31
    const int lcol = (lane & 7) + ((lane >> 3) & 1) * 8, lrow = ((lane >> 4) & 1) * 4;
    warp_ring(
        packs, sg.cb + warp, sg.ce, TC_WARPS, sdesc, lane,
        [&](int st, const QTTPack& pk) {
            stage_columns<16, 16>(ring + st * TC_STAGE_T32, TC_A32T_STRIDE, A, pk, units, lane);
        },
        [&](int st, const QTTPack& pk) {
            const uint8_t* sa = ring + st * TC_STAGE_T32;
            int col0 = 0;
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const QTTChunk& ch = pk.p[q];
                if (ch.nc == 0) continue;
                float d[4] = {0.f, 0.f, 0.f, 0.f};
                const uint8_t* base = sa + min(col0 + lcol, 15) * TC_A32T_STRIDE + 4 * lrow;
#pragma unroll
                for (int ks = 0; ks < 8; ++ks) {
                    if (ks >= nks) break;
                    uint32_t a[4];
                    ldsm_x4(a, base + 32 * ks);
                    mma_tf32x3(d, a, bb[ks], bs[ks]);
                }
                const double f0 = double(ch.scale) * inv0, f1 = double(ch.scale) * inv1;
                tt_store(ch, g, 2 * t, double(d[0]) * f0, om, part, alpha, add);
                tt_store(ch, g, 2 * t + 1, double(d[1]) * f1, om, part, alpha, add);
                tt_store(ch, g + 8, 2 * t, double(d[2]) * f0, om, part, alpha, add);
                tt_store(ch, g + 8, 2 * t + 1, double(d[3]) * f1, om, part, alpha, add);
                col0 += ch.nc;
            }
        });
}

// N-form on TF32 tiles.  A 32-bit fragment cannot be transposed by
// ldmatrix, so a lane reads 16-byte runs of 4 rows: lane (g, t) takes rows
// 4g .. 4g+3 and 32+4g .. 32+4g+3 of chunk columns 8kt + t and 8kt + t + 4,
// and m-tile i uses rows 4g + 2i, 4g + 2i + 1 (i < 2), or 32 + 4g + 2(i-2)
// + {0, 1}, as its fragment rows g and g + 8.  The shared stride of 288 bytes
// keeps these reads free of bank conflicts.
__global__ void __launch_bounds__(TC_WARPS * 32)
k_nform_tc32(const NSeg* __restrict__ segs, const QNPack* __restrict__ packs, const uint8_t* __restrict__ A,
             const double* __restrict__ vx, const double* __restrict__ vt, OutMap om, double alpha, int add) {
    extern __shared__ __align__(16) uint8_t smem[];
    const NSeg sg = segs[blockIdx.x];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, t = lane & 3;
    uint8_t* ring = smem + warp * (TC_STAGES * TC_STAGE_N32);
    QNPack* sdesc = reinterpret_cast<QNPack*>(smem + TC_WARPS * TC_STAGES * TC_STAGE_N32) + warp * TC_STAGES;
    const int units = sg.ld / 4;
    const bool hi_rows = 32 < sg.ld;
    // accumulators: rows 4g + r and 32 + 4g + r (r < 4) -> acc[r] / acc[4 + r]
    double acc[8][2];
#pragma unroll
    for (int r = 0; r < 8; ++r) acc[r][0] = acc[r][1] = 0.0;
    warp_ring(
        packs, sg.cb + warp, sg.ce, TC_WARPS, sdesc, lane,
        [&](int st, const QNPack& pk) {
            uint8_t* sa = ring + st * TC_STAGE_N32;
            stage_columns<16, 16>(sa, TC_A32N_STRIDE, A, pk, units, lane);
            stage_vector<16>(sa + 16 * TC_A32N_STRIDE, vx, vt, pk, lane);
        },
        [&](int st, const QNPack& pk) {
            const uint8_t* sa = ring + st * TC_STAGE_N32;
            const double* sv = reinterpret_cast<const double*>(sa + 16 * TC_A32N_STRIDE);
            int col0 = 0;
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const QNChunk& ch = pk.p[q];
                if (ch.nc == 0) continue;
                const int nkt = ch.nc > 8 ? 2 : 1;
                // vector operand: columns 8kt + t and 8kt + t + 4, right-hand side g
                double bv[2][2];
                int E = 0;
#pragma unroll
                for (int kt = 0; kt < 2; ++kt)
#pragma unroll
                    for (int j = 0; j < 2; ++j) {
                        const int col = 8 * kt + t + 4 * j;
                        const double x = col < ch.nc ? sv[(col0 + col) * (TC_V_STRIDE / 8) + g] : 0.0;
                        bv[kt][j] = x;
                        E = max(E, dexp(x));
                    }
                E = quad_max(E);
                const double s = exp_scale(E);
                const double f0 = double(ch.scale) * exp_unscale(__shfl_sync(0xffffffffu, E, 8 * t));
                const double f1 = double(ch.scale) * exp_unscale(__shfl_sync(0xffffffffu, E, 8 * t + 4));
                float d[4][4];
#pragma unroll
                for (int i = 0; i < 4; ++i) d[i][0] = d[i][1] = d[i][2] = d[i][3] = 0.f;
#pragma unroll
                for (int kt = 0; kt < 2; ++kt) {
                    if (kt >= nkt) break;
                    uint32_t bb[2], bs[2];
                    tf32_split(float(bv[kt][0] * s), bb[0], bs[0]);
                    tf32_split(float(bv[kt][1] * s), bb[1], bs[1]);
                    const uint8_t* ca = sa + min(col0 + 8 * kt + t, 15) * TC_A32N_STRIDE + 16 * g;
                    const uint8_t* cb = sa + min(col0 + 8 * kt + t + 4, 15) * TC_A32N_STRIDE + 16 * g;
                    const uint4 La0 = *reinterpret_cast<const uint4*>(ca);
                    const uint4 Lb0 = *reinterpret_cast<const uint4*>(cb);
                    const uint32_t a0[4] = {La0.x, La0.y, Lb0.x, Lb0.y};
                    const uint32_t a1[4] = {La0.z, La0.w, Lb0.z, Lb0.w};
                    mma_tf32x3(d[0], a0, bb, bs);
                    mma_tf32x3(d[1], a1, bb, bs);
                    if (hi_rows) {
                        const uint4 La1 = *reinterpret_cast<const uint4*>(ca + 128);
                        const uint4 Lb1 = *reinterpret_cast<const uint4*>(cb + 128);
                        const uint32_t a2[4] = {La1.x, La1.y, Lb1.x, Lb1.y};
                        const uint32_t a3[4] = {La1.z, La1.w, Lb1.z, Lb1.w};
                        mma_tf32x3(d[2], a2, bb, bs);
                        mma_tf32x3(d[3], a3, bb, bs);
                    }
                }
                // m-tile i: fragment row g -> local row 2i, row g + 8 -> 2i + 1
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    acc[2 * i][0] = fma(double(d[i][0]), f0, acc[2 * i][0]);
                    acc[2 * i][1] = fma(double(d[i][1]), f1, acc[2 * i][1]);
                    acc[2 * i + 1][0] = fma(double(d[i][2]), f0, acc[2 * i + 1][0]);
                    acc[2 * i + 1][1] = fma(double(d[i][3]), f1, acc[2 * i + 1][1]);
                }
                col0 += ch.nc;
            }
        });
    __syncthreads();
    double* red = reinterpret_cast<double*>(smem);
    // local row l < 4 is tile row 4g + l, l >= 4 is 32 + 4g + (l - 4)
#pragma unroll
    for (int l = 0; l < 8; ++l) {
        const int row = (l < 4 ? 0 : 32) + 4 * g + (l & 3);
        red[(warp * TILE + row) * MR_RB + 2 * t] = acc[l][0];
        red[(warp * TILE + row) * MR_RB + 2 * t + 1] = acc[l][1];
    }
    __syncthreads();
    nform_store(red, sg, om, alpha, add);
}

}  // namespace hlrc
