// One-pass wide multi-right-hand-side product of 16-bit (FP16 / BF16)
// H-matrix stores on the Blackwell tensor cores (tcgen05.mma, accumulators in
// tensor memory): up to WIDE_RHS = 64 vectors per pass, the matrix streamed
// once.  This is the block apply of lrmatrix::apply_add on a blas::matrix X
// (include/hlr/matrix/lrmatrix.hh:681-746: T = V^H X, Y += U T) and of the
// dense leaves, over all leaves of the flattened layout at once.
//
// Vectors.  kind::f16 MMAs take two 16-bit operands of the same type, so
// every vector entry v (FP64) enters as two 16-bit terms, hi = round(v s)
// and lo = round(v s - hi), which keep about 22 (FP16) or 16 (BF16)
// significant bits; the storage rounding of the matrix stays the dominant
// error.  The terms of the 64 vectors of one entry form a 256-byte "split
// row" (term 2r = hi of vector r, 2r + 1 = lo), so hi and lo of a vector end
// up in neighbouring accumulator lanes (N-form) or columns (T-form).
//   x: one power-of-two scale 2^g_r per vector (max |x_r| 2^g_r in
//      [2^13, 2^14)), split once per pass into xs.
//   t = V^T x (per low-rank column, times 2^g_r): the T-form epilogue writes
//      it as a split row with its own power-of-two exponent e (the row's
//      largest |t| 2^g_r 2^-e in [2^13, 2^14)), into ts and texp.
//
// Kernels (op N):
//   k_wide_xmax / k_wide_xsplit   x -> xs (and g_r)
//   k_ttform_wide   one CTA per input tile: t = V^T x for the tile's run of V
//                   columns; A = 128 columns (K-major), B = the tile's xs
//                   rows (MN-major), D = 128 columns x 128 terms in TMEM
//                   (two buffers, so the epilogue of one block overlaps the
//                   MMAs of the next); single-tile outputs go straight to
//                   ts, the others to FP32 partials
//   k_ttfinish_wide   partials of multi-tile outputs summed in tile order
//                   (FP64), then split into ts
//   k_nform_wide    one CTA per output tile: y += U t + D x over the tile's
//                   run of columns; A = 128 terms of 32 columns (MN-major,
//                   gathered split rows), B = the 32 matrix columns
//                   (MN-major), D = 128 terms x 64 rows in TMEM
//
// Scales in the N-form.  Column c of the run carries its chunk's scale s_c
// and (t columns) the exponent e of its split row, f_c = s_c 2^e.  The CTA
// first finds the largest f over its run, F, and multiplies the staged
// matrix column by f_c / F (a power of two <= 1, exact unless the values
// drop below the 16-bit range, where they are negligible against the run's
// largest terms), so that one accumulator serves the whole run:
// y_r += alpha F 2^-g_r (acc_hi + acc_lo).  The tensor cores accumulate in
// FP32 over WIDE_FLUSH stages (64 columns) into one of two TMEM buffers; the
// epilogue warps add each finished buffer to an FP64 accumulator in shared
// memory while the MMAs fill the other, so long runs keep FP64 sums.
//
// Roles (224 threads): warps 0-3 read the accumulators (warp w reads TMEM
// lanes 32w .. 32w + 31), warp 4 allocates TMEM and issues the MMAs (one
// thread), warps 5-6 stage operands with 16-byte cp.async copies into the
// 128-byte-swizzled layouts, zero-filling everything outside the run.
// Stages are handed over with mbarriers: "full" (copies landed, made
// visible to the tensor cores' proxy, 64 producer arrivals), "empty" (the
// stage's MMAs completed, tcgen05.commit).  Every wait is bounded
// (tc5::mbar_wait) and checks a device error flag, so a wait that runs out
// sets bit 1 of the error word and all CTAs leave quickly, with their copies
// drained, their MMAs completed and their TMEM freed.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "kernels_mr.cuh"
#include "layout.hpp"
#include "tc5.cuh"

namespace hlrc {

constexpr int WIDE_RHS = 64;          // vectors per pass
constexpr int WIDE_TERMS = 128;       // 16-bit terms per split row
constexpr int WIDE_ROWB = 256;        // bytes per split row
constexpr int WIDE_THREADS = 224;     // 4 epilogue warps, 1 MMA warp, 2 producer warps
constexpr int WIDE_PRODUCERS = 64;
constexpr int WIDE_NS_N = 6;          // N-form stages (32 columns each): 2 CTAs per SM
constexpr int WIDE_FLUSH = 2;         // N-form stages per FP32 accumulation (64 columns), then added in FP64
constexpr int WIDE_NS_T = 4;          // tile T-form stages (128 columns each): 2 CTAs per SM (TMEM: 256 columns each)
constexpr int WIDE_LAG_N = WIDE_NS_N - 2;   // copy groups a producer keeps in flight
constexpr int WIDE_LAG_T = WIDE_NS_T - 1;
constexpr int WIDE_ERR_WAIT = 2;      // device error word bit: a wait of a wide kernel ran out

// N-form stage: A (vector terms, 2 M-atoms x 4 K-atoms) 8 KB, B (matrix, 4 K-atoms) 4 KB
constexpr int WIDE_N_STAGE = 12288;
// N-form FP64 accumulator in shared memory: [vector][row], rows padded to 65
// (the 16 lanes that add one row of 16 vectors hit 16 different bank pairs)
constexpr int WIDE_ACC_LD = TILE + 1;
constexpr int WIDE_ACC_BYTES = WIDE_RHS * WIDE_ACC_LD * 8;
// tile T-form: B (the tile's split rows: 2 N-atoms x 8 K-atoms) 16 KB, stages of A (16 M-atoms) 16 KB
constexpr int WIDE_T_B = 16384;
constexpr int WIDE_T_STAGE = 16384;
constexpr int WIDE_BAR_BYTES = 256;   // mbarriers and the TMEM address
constexpr int wide_smem_n() { return 1024 + WIDE_NS_N * WIDE_N_STAGE + WIDE_ACC_BYTES + WIDE_BAR_BYTES; }
constexpr int wide_smem_t() { return 1024 + WIDE_T_B + WIDE_NS_T * WIDE_T_STAGE + WIDE_BAR_BYTES; }

template <int FMT> struct WideT;
template <> struct WideT<FMT_F16> {
    using h2 = __half2;
    static __device__ __forceinline__ uint16_t bits(double v) { return __half_as_ushort(__double2half(v)); }
    static __device__ __forceinline__ double val(uint16_t b) { return double(__half2float(__ushort_as_half(b))); }
    static __device__ __forceinline__ h2 pow2(int d) {   // 2^d for d <= 0 (0 below the subnormal range)
        return __float2half2_rn(d < -24 ? 0.0f : ldexpf(1.0f, d));
    }
    static __device__ __forceinline__ uint32_t mul(uint32_t a, h2 f) {
        h2 x = *reinterpret_cast<h2*>(&a);
        x = __hmul2(x, f);
        return *reinterpret_cast<uint32_t*>(&x);
    }
    static constexpr bool bf16 = false;
};
template <> struct WideT<FMT_BF16> {
    using h2 = __nv_bfloat162;
    static __device__ __forceinline__ uint16_t bits(double v) { return __bfloat16_as_ushort(__double2bfloat16(v)); }
    static __device__ __forceinline__ double val(uint16_t b) {
        return double(__bfloat162float(__ushort_as_bfloat16(b)));
    }
    static __device__ __forceinline__ h2 pow2(int d) {
        return __float2bfloat162_rn(d < -126 ? 0.0f : ldexpf(1.0f, d));
    }
    static __device__ __forceinline__ uint32_t mul(uint32_t a, h2 f) {
        h2 x = *reinterpret_cast<h2*>(&a);
        x = __hmul2(x, f);
        return *reinterpret_cast<uint32_t*>(&x);
    }
    static constexpr bool bf16 = true;
};

// the two 16-bit terms of v (already scaled), packed lo-term high
template <int FMT>
__device__ __forceinline__ uint32_t wide_split(double v) {
    using W = WideT<FMT>;
    const uint16_t hi = W::bits(v);
    const uint16_t lo = W::bits(v - W::val(hi));
    return uint32_t(hi) | (uint32_t(lo) << 16);
}

// exponent of the largest |v| (ilogb), or INT_MIN-like sentinel for 0
constexpr int WIDE_NOEXP = -100000;
__device__ __forceinline__ int wide_ilogb(double a) { return a > 0.0 ? ilogb(a) : WIDE_NOEXP; }

// error flag shared by all CTAs of a pass: a bounded wait that ran out
__device__ __forceinline__ bool wide_aborted(const int* err) {
    return (*reinterpret_cast<const volatile int*>(err) & WIDE_ERR_WAIT) != 0;
}
__device__ __forceinline__ bool wide_wait(uint64_t* bar, uint32_t parity, int* err) {
    if (tc5::mbar_try(bar, parity)) return true;
    const uint64_t t0 = tc5::globaltimer();
    for (uint32_t it = 1;; ++it) {
        if (tc5::mbar_try(bar, parity)) return true;
        if ((it & 63u) == 0u) {
            if (wide_aborted(err)) return false;
            if (tc5::globaltimer() - t0 > tc5::WAIT_LIMIT_NS) {
                atomicOr(err, WIDE_ERR_WAIT);
                return false;
            }
        }
    }
}

// ------------------------------------------------------------- x -> xs
// largest |x| of each vector: xmax[r] (as the bits of a non-negative double,
// which order like unsigned integers), zeroed before the launch
__global__ void __launch_bounds__(256)
k_wide_xmax(const double* __restrict__ X, int64_t ldx, int64_t n, int nr, unsigned long long* xmax) {
    const int r = blockIdx.y;
    double m = 0.0;
    for (int64_t i = int64_t(blockIdx.x) * 256 + threadIdx.x; i < n; i += int64_t(gridDim.x) * 256)
        m = fmax(m, fabs(X[i + int64_t(r) * ldx]));
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    __shared__ double red[8];
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < 8; ++w) m = fmax(m, red[w]);
        if (r < nr && m > 0.0) atomicMax(xmax + r, static_cast<unsigned long long>(__double_as_longlong(m)));
    }
}

// g_r = 13 - ilogb(max |x_r|) (0 for a zero vector)
__device__ __forceinline__ int wide_xg(const unsigned long long* xmax, int r) {
    const double m = __longlong_as_double(static_cast<long long>(xmax[r]));
    return m > 0.0 ? 13 - ilogb(m) : 0;
}

// xs[i] = split row of entry i: 64 entries x 64 vectors per block, read
// column by column (coalesced), written row by row through shared memory;
// vectors r >= nr are zero.  Also writes g[] (block 0).
template <int FMT>
__global__ void __launch_bounds__(256)
k_wide_xsplit(const double* __restrict__ X, int64_t ldx, int64_t n, int nr, const unsigned long long* xmax,
              uint32_t* __restrict__ xs, int* __restrict__ g) {
    __shared__ double tile[WIDE_RHS][TILE + 1];
    __shared__ double sc[WIDE_RHS];
    const int64_t i0 = int64_t(blockIdx.x) * TILE;
    if (threadIdx.x < WIDE_RHS) {
        const int gr = threadIdx.x < nr ? wide_xg(xmax, threadIdx.x) : 0;
        sc[threadIdx.x] = ldexp(1.0, gr);
        if (blockIdx.x == 0) g[threadIdx.x] = gr;
    }
    for (int k = threadIdx.x; k < WIDE_RHS * TILE; k += 256) {
        const int r = k / TILE, i = k % TILE;
        tile[r][i] = (r < nr && i0 + i < n) ? X[i0 + i + int64_t(r) * ldx] : 0.0;
    }
    __syncthreads();
    // thread: entry i, vectors 2p, 2p + 1 (p < 32) -> one 8-byte unit of the row
    for (int k = threadIdx.x; k < TILE * 32; k += 256) {
        const int i = k / 32, p = k % 32;
        if (i0 + i >= n) continue;
        const uint32_t a = wide_split<FMT>(tile[2 * p][i] * sc[2 * p]);
        const uint32_t b = wide_split<FMT>(tile[2 * p + 1][i] * sc[2 * p + 1]);
        uint2* o = reinterpret_cast<uint2*>(xs + (i0 + i) * (WIDE_TERMS / 2)) + p;
        *o = make_uint2(a, b);
    }
}

// split row of 64 values (already times 2^g_r) with its own exponent e:
// |v| 2^-e < 2^14; a lane holds vectors 2l, 2l + 1
template <int FMT>
__device__ __forceinline__ void wide_store_row(double v0, double v1, uint32_t* __restrict__ row, int8_t* texp,
                                               int lane) {
    int e = max(wide_ilogb(fabs(v0)), wide_ilogb(fabs(v1)));
    for (int o = 16; o > 0; o >>= 1) e = max(e, __shfl_xor_sync(0xffffffffu, e, o));
    e = e == WIDE_NOEXP ? 0 : min(120, max(-120, e - 13));
    const uint32_t a = wide_split<FMT>(ldexp(v0, -e)), b = wide_split<FMT>(ldexp(v1, -e));
    reinterpret_cast<uint2*>(row)[lane] = make_uint2(a, b);
    if (lane == 0) *texp = int8_t(e);
}

// Partials of multi-tile outputs (FP32, 64 per entry: part[entry * 64 + r]):
// group g sums slots i < nslots of its nc columns, slot i of column j at
// entry slot0 + i * nc + j, in tile order (FP64).  One warp per group, its
// columns one after the other; lane l takes vectors 2l, 2l + 1.  TO_PART:
// the first level of a two-level finish, written as FP32 partials at entry
// g.out + j; otherwise the sums become split rows of ts (entry g.out + j)
// with their exponents.
template <int FMT, bool TO_PART>
__global__ void __launch_bounds__(256)
k_ttfinish_wide(const TGroup* __restrict__ groups, int ngroups, float* part, uint32_t* __restrict__ ts,
                int8_t* __restrict__ texp) {
    const int gid = int(blockIdx.x) * 8 + int(threadIdx.x >> 5);
    if (gid >= ngroups) return;
    const int lane = threadIdx.x & 31;
    const TGroup gr = groups[gid];
    const size_t step = size_t(gr.nc) * 32;
    for (uint32_t j = 0; j < gr.nc; ++j) {
        const float2* p = reinterpret_cast<const float2*>(part) + (size_t(gr.slot0) + j) * 32 + lane;
        double s0[2] = {0.0, 0.0}, s1[2] = {0.0, 0.0};
        uint32_t i = 0;
        for (; i + 2 <= gr.nslots; i += 2) {
            const float2 a = __ldcs(p + size_t(i) * step), b = __ldcs(p + size_t(i + 1) * step);
            s0[0] += a.x; s1[0] += a.y; s0[1] += b.x; s1[1] += b.y;
        }
        if (i < gr.nslots) {
            const float2 a = __ldcs(p + size_t(i) * step);
            s0[0] += a.x; s1[0] += a.y;
        }
        const double v0 = s0[0] + s0[1], v1 = s1[0] + s1[1];
        const size_t e = size_t(gr.out) + j;
        if constexpr (TO_PART) {
            reinterpret_cast<float2*>(part)[e * 32 + lane] = make_float2(float(v0), float(v1));
        } else {
            wide_store_row<FMT>(v0, v1, ts + e * (WIDE_TERMS / 2), texp + e, lane);
        }
    }
}

// ------------------------------------------------------------ tile T-form
// t (x 2^g) of the columns of each tile's run of V: a CTA per run (MSeg),
// 128 columns per block.  Column m of a block at run column c = 128 b + m:
// its 64 values (x 2^g) -> split row of ts (MCol: output entry | MC_DIRECT)
// or FP32 partial entry.
template <int FMT>
__global__ void __launch_bounds__(WIDE_THREADS, 2)
k_ttform_wide(const MSeg* __restrict__ segs, const MCol* __restrict__ cols, const uint8_t* __restrict__ A,
              const uint32_t* __restrict__ xs, uint32_t* __restrict__ ts, int8_t* __restrict__ texp,
              float* __restrict__ part, int* err) {
    using namespace tc5;
    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    uint8_t* sm = smem_raw + (((raw + 1023u) & ~1023u) - raw);
    uint8_t* sB = sm;                                   // the tile's split rows
    uint8_t* sA = sm + WIDE_T_B;                        // stages
    uint64_t* full = reinterpret_cast<uint64_t*>(sA + WIDE_NS_T * WIDE_T_STAGE);
    uint64_t* empty = full + WIDE_NS_T;
    uint64_t* tfull = empty + WIDE_NS_T;                // accumulator buffers ready
    uint64_t* tempty = tfull + 2;                       // accumulator buffers read
    uint64_t* done = tempty + 2;
    uint32_t* tslot = reinterpret_cast<uint32_t*>(done + 1);

    const MSeg sg = segs[blockIdx.x];
    const int ncols = int(sg.ncols);
    const int nblk = (ncols + 127) / 128;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (nblk == 0) return;
    if (threadIdx.x == 0) {
        for (int i = 0; i < WIDE_NS_T; ++i) {
            mbar_init(full + i, WIDE_PRODUCERS);
            mbar_init(empty + i, 1);
        }
        for (int i = 0; i < 2; ++i) {
            mbar_init(tfull + i, 1);
            mbar_init(tempty + i, 128);
        }
        mbar_init(done, 1);
        mbar_init_fence();
    }
    if (warp == 4) tmem_alloc(tslot, 256);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;
    const uint8_t* base = A + size_t(sg.a16) * 16;
    const int colb = int(sg.ld) * 2;
    const MCol* ctab = cols + sg.col0;

    if (warp >= 5) {
        // ---------------------------------------------------- producers
        const int p = threadIdx.x - 160;
        const uint32_t b0 = smem_u32(sB), a0 = smem_u32(sA);
        // the tile's split rows (B operand, 1024 units): row k (tile entry),
        // unit u -> N-atom u / 8 (8 KB apart), K-atom k / 8, row k % 8
        for (int q = p; q < 1024; q += WIDE_PRODUCERS) {
            const int k = q >> 4, u = q & 15;
            const bool ok = k < int(sg.rows);
            const uint32_t dst = b0 + uint32_t(u >> 3) * 8192u + uint32_t(k >> 3) * 1024u + swz(k & 7, u & 7);
            tc5::cp16(dst, ok ? static_cast<const void*>(xs + (size_t(sg.vo) + k) * (WIDE_TERMS / 2) + u * 4)
                         : static_cast<const void*>(xs),
                 ok ? 16u : 0u);
        }
        bool ok = true;
        for (int s = 0; s < nblk && ok; ++s) {
            const int slot = s % WIDE_NS_T;
            if (s >= WIDE_NS_T) ok = wide_wait(empty + slot, uint32_t((s / WIDE_NS_T) - 1) & 1u, err);
            if (!ok) break;
            // 128 columns x 8 units: column m (M index) -> atom m / 8, row m % 8; unit j = rows 8j..8j+7
            const uint32_t sa = a0 + uint32_t(slot) * WIDE_T_STAGE;
            for (int q = p; q < 1024; q += WIDE_PRODUCERS) {
                const int m = q >> 3, j = q & 7;
                const int c = 128 * s + m;
                const bool v = c < ncols && 8 * j < int(sg.ld);
                const uint32_t dst = sa + uint32_t(m >> 3) * 1024u + swz(m & 7, j);
                tc5::cp16(dst, v ? static_cast<const void*>(base + size_t(c) * colb + 16 * j) : static_cast<const void*>(A),
                     v ? 16u : 0u);
            }
            tc5::cp_commit();
            if (s >= WIDE_LAG_T) {
                tc5::cp_wait<WIDE_LAG_T>();
                fence_async_smem();
                mbar_arrive(full + (s - WIDE_LAG_T) % WIDE_NS_T);
            }
        }
        tc5::cp_wait<0>();
        fence_async_smem();
        if (ok)
            for (int s = max(0, nblk - WIDE_LAG_T); s < nblk; ++s) mbar_arrive(full + s % WIDE_NS_T);
    } else if (warp == 4) {
        // ------------------------------------------------------- MMA issue
        if (lane == 0) {
            constexpr uint32_t ID = tc5::idesc_f16(128, 128, WideT<FMT>::bf16, false, true);
            const uint32_t a0 = smem_u32(sA), b0 = smem_u32(sB);
            bool ok = true;
            for (int s = 0; s < nblk; ++s) {
                const int slot = s % WIDE_NS_T, buf = s & 1;
                ok = wide_wait(full + slot, uint32_t(s / WIDE_NS_T) & 1u, err);
                if (ok && s >= 2) ok = wide_wait(tempty + buf, uint32_t((s >> 1) - 1) & 1u, err);
                if (!ok) break;
                tc_fence_after();
                const uint32_t d = tmem + uint32_t(buf) * 128u;
                const uint32_t sa = a0 + uint32_t(slot) * WIDE_T_STAGE;
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    mma_f16(d, sdesc(sa + 32u * j, 16u, 1024u), sdesc(b0 + 2048u * j, 8192u, 1024u), ID, j > 0);
                mma_commit(empty + slot);
                mma_commit(tfull + buf);
            }
            // every MMA issued has completed before TMEM is freed (this wait
            // does not give up on the error flag: MMAs always finish)
            mma_commit(done);
            if (!mbar_wait(done, 0u)) atomicOr(err, WIDE_ERR_WAIT);
        }
        __syncwarp();
    } else {
        // -------------------------------------------------------- epilogue
        const uint32_t lanebase = tmem + (uint32_t(32 * warp) << 16);
        for (int s = 0; s < nblk; ++s) {
            const int buf = s & 1;
            // warp-uniform: the TMEM loads below are collective
            if (!__all_sync(0xffffffffu, wide_wait(tfull + buf, uint32_t(s >> 1) & 1u, err))) break;
            tc_fence_after();
            const int m = 32 * warp + lane, c = 128 * s + m;
            const bool have = c < ncols;
            const MCol mc = have ? ctab[c] : MCol{0u, 0.f};
            const uint32_t ta = lanebase + uint32_t(buf) * 128u;
            const double sc = double(mc.scale);
            const bool direct = (mc.idx & MC_DIRECT) != 0;
            // TMEM loads are collective: every lane runs both passes, and
            // only the stores depend on the lane's column.  Pass 1: the
            // column's largest value (the exponent of its split row); pass
            // 2: the split terms (direct outputs) or the FP32 partials.
            int ex = WIDE_NOEXP;
#pragma unroll 1
            for (int h = 0; h < 4; ++h) {
                float f[32];
                tc5::tmem_ld32(ta + uint32_t(32 * h), f);
#pragma unroll
                for (int i = 0; i < 16; ++i)
                    ex = max(ex, wide_ilogb(fabs((double(f[2 * i]) + double(f[2 * i + 1])) * sc)));
            }
            ex = ex == WIDE_NOEXP ? 0 : min(120, max(-120, ex - 13));
            uint4* row = reinterpret_cast<uint4*>(ts + size_t(mc.idx & ~MC_DIRECT) * (WIDE_TERMS / 2));
            float4* o = reinterpret_cast<float4*>(part + size_t(mc.idx & ~MC_DIRECT) * WIDE_RHS);
#pragma unroll 1
            for (int h = 0; h < 4; ++h) {
                float f[32];
                tc5::tmem_ld32(ta + uint32_t(32 * h), f);
                if (!have) continue;
                if (direct) {
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        uint32_t w[4];
#pragma unroll
                        for (int i = 0; i < 4; ++i) {
                            const int k = 4 * q + i;
                            w[i] = wide_split<FMT>(ldexp((double(f[2 * k]) + double(f[2 * k + 1])) * sc, -ex));
                        }
                        row[4 * h + q] = make_uint4(w[0], w[1], w[2], w[3]);
                    }
                } else {
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        float w[4];
#pragma unroll
                        for (int i = 0; i < 4; ++i) {
                            const int k = 4 * q + i;
                            w[i] = float((double(f[2 * k]) + double(f[2 * k + 1])) * sc);
                        }
                        o[4 * h + q] = make_float4(w[0], w[1], w[2], w[3]);
                    }
                }
            }
            if (have && direct) texp[mc.idx & ~MC_DIRECT] = int8_t(ex);
            tc_fence_before();
            mbar_arrive(tempty + buf);
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 4) {
        tc_fence_after();
        tmem_dealloc(tmem, 256);
    }
}

// ----------------------------------------------------------------- N-form
// y (+)= alpha op(M) X for the WIDE_RHS vectors: a CTA per output tile's run
// (MSeg), 32 columns per stage.  om maps (row, vector) to y.
template <int FMT>
__global__ void __launch_bounds__(WIDE_THREADS, 2)
k_nform_wide(const MSeg* __restrict__ segs, const MCol* __restrict__ cols, const uint8_t* __restrict__ A,
             const uint32_t* __restrict__ xs, const uint32_t* __restrict__ ts, const int8_t* __restrict__ texp,
             const int* __restrict__ g, OutMap om, double alpha, int add, int* err) {
    using namespace tc5;
    using W = WideT<FMT>;
    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    uint8_t* sm = smem_raw + (((raw + 1023u) & ~1023u) - raw);
    double* acc = reinterpret_cast<double*>(sm + WIDE_NS_N * WIDE_N_STAGE);   // [r][row], ld WIDE_ACC_LD
    uint64_t* full = reinterpret_cast<uint64_t*>(sm + WIDE_NS_N * WIDE_N_STAGE + WIDE_ACC_BYTES);
    uint64_t* empty = full + WIDE_NS_N;
    uint64_t* tfull = empty + WIDE_NS_N;                // accumulator buffers ready
    uint64_t* tempty = tfull + 2;                       // accumulator buffers drained
    uint64_t* done = tempty + 2;
    uint32_t* tslot = reinterpret_cast<uint32_t*>(done + 1);
    int* sref = reinterpret_cast<int*>(tslot + 1);      // largest column exponent of the run
    int* wred = sref + 1;                               // per-warp maxima (7)

    const MSeg sg = segs[blockIdx.x];
    const int ncols = int(sg.ncols);
    const int nst = (ncols + 31) / 32;
    const int ngrp = (nst + WIDE_FLUSH - 1) / WIDE_FLUSH;   // FP32 accumulations
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (nst == 0) return;
    const MCol* ctab = cols + sg.col0;
    // exponent of column c's factor: its chunk scale times 2^e of its split row
    auto col_exp = [&](const MCol& m) {
        const int es = ilogbf(m.scale);
        return (m.idx & VEC_T) ? es + int(texp[m.idx & ~VEC_T]) : es;
    };
    int emax = WIDE_NOEXP;
    for (int c = threadIdx.x; c < ncols; c += WIDE_THREADS) emax = max(emax, col_exp(ctab[c]));
    for (int o = 16; o > 0; o >>= 1) emax = max(emax, __shfl_xor_sync(0xffffffffu, emax, o));
    if (lane == 0) wred[warp] = emax;
    for (int i = threadIdx.x; i < WIDE_RHS * WIDE_ACC_LD; i += WIDE_THREADS) acc[i] = 0.0;
    if (threadIdx.x == 0) {
        for (int i = 0; i < WIDE_NS_N; ++i) {
            mbar_init(full + i, WIDE_PRODUCERS);
            mbar_init(empty + i, 1);
        }
        for (int i = 0; i < 2; ++i) {
            mbar_init(tfull + i, 1);
            mbar_init(tempty + i, 128);
        }
        mbar_init(done, 1);
        mbar_init_fence();
    }
    if (warp == 4) tmem_alloc(tslot, 128);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (threadIdx.x == 0) {
        int m = wred[0];
        for (int w = 1; w < WIDE_THREADS / 32; ++w) m = max(m, wred[w]);
        *sref = m;
    }
    __syncthreads();
    const int E = *sref;
    const uint32_t tmem = *tslot;

    if (warp >= 5) {
        // ---------------------------------------------------- producers
        // thread p stages column p / 2 of every stage: half p % 2 of its
        // split row (8 units, M-atom p % 2) and units 4 (p % 2) .. +3 of the
        // matrix column
        const int p = threadIdx.x - 160, k = p >> 1, half = p & 1;
        const uint8_t* base = A + size_t(sg.a16) * 16;
        const int colb = int(sg.ld) * 2;
        const uint32_t s0 = smem_u32(sm);
        typename W::h2 fac[WIDE_LAG_N + 1];
        bool ok = true;
        for (int s = 0; s < nst && ok; ++s) {
            const int slot = s % WIDE_NS_N;
            if (s >= WIDE_NS_N) ok = wide_wait(empty + slot, uint32_t((s / WIDE_NS_N) - 1) & 1u, err);
            if (!ok) break;
            const int c = 32 * s + k;
            const bool have = c < ncols;
            const MCol mc = have ? ctab[c] : MCol{0u, 1.f};
            fac[s % (WIDE_LAG_N + 1)] = W::pow2(have ? col_exp(mc) - E : 0);
            const uint32_t* vrow = (mc.idx & VEC_T) ? ts + size_t(mc.idx & ~VEC_T) * (WIDE_TERMS / 2)
                                                    : xs + size_t(mc.idx) * (WIDE_TERMS / 2);
            const uint32_t sa = s0 + uint32_t(slot) * WIDE_N_STAGE, sb = sa + 8192u;
            // vector terms: unit u of the row -> M-atom u / 8 (4 KB apart), K-atom k / 8, row k % 8
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                const int u = 8 * half + i;
                tc5::cp16(sa + uint32_t(half) * 4096u + uint32_t(k >> 3) * 1024u + swz(k & 7, i),
                          have ? static_cast<const void*>(vrow + 4 * u) : static_cast<const void*>(xs), have ? 16u : 0u);
            }
            // matrix column: unit j (rows 8j .. 8j+7) -> K-atom k / 8, row k % 8
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int j = 4 * half + i;
                const bool v = have && 8 * j < int(sg.ld);
                tc5::cp16(sb + uint32_t(k >> 3) * 1024u + swz(k & 7, j),
                          v ? static_cast<const void*>(base + size_t(c) * colb + 16 * j) : static_cast<const void*>(A),
                          v ? 16u : 0u);
            }
            tc5::cp_commit();
            auto finish = [&](int sd) {   // stage sd has landed: scale its matrix column, hand it over
                const typename W::h2 f = fac[sd % (WIDE_LAG_N + 1)];
                uint8_t* col = sm + (sd % WIDE_NS_N) * WIDE_N_STAGE + 8192 + (k >> 3) * 1024;
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    uint4* q = reinterpret_cast<uint4*>(col + swz(k & 7, 4 * half + i));
                    uint4 w = *q;
                    w.x = W::mul(w.x, f); w.y = W::mul(w.y, f); w.z = W::mul(w.z, f); w.w = W::mul(w.w, f);
                    *q = w;
                }
                fence_async_smem();
                mbar_arrive(full + sd % WIDE_NS_N);
            };
            if (s >= WIDE_LAG_N) {
                tc5::cp_wait<WIDE_LAG_N>();
                finish(s - WIDE_LAG_N);
            }
            if (s == nst - 1) {
                tc5::cp_wait<0>();
                for (int sd = max(0, nst - WIDE_LAG_N); sd < nst; ++sd) finish(sd);
            }
        }
        tc5::cp_wait<0>();
    } else if (warp == 4) {
        // ------------------------------------------------------- MMA issue
        // group q (stages WIDE_FLUSH q ..) accumulates into buffer q % 2
        if (lane == 0) {
            constexpr uint32_t ID = tc5::idesc_f16(128, 64, WideT<FMT>::bf16, true, true);
            const uint32_t s0 = smem_u32(sm);
            bool ok = true;
            for (int s = 0; s < nst && ok; ++s) {
                const int slot = s % WIDE_NS_N, q = s / WIDE_FLUSH, buf = q & 1;
                const bool first = s % WIDE_FLUSH == 0, last = s % WIDE_FLUSH == WIDE_FLUSH - 1 || s == nst - 1;
                if (first && q >= 2) ok = wide_wait(tempty + buf, uint32_t((q >> 1) - 1) & 1u, err);
                if (ok) ok = wide_wait(full + slot, uint32_t(s / WIDE_NS_N) & 1u, err);
                if (!ok) break;
                tc_fence_after();
                const uint32_t sa = s0 + uint32_t(slot) * WIDE_N_STAGE, sb = sa + 8192u;
                const uint32_t d = tmem + uint32_t(buf) * 64u;
#pragma unroll
                for (int j = 0; j < 2; ++j)
                    mma_f16(d, sdesc(sa + 2048u * j, 4096u, 1024u), sdesc(sb + 2048u * j, 4096u, 1024u), ID,
                            (!first || j > 0) ? 1u : 0u);
                mma_commit(empty + slot);
                if (last) mma_commit(tfull + buf);
            }
            // every MMA issued has completed before TMEM is freed (this wait
            // does not give up on the error flag: MMAs always finish)
            mma_commit(done);
            if (!mbar_wait(done, 0u)) atomicOr(err, WIDE_ERR_WAIT);
        }
        __syncwarp();
    } else {
        // -------------------------------------------------------- epilogue
        // lane m = term m: vector m / 2, hi (even) or lo (odd); the even lane
        // adds hi + lo of its vector's 64 rows to the FP64 accumulator
        const uint32_t la = tmem + (uint32_t(32 * warp) << 16);
        const int m = 32 * warp + lane;
        double* arow = acc + (m >> 1) * WIDE_ACC_LD;
        bool ok = true;
        for (int q = 0; q < ngrp; ++q) {
            const int buf = q & 1;
            ok = __all_sync(0xffffffffu, wide_wait(tfull + buf, uint32_t(q >> 1) & 1u, err));
            if (!ok) break;
            tc_fence_after();
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                float f[32];
                tmem_ld32(la + uint32_t(buf) * 64u + uint32_t(32 * h), f);
#pragma unroll
                for (int i = 0; i < 32; ++i) {
                    const float o = __shfl_xor_sync(0xffffffffu, f[i], 1);
                    if ((lane & 1) == 0) arow[32 * h + i] += double(f[i]) + double(o);
                }
            }
            tc_fence_before();
            mbar_arrive(tempty + buf);
        }
        asm volatile("bar.sync 1, 128;\n" ::: "memory");
        ok = __all_sync(0xffffffffu, ok) && !wide_aborted(err);
        if (ok) {
            for (int q = threadIdx.x; q < WIDE_RHS * TILE; q += 128) {
                const int r = q / TILE, row = q % TILE;
                if (r >= om.nr || row >= int(sg.rows)) continue;
                const double val = ldexp(acc[r * WIDE_ACC_LD + row], E - g[r]);
                double* o = om.base + int64_t(sg.vo + row) * om.rs + int64_t(r) * om.cs;
                if (add) *o += alpha * val;
                else *o = val;
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 4) {
        tc_fence_after();
        tmem_dealloc(tmem, 128);
    }
}

}  // namespace hlrc
