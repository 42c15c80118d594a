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
//   t = V^T x (per low-rank column i, times 2^g_r): split rows with a static
//      exponent c_i (2^c_i > ||V(:,i)||_1, so |t_i| 2^g_r 2^-c_i < 2^14),
//      into ts; c_i comes from the planner (WidePlan::t_exp).
//
// Kernels (op N):
//   k_wide_xmax / k_wide_xsplit   x -> xs (and g_r)
//   k_ctform_wide   one CTA per unit of the column-cluster T-form: the V
//                   slabs of blocks sharing a column cluster, stacked as the
//                   N operand (<= 128 columns, K-major), times the split rows
//                   of one column tile as the M operand (128 terms,
//                   MN-major), accumulated over all the unit's tiles in TMEM;
//                   t rows go straight to ts (or, for a piece of a long
//                   cluster, to FP32 partials)
//   k_ttfinish_wide   partials of the pieces summed in piece order (FP64),
//                   then split into ts
//   k_nform_wide    one CTA per output tile: y += U t + D x over the tile's
//                   run of columns; A = 128 terms of 32 columns (MN-major,
//                   gathered split rows), B = the 32 matrix columns
//                   (MN-major), D = 128 terms x 64 rows in TMEM
//
// Scales in the N-form.  Column c of the run has the factor f_c = its chunk
// scale (x columns) or its chunk scale times 2^c_i (t columns); with F = 2^E
// the largest f over the run, the staged matrix column is multiplied by
// f_c / F (a power of two <= 1: exact unless the values drop below the
// 16-bit range, where they are negligible against the run's largest terms),
// so that one accumulator serves the whole run:
// y_r += alpha F 2^-g_r (acc_hi + acc_lo).  All factors are fixed at upload
// (WCol, E per run).  The tensor cores accumulate in FP32 over WIDE_FLUSH
// stages (64 columns) into one of two TMEM buffers; the epilogue warps add
// each finished buffer to an FP64 accumulator in shared memory while the
// MMAs fill the other, so long runs keep FP64 sums.
//
// Roles (224 threads): warps 0-3 read the accumulators (warp w reads TMEM
// lanes 32w .. 32w + 31), warp 4 allocates TMEM and issues the MMAs (one
// thread), warps 5-6 stage operands with cp.async copies into the
// 128-byte-swizzled layouts, zero-filling everything outside the data.
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
constexpr int WIDE_NS_C = 3;          // column-cluster T-form stages (one tile each): 2 CTAs per SM
constexpr int WIDE_LAG_N = WIDE_NS_N - 2;   // copy groups a producer keeps in flight
constexpr int WIDE_LAG_C = WIDE_NS_C - 1;
constexpr int WIDE_PF = WIDE_LAG_N + 1;     // N-form: column-table entries prefetched this many stages ahead
constexpr int WIDE_WQ = WIDE_PF + WIDE_LAG_N + 1;   // ring of prefetched column-table entries
constexpr int WIDE_ERR_WAIT = 2;      // device error word bit: a wait of a wide kernel ran out
constexpr uint32_t WT_EMPTY = 0xffffffffu;   // stacked column without data

// N-form stage: A (vector terms, 2 M-atoms x 4 K-atoms) 8 KB, B (matrix, 4 K-atoms) 4 KB
constexpr int WIDE_N_STAGE = 12288;
// N-form FP64 accumulator in shared memory: [vector][row], rows padded to 65
// (the 16 lanes that add one row of 16 vectors hit 16 different bank pairs)
constexpr int WIDE_ACC_LD = TILE + 1;
constexpr int WIDE_ACC_BYTES = WIDE_RHS * WIDE_ACC_LD * 8;
constexpr int WIDE_WQ_BYTES = WIDE_WQ * WIDE_PRODUCERS * 8;
// column-cluster T-form stage: A (split rows of a tile: 2 M-atoms x 8 K-atoms)
// 16 KB, B (<= 128 stacked V columns: 16 atoms) 16 KB
constexpr int WIDE_C_STAGE = 32768;
constexpr int WIDE_C_TABLES = WT_MAXB * 16 + WT_MAXN * 4 + WT_MAXT * WT_MAXB * 4;
constexpr int WIDE_BAR_BYTES = 256;   // mbarriers and the TMEM address
constexpr int wide_smem_n() {
    return 1024 + WIDE_NS_N * WIDE_N_STAGE + WIDE_ACC_BYTES + WIDE_WQ_BYTES + WIDE_BAR_BYTES;
}
constexpr int wide_smem_c() { return 1024 + WIDE_NS_C * WIDE_C_STAGE + WIDE_C_TABLES + WIDE_BAR_BYTES; }
static_assert(WIDE_NS_C * WIDE_C_STAGE >= WT_MAXN * WIDE_TERMS * 4, "T-form epilogue transpose fits the stages");

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

// the same from an FP32 value (FP32 keeps 24 bits, the split 22 or 16)
template <int FMT>
__device__ __forceinline__ uint32_t wide_split_f(float v) {
    if constexpr (FMT == FMT_F16) {
        const __half hi = __float2half_rn(v);
        const __half lo = __float2half_rn(v - __half2float(hi));
        return uint32_t(__half_as_ushort(hi)) | (uint32_t(__half_as_ushort(lo)) << 16);
    } else {
        const __nv_bfloat16 hi = __float2bfloat16_rn(v);
        const __nv_bfloat16 lo = __float2bfloat16_rn(v - __bfloat162float(hi));
        return uint32_t(__bfloat16_as_ushort(hi)) | (uint32_t(__bfloat16_as_ushort(lo)) << 16);
    }
}

// exponent of the largest |v| (ilogb), or INT_MIN-like sentinel for 0
constexpr int WIDE_NOEXP = -100000;
__device__ __forceinline__ int wide_ilogb(double a) { return a > 0.0 ? ilogb(a) : WIDE_NOEXP; }

// Wait bound of the kernels that hand work over with mbarriers, and the
// test hook of hlrc_debug_waits: skip != 0 leaves the first hand-over of
// every CTA undone (its producers never signal stage 0), so that the
// consumer's wait runs out, as a wait on a flag that nothing sets.
struct WaitCfg {
    uint64_t limit_ns;
    int skip;
};

// error flag shared by all CTAs of a pass: a bounded wait that ran out
__device__ __forceinline__ bool wide_aborted(const int* err) {
    return (*reinterpret_cast<const volatile int*>(err) & WIDE_ERR_WAIT) != 0;
}
__device__ __forceinline__ bool wide_wait(uint64_t* bar, uint32_t parity, int* err, uint64_t limit_ns) {
    if (tc5::mbar_try(bar, parity)) return true;
    const uint64_t t0 = tc5::globaltimer();
    for (uint32_t it = 1;; ++it) {
        if (tc5::mbar_try(bar, parity)) return true;
        if ((it & 63u) == 0u) {
            if (wide_aborted(err)) return false;
            if (tc5::globaltimer() - t0 > limit_ns) {
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

// split row of 64 values (times 2^g_r) with the static exponent e of its t
// entry; a lane holds vectors 2l, 2l + 1
template <int FMT>
__device__ __forceinline__ void wide_store_row(double v0, double v1, int e, uint32_t* __restrict__ row, int lane) {
    reinterpret_cast<uint2*>(row)[lane] = make_uint2(wide_split<FMT>(ldexp(v0, -e)), wide_split<FMT>(ldexp(v1, -e)));
}

// Partials of the pieces of long column clusters (FP32, 64 per entry:
// part[entry * 64 + r]): group g sums pieces i < nslots of its nc columns,
// piece i of column j at entry slot0 + i * nc + j, in piece order (FP64),
// into the split rows of ts (entry g.out + j).  One warp per group, its
// columns one after the other; lane l takes vectors 2l, 2l + 1.
template <int FMT>
__global__ void __launch_bounds__(256)
k_ttfinish_wide(const TGroup* __restrict__ groups, int ngroups, const float* __restrict__ part,
                uint32_t* __restrict__ ts, const int8_t* __restrict__ texp) {
    const int gid = int(blockIdx.x) * 8 + int(threadIdx.x >> 5);
    if (gid >= ngroups) return;
    const int lane = threadIdx.x & 31;
    const TGroup gr = groups[gid];
    const size_t step = size_t(gr.nc) * 32;
    for (uint32_t j = 0; j < gr.nc; ++j) {
        const float2* p = reinterpret_cast<const float2*>(part) + (size_t(gr.slot0) + j) * 32 + lane;
        double s0[2] = {0.0, 0.0}, s1[2] = {0.0, 0.0};
        uint32_t i = 0;
        // eight loads in flight, then the same sums in the same order
        for (; i + 8 <= gr.nslots; i += 8) {
            float2 v[8];
#pragma unroll
            for (int a = 0; a < 8; ++a) v[a] = __ldcs(p + size_t(i + a) * step);
#pragma unroll
            for (int a = 0; a < 8; ++a) {
                s0[a & 1] += v[a].x;
                s1[a & 1] += v[a].y;
            }
        }
        for (; i + 2 <= gr.nslots; i += 2) {
            const float2 a = __ldcs(p + size_t(i) * step), b = __ldcs(p + size_t(i + 1) * step);
            s0[0] += a.x; s1[0] += a.y; s0[1] += b.x; s1[1] += b.y;
        }
        if (i < gr.nslots) {
            const float2 a = __ldcs(p + size_t(i) * step);
            s0[0] += a.x; s1[0] += a.y;
        }
        const size_t e = size_t(gr.out) + j;
        wide_store_row<FMT>(s0[0] + s0[1], s1[0] + s1[1], int(texp[e]), ts + e * (WIDE_TERMS / 2), lane);
    }
}

// ------------------------------------------------------ column-cluster T-form
// One CTA per unit (WTUnit): for each of its tiles, A = the tile's split rows
// of x (M = 128 terms, K = 64 tile rows, MN-major) and B = the V slabs of the
// unit's blocks in that tile (N = the stacked columns, K-major); D (128 terms
// x N) accumulates over all tiles.  The epilogue transposes D through shared
// memory and writes one split row (or FP32 partial) per column.
template <int FMT>
__global__ void __launch_bounds__(WIDE_THREADS, 2)
k_ctform_wide(const WTUnit* __restrict__ units, const WTBlk* __restrict__ blks, const uint32_t* __restrict__ slabs,
              const WTTile* __restrict__ tiles, const uint8_t* __restrict__ A, const uint32_t* __restrict__ xs,
              uint32_t* __restrict__ ts, const int8_t* __restrict__ texp, float* __restrict__ part, int* err,
              WaitCfg wc) {
    using namespace tc5;
    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    uint8_t* sm = smem_raw + (((raw + 1023u) & ~1023u) - raw);
    WTBlk* sblk = reinterpret_cast<WTBlk*>(sm + WIDE_NS_C * WIDE_C_STAGE);
    uint32_t* scol = reinterpret_cast<uint32_t*>(sblk + WT_MAXB);           // stacked column -> (block << 16) | column
    uint32_t* sslab = scol + WT_MAXN;                                       // [tile][block] store offsets / 16
    uint64_t* full = reinterpret_cast<uint64_t*>(sslab + WT_MAXT * WT_MAXB);
    uint64_t* empty = full + WIDE_NS_C;
    uint64_t* accf = empty + WIDE_NS_C;
    uint32_t* tslot = reinterpret_cast<uint32_t*>(accf + 1);

    const WTUnit u = units[blockIdx.x];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nt = u.ntiles, nb = u.nblk, nc = u.ncols, npad = (nc + 15) & ~15;
    if (nt == 0 || nc == 0) return;
    for (int j = threadIdx.x; j < nb; j += WIDE_THREADS) sblk[j] = blks[u.blk0 + j];
    for (int i = threadIdx.x; i < nt * nb; i += WIDE_THREADS) sslab[i] = slabs[u.slab0 + i];
    if (threadIdx.x == 0) {
        for (int i = 0; i < WIDE_NS_C; ++i) {
            mbar_init(full + i, WIDE_PRODUCERS);
            mbar_init(empty + i, 1);
        }
        mbar_init(accf, 1);
        mbar_init_fence();
    }
    if (warp == 4) tmem_alloc(tslot, 128);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    // stacked column -> (block, column); columns between a block's rank and
    // its 8-column boundary stay empty (zero-filled, not written out)
    for (int n = threadIdx.x; n < WT_MAXN; n += WIDE_THREADS) scol[n] = WT_EMPTY;
    __syncthreads();
    for (int j = threadIdx.x; j < nb; j += WIDE_THREADS)
        for (int l = 0; l < sblk[j].k; ++l) scol[sblk[j].off + l] = (uint32_t(j) << 16) | uint32_t(l);
    __syncthreads();
    const uint32_t tmem = *tslot;

    if (warp >= 5) {
        // ---------------------------------------------------- producers
        const int p = threadIdx.x - 160;
        const uint32_t s0 = smem_u32(sm);
        bool ok = true;
        for (int q = 0; q < nt && ok; ++q) {
            const int slot = q % WIDE_NS_C;
            if (q >= WIDE_NS_C) ok = wide_wait(empty + slot, uint32_t((q / WIDE_NS_C) - 1) & 1u, err, wc.limit_ns);
            if (!ok) break;
            const WTTile tl = tiles[u.tile0 + q];
            const uint32_t sa = s0 + uint32_t(slot) * WIDE_C_STAGE, sb = sa + 16384u;
            // A: split row k (tile entry), unit v -> M-atom v / 8 (8 KB apart), K-atom k / 8, row k % 8
            for (int i = p; i < 1024; i += WIDE_PRODUCERS) {
                const int k = i >> 4, v = i & 15;
                const bool in = k < int(tl.rows);
                tc5::cp16(sa + uint32_t(v >> 3) * 8192u + uint32_t(k >> 3) * 1024u + swz(k & 7, v & 7),
                          in ? static_cast<const void*>(xs + (size_t(tl.v_off) + k) * (WIDE_TERMS / 2) + v * 4)
                             : static_cast<const void*>(xs),
                          in ? 16u : 0u);
            }
            // B: stacked column n, unit jj (tile rows 8jj .. 8jj+7) -> atom n / 8, row n % 8
            for (int i = p; i < npad * 8; i += WIDE_PRODUCERS) {
                const int n = i >> 3, jj = i & 7;
                const uint32_t cm = n < nc ? scol[n] : WT_EMPTY;
                const bool in = cm != WT_EMPTY && 8 * jj < int(tl.ld);
                const uint8_t* src = A;
                if (in)
                    src = A + size_t(sslab[q * nb + int(cm >> 16)]) * 16 + size_t(cm & 0xffffu) * tl.ld * 2 + 16 * jj;
                tc5::cp16(sb + uint32_t(n >> 3) * 1024u + swz(n & 7, jj), src, in ? 16u : 0u);
            }
            tc5::cp_commit();
            if (q >= WIDE_LAG_C) {
                tc5::cp_wait<WIDE_LAG_C>();
                fence_async_smem();
                if (!(wc.skip && q == WIDE_LAG_C)) mbar_arrive(full + (q - WIDE_LAG_C) % WIDE_NS_C);
            }
        }
        tc5::cp_wait<0>();
        fence_async_smem();
        if (ok)
            for (int q = max(0, nt - WIDE_LAG_C); q < nt; ++q)
                if (!(wc.skip && q == 0)) mbar_arrive(full + q % WIDE_NS_C);
    } else if (warp == 4) {
        // ------------------------------------------------------- MMA issue
        if (lane == 0) {
            const uint32_t id = tc5::idesc_f16(128, npad, WideT<FMT>::bf16, true, false);
            const uint32_t s0 = smem_u32(sm);
            for (int q = 0; q < nt; ++q) {
                const int slot = q % WIDE_NS_C;
                if (!wide_wait(full + slot, uint32_t(q / WIDE_NS_C) & 1u, err, wc.limit_ns)) break;
                tc_fence_after();
                const uint32_t sa = s0 + uint32_t(slot) * WIDE_C_STAGE, sb = sa + 16384u;
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    mma_f16(tmem, sdesc(sa + 2048u * j, 8192u, 1024u), sdesc(sb + 32u * j, 16u, 1024u), id,
                            (q > 0 || j > 0) ? 1u : 0u);
                mma_commit(empty + slot);
            }
            // every MMA issued has completed before the epilogue reads TMEM
            // and before TMEM is freed (this wait does not give up on the
            // error flag: MMAs always finish)
            mma_commit(accf);
            if (!mbar_wait(accf, 0u, wc.limit_ns)) atomicOr(err, WIDE_ERR_WAIT);
        }
        __syncwarp();
    } else {
        // -------------------------------------------------------- epilogue
        bool ok = __all_sync(0xffffffffu, wide_wait(accf, 0u, err, wc.limit_ns) && !wide_aborted(err));
        tc_fence_after();
        // every stage has been consumed: the stage memory holds the
        // transpose red[n][m] (FP32, 128 terms per stacked column)
        float* red = reinterpret_cast<float*>(sm);
        if (ok) {
            const uint32_t la = tmem + (uint32_t(32 * warp) << 16);
            const int m = 32 * warp + lane;
            for (int c = 0; c < npad; c += 32) {
                float f[32];
                tmem_ld32(la + uint32_t(c), f);
#pragma unroll
                for (int i = 0; i < 32; ++i)
                    if (c + i < nc) red[(c + i) * WIDE_TERMS + m] = f[i];
            }
        }
        tc_fence_before();
        asm volatile("bar.sync 1, 128;\n" ::: "memory");
        if (__all_sync(0xffffffffu, ok)) {
            for (int n = warp; n < nc; n += 4) {
                const uint32_t cm = scol[n];
                if (cm == WT_EMPTY) continue;
                const WTBlk& b = sblk[cm >> 16];
                const int l = int(cm & 0xffffu);
                const float4 t4 = reinterpret_cast<const float4*>(red + n * WIDE_TERMS)[lane];
                const double sc = double(b.scale);
                const double v0 = (double(t4.x) + double(t4.y)) * sc, v1 = (double(t4.z) + double(t4.w)) * sc;
                if (u.npieces == 1) {
                    const size_t e = size_t(b.toff) + size_t(l);
                    wide_store_row<FMT>(v0, v1, int(texp[e]), ts + e * (WIDE_TERMS / 2), lane);
                } else {
                    const size_t e = size_t(b.pbase) + size_t(u.piece) * b.k + size_t(l);
                    reinterpret_cast<float2*>(part)[e * 32 + lane] = make_float2(float(v0), float(v1));
                }
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

// ----------------------------------------------------------------- N-form
// y (+)= alpha op(M) X for the WIDE_RHS vectors: a CTA per output tile's run
// (MSeg; E = the run's factor exponent in MSeg.pad), 32 columns per stage;
// wcol[col0 + c]: the vector entry and factor of run column c.  om maps
// (row, vector) to y.
template <int FMT>
__global__ void __launch_bounds__(WIDE_THREADS, 2)
k_nform_wide(const MSeg* __restrict__ segs, const WCol* __restrict__ wcol, const uint8_t* __restrict__ A,
             const uint32_t* __restrict__ xs, const uint32_t* __restrict__ ts, const int* __restrict__ g, OutMap om,
             double alpha, int add, int* err, WaitCfg wc) {
    using namespace tc5;
    using W = WideT<FMT>;
    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    uint8_t* sm = smem_raw + (((raw + 1023u) & ~1023u) - raw);
    double* acc = reinterpret_cast<double*>(sm + WIDE_NS_N * WIDE_N_STAGE);   // [r][row], ld WIDE_ACC_LD
    uint2* wq = reinterpret_cast<uint2*>(sm + WIDE_NS_N * WIDE_N_STAGE + WIDE_ACC_BYTES);   // [slot][producer]
    uint64_t* full = reinterpret_cast<uint64_t*>(sm + WIDE_NS_N * WIDE_N_STAGE + WIDE_ACC_BYTES + WIDE_WQ_BYTES);
    uint64_t* empty = full + WIDE_NS_N;
    uint64_t* tfull = empty + WIDE_NS_N;                // accumulator buffers ready
    uint64_t* tempty = tfull + 2;                       // accumulator buffers drained
    uint64_t* done = tempty + 2;
    uint32_t* tslot = reinterpret_cast<uint32_t*>(done + 1);

    const MSeg sg = segs[blockIdx.x];
    const int ncols = int(sg.ncols);
    const int nst = (ncols + 31) / 32;
    const int ngrp = (nst + WIDE_FLUSH - 1) / WIDE_FLUSH;   // FP32 accumulations
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (nst == 0) return;
    const int E = int(sg.pad);
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
    const uint32_t tmem = *tslot;

    if (warp >= 5) {
        // ---------------------------------------------------- producers
        // thread p stages column k = p / 2 of every stage: half p % 2 of its
        // split row (8 units, M-atom p % 2) and units 4 (p % 2) .. +3 of the
        // matrix column.  Its column-table entries arrive WIDE_PF stages
        // ahead in the shared ring wq (cp.async, so no load stalls the
        // loop); an entry stays there until its stage has been handed over.
        const int p = threadIdx.x - 160, k = p >> 1, half = p & 1;
        const uint8_t* base = A + size_t(sg.a16) * 16;
        const int colb = int(sg.ld) * 2;
        const uint32_t s0 = smem_u32(sm);
        const WCol* wtab = wcol + sg.col0;
        auto prefetch = [&](int st) {   // column-table entry of stage st into its ring slot
            const int c = 32 * st + k;
            const bool in = c < ncols;
            asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(
                             smem_u32(wq + (st % WIDE_WQ) * WIDE_PRODUCERS + p)),
                         "l"(in ? static_cast<const void*>(wtab + c) : static_cast<const void*>(wcol)), "r"(in ? 8u : 0u)
                         : "memory");
        };
        for (int st = 0; st < WIDE_PF && st < nst; ++st) prefetch(st);
        tc5::cp_commit();
        tc5::cp_wait<0>();
        auto finish = [&](int sd) {   // stage sd has landed: scale its matrix column, hand it over
            const uint32_t fb = wq[(sd % WIDE_WQ) * WIDE_PRODUCERS + p].y;
            const typename W::h2 f = *reinterpret_cast<const typename W::h2*>(&fb);
            uint8_t* col = sm + (sd % WIDE_NS_N) * WIDE_N_STAGE + 8192 + (k >> 3) * 1024;
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                uint4* q = reinterpret_cast<uint4*>(col + swz(k & 7, 4 * half + i));
                uint4 w = *q;
                w.x = W::mul(w.x, f); w.y = W::mul(w.y, f); w.z = W::mul(w.z, f); w.w = W::mul(w.w, f);
                *q = w;
            }
            fence_async_smem();
            if (!(wc.skip && sd == 0)) mbar_arrive(full + sd % WIDE_NS_N);
        };
        bool ok = true;
        for (int s = 0; s < nst && ok; ++s) {
            const int slot = s % WIDE_NS_N;
            if (s >= WIDE_NS_N) ok = wide_wait(empty + slot, uint32_t((s / WIDE_NS_N) - 1) & 1u, err, wc.limit_ns);
            if (!ok) break;
            const int c = 32 * s + k;
            const bool have = c < ncols;
            const uint2 wce = wq[(s % WIDE_WQ) * WIDE_PRODUCERS + p];
            const uint32_t idx = wce.x;
            const uint32_t* vrow = (idx & VEC_T) ? ts + size_t(idx & ~VEC_T) * (WIDE_TERMS / 2)
                                                 : xs + size_t(idx) * (WIDE_TERMS / 2);
            const uint32_t sa = s0 + uint32_t(slot) * WIDE_N_STAGE, sb = sa + 8192u;
            // vector terms: unit u of the row -> M-atom u / 8 (4 KB apart), K-atom k / 8, row k % 8
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                const int uu = 8 * half + i;
                tc5::cp16(sa + uint32_t(half) * 4096u + uint32_t(k >> 3) * 1024u + swz(k & 7, i),
                          have ? static_cast<const void*>(vrow + 4 * uu) : static_cast<const void*>(xs),
                          have ? 16u : 0u);
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
            if (s + WIDE_PF < nst) prefetch(s + WIDE_PF);
            tc5::cp_commit();
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
                if (first && q >= 2) ok = wide_wait(tempty + buf, uint32_t((q >> 1) - 1) & 1u, err, wc.limit_ns);
                if (ok) ok = wide_wait(full + slot, uint32_t(s / WIDE_NS_N) & 1u, err, wc.limit_ns);
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
            if (!mbar_wait(done, 0u, wc.limit_ns)) atomicOr(err, WIDE_ERR_WAIT);
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
            ok = __all_sync(0xffffffffu, wide_wait(tfull + buf, uint32_t(q >> 1) & 1u, err, wc.limit_ns));
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
