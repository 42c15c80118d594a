// The 64-vector product of 16-bit H stores with TMA operand staging (full
// 64-row tiles; ragged tiles keep the cp.async kernels of kernels_wide.cuh).
//
// The same products as kernels_wide.cuh (split rows, static exponents, FP32
// tensor-core accumulation drained to FP64), but every operand tile reaches
// shared memory through 2-D TMA loads (cp.async.bulk.tensor, no multicast,
// this GPU's own memory) with the 128-byte swizzle the MMA descriptors
// expect, issued by one producer thread per CTA and completing on the
// stage's mbarrier: no load passes through the L1/LSU path and no producer
// thread waits on data.  Tensor maps (CUtensorMap, built on the host):
//   store, box 64 x 16 and 64 x 8: the store seen as rows of 128 bytes, so
//     one row is one column of a full-height 16-bit slab;
//   xs / ts, box 64 x 16 and 64 x 64: the split rows (256 bytes), read in two
//     halves of 64 terms (the two M atoms of the vector operand).
//
// N-form (k_nform_wtma): a CTA per full-height output tile; a stage is a run
// of <= 32 columns with consecutive vector entries (WStage), 16 or 32 rows
// of both operands; matrix rows past the run's columns (the next run's
// data) are zeroed by the MMA warp before its MMAs.  All of a tile's columns
// have factor 1 (the store's row-group scales), so the staged data is used
// as it lands, and the whole run accumulates in one FP32 TMEM accumulator
// (FP32 accumulation per output tile, FP64 y), drained once.
//
// Column-cluster T-form (k_ctform_wtma): persistent CTAs, each taking every
// (gridDim)-th unit; a stage is one tile of a unit: its split rows of x
// (64 x 128 terms) and the units' V columns in 8-column boxes (stacked
// blocks start on multiples of 8; the columns between a block's rank and
// its 8-column boundary hold the neighbouring slab's data, whose results
// nobody reads).  The accumulator alternates between two TMEM buffers per
// unit, so the epilogue of one unit overlaps the loads and MMAs of the next.
#pragma once

#include <cuda.h>

#include "kernels_wide.cuh"

namespace hlrc {

constexpr int WTMA_THREADS = 192;     // N-form: 4 epilogue warps, MMA warp, producer warp
constexpr int WTMA_THREADS_C = 320;   // T-form: 8 epilogue warps (two per TMEM lane quarter), MMA, producer
constexpr int WTMA_EPI_C = 256;       // T-form epilogue threads
#ifndef HLRC_WTMA_NS_N
#define HLRC_WTMA_NS_N 4
#endif
constexpr int WTMA_NS_N = HLRC_WTMA_NS_N;   // N-form stages (12 KB each; 4 CTAs per SM at 4)
constexpr int WTMA_NS_C = 3;          // T-form stages (32 KB each)
constexpr int WTMA_RED_COLS = 16;     // T-form epilogue: columns per TMEM load
constexpr int wtma_smem_n() { return 1024 + WTMA_NS_N * WIDE_N_STAGE + 64 + WIDE_BAR_BYTES; }
constexpr int wtma_smem_c() { return 1024 + WTMA_NS_C * WIDE_C_STAGE + 2 * WT_MAXN * 16 + WIDE_BAR_BYTES; }

// 16 consecutive FP32 columns of the warp's 32 lanes (as tmem_ld32)
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n\t"
        "tcgen05.wait::ld.sync.aligned;\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// AND of p over the T-form's 256 epilogue threads, which all arrive
// (named barrier 1)
__device__ __forceinline__ bool bar_and_epi(bool p) {
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred pi, po;\n\tsetp.ne.u32 pi, %1, 0;\n\tbar.red.and.pred po, 1, 256, pi;\n\t"
        "selp.u32 %0, 1, 0, po;\n\t}\n"
        : "=r"(r)
        : "r"(uint32_t(p))
        : "memory");
    return r != 0;
}
__device__ __forceinline__ void bar_epi() { asm volatile("bar.sync 1, 256;\n" ::: "memory"); }

// ----------------------------------------------------------------- N-form
template <int FMT>
__global__ void __launch_bounds__(WTMA_THREADS, 4)
k_nform_wtma(const WSeg* __restrict__ segs, const WStage* __restrict__ stages, const __grid_constant__ CUtensorMap tm_a,
             const __grid_constant__ CUtensorMap tm_x, const __grid_constant__ CUtensorMap tm_t,
             const int* __restrict__ g, OutMap om, double alpha, int* err, WaitCfg wc) {
    using namespace tc5;
    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    uint8_t* sm = smem_raw + (((raw + 1023u) & ~1023u) - raw);
    int* snc = reinterpret_cast<int*>(sm + WTMA_NS_N * WIDE_N_STAGE);   // columns per slot
    uint64_t* full = reinterpret_cast<uint64_t*>(snc + 16);
    uint64_t* empty = full + WTMA_NS_N;
    uint64_t* tfull = empty + WTMA_NS_N;
    uint64_t* done = tfull + 1;
    uint32_t* tslot = reinterpret_cast<uint32_t*>(done + 1);

    const WSeg sg = segs[blockIdx.x];
    const int nst = int(sg.nst);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (nst == 0) return;
    if (threadIdx.x == 0) {
        for (int i = 0; i < WTMA_NS_N; ++i) {
            mbar_init(full + i, 1);
            mbar_init(empty + i, 1);
        }
        mbar_init(tfull, 1);
        mbar_init(done, 1);
        mbar_init_fence();
    }
    if (warp == 4) tmem_alloc(tslot, 64);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;
    const uint32_t s0 = smem_u32(sm);

    if (warp == 5) {
        // ---------------------------------------------------- producer
        if (lane == 0) {
            const WStage* st = stages + sg.st0;
            // stage descriptors are read 8 stages ahead (one register set
            // per position of the unrolled group)
            WStage pre[8];
#pragma unroll
            for (int i = 0; i < 8; ++i) pre[i] = i < nst ? st[i] : WStage{0u, 0u, 0u};
            bool ok = true;
            int last = -1;   // the last stage whose loads were issued
            for (int b = 0; b < nst && ok; b += 8) {
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    const int s = b + i;
                    if (s >= nst || !ok) break;
                    const WStage d = pre[i];
                    if (s + 8 < nst) pre[i] = st[s + 8];
                    const int slot = s % WTMA_NS_N;
                    if (s >= WTMA_NS_N) ok = wide_wait(empty + slot, uint32_t((s / WTMA_NS_N) - 1) & 1u, err, wc.limit_ns);
                    if (!ok) break;
                    const int R = d.nc <= 16 ? 16 : 32;
                    snc[slot] = int(d.nc);
                    if (wc.skip && s == 0) continue;   // test hook: stage 0 is never handed over
                    mbar_arrive_tx(full + slot, uint32_t(384 * R));
                    const uint32_t sa = s0 + uint32_t(slot) * WIDE_N_STAGE, sb = sa + 8192u;
                    const void* tv = (d.e0 & VEC_T) ? static_cast<const void*>(&tm_t) : static_cast<const void*>(&tm_x);
                    const int e = int(d.e0 & ~VEC_T);
                    for (int h = 0; h < R / 16; ++h) {
                        tma_load_2d(sb + 2048u * h, &tm_a, 0, int(d.srow) + 16 * h, full + slot);
                        tma_load_2d(sa + 2048u * h, tv, 0, e + 16 * h, full + slot);
                        tma_load_2d(sa + 4096u + 2048u * h, tv, 64, e + 16 * h, full + slot);
                    }
                    last = s;
                }
            }
            // no load may still be in flight when the CTA ends: wait for the
            // stages not known to be consumed (returns at once when they were)
            for (int sd = max(0, last - WTMA_NS_N + 1); sd <= last; ++sd)
                if (!(wc.skip && sd == 0)) mbar_wait(full + sd % WTMA_NS_N, uint32_t(sd / WTMA_NS_N) & 1u, wc.limit_ns);
        }
        __syncwarp();
    } else if (warp == 4) {
        // ------------------------------------------------ zero + MMA issue
        constexpr uint32_t ID16 = tc5::idesc_f16(128, 64, WideT<FMT>::bf16, true, true);
        bool ok = true;
        for (int s = 0; s < nst && ok; ++s) {
            const int slot = s % WTMA_NS_N;
            bool w = true;
            if (lane == 0) w = wide_wait(full + slot, uint32_t(s / WTMA_NS_N) & 1u, err, wc.limit_ns);
            ok = __shfl_sync(0xffffffffu, w, 0);
            if (!ok) break;
            __syncwarp();   // lane 0's wait orders the producer's snc write before these reads
            const int nc = snc[slot], R = nc <= 16 ? 16 : 32;
            // matrix rows (columns of the run) past nc hold the next run's data
            if (nc < R) {
                uint8_t* sb = sm + slot * WIDE_N_STAGE + 8192;
                for (int u = lane; u < (R - nc) * 8; u += 32) {
                    const int k = nc + (u >> 3);
                    *reinterpret_cast<uint4*>(sb + (k >> 3) * 1024 + (k & 7) * 128 + (u & 7) * 16) = make_uint4(0u, 0u, 0u, 0u);
                }
                fence_async_smem();
            }
            __syncwarp();
            if (lane == 0) {
                tc_fence_after();
                const uint32_t sa = s0 + uint32_t(slot) * WIDE_N_STAGE, sb = sa + 8192u;
                for (int j = 0; j < R / 16; ++j)
                    mma_f16(tmem, sdesc(sa + 2048u * j, 4096u, 1024u), sdesc(sb + 2048u * j, 4096u, 1024u), ID16,
                            (s > 0 || j > 0) ? 1u : 0u);
                mma_commit(empty + slot);
                if (s == nst - 1) mma_commit(tfull);
            }
            __syncwarp();
        }
        if (lane == 0) {
            mma_commit(done);
            if (!mbar_wait(done, 0u, wc.limit_ns)) atomicOr(err, WIDE_ERR_WAIT);
        }
        __syncwarp();
    } else {
        // -------------------------------------------------------- epilogue
        // lane m holds term m (vector m / 2, high or low part) of the 64
        // rows, read 16 rows at a time; the two lanes of a vector exchange
        // their terms, and the high-part lane adds rows 0-31 to y, the
        // low-part lane rows 32-63
        const uint32_t la = tmem + (uint32_t(32 * warp) << 16);
        const int m = 32 * warp + lane, r = m >> 1;
        const bool lo = (m & 1) != 0;
        const bool ok = __all_sync(0xffffffffu, wide_wait(tfull, 0u, err, wc.limit_ns)) && !wide_aborted(err);
        if (ok) {
            tc_fence_after();
            const double fr = r < om.nr ? alpha * ldexp(1.0, sg.E - g[r]) : 0.0;
            double* o = om.base + int64_t(sg.out) * om.rs + int64_t(r) * om.cs;
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                float f[16];
                tmem_ld16(la + uint32_t(16 * q), f);
                const bool own = (q >= 2) == lo;
#pragma unroll
                for (int i = 0; i < 16; ++i) {
                    const float other = __shfl_xor_sync(0xffffffffu, f[i], 1);
                    if (own && r < om.nr) o[int64_t(16 * q + i) * om.rs] += fr * (double(f[i]) + double(other));
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 4) {
        tc_fence_after();
        tmem_dealloc(tmem, 64);
    }
}

// ------------------------------------------------- column-cluster T-form
template <int FMT>
__global__ void __launch_bounds__(WTMA_THREADS_C, 2)
k_ctform_wtma(const WTUnit* __restrict__ units, int nunits, const WTBlk* __restrict__ blks,
              const uint32_t* __restrict__ slabs, const WTTile* __restrict__ tiles, const WCDst* __restrict__ ctab,
              const __grid_constant__ CUtensorMap tm_s8, const __grid_constant__ CUtensorMap tm_x64,
              uint32_t* __restrict__ ts, float* __restrict__ part, int* err, WaitCfg wc) {
    using namespace tc5;
    constexpr int MMA_WARP = 8, PROD_WARP = 9;
    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    uint8_t* sm = smem_raw + (((raw + 1023u) & ~1023u) - raw);
    // two buffers of a unit's column table (output entry, factor, static
    // exponent per stacked column), the next unit's copied in while the
    // current one is written out
    WCDst* stab = reinterpret_cast<WCDst*>(sm + WTMA_NS_C * WIDE_C_STAGE);
    uint64_t* full = reinterpret_cast<uint64_t*>(stab + 2 * WT_MAXN);
    uint64_t* empty = full + WTMA_NS_C;
    uint64_t* tfull = empty + WTMA_NS_C;
    uint64_t* tempty = tfull + 2;
    uint64_t* done = tempty + 2;
    uint32_t* tslot = reinterpret_cast<uint32_t*>(done + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (int(blockIdx.x) >= nunits) return;
    if (threadIdx.x == 0) {
        for (int i = 0; i < WTMA_NS_C; ++i) {
            mbar_init(full + i, 1);
            mbar_init(empty + i, 1);
        }
        for (int i = 0; i < 2; ++i) {
            mbar_init(tfull + i, 1);
            mbar_init(tempty + i, WTMA_EPI_C);
        }
        mbar_init(done, 1);
        mbar_init_fence();
    }
    if (warp == MMA_WARP) tmem_alloc(tslot, 256);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;
    const uint32_t s0 = smem_u32(sm);

    if (warp == PROD_WARP) {
        // ---------------------------------------------------- producer warp
        // lane j stages block j of the unit (its V columns in 8-column
        // boxes); lane 0 also the split rows of x and the stage's byte count
        bool ok = true;
        int s = 0, last = -1;   // last: the last stage whose loads were issued
        for (int ui = int(blockIdx.x); ui < nunits && ok; ui += int(gridDim.x)) {
            const WTUnit u = units[ui];
            const bool mine = lane < int(u.nblk);
            int boxes = 0, off = 0;
            if (mine) {
                const WTBlk b = blks[u.blk0 + lane];
                boxes = (int(b.k) + 7) / 8;
                off = int(b.off);
            }
            int bytes = 1024 * boxes;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) bytes += __shfl_xor_sync(0xffffffffu, bytes, o);
            uint32_t a16n = mine ? slabs[u.slab0 + lane] : 0u;   // tile 0, read ahead tile by tile
            for (int q = 0; q < int(u.ntiles); ++q, ++s) {
                const int slot = s % WTMA_NS_C;
                bool w = true;
                if (lane == 0 && s >= WTMA_NS_C) w = wide_wait(empty + slot, uint32_t((s / WTMA_NS_C) - 1) & 1u, err, wc.limit_ns);
                ok = __shfl_sync(0xffffffffu, w, 0);
                if (!ok) break;
                const uint32_t a16 = a16n;
                if (mine && q + 1 < int(u.ntiles)) a16n = slabs[u.slab0 + (q + 1) * u.nblk + lane];
                if (wc.skip && s == 0) continue;   // test hook: stage 0 is never handed over
                const uint32_t sa = s0 + uint32_t(slot) * WIDE_C_STAGE, sb = sa + 16384u;
                if (lane == 0) {
                    mbar_arrive_tx(full + slot, uint32_t(16384 + bytes));
                    const int v0 = int(tiles[u.tile0 + q].v_off);
                    tma_load_2d(sa, &tm_x64, 0, v0, full + slot);
                    tma_load_2d(sa + 8192u, &tm_x64, 64, v0, full + slot);
                }
                __syncwarp();
                for (int h = 0; h < boxes; ++h)
                    tma_load_2d(sb + uint32_t(off / 8 + h) * 1024u, &tm_s8, 0, int(a16 / 8) + 8 * h, full + slot);
                last = s;
            }
        }
        // no load may still be in flight when the CTA ends (see the N-form)
        if (lane == 0)
            for (int sd = max(0, last - WTMA_NS_C + 1); sd <= last; ++sd)
                if (!(wc.skip && sd == 0)) mbar_wait(full + sd % WTMA_NS_C, uint32_t(sd / WTMA_NS_C) & 1u, wc.limit_ns);
        __syncwarp();
    } else if (warp == MMA_WARP) {
        // ------------------------------------------------------- MMA issue
        if (lane == 0) {
            bool ok = true;
            int s = 0, i = 0;
            for (int ui = int(blockIdx.x); ui < nunits && ok; ui += int(gridDim.x), ++i) {
                const WTUnit u = units[ui];
                const int buf = i & 1;
                const int npad = (int(u.ncols) + 15) & ~15;
                const uint32_t id = tc5::idesc_f16(128, npad, WideT<FMT>::bf16, true, false);
                if (i >= 2) ok = wide_wait(tempty + buf, uint32_t((i >> 1) - 1) & 1u, err, wc.limit_ns);
                const uint32_t d = tmem + uint32_t(buf) * 128u;
                for (int q = 0; q < int(u.ntiles) && ok; ++q, ++s) {
                    const int slot = s % WTMA_NS_C;
                    ok = wide_wait(full + slot, uint32_t(s / WTMA_NS_C) & 1u, err, wc.limit_ns);
                    if (!ok) break;
                    tc_fence_after();
                    const uint32_t sa = s0 + uint32_t(slot) * WIDE_C_STAGE, sb = sa + 16384u;
#pragma unroll
                    for (int j = 0; j < 4; ++j)
                        mma_f16(d, sdesc(sa + 2048u * j, 8192u, 1024u), sdesc(sb + 32u * j, 16u, 1024u), id,
                                (q > 0 || j > 0) ? 1u : 0u);
                    mma_commit(empty + slot);
                }
                if (ok) mma_commit(tfull + buf);
            }
            mma_commit(done);
            if (!mbar_wait(done, 0u, wc.limit_ns)) atomicOr(err, WIDE_ERR_WAIT);
        }
        __syncwarp();
    } else {
        // -------------------------------------------------------- epilogue
        // warps w and w + 4 read TMEM lanes 32 (w % 4) ... (term m = lane
        // quarter row), alternating 16-column groups; the two lanes of a
        // vector exchange halves, the high-part lane sums hi + lo for the
        // even columns, the low-part lane for the odd ones, and each stores
        // its columns' entries of vector r = m / 2.  The column tables come
        // from the host-built table (WT_MAXN entries per unit), copied one
        // unit ahead.
        const int et = threadIdx.x;                 // 0 .. 255
        const uint32_t la0 = tmem + (uint32_t(32 * (warp & 3)) << 16);
        const int m = 32 * (warp & 3) + lane, r = m >> 1, odd = m & 1;
        const int half = warp >> 2;
        auto prefetch = [&](int uix, int b) {
            if (uix < nunits && et < WT_MAXN)
                tc5::cp16(smem_u32(stab + b * WT_MAXN + et), ctab + size_t(uix) * WT_MAXN + et, 16u);
            tc5::cp_commit();
        };
        prefetch(int(blockIdx.x), 0);
        WTUnit un = units[blockIdx.x];
        int i = 0;
        for (int ui = int(blockIdx.x); ui < nunits; ui += int(gridDim.x), ++i) {
            const int buf = i & 1;
            const WTUnit u = un;
            const int nxt = ui + int(gridDim.x);
            if (nxt < nunits) un = units[nxt];
            // all eight warps take the same branch (the named barriers below
            // need every one of them)
            if (!bar_and_epi(wide_wait(tfull + buf, uint32_t(i >> 1) & 1u, err, wc.limit_ns))) break;
            tc_fence_after();
            prefetch(nxt, buf ^ 1);
            tc5::cp_wait<1>();   // this unit's table has landed (own copies) ...
            bar_epi();      // ... and everyone's
            const WCDst* tab = stab + buf * WT_MAXN;
            const int nc = int(u.ncols);
            const bool final_t = u.npieces == 1;
            const uint32_t la = la0 + uint32_t(buf) * 128u;
            for (int c0 = 16 * half; c0 < nc; c0 += 32) {
                float f[16];
                tmem_ld16(la + uint32_t(c0), f);
#pragma unroll
                for (int k = 0; k < 8; ++k) {
                    const float other = __shfl_xor_sync(0xffffffffu, odd ? f[2 * k] : f[2 * k + 1], 1);
                    const WCDst d = tab[c0 + 2 * k + odd];   // < WT_MAXN: c0 <= 112
                    // hi + lo terms, times the chunk scale and (t rows) 2^-c: FP32
                    const float v = ((odd ? f[2 * k + 1] : f[2 * k]) + other) * d.fac;
                    if (d.dst != WT_NODST) {
                        if (final_t) ts[size_t(d.dst) * (WIDE_TERMS / 2) + r] = wide_split_f<FMT>(v);
                        else part[size_t(d.dst) * WIDE_RHS + r] = v;
                    }
                }
            }
            tc_fence_before();
            mbar_arrive(tempty + buf);
            // the next prefetch overwrites this buffer only after every thread is done
            bar_epi();
        }
        tc5::cp_wait<0>();   // no copy in flight at exit
    }
    tc_fence_before();
    __syncthreads();
    if (warp == MMA_WARP) {
        tc_fence_after();
        tmem_dealloc(tmem, 256);
    }
}

}  // namespace hlrc
