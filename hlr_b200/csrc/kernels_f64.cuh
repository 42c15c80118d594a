// FP64 batched GEMV kernels of the H / uniform-H product (sm_100a).
//
// Both kernels stream the matrix slabs with 128-bit loads marked
// evict-first (each matrix byte is read exactly once per product) while the
// small vectors x / t stay cache resident.
#pragma once

#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include "layout.hpp"

namespace hlrc {

namespace cg = cooperative_groups;

__device__ __forceinline__ double2 ld_stream(const double* p) {
    return __ldcs(reinterpret_cast<const double2*>(p));
}

// Programmatic dependent launch.  The one-vector kernels are launched so
// that the next kernel in the stream may start while they run: each lets
// its successor launch as soon as it has started (pdl_trigger), reads only
// its static descriptors before pdl_wait, and after pdl_wait (which returns
// once the preceding kernel has completed and its writes are visible) reads
// and writes the vectors.  Without the launch attribute both are no-ops.
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }

// Butterfly transpose-reduction of N per-lane column partials (N = 2^g,
// g <= 5): at each step a lane keeps one half of its values and trades the
// other half with its partner, so 32 columns cost 31 shuffles instead of
// 5 * 32.  Afterwards p[0] holds the warp total of column lane >> (5 - g).
template <int N, int O, typename T = double>
struct TransposeReduce {
    static __device__ __forceinline__ void run(T* p, int lane) {
        if constexpr (N > 1) {
            constexpr int H = N / 2;
            const bool up = (lane & O) != 0;
#pragma unroll
            for (int j = 0; j < H; ++j) {
                const T send = up ? p[j] : p[j + H];
                const T keep = up ? p[j + H] : p[j];
                p[j] = keep + __shfl_xor_sync(0xffffffffu, send, O);
            }
            if constexpr (O > 1) TransposeReduce<H, O / 2, T>::run(p, lane);
        } else {
            p[0] += __shfl_xor_sync(0xffffffffu, p[0], O);
            if constexpr (O > 1) TransposeReduce<1, O / 2, T>::run(p, lane);
        }
    }
};

template <int N> struct Log2;
template <> struct Log2<8> { static constexpr int v = 3; };
template <> struct Log2<16> { static constexpr int v = 4; };
template <> struct Log2<32> { static constexpr int v = 5; };

// N-form: one CTA (W warps) per output tile; chunk c goes to warp c % W;
// lane l owns rows 2l, 2l+1; warps are summed in index order.
template <int W>
__global__ void __launch_bounds__(W * 32)
k_nform_f64(const NSeg* __restrict__ segs, const NChunk* __restrict__ chunks, const double* __restrict__ A,
            const double* __restrict__ vx, const double* __restrict__ vt, double* __restrict__ out, double alpha,
            int add) {
    __shared__ double red[W][TILE];
    pdl_trigger();
    const NSeg sg = segs[blockIdx.x];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int r = 2 * lane;
    const bool active = r < sg.ld;
    double acc0 = 0.0, acc1 = 0.0;
    pdl_wait();
    for (uint32_t c = sg.cb + warp; c < sg.ce; c += W) {
        const NChunk ch = chunks[c];
        const double* v = (ch.v_off & VEC_T) ? vt + (ch.v_off & ~VEC_T) : vx + ch.v_off;
        if (active) {
            const double* a = A + ch.a_off + r;
            double2 m[NCHUNK];
            double vv[NCHUNK];
#pragma unroll
            for (int j = 0; j < NCHUNK; ++j) {
                if (j < ch.nc) {
                    m[j] = ld_stream(a + size_t(j) * sg.ld);
                    vv[j] = __ldg(v + j);
                } else {
                    m[j] = make_double2(0.0, 0.0);
                    vv[j] = 0.0;
                }
            }
#pragma unroll
            for (int j = 0; j < NCHUNK; ++j) {
                acc0 = fma(m[j].x, vv[j], acc0);
                acc1 = fma(m[j].y, vv[j], acc1);
            }
        }
    }
    red[warp][r] = acc0;
    red[warp][r + 1] = acc1;
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

// Tree entries of a sweep pass (device copies of the planner's arrays) and
// the maxima that size the CTAs' shared memory (tree_smem_bytes).
struct TreeArgs {
    const int* cta_begin;      // levels of subtree b: [cta_begin[b], cta_begin[b+1])
    const int* level;          // segments of level g: [level[g], level[g+1])
    const int* part;           // rank r of level g: segments [part[g*(TC+1)+r], part[g*(TC+1)+r+1])
    const int* seg;            // mirror slot of each segment's first row
    const TreeChunk* chunk;    // stage offset (owner's stage) and mirror slot of each chunk
    const TreeExt* ext;        // coefficients copied in from outside the subtree
    const int* cta_ext;        // subtree b's entries of ext: [cta_ext[b], cta_ext[b+1])
    int stage, mirror, levels, segs, chunks, items;
};

// Bulk copies (TMA, no multicast) into this CTA's shared memory, completed
// on an mbarrier per level.
__device__ __forceinline__ unsigned tree_saddr(const void* p) {
    return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void tree_bar_init(uint64_t* bar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(tree_saddr(bar)) : "memory");
}
__device__ __forceinline__ void tree_bar_init_fence() {
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ void tree_bar_expect(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.expect_tx.relaxed.cta.shared::cta.b64 [%0], %1;\n" ::"r"(tree_saddr(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void tree_bar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(tree_saddr(bar)) : "memory");
}
__device__ __forceinline__ void tree_bulk(double* dst, const double* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                     tree_saddr(dst)),
                 "l"(src), "r"(bytes), "r"(tree_saddr(bar))
                 : "memory");
}
// Waits for phase 0 of the barrier for at most limit_ns of wall-clock time
// (%globaltimer); false when the time ran out.
__device__ __forceinline__ uint64_t tree_clock() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
    return t;
}
__device__ __forceinline__ bool tree_bar_wait(uint64_t* bar, uint64_t limit_ns) {
    const uint64_t t0 = tree_clock();
    for (uint32_t i = 0;; ++i) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(tree_saddr(bar))
            : "memory");
        if (done) return true;
        if ((i & 15u) == 15u && tree_clock() - t0 > limit_ns) return false;
    }
}

// Tree sweep of the H^2 transfers: one cluster of TREE_CLUSTER CTAs per
// subtree runs its levels one after the other; rank r of the cluster
// computes its run of each level's segments.  Prologue (every CTA): the
// subtree's segment and chunk descriptors are loaded; the matrix data of the
// CTA's own chunks is copied into its stage by bulk copies (one per chunk,
// each thread expecting the bytes of its own copies on the level's barrier),
// so that the copies of later levels overlap the work of earlier ones; the
// coefficients the subtree reads from outside (the leaves' going up, the
// subtree root's going down) and, when adding, the current values of the
// CTA's outputs are loaded into its mirror.  Level g: the CTA waits for its
// own copies of the level; its chunks go to the half-warps (two rows per
// lane, 32-row blocks), each writing a column partial to shared memory;
// after a barrier every output row sums its segment's partials in chunk
// order, and the result goes to the mirrors of all CTAs of the cluster
// (distributed shared memory) and to the output array; a cluster barrier
// ends the level.  Summation order is fixed: the result is deterministic.
// A copy that never completes stops the CTA's work: it sets bit 0 of the
// error word, keeps taking part in the cluster barriers, and waits
// (bounded) for its other copies before returning.  Each wait lasts at most
// wait_ns; skip != 0 (the test hook of hlrc_debug_waits) announces 16 bytes
// more on the first level's barrier than its copies deliver, so that its
// wait runs out with no copy left in flight.
template <int W>
__global__ void __cluster_dims__(TREE_CLUSTER, 1, 1) __launch_bounds__(W * 32)
k_ntree_f64(const NSeg* __restrict__ segs, const NChunk* __restrict__ chunks, TreeArgs t,
            const double* __restrict__ A, const double* vx, const double* vt, double* out, double alpha, int add,
            int* err, uint64_t wait_ns, int skip) {
    constexpr int TC = TREE_CLUSTER;
    pdl_trigger();
    cg::cluster_group cl = cg::this_cluster();
    const int rank = int(cl.block_rank());
    const int sub = int(blockIdx.x) / TC;
    extern __shared__ double2 tree_smem[];
    double* stage = reinterpret_cast<double*>(tree_smem);
    double2* part2 = tree_smem + t.stage / 2;
    double* mirror = reinterpret_cast<double*>(part2 + size_t(t.items) * (TILE / 2));
    uint64_t* bars = reinterpret_cast<uint64_t*>(mirror + ((t.mirror + 1) & ~1));
    NSeg* sseg = reinterpret_cast<NSeg*>(bars + ((t.levels + 1) & ~1));
    int* sseg_m = reinterpret_cast<int*>(sseg + t.segs);
    NChunk* sch = reinterpret_cast<NChunk*>(sseg_m + ((t.segs + 3) & ~3));
    TreeChunk* sct = reinterpret_cast<TreeChunk*>(sch + t.chunks);
    int* srun = reinterpret_cast<int*>(sct + t.chunks);   // [2 * level]: this rank's run of the level's segments
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int g0 = t.cta_begin[sub], g1 = t.cta_begin[sub + 1], nlev = g1 - g0;
    const int S0 = t.level[g0], nseg = t.level[g1] - S0;
    const uint32_t C0 = segs[S0].cb, nch = segs[S0 + nseg - 1].ce - C0;
    if (tid == 0) {
        for (int i = 0; i < nlev; ++i) tree_bar_init(&bars[i]);
        tree_bar_init_fence();
    }
    for (int i = tid; i < nseg; i += W * 32) {
        sseg[i] = segs[S0 + i];
        sseg_m[i] = t.seg[S0 + i];
    }
    for (uint32_t i = tid; i < nch; i += W * 32) {
        sch[i] = chunks[C0 + i];
        sct[i] = t.chunk[C0 + i];
    }
    for (int i = tid; i < 2 * nlev; i += W * 32) srun[i] = t.part[size_t(g0 + i / 2) * (TC + 1) + rank + (i & 1)] - S0;
    __syncthreads();
    for (int gi = 0; gi < nlev; ++gi) {   // own matrix data: chunk k of the level's run to thread k % (32 W)
        const int sb = srun[2 * gi], se = srun[2 * gi + 1];
        if (sb >= se) continue;
        const uint32_t k0 = sseg[sb].cb, k1 = sseg[se - 1].ce;
        uint32_t bytes = 0;
        int si = sb;
        for (uint32_t c = k0 + tid; c < k1; c += W * 32) {
            while (c >= sseg[si].ce) ++si;
            bytes += uint32_t(sch[c - C0].nc) * sseg[si].ld * uint32_t(sizeof(double));
        }
        if (bytes == 0) continue;
        tree_bar_expect(&bars[gi], bytes);
        si = sb;
        for (uint32_t c = k0 + tid; c < k1; c += W * 32) {
            while (c >= sseg[si].ce) ++si;
            const NChunk ch = sch[c - C0];
            tree_bulk(stage + sct[c - C0].stage, A + ch.a_off, uint32_t(ch.nc) * sseg[si].ld * uint32_t(sizeof(double)),
                      &bars[gi]);
        }
    }
    if (skip && tid == 0 && nlev > 0) tree_bar_expect(&bars[0], 16u);
    __syncthreads();   // every expectation is set: the one arrival may complete a phase
    if (tid == 0)
        for (int i = 0; i < nlev; ++i) tree_bar_arrive(&bars[i]);
    // the matrix copies above read static data; the vectors below are
    // written by the preceding kernel
    pdl_wait();
    for (int e = t.cta_ext[sub] + tid; e < t.cta_ext[sub + 1]; e += W * 32) {
        const TreeExt x = t.ext[e];
        mirror[x.mirror] = __ldcg((x.v_off & VEC_T) ? vt + (x.v_off & ~VEC_T) : vx + x.v_off);
    }
    if (add)
        for (int gi = 0; gi < nlev; ++gi) {
            for (int q = srun[2 * gi] + warp; q < srun[2 * gi + 1]; q += W)
                for (int i = lane; i < sseg[q].rows; i += 32) mirror[sseg_m[q] + i] = __ldcg(out + sseg[q].out + i);
        }
    cl.sync();   // every CTA of the cluster runs before any writes into its mirror
    const int hw = 2 * warp + (lane >> 4), l16 = lane & 15;
    bool failed = false;
    for (int gi = 0; gi < nlev; ++gi) {
        const bool ok = failed || tree_bar_wait(&bars[gi], wait_ns);
        if (__syncthreads_or(!ok)) {
            if (tid == 0 && !failed) atomicOr(err, 1);
            failed = true;
        }
        if (!failed) {
            const int sb = srun[2 * gi], se = srun[2 * gi + 1];
            const uint32_t k0 = sb < se ? sseg[sb].cb : 0, k1 = sb < se ? sseg[se - 1].ce : 0;
            int si = sb;
            for (uint32_t c = k0 + hw; c < k1; c += 2 * W) {
                while (c >= sseg[si].ce) ++si;
                const int ld = sseg[si].ld;
                const NChunk ch = sch[c - C0];
                const TreeChunk tc = sct[c - C0];
                const double* v = mirror + tc.mirror;
                for (int rr = 2 * l16; rr < ld; rr += 32) {
                    const double* a = stage + tc.stage + rr;
                    double acc0 = 0.0, acc1 = 0.0;
#pragma unroll
                    for (int j = 0; j < NCHUNK; ++j)
                        if (j < ch.nc) {
                            const double2 m = *reinterpret_cast<const double2*>(a + j * ld);
                            acc0 = fma(m.x, v[j], acc0);
                            acc1 = fma(m.y, v[j], acc1);
                        }
                    part2[size_t(c - k0) * (TILE / 2) + rr / 2] = make_double2(acc0, acc1);
                }
            }
            __syncthreads();
            const double* part = reinterpret_cast<const double*>(part2);
            for (int i = tid; i < (se - sb) * TILE; i += W * 32) {
                const int q = sb + i / TILE, row = i % TILE;
                const NSeg sg = sseg[q];
                if (row < sg.rows) {
                    double sum = 0.0;
                    for (uint32_t c = sg.cb; c < sg.ce; ++c) sum += part[size_t(c - k0) * TILE + row];
                    const int slot = sseg_m[q] + row;
                    const double y = add ? mirror[slot] + alpha * sum : sum;
#pragma unroll
                    for (int r = 0; r < TC; ++r) *cl.map_shared_rank(mirror + slot, r) = y;
                    out[sg.out + row] = y;
                }
            }
        }
        cl.sync();   // the level's rows are in every mirror; partials free
    }
    if (failed)
        for (int k = 0; k < nlev; ++k) tree_bar_wait(&bars[k], wait_ns);
}

// T-form: one warp per unit; lane l owns rows 2l, 2l+1 of every slab and
// keeps NC column partials in registers; one transpose-reduction per unit.
template <int NC>
__global__ void __launch_bounds__(256)
k_tform_f64(const TUnit* __restrict__ units, int nunits, const TSlab* __restrict__ slabs,
            const double* __restrict__ A, const double* __restrict__ vin, double* __restrict__ out,
            double* __restrict__ part, double alpha, int add) {
    pdl_trigger();
    const int wid = blockIdx.x * 8 + (threadIdx.x >> 5);
    if (wid >= nunits) return;
    const int lane = threadIdx.x & 31;
    const TUnit u = units[wid];
    pdl_wait();
    double p[NC];
#pragma unroll
    for (int j = 0; j < NC; ++j) p[j] = 0.0;
    const int r = 2 * lane;
    // the next slab's descriptor is fetched one iteration ahead so that its
    // latency overlaps the current slab's loads
    TSlab sl = u.sb < u.se ? slabs[u.sb] : TSlab{0, 0, 0, 0};
    for (uint32_t s = u.sb; s < u.se; ++s) {
        const TSlab cur = sl;
        if (s + 1 < u.se) sl = slabs[s + 1];
        if (r < cur.ld) {
            const double v0 = (r < cur.rows) ? __ldg(vin + cur.v_off + r) : 0.0;
            const double v1 = (r + 1 < cur.rows) ? __ldg(vin + cur.v_off + r + 1) : 0.0;
            const double* a = A + cur.a_off + size_t(u.c0) * cur.ld + r;
            double2 m[NC];
#pragma unroll
            for (int j = 0; j < NC; ++j) m[j] = (j < u.nc) ? ld_stream(a + size_t(j) * cur.ld) : make_double2(0.0, 0.0);
#pragma unroll
            for (int j = 0; j < NC; ++j) p[j] = fma(m[j].y, v1, fma(m[j].x, v0, p[j]));
        }
    }
    TransposeReduce<NC, 16>::run(p, lane);
    constexpr int SH = 5 - Log2<NC>::v;
    const int c = lane >> SH;
    if ((lane & ((1 << SH) - 1)) == 0 && c < u.nc) {
        if (u.flags & TU_DIRECT) {
            double* o = out + u.out + c;
            if (add) *o += alpha * p[0];
            else *o = p[0];
        } else {
            part[size_t(u.out) * 32 + c] = p[0];
        }
    }
}

// Tile T-form: one CTA (W warps) per input tile; x restricted to the tile
// stays in registers (lane l holds rows 2l, 2l+1); chunk c goes to warp
// c % W and is reduced on its own (8 columns -> one transpose-reduction).
template <int W>
__global__ void __launch_bounds__(W * 32)
k_ttform_f64(const TTSeg* __restrict__ segs, const TTChunk* __restrict__ chunks, const double* __restrict__ A,
             const double* __restrict__ vin, double* __restrict__ out, double* __restrict__ part, double alpha,
             int add) {
    pdl_trigger();
    const TTSeg sg = segs[blockIdx.x];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int r = 2 * lane;
    const bool active = r < sg.ld;
    pdl_wait();
    const double v0 = (r < sg.rows) ? __ldg(vin + sg.v_off + r) : 0.0;
    const double v1 = (r + 1 < sg.rows) ? __ldg(vin + sg.v_off + r + 1) : 0.0;
    // software pipeline: the loads of chunk c + W are issued before chunk c
    // is reduced and written; descriptors are fetched two iterations ahead
    uint32_t c = sg.cb + warp;
    if (c >= sg.ce) return;
    TTChunk cur = chunks[c], nxt{0, 0, 0, 0};
    if (c + W < sg.ce) nxt = chunks[c + W];
    double2 m[TCOLS];
    auto issue = [&](const TTChunk& q) {
        const double* a = A + q.a_off + r;
#pragma unroll
        for (int j = 0; j < TCOLS; ++j)
            m[j] = (active && j < q.nc) ? ld_stream(a + size_t(j) * sg.ld) : make_double2(0.0, 0.0);
    };
    issue(cur);
    for (; c < sg.ce; c += W) {
        double p[TCOLS];
#pragma unroll
        for (int j = 0; j < TCOLS; ++j) p[j] = fma(m[j].y, v1, m[j].x * v0);
        const TTChunk ch = cur;
        if (c + W < sg.ce) {
            cur = nxt;
            issue(cur);
            if (c + 2 * W < sg.ce) nxt = chunks[c + 2 * W];
        }
        TransposeReduce<TCOLS, 16>::run(p, lane);
        constexpr int SH = 5 - Log2<TCOLS>::v;
        const int col = lane >> SH;
        if ((lane & ((1 << SH) - 1)) == 0 && col < ch.nc) {
            if (ch.flags & TT_DIRECT) {
                double* o = out + ch.out + col;
                if (add) *o += alpha * p[0];
                else *o = p[0];
            } else {
                part[ch.out + col] = p[0];
            }
        }
    }
}

// Sums the per-tile partials of multi-tile tile-T-form outputs in tile order
// (one-vector products; a warp per output, lanes over its columns).
__global__ void __launch_bounds__(256)
k_ttfinish_f64(const TGroup* __restrict__ groups, int ngroups, const double* __restrict__ part,
               double* __restrict__ out, double alpha, int add) {
    pdl_trigger();
    const int gid = blockIdx.x * 8 + (threadIdx.x >> 5);
    if (gid >= ngroups) return;
    const int lane = threadIdx.x & 31;
    const TGroup g = groups[gid];
    pdl_wait();
    for (uint32_t j = lane; j < g.nc; j += 32) {
        // four interleaved partial sums keep four loads in flight; they are
        // combined in a fixed order, so the result is deterministic
        const double* p = part + size_t(g.slot0) + j;
        double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
        uint32_t i = 0;
        // sixteen loads in flight, then the same sums in the same order
        for (; i + 16 <= g.nslots; i += 16) {
            double v[16];
#pragma unroll
            for (int q = 0; q < 16; ++q) v[q] = p[size_t(i + q) * g.nc];
#pragma unroll
            for (int q = 0; q < 16; q += 4) {
                s0 += v[q];
                s1 += v[q + 1];
                s2 += v[q + 2];
                s3 += v[q + 3];
            }
        }
        for (; i + 4 <= g.nslots; i += 4) {
            s0 += p[size_t(i) * g.nc];
            s1 += p[size_t(i + 1) * g.nc];
            s2 += p[size_t(i + 2) * g.nc];
            s3 += p[size_t(i + 3) * g.nc];
        }
        for (; i < g.nslots; ++i) s0 += p[size_t(i) * g.nc];
        const double s = (s0 + s1) + (s2 + s3);
        double* o = out + g.out + j;
        if (add) *o += alpha * s;
        else *o = s;
    }
}

// Sums the partial slots of multi-unit T-form outputs in slot order.
__global__ void __launch_bounds__(256)
k_tfinish_f64(const TGroup* __restrict__ groups, int ngroups, const double* __restrict__ part,
              double* __restrict__ out, double alpha, int add) {
    pdl_trigger();
    const int gid = blockIdx.x * 8 + (threadIdx.x >> 5);
    if (gid >= ngroups) return;
    const int lane = threadIdx.x & 31;
    const TGroup g = groups[gid];
    pdl_wait();
    if (lane >= int(g.nc)) return;
    double s = 0.0;
    for (uint32_t i = 0; i < g.nslots; ++i) s += part[size_t(g.slot0 + i) * 32 + lane];
    double* o = out + g.out + lane;
    if (add) *o += alpha * s;
    else *o = s;
}

}  // namespace hlrc
