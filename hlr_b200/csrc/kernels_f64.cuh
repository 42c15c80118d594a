// FP64 batched GEMV kernels of the H / uniform-H product (sm_100a).
//
// Both kernels stream the matrix slabs with 128-bit loads marked
// evict-first (each matrix byte is read exactly once per product) while the
// small vectors x / t stay cache resident.
#pragma once

#include <cuda_runtime.h>

#include "layout.hpp"

namespace hlrc {

__device__ __forceinline__ double2 ld_stream(const double* p) {
    return __ldcs(reinterpret_cast<const double2*>(p));
}

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
    const NSeg sg = segs[blockIdx.x];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int r = 2 * lane;
    const bool active = r < sg.ld;
    double acc0 = 0.0, acc1 = 0.0;
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

// T-form: one warp per unit; lane l owns rows 2l, 2l+1 of every slab and
// keeps NC column partials in registers; one transpose-reduction per unit.
template <int NC>
__global__ void __launch_bounds__(256)
k_tform_f64(const TUnit* __restrict__ units, int nunits, const TSlab* __restrict__ slabs,
            const double* __restrict__ A, const double* __restrict__ vin, double* __restrict__ out,
            double* __restrict__ part, double alpha, int add) {
    const int wid = blockIdx.x * 8 + (threadIdx.x >> 5);
    if (wid >= nunits) return;
    const int lane = threadIdx.x & 31;
    const TUnit u = units[wid];
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
    const TTSeg sg = segs[blockIdx.x];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int r = 2 * lane;
    const bool active = r < sg.ld;
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

// Sums the per-tile partials of multi-tile tile-T-form outputs in tile order.
__global__ void __launch_bounds__(256)
k_ttfinish_f64(const TGroup* __restrict__ groups, int ngroups, const double* __restrict__ part,
               double* __restrict__ out, double alpha, int add) {
    const int gid = blockIdx.x * 8 + (threadIdx.x >> 5);
    if (gid >= ngroups) return;
    const int lane = threadIdx.x & 31;
    const TGroup g = groups[gid];
    for (uint32_t j = lane; j < g.nc; j += 32) {
        // four interleaved partial sums keep four loads in flight; they are
        // combined in a fixed order, so the result is deterministic
        const double* p = part + size_t(g.slot0) + j;
        double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
        uint32_t i = 0;
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
    const int gid = blockIdx.x * 8 + (threadIdx.x >> 5);
    if (gid >= ngroups) return;
    const int lane = threadIdx.x & 31;
    const TGroup g = groups[gid];
    if (lane >= int(g.nc)) return;
    double s = 0.0;
    for (uint32_t i = 0; i < g.nslots; ++i) s += part[size_t(g.slot0 + i) * 32 + lane];
    double* o = out + g.out + lane;
    if (add) *o += alpha * s;
    else *o = s;
}

}  // namespace hlrc
