// Multi-right-hand-side products: the matrix is streamed once per block of
// MR_RB right-hand sides instead of once per vector.  This file holds the
// block layout helpers, the partial-sum finish and the FP64 kernels (FP64
// tensor cores); the reduced-precision kernels are in kernels_tc.cuh.
//
// Vector operands are row-major blocks (entry (i, r) at i * RB + r), so the
// RB values that multiply one matrix column are contiguous: the caller's
// column-major X is transposed into that form first, and the coefficient
// workspaces (t, uy, partial sums) use it throughout.  Outputs go through
// (row stride, column stride) pairs, so the same kernel writes row-major
// coefficients or the caller's column-major Y.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>

#include "kernels_f64.cuh"
#include "layout.hpp"

namespace hlrc {

constexpr int MR_RB = 8;   // right-hand sides per block (kernels, finish, workspaces)

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

// Finish of the multi-vector tile T-form with a flat thread map: a CTA takes
// gpb (at most FIN_GROUPS, fin_gpb) consecutive groups, and each thread one
// vector of VEC entries of them (output column j, right-hand sides k ..
// k+VEC-1), NR right-hand sides per partial entry.  Slot i of a group holds
// its entries at part[(slot0 + i*nc + j)*NR + k].  Each entry is summed in a
// fixed order: four FP64 accumulators, slot a going to accumulator a mod 4
// when a < (nslots rounded down to a multiple of 4) and to the first
// otherwise, each accumulator taking its slots in increasing order; the
// result is (s0 + s1) + (s2 + s3).  The loads of FIN_BATCH slots are issued
// before their sums, so a short group (a few slots of a few columns, the
// common case) costs one round trip, and the short groups of a CTA fill its
// threads together.  TO_PART writes the sums (as T) to
// part_out[(out + j)*NR + k] (the first level of long outputs); otherwise
// they go to the output map, with alpha/add.  (The one-vector finish,
// k_ttfinish_f64, keeps a warp per output: for one vector that measured
// faster.)
constexpr int FIN_GROUPS = 32;
constexpr int FIN_BATCH = 8;

// Groups per CTA of a finish launch: about 16 CTAs per SM of the 148, so
// that few long groups (the first level) still spread over the GPU.
inline int fin_gpb(int ngroups) {
    constexpr int target = 148 * 16;
    return std::max(1, std::min(FIN_GROUPS, (ngroups + target - 1) / target));
}

template <typename T, int VEC> struct FinVec { using type = T; };
template <> struct FinVec<float, 2> { using type = float2; };
template <> struct FinVec<double, 2> { using type = double2; };

template <int NR, typename T, bool TO_PART>
__global__ void __launch_bounds__(256)
k_ttfinish_flat(const TGroup* __restrict__ groups, int ngroups, int gpb, const T* part, OutMap om, T* part_out,
                double alpha, int add) {
    // 8-byte (FP32 pairs) or 16-byte (FP64 pairs) loads
    constexpr int VEC = NR % 2 == 0 ? 2 : 1;
    constexpr int PER = NR / VEC;   // vectors per column entry
    using V = typename FinVec<T, VEC>::type;
    static_assert(sizeof(V) == VEC * sizeof(T), "vector type");
    static_assert(FIN_BATCH % 4 == 0, "a batch keeps the accumulator of a slot at a mod 4");
    __shared__ TGroup sg[FIN_GROUPS];
    __shared__ uint32_t pre[FIN_GROUPS + 1];
    pdl_trigger();
    const int g0 = int(blockIdx.x) * gpb;
    const int ng = min(gpb, ngroups - g0);
    if (int(threadIdx.x) < ng) sg[threadIdx.x] = groups[g0 + int(threadIdx.x)];
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t acc = 0;
        for (int q = 0; q < ng; ++q) {
            pre[q] = acc;
            acc += sg[q].nc * uint32_t(PER);
        }
        pre[ng] = acc;
    }
    __syncthreads();
    pdl_wait();
    const uint32_t total = pre[ng];
    int lo = 0;   // the group holding item `it` (pre[lo] <= it < pre[lo + 1]); items only move forward
    for (uint32_t it = threadIdx.x; it < total; it += blockDim.x) {
        while (pre[lo + 1] <= it) ++lo;
        const TGroup g = sg[lo];
        const uint32_t e = it - pre[lo];
        const uint32_t j = e / PER;
        const int k = int(e % PER) * VEC;
        if (k >= om.nr) continue;
        const size_t stride = size_t(g.nc) * PER;
        const V* p = reinterpret_cast<const V*>(part + size_t(g.slot0) * NR) + e;
        const uint32_t f4 = g.nslots & ~3u;
        double s[4][VEC] = {};
        for (uint32_t i = 0; i < g.nslots; i += FIN_BATCH) {
            V v[FIN_BATCH];
#pragma unroll
            for (int a = 0; a < FIN_BATCH; ++a)
                if (i + a < g.nslots) v[a] = __ldcs(p + (i + a) * stride);
#pragma unroll
            for (int a = 0; a < FIN_BATCH; ++a) {
                const uint32_t sl = i + a;
                if (sl >= g.nslots) break;
                const T* x = reinterpret_cast<const T*>(&v[a]);
                if (sl < f4) {   // i is a multiple of 4: sl mod 4 == a mod 4
#pragma unroll
                    for (int q = 0; q < VEC; ++q) s[a & 3][q] += double(x[q]);
                } else {
#pragma unroll
                    for (int q = 0; q < VEC; ++q) s[0][q] += double(x[q]);
                }
            }
        }
#pragma unroll
        for (int q = 0; q < VEC; ++q) {
            const double r = (s[0][q] + s[1][q]) + (s[2][q] + s[3][q]);
            if constexpr (TO_PART) {
                part_out[size_t(g.out + j) * NR + k + q] = T(r);
            } else {
                if (k + q >= om.nr) break;
                double* o = om.base + int64_t(g.out + j) * om.rs + int64_t(k + q) * om.cs;
                if (add) *o += alpha * r;
                else *o = r;
            }
        }
    }
}

// ------------------------------------------------------ FP64 tensor cores
// The same two forms on FP64 tensor cores (mma.sync m8n8k4, FP64 products
// and sums), all MR_RB vectors in one launch.  A lane's 16-byte load is two
// consecutive rows of one column; the contraction / output rows of the MMA
// are mapped onto them as follows.
//   N-form: contraction = chunk columns 4kt + t; m-tile i = 2p + b takes
//     tile row 16p + 2g + b as its fragment row g.
//   tile T-form: contraction = tile rows, k-step s = 2j + b maps fragment
//     k = t to row 8j + 2t + b; the output rows are the chunk's 8 columns.

__device__ __forceinline__ void dmma(double (&d)[2], double a, double b) {
    asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
        : "+d"(d[0]), "+d"(d[1])
        : "d"(a), "d"(b));
}

// Both kernels keep two operand sets in registers: the loads of chunk
// c + W are in flight while chunk c is multiplied, and chunk descriptors are
// read two chunks ahead.
template <int W>
__global__ void __launch_bounds__(W * 32, 2)
k_nform_dmma(const NSeg* __restrict__ segs, const NChunk* __restrict__ chunks, const double* __restrict__ A,
             const double* __restrict__ vx, const double* __restrict__ vt, OutMap om, double alpha, int add) {
    __shared__ double red[W][TILE][MR_RB];
    const NSeg sg = segs[blockIdx.x];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, t = lane & 3;
    // acc[2p + b]: tile row 16p + 2g + b, right-hand sides 2t, 2t+1
    double acc[8][2];
#pragma unroll
    for (int i = 0; i < 8; ++i) acc[i][0] = acc[i][1] = 0.0;
    // operands of one chunk: k-step kt = column 4kt + t; m[kt][p] = rows
    // 16p + 2g, +1; b[kt] = vector entry of that column, right-hand side g
    auto issue = [&](const NChunk& q, double2 (&m)[2][4], double (&b)[2]) {
        const double* v = (q.v_off & VEC_T) ? vt + size_t(q.v_off & ~VEC_T) * MR_RB : vx + size_t(q.v_off) * MR_RB;
        const double* a = A + q.a_off;
#pragma unroll
        for (int kt = 0; kt < 2; ++kt) {
            const int col = 4 * kt + t;
            const bool okc = col < q.nc;
            b[kt] = okc ? __ldg(v + size_t(col) * MR_RB + g) : 0.0;
#pragma unroll
            for (int p = 0; p < 4; ++p) {
                const int row = 16 * p + 2 * g;
                m[kt][p] = (okc && row < sg.ld) ? ld_stream(a + size_t(col) * sg.ld + row) : make_double2(0.0, 0.0);
            }
        }
    };
    auto compute = [&](const double2 (&m)[2][4], const double (&b)[2]) {
#pragma unroll
        for (int kt = 0; kt < 2; ++kt)
#pragma unroll
            for (int p = 0; p < 4; ++p) {
                dmma(acc[2 * p], m[kt][p].x, b[kt]);
                dmma(acc[2 * p + 1], m[kt][p].y, b[kt]);
            }
    };
    uint32_t c = sg.cb + warp;
    if (c < sg.ce) {
        const NChunk none{0, 0, 0, 0};
        double2 mA[2][4], mB[2][4];
        double bA[2], bB[2];
        issue(chunks[c], mA, bA);
        NChunk qn = c + W < sg.ce ? chunks[c + W] : none;
        for (;;) {
            const bool hasB = c + W < sg.ce;
            const NChunk qnn = c + 2 * W < sg.ce ? chunks[c + 2 * W] : none;
            if (hasB) issue(qn, mB, bB);
            compute(mA, bA);
            if (!hasB) break;
            c += W;
            const bool hasA = c + W < sg.ce;
            const NChunk q3 = c + 2 * W < sg.ce ? chunks[c + 2 * W] : none;
            if (hasA) issue(qnn, mA, bA);
            compute(mB, bB);
            if (!hasA) break;
            c += W;
            qn = q3;
        }
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int row = 16 * (i >> 1) + 2 * g + (i & 1);
        red[warp][row][2 * t] = acc[i][0];
        red[warp][row][2 * t + 1] = acc[i][1];
    }
    __syncthreads();
    for (int i = threadIdx.x; i < TILE * MR_RB; i += W * 32) {
        const int row = i % TILE, k = i / TILE;
        if (row >= sg.rows || k >= om.nr) continue;
        double s = 0.0;
#pragma unroll
        for (int w = 0; w < W; ++w) s += red[w][row][k];
        double* o = om.base + int64_t(sg.out + row) * om.rs + int64_t(k) * om.cs;
        if (add) *o += alpha * s;
        else *o = s;
    }
}

template <int W>
__global__ void __launch_bounds__(W * 32, 2)
k_ttform_dmma(const TTSeg* __restrict__ segs, const TTChunk* __restrict__ chunks, const double* __restrict__ A,
              const double* __restrict__ vin, OutMap om, double* __restrict__ part, double alpha, int add) {
    const TTSeg sg = segs[blockIdx.x];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, t = lane & 3;
    // x of the lane: rows 8j + 2t + b (j < 8, b < 2), right-hand side g
    double xv[16];
#pragma unroll
    for (int j = 0; j < 8; ++j)
#pragma unroll
        for (int b = 0; b < 2; ++b) {
            const int row = 8 * j + 2 * t + b;
            xv[2 * j + b] = row < sg.rows ? __ldg(vin + size_t(sg.v_off + row) * MR_RB + g) : 0.0;
        }
    // operands of one chunk: column g, rows 8j + 2t, +1
    auto issue = [&](const TTChunk& q, double2 (&m)[8]) {
        const bool okc = g < q.nc;
        const double* a = A + q.a_off + size_t(g) * sg.ld;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int row = 8 * j + 2 * t;
            m[j] = (okc && row < sg.ld) ? ld_stream(a + row) : make_double2(0.0, 0.0);
        }
    };
    auto finish = [&](const TTChunk& q, const double2 (&m)[8]) {
        double d[2] = {0.0, 0.0};
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            dmma(d, m[j].x, xv[2 * j]);
            dmma(d, m[j].y, xv[2 * j + 1]);
        }
        // d[e]: chunk column g, right-hand side 2t + e
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            const int n = 2 * t + e;
            if (g >= q.nc || n >= om.nr) continue;
            if (q.flags & TT_DIRECT) {
                double* o = om.base + int64_t(q.out + g) * om.rs + int64_t(n) * om.cs;
                if (add) *o += alpha * d[e];
                else *o = d[e];
            } else {
                part[size_t(q.out + g) * MR_RB + n] = d[e];
            }
        }
    };
    uint32_t c = sg.cb + warp;
    if (c >= sg.ce) return;
    const TTChunk none{0, 0, 0, 0};
    double2 mA[8], mB[8];
    TTChunk qA = chunks[c];
    issue(qA, mA);
    TTChunk qB = c + W < sg.ce ? chunks[c + W] : none;
    for (;;) {
        const bool hasB = c + W < sg.ce;
        const TTChunk qnn = c + 2 * W < sg.ce ? chunks[c + 2 * W] : none;
        if (hasB) issue(qB, mB);
        finish(qA, mA);
        if (!hasB) break;
        c += W;
        const bool hasA = c + W < sg.ce;
        const TTChunk q3 = c + 2 * W < sg.ce ? chunks[c + 2 * W] : none;
        qA = qnn;
        if (hasA) issue(qA, mA);
        finish(qB, mB);
        if (!hasA) break;
        c += W;
        qB = q3;
    }
}

}  // namespace hlrc
