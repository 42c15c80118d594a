// Device assembly of H-matrix leaves (see host/build_gpu.hpp).
//
//   dense leaves : one CTA per leaf evaluates the kernel function
//   ACA          : one CTA per admissible leaf, the steps of the host ACA
//                  (approx/aca.hh:118-225, 328-436; host/build.cpp aca()):
//                  residual column at the pivot column, pivot row = argmax
//                  |column| (zero test eps_mach^2), column / pivot, residual
//                  row, next column = argmax |row| over unused columns,
//                  stop when |u||v| < eps |U V^T|_F (estimate), keeping that
//                  pair.  Block-wide reductions replace the sequential loops.
//   truncation   : one CTA per leaf, as approx/svd.hh:94-209 (host/build.cpp
//                  truncate()): Householder QR of both factors, one-sided
//                  Jacobi SVD of R_U R_V^T (round-robin pair order),
//                  sigma_i > eps sigma_0 kept, Q factors applied to the kept
//                  singular vectors, singular values multiplied into the
//                  factor with fewer rows.
// The two phases are separate launches: the ACA ranks size the output.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "common.hpp"
#include "host/build_gpu.hpp"

namespace hlrc {
namespace {

constexpr int BT = 256;   // threads per CTA of the construction kernels
constexpr int BW = BT / 32;

struct DevProblem {
    int kind, dim;
    const double* pts;
    const double* wts;
    double ell, nugget, h;
};

__device__ __forceinline__ double dev_entry(const DevProblem& P, int64_t i, int64_t j) {
    if (P.kind == HLRC_PROBLEM_LOG1D) {
        if (i == j) return P.h * (log(P.h) - 1.0);
        return log(fabs(P.pts[i] - P.pts[j]));
    }
    const double* a = P.pts + 3 * i;
    const double* b = P.pts + 3 * j;
    const double dx = a[0] - b[0], dy = a[1] - b[1], dz = a[2] - b[2];
    const double r = sqrt(dx * dx + dy * dy + dz * dz);
    if (P.kind == HLRC_PROBLEM_EXP3D) {
        double v = exp(-r / P.ell);
        if (i == j) v += P.nugget;
        return v;
    }
    // LAPLACE_SPH
    if (i == j) return 0.5 * sqrt(P.wts[i]) / sqrt(M_PI);
    return P.wts[j] / (4.0 * M_PI * r);
}

struct DenseTask {
    int64_t row0, col0, off;
    int32_t m, n;
};

struct LrTask {
    int64_t row0, col0;
    int32_t m, n;
    int32_t cap;        // ACA columns available (<= min(m, n, GPU_ACA_MAX_RANK))
    int32_t k;          // ACA rank (written by k_aca)
    int64_t su, sv;     // ACA factors in the scratch (m x cap, n x cap)
    int64_t ou, ov, os; // output U (m x k), V (n x k), singular values (k)
    int64_t sm;         // small scratch: R_U, R_V, M, J (k x k each), beta_U, beta_V (k each)
    int32_t kk;         // truncated rank (written by k_trunc)
    int32_t pad;
};

// ---------------------------------------------------------- reductions
// sum over the CTA, every thread gets the result; fixed order
__device__ double block_sum(double v, double* red) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __syncthreads();
    if (lane == 0) red[w] = v;
    __syncthreads();
    double s = 0.0;
    for (int i = 0; i < BW; ++i) s += red[i];
    return s;
}

// (|value| largest, index smallest among equal) over the CTA; idx < 0 for none
__device__ void block_argmax(double& av, int& idx, double* redv, int* redi) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int o = 16; o > 0; o >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, av, o);
        const int oi = __shfl_xor_sync(0xffffffffu, idx, o);
        if (oi >= 0 && (idx < 0 || ov > av || (ov == av && oi < idx))) { av = ov; idx = oi; }
    }
    __syncthreads();
    if (lane == 0) { redv[w] = av; redi[w] = idx; }
    __syncthreads();
    av = -1.0;
    idx = -1;
    for (int i = 0; i < BW; ++i)
        if (redi[i] >= 0 && (idx < 0 || redv[i] > av || (redv[i] == av && redi[i] < idx))) { av = redv[i]; idx = redi[i]; }
}

// ---------------------------------------------------------- dense leaves
__global__ void __launch_bounds__(BT) k_dense(const DenseTask* __restrict__ tasks, DevProblem P, double* __restrict__ out) {
    const DenseTask t = tasks[blockIdx.x];
    const int64_t tot = int64_t(t.m) * t.n;
    for (int64_t e = threadIdx.x; e < tot; e += BT) {
        const int64_t i = e % t.m, j = e / t.m;
        out[t.off + e] = dev_entry(P, t.row0 + i, t.col0 + j);
    }
}

// ------------------------------------------------------------------ ACA
// dynamic shared memory: cap doubles (pivot row / column coefficients) and
// ceil(n / 32) words (used columns)
__global__ void __launch_bounds__(BT) k_aca(LrTask* __restrict__ tasks, DevProblem P, double* __restrict__ scr,
                                            double eps, int* __restrict__ err) {
    extern __shared__ double dyn[];
    __shared__ double redv[BW];
    __shared__ int redi[BW];
    __shared__ double du[GPU_ACA_MAX_RANK], dv[GPU_ACA_MAX_RANK];
    LrTask& T = tasks[blockIdx.x];
    const int m = T.m, n = T.n, cap = T.cap;
    double* U = scr + T.su;   // m x cap
    double* V = scr + T.sv;   // n x cap
    double* coef = dyn;       // cap
    uint32_t* used = reinterpret_cast<uint32_t*>(dyn + cap);
    const int nw = (n + 31) / 32;
    for (int i = threadIdx.x; i < nw; i += BT) used[i] = 0u;
    const double zero_val = 4.930380657631324e-32;   // eps_mach^2 (2^-104)
    const int max_rank = min(m, n);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int k = 0, pc = 0;
    double norm_M = 0.0;
    bool overflow = false;
    __syncthreads();
    for (int it = 0; it < max_rank; ++it) {
        if (k >= cap) { overflow = true; break; }
        if (threadIdx.x == 0) used[pc >> 5] |= 1u << (pc & 31);
        for (int l = threadIdx.x; l < k; l += BT) coef[l] = V[int64_t(l) * n + pc];
        __syncthreads();
        // residual column at pc into U(:, k); pivot row
        double* col = U + int64_t(k) * m;
        double amax = -1.0;
        int pr = -1;
        for (int i = threadIdx.x; i < m; i += BT) {
            double c = dev_entry(P, T.row0 + i, T.col0 + pc);
            for (int l = 0; l < k; ++l) c -= coef[l] * U[int64_t(l) * m + i];
            col[i] = c;
            if (fabs(c) > amax) { amax = fabs(c); pr = i; }
        }
        block_argmax(amax, pr, redv, redi);
        if (pr < 0) break;             // no comparable entry (NaN column)
        const double maxv = col[pr];   // written by the thread that owns pr, visible after the barriers
        // every thread has read the pivot before its owner scales it below
        __syncthreads();
        if (fabs(maxv) <= zero_val) break;
        const double inv = 1.0 / maxv;
        double ss = 0.0;
        for (int i = threadIdx.x; i < m; i += BT) {
            const double c = col[i] * inv;
            col[i] = c;
            ss += c * c;
        }
        const double ncol = block_sum(ss, redv);
        for (int l = threadIdx.x; l < k; l += BT) coef[l] = U[int64_t(l) * m + pr];
        __syncthreads();
        // residual row at pr into V(:, k); next column over the unused ones
        double* row = V + int64_t(k) * n;
        double rmax = 0.0;
        int mj = -1;
        ss = 0.0;
        for (int j = threadIdx.x; j < n; j += BT) {
            double r = dev_entry(P, T.row0 + pr, T.col0 + j);
            for (int l = 0; l < k; ++l) r -= coef[l] * V[int64_t(l) * n + j];
            row[j] = r;
            ss += r * r;
            const bool un = !(used[j >> 5] & (1u << (j & 31)));
            if (un && fabs(r) > rmax) { rmax = fabs(r); mj = j; }
        }
        const double nrow = block_sum(ss, redv);
        if (mj < 0) rmax = -1.0;
        block_argmax(rmax, mj, redv, redi);
        if (mj < 0) {   // no unused column with a nonzero entry: the first unused one
            int first = -1;
            for (int j = threadIdx.x; j < n; j += BT)
                if (!(used[j >> 5] & (1u << (j & 31)))) { first = j; break; }
            double z = 0.0;
            if (first < 0) z = -1.0;
            block_argmax(z, first, redv, redi);
            mj = first;
        }
        const double norm_i = sqrt(ncol) * sqrt(nrow);
        if (norm_i < eps * norm_M) {
            ++k;
            break;
        }
        // |U V^T|_F^2 update: 2 sum_l (u_l . col)(v_l . row)
        for (int l = w; l < k; l += BW) {
            double a = 0.0, b = 0.0;
            for (int i = lane; i < m; i += 32) a += U[int64_t(l) * m + i] * col[i];
            for (int j = lane; j < n; j += 32) b += V[int64_t(l) * n + j] * row[j];
            for (int o = 16; o > 0; o >>= 1) {
                a += __shfl_xor_sync(0xffffffffu, a, o);
                b += __shfl_xor_sync(0xffffffffu, b, o);
            }
            if (lane == 0) { du[l] = a; dv[l] = b; }
        }
        __syncthreads();
        double upd = norm_i * norm_i;
        for (int l = 0; l < k; ++l) upd += 2.0 * du[l] * dv[l];
        norm_M = sqrt(norm_M * norm_M + fabs(upd));
        ++k;
        if (mj < 0) break;
        pc = mj;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        T.k = k;
        if (overflow) atomicOr(err, 1);
    }
}

// ------------------------------------------------------------ truncation
// Householder QR of A (rows x k, ld = rows) in place: column j keeps R's
// entries above the diagonal and below it the reflector v_j (v_j[0] on the
// diagonal); R(j, j) goes to R (k x k, column-major) with the rest of R;
// beta_j = 2 / |v_j|^2 (0: no reflection).
__device__ void house_qr(double* A, int rows, int k, double* R, double* beta, double* red) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int j = 0; j < k; ++j) {
        double* x = A + int64_t(j) * rows + j;
        const int len = rows - j;
        double ss = 0.0;
        for (int i = threadIdx.x; i < len; i += BT) ss += x[i] * x[i];
        ss = block_sum(ss, red);
        const double x0 = x[0];
        const double nx = sqrt(ss);
        double b = 0.0, alpha = 0.0;
        if (nx > 0.0) {
            alpha = x0 > 0 ? -nx : nx;
            const double v0 = x0 - alpha;
            const double vn2 = ss - x0 * x0 + v0 * v0;
            b = vn2 > 0 ? 2.0 / vn2 : 0.0;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            if (nx > 0.0) x[0] = x0 - alpha;
            beta[j] = b;
            R[int64_t(j) * k + j] = alpha;
        }
        __syncthreads();
        if (b != 0.0) {
            for (int c = j + 1 + w; c < k; c += BW) {
                double* y = A + int64_t(c) * rows + j;
                double s = 0.0;
                for (int i = lane; i < len; i += 32) s += x[i] * y[i];
                for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
                s *= b;
                for (int i = lane; i < len; i += 32) y[i] -= s * x[i];
            }
        }
        __syncthreads();
    }
    // R above the diagonal, zeros below
    for (int e = threadIdx.x; e < k * k; e += BT) {
        const int i = e % k, c = e / k;
        if (i < c) R[e] = A[int64_t(c) * rows + i];
        else if (i > c) R[e] = 0.0;
    }
    __syncthreads();
}

// B (rows x nc, ld rows) := Q B, Q = H_0 ... H_{k-1} from house_qr
__device__ void apply_q(const double* A, int rows, int k, const double* beta, double* B, int nc) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int j = k - 1; j >= 0; --j) {
        const double b = beta[j];
        if (b != 0.0) {
            const double* v = A + int64_t(j) * rows + j;
            const int len = rows - j;
            for (int c = w; c < nc; c += BW) {
                double* y = B + int64_t(c) * rows + j;
                double s = 0.0;
                for (int i = lane; i < len; i += 32) s += v[i] * y[i];
                for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
                s *= b;
                for (int i = lane; i < len; i += 32) y[i] -= s * v[i];
            }
        }
        __syncthreads();
    }
}

// One-sided Jacobi on the columns of M (k x k): M J = U S with J
// orthogonal (accumulated in J); round-robin pairs, a warp per pair.
__device__ void jacobi(double* M, double* J, int k, int* cnt) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int e = threadIdx.x; e < k * k; e += BT) J[e] = (e % k == e / k) ? 1.0 : 0.0;
    const int K = k + (k & 1);            // players (a dummy when k is odd)
    const int npair = K / 2;
    __syncthreads();
    for (int sweep = 0; sweep < 80; ++sweep) {
        if (threadIdx.x == 0) *cnt = 0;
        __syncthreads();
        int rot = 0;
        for (int r = 0; r < K - 1; ++r) {
            for (int pi = w; pi < npair; pi += BW) {
                int p = pi == 0 ? K - 1 : (K - 1 - pi + r) % (K - 1);
                int q = (pi + r) % (K - 1);
                if (p > q) { const int t = p; p = q; q = t; }
                if (q >= k) continue;     // the dummy
                double* mp = M + int64_t(p) * k;
                double* mq = M + int64_t(q) * k;
                double a = 0.0, b = 0.0, g = 0.0;
                for (int i = lane; i < k; i += 32) {
                    a += mp[i] * mp[i];
                    b += mq[i] * mq[i];
                    g += mp[i] * mq[i];
                }
                for (int o = 16; o > 0; o >>= 1) {
                    a += __shfl_xor_sync(0xffffffffu, a, o);
                    b += __shfl_xor_sync(0xffffffffu, b, o);
                    g += __shfl_xor_sync(0xffffffffu, g, o);
                }
                if (a == 0.0 || b == 0.0 || fabs(g) <= 1e-15 * sqrt(a * b)) continue;
                ++rot;
                const double zeta = (b - a) / (2.0 * g);
                const double t = (zeta >= 0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
                const double c = 1.0 / sqrt(1.0 + t * t), s = c * t;
                double* jp = J + int64_t(p) * k;
                double* jq = J + int64_t(q) * k;
                for (int i = lane; i < k; i += 32) {
                    const double x = mp[i], y = mq[i];
                    mp[i] = c * x - s * y;
                    mq[i] = s * x + c * y;
                    const double u = jp[i], v = jq[i];
                    jp[i] = c * u - s * v;
                    jq[i] = s * u + c * v;
                }
            }
            __syncthreads();
        }
        if (lane == 0 && rot > 0) atomicAdd(cnt, rot);
        __syncthreads();
        const int total = *cnt;
        __syncthreads();
        if (total == 0) break;
    }
}

__global__ void __launch_bounds__(BT) k_trunc(LrTask* __restrict__ tasks, const double* __restrict__ scr_c,
                                              double* __restrict__ scr, double* __restrict__ small,
                                              double* __restrict__ out, double eps) {
    __shared__ double red[BW];
    __shared__ double sig[GPU_ACA_MAX_RANK];
    __shared__ int ord[GPU_ACA_MAX_RANK];
    __shared__ int cnt;
    (void)scr_c;
    LrTask& T = tasks[blockIdx.x];
    const int m = T.m, n = T.n, k = T.k;
    if (k == 0) {
        if (threadIdx.x == 0) T.kk = 0;
        return;
    }
    double* U = scr + T.su;
    double* V = scr + T.sv;
    double* RU = small + T.sm;
    double* RV = RU + int64_t(k) * k;
    double* M = RV + int64_t(k) * k;
    double* J = M + int64_t(k) * k;
    double* bu = J + int64_t(k) * k;
    double* bv = bu + k;
    house_qr(U, m, k, RU, bu, red);
    house_qr(V, n, k, RV, bv, red);
    // M = R_U R_V^T
    for (int e = threadIdx.x; e < k * k; e += BT) {
        const int i = e % k, j = e / k;
        double s = 0.0;
        for (int l = max(i, j); l < k; ++l) s += RU[int64_t(l) * k + i] * RV[int64_t(l) * k + j];
        M[e] = s;
    }
    __syncthreads();
    jacobi(M, J, k, &cnt);
    // singular values and their descending order (stable)
    for (int j = threadIdx.x; j < k; j += BT) {
        double s = 0.0;
        for (int i = 0; i < k; ++i) s += M[int64_t(j) * k + i] * M[int64_t(j) * k + i];
        sig[j] = sqrt(s);
    }
    __syncthreads();
    for (int j = threadIdx.x; j < k; j += BT) {
        int rk = 0;
        for (int i = 0; i < k; ++i) rk += (sig[i] > sig[j] || (sig[i] == sig[j] && i < j)) ? 1 : 0;
        ord[rk] = j;
    }
    __syncthreads();
    const double smax = sig[ord[0]];
    int kk = 0;
    if (smax > 0.0)
        while (kk < k && sig[ord[kk]] > eps * smax) ++kk;
    double* W = out + T.ou;   // m x kk
    double* X = out + T.ov;   // n x kk
    // W = Q_U [U~_kk; 0], X = Q_V [J_kk; 0]
    for (int64_t e = threadIdx.x; e < int64_t(m) * kk; e += BT) {
        const int i = int(e % m), c = int(e / m);
        const int j = ord[c];
        W[e] = i < k ? M[int64_t(j) * k + i] / sig[j] : 0.0;
    }
    for (int64_t e = threadIdx.x; e < int64_t(n) * kk; e += BT) {
        const int i = int(e % n), c = int(e / n);
        X[e] = i < k ? J[int64_t(ord[c]) * k + i] : 0.0;
    }
    __syncthreads();
    apply_q(U, m, k, bu, W, kk);
    apply_q(V, n, k, bv, X, kk);
    // singular values into the factor with fewer rows
    double* Tm = m < n ? W : X;
    const int tr = m < n ? m : n;
    for (int64_t e = threadIdx.x; e < int64_t(tr) * kk; e += BT) Tm[e] *= sig[ord[int(e / tr)]];
    for (int c = threadIdx.x; c < kk; c += BT) out[T.os + c] = sig[ord[c]];
    if (threadIdx.x == 0) T.kk = kk;
}

struct DevBuf {
    void* p = nullptr;
    ~DevBuf() { if (p) cudaFree(p); }
};

}  // namespace

hlrc_status gpu_copy_to_host(double* dst, const double* src, int64_t n) {
    if (n <= 0) return HLRC_OK;
    const cudaError_t e = cudaMemcpy(dst, src, size_t(n) * sizeof(double), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return fail(HLRC_ERR_CUDA, "device-to-host copy of leaf data: %s", cudaGetErrorString(e));
    return HLRC_OK;
}

hlrc_status gpu_free(void* p) {
    if (p) cudaFree(p);
    return HLRC_OK;
}

hlrc_status gpu_assemble(const GpuProblem& P, std::vector<GpuLeaf>& leaves, double eps, double** arena,
                         int64_t* arena_doubles) {
    *arena = nullptr;
    *arena_doubles = 0;
    auto cerr = [](cudaError_t e, const char* what) {
        cudaGetLastError();
        return fail(HLRC_ERR_CUDA, "device construction: %s: %s", what, cudaGetErrorString(e));
    };
    cudaError_t e;
    // points and weights
    DevBuf dpts, dwts;
    const size_t npts = size_t(P.n) * size_t(P.dim);
    if ((e = cudaMalloc(&dpts.p, std::max<size_t>(8, npts * 8))) != cudaSuccess) return cerr(e, "points");
    if ((e = cudaMemcpy(dpts.p, P.pts, npts * 8, cudaMemcpyHostToDevice)) != cudaSuccess) return cerr(e, "points");
    if (P.wts) {
        if ((e = cudaMalloc(&dwts.p, size_t(P.n) * 8)) != cudaSuccess) return cerr(e, "weights");
        if ((e = cudaMemcpy(dwts.p, P.wts, size_t(P.n) * 8, cudaMemcpyHostToDevice)) != cudaSuccess)
            return cerr(e, "weights");
    }
    const DevProblem DP{P.kind, P.dim, static_cast<const double*>(dpts.p), static_cast<const double*>(dwts.p),
                        P.ell, P.nugget, P.h};
    // task lists: dense leaves go straight to their final place, admissible
    // ones to the ACA scratch; larger leaves first (load balance)
    std::vector<DenseTask> dt;
    std::vector<LrTask> lt;
    std::vector<size_t> lr_leaf;
    int64_t dense_total = 0, scratch = 0, max_n = 1;
    for (size_t i = 0; i < leaves.size(); ++i) {
        GpuLeaf& L = leaves[i];
        if (L.nrows <= 0 || L.ncols <= 0) { L.rank = 0; continue; }
        if (L.nrows >= (int64_t(1) << 31) || L.ncols >= (int64_t(1) << 31))
            return fail(HLRC_ERR_SHAPE, "device construction: leaf dimension above 2^31");
        if (L.kind == HLRC_LEAF_DENSE) {
            L.d = dense_total;
            dt.push_back(DenseTask{L.row0, L.col0, dense_total, int32_t(L.nrows), int32_t(L.ncols)});
            dense_total += L.nrows * L.ncols;
        } else {
            LrTask t{};
            t.row0 = L.row0; t.col0 = L.col0;
            t.m = int32_t(L.nrows); t.n = int32_t(L.ncols);
            t.cap = int32_t(std::min<int64_t>({L.nrows, L.ncols, int64_t(GPU_ACA_MAX_RANK)}));
            t.su = scratch;
            scratch += L.nrows * t.cap;
            t.sv = scratch;
            scratch += L.ncols * t.cap;
            max_n = std::max<int64_t>(max_n, L.ncols);
            lt.push_back(t);
            lr_leaf.push_back(i);
        }
    }
    std::vector<size_t> ord(lt.size());
    for (size_t i = 0; i < ord.size(); ++i) ord[i] = i;
    std::stable_sort(ord.begin(), ord.end(), [&](size_t a, size_t b) {
        return int64_t(lt[a].m) * lt[a].n > int64_t(lt[b].m) * lt[b].n;
    });
    {
        std::vector<LrTask> lt2(lt.size());
        std::vector<size_t> leaf2(lt.size());
        for (size_t i = 0; i < ord.size(); ++i) { lt2[i] = lt[ord[i]]; leaf2[i] = lr_leaf[ord[i]]; }
        lt.swap(lt2);
        lr_leaf.swap(leaf2);
    }
    DevBuf dout_dense, dscr, derr, dtasks, ddense;
    // phase 1: ACA into the scratch (and the dense leaves into their own buffer)
    if ((e = cudaMalloc(&derr.p, sizeof(int))) != cudaSuccess) return cerr(e, "error flag");
    if ((e = cudaMemset(derr.p, 0, sizeof(int))) != cudaSuccess) return cerr(e, "error flag");
    if (!lt.empty()) {
        if ((e = cudaMalloc(&dscr.p, size_t(std::max<int64_t>(1, scratch)) * 8)) != cudaSuccess)
            return cerr(e, "ACA scratch");
        if ((e = cudaMalloc(&dtasks.p, lt.size() * sizeof(LrTask))) != cudaSuccess) return cerr(e, "tasks");
        if ((e = cudaMemcpy(dtasks.p, lt.data(), lt.size() * sizeof(LrTask), cudaMemcpyHostToDevice)) != cudaSuccess)
            return cerr(e, "tasks");
        const size_t smem = size_t(GPU_ACA_MAX_RANK) * 8 + size_t((max_n + 31) / 32) * 4;
        if (smem > 48 * 1024 &&
            (e = cudaFuncSetAttribute(k_aca, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem))) != cudaSuccess)
            return cerr(e, "ACA shared memory");
        k_aca<<<unsigned(lt.size()), BT, smem>>>(static_cast<LrTask*>(dtasks.p), DP, static_cast<double*>(dscr.p), eps,
                                                 static_cast<int*>(derr.p));
        if ((e = cudaGetLastError()) != cudaSuccess) return cerr(e, "ACA launch");
        if ((e = cudaMemcpy(lt.data(), dtasks.p, lt.size() * sizeof(LrTask), cudaMemcpyDeviceToHost)) != cudaSuccess)
            return cerr(e, "ACA");
        int flag = 0;
        if ((e = cudaMemcpy(&flag, derr.p, sizeof(int), cudaMemcpyDeviceToHost)) != cudaSuccess) return cerr(e, "ACA");
        if (flag) return fail(HLRC_ERR_SHAPE, "device construction: an ACA did not converge within rank %d",
                              GPU_ACA_MAX_RANK);
    }
    // phase 2: the output arena (dense leaves, U, V, singular values at the
    // ACA ranks) and the small scratch of the truncation
    int64_t total = dense_total, small = 0;
    for (LrTask& t : lt) {
        t.ou = total; total += int64_t(t.m) * t.k;
        t.ov = total; total += int64_t(t.n) * t.k;
        t.os = total; total += t.k;
        t.sm = small; small += 4 * int64_t(t.k) * t.k + 2 * int64_t(t.k);
    }
    double* out = nullptr;
    if ((e = cudaMalloc(&out, size_t(std::max<int64_t>(1, total)) * 8)) != cudaSuccess) return cerr(e, "leaf arena");
    DevBuf own_out;
    own_out.p = out;
    if (!dt.empty()) {
        if ((e = cudaMalloc(&ddense.p, dt.size() * sizeof(DenseTask))) != cudaSuccess) return cerr(e, "dense tasks");
        if ((e = cudaMemcpy(ddense.p, dt.data(), dt.size() * sizeof(DenseTask), cudaMemcpyHostToDevice)) != cudaSuccess)
            return cerr(e, "dense tasks");
        k_dense<<<unsigned(dt.size()), BT>>>(static_cast<const DenseTask*>(ddense.p), DP, out);
        if ((e = cudaGetLastError()) != cudaSuccess) return cerr(e, "dense launch");
    }
    if (!lt.empty()) {
        DevBuf dsmall;
        if ((e = cudaMalloc(&dsmall.p, size_t(std::max<int64_t>(1, small)) * 8)) != cudaSuccess)
            return cerr(e, "truncation scratch");
        if ((e = cudaMemcpy(dtasks.p, lt.data(), lt.size() * sizeof(LrTask), cudaMemcpyHostToDevice)) != cudaSuccess)
            return cerr(e, "tasks");
        k_trunc<<<unsigned(lt.size()), BT>>>(static_cast<LrTask*>(dtasks.p), static_cast<const double*>(dscr.p),
                                             static_cast<double*>(dscr.p), static_cast<double*>(dsmall.p), out, eps);
        if ((e = cudaGetLastError()) != cudaSuccess) return cerr(e, "truncation launch");
        if ((e = cudaMemcpy(lt.data(), dtasks.p, lt.size() * sizeof(LrTask), cudaMemcpyDeviceToHost)) != cudaSuccess)
            return cerr(e, "truncation");
    }
    if ((e = cudaDeviceSynchronize()) != cudaSuccess) return cerr(e, "construction");
    for (size_t i = 0; i < lt.size(); ++i) {
        GpuLeaf& L = leaves[lr_leaf[i]];
        L.rank = lt[i].kk;
        L.u = lt[i].ou;
        L.v = lt[i].ov;
        L.s = lt[i].os;
    }
    own_out.p = nullptr;
    *arena = out;
    *arena_doubles = total;
    return HLRC_OK;
}

}  // namespace hlrc
