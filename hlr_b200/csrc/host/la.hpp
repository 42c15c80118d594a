// Small dense linear algebra for the host-side matrix construction:
// column-major matrices, Householder QR with explicit Q and one-sided Jacobi
// SVD.  HLR reaches LAPACK through HLIBpro's BLAS layer
// (include/hlr/arith/blas.hh: qr, svd); neither HLIBpro nor a system LAPACK is
// available, so these are written from the textbook algorithms
// (Householder: Golub & Van Loan 5.2; one-sided Jacobi: Hestenes 1958,
// Demmel & Veselic 1992).
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <vector>

namespace hlrc {

struct Mat {
    int64_t m = 0, n = 0;
    std::vector<double> a;
    Mat() = default;
    Mat(int64_t m_, int64_t n_) : m(m_), n(n_), a(size_t(m_ * n_), 0.0) {}
    double&       operator()(int64_t i, int64_t j)       { return a[size_t(i + j * m)]; }
    const double& operator()(int64_t i, int64_t j) const { return a[size_t(i + j * m)]; }
    double*       col(int64_t j)       { return a.data() + j * m; }
    const double* col(int64_t j) const { return a.data() + j * m; }
};

inline double dot(const double* x, const double* y, int64_t n) {
    double s = 0;
    for (int64_t i = 0; i < n; ++i) s += x[i] * y[i];
    return s;
}
inline double nrm2(const double* x, int64_t n) {
    // scaled to avoid overflow/underflow of the squares
    double scale = 0, ssq = 1;
    for (int64_t i = 0; i < n; ++i) {
        if (x[i] != 0) {
            double ax = std::fabs(x[i]);
            if (scale < ax) { ssq = 1 + ssq * (scale / ax) * (scale / ax); scale = ax; }
            else            { ssq += (ax / scale) * (ax / scale); }
        }
    }
    return scale * std::sqrt(ssq);
}

// C = A * B  (A: m x k, B: k x n)
inline Mat prod(const Mat& A, const Mat& B) {
    Mat C(A.m, B.n);
    for (int64_t j = 0; j < B.n; ++j)
        for (int64_t l = 0; l < A.n; ++l) {
            const double b = B(l, j);
            if (b == 0) continue;
            const double* a = A.col(l);
            double* c = C.col(j);
            for (int64_t i = 0; i < A.m; ++i) c[i] += a[i] * b;
        }
    return C;
}
// C = A^T * B  (A: k x m, B: k x n)
inline Mat prod_tn(const Mat& A, const Mat& B) {
    Mat C(A.n, B.n);
    for (int64_t j = 0; j < B.n; ++j)
        for (int64_t i = 0; i < A.n; ++i) C(i, j) = dot(A.col(i), B.col(j), A.m);
    return C;
}
// C = A * B^T  (A: m x k, B: n x k)
inline Mat prod_nt(const Mat& A, const Mat& B) {
    Mat C(A.m, B.m);
    for (int64_t l = 0; l < A.n; ++l)
        for (int64_t j = 0; j < B.m; ++j) {
            const double b = B(j, l);
            if (b == 0) continue;
            const double* a = A.col(l);
            double* c = C.col(j);
            for (int64_t i = 0; i < A.m; ++i) c[i] += a[i] * b;
        }
    return C;
}

// Householder QR of A (m x n, m >= n): A = Q R, Q (m x n) with orthonormal
// columns (explicit), R (n x n) upper triangular.  A is overwritten by Q.
inline void qr(Mat& A, Mat& R) {
    const int64_t m = A.m, n = A.n;
    R = Mat(n, n);
    if (n == 0) return;
    std::vector<double> vs(size_t(m * n), 0.0);  // Householder vectors (column j starts at row j)
    std::vector<double> beta(size_t(n), 0.0);
    for (int64_t j = 0; j < n && j < m; ++j) {
        double* x = A.col(j) + j;
        const int64_t len = m - j;
        const double nx = nrm2(x, len);
        double* v = vs.data() + j * m + j;
        if (nx == 0.0) { beta[j] = 0; R(j, j) = 0; for (int64_t i = 0; i < len; ++i) v[i] = 0; continue; }
        const double alpha = (x[0] > 0) ? -nx : nx;
        for (int64_t i = 0; i < len; ++i) v[i] = x[i];
        v[0] -= alpha;
        const double vn2 = dot(v, v, len);
        beta[j] = (vn2 > 0) ? 2.0 / vn2 : 0.0;
        // apply to remaining columns
        for (int64_t c = j; c < n; ++c) {
            double* y = A.col(c) + j;
            const double s = beta[j] * dot(v, y, len);
            for (int64_t i = 0; i < len; ++i) y[i] -= s * v[i];
        }
    }
    for (int64_t j = 0; j < n; ++j)
        for (int64_t i = 0; i <= j && i < m; ++i) R(i, j) = A(i, j);
    // explicit Q: apply reflectors backwards to [I; 0]
    for (int64_t j = 0; j < n; ++j) {
        double* q = A.col(j);
        for (int64_t i = 0; i < m; ++i) q[i] = (i == j) ? 1.0 : 0.0;
    }
    for (int64_t j = std::min(n, m) - 1; j >= 0; --j) {
        const double* v = vs.data() + j * m + j;
        const int64_t len = m - j;
        if (beta[j] == 0) continue;
        for (int64_t c = j; c < n; ++c) {
            double* y = A.col(c) + j;
            const double s = beta[j] * dot(v, y, len);
            for (int64_t i = 0; i < len; ++i) y[i] -= s * v[i];
        }
    }
}

// One-sided Jacobi SVD of A (m x n): A = U diag(S) V^T with S descending.
// U: m x r, V: n x r, r = min(m, n).
inline void svd(const Mat& A, Mat& U, std::vector<double>& S, Mat& V) {
    const bool trans = A.m < A.n;
    Mat W;
    if (!trans) W = A;
    else {
        W = Mat(A.n, A.m);
        for (int64_t j = 0; j < A.n; ++j)
            for (int64_t i = 0; i < A.m; ++i) W(j, i) = A(i, j);
    }
    const int64_t m = W.m, n = W.n;   // m >= n
    Mat Vj(n, n);
    for (int64_t i = 0; i < n; ++i) Vj(i, i) = 1.0;
    const double tol = 1e-15;
    std::vector<double> nrm(static_cast<size_t>(n));
    for (int64_t j = 0; j < n; ++j) nrm[j] = dot(W.col(j), W.col(j), m);
    for (int sweep = 0; sweep < 80; ++sweep) {
        int64_t rotations = 0;
        for (int64_t p = 0; p < n - 1; ++p) {
            for (int64_t q = p + 1; q < n; ++q) {
                const double alpha = nrm[p], beta = nrm[q];
                if (alpha == 0.0 || beta == 0.0) continue;
                const double gamma = dot(W.col(p), W.col(q), m);
                if (std::fabs(gamma) <= tol * std::sqrt(alpha * beta)) continue;
                ++rotations;
                const double zeta = (beta - alpha) / (2.0 * gamma);
                const double t = (zeta >= 0 ? 1.0 : -1.0) / (std::fabs(zeta) + std::sqrt(1.0 + zeta * zeta));
                const double c = 1.0 / std::sqrt(1.0 + t * t), s = c * t;
                double* wp = W.col(p); double* wq = W.col(q);
                for (int64_t i = 0; i < m; ++i) {
                    const double a = wp[i], b = wq[i];
                    wp[i] = c * a - s * b;
                    wq[i] = s * a + c * b;
                }
                double* vp = Vj.col(p); double* vq = Vj.col(q);
                for (int64_t i = 0; i < n; ++i) {
                    const double a = vp[i], b = vq[i];
                    vp[i] = c * a - s * b;
                    vq[i] = s * a + c * b;
                }
                nrm[p] = dot(wp, wp, m);
                nrm[q] = dot(wq, wq, m);
            }
        }
        if (rotations == 0) break;
    }
    std::vector<double> sig(static_cast<size_t>(n));
    for (int64_t j = 0; j < n; ++j) sig[j] = nrm2(W.col(j), m);
    std::vector<int64_t> ord(static_cast<size_t>(n));
    std::iota(ord.begin(), ord.end(), 0);
    std::stable_sort(ord.begin(), ord.end(), [&](int64_t a, int64_t b) { return sig[a] > sig[b]; });
    Mat Uo(m, n), Vo(n, n);
    S.assign(size_t(n), 0.0);
    for (int64_t jj = 0; jj < n; ++jj) {
        const int64_t j = ord[jj];
        S[jj] = sig[j];
        const double inv = sig[j] > 0 ? 1.0 / sig[j] : 0.0;
        for (int64_t i = 0; i < m; ++i) Uo(i, jj) = W(i, j) * inv;
        for (int64_t i = 0; i < n; ++i) Vo(i, jj) = Vj(i, j);
    }
    if (!trans) { U = std::move(Uo); V = std::move(Vo); }
    else        { U = std::move(Vo); V = std::move(Uo); }
}

// Truncation rank for relative precision eps in the spectral norm:
// keep sigma_i > eps * sigma_0 (HLIBpro TTruncAcc::trunc_rank, relative
// precision, restated; approx/accuracy.hh:17-26 aliases it).
inline int64_t trunc_rank(const std::vector<double>& S, double eps) {
    if (S.empty() || S[0] <= 0) return 0;
    const double thr = eps * S[0];
    int64_t k = 0;
    while (k < int64_t(S.size()) && S[k] > thr) ++k;
    return k;
}

}  // namespace hlrc
