// Host-side construction of the test matrices: point sets and coefficient
// functions, BSP cluster tree, block tree with standard admissibility, ACA
// with maximum-pivot search, SVD recompression, and shared (uniform) cluster
// bases.  HLR delegates clustering and admissibility to HLIBpro, which is not
// available, so those parts are restated from their documented behaviour:
//
//   cluster tree  : TBSPCTBuilder + TCardBSPPartStrat(adaptive_split_axis)
//                   (programs/common/common.hh:205-277, src/cluster/h.cc:21-55)
//   block tree    : TBCBuilder + TStdGeomAdmCond(eta, use_min_diam)
//                   (programs/common/common.hh:279-323)
//   ACA           : approx::aca with aca_pivot_max (approx/aca.hh:118-225,
//                   328-436), wrapped by bem::aca_lrapx (bem/aca.hh:28-79)
//   recompression : approx::svd_ortho / svd (approx/svd.hh:94-209)
//   uniform bases : tbb/detail/uniform_matrix.hh:328-523 (block row W_t =
//                   [U_i R_i^T], column_basis, S_r = V_t^T U_i, S = S_r S_c^T)
//   point sets    : src/apps/radial.cc:41-50 (randcube, mt19937_64 seed 1)
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <random>
#include <vector>

#include <omp.h>

#include "../common.hpp"
#include "build_gpu.hpp"
#include "la.hpp"

namespace hlrc {

// ---------------------------------------------------------------- problems
struct Problem {
    int kind = 0;
    int dim = 1;
    int64_t n = 0;
    std::vector<double> pts;     // n x dim, internal order
    std::vector<double> wts;     // LAPLACE_SPH: areas, internal order
    std::vector<int64_t> perm;   // internal -> external
    double ell = 0.1, nugget = 0.0, h = 0.0;

    const double* p(int64_t i) const { return pts.data() + i * dim; }

    double entry(int64_t i, int64_t j) const {
        switch (kind) {
            case HLRC_PROBLEM_LOG1D: {
                if (i == j) return h * (std::log(h) - 1.0);
                return std::log(std::fabs(pts[i] - pts[j]));
            }
            case HLRC_PROBLEM_EXP3D: {
                const double* a = p(i); const double* b = p(j);
                const double dx = a[0] - b[0], dy = a[1] - b[1], dz = a[2] - b[2];
                const double r = std::sqrt(dx * dx + dy * dy + dz * dz);
                double v = std::exp(-r / ell);
                if (i == j) v += nugget;
                return v;
            }
            case HLRC_PROBLEM_LAPLACE_SPH: {
                if (i == j) return 0.5 * std::sqrt(wts[i]) / std::sqrt(M_PI);
                const double* a = p(i); const double* b = p(j);
                const double dx = a[0] - b[0], dy = a[1] - b[1], dz = a[2] - b[2];
                const double r = std::sqrt(dx * dx + dy * dy + dz * dz);
                return wts[j] / (4.0 * M_PI * r);
            }
        }
        return 0.0;
    }
};

// uniform double in [0,1) from the raw 64-bit Mersenne twister output; the
// mapping is spelled out so the point sets do not depend on the standard
// library's distribution implementation
static inline double u01(std::mt19937_64& g) { return double(g() >> 11) * 0x1.0p-53; }

static void make_points(const hlrc_problem& pr, std::vector<double>& pts, std::vector<double>& wts, int& dim) {
    std::mt19937_64 g(pr.seed);
    if (pr.kind == HLRC_PROBLEM_LOG1D) {
        dim = 1;
        pts.resize(size_t(pr.n));
        for (int64_t i = 0; i < pr.n; ++i) pts[i] = u01(g);
    } else if (pr.kind == HLRC_PROBLEM_EXP3D) {
        dim = 3;
        pts.resize(size_t(pr.n * 3));
        for (int64_t i = 0; i < pr.n; ++i) {  // x, y, z drawn in this order
            pts[3 * i + 0] = u01(g);
            pts[3 * i + 1] = u01(g);
            pts[3 * i + 2] = u01(g);
        }
    } else {
        // octahedron refined `refine` times, new vertices projected onto the
        // unit sphere after each refinement; flat-triangle centroids and areas
        dim = 3;
        struct Tri { double v[3][3]; };
        std::vector<Tri> tris;
        const double P[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
        const int F[8][3] = {{0, 2, 4}, {2, 1, 4}, {1, 3, 4}, {3, 0, 4}, {2, 0, 5}, {1, 2, 5}, {3, 1, 5}, {0, 3, 5}};
        for (auto& f : F) {
            Tri t;
            for (int k = 0; k < 3; ++k) for (int d = 0; d < 3; ++d) t.v[k][d] = P[f[k]][d];
            tris.push_back(t);
        }
        auto mid = [](const double* a, const double* b, double* o) {
            double s = 0;
            for (int d = 0; d < 3; ++d) { o[d] = 0.5 * (a[d] + b[d]); s += o[d] * o[d]; }
            s = std::sqrt(s);
            for (int d = 0; d < 3; ++d) o[d] /= s;
        };
        for (int r = 0; r < pr.refine; ++r) {
            std::vector<Tri> nt;
            nt.reserve(tris.size() * 4);
            for (auto& t : tris) {
                double m01[3], m12[3], m20[3];
                mid(t.v[0], t.v[1], m01); mid(t.v[1], t.v[2], m12); mid(t.v[2], t.v[0], m20);
                auto push = [&](const double* a, const double* b, const double* c) {
                    Tri u;
                    for (int d = 0; d < 3; ++d) { u.v[0][d] = a[d]; u.v[1][d] = b[d]; u.v[2][d] = c[d]; }
                    nt.push_back(u);
                };
                push(t.v[0], m01, m20);
                push(m01, t.v[1], m12);
                push(m20, m12, t.v[2]);
                push(m01, m12, m20);
            }
            tris.swap(nt);
        }
        const int64_t n = int64_t(tris.size());
        pts.resize(size_t(n * 3));
        wts.resize(static_cast<size_t>(n));
        for (int64_t i = 0; i < n; ++i) {
            const Tri& t = tris[i];
            double e1[3], e2[3];
            for (int d = 0; d < 3; ++d) {
                pts[3 * i + d] = (t.v[0][d] + t.v[1][d] + t.v[2][d]) / 3.0;
                e1[d] = t.v[1][d] - t.v[0][d];
                e2[d] = t.v[2][d] - t.v[0][d];
            }
            const double cx = e1[1] * e2[2] - e1[2] * e2[1];
            const double cy = e1[2] * e2[0] - e1[0] * e2[2];
            const double cz = e1[0] * e2[1] - e1[1] * e2[0];
            wts[i] = 0.5 * std::sqrt(cx * cx + cy * cy + cz * cz);
        }
    }
}

// ---------------------------------------------------------------- clusters
struct Cluster {
    int64_t ofs = 0, size = 0;
    double bmin[3] = {0, 0, 0}, bmax[3] = {0, 0, 0};
    int son[2] = {-1, -1};
    int level = 0;
    bool leaf() const { return son[0] < 0; }
};

struct ClusterTree {
    std::vector<Cluster> cl;   // cl[0] = root
};

static double diam(const Cluster& c, int dim) {
    double s = 0;
    for (int d = 0; d < dim; ++d) { const double e = c.bmax[d] - c.bmin[d]; s += e * e; }
    return std::sqrt(s);
}
static double dist(const Cluster& a, const Cluster& b, int dim) {
    double s = 0;
    for (int d = 0; d < dim; ++d) {
        double g = 0;
        if (a.bmax[d] < b.bmin[d]) g = b.bmin[d] - a.bmax[d];
        else if (b.bmax[d] < a.bmin[d]) g = a.bmin[d] - b.bmax[d];
        s += g * g;
    }
    return std::sqrt(s);
}

// Binary space partitioning with cardinality-balanced splits along the
// longest bounding-box axis; clusters with <= leaf points are leaves.
static void build_ct(const std::vector<double>& pts, int dim, int64_t n, int leaf, ClusterTree& ct,
                     std::vector<int64_t>& perm) {
    perm.resize(static_cast<size_t>(n));
    std::iota(perm.begin(), perm.end(), 0);
    ct.cl.clear();
    struct Item { int id; };
    ct.cl.push_back(Cluster{});
    ct.cl[0].ofs = 0; ct.cl[0].size = n; ct.cl[0].level = 0;
    std::vector<int> stack{0};
    while (!stack.empty()) {
        const int id = stack.back(); stack.pop_back();
        Cluster c = ct.cl[id];
        for (int d = 0; d < dim; ++d) { c.bmin[d] = 1e300; c.bmax[d] = -1e300; }
        for (int64_t i = c.ofs; i < c.ofs + c.size; ++i)
            for (int d = 0; d < dim; ++d) {
                const double v = pts[size_t(perm[i] * dim + d)];
                c.bmin[d] = std::min(c.bmin[d], v);
                c.bmax[d] = std::max(c.bmax[d], v);
            }
        if (c.size > leaf) {
            int ax = 0;
            double best = -1;
            for (int d = 0; d < dim; ++d)
                if (c.bmax[d] - c.bmin[d] > best) { best = c.bmax[d] - c.bmin[d]; ax = d; }
            const int64_t half = c.size / 2;
            auto b = perm.begin() + c.ofs;
            // stable ordering inside each half: sort by coordinate, ties by index
            std::sort(b, b + c.size, [&](int64_t p, int64_t q) {
                const double vp = pts[size_t(p * dim + ax)], vq = pts[size_t(q * dim + ax)];
                return vp < vq || (vp == vq && p < q);
            });
            Cluster s0, s1;
            s0.ofs = c.ofs; s0.size = half; s0.level = c.level + 1;
            s1.ofs = c.ofs + half; s1.size = c.size - half; s1.level = c.level + 1;
            c.son[0] = int(ct.cl.size());
            c.son[1] = int(ct.cl.size()) + 1;
            ct.cl.push_back(s0);
            ct.cl.push_back(s1);
            stack.push_back(c.son[1]);
            stack.push_back(c.son[0]);
        }
        ct.cl[id] = c;
    }
}

// ---------------------------------------------------------------- leaves
struct Leaf {
    int rc = 0, cc = 0;          // row / column cluster ids
    int64_t row0 = 0, nrows = 0, col0 = 0, ncols = 0;
    int kind = HLRC_LEAF_DENSE;
    int rank = 0;
    std::vector<double> D, U, V, sv;
};

static void build_bt(const ClusterTree& ct, int dim, double eta, int rc, int cc, std::vector<Leaf>& leaves) {
    const Cluster& r = ct.cl[rc];
    const Cluster& c = ct.cl[cc];
    const bool adm = std::min(diam(r, dim), diam(c, dim)) <= eta * dist(r, c, dim);
    if (adm || r.leaf() || c.leaf()) {
        Leaf l;
        l.rc = rc; l.cc = cc;
        l.row0 = r.ofs; l.nrows = r.size; l.col0 = c.ofs; l.ncols = c.size;
        l.kind = adm ? HLRC_LEAF_LOWRANK : HLRC_LEAF_DENSE;
        leaves.push_back(std::move(l));
        return;
    }
    for (int i = 0; i < 2; ++i)
        for (int j = 0; j < 2; ++j) build_bt(ct, dim, eta, r.son[i], c.son[j], leaves);
}

// ACA with maximum pivot search (approx/aca.hh:118-225, 328-436):
// column residual -> pivot row = argmax |column|; stop if |max| <= eps_mach^2;
// scale column by 1/max; row residual; next column = argmax |row| over unused
// columns; stop when |u||v| < eps * |U V^T|_F (estimate), keeping that pair.
static void aca(const Problem& P, int64_t r0, int64_t m, int64_t c0, int64_t n, double eps, Mat& U, Mat& V) {
    const double zero_val = std::numeric_limits<double>::epsilon() * std::numeric_limits<double>::epsilon();
    std::vector<std::vector<double>> Us, Vs;
    std::vector<char> used_cols(size_t(n), 0);
    int64_t next_col = 0;
    double norm_M = 0;
    const int64_t max_rank = std::min(m, n);
    for (int64_t it = 0; it < max_rank; ++it) {
        const int64_t pc = next_col;
        used_cols[pc] = 1;
        std::vector<double> col(static_cast<size_t>(m)), row(static_cast<size_t>(n));
        for (int64_t i = 0; i < m; ++i) col[i] = P.entry(r0 + i, c0 + pc);
        for (size_t l = 0; l < Us.size(); ++l) {
            const double f = Vs[l][pc];
            const double* u = Us[l].data();
            for (int64_t i = 0; i < m; ++i) col[i] -= f * u[i];
        }
        int64_t pr = 0;
        double amax = -1;
        for (int64_t i = 0; i < m; ++i)
            if (std::fabs(col[i]) > amax) { amax = std::fabs(col[i]); pr = i; }
        const double maxv = col[pr];
        if (std::fabs(maxv) <= zero_val) break;
        const double inv = 1.0 / maxv;
        for (int64_t i = 0; i < m; ++i) col[i] *= inv;
        for (int64_t j = 0; j < n; ++j) row[j] = P.entry(r0 + pr, c0 + j);
        for (size_t l = 0; l < Us.size(); ++l) {
            const double f = Us[l][pr];
            const double* v = Vs[l].data();
            for (int64_t j = 0; j < n; ++j) row[j] -= f * v[j];
        }
        double maxr = 0;
        int64_t mj = -1;
        for (int64_t j = 0; j < n; ++j)
            if (!used_cols[j] && std::fabs(row[j]) > maxr) { maxr = std::fabs(row[j]); mj = j; }
        if (mj < 0)
            for (int64_t j = 0; j < n; ++j)
                if (!used_cols[j]) { mj = j; break; }
        next_col = mj;

        const double norm_i = nrm2(col.data(), m) * nrm2(row.data(), n);
        if (norm_i < eps * norm_M) {
            Us.push_back(std::move(col));
            Vs.push_back(std::move(row));
            break;
        }
        double upd = norm_i * norm_i;
        for (size_t l = 0; l < Us.size(); ++l)
            upd += 2.0 * dot(Us[l].data(), col.data(), m) * dot(Vs[l].data(), row.data(), n);
        norm_M = std::sqrt(norm_M * norm_M + std::fabs(upd));
        Us.push_back(std::move(col));
        Vs.push_back(std::move(row));
        if (next_col < 0) break;
    }
    const int64_t k = int64_t(Us.size());
    U = Mat(m, k);
    V = Mat(n, k);
    for (int64_t l = 0; l < k; ++l) {
        std::memcpy(U.col(l), Us[l].data(), size_t(m) * sizeof(double));
        std::memcpy(V.col(l), Vs[l].data(), size_t(n) * sizeof(double));
    }
}

// SVD recompression of U V^T (approx/svd.hh:94-209): QR of both factors,
// SVD of R_U R_V^T, truncation, then the singular values are multiplied into
// the factor with fewer rows.  If the rank is not below min(m, n) the block
// is formed and decomposed directly.
static void truncate(Mat& U, Mat& V, double eps, std::vector<double>& sv_out) {
    const int64_t m = U.m, n = V.m, k = U.n;
    sv_out.clear();
    if (k == 0) return;
    Mat W, X;
    std::vector<double> S;
    int64_t kk;
    if (k >= std::min(m, n)) {
        Mat M = prod_nt(U, V);
        Mat Us, Vs;
        svd(M, Us, S, Vs);
        kk = trunc_rank(S, eps);
        W = Mat(m, kk); X = Mat(n, kk);
        for (int64_t j = 0; j < kk; ++j) {
            std::memcpy(W.col(j), Us.col(j), size_t(m) * sizeof(double));
            std::memcpy(X.col(j), Vs.col(j), size_t(n) * sizeof(double));
        }
    } else {
        Mat QU = U, RU, QV = V, RV;
        qr(QU, RU);
        qr(QV, RV);
        Mat R = prod_nt(RU, RV);
        Mat Us, Vs;
        svd(R, Us, S, Vs);
        kk = trunc_rank(S, eps);
        Mat Uk(k, kk), Vk(k, kk);
        for (int64_t j = 0; j < kk; ++j) {
            std::memcpy(Uk.col(j), Us.col(j), size_t(k) * sizeof(double));
            std::memcpy(Vk.col(j), Vs.col(j), size_t(k) * sizeof(double));
        }
        W = prod(QU, Uk);
        X = prod(QV, Vk);
    }
    sv_out.assign(S.begin(), S.begin() + kk);
    Mat& T = (W.m < X.m) ? W : X;
    for (int64_t j = 0; j < kk; ++j) {
        double* c = T.col(j);
        for (int64_t i = 0; i < T.m; ++i) c[i] *= S[j];
    }
    U = std::move(W);
    V = std::move(X);
}

// column_basis (approx/svd.hh:615-735): left singular vectors of M truncated
// to relative precision eps; direct SVD when M is wide, else QR first.
static Mat column_basis(const Mat& M, double eps, std::vector<double>& sv) {
    sv.clear();
    if (M.n == 0) return Mat(M.m, 0);
    Mat Uf;
    std::vector<double> S;
    if (M.n > M.m / 2) {
        Mat Vs;
        svd(M, Uf, S, Vs);
    } else {
        Mat Q = M, R, Ur, Vs;
        qr(Q, R);
        svd(R, Ur, S, Vs);
        Uf = prod(Q, Ur);
    }
    const int64_t k = trunc_rank(S, eps);
    Mat B(M.m, k);
    for (int64_t j = 0; j < k; ++j) std::memcpy(B.col(j), Uf.col(j), size_t(M.m) * sizeof(double));
    sv.assign(S.begin(), S.begin() + k);
    return B;
}

struct Basis {
    int64_t ofs = 0, size = 0;
    Mat V;
    std::vector<double> sv;
};

// Node of a nested cluster basis: an explicit basis at the leaves, and the
// transfer matrix to the parent's basis everywhere but at the root
// (matrix/nested_cluster_basis.hh).
struct NBasis {
    int64_t ofs = 0, size = 0;
    int rank = 0;
    Mat V;   // leaves: size x rank
    Mat E;   // non-root: rank x parent rank
};

struct UniBlock {
    int leaf = 0;      // index into leaves
    Mat S;             // coupling k_row x k_col
};

struct HBuild {
    hlrc_problem pr{};
    Problem P;
    ClusterTree ct;
    std::vector<Leaf> leaves;
    std::vector<hlrc_block> desc_blocks;
    // uniform
    bool uniform = false;
    std::vector<Basis> rowcb, colcb;               // indexed by cluster id
    std::vector<Mat> coupling;                     // per leaf (empty for dense)
    std::vector<hlrc_basis> desc_rowb, desc_colb;
    std::vector<hlrc_uniform_block> desc_ublocks;
    // H^2 (nested bases)
    bool nested = false;
    std::vector<NBasis> rowh2, colh2;              // indexed by cluster id
    std::vector<Mat> h2coupling;                   // per leaf (empty for dense)
    std::vector<hlrc_h2_cluster> desc_rowh2, desc_colh2;
    std::vector<hlrc_uniform_block> desc_h2blocks;
    double seconds = 0;
    int max_rank = 0;
    int64_t bytes = 0;
};

static void build_uniform(HBuild& B, double eps) {
    const auto& ct = B.ct;
    const int nc = int(ct.cl.size());
    std::vector<std::vector<int>> rowlist(static_cast<size_t>(nc)), collist(static_cast<size_t>(nc));
    for (int i = 0; i < int(B.leaves.size()); ++i) {
        const Leaf& l = B.leaves[i];
        if (l.kind == HLRC_LEAF_LOWRANK && l.rank > 0) {
            rowlist[l.rc].push_back(i);
            collist[l.cc].push_back(i);
        }
    }
    B.rowcb.assign(size_t(nc), Basis{});
    B.colcb.assign(size_t(nc), Basis{});
    // row bases: W_t = [U_i R_i^T], V_i = Q_i R_i; column bases symmetric
    #pragma omp parallel for schedule(dynamic, 1)
    for (int c = 0; c < 2 * nc; ++c) {
        const bool row = c < nc;
        const int t = row ? c : c - nc;
        const auto& lst = row ? rowlist[t] : collist[t];
        Basis& bs = row ? B.rowcb[t] : B.colcb[t];
        bs.ofs = ct.cl[t].ofs;
        bs.size = ct.cl[t].size;
        if (lst.empty()) { bs.V = Mat(bs.size, 0); continue; }
        int64_t tot = 0;
        for (int i : lst) tot += B.leaves[i].rank;
        Mat W(bs.size, tot);
        int64_t pos = 0;
        for (int i : lst) {
            const Leaf& l = B.leaves[i];
            const int64_t k = l.rank;
            Mat A(row ? l.nrows : l.ncols, k), O(row ? l.ncols : l.nrows, k);
            std::memcpy(A.a.data(), (row ? l.U : l.V).data(), A.a.size() * sizeof(double));
            std::memcpy(O.a.data(), (row ? l.V : l.U).data(), O.a.size() * sizeof(double));
            Mat R;
            qr(O, R);
            Mat AR = prod_nt(A, R);
            for (int64_t j = 0; j < k; ++j) std::memcpy(W.col(pos + j), AR.col(j), size_t(bs.size) * sizeof(double));
            pos += k;
        }
        bs.V = column_basis(W, eps, bs.sv);
    }
    B.coupling.assign(B.leaves.size(), Mat());
    #pragma omp parallel for schedule(dynamic, 4)
    for (int i = 0; i < int(B.leaves.size()); ++i) {
        const Leaf& l = B.leaves[i];
        if (l.kind != HLRC_LEAF_LOWRANK) continue;
        const Basis& rb = B.rowcb[l.rc];
        const Basis& cb = B.colcb[l.cc];
        const int64_t k = l.rank;
        Mat U(l.nrows, k), V(l.ncols, k);
        if (k > 0) {
            std::memcpy(U.a.data(), l.U.data(), U.a.size() * sizeof(double));
            std::memcpy(V.a.data(), l.V.data(), V.a.size() * sizeof(double));
        }
        Mat Sr = prod_tn(rb.V, U);   // k_t x k
        Mat Sc = prod_tn(cb.V, V);   // k_s x k
        B.coupling[i] = prod_nt(Sr, Sc);   // k_t x k_s
    }
    // descriptors
    B.desc_rowb.resize(static_cast<size_t>(nc));
    B.desc_colb.resize(static_cast<size_t>(nc));
    for (int t = 0; t < nc; ++t) {
        for (int s = 0; s < 2; ++s) {
            const Basis& bs = s == 0 ? B.rowcb[t] : B.colcb[t];
            hlrc_basis& d = s == 0 ? B.desc_rowb[t] : B.desc_colb[t];
            d.ofs = bs.ofs; d.size = bs.size; d.rank = int32_t(bs.V.n); d.pad_ = 0;
            d.V = bs.V.a.empty() ? nullptr : bs.V.a.data();
            d.ldv = std::max<int64_t>(1, bs.size);
        }
    }
    B.desc_ublocks.resize(B.leaves.size());
    for (size_t i = 0; i < B.leaves.size(); ++i) {
        const Leaf& l = B.leaves[i];
        hlrc_uniform_block& d = B.desc_ublocks[i];
        std::memset(&d, 0, sizeof(d));
        d.row0 = l.row0; d.nrows = l.nrows; d.col0 = l.col0; d.ncols = l.ncols;
        d.kind = l.kind;
        if (l.kind == HLRC_LEAF_LOWRANK) {
            d.row_basis = l.rc; d.col_basis = l.cc;
            d.S = B.coupling[i].a.empty() ? nullptr : B.coupling[i].a.data();
            d.lds = std::max<int64_t>(1, B.coupling[i].m);
        } else {
            d.D = l.D.data(); d.ldd = l.nrows;
        }
    }
}


// Nested (H^2) cluster bases from the admissible leaves, bottom-up.  The
// basis of cluster t must span the rows of t of every admissible block of t
// and of its ancestors (the total cluster basis), weighted by the other
// factor: a block b = U_b V_b^T contributes U_b|_t R_b^T with V_b = Q_b R_b.
//   leaf t:   V_t = column_basis([U_b|_t R_b^T]_b)                  (size x k_t)
//   parent t: Q_t = column_basis([P_t1[b] R_b^T ; P_t2[b] R_b^T]_b) and
//             E_ti = rows of Q_t for son i, so V_t = [V_t1 E_t1; V_t2 E_t2]
// where P_t[b] = V_t^T U_b|_t is carried upwards as P_t = sum_i E_ti^T P_ti.
// The column bases are the same with the roles of U_b and V_b exchanged.
// Couplings: S_b = P_rc[b] (P'_cc[b])^T, the projections at the block's own
// clusters.
static void build_nested(HBuild& B, double eps, bool row, std::vector<NBasis>& nb, std::vector<std::vector<Mat>>& own) {
    const auto& ct = B.ct;
    const int nc = int(ct.cl.size());
    std::vector<int> parent(static_cast<size_t>(nc), -1);
    for (int t = 0; t < nc; ++t)
        for (int i = 0; i < 2; ++i)
            if (ct.cl[t].son[i] >= 0) parent[size_t(ct.cl[t].son[i])] = t;
    std::vector<std::vector<int>> lst(static_cast<size_t>(nc));   // admissible leaves by own cluster
    for (int i = 0; i < int(B.leaves.size()); ++i) {
        const Leaf& l = B.leaves[i];
        if (l.kind == HLRC_LEAF_LOWRANK && l.rank > 0) lst[size_t(row ? l.rc : l.cc)].push_back(i);
    }
    // R factors of the other factor, per leaf
    std::vector<Mat> R(B.leaves.size());
    #pragma omp parallel for schedule(dynamic, 8)
    for (int i = 0; i < int(B.leaves.size()); ++i) {
        const Leaf& l = B.leaves[i];
        if (l.kind != HLRC_LEAF_LOWRANK || l.rank == 0) continue;
        Mat O(row ? l.ncols : l.nrows, l.rank);
        std::memcpy(O.a.data(), (row ? l.V : l.U).data(), O.a.size() * sizeof(double));
        qr(O, R[size_t(i)]);
    }
    // total lists: own leaves, then the ancestors'
    std::vector<std::vector<int>> tot(static_cast<size_t>(nc));
    for (int t = 0; t < nc; ++t) {
        for (int a = t; a >= 0; a = parent[size_t(a)]) tot[size_t(t)].insert(tot[size_t(t)].end(), lst[size_t(a)].begin(), lst[size_t(a)].end());
    }
    int maxlev = 0;
    for (const Cluster& c : ct.cl) maxlev = std::max(maxlev, c.level);
    nb.assign(size_t(nc), NBasis{});
    own.assign(size_t(nc), {});
    std::vector<std::vector<Mat>> P(static_cast<size_t>(nc));   // P[t][j] for leaf tot[t][j]
    for (int lev = maxlev; lev >= 0; --lev) {
        std::vector<int> cls;
        for (int t = 0; t < nc; ++t)
            if (ct.cl[t].level == lev) cls.push_back(t);
        #pragma omp parallel for schedule(dynamic, 1)
        for (int ci = 0; ci < int(cls.size()); ++ci) {
            const int t = cls[size_t(ci)];
            const Cluster& c = ct.cl[t];
            NBasis& bs = nb[size_t(t)];
            bs.ofs = c.ofs;
            bs.size = c.size;
            const auto& L = tot[size_t(t)];
            int64_t cols = 0;
            for (int i : L) cols += B.leaves[size_t(i)].rank;
            // the rows of U_b in t (row side) or of V_b (column side)
            auto factor_rows = [&](int i) {
                const Leaf& l = B.leaves[size_t(i)];
                const int64_t m = row ? l.nrows : l.ncols, o = c.ofs - (row ? l.row0 : l.col0);
                const std::vector<double>& F = row ? l.U : l.V;
                Mat A(c.size, l.rank);
                for (int64_t j = 0; j < l.rank; ++j)
                    std::memcpy(A.col(j), F.data() + j * m + o, size_t(c.size) * sizeof(double));
                return A;
            };
            std::vector<double> sv;
            if (c.leaf()) {
                Mat Z(c.size, cols);
                int64_t pos = 0;
                for (int i : L) {
                    const Mat AR = prod_nt(factor_rows(i), R[size_t(i)]);
                    std::memcpy(Z.col(pos), AR.a.data(), AR.a.size() * sizeof(double));
                    pos += AR.n;
                }
                bs.V = cols > 0 ? column_basis(Z, eps, sv) : Mat(c.size, 0);
                bs.rank = int(bs.V.n);
                P[size_t(t)].resize(L.size());
                for (size_t j = 0; j < L.size(); ++j) P[size_t(t)][j] = prod_tn(bs.V, factor_rows(L[j]));
            } else {
                const int s0 = c.son[0], s1 = c.son[1];
                const int k0 = s0 >= 0 ? nb[size_t(s0)].rank : 0, k1 = s1 >= 0 ? nb[size_t(s1)].rank : 0;
                // son j's list starts with its own leaves; t's list is its tail
                auto son_proj = [&](int s, size_t j) -> const Mat& {
                    const size_t off = tot[size_t(s)].size() - L.size();
                    return P[size_t(s)][off + j];
                };
                Mat Z(k0 + k1, cols);
                int64_t pos = 0;
                for (size_t j = 0; j < L.size(); ++j) {
                    const Mat& Rb = R[size_t(L[j])];
                    if (k0 > 0) {
                        const Mat A = prod_nt(son_proj(s0, j), Rb);
                        for (int64_t q = 0; q < A.n; ++q)
                            for (int64_t r = 0; r < k0; ++r) Z(r, pos + q) = A(r, q);
                    }
                    if (k1 > 0) {
                        const Mat A = prod_nt(son_proj(s1, j), Rb);
                        for (int64_t q = 0; q < A.n; ++q)
                            for (int64_t r = 0; r < k1; ++r) Z(k0 + r, pos + q) = A(r, q);
                    }
                    pos += Rb.n;
                }
                const Mat Q = (cols > 0 && k0 + k1 > 0) ? column_basis(Z, eps, sv) : Mat(k0 + k1, 0);
                bs.rank = int(Q.n);
                for (int si = 0; si < 2; ++si) {
                    const int s = c.son[si];
                    if (s < 0) continue;
                    const int ks = si == 0 ? k0 : k1, r0 = si == 0 ? 0 : k0;
                    Mat E(ks, Q.n);
                    for (int64_t q = 0; q < Q.n; ++q)
                        for (int64_t r = 0; r < ks; ++r) E(r, q) = Q(r0 + r, q);
                    nb[size_t(s)].E = std::move(E);
                }
                P[size_t(t)].resize(L.size());
                for (size_t j = 0; j < L.size(); ++j) {
                    Mat Pj(bs.rank, B.leaves[size_t(L[j])].rank);
                    for (int si = 0; si < 2; ++si) {
                        const int s = c.son[si];
                        if (s < 0 || nb[size_t(s)].rank == 0) continue;
                        const Mat A = prod_tn(nb[size_t(s)].E, son_proj(s, j));
                        for (size_t e = 0; e < A.a.size(); ++e) Pj.a[e] += A.a[e];
                    }
                    P[size_t(t)][j] = std::move(Pj);
                }
            }
        }
        // a cluster's own blocks keep their projections (couplings); the
        // rest of the sons' projections is no longer needed
        for (int t : cls) {
            own[size_t(t)].assign(P[size_t(t)].begin(), P[size_t(t)].begin() + long(lst[size_t(t)].size()));
            for (int si = 0; si < 2; ++si)
                if (ct.cl[t].son[si] >= 0) std::vector<Mat>().swap(P[size_t(ct.cl[t].son[si])]);
        }
    }
}

static void build_h2(HBuild& B, double eps) {
    const auto& ct = B.ct;
    const int nc = int(ct.cl.size());
    std::vector<std::vector<Mat>> ownr, ownc;
    build_nested(B, eps, true, B.rowh2, ownr);
    build_nested(B, eps, false, B.colh2, ownc);
    // couplings S_b = (V_t^T U_b)(W_s^T V_b)^T; a leaf's position in its
    // cluster's own list is its rank among that cluster's admissible leaves
    std::vector<int> posr(B.leaves.size(), -1), posc(B.leaves.size(), -1);
    std::vector<int> cntr(static_cast<size_t>(nc), 0), cntc(static_cast<size_t>(nc), 0);
    for (size_t i = 0; i < B.leaves.size(); ++i) {
        const Leaf& l = B.leaves[i];
        if (l.kind != HLRC_LEAF_LOWRANK || l.rank == 0) continue;
        posr[i] = cntr[size_t(l.rc)]++;
        posc[i] = cntc[size_t(l.cc)]++;
    }
    B.h2coupling.assign(B.leaves.size(), Mat());
    for (size_t i = 0; i < B.leaves.size(); ++i) {
        const Leaf& l = B.leaves[i];
        if (l.kind != HLRC_LEAF_LOWRANK) continue;
        if (l.rank == 0) { B.h2coupling[i] = Mat(B.rowh2[size_t(l.rc)].rank, B.colh2[size_t(l.cc)].rank); continue; }
        B.h2coupling[i] = prod_nt(ownr[size_t(l.rc)][size_t(posr[i])], ownc[size_t(l.cc)][size_t(posc[i])]);
    }
    std::vector<int> parent(static_cast<size_t>(nc), -1);
    for (int t = 0; t < nc; ++t)
        for (int j = 0; j < 2; ++j)
            if (ct.cl[t].son[j] >= 0) parent[size_t(ct.cl[t].son[j])] = t;
    for (int side = 0; side < 2; ++side) {
        const std::vector<NBasis>& nbv = side == 0 ? B.rowh2 : B.colh2;
        std::vector<hlrc_h2_cluster>& out = side == 0 ? B.desc_rowh2 : B.desc_colh2;
        out.assign(size_t(nc), hlrc_h2_cluster{});
        for (int t = 0; t < nc; ++t) {
            const NBasis& b = nbv[size_t(t)];
            hlrc_h2_cluster& d = out[size_t(t)];
            std::memset(&d, 0, sizeof(d));
            d.ofs = b.ofs; d.size = b.size;
            d.son[0] = ct.cl[t].son[0]; d.son[1] = ct.cl[t].son[1];
            d.parent = parent[size_t(t)];
            d.rank = b.rank;
            d.V = b.V.a.empty() ? nullptr : b.V.a.data();
            d.ldv = std::max<int64_t>(1, b.size);
            d.E = b.E.a.empty() ? nullptr : b.E.a.data();
            d.lde = std::max<int64_t>(1, b.E.m);
        }
    }
    B.desc_h2blocks.resize(B.leaves.size());
    for (size_t i = 0; i < B.leaves.size(); ++i) {
        const Leaf& l = B.leaves[i];
        hlrc_uniform_block& d = B.desc_h2blocks[i];
        std::memset(&d, 0, sizeof(d));
        d.row0 = l.row0; d.nrows = l.nrows; d.col0 = l.col0; d.ncols = l.ncols;
        d.kind = l.kind;
        if (l.kind == HLRC_LEAF_LOWRANK) {
            d.row_basis = l.rc; d.col_basis = l.cc;
            d.S = B.h2coupling[i].a.empty() ? nullptr : B.h2coupling[i].a.data();
            d.lds = std::max<int64_t>(1, B.h2coupling[i].m);
        } else {
            d.D = l.D.data(); d.ldd = l.nrows;
        }
    }
}

}  // namespace hlrc

using namespace hlrc;

struct hlrc_hbuild_s {
    HBuild b;
    double* dev_arena = nullptr;   // on_device builds: the leaf data (until fetched)
    int64_t dev_doubles = 0;
    std::vector<GpuLeaf> gl;       // per leaf: offsets into dev_arena
    std::vector<double> host_arena;   // fetched on_device builds: the same data on the host
    ~hlrc_hbuild_s() { gpu_free(dev_arena); }
};

extern "C" hlrc_status hlrc_build(const hlrc_problem* prob, hlrc_hbuild* out) {
    clear_error();
    if (!prob || !out) return fail(HLRC_ERR_ARG, "hlrc_build: null argument");
    if (prob->kind < 0 || prob->kind > 2) return fail(HLRC_ERR_ARG, "hlrc_build: unknown problem kind %d", prob->kind);
    if (prob->leaf_size < 2) return fail(HLRC_ERR_ARG, "hlrc_build: leaf_size must be >= 2");
    if (prob->kind != HLRC_PROBLEM_LAPLACE_SPH && prob->n < 1) return fail(HLRC_ERR_ARG, "hlrc_build: n must be >= 1");
    if (!(prob->eps > 0) || !(prob->eta > 0)) return fail(HLRC_ERR_ARG, "hlrc_build: eps and eta must be > 0");
    if (prob->on_device && (prob->uniform || prob->nested))
        return fail(HLRC_ERR_ARG, "hlrc_build: on_device builds the H form only (uniform and nested need host leaves)");
    const auto t0 = std::chrono::steady_clock::now();
    auto h = std::make_unique<hlrc_hbuild_s>();
    HBuild& B = h->b;
    B.pr = *prob;
    const int nthreads = prob->nthreads > 0 ? prob->nthreads : omp_get_max_threads();
    std::vector<double> pts, wts;
    int dim = 1;
    make_points(*prob, pts, wts, dim);
    const int64_t n = int64_t(pts.size()) / dim;
    build_ct(pts, dim, n, prob->leaf_size, B.ct, B.P.perm);
    Problem& P = B.P;
    P.kind = prob->kind; P.dim = dim; P.n = n;
    P.ell = prob->ell > 0 ? prob->ell : 0.1;
    P.nugget = prob->nugget;
    P.h = 1.0 / double(n);
    P.pts.resize(pts.size());
    for (int64_t i = 0; i < n; ++i)
        for (int d = 0; d < dim; ++d) P.pts[size_t(i * dim + d)] = pts[size_t(P.perm[i] * dim + d)];
    if (!wts.empty()) {
        P.wts.resize(static_cast<size_t>(n));
        for (int64_t i = 0; i < n; ++i) P.wts[i] = wts[size_t(P.perm[i])];
    }
    build_bt(B.ct, dim, prob->eta, 0, 0, B.leaves);

    // assemble leaves, most expensive first for load balance
    std::vector<int> order(B.leaves.size());
    std::iota(order.begin(), order.end(), 0);
    std::sort(order.begin(), order.end(), [&](int a, int b) {
        const auto ca = B.leaves[a].nrows * B.leaves[a].ncols, cb = B.leaves[b].nrows * B.leaves[b].ncols;
        return ca > cb || (ca == cb && a < b);
    });
    const double eps = prob->eps;
    if (prob->on_device) {
        GpuProblem gp;
        gp.kind = P.kind; gp.dim = P.dim; gp.n = P.n;
        gp.pts = P.pts.data();
        gp.wts = P.wts.empty() ? nullptr : P.wts.data();
        gp.ell = P.ell; gp.nugget = P.nugget; gp.h = P.h;
        h->gl.resize(B.leaves.size());
        for (size_t i = 0; i < B.leaves.size(); ++i) {
            const Leaf& l = B.leaves[i];
            GpuLeaf& g = h->gl[i];
            g.row0 = l.row0; g.nrows = l.nrows; g.col0 = l.col0; g.ncols = l.ncols; g.kind = l.kind;
        }
        const hlrc_status st = gpu_assemble(gp, h->gl, eps, &h->dev_arena, &h->dev_doubles);
        if (st != HLRC_OK) return st;
        B.desc_blocks.resize(B.leaves.size());
        for (size_t i = 0; i < B.leaves.size(); ++i) {
            Leaf& l = B.leaves[i];
            const GpuLeaf& g = h->gl[i];
            l.rank = g.rank;
            hlrc_block& d = B.desc_blocks[i];
            std::memset(&d, 0, sizeof(d));
            d.row0 = l.row0; d.nrows = l.nrows; d.col0 = l.col0; d.ncols = l.ncols;
            d.kind = l.kind; d.rank = l.rank;
            if (l.kind == HLRC_LEAF_DENSE) {
                d.D = g.d >= 0 ? h->dev_arena + g.d : nullptr;
                d.ldd = std::max<int64_t>(1, l.nrows);
                B.bytes += l.nrows * l.ncols * 8;
            } else {
                d.U = l.rank ? h->dev_arena + g.u : nullptr; d.ldu = std::max<int64_t>(1, l.nrows);
                d.V = l.rank ? h->dev_arena + g.v : nullptr; d.ldv = std::max<int64_t>(1, l.ncols);
                d.sv = l.rank ? h->dev_arena + g.s : nullptr;
                B.bytes += (l.nrows + l.ncols) * l.rank * 8;
                B.max_rank = std::max(B.max_rank, l.rank);
            }
        }
        B.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        *out = h.release();
        return HLRC_OK;
    }
    #pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
    for (int oi = 0; oi < int(order.size()); ++oi) {
        Leaf& l = B.leaves[order[oi]];
        if (l.kind == HLRC_LEAF_DENSE) {
            l.D.resize(size_t(l.nrows * l.ncols));
            for (int64_t j = 0; j < l.ncols; ++j)
                for (int64_t i = 0; i < l.nrows; ++i) l.D[size_t(i + j * l.nrows)] = P.entry(l.row0 + i, l.col0 + j);
        } else {
            Mat U, V;
            aca(P, l.row0, l.nrows, l.col0, l.ncols, eps, U, V);
            truncate(U, V, eps, l.sv);
            l.rank = int(U.n);
            l.U = std::move(U.a);
            l.V = std::move(V.a);
        }
    }
    B.desc_blocks.resize(B.leaves.size());
    for (size_t i = 0; i < B.leaves.size(); ++i) {
        const Leaf& l = B.leaves[i];
        hlrc_block& d = B.desc_blocks[i];
        std::memset(&d, 0, sizeof(d));
        d.row0 = l.row0; d.nrows = l.nrows; d.col0 = l.col0; d.ncols = l.ncols;
        d.kind = l.kind; d.rank = l.rank;
        if (l.kind == HLRC_LEAF_DENSE) {
            d.D = l.D.data(); d.ldd = l.nrows;
            B.bytes += int64_t(l.D.size()) * 8;
        } else {
            d.U = l.rank ? l.U.data() : nullptr; d.ldu = std::max<int64_t>(1, l.nrows);
            d.V = l.rank ? l.V.data() : nullptr; d.ldv = std::max<int64_t>(1, l.ncols);
            d.sv = l.rank ? l.sv.data() : nullptr;
            B.bytes += int64_t(l.U.size() + l.V.size()) * 8;
            B.max_rank = std::max(B.max_rank, l.rank);
        }
    }
    if (prob->uniform) {
        B.uniform = true;
        omp_set_num_threads(nthreads);
        build_uniform(B, eps);
    }
    if (prob->nested) {
        B.nested = true;
        omp_set_num_threads(nthreads);
        build_h2(B, eps);
    }
    B.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    *out = h.release();
    return HLRC_OK;
}

extern "C" hlrc_status hlrc_build_h_desc(hlrc_hbuild B, hlrc_h_desc* out) {
    if (!B || !out) return fail(HLRC_ERR_ARG, "hlrc_build_h_desc: null argument");
    out->nrows = B->b.P.n;
    out->ncols = B->b.P.n;
    out->nblocks = int64_t(B->b.desc_blocks.size());
    out->blocks = B->b.desc_blocks.data();
    return HLRC_OK;
}

extern "C" hlrc_status hlrc_build_uniform_desc(hlrc_hbuild B, hlrc_uniform_desc* out) {
    if (!B || !out) return fail(HLRC_ERR_ARG, "hlrc_build_uniform_desc: null argument");
    if (!B->b.uniform) return fail(HLRC_ERR_ARG, "hlrc_build_uniform_desc: problem was built without uniform=1");
    out->nrows = B->b.P.n;
    out->ncols = B->b.P.n;
    out->nrow_bases = int64_t(B->b.desc_rowb.size());
    out->row_bases = B->b.desc_rowb.data();
    out->ncol_bases = int64_t(B->b.desc_colb.size());
    out->col_bases = B->b.desc_colb.data();
    out->nblocks = int64_t(B->b.desc_ublocks.size());
    out->blocks = B->b.desc_ublocks.data();
    return HLRC_OK;
}

extern "C" hlrc_status hlrc_build_h2_desc(hlrc_hbuild B, hlrc_h2_desc* out) {
    if (!B || !out) return fail(HLRC_ERR_ARG, "hlrc_build_h2_desc: null argument");
    if (!B->b.nested) return fail(HLRC_ERR_ARG, "hlrc_build_h2_desc: problem was built without nested=1");
    out->nrows = B->b.P.n;
    out->ncols = B->b.P.n;
    out->nrow_clusters = int64_t(B->b.desc_rowh2.size());
    out->row_clusters = B->b.desc_rowh2.data();
    out->ncol_clusters = int64_t(B->b.desc_colh2.size());
    out->col_clusters = B->b.desc_colh2.data();
    out->nblocks = int64_t(B->b.desc_h2blocks.size());
    out->blocks = B->b.desc_h2blocks.data();
    return HLRC_OK;
}

extern "C" hlrc_status hlrc_build_points(hlrc_hbuild B, const double** pts, int* dim, int64_t* n) {
    if (!B || !pts || !dim || !n) return fail(HLRC_ERR_ARG, "hlrc_build_points: null argument");
    *pts = B->b.P.pts.data();
    *dim = B->b.P.dim;
    *n = B->b.P.n;
    return HLRC_OK;
}

extern "C" hlrc_status hlrc_build_weights(hlrc_hbuild B, const double** w) {
    if (!B || !w) return fail(HLRC_ERR_ARG, "hlrc_build_weights: null argument");
    *w = B->b.P.wts.empty() ? nullptr : B->b.P.wts.data();
    return HLRC_OK;
}

extern "C" hlrc_status hlrc_build_perm(hlrc_hbuild B, const int64_t** perm) {
    if (!B || !perm) return fail(HLRC_ERR_ARG, "hlrc_build_perm: null argument");
    *perm = B->b.P.perm.data();
    return HLRC_OK;
}

extern "C" hlrc_status hlrc_build_stats(hlrc_hbuild B, double* seconds, int64_t* nleaves, int32_t* max_rank,
                                        int64_t* bytes) {
    if (!B) return fail(HLRC_ERR_ARG, "hlrc_build_stats: null argument");
    if (seconds) *seconds = B->b.seconds;
    if (nleaves) *nleaves = int64_t(B->b.leaves.size());
    if (max_rank) *max_rank = B->b.max_rank;
    if (bytes) *bytes = B->b.bytes;
    return HLRC_OK;
}

extern "C" hlrc_status hlrc_build_leaves_on_device(hlrc_hbuild B, int* on_device) {
    if (!B || !on_device) return fail(HLRC_ERR_ARG, "hlrc_build_leaves_on_device: null argument");
    *on_device = B->dev_arena ? 1 : 0;
    return HLRC_OK;
}

extern "C" hlrc_status hlrc_build_fetch(hlrc_hbuild B) {
    clear_error();
    if (!B) return fail(HLRC_ERR_ARG, "hlrc_build_fetch: null argument");
    if (!B->dev_arena) return HLRC_OK;
    HBuild& b = B->b;
    // one bulk copy of the arena; the descriptors keep their offsets
    B->host_arena.resize(size_t(std::max<int64_t>(1, B->dev_doubles)));
    const hlrc_status st = gpu_copy_to_host(B->host_arena.data(), B->dev_arena, B->dev_doubles);
    if (st != HLRC_OK) return st;
    double* h = B->host_arena.data();
    for (size_t i = 0; i < b.leaves.size(); ++i) {
        const Leaf& l = b.leaves[i];
        const GpuLeaf& g = B->gl[i];
        hlrc_block& d = b.desc_blocks[i];
        if (l.kind == HLRC_LEAF_DENSE) {
            d.D = g.d >= 0 && l.nrows * l.ncols > 0 ? h + g.d : nullptr;
        } else if (l.rank > 0) {
            d.U = h + g.u; d.V = h + g.v; d.sv = h + g.s;
        }
    }
    gpu_free(B->dev_arena);
    B->dev_arena = nullptr;
    B->dev_doubles = 0;
    return HLRC_OK;
}

extern "C" hlrc_status hlrc_build_free(hlrc_hbuild B) {
    delete B;
    return HLRC_OK;
}

extern "C" double hlrc_build_entry(hlrc_hbuild B, int64_t i, int64_t j) {
    if (!B || i < 0 || j < 0 || i >= B->b.P.n || j >= B->b.P.n) return std::nan("");
    return B->b.P.entry(i, j);
}
