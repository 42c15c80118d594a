// Runs the HLR-side adapter of INTEGRATION.md (extracted into arith.hh by
// tests/test_capi_c.py) on a 2 x 2 block matrix: dense diagonal leaves and
// low-rank off-diagonal leaves, as HLR's block tree would hold them.  The
// result of hlr::cuda::mul_vec is compared with the dense product of the
// same matrix.  "--dry" only flattens (no GPU).
#include <cmath>
#include <cstdio>
#include <cstring>

#include "arith.hh"

using namespace hlr;

static double val(int64_t i, int64_t j, int salt) { return std::sin(0.37 * double(i + 1) + 0.11 * double(j) * salt); }

int main(int argc, char** argv) {
    const bool dry = argc > 1 && std::strcmp(argv[1], "--dry") == 0;
    const int64_t h = 64, n = 2 * h;
    Hpro::TBlockMatrix<double> A;
    A.r = {0, n - 1};
    A.c = {0, n - 1};
    A.nbr = A.nbc = 2;
    std::vector<double> full(size_t(n * n), 0.0);   // the same matrix, dense
    for (uint j = 0; j < 2; ++j)
        for (uint i = 0; i < 2; ++i) {
            const int64_t r0 = i * h, c0 = j * h;
            if (i == j) {
                auto D = std::make_unique<matrix::dense_matrix<double>>();
                D->r = {r0, r0 + h - 1};
                D->c = {c0, c0 + h - 1};
                D->M = blas::matrix<double>(h, h);
                for (int64_t c = 0; c < h; ++c)
                    for (int64_t r = 0; r < h; ++r) {
                        D->M(r, c) = val(r0 + r, c0 + c, 1) + (r == c ? 4.0 : 0.0);
                        full[size_t((r0 + r) + (c0 + c) * n)] = D->M(r, c);
                    }
                A.sub.push_back(std::move(D));
            } else {
                const int64_t k = 2 + int64_t(i);
                auto R = std::make_unique<matrix::lrmatrix<double>>();
                R->r = {r0, r0 + h - 1};
                R->c = {c0, c0 + h - 1};
                R->u = blas::matrix<double>(h, k);
                R->v = blas::matrix<double>(h, k);
                for (int64_t l = 0; l < k; ++l)
                    for (int64_t r = 0; r < h; ++r) {
                        R->u(r, l) = val(r0 + r, l, 2);
                        R->v(r, l) = val(c0 + r, l, 3);
                    }
                for (int64_t c = 0; c < h; ++c)
                    for (int64_t r = 0; r < h; ++r) {
                        double s = 0;
                        for (int64_t l = 0; l < k; ++l) s += R->u(r, l) * R->v(c, l);
                        full[size_t((r0 + r) + (c0 + c) * n)] = s;
                    }
                A.sub.push_back(std::move(R));
            }
        }
    std::vector<hlrc_block> leaves;
    cuda::collect(static_cast<const Hpro::TMatrix<double>&>(A), leaves);
    std::printf("flattened %zu leaves\n", leaves.size());
    if (dry) return leaves.size() == 4 ? 0 : 1;

    try {
        auto G = cuda::upload(A);
        vector::scalar_vector<double> x, y;
        x.x.v.resize(size_t(n));
        y.x.v.assign(size_t(n), 0.5);
        for (int64_t i = 0; i < n; ++i) x.x.v[size_t(i)] = std::cos(0.3 * double(i));
        cuda::mul_vec(2.0, Hpro::apply_normal, G, x, y);     // y += 2 A x
        cuda::mul_vec(-1.0, Hpro::apply_transposed, G, x, y);  // y -= A^T x
        double d = 0, r = 0;
        for (int64_t i = 0; i < n; ++i) {
            double ref = 0.5;
            for (int64_t j = 0; j < n; ++j)
                ref += 2.0 * full[size_t(i + j * n)] * x.x.v[size_t(j)] - full[size_t(j + i * n)] * x.x.v[size_t(j)];
            d += (y.x.v[size_t(i)] - ref) * (y.x.v[size_t(i)] - ref);
            r += ref * ref;
        }
        std::printf("rel. error %.3e vs the dense product\n", std::sqrt(d / r));
        return std::sqrt(d / r) <= 1e-13 ? 0 : 1;
    } catch (const std::exception& e) {
        std::printf("error: %s\n", e.what());
        return 2;
    }
}
