/*
 * A plain C caller of the hlrc ABI: what a C or C++ program (HLR's adapter,
 * an MPI code) does to use the product, compiled and linked like one.
 *
 * It builds a 3D exponential-covariance H-matrix with the library's host
 * construction (hlrc_build), uploads it (hlrc_upload_h), creates two
 * workspaces and runs products of the one immutable handle on two CUDA
 * streams at once (hlrc_mvm_ws), as HLR's TBB product may be called from two
 * threads on one matrix with different y (include/hlr/tbb/arith.hh:312-323).
 * Both results are compared with the oracle's restatement of hlr::seq::mul_vec
 * (oracle/oracle.c, linked as the checker) at the FP64 parity bound 1e-13.
 *
 *   two_streams --dry   no GPU needed: build, dry-run plan, report sizes
 *   two_streams         the full run (needs a CUDA device)
 * Exit status 0 = pass.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <cuda_runtime.h>

#include "hlrc.h"

/* the checker (oracle/liboracle.so) */
int oracle_hmvm_seq(const hlrc_h_desc* d, double alpha, int op, const double* x, double* y);

#define CHECK(call)                                                                    \
    do {                                                                               \
        hlrc_status st_ = (call);                                                      \
        if (st_ != HLRC_OK) {                                                          \
            fprintf(stderr, "%s failed (%d): %s\n", #call, (int)st_, hlrc_last_error()); \
            return 2;                                                                  \
        }                                                                              \
    } while (0)
#define CUDA(call)                                                                             \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess) {                                                               \
            fprintf(stderr, "%s failed: %s\n", #call, cudaGetErrorString(e_));                \
            return 2;                                                                          \
        }                                                                                      \
    } while (0)

static double rel_err(const double* a, const double* b, int64_t n) {
    double d = 0, r = 0;
    for (int64_t i = 0; i < n; ++i) {
        d += (a[i] - b[i]) * (a[i] - b[i]);
        r += b[i] * b[i];
    }
    return sqrt(d / (r > 0 ? r : 1));
}

/* x ~ deterministic pseudo-random values in [-1, 1) */
static void fill(double* x, int64_t n, unsigned seed) {
    unsigned s = seed * 2654435761u + 1u;
    for (int64_t i = 0; i < n; ++i) {
        s = s * 1664525u + 1013904223u;
        x[i] = (double)(s >> 8) / (double)(1u << 23) - 1.0;
    }
}

int main(int argc, char** argv) {
    const int dry = argc > 1 && strcmp(argv[1], "--dry") == 0;
    hlrc_problem p;
    memset(&p, 0, sizeof(p));
    p.kind = HLRC_PROBLEM_EXP3D;
    p.leaf_size = 64;
    p.n = 8192;
    p.seed = 1;
    p.eta = 2.0;
    p.eps = 1e-6;
    p.ell = 0.1;
    p.nugget = 1e-4;
    hlrc_hbuild B = NULL;
    CHECK(hlrc_build(&p, &B));
    hlrc_h_desc d;
    CHECK(hlrc_build_h_desc(B, &d));
    hlrc_info info;
    CHECK(hlrc_plan_info_h(&d, NULL, &info));
    printf("n %lld leaves %lld matrix_bytes %lld scratch_bytes %lld\n", (long long)info.n_rows,
           (long long)(info.n_dense + info.n_lowrank), (long long)info.matrix_bytes, (long long)info.scratch_bytes);
    if (info.scratch_bytes <= 0 || info.matrix_bytes <= 0) return 1;
    if (dry) {
        CHECK(hlrc_build_free(B));
        printf("dry run ok\n");
        return 0;
    }

    const int64_t n = d.nrows;
    const int nrhs = 3;   /* several vectors per product: ld = n */
    hlrc_hmat M = NULL;
    hlrc_options o;
    hlrc_default_options(&o);
    o.max_nrhs = nrhs;
    CHECK(hlrc_upload_h(&d, &o, &M));
    hlrc_workspace W[2] = {NULL, NULL};
    CHECK(hlrc_workspace_create(M, nrhs, &W[0]));
    CHECK(hlrc_workspace_create(M, 1, &W[1]));
    cudaStream_t s[2];
    CUDA(cudaStreamCreateWithFlags(&s[0], cudaStreamNonBlocking));
    CUDA(cudaStreamCreateWithFlags(&s[1], cudaStreamNonBlocking));

    const size_t bytes = (size_t)n * nrhs * sizeof(double);
    double *hx[2], *hy[2], *dx[2], *dy[2];
    const double alpha[2] = {2.0, -0.75};
    const int op[2] = {HLRC_OP_N, HLRC_OP_T};
    const int vecs[2] = {nrhs, 1};
    for (int k = 0; k < 2; ++k) {
        hx[k] = (double*)malloc(bytes);
        hy[k] = (double*)calloc((size_t)n * nrhs, sizeof(double));
        fill(hx[k], n * nrhs, 7u + (unsigned)k);
        CUDA(cudaMalloc((void**)&dx[k], bytes));
        CUDA(cudaMalloc((void**)&dy[k], bytes));
        CUDA(cudaMemcpy(dx[k], hx[k], bytes, cudaMemcpyHostToDevice));
        CUDA(cudaMemset(dy[k], 0, bytes));
    }
    /* interleave several products on both streams; each stream owns its
       workspace, the handle is shared */
    const int reps = 5;
    for (int r = 0; r < reps; ++r)
        for (int k = 0; k < 2; ++k)
            CHECK(hlrc_mvm_ws(M, W[k], alpha[k], op[k], dx[k], dy[k], vecs[k], n, n, s[k]));
    CUDA(cudaStreamSynchronize(s[0]));
    CUDA(cudaStreamSynchronize(s[1]));

    double worst = 0;
    double* yref = (double*)malloc((size_t)n * sizeof(double));
    for (int k = 0; k < 2; ++k) {
        CUDA(cudaMemcpy(hy[k], dy[k], bytes, cudaMemcpyDeviceToHost));
        for (int j = 0; j < vecs[k]; ++j) {
            memset(yref, 0, (size_t)n * sizeof(double));
            if (oracle_hmvm_seq(&d, alpha[k] * reps, op[k], hx[k] + (size_t)j * n, yref) != 0) return 2;
            const double e = rel_err(hy[k] + (size_t)j * n, yref, n);
            printf("stream %d op %d vector %d: rel. error %.3e vs oracle\n", k, op[k], j, e);
            if (e > worst) worst = e;
        }
    }
    for (int k = 0; k < 2; ++k) {
        CHECK(hlrc_workspace_free(W[k]));
        cudaFree(dx[k]);
        cudaFree(dy[k]);
        cudaStreamDestroy(s[k]);
        free(hx[k]);
        free(hy[k]);
    }
    free(yref);
    CHECK(hlrc_free(M));
    CHECK(hlrc_build_free(B));
    printf("worst %.3e\n", worst);
    return worst <= 1e-13 ? 0 : 1;
}
