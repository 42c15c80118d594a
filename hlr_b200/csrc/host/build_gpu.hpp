// Device assembly of the leaves of an H-matrix whose cluster and block
// trees were built on the host (build.cpp): dense leaves are evaluated from
// the kernel function, admissible leaves are approximated by ACA with
// maximum-pivot search and recompressed by QR + SVD, all on the GPU, with
// the results left in one device arena.
#pragma once

#include <cstdint>
#include <vector>

#include "hlrc.h"

namespace hlrc {

// The kernel function of a test problem (internal point order), host arrays.
struct GpuProblem {
    int kind = 0;
    int dim = 1;
    int64_t n = 0;
    const double* pts = nullptr;   // n x dim, row-major
    const double* wts = nullptr;   // LAPLACE_SPH: per-point weights, else null
    double ell = 0.1, nugget = 0.0, h = 0.0;
};

// One leaf: the index sets and kind in; rank and the element offsets of its
// data in the arena out (column-major: D nrows x ncols, U nrows x rank,
// V ncols x rank, sv rank singular values in descending order).
struct GpuLeaf {
    int64_t row0 = 0, nrows = 0, col0 = 0, ncols = 0;
    int kind = HLRC_LEAF_DENSE;
    int rank = 0;
    int64_t d = -1, u = -1, v = -1, s = -1;
};

// Largest ACA rank of one block on the device; a block whose approximation
// has not converged at this rank fails the build (HLRC_ERR_SHAPE).
constexpr int GPU_ACA_MAX_RANK = 128;

// Assembles every leaf on the current CUDA device.  On success *arena is a
// cudaMalloc'ed buffer of *arena_doubles doubles holding all leaf data (the
// caller frees it with cudaFree).
hlrc_status gpu_assemble(const GpuProblem& P, std::vector<GpuLeaf>& leaves, double eps, double** arena,
                         int64_t* arena_doubles);

// Copies n doubles from device memory to the host.
hlrc_status gpu_copy_to_host(double* dst, const double* src, int64_t n);
hlrc_status gpu_free(void* p);

}  // namespace hlrc
