// Device roofs measured by the library itself, for the roofline reports of
// its products.  No counterpart in the reference.
//
// hlrc_fp64_peak: the FP64 tensor-core (DMMA) throughput.  Every warp runs a
// register-resident chain of mma.sync m8n8k4 f64 instructions (512 flops
// each) on eight independent accumulators, so the pipe, not memory or
// latency, bounds the loop; CUDA events time one launch after a warm-up.
// This is the compute roof of FP64 products with several right-hand sides
// (the 8-vector DMMA kernels), whose arithmetic intensity grows with the
// vector count: roof = min(HBM bandwidth x intensity, this peak).
#include <cuda_runtime.h>

#include "common.hpp"
#include "hlrc.h"

namespace {

// one m8n8k4 FP64 MMA, d += a b (the kernels' headers define kernels, so
// this file keeps its own copy of the instruction wrapper)
__device__ __forceinline__ void dmma(double (&d)[2], double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                 : "+d"(d[0]), "+d"(d[1])
                 : "d"(a), "d"(b));
}

__global__ void __launch_bounds__(256) k_fp64_peak(int iters, double* sink) {
    double d[8][2];
#pragma unroll
    for (int j = 0; j < 8; ++j) d[j][0] = d[j][1] = 0.0;
    const double a = 1e-3 * double(threadIdx.x + 1), b = 1.0 + 1e-6 * double(blockIdx.x);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int j = 0; j < 8; ++j) dmma(d[j], a, b);
    }
    double s = 0.0;
#pragma unroll
    for (int j = 0; j < 8; ++j) s += d[j][0] + d[j][1];
    if (s == -1.0) sink[0] = s;   // never true: keeps the chain alive
}

}  // namespace

extern "C" hlrc_status hlrc_fp64_peak(int device, double* tflops) {
    using hlrc::fail;
    hlrc::clear_error();
    if (!tflops) return fail(HLRC_ERR_ARG, "hlrc_fp64_peak: tflops is NULL");
    *tflops = 0.0;
    int prev = -1;
    if (cudaGetDevice(&prev) != cudaSuccess) return fail(HLRC_ERR_CUDA, "cudaGetDevice failed");
    if (device >= 0 && cudaSetDevice(device) != cudaSuccess) return fail(HLRC_ERR_CUDA, "cannot select device %d", device);
    int dev = device >= 0 ? device : prev, sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int blocks = 4 * (sms > 0 ? sms : 148), threads = 256;
    double* sink = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    hlrc_status st = HLRC_OK;
    float ms = 0.f;
    int iters = 1 << 12;
    if (cudaMalloc(&sink, sizeof(double)) != cudaSuccess || cudaEventCreate(&e0) != cudaSuccess ||
        cudaEventCreate(&e1) != cudaSuccess) {
        st = fail(HLRC_ERR_CUDA, "hlrc_fp64_peak: setup failed");
    } else {
        k_fp64_peak<<<blocks, threads>>>(iters, sink);   // warm-up, and a first estimate
        for (int rep = 0; rep < 3 && st == HLRC_OK; ++rep) {
            cudaEventRecord(e0);
            k_fp64_peak<<<blocks, threads>>>(iters, sink);
            cudaEventRecord(e1);
            if (cudaEventSynchronize(e1) != cudaSuccess) { st = fail(HLRC_ERR_CUDA, "hlrc_fp64_peak: launch failed"); break; }
            cudaEventElapsedTime(&ms, e0, e1);
            if (ms >= 100.f) break;
            iters = int(double(iters) * 150.0 / double(ms > 0.01f ? ms : 0.01f));   // aim at ~150 ms
            if (iters > (1 << 24)) iters = 1 << 24;
        }
    }
    if (st == HLRC_OK && ms > 0.f) {
        const double flops = double(blocks) * (threads / 32) * double(iters) * 8.0 * 512.0;
        *tflops = flops / (double(ms) * 1e-3) / 1e12;
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(sink);
    if (prev >= 0) cudaSetDevice(prev);
    return st;
}
