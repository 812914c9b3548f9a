// Diagnostic: measured CUDA-core FMA throughput of this device, the
// denominator of the PBS roofline (the driver-measured peaks cover HBM copy
// and bf16 tensor GEMMs only).  Each thread runs 8 independent FMA chains so
// the pipe, not the dependency latency, sets the rate.
#include <cuda_runtime.h>

#include "cufhedb_b200.h"

namespace {

template <typename T>
__global__ void fma_loop(T *out, int iters, T a, T b)
{
    T x[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) x[k] = (T)(threadIdx.x + k);
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < 8; ++k) x[k] = x[k] * a + b;
    }
    T s = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) s += x[k];
    if (s == (T)-1.2345) out[0] = s;   // keeps the chains live
}

}  // namespace

extern "C" CUFHEDB_API int cufhedb_measure_fma_peak(int device, int fp64, double *tflops)
{
    if (!tflops) return CUFHEDB_ERR_ARG;
    int prev = -1;
    if (cudaGetDevice(&prev) != cudaSuccess) return CUFHEDB_ERR_CUDA;
    // the caller's current device is given back on every return below
    struct Restore {
        int dev;
        ~Restore() { cudaSetDevice(dev); }
    } restore{prev};
    if (cudaSetDevice(device) != cudaSuccess) return CUFHEDB_ERR_CUDA;
    cudaDeviceProp p;
    if (cudaGetDeviceProperties(&p, device) != cudaSuccess) return CUFHEDB_ERR_CUDA;
    const int blocks = p.multiProcessorCount * 8, threads = 256, iters = 1 << 14;
    void *out = nullptr;
    if (cudaMalloc(&out, 16) != cudaSuccess) return CUFHEDB_ERR_OOM;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 1e30f;
    for (int rep = 0; rep < 4; ++rep) {
        cudaEventRecord(e0);
        if (fp64) fma_loop<double><<<blocks, threads>>>((double *)out, iters, 0.999999, 1e-7);
        else fma_loop<float><<<blocks, threads>>>((float *)out, iters, 0.999999f, 1e-7f);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0 && ms < best) best = ms;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (cudaGetLastError() != cudaSuccess) return CUFHEDB_ERR_CUDA;
    const double flop = 2.0 * 8.0 * iters * (double)blocks * threads;
    *tflops = flop / (best * 1e-3) / 1e12;
    return CUFHEDB_OK;
}
