// Internal: the context object behind the C ABI, and the enqueue helpers the
// operator layer shares with capi.cu (not exported).
#pragma once
#include <cstdint>
#include <mutex>

#include "cufhedb_b200.h"
#include "fft_f32.cuh"
#include "fft_f64.cuh"
#include "fft1024_f64.cuh"
#include "pbs_common.cuh"

using namespace cfdb;

struct cufhedb_ctx {
    int device = 0;
    int num_sms = 0;
    Fft512Tables *tab512 = nullptr;   // device copy of the lvl1 transform tables
    Fft512TablesF *tab512f = nullptr; // the same tables in FP32 (split-precision path)
    float4 *bk01_split = nullptr;     // split-precision lvl01 key (hi/lo limbs, FP32)
    Fft1024Tables *tab1024 = nullptr; // lvl2 transform tables
    double2 *bk02 = nullptr;          // FFT-domain lvl02 key, chunk layout
    uint64_t *bk02_int = nullptr;     // integer lvl02 key (when loaded or generated)
    double2 *bk01 = nullptr;          // FFT-domain lvl01 key, chunk layout
    uint32_t *bk01_int = nullptr;     // integer lvl01 key (when loaded or generated)
    uint32_t *ksk[3] = {nullptr, nullptr, nullptr};   // lvl10, lvl20, lvl21
    int *err = nullptr;               // device failure word
    cudaStream_t io = nullptr;        // stream of the host-buffer entry points
    std::mutex io_mu;
    bool have_sk = false;
    // measured time of one full pass of each launch shape (PBS01_SHAPES per
    // precision FP64 / split / split with the tensor-core stage, PBS02_SHAPES);
    // all equal until the autotuner runs
    float pbs01_pass_ms[3][NSHAPES] = {{1.0f, 1.0f, 1.0f}, {1.0f, 1.0f, 1.0f}, {1.0f, 1.0f, 1.0f}};
    float pbs02_pass_ms[NSHAPES] = {1.0f, 1.0f, 1.0f};
    uint32_t *s0_d = nullptr, *s1_d = nullptr;
    uint64_t *s2_d = nullptr;
    // device address of the allocation-free gate's fixed intermediate
    // (noalloc.cu), looked up when the context is created
    uint32_t *noalloc_scratch = nullptr;
};

namespace cfdb {
// Makes `dev` the calling thread's current device for the guard's lifetime
// and gives the caller back its own current device afterwards.
struct DeviceGuard {
    int prev = -1;
    DeviceGuard() = default;
    explicit DeviceGuard(int dev) { set(dev); }
    DeviceGuard(const DeviceGuard &) = delete;
    DeviceGuard &operator=(const DeviceGuard &) = delete;
    cudaError_t set(int dev)
    {
        int cur = -1;
        cudaError_t e = cudaGetDevice(&cur);
        if (e != cudaSuccess) return e;
        if (cur == dev) return cudaSuccess;
        e = cudaSetDevice(dev);
        if (e == cudaSuccess && prev < 0) prev = cur;
        return e;
    }
    ~DeviceGuard()
    {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

// Device buffers that kernels read or write as w-byte words must start on a
// w-byte boundary (a misaligned word access is a device fault, which loses the
// context): every entry point checks its buffers and refuses misaligned ones.
inline bool aligned_to(const void *p, size_t w) { return ((uintptr_t)p % w) == 0; }

// device address of the allocation-free gate's intermediate on the current
// device (noalloc.cu); loads that module, so the array is reserved then
cudaError_t noalloc_scratch_address(uint32_t **out);
int set_error(int code, const char *msg);
int cuda_error(cudaError_t e, const char *what);
// PBS01 / PBS02 of a device batch with an optional constant added to each output's b
int pbs01_run(cufhedb_ctx *ctx, const uint32_t *in, uint32_t *out, int B, const TestVec &tv, uint32_t b_add,
              int precision, cudaStream_t st);
int pbs02_run(cufhedb_ctx *ctx, const uint32_t *in, uint64_t *out, int B, const TestVec &tv, uint64_t b_add,
              cudaStream_t st);
// IKS of a device batch; kind 10 (32-bit input, optional second input and offset)
// or 20 / 21 (64-bit input, offset added to b before rescaling)
int iks_run(cufhedb_ctx *ctx, int kind, const void *in, const uint32_t *in_b, int sa, int sb, uint64_t offset,
            uint32_t *out, int B, cudaStream_t st);
}  // namespace cfdb
