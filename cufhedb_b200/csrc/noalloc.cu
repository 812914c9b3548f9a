// Allocation-free variant of the batched two-input gate (cufhedb_gate_lvl1).
//
// cufhedb_gate_lvl1 takes its key-switched lvl0 intermediate (B x 673 words)
// from the stream-ordered allocator on every call.  Some callers cannot let a
// library allocate device memory while they run: a database engine that
// reserves and accounts for all device memory when it starts, or a host
// process whose allocator owns the device and treats any other allocation as
// an error.  cufhedb_gate_lvl1_noalloc serves them: its intermediate lives in
// one fixed array in this file, so a call allocates nothing on the device or
// the host.
//
// Limits and sharing:
//  * at most NOALLOC_MAX_GATES gates per call (larger batches are rejected
//    with CUFHEDB_ERR_ARG; split them into several calls);
//  * the array (NOALLOC_MAX_GATES x 673 x 4 bytes = 2.63 MiB) exists once per
//    GPU that loads this library and stays reserved until the process exits;
//  * every call on a device uses the same array: calls whose work overlaps on
//    the GPU (different streams, or different host threads without ordering)
//    race on it; order them on one stream.  The array keeps the last call's
//    contents; every word a call reads is first written by that call.
//  * the first call on each device looks up the device address of the array
//    (cudaGetSymbolAddress) with that device current; make that first call
//    before any stream capture begins.
#include <mutex>
#include <string>

#include "common.cuh"
#include "cufhedb_b200.h"

namespace cfdb {
int set_error(int code, const char *msg);
int ctx_device(const cufhedb_ctx *ctx);
int gate_enqueue_into(cufhedb_ctx *ctx, int gate, const uint32_t *ca, const uint32_t *cb, uint32_t *out, int B,
                      int precision, cudaStream_t st, uint32_t *scratch_lvl0);
}  // namespace cfdb

namespace {

constexpr int NOALLOC_MAX_GATES = 1024;
constexpr int kMaxDevices = 64;

// the lvl0 intermediate of up to NOALLOC_MAX_GATES gates
static __device__ __align__(256) uint32_t g_gate_scratch[NOALLOC_MAX_GATES * (cfdb::N0 + 1)];

std::mutex g_mu;
uint32_t *g_scratch_addr[kMaxDevices] = {};

// device address of g_gate_scratch on `dev` (current device), looked up once
int scratch_for(int dev, uint32_t **out)
{
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_addr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_gate_scratch);
        if (e != cudaSuccess) {
            std::string m = std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e);
            return cfdb::set_error(CUFHEDB_ERR_CUDA, m.c_str());
        }
        g_scratch_addr[dev] = static_cast<uint32_t *>(p);
    }
    *out = g_scratch_addr[dev];
    return CUFHEDB_OK;
}

}  // namespace

extern "C" CUFHEDB_API int cufhedb_gate_lvl1_noalloc(cufhedb_ctx *ctx, int gate, const uint32_t *ca,
                                                     const uint32_t *cb, uint32_t *out, int B, int precision,
                                                     cufhedb_stream_t stream)
{
    if (!ctx) return cfdb::set_error(CUFHEDB_ERR_ARG, "ctx is null");
    if (B < 0) return cfdb::set_error(CUFHEDB_ERR_ARG, "negative batch");
    if (B > NOALLOC_MAX_GATES)
        return cfdb::set_error(CUFHEDB_ERR_ARG,
                               "batch exceeds the allocation-free limit of 1024 gates per call; split the batch");
    if (B == 0) return CUFHEDB_OK;
    if (!ca || !cb || !out) return cfdb::set_error(CUFHEDB_ERR_ARG, "null buffer");
    const int dev = cfdb::ctx_device(ctx);
    if (dev < 0 || dev >= kMaxDevices) return cfdb::set_error(CUFHEDB_ERR_ARG, "device index out of range");
    if (cudaSetDevice(dev) != cudaSuccess) return cfdb::set_error(CUFHEDB_ERR_CUDA, "cudaSetDevice failed");
    uint32_t *scratch = nullptr;
    int rc = scratch_for(dev, &scratch);
    if (rc != CUFHEDB_OK) return rc;
    return cfdb::gate_enqueue_into(ctx, gate, ca, cb, out, B, precision, (cudaStream_t)stream, scratch);
}
