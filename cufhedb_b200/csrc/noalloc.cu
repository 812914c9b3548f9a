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
//    cufhedb_ctx_create looks up its device address (which loads this file's
//    module, and so reserves the array) with the context's device current, so
//    the reservation happens when the context is created, never inside a call;
//  * every call on a device uses the same array: calls whose work overlaps on
//    the GPU (different streams, different contexts on one device, or
//    different host threads without ordering) race on it; order them on one
//    stream.  The array keeps the last call's contents; every word a call
//    reads is first written by that call.
#include <string>

#include "common.cuh"
#include "cufhedb_b200.h"
#include "ctx.cuh"

namespace cfdb {
int gate_enqueue_into(cufhedb_ctx *ctx, int gate, const uint32_t *ca, const uint32_t *cb, uint32_t *out, int B,
                      int precision, cudaStream_t st, uint32_t *scratch_lvl0);
}  // namespace cfdb

namespace {

constexpr int NOALLOC_MAX_GATES = 1024;

// the lvl0 intermediate of up to NOALLOC_MAX_GATES gates
static __device__ __align__(256) uint32_t g_gate_scratch[NOALLOC_MAX_GATES * (cfdb::N0 + 1)];

}  // namespace

namespace cfdb {

cudaError_t noalloc_scratch_address(uint32_t **out)
{
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_gate_scratch);
    *out = (e == cudaSuccess) ? static_cast<uint32_t *>(p) : nullptr;
    return e;
}

}  // namespace cfdb

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
    if (!ctx->noalloc_scratch) return cfdb::set_error(CUFHEDB_ERR_CUDA, "allocation-free intermediate not set up");
    cfdb::DeviceGuard guard;
    if (guard.set(ctx->device) != cudaSuccess) return cfdb::set_error(CUFHEDB_ERR_CUDA, "cudaSetDevice failed");
    return cfdb::gate_enqueue_into(ctx, gate, ca, cb, out, B, precision, (cudaStream_t)stream,
                                   ctx->noalloc_scratch);
}
