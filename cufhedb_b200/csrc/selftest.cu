// Self-test of the bounded waits: a key ring (ring.cuh) whose first chunk is
// never issued, so every consumer's wait for it runs out.  The kernel must
// then record DEV_TIMEOUT_FULL in the context's error word, raise the ring's
// abort flag so that no other warp waits, skip the refill, skip the drain
// (nothing was issued) and return; the host reads the code through
// cufhedb_sync and the context stays usable.  No copy is issued and no
// memory outside the block's own shared memory is touched.
#include "ctx.cuh"
#include "ring.cuh"

namespace cfdb {

namespace {

constexpr int ST_S = 2, ST_CHUNK = 16, ST_W = 2;

__global__ void __launch_bounds__(ST_W * 32) ring_timeout_selftest_kernel(int *err, uint32_t limit)
{
    __shared__ __align__(128) unsigned char smem[RING_HEADER_BYTES + ST_S * ST_CHUNK];
    KeyRing<ST_S, ST_CHUNK, ST_W> ring{reinterpret_cast<RingHeader *>(smem), smem + RING_HEADER_BYTES, nullptr, 1u,
                                       2u, limit};
    const int lane = threadIdx.x & 31;
    if (threadIdx.x == 0) ring.init_by_thread0();
    __syncthreads();
    // no prologue: chunk 0 never lands
    ring.acquire(0, err);
    ring.release(0, lane);
    __syncthreads();
    if (threadIdx.x == 0) ring.drain_by_thread0(err);
}

}  // namespace

}  // namespace cfdb

using namespace cfdb;

int cufhedb_selftest_wait_timeout(cufhedb_ctx *ctx, uint32_t polls)
{
    if (!ctx) return set_error(CUFHEDB_ERR_ARG, "ctx is null");
    if (polls == 0 || polls > (1u << 20)) return set_error(CUFHEDB_ERR_ARG, "polls must be in [1, 2^20]");
    DeviceGuard guard(ctx->device);
    ring_timeout_selftest_kernel<<<1, ST_W * 32>>>(ctx->err, polls);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_error(e, "wait self-test launch");
    return cufhedb_sync(ctx, nullptr);
}
