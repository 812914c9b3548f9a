// Shared-memory key ring of the persistent PBS kernels, without a producer
// warp.  The bootstrapping key streams through S slots of CHUNK bytes each
// (bulk copies completing on one mbarrier per slot).  Thread 0 issues the
// first S chunks; afterwards the last of the W consumer warps to release a
// slot refills it with the chunk S positions further on, so every warp of the
// block runs the math and the register file is shared by consumers only.
//
// Every wait is bounded: a consumer that gives up raises the block's abort
// flag, after which no warp waits and no chunk is issued; at the end thread 0
// waits (bounded) for the last copy issued into every slot, so no copy lands
// after the block has exited.
#pragma once
#include "common.cuh"

namespace cfdb {

struct RingHeader {
    static constexpr int MAX_S = 8;
    uint64_t full[MAX_S];   // per slot: the chunk's bytes have landed
    uint64_t empty[MAX_S];  // per slot: all consumers released it (producer-warp ring)
    int relcnt[MAX_S];      // releases seen by each slot (ring without producer)
    int issued[MAX_S];      // chunks issued into each slot
    int abort;              // set when any wait gave up
    int pad[7];
};
static_assert(sizeof(RingHeader) <= 256, "ring header");
constexpr int RING_HEADER_BYTES = 256;

template <int S, int CHUNK, int W>
struct KeyRing {
    static_assert(S <= RingHeader::MAX_S, "ring depth");
    RingHeader *h;
    unsigned char *slots;       // S x CHUNK bytes, 128-byte aligned
    const unsigned char *src;   // the key: `per_pass` chunks, CHUNK bytes each
    uint32_t per_pass;          // chunks in one pass over the key
    uint32_t total;             // chunks this block consumes (passes x per_pass)
    uint32_t limit = WAIT_LIMIT;   // polls per bounded wait

    __device__ __forceinline__ void init_by_thread0()
    {
        h->abort = 0;
        for (int s = 0; s < S; ++s) {
            mbar_init(&h->full[s], 1);
            h->relcnt[s] = 0;
            h->issued[s] = 0;
        }
        fence_barrier_init();
    }

    __device__ __forceinline__ void issue(uint32_t ch)
    {
        const int s = ch % S;
        ++h->issued[s];
        mbar_arrive_expect_tx(&h->full[s], CHUNK);
        bulk_g2s(slots + (size_t)s * CHUNK, src + (size_t)(ch % per_pass) * CHUNK, CHUNK, &h->full[s]);
    }

    // after __syncthreads() following init
    __device__ __forceinline__ void prologue_by_thread0()
    {
        for (uint32_t ch = 0; ch < (uint32_t)S && ch < total; ++ch) issue(ch);
    }

    __device__ __forceinline__ bool aborted() const { return *(volatile int *)&h->abort != 0; }

    // waits for chunk c; returns its slot's data
    __device__ __forceinline__ const unsigned char *acquire(uint32_t c, int *err)
    {
        const int s = c % S;
        if (!aborted() && !mbar_wait(&h->full[s], (c / S) & 1, limit)) {
            report_error(err, DEV_TIMEOUT_FULL);
            *(volatile int *)&h->abort = 1;
        }
        return slots + (size_t)s * CHUNK;
    }

    // One call per warp after its last read of chunk c (all lanes; lane 0
    // acts).  The slot's counter counts releases; the warp whose release is
    // the W-th for this use of the slot refills it with chunk c + S without
    // waiting for anyone (ring_release orders every warp's reads first).
    __device__ __forceinline__ void release(uint32_t c, int lane)
    {
        __syncwarp();
        if (lane == 0) {
            const int s = c % S;
            if (ring_release(&h->relcnt[s], c / S, W) && c + S < total && !aborted()) {
                fence_proxy_async_smem();
                issue(c + S);
            }
        }
    }

    // after the block's final __syncthreads()
    __device__ __forceinline__ void drain_by_thread0(int *err)
    {
        if (!aborted()) return;
        for (int s = 0; s < S; ++s)
            if (h->issued[s] > 0 && !mbar_wait(&h->full[s], (uint32_t)(h->issued[s] - 1) & 1, limit))
                report_error(err, DEV_TIMEOUT_DRAIN);
    }
};

// The same ring fed by a dedicated producer warp (one elected lane): it
// waits for each slot's `empty` barrier (all W consumers released the slot)
// and issues the next chunk at once.  Costs a warp slot but takes the
// refill latency off the consumers; which form is faster depends on the
// kernel, so both exist.
template <int S, int CHUNK, int W>
struct ProducerRing {
    static_assert(S <= RingHeader::MAX_S, "ring depth");
    RingHeader *h;
    unsigned char *slots;
    const unsigned char *src;
    uint32_t per_pass;
    uint32_t total;

    __device__ __forceinline__ void init_by_thread0()
    {
        h->abort = 0;
        for (int s = 0; s < S; ++s) {
            mbar_init(&h->full[s], 1);
            mbar_init(&h->empty[s], W);
        }
        fence_barrier_init();
    }

    __device__ __forceinline__ bool aborted() const { return *(volatile int *)&h->abort != 0; }

    // the producer warp's whole job (lane 0 acts); drains its own copies
    __device__ __forceinline__ void run_producer(int lane, int *err)
    {
        if (lane != 0) return;
        uint32_t c = 0;
        for (; c < total && !aborted(); ++c) {
            const int s = c % S;
            if (c >= (uint32_t)S && !mbar_wait(&h->empty[s], ((c / S) - 1) & 1)) {
                report_error(err, DEV_TIMEOUT_EMPTY);
                *(volatile int *)&h->abort = 1;
                break;
            }
            mbar_arrive_expect_tx(&h->full[s], CHUNK);
            bulk_g2s(slots + (size_t)s * CHUNK, src + (size_t)(c % per_pass) * CHUNK, CHUNK, &h->full[s]);
        }
        // no copy may still be in flight when the block exits
        for (uint32_t k = (c > (uint32_t)S ? c - S : 0); k < c; ++k)
            if (!mbar_wait(&h->full[k % S], (k / S) & 1)) report_error(err, DEV_TIMEOUT_DRAIN);
    }

    __device__ __forceinline__ const unsigned char *acquire(uint32_t c, int *err)
    {
        const int s = c % S;
        if (!aborted() && !mbar_wait(&h->full[s], (c / S) & 1)) {
            report_error(err, DEV_TIMEOUT_FULL);
            *(volatile int *)&h->abort = 1;
        }
        return slots + (size_t)s * CHUNK;
    }

    __device__ __forceinline__ void release(uint32_t c, int lane)
    {
        __syncwarp();
        if (lane == 0) mbar_arrive(&h->empty[c % S]);
    }
};

// number of groups block `b` of `grid` processes out of `ngroups` (round robin)
__device__ __forceinline__ int groups_of_block(int ngroups, int b, int grid)
{
    return b < ngroups ? (ngroups - 1 - b) / grid + 1 : 0;
}

}  // namespace cfdb
