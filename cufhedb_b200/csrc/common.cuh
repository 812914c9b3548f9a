// Shared device-side definitions for the cufhedb_b200 PBS engine (sm_100a).
//
// Parameter set: the reference's default TFHEpp profile,
// thirdparty/TFHEpp/include/params/128bit.hpp:7-83.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace cfdb {

// lvl0 LWE, lvl1 / lvl2 TRLWE + gadget, key-switching parameters
constexpr int N0 = 672;
constexpr int N1 = 1024, L1 = 3, BGBIT1 = 6;
// per-warp transpose scratch of the 512-point transforms: 32 rows of 16
// values padded to 17 (fft_f64.cuh, fft_f32.cuh)
constexpr int FFT512_XP = 32 * 17;
constexpr int N2 = 2048, L2 = 4, BGBIT2 = 9;
constexpr int KS10_BASEBIT = 10, KS10_T = 2;
constexpr int KS20_BASEBIT = 10, KS20_T = 2;
constexpr int KS21_BASEBIT = 3, KS21_T = 10;
// Key-switching key rows live in HBM with their words padded to a multiple of
// four (16 bytes: lvl0 rows 673 -> 676 words, lvl1 rows 1025 -> 1028), the
// pad words zero, so that the gather reads each row with 16-byte loads.
__host__ __device__ constexpr int ksk_pitch(int row_words) { return (row_words + 3) & ~3; }

// gadget decomposition constants (thirdparty/TFHEpp/src/trgsw.cpp:9-39)
constexpr uint32_t DEC1_OFFSET = (32u << 26) + (32u << 20) + (32u << 14);   // sum Bg/2 * 2^(32-i*Bgbit)
constexpr uint32_t DEC1_ROUND = 1u << (32 - L1 * BGBIT1 - 1);
// Signed digit extraction: with x = (t + DEC1_OFFSET + DEC1_ROUND) ^ DEC1_XOR,
// digit d of t is the sign-extended 6-bit field of x at bit 32 - 6 (d + 1).
// ((u ^ 32) read as a signed 6-bit number is u - 32 for every 6-bit u, the
// "- Bg/2" of trgsw.cpp:31.)
constexpr uint32_t DEC1_XOR = (32u << 26) | (32u << 20) | (32u << 14);
constexpr uint64_t DEC2_OFFSET = (256ull << 55) + (256ull << 46) + (256ull << 37) + (256ull << 28);
constexpr uint64_t DEC2_ROUND = 1ull << (64 - L2 * BGBIT2 - 1);

// error codes written by kernels into the context's device error word
enum : int {
    DEV_OK = 0,
    DEV_TIMEOUT_FULL = 1,    // consumer gave up waiting for a key chunk
    DEV_TIMEOUT_EMPTY = 2,   // producer gave up waiting for a free ring slot
    DEV_TIMEOUT_DRAIN = 3,   // producer gave up waiting for its last copies
    DEV_TIMEOUT_MMA = 4,     // a warp gave up waiting for its tensor-core product
    DEV_TIMEOUT_ROW = 5,     // a warp gave up waiting for a TRGSW row it copies in
};

// bounded waits: polls of mbarrier.try_wait (each poll may suspend in hardware
// for a short system-defined time), ~ a few seconds at most
constexpr uint32_t WAIT_LIMIT = 1u << 24;

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// make mbarrier initialisation visible to the async (bulk-copy) proxy
__device__ __forceinline__ void fence_barrier_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// returns false if the phase did not complete within `limit` polls
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, uint32_t limit = WAIT_LIMIT)
{
    for (uint32_t it = 0; it < limit; ++it)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

// orders this thread's earlier generic-proxy shared-memory accesses before
// its later async-proxy ones (a bulk copy into memory just read)
__device__ __forceinline__ void fence_proxy_async_smem()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Release of a key-ring slot by one consumer warp (called by one lane): the
// slot's counter counts releases; true for the last of the `consumers`
// releases of the slot's `use`-th chunk, whose caller then refills the slot.
// The fences order every warp's reads of the slot before the refill.
__device__ __forceinline__ bool ring_release(int *cnt, uint32_t use, int consumers)
{
    __threadfence_block();
    const int old = atomicAdd(cnt, 1);
    const bool last = old == (int)(use + 1) * consumers - 1;
    if (last) __threadfence_block();
    return last;
}

// one bulk (TMA-engine) copy global -> this CTA's shared memory, completing
// `bytes` of transaction count on `bar`.  Both addresses 16-byte aligned,
// bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void *smem_dst, const void *gsrc, uint32_t bytes, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(smem_dst)),
        "l"(gsrc), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

// asks L2 to fetch [gsrc, gsrc + bytes) ahead of its use (no data returned;
// gsrc 16-byte aligned, bytes a multiple of 16)
__device__ __forceinline__ void bulk_prefetch_l2(const void *gsrc, uint32_t bytes)
{
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(gsrc), "r"(bytes) : "memory");
}
// the same for a buffer whose alignment the caller does not control (a hint:
// nothing is done unless gsrc is 16-byte aligned)
__device__ __forceinline__ void bulk_prefetch_l2_if_aligned(const void *gsrc, uint32_t bytes)
{
    if ((reinterpret_cast<uintptr_t>(gsrc) & 15u) == 0 && (bytes & 15u) == 0) bulk_prefetch_l2(gsrc, bytes);
}

// signed Bg-bit field d (0 = most significant) of x: two plain shifts, the
// field moved to the top and sign-extended back down
__device__ __forceinline__ int digit_field1(uint32_t x, int d)
{
    return (int)(x << (BGBIT1 * d)) >> (32 - BGBIT1);
}

__device__ __forceinline__ void report_error(int *err, int code)
{
    if (err) atomicCAS(err, 0, code);
}

// ---- complex helpers --------------------------------------------------------
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b)
{
    return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
// a * conj(b)
__device__ __forceinline__ double2 cmulc(double2 a, double2 b)
{
    return make_double2(fma(a.x, b.x, a.y * b.y), fma(a.y, b.x, -a.x * b.y));
}
// acc += a * b
__device__ __forceinline__ void cfma(double2 &acc, double2 a, double2 b)
{
    acc.x = fma(a.x, b.x, acc.x);
    acc.x = fma(-a.y, b.y, acc.x);
    acc.y = fma(a.x, b.y, acc.y);
    acc.y = fma(a.y, b.x, acc.y);
}

__device__ __forceinline__ double2 shfl_xor2(double2 v, int m)
{
    return make_double2(__shfl_xor_sync(0xffffffffu, v.x, m), __shfl_xor_sync(0xffffffffu, v.y, m));
}

}  // namespace cfdb
