// Stage 1 of the split-precision forward transform on the 5th-generation
// tensor cores (tcgen05), for the lvl01 PBS kernel's SPLIT32_TC path.
//
// In the FP32 transform (fft_f32.cuh) lane L of a warp holds, for one digit
// polynomial, x[m2] = d(L + 32 m2) + i d(L + 32 m2 + 512), m2 < 16, the signed
// Bg = 2^6 digits (|d| <= 32, exact in FP16), and its first step is
//   X[q] = sum_m2 x[m2] e^{2 pi i m2 / 64} e^{2 pi i m2 q / 16}
//        = sum_m2 x[m2] e^{2 pi i m2 (1 + 4 q) / 64},       q < 16
// (the per-register part of the twist, cw64, then the 16-point DFT fdft16).
// Over the 32 lanes that is a product of a 32 x 32 real matrix A (row = lane;
// columns: the 16 real, then the 16 imaginary parts of x) with a constant
// 32 x 32 real matrix B (output columns: the 16 real, then the 16 imaginary
// parts of X):
//   B[m][q] = c,  B[m][16 + q] = s,  B[16 + m][q] = -s,  B[16 + m][16 + q] = c,
//   c + i s = e^{2 pi i m (1 + 4 q) / 64}.
// B is split into two FP16 limbs, B = Bhi + Blo (Bhi = fp16(B), Blo =
// fp16(B - Bhi): |B - Bhi - Blo| <= 2^-23), and each warp computes
// D = A Bhi + A Blo with kind::f16 MMAs accumulating in FP32 in tensor memory:
// the products of the exact digits with the limbs are exact in FP32, so D
// carries FP32 accumulation rounding only, as the CUDA-core stage does.
//
// The consumer warps work in groups of four (one per sub-partition).  A group
// has its own 256 tensor-memory columns: D for the six digit polynomials of a
// CMux (6 x 32 FP32 columns, each on a 32-column boundary) and A for the
// three digits of one polynomial (3 x 16 columns: 32 FP16 per row, two per
// 32-bit column).  Each warp writes its 32 rows into the 32 lanes of its
// sub-partition (tcgen05.st), the group meets at a named barrier, one lane of
// its first warp issues a polynomial's M = 128 MMAs (A from tensor memory, B
// from shared memory) for all four warps and commits them to that
// polynomial's mbarrier, and each warp reads its own 32 rows of D back
// (tcgen05.ld).
#pragma once
#include <cuda_fp16.h>

#include <cmath>
#include <cstdint>
#include <cstring>

#include "common.cuh"

namespace cfdb {

// one limb of B: 32 (N) x 32 (K) FP16 in the canonical K-major layout without
// swizzle: 8-row x 16-byte core matrices, K-adjacent ones 128 bytes apart
// (leading byte offset), 8-row groups 512 bytes apart (stride byte offset)
constexpr int TC_B_HALVES = 32 * 32;
constexpr uint32_t TC_B_LBO = 128, TC_B_SBO = 512;

__host__ __device__ inline int tc_b_index(int n, int k)
{
    return (n / 8) * (int)(TC_B_SBO / 2) + (k / 8) * (int)(TC_B_LBO / 2) + (n % 8) * 8 + (k % 8);
}

// the two limbs of B as FP16 bit patterns, in tc_b_index order (host)
inline void build_stage1_b(uint16_t hi[TC_B_HALVES], uint16_t lo[TC_B_HALVES])
{
    const long double pi = 3.141592653589793238462643383279502884L;
    for (int k = 0; k < 32; ++k)
        for (int n = 0; n < 32; ++n) {
            const int m = k % 16, q = n % 16;
            const long double ang = 2.0L * pi * (long double)(m * (1 + 4 * q)) / 64.0L;
            const double c = (double)cosl(ang), s = (double)sinl(ang);
            const double v = (k < 16) ? (n < 16 ? c : s) : (n < 16 ? -s : c);
            const __half h = __float2half_rn((float)v);
            const __half l = __float2half_rn((float)(v - (double)__half2float(h)));
            std::memcpy(&hi[tc_b_index(n, k)], &h, 2);
            std::memcpy(&lo[tc_b_index(n, k)], &l, 2);
        }
}

// instruction descriptor of kind::f16: D FP32, A and B FP16, both K-major,
// N = 32, M = 128 (bits: D format [4,6), A format [7,10), B format [10,13),
// A / B major 15 / 16, N >> 3 at [17,23), M >> 4 at [24,29))
constexpr uint32_t TC_IDESC = (1u << 4) | ((32u >> 3) << 17) | ((128u >> 4) << 24);

// shared-memory matrix descriptor: start address, leading / stride byte
// offsets (all >> 4), descriptor version 1 at bit 46, no swizzle
__device__ __forceinline__ uint64_t tc_smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// ---- tensor-memory allocation (one whole warp) ------------------------------
__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// this lane's 16 32-bit columns at taddr (lane field = the warp's
// sub-partition); tmem_wait_st() before anything reads them
__device__ __forceinline__ void tmem_st16(uint32_t taddr, const uint32_t v[16])
{
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
        "%14, %15, %16};" ::"r"(taddr),
        "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7]), "r"(v[8]),
        "r"(v[9]), "r"(v[10]), "r"(v[11]), "r"(v[12]), "r"(v[13]), "r"(v[14]), "r"(v[15])
        : "memory");
}
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t v[32])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
        "%14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
          "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
          "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// D (+)= A B, A from tensor memory, B from shared memory (one thread)
__device__ __forceinline__ void umma_ts(uint32_t d_tmem, uint32_t a_tmem, uint64_t b_desc, uint32_t accumulate)
{
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %3, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], [%1], %2, %4, p;\n}\n" ::"r"(d_tmem),
        "r"(a_tmem), "l"(b_desc), "r"(accumulate), "r"(TC_IDESC)
        : "memory");
}

// the mbarrier completes one phase when this thread's MMAs so far are done
__device__ __forceinline__ void umma_commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

// The A row of digit polynomial d (0..2) from the cached decomposition words
// (digit_words1 layout: w[2 m2] for coefficient L + 32 m2, w[2 m2 + 1] for
// L + 32 m2 + 512) as 16 FP16 pairs, K order: x_re[0..15], then x_im[0..15],
// the lower K index in the low half of each 32-bit column.
__device__ __forceinline__ void tc_a_row(uint32_t a[16], const uint32_t w[32], int d)
{
#pragma unroll
    for (int c = 0; c < 16; ++c) {
        const int h = c >> 3, m2 = 2 * (c & 7);
        const float lo = (float)digit_field1(w[2 * m2 + h], d);
        const float hi = (float)digit_field1(w[2 * (m2 + 1) + h], d);
        const __half2 p = __floats2half2_rn(lo, hi);
        a[c] = *reinterpret_cast<const uint32_t *>(&p);
    }
}

}  // namespace cfdb
