// Batched lvl0 -> lvl1 programmable bootstrapping, split-precision FP32 path.
//
// Same algorithm as pbs01_f64.cu (TFHEpp GateBootstrappingTLWE2TLWEFFT
// <lvl01param>, src/gatebootstrapping.cpp:14-23), with every transform and
// product in FP32.  Precision plan (the 32-bit torus needs products exact to
// well below the bootstrapping noise, which FP32 alone cannot give):
//   * each integer key polynomial b is split into limbs
//       hi = round(b / 2^24) in [-128, 128],  lo = b - hi * 2^24 in [-2^23, 2^23);
//     both are transformed in FP64 on the device at key-load time and stored
//     as FP32 frequency values;
//   * per CMux the 6 digit polynomials (|d| <= 32) are transformed in FP32 and
//     multiplied into four FP32 accumulators (hi/lo x 2 output polynomials);
//   * the hi accumulators' inverse transforms are rounded to integers, which is
//     exact: sum_r d_r * hi_r has rms magnitude ~2^16.7, so FP32 round-off
//     (~2^-21.5 relative) leaves an error ~0.04, a 12-sigma margin below 1/2;
//     then hi * 2^24 is taken modulo 2^32;
//   * the lo accumulators' inverse transforms (rms ~2^32.7) are rounded to
//     64-bit integers; their FP32 round-off (~2^11) is ~2^-6 of the per-CMux
//     bootstrapping noise standard deviation (~2^17.8), i.e. it adds about
//     0.03 % to the noise variance.
// Kernel layout and key streaming are those of the FP64 kernel; the key ring
// slots hold (hi, lo) float pairs in the same 16 KB per TRGSW row.
#include "fft_f32.cuh"
#include "pbs_common.cuh"
#include "ring.cuh"
#include "tc_stage1.cuh"

#include <type_traits>

namespace cfdb {

template <int W, int S, int TBYTES>
struct Pbs01SplitSmem {
    static constexpr int RING_OFF = RING_HEADER_BYTES;
    static constexpr int CHUNK_BYTES = 16384;   // 16 slots x 2 outputs x 32 lanes x float4(hi, lo)
    static constexpr int TAB_OFF = RING_OFF + S * CHUNK_BYTES;
    static constexpr int WARP_OFF = TAB_OFF + (TBYTES + 127) / 128 * 128;
    static constexpr int XP_BYTES = FFT512_XP * 8;
    static constexpr int ACC_BYTES = 2 * N1 * 4;
    static constexpr int ABAR_BYTES = ((N0 * 2) + 127) / 128 * 128;
    static constexpr int PER_WARP = XP_BYTES + ACC_BYTES + ABAR_BYTES;
    // tensor-core stage 1 only: the two FP16 limbs of B, one mbarrier per
    // warp, the tensor-memory base address
    static constexpr int TC_OFF = (WARP_OFF + W * PER_WARP + 1023) / 1024 * 1024;
    static constexpr int TC_B_BYTES = 2 * TC_B_HALVES * 2;
    static constexpr int TC_BAR_OFF = TC_OFF + TC_B_BYTES;
    static constexpr int TC_SLOT_OFF = TC_BAR_OFF + 8 * 16;
    static constexpr int TOTAL_TC = TC_SLOT_OFF + 16;
    static constexpr int TOTAL = WARP_OFF + W * PER_WARP;
};

// the decomposition words of (X^a - 1) * poly, once per polynomial:
// w[2 m2 + h] = (((X^a - 1) poly)[m + 512 h] + offset + round) ^ DEC1_XOR,
// m = lane + 32 m2; each of the l = 3 digits is then a field of these words
__device__ __forceinline__ void digit_words1(uint32_t w[32], const uint32_t *poly, uint32_t abar, int lane)
{
#pragma unroll
    for (int m2 = 0; m2 < 16; ++m2) {
        const int m = lane + 32 * m2;
        w[2 * m2] = ((rot_coef<N1>(poly, m, abar) - poly[m]) + DEC1_OFFSET + DEC1_ROUND) ^ DEC1_XOR;
        w[2 * m2 + 1] = ((rot_coef<N1>(poly, m + 512, abar) - poly[m + 512]) + DEC1_OFFSET + DEC1_ROUND) ^ DEC1_XOR;
    }
}

// v[m2] = (dig_d(m) + i dig_d(m+512)) * w^{32 m2} from the cached words: the
// per-register part of the twist (ffft512_fwd_tw applies the lane's part)
__device__ __forceinline__ void digits_from_words_f(float2 v[16], const uint32_t w[32], int d)
{
#pragma unroll
    for (int m2 = 0; m2 < 16; ++m2) {
        const int d0 = digit_field1(w[2 * m2], d), d1 = digit_field1(w[2 * m2 + 1], d);
        v[m2] = cw64(make_float2((float)d0, (float)d1), m2);
    }
}

// round(h) * 2^24 mod 2^32 without a conversion instruction: adding
// 1.5 * 2^23 leaves round-to-nearest-even of h in the low mantissa bits
// (|h| < 2^22, ~40 standard deviations of the hi products), and the term
// needs only their low 8 bits.  Same bits as __float2int_rn(h) << 24, on the
// FMA and ALU pipes instead of the conversion unit (measured: 1,024 PBS
// 9.73 -> 9.41 ms, 1,184 in the 8-per-CTA shape 10.95 -> 10.5 ms; building
// the digits from their bits the same way measured slower in both shapes, so
// they keep the int -> float conversion)
__device__ __forceinline__ uint32_t hi_term(float h)
{
    return __float_as_uint(h + 12582912.0f) << 24;
}

// poly[m] += round(hi_m) * 2^24 + round(lo_m) (mod 2^32), one read-modify-write
// of the accumulator per polynomial.  f holds the hi and lo limbs of one
// output as pairs, inverse-transformed together.  The hi limb's products
// round exactly; the lo limb's FP32 error stays far below the bootstrapping
// noise.
__device__ __forceinline__ void add_inverse_split(uint32_t *poly, CP f[16], unsigned long long *xp, int lane,
                                                  const Fft512TablesFold &T)
{
    pfft512_inv<true>(f, xp, T, lane);
#pragma unroll
    for (int m2 = 0; m2 < 16; ++m2) {
        const int m = lane + 32 * m2;
        const CP y = untwist_m2(f[m2], m2);
        const float2 re = unpk2(y.re), im = unpk2(y.im);   // (hi, lo) of coefficients m and m + 512
        poly[m] += hi_term(re.x) + (uint32_t)__float2ll_rn(re.y);
        poly[m + 512] += hi_term(im.x) + (uint32_t)__float2ll_rn(im.y);
    }
}

// f += v * k for both limbs of one output: k = (hi.re, lo.re, hi.im, lo.im),
// vr = (v.re, v.re), vi = (v.im, v.im), nvi = (-v.im, -v.im)
__device__ __forceinline__ void pmac(CP &f, unsigned long long vr, unsigned long long vi, unsigned long long nvi,
                                     float4 k)
{
    const unsigned long long kr = pk2(k.x, k.y), ki = pk2(k.z, k.w);
    f.re = f2(nvi, ki, f2(vr, kr, f.re));
    f.im = f2(vi, kr, f2(vr, ki, f.im));
}
__device__ __forceinline__ CP pmul_first(unsigned long long vr, unsigned long long vi, unsigned long long nvi, float4 k)
{
    const unsigned long long kr = pk2(k.x, k.y), ki = pk2(k.z, k.w);
    return CP{f2(nvi, ki, m2(vr, kr)), f2(vi, kr, m2(vr, ki))};
}

// Tensor-core stage 1 (tc_stage1.cuh), shared by the warps of a group of
// four (warps 0-3 and 4-7; a producer warp takes no part), one polynomial at
// a time: when a polynomial's decomposition words are formed, each warp
// writes the A rows of all three of its digit polynomials into its own
// sub-partition's lanes of the group's A columns (the words are dead right
// after), the group meets at a named barrier, and one lane of the group's
// first warp issues the polynomial's three M = 128 products into three of the
// group's six D buffers and commits them to the polynomial's mbarrier.
// Polynomial 0's products are issued at the start of a CMux and taken at
// digit 0; polynomial 1's are issued at digit 1 (A is free again: every
// warp waited for polynomial 0's products at digit 0) and run under the
// transforms of digits 1 and 2.  Per group (256 columns): D 6 x 32 columns
// first, each on a 32-column boundary, then A 3 x 16.
// Every warp takes part in every step, active or not (a warp whose rotation
// is 0 for this CMux writes no rows and reads no result), so the barriers and
// the buffer reuse stay in step.  Addresses are recomputed from the block's
// shared memory and the warp index at each use (the kernel runs at the
// 255-register limit).
constexpr uint32_t TC_D_COLS = 6 * 32, TC_GROUP_COLS = 256;   // D at [0, 192), A at [192, 240)

template <class L, int W>
struct TcStage {
    unsigned char *smem;
    uint32_t phase;     // per polynomial (bits 0, 1): parity of its next completion

    __device__ __forceinline__ static int group(int warp) { return warp >> 2; }
    __device__ __forceinline__ uint32_t tbase() const
    {
        return *reinterpret_cast<const volatile uint32_t *>(smem + L::TC_SLOT_OFF);
    }
    __device__ __forceinline__ uint32_t lanes(int warp) const
    {
        return tbase() + TC_GROUP_COLS * group(warp) + ((32u * (warp & 3)) << 16);
    }
    __device__ __forceinline__ uint64_t *bar(int warp, int poly) const
    {
        return reinterpret_cast<uint64_t *>(smem + L::TC_BAR_OFF) + 2 * group(warp) + poly;
    }
    // A(d) <- the digit-d row of this lane, d < 3 (only when active), then the
    // group meets and its first warp issues D(3 poly + d) = A(d) (Bhi + Blo)
    __device__ __forceinline__ void put_issue(const uint32_t *w, bool active, int poly, int warp, int lane)
    {
        if (active) {
#pragma unroll 1
            for (int d = 0; d < L1; ++d) {
                uint32_t a[16];
                tc_a_row(a, w, d);
                tmem_st16(lanes(warp) + TC_D_COLS + 16 * d, a);
            }
            tmem_wait_st();
        }
        tc_fence_before();
        if (group(warp) == 0) asm volatile("bar.sync 2, %0;" ::"n"(32 * (W < 4 ? W : 4)) : "memory");
        else asm volatile("bar.sync 3, %0;" ::"n"(32 * (W > 4 ? W - 4 : 1)) : "memory");
        if ((warp & 3) == 0 && lane == 0) {
            tc_fence_after();
            const uint32_t gcol = tbase() + TC_GROUP_COLS * group(warp);
            const uint32_t b = smem_u32(smem + L::TC_OFF), limb = TC_B_HALVES * 2, kstep = 2 * TC_B_LBO;
#pragma unroll
            for (int d = 0; d < L1; ++d) {
                const uint32_t a = gcol + TC_D_COLS + 16 * d, dcol = gcol + 32 * (L1 * poly + d);
                umma_ts(dcol, a, tc_smem_desc(b, TC_B_LBO, TC_B_SBO), 0);
                umma_ts(dcol, a + 8, tc_smem_desc(b + kstep, TC_B_LBO, TC_B_SBO), 1);
                umma_ts(dcol, a, tc_smem_desc(b + limb, TC_B_LBO, TC_B_SBO), 1);
                umma_ts(dcol, a + 8, tc_smem_desc(b + limb + kstep, TC_B_LBO, TC_B_SBO), 1);
            }
            umma_commit(bar(warp, poly));
        }
        __syncwarp();
    }
    // waits for a polynomial's three products
    __device__ __forceinline__ void wait(int poly, int warp, int *err)
    {
        if (!mbar_wait(bar(warp, poly), (phase >> poly) & 1)) report_error(err, DEV_TIMEOUT_MMA);
        phase ^= 1u << poly;
        tc_fence_after();
    }
    // this lane's row of digit polynomial r's product (only when active):
    // v[q] = X[q]
    __device__ __forceinline__ void take(float2 v[16], bool active, int r, int warp)
    {
        if (active) {
            uint32_t x[32];
            tmem_ld32(lanes(warp) + 32 * r, x);
#pragma unroll
            for (int q = 0; q < 16; ++q) v[q] = make_float2(__uint_as_float(x[q]), __uint_as_float(x[16 + q]));
        }
        tc_fence_before();
        __syncwarp();
    }
};

template <int W>
constexpr uint32_t tc_cols()
{
    return ((W + 3) / 4) * TC_GROUP_COLS <= 256 ? 256u : 512u;
}
static_assert(2 * TC_GROUP_COLS <= 512 && TC_D_COLS + 3 * 16 <= TC_GROUP_COLS,
              "two groups' columns within one SM's tensor memory");

// W consumer warps, plus a producer warp when PRODUCER (ring.cuh has both
// feeds; the launch picks per shape, see launch_pbs01_split).  TC: the first
// step of every digit transform runs on the tensor cores (tc_stage1.cuh), the
// rest as in the CUDA-core path.
template <int W, int S, bool PRODUCER, bool TC>
__global__ void __launch_bounds__((W + (PRODUCER ? 1 : 0)) * 32, 1) pbs01_split_kernel(Pbs01Args a)
{
    // the folded tables (fft_f32.cuh): the twist and untwist ride on the
    // stage-1 twiddles, so the kernel reads 12.3 KB of tables instead of 24.4
    using TT = Fft512TablesFold;
    using L = Pbs01SplitSmem<W, S, (int)sizeof(TT)>;
    extern __shared__ __align__(128) unsigned char smem[];
    TT *T = reinterpret_cast<TT *>(smem + L::TAB_OFF);
    const int ngroups = (a.B + W - 1) / W;
    constexpr int CHUNKS = N0 * 2 * L1;
    using Feed = std::conditional_t<PRODUCER, ProducerRing<S, L::CHUNK_BYTES, W>, KeyRing<S, L::CHUNK_BYTES, W>>;
    Feed ring{reinterpret_cast<RingHeader *>(smem), smem + L::RING_OFF, reinterpret_cast<const unsigned char *>(a.bk),
              (uint32_t)CHUNKS, (uint32_t)groups_of_block(ngroups, blockIdx.x, gridDim.x) * CHUNKS};

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint64_t *tc_bars = reinterpret_cast<uint64_t *>(smem + L::TC_BAR_OFF);
    uint32_t *tc_slot = reinterpret_cast<uint32_t *>(smem + L::TC_SLOT_OFF);
    if (threadIdx.x == 0) {
        ring.init_by_thread0();
        if constexpr (TC) {
            for (int k = 0; k < 4; ++k) mbar_init(&tc_bars[k], 1);   // 2 groups x 2 buffers
            fence_barrier_init();
        }
    }
    if constexpr (TC) {
        if (warp == 0) tmem_alloc(tc_slot, tc_cols<W>());
    }
    {
        const Fft512TablesF *all = reinterpret_cast<const Fft512TablesF *>(a.tables);
        const float4 *src = reinterpret_cast<const float4 *>(&all->fold);
        float4 *dst = reinterpret_cast<float4 *>(T);
        for (int i = threadIdx.x; i < (int)(sizeof(TT) / 16); i += blockDim.x) dst[i] = src[i];
        if constexpr (TC) {
            const float4 *bs = reinterpret_cast<const float4 *>(&all->tc_b[0][0]);
            float4 *bd = reinterpret_cast<float4 *>(smem + L::TC_OFF);
            for (int i = threadIdx.x; i < L::TC_B_BYTES / 16; i += blockDim.x) bd[i] = bs[i];
            fence_proxy_async_smem();   // B is read by the tensor cores (async proxy)
        }
    }
    if constexpr (TC) tc_fence_before();
    __syncthreads();
    if constexpr (TC) tc_fence_after();
    if constexpr (PRODUCER) {
        if (warp == W) {
            ring.run_producer(lane, a.err);
            return;
        }
    } else {
        if (threadIdx.x == 0) ring.prologue_by_thread0();
    }

    TcStage<L, W> tc{smem, 0u};

    unsigned char *wb = smem + L::WARP_OFF + warp * L::PER_WARP;
    unsigned long long *xp = reinterpret_cast<unsigned long long *>(wb);
    uint32_t *acc = reinterpret_cast<uint32_t *>(wb + L::XP_BYTES);
    uint16_t *abar_s = reinterpret_cast<uint16_t *>(wb + L::XP_BYTES + L::ACC_BYTES);

    uint32_t c = 0;
    for (int g = blockIdx.x; g < ngroups; g += gridDim.x) {
        const int ct = g * W + warp;
        const bool valid = ct < a.B;
        uint32_t bbar = 2 * N1;
        if (valid) {
            const uint32_t *in = a.in + (size_t)ct * (N0 + 1);
            for (int i = lane; i < N0; i += 32) abar_s[i] = (uint16_t)((in[i] + (1u << 20)) >> 21);
            bbar = 2 * N1 - (in[N0] >> 21);
        }
        for (int j = lane; j < N1; j += 32) {
            acc[j] = 0;
            acc[N1 + j] = testvec_rot1(a.tv, j, bbar);
        }
        __syncwarp();
        if constexpr (TC) {
            // polynomial 0's products of CMux 0; those of every later CMux are
            // issued between the previous CMux's two inverse transforms
            const uint32_t ab0 = valid ? abar_s[0] : 0u;
            uint32_t w0[32];
            if (ab0) digit_words1(w0, acc, ab0, lane);
            tc.put_issue(w0, ab0 != 0, 0, warp, lane);
        }

        for (int i = 0; i < N0; ++i) {
            const uint32_t ab = valid ? abar_s[i] : 0u;
            const bool active = ab != 0;
            CP f0[16], f1[16];
            uint32_t w[32];
#pragma unroll 1
            for (int r = 0; r < 2 * L1; ++r, ++c) {
                float2 v[16];
                if constexpr (TC) {
                    if (r == 1) {
                        // polynomial 1's products, under the transforms of
                        // digits 1 and 2
                        if (active) digit_words1(w, acc + N1, ab, lane);
                        tc.put_issue(w, active, 1, warp, lane);
                    }
                    if (r % L1 == 0) tc.wait(r / L1, warp, a.err);
                    tc.take(v, active, r, warp);
                } else {
                    if (active && r % L1 == 0) digit_words1(w, acc + (r / L1) * N1, ab, lane);
                }
                const float4 *bkc = reinterpret_cast<const float4 *>(ring.acquire(c, a.err));
                if (active) {
                    if constexpr (!TC) {
                        digits_from_words_f(v, w, r % L1);
                        fdft16<1>(v);
                    }
                    ffft512_fwd_tw_rest(v, reinterpret_cast<float2 *>(xp), *T, lane);
                    if (r == 0) {
#pragma unroll
                        for (int s = 0; s < 16; ++s) {
                            const float4 k0 = bkc[(2 * s) * 32 + lane], k1 = bkc[(2 * s + 1) * 32 + lane];
                            const unsigned long long vr = pk2(v[s].x, v[s].x), vi = pk2(v[s].y, v[s].y),
                                                     nvi = pk2(-v[s].y, -v[s].y);
                            f0[s] = pmul_first(vr, vi, nvi, k0);
                            f1[s] = pmul_first(vr, vi, nvi, k1);
                        }
                    } else {
#pragma unroll
                        for (int s = 0; s < 16; ++s) {
                            const float4 k0 = bkc[(2 * s) * 32 + lane], k1 = bkc[(2 * s + 1) * 32 + lane];
                            const unsigned long long vr = pk2(v[s].x, v[s].x), vi = pk2(v[s].y, v[s].y),
                                                     nvi = pk2(-v[s].y, -v[s].y);
                            pmac(f0[s], vr, vi, nvi, k0);
                            pmac(f1[s], vr, vi, nvi, k1);
                        }
                    }
                }
                ring.release(c, lane);
            }
            if constexpr (TC) {
                if (active) {
                    add_inverse_split(acc, f0, xp, lane, *T);
                    __syncwarp();
                }
                if (i + 1 < N0) {
                    // the next CMux's polynomial 0 is final here: its products
                    // run under this CMux's second inverse transform
                    const uint32_t abn = valid ? abar_s[i + 1] : 0u;
                    if (abn) digit_words1(w, acc, abn, lane);
                    tc.put_issue(w, abn != 0, 0, warp, lane);
                }
                if (active) {
                    add_inverse_split(acc + N1, f1, xp, lane, *T);
                    __syncwarp();
                }
            } else if (active) {
                add_inverse_split(acc, f0, xp, lane, *T);
                add_inverse_split(acc + N1, f1, xp, lane, *T);
                __syncwarp();
            }
        }
        if (valid) {
            uint32_t *o = a.out + (size_t)ct * (N1 + 1);
            for (int j = lane; j < N1; j += 32) o[j] = j == 0 ? acc[0] : (uint32_t)(0u - acc[N1 - j]);
            if (lane == 0) o[N1] = acc[N1] + a.out_b_add;
        }
        __syncwarp();
    }
    if constexpr (TC) {
        // every product of every warp was waited for; then the columns are freed
        tc_fence_before();
        asm volatile("bar.sync 1, %0;" ::"r"(W * 32) : "memory");
        if (warp == 0) {
            tc_fence_after();
            tmem_dealloc(*tc_slot, tc_cols<W>());
        }
    }
    if constexpr (!PRODUCER) {
        __syncthreads();
        if (threadIdx.x == 0) ring.drain_by_thread0(a.err);
    }
}

// key-ring depth: 7 slots with 7 (or 4) ciphertexts per CTA (more than one
// CMux of key rows in flight), 6 with 8 (shared memory)
template <int W>
constexpr int PBS01S_S = W == 8 ? 6 : 7;

template <int W>
using SplitLayout = Pbs01SplitSmem<W, PBS01S_S<W>, (int)sizeof(Fft512TablesFold)>;

template <int W, bool TC>
constexpr int split_smem_bytes()
{
    return TC ? SplitLayout<W>::TOTAL_TC : SplitLayout<W>::TOTAL;
}

// 7 and 4 ciphertexts per CTA run with a producer warp (8 or 5 warps), 8 per
// CTA without one (8 warps): at most 2 warps per SM sub-partition (up to 255
// registers); 4 per CTA leaves one consumer warp per sub-partition
template <int W>
constexpr bool PBS01S_PROD = W != 8;

template <int W, bool TC>
static cudaError_t launch_pbs01_split_t(const Pbs01Args &a, int grid, cudaStream_t st)
{
    constexpr bool PROD = PBS01S_PROD<W>;
    static_assert(split_smem_bytes<W, TC>() <= 227 * 1024, "shared memory budget");
    pbs01_split_kernel<W, PBS01S_S<W>, PROD, TC>
        <<<grid, (W + (PROD ? 1 : 0)) * 32, split_smem_bytes<W, TC>(), st>>>(a);
    return cudaGetLastError();
}

template <bool TC>
static cudaError_t launch_split_any(const Pbs01Args &a, int num_sms, int w, cudaStream_t st)
{
    if (a.B <= 0) return cudaSuccess;
    const int groups = (a.B + w - 1) / w;
    const int grid = groups < num_sms ? groups : num_sms;
    if (w == 7) return launch_pbs01_split_t<7, TC>(a, grid, st);
    if (w == 8) return launch_pbs01_split_t<8, TC>(a, grid, st);
    if (w == 4) return launch_pbs01_split_t<4, TC>(a, grid, st);
    return cudaErrorInvalidValue;
}

cudaError_t launch_pbs01_split(const Pbs01Args &a, int num_sms, int w, cudaStream_t st)
{
    return launch_split_any<false>(a, num_sms, w, st);
}

cudaError_t launch_pbs01_split_tc(const Pbs01Args &a, int num_sms, int w, cudaStream_t st)
{
    return launch_split_any<true>(a, num_sms, w, st);
}

template <int W, bool TC>
static cudaError_t init_pbs01_split_t()
{
    return cudaFuncSetAttribute(pbs01_split_kernel<W, PBS01S_S<W>, PBS01S_PROD<W>, TC>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, split_smem_bytes<W, TC>());
}

cudaError_t init_pbs01_split()
{
    cudaError_t e = init_pbs01_split_t<7, false>();
    if (e == cudaSuccess) e = init_pbs01_split_t<8, false>();
    if (e == cudaSuccess) e = init_pbs01_split_t<4, false>();
    if (e == cudaSuccess) e = init_pbs01_split_t<7, true>();
    if (e == cudaSuccess) e = init_pbs01_split_t<8, true>();
    if (e == cudaSuccess) e = init_pbs01_split_t<4, true>();
    return e;
}

}  // namespace cfdb
