// The lvl2 ring (N = 2048, 64-bit torus, l = 4, Bg = 2^9) in FP64: batched
// lvl0 -> lvl2 programmable bootstrapping, batched lvl2 external products,
// standalone TwistIFFT / TwistFFT<lvl2param>, and key preparation.
//
// Restates GateBootstrappingTLWE2TLWEFFT<lvl02param> (thirdparty/TFHEpp/src/
// gatebootstrapping.cpp:14-23, BlindRotate at include/gatebootstrapping.hpp:
// 15-43 with domain lvl0, target lvl2: bbar = 2N - (b >> 20), abar_i =
// (a_i + 2^19) >> 20) and trgswfftExternalProduct<lvl2param> (src/trgsw.cpp:
// 77-103).  The conversions follow TFHEpp's 64-bit torus FFT: int64 -> double
// rounding on the way in, truncation toward zero modulo 2^64 on the way out;
// FP64 keeps ~53 bits of a 64-bit torus value, the intrinsic precision of this
// path (TFHEpp's own round trip error bound is 2^14, test/polymul.cpp:57-68).
//
// Layout: four warps (T2 = 128 threads, 8 complex values each) per ciphertext,
// P ciphertexts per CTA and no producer warp (ring.cuh KeyRing: the last warp
// to release a slot refills it).  The key streams through the shared-memory
// ring in 16 KB chunks, one per (CMux i, TRGSW row r, output o), shared by all
// ciphertexts of the CTA; a chunk is stored [slot s][thread u], so each thread
// reads exactly the frequencies it owns.
#include "fft1024_f64.cuh"
#include "lvl2.cuh"
#include "ring.cuh"

namespace cfdb {

namespace {

constexpr uint64_t DEC2_XOR = (256ull << 55) | (256ull << 46) | (256ull << 37) | (256ull << 28);

// signed 9-bit field d (0 = most significant) of x, sign-extended by two
// shifts; the field lies in the top word after the first, so the second
// shift and the conversion to double work on 32 bits
__device__ __forceinline__ int digit_field2(uint64_t x, int d)
{
    return (int)((x << (BGBIT2 * d)) >> 32) >> (32 - BGBIT2);
}

// digit-extraction words of (X^a - 1) * poly (or of poly when ROT is false)
// at m = t + 128 j and m + 1024: x = (c + offset + round) ^ DEC2_XOR, from
// which every digit is two shifts (all four digits of a polynomial from one
// load of the accumulator)
template <bool ROT>
__device__ __forceinline__ void digit_words2(uint64_t x[16], const uint64_t *poly, uint32_t abar, int t)
{
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const int m = t + T2 * j;
        uint64_t c0 = poly[m], c1 = poly[m + 1024];
        if (ROT) {
            c0 = rot_coef<N2>(poly, m, abar) - c0;
            c1 = rot_coef<N2>(poly, m + 1024, abar) - c1;
        }
        x[2 * j] = (c0 + DEC2_OFFSET + DEC2_ROUND) ^ DEC2_XOR;
        x[2 * j + 1] = (c1 + DEC2_OFFSET + DEC2_ROUND) ^ DEC2_XOR;
    }
}

// digit d, twisted by W_32^j (fft8x folds the rest of the twist):
// v[j] = (dig_d(m) + i dig_d(m+1024)) * W_32^j, m = t + 128 j
__device__ __forceinline__ void digits2(double2 v[8], const uint64_t x[16], int d)
{
#pragma unroll
    for (int j = 0; j < 8; ++j)
        v[j] = cx_w32<1>(make_double2((double)digit_field2(x[2 * j], d), (double)digit_field2(x[2 * j + 1], d)), j);
}

// poly[m] += round-toward-zero of the inverse transform, m = t + 128 j
__device__ __forceinline__ void add_inverse2(uint64_t *poly, const double2 v[8], int t)
{
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const int m = t + T2 * j;
        const double2 y = cx_w32<-1>(v[j], j);
        poly[m] += f64_to_torus64(y.x * (1.0 / 1024.0));
        poly[m + 1024] += f64_to_torus64(y.y * (1.0 / 1024.0));
    }
}

template <int P, int S>
struct Pbs02Smem {
    static constexpr int CHUNK_BYTES = 16384;   // one (row, output): 1024 complex
    static constexpr int RING_OFF = RING_HEADER_BYTES;
    static constexpr int TAB_OFF = RING_OFF + S * CHUNK_BYTES;
    static constexpr int GROUP_OFF = TAB_OFF + ((int)sizeof(Fft1024Tables) + 127) / 128 * 128;
    static constexpr int XP_BYTES = FFT8X_XP<T2> * 16;
    static constexpr int ACC_BYTES = 2 * N2 * 8;
    static constexpr int ABAR_BYTES = ((N0 * 2) + 127) / 128 * 128;
    static constexpr int PER_GROUP = XP_BYTES + ACC_BYTES + ABAR_BYTES;
    static constexpr int TOTAL = GROUP_OFF + P * PER_GROUP;
};

// Key ring without a producer warp (ring.cuh): every warp runs the math, and
// the block's registers are shared by the consumer warps alone.
template <int P, int S>
__global__ void __launch_bounds__(4 * P * 32, 1) pbs02_f64_kernel(Pbs02Args a)
{
    using L = Pbs02Smem<P, S>;
    constexpr int W = 4 * P;   // warps, all consumers
    extern __shared__ __align__(128) unsigned char smem[];
    Fft1024Tables *T = reinterpret_cast<Fft1024Tables *>(smem + L::TAB_OFF);
    const int ngroups = (a.B + P - 1) / P;
    constexpr int CHUNKS = N0 * 2 * L2 * 2;
    KeyRing<S, L::CHUNK_BYTES, W> ring{reinterpret_cast<RingHeader *>(smem), smem + L::RING_OFF,
                                    reinterpret_cast<const unsigned char *>(a.bk), (uint32_t)CHUNKS,
                                    (uint32_t)groups_of_block(ngroups, blockIdx.x, gridDim.x) * CHUNKS};

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) ring.init_by_thread0();
    {
        const double2 *src = reinterpret_cast<const double2 *>(a.tables);
        double2 *dst = reinterpret_cast<double2 *>(T);
        for (int i = threadIdx.x; i < (int)(sizeof(Fft1024Tables) / 16); i += blockDim.x) dst[i] = src[i];
    }
    __syncthreads();
    if (threadIdx.x == 0) ring.prologue_by_thread0();

    const int gr = warp >> 2, t = threadIdx.x & (T2 - 1), bar = 1 + gr;
    unsigned char *pb = smem + L::GROUP_OFF + gr * L::PER_GROUP;
    double2 *xp = reinterpret_cast<double2 *>(pb);
    uint64_t *acc = reinterpret_cast<uint64_t *>(pb + L::XP_BYTES);
    uint16_t *abar_s = reinterpret_cast<uint16_t *>(pb + L::XP_BYTES + L::ACC_BYTES);

    uint32_t c = 0;
    for (int g = blockIdx.x; g < ngroups; g += gridDim.x) {
        const int ct = g * P + gr;
        const bool valid = ct < a.B;
        uint32_t bbar = 2 * N2;
        if (valid) {
            const uint32_t *in = a.in + (size_t)ct * (N0 + 1);
            for (int i = t; i < N0; i += T2) abar_s[i] = (uint16_t)((in[i] + (1u << 19)) >> 20);
            bbar = 2 * N2 - (in[N0] >> 20);
        }
        for (int j = t; j < N2; j += T2) {
            acc[j] = 0;
            acc[N2 + j] = testvec_rot2(a.tv, j, bbar);
        }
        group_sync<T2>(bar);

        for (int i = 0; i < N0; ++i) {
            const uint32_t ab = valid ? abar_s[i] : 0u;
            const bool active = ab != 0;
            double2 f0[8], f1[8];
            uint64_t xw[16];
#pragma unroll 1
            for (int r = 0; r < 2 * L2; ++r) {
                double2 v[8];
                if (active) {
                    if (r % L2 == 0) digit_words2<true>(xw, acc + (r / L2) * N2, ab, t);
                    digits2(v, xw, r % L2);
                    fft8x_fwd<double2, T2>(v, xp, *T, t, bar);
                }
#pragma unroll
                for (int o = 0; o < 2; ++o, ++c) {
                    const double2 *bkc = reinterpret_cast<const double2 *>(ring.acquire(c, a.err));
                    if (active) {
                        if (o == 0) {
                            if (r == 0) {
#pragma unroll
                                for (int s = 0; s < 8; ++s) f0[s] = cx_mul(v[s], bkc[s * T2 + t]);
                            } else {
#pragma unroll
                                for (int s = 0; s < 8; ++s) cx_fma(f0[s], v[s], bkc[s * T2 + t]);
                            }
                        } else {
                            if (r == 0) {
#pragma unroll
                                for (int s = 0; s < 8; ++s) f1[s] = cx_mul(v[s], bkc[s * T2 + t]);
                            } else {
#pragma unroll
                                for (int s = 0; s < 8; ++s) cx_fma(f1[s], v[s], bkc[s * T2 + t]);
                            }
                        }
                    }
                    ring.release(c, lane);
                }
            }
            if (active) {
                fft8x_inv<double2, T2>(f0, xp, *T, t, bar);
                add_inverse2(acc, f0, t);
                fft8x_inv<double2, T2>(f1, xp, *T, t, bar);
                add_inverse2(acc + N2, f1, t);
            }
            group_sync<T2>(bar);
        }
        if (valid) {
            uint64_t *o = a.out + (size_t)ct * (N2 + 1);
            for (int j = t; j < N2; j += T2) o[j] = j == 0 ? acc[0] : 0ull - acc[N2 - j];
            if (t == 0) o[N2] = acc[N2] + a.out_b_add;
        }
        group_sync<T2>(bar);
    }
    __syncthreads();
    if (threadIdx.x == 0) ring.drain_by_thread0(a.err);
}

// integer polynomials [rows][2][2048] (64-bit torus) -> chunk layout
// [rows][2 o][8 s][128 u] complex (one 1024-complex chunk per (row, o))
__global__ void __launch_bounds__(T2) bk_fft2_kernel(double2 *dst, const uint64_t *src, const Fft1024Tables *T)
{
    __shared__ double2 xp_s[FFT8X_XP<T2>];
    const int t = threadIdx.x;
    const size_t poly = blockIdx.x;
    const uint64_t *p = src + poly * N2;
    double2 v[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const int m = t + T2 * j;
        v[j] = cx_w32<1>(make_double2(__ll2double_rn((long long)p[m]), __ll2double_rn((long long)p[m + 1024])), j);
    }
    fft8x_fwd<double2, T2>(v, xp_s, *T, t, 1);
    double2 *d = dst + poly * 1024;
#pragma unroll
    for (int s = 0; s < 8; ++s) d[s * T2 + t] = v[s];
}

__device__ __forceinline__ int bitrev10(int x) { return (int)(__brev((unsigned)x) >> 22); }

// TFHEpp BootstrappingKeyFFT<lvl02param> / TRGSWFFT<lvl2param> rows (re | im
// halves, bit-reversed order) -> chunk layout
__global__ void bk_permute2_kernel(double2 *dst, const double *src, int rows)
{
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;   // (poly, s, u)
    if (e >= (size_t)rows * 2 * 1024) return;
    const int u = (int)(e & (T2 - 1)), s = (int)((e >> 7) & 7);
    const size_t poly = e >> 10;
    const int idx = bitrev10(fft1024_freq(u, s));
    const double *p = src + poly * N2;
    dst[e] = make_double2(p[idx], p[idx + 1024]);
}

__global__ void __launch_bounds__(T2) twist_ifft2_kernel(double *out, const uint64_t *in, const Fft1024Tables *T)
{
    __shared__ double2 xp_s[FFT8X_XP<T2>];
    const int t = threadIdx.x;
    const size_t p = blockIdx.x;
    const uint64_t *x = in + p * N2;
    double2 v[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const int m = t + T2 * j;
        v[j] = cx_w32<1>(make_double2(__ll2double_rn((long long)x[m]), __ll2double_rn((long long)x[m + 1024])), j);
    }
    fft8x_fwd<double2, T2>(v, xp_s, *T, t, 1);
    double *o = out + p * N2;
#pragma unroll
    for (int s = 0; s < 8; ++s) {
        const int idx = bitrev10(fft1024_freq(t, s));
        o[idx] = v[s].x;
        o[idx + 1024] = v[s].y;
    }
}

__global__ void __launch_bounds__(T2) twist_fft2_kernel(uint64_t *out, const double *in, const Fft1024Tables *T)
{
    __shared__ double2 xp_s[FFT8X_XP<T2>];
    const int t = threadIdx.x;
    const size_t p = blockIdx.x;
    const double *x = in + p * N2;
    double2 v[8];
#pragma unroll
    for (int s = 0; s < 8; ++s) {
        const int idx = bitrev10(fft1024_freq(t, s));
        v[s] = make_double2(x[idx], x[idx + 1024]);
    }
    fft8x_inv<double2, T2>(v, xp_s, *T, t, 1);
    uint64_t *o = out + p * N2;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const int m = t + T2 * j;
        const double2 y = cx_w32<-1>(v[j], j);
        o[m] = f64_to_torus64(y.x * (1.0 / 1024.0));
        o[m + 1024] = f64_to_torus64(y.y * (1.0 / 1024.0));
    }
}

// one product per 128-thread block; trgsw prepared: [8 rows][2 o][1024] complex
__global__ void __launch_bounds__(T2) extprod2_kernel(ExtProd2Args a)
{
    __shared__ double2 xp_s[FFT8X_XP<T2>];
    const int t = threadIdx.x;
    const size_t p = blockIdx.x;
    const Fft1024Tables &T = *a.tables;
    const uint64_t *in = a.trlwe + p * 2 * N2;
    const double2 *g = a.trgsw + (a.shared ? 0 : p * 2 * L2 * 2 * 1024);
    // the TRGSW rows two ahead of the one in use are fetched into L2 (32 KB
    // per row: both outputs), so the loads after each transform find them there
    constexpr uint32_t ROW_BYTES = 2 * 1024 * sizeof(double2);
    auto prefetch = [&](int r0, int n) {
        if (a.shared || t != 0) return;
        for (int k = r0; k < r0 + n && k < 2 * L2; ++k)
            bulk_prefetch_l2(reinterpret_cast<const unsigned char *>(g) + (size_t)k * ROW_BYTES, ROW_BYTES);
    };
    prefetch(0, 2);
    if (t == 0) bulk_prefetch_l2_if_aligned(in, 2 * N2 * sizeof(uint64_t));   // the TRLWE, read per digit polynomial
    double2 f0[8], f1[8];
#pragma unroll 1
    for (int r = 0; r < 2 * L2; ++r) {
        double2 v[8];
        uint64_t xw[16];
        prefetch(r + 2, 1);
        digit_words2<false>(xw, in + (r / L2) * N2, 0, t);
        digits2(v, xw, r % L2);
        fft8x_fwd<double2, T2>(v, xp_s, T, t, 1);
        const double2 *g0 = g + ((size_t)r * 2) * 1024, *g1 = g0 + 1024;
        if (r == 0) {
#pragma unroll
            for (int s = 0; s < 8; ++s) {
                f0[s] = cx_mul(v[s], g0[s * T2 + t]);
                f1[s] = cx_mul(v[s], g1[s * T2 + t]);
            }
        } else {
#pragma unroll
            for (int s = 0; s < 8; ++s) {
                cx_fma(f0[s], v[s], g0[s * T2 + t]);
                cx_fma(f1[s], v[s], g1[s * T2 + t]);
            }
        }
    }
    uint64_t *o = a.out + p * 2 * N2;
    fft8x_inv<double2, T2>(f0, xp_s, T, t, 1);
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const int m = t + T2 * j;
        const double2 y = cx_w32<-1>(f0[j], j);
        o[m] = f64_to_torus64(y.x * (1.0 / 1024.0));
        o[m + 1024] = f64_to_torus64(y.y * (1.0 / 1024.0));
    }
    fft8x_inv<double2, T2>(f1, xp_s, T, t, 1);
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const int m = t + T2 * j;
        const double2 y = cx_w32<-1>(f1[j], j);
        o[N2 + m] = f64_to_torus64(y.x * (1.0 / 1024.0));
        o[N2 + m + 1024] = f64_to_torus64(y.y * (1.0 / 1024.0));
    }
}

// key-ring depth per shape: what the shared memory left by P ciphertexts holds
template <int P>
constexpr int PBS02_S = P == 3 ? 4 : P == 2 ? 7 : 8;

}  // namespace

template <int P>
static cudaError_t launch_pbs02_t(const Pbs02Args &a, int num_sms, cudaStream_t st)
{
    using L = Pbs02Smem<P, PBS02_S<P>>;
    static_assert(L::TOTAL <= 227 * 1024, "shared memory budget");
    const int groups = (a.B + P - 1) / P;
    pbs02_f64_kernel<P, PBS02_S<P>><<<groups < num_sms ? groups : num_sms, 4 * P * 32, L::TOTAL, st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_pbs02_f64(const Pbs02Args &a, int num_sms, int p, cudaStream_t st)
{
    if (a.B <= 0) return cudaSuccess;
    if (p == 3) return launch_pbs02_t<3>(a, num_sms, st);
    if (p == 2) return launch_pbs02_t<2>(a, num_sms, st);
    if (p == 1) return launch_pbs02_t<1>(a, num_sms, st);
    return cudaErrorInvalidValue;
}

template <int P>
static cudaError_t init_pbs02_t()
{
    return cudaFuncSetAttribute(pbs02_f64_kernel<P, PBS02_S<P>>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                Pbs02Smem<P, PBS02_S<P>>::TOTAL);
}

cudaError_t init_pbs02_f64()
{
    cudaError_t e = init_pbs02_t<3>();
    if (e == cudaSuccess) e = init_pbs02_t<2>();
    if (e == cudaSuccess) e = init_pbs02_t<1>();
    return e;
}

cudaError_t bk02_to_fft(double2 *dst, const uint64_t *src, int rows, const Fft1024Tables *T, cudaStream_t st)
{
    if (rows <= 0) return cudaSuccess;
    bk_fft2_kernel<<<rows * 2, T2, 0, st>>>(dst, src, T);
    return cudaGetLastError();
}

cudaError_t bkfft02_permute(double2 *dst, const double *src, int rows, cudaStream_t st)
{
    const size_t n = (size_t)rows * 2 * 1024;
    bk_permute2_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(dst, src, rows);
    return cudaGetLastError();
}

cudaError_t launch_twist_ifft2(double *out, const uint64_t *in, int B, const Fft1024Tables *T, cudaStream_t st)
{
    if (B <= 0) return cudaSuccess;
    twist_ifft2_kernel<<<B, T2, 0, st>>>(out, in, T);
    return cudaGetLastError();
}

cudaError_t launch_twist_fft2(uint64_t *out, const double *in, int B, const Fft1024Tables *T, cudaStream_t st)
{
    if (B <= 0) return cudaSuccess;
    twist_fft2_kernel<<<B, T2, 0, st>>>(out, in, T);
    return cudaGetLastError();
}

cudaError_t launch_extprod2(const ExtProd2Args &a, cudaStream_t st)
{
    if (a.B <= 0) return cudaSuccess;
    extprod2_kernel<<<a.B, T2, 0, st>>>(a);
    return cudaGetLastError();
}

}  // namespace cfdb
