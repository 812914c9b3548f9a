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
// Layout: two warps per ciphertext (the 1024-point transform of
// fft1024_f64.cuh), 2 ciphertexts and one bulk-copy producer warp per CTA.
// The key streams through the shared-memory ring in 16 KB chunks, one per
// (CMux i, TRGSW row r, output o), shared by both ciphertexts of the CTA.
#include "fft1024_f64.cuh"
#include "lvl2.cuh"

namespace cfdb {

namespace {

constexpr uint64_t DEC2_XOR = (256ull << 55) | (256ull << 46) | (256ull << 37) | (256ull << 28);

// signed 9-bit field d (0 = most significant) of x, sign-extended by two shifts
__device__ __forceinline__ long long digit_field2(uint64_t x, int d)
{
    return (long long)(x << (BGBIT2 * d)) >> (64 - BGBIT2);
}

// digit d of (X^a - 1) * poly (or of poly when a == 0 and plain), twisted:
// v[m2] = (dig_d(m) + i dig_d(m+1024)) * w^m, m = t + 64 m2
template <bool ROT>
__device__ __forceinline__ void digits2(double2 v[16], const uint64_t *poly, uint32_t abar, int d, int t,
                                        const Fft1024Tables &T)
{
#pragma unroll
    for (int m2 = 0; m2 < 16; ++m2) {
        const int m = t + 64 * m2;
        uint64_t c0 = poly[m], c1 = poly[m + 1024];
        if (ROT) {
            c0 = rot_coef<N2>(poly, m, abar) - c0;
            c1 = rot_coef<N2>(poly, m + 1024, abar) - c1;
        }
        const long long d0 = digit_field2((c0 + DEC2_OFFSET + DEC2_ROUND) ^ DEC2_XOR, d);
        const long long d1 = digit_field2((c1 + DEC2_OFFSET + DEC2_ROUND) ^ DEC2_XOR, d);
        v[m2] = cmul(make_double2((double)d0, (double)d1), T.twist[m2 * 64 + t]);
    }
}

template <int W, int S>
struct Pbs02Smem {
    static constexpr int ABORT_OFF = 96;       // int: set when any wait gave up
    static constexpr int RING_OFF = 128;
    static constexpr int CHUNK_BYTES = 16384;   // one (row, output): 1024 complex
    static constexpr int TAB_OFF = RING_OFF + S * CHUNK_BYTES;
    static constexpr int PAIR_OFF = TAB_OFF + ((int)sizeof(Fft1024Tables) + 127) / 128 * 128;
    static constexpr int XP_BYTES = 1024 * 16;
    static constexpr int ACC_BYTES = 2 * N2 * 8;
    static constexpr int ABAR_BYTES = ((N0 * 2) + 127) / 128 * 128;
    static constexpr int PER_PAIR = XP_BYTES + ACC_BYTES + ABAR_BYTES;
    static constexpr int TOTAL = PAIR_OFF + (W / 2) * PER_PAIR;
};

template <int W, int S>
__global__ void __launch_bounds__((W + 1) * 32, 1) pbs02_f64_kernel(Pbs02Args a)
{
    using L = Pbs02Smem<W, S>;
    extern __shared__ __align__(128) unsigned char smem[];
    uint64_t *full = reinterpret_cast<uint64_t *>(smem);
    uint64_t *empty = full + S;
    double2 *ring = reinterpret_cast<double2 *>(smem + L::RING_OFF);
    Fft1024Tables *T = reinterpret_cast<Fft1024Tables *>(smem + L::TAB_OFF);
    // The two warps of a ciphertext meet at named barriers, so a warp that
    // gives up a bounded wait must not leave: it raises `abort`, after which
    // every warp skips the remaining waits and runs to the end of the kernel.
    volatile int *abort_flag = reinterpret_cast<volatile int *>(smem + L::ABORT_OFF);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        *abort_flag = 0;
        for (int s = 0; s < S; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], W);
        }
        fence_barrier_init();
    }
    {
        const double2 *src = reinterpret_cast<const double2 *>(a.tables);
        double2 *dst = reinterpret_cast<double2 *>(T);
        for (int i = threadIdx.x; i < (int)(sizeof(Fft1024Tables) / 16); i += blockDim.x) dst[i] = src[i];
    }
    __syncthreads();

    constexpr int P = W / 2;   // ciphertexts per CTA
    const int ngroups = (a.B + P - 1) / P;
    constexpr int CHUNKS = N0 * 2 * L2 * 2;

    if (warp == W) {
        if (lane == 0) {
            uint32_t c = 0;
            bool ok = true;
            for (int g = blockIdx.x; g < ngroups && ok; g += gridDim.x) {
                for (int ch = 0; ch < CHUNKS; ++ch, ++c) {
                    const int slot = c % S;
                    if (c >= (uint32_t)S && !mbar_wait(&empty[slot], ((c / S) - 1) & 1)) {
                        report_error(a.err, DEV_TIMEOUT_EMPTY);
                        *abort_flag = 1;
                        ok = false;
                        break;
                    }
                    mbar_arrive_expect_tx(&full[slot], L::CHUNK_BYTES);
                    bulk_g2s(ring + slot * 1024, a.bk + (size_t)ch * 1024, L::CHUNK_BYTES, &full[slot]);
                }
            }
            for (uint32_t k = (c > (uint32_t)S ? c - S : 0); k < c; ++k)
                if (!mbar_wait(&full[k % S], (k / S) & 1)) report_error(a.err, DEV_TIMEOUT_DRAIN);
        }
        return;
    }

    const int pr = warp >> 1, t = threadIdx.x & 63, bar = 1 + pr;
    unsigned char *pb = smem + L::PAIR_OFF + pr * L::PER_PAIR;
    double2 *xp = reinterpret_cast<double2 *>(pb);
    uint64_t *acc = reinterpret_cast<uint64_t *>(pb + L::XP_BYTES);
    uint16_t *abar_s = reinterpret_cast<uint16_t *>(pb + L::XP_BYTES + L::ACC_BYTES);

    uint32_t c = 0;
    for (int g = blockIdx.x; g < ngroups; g += gridDim.x) {
        const int ct = g * P + pr;
        const bool valid = ct < a.B;
        uint32_t bbar = 2 * N2;
        if (valid) {
            const uint32_t *in = a.in + (size_t)ct * (N0 + 1);
            for (int i = t; i < N0; i += 64) abar_s[i] = (uint16_t)((in[i] + (1u << 19)) >> 20);
            bbar = 2 * N2 - (in[N0] >> 20);
        }
        for (int j = t; j < N2; j += 64) {
            acc[j] = 0;
            acc[N2 + j] = testvec_rot2(a.tv, j, bbar);
        }
        pair_sync(bar);

        for (int i = 0; i < N0; ++i) {
            const uint32_t ab = valid ? abar_s[i] : 0u;
            const bool active = ab != 0;
            double2 f0[16], f1[16];
#pragma unroll 1
            for (int r = 0; r < 2 * L2; ++r) {
                double2 v[16];
                if (active) {
                    digits2<true>(v, acc + (r / L2) * N2, ab, r % L2, t, *T);
                    fft1024_fwd(v, xp, *T, t, bar);
                }
#pragma unroll
                for (int o = 0; o < 2; ++o, ++c) {
                    const int slot = c % S;
                    if (!*abort_flag && !mbar_wait(&full[slot], (c / S) & 1)) {
                        report_error(a.err, DEV_TIMEOUT_FULL);
                        *abort_flag = 1;
                    }
                    if (active) {
                        const double2 *bkc = ring + slot * 1024;
                        if (o == 0) {
                            if (r == 0) {
#pragma unroll
                                for (int s = 0; s < 16; ++s) f0[s] = cmul(v[s], bkc[s * 64 + t]);
                            } else {
#pragma unroll
                                for (int s = 0; s < 16; ++s) cfma(f0[s], v[s], bkc[s * 64 + t]);
                            }
                        } else {
                            if (r == 0) {
#pragma unroll
                                for (int s = 0; s < 16; ++s) f1[s] = cmul(v[s], bkc[s * 64 + t]);
                            } else {
#pragma unroll
                                for (int s = 0; s < 16; ++s) cfma(f1[s], v[s], bkc[s * 64 + t]);
                            }
                        }
                    }
                    __syncwarp();
                    if (lane == 0) mbar_arrive(&empty[slot]);
                }
            }
            if (active) {
                fft1024_inv(f0, xp, *T, t, bar);
#pragma unroll
                for (int m2 = 0; m2 < 16; ++m2) {
                    const int m = t + 64 * m2;
                    const double2 y = cmulc(f0[m2], T->twist[m2 * 64 + t]);
                    acc[m] += f64_to_torus64(y.x * (1.0 / 1024.0));
                    acc[m + 1024] += f64_to_torus64(y.y * (1.0 / 1024.0));
                }
                fft1024_inv(f1, xp, *T, t, bar);
#pragma unroll
                for (int m2 = 0; m2 < 16; ++m2) {
                    const int m = t + 64 * m2;
                    const double2 y = cmulc(f1[m2], T->twist[m2 * 64 + t]);
                    acc[N2 + m] += f64_to_torus64(y.x * (1.0 / 1024.0));
                    acc[N2 + m + 1024] += f64_to_torus64(y.y * (1.0 / 1024.0));
                }
            }
            pair_sync(bar);
        }
        if (valid) {
            uint64_t *o = a.out + (size_t)ct * (N2 + 1);
            for (int j = t; j < N2; j += 64) o[j] = j == 0 ? acc[0] : 0ull - acc[N2 - j];
            if (t == 0) o[N2] = acc[N2] + a.out_b_add;
        }
        pair_sync(bar);
    }
}

// integer polynomials [rows][2][2048] (64-bit torus) -> chunk layout
// [rows][2 o][16 s][64 t] complex (one 1024-complex chunk per (row, o))
__global__ void __launch_bounds__(128) bk_fft2_kernel(double2 *dst, const uint64_t *src, int rows,
                                                      const Fft1024Tables *T)
{
    __shared__ double2 xp_s[2][1024];
    const int pr = threadIdx.x >> 6, t = threadIdx.x & 63;
    const int poly = blockIdx.x * 2 + pr;
    if (poly >= rows * 2) return;   // uniform per pair; the grid covers pairs exactly
    const uint64_t *p = src + (size_t)poly * N2;
    double2 v[16];
#pragma unroll
    for (int m2 = 0; m2 < 16; ++m2) {
        const int m = t + 64 * m2;
        v[m2] = cmul(make_double2(__ll2double_rn((long long)p[m]), __ll2double_rn((long long)p[m + 1024])),
                     T->twist[m2 * 64 + t]);
    }
    fft1024_fwd(v, xp_s[pr], *T, t, 1 + pr);
    double2 *d = dst + (size_t)poly * 1024;
#pragma unroll
    for (int s = 0; s < 16; ++s) d[s * 64 + t] = v[s];
}

__device__ __forceinline__ int bitrev10(int x) { return (int)(__brev((unsigned)x) >> 22); }

// TFHEpp BootstrappingKeyFFT<lvl02param> / TRGSWFFT<lvl2param> rows (re | im
// halves, bit-reversed order) -> chunk layout
__global__ void bk_permute2_kernel(double2 *dst, const double *src, int rows)
{
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;   // (poly, s, t)
    if (e >= (size_t)rows * 2 * 1024) return;
    const int t = (int)(e & 63), s = (int)((e >> 6) & 15);
    const size_t poly = e >> 10;
    const int idx = bitrev10(fft1024_freq(t, s));
    const double *p = src + poly * N2;
    dst[e] = make_double2(p[idx], p[idx + 1024]);
}

__global__ void __launch_bounds__(128) twist_ifft2_kernel(double *out, const uint64_t *in, int B,
                                                          const Fft1024Tables *T)
{
    __shared__ double2 xp_s[2][1024];
    const int pr = threadIdx.x >> 6, t = threadIdx.x & 63;
    const int p = blockIdx.x * 2 + pr;
    if (p >= B) return;
    const uint64_t *x = in + (size_t)p * N2;
    double2 v[16];
#pragma unroll
    for (int m2 = 0; m2 < 16; ++m2) {
        const int m = t + 64 * m2;
        v[m2] = cmul(make_double2(__ll2double_rn((long long)x[m]), __ll2double_rn((long long)x[m + 1024])),
                     T->twist[m2 * 64 + t]);
    }
    fft1024_fwd(v, xp_s[pr], *T, t, 1 + pr);
    double *o = out + (size_t)p * N2;
#pragma unroll
    for (int s = 0; s < 16; ++s) {
        const int idx = bitrev10(fft1024_freq(t, s));
        o[idx] = v[s].x;
        o[idx + 1024] = v[s].y;
    }
}

__global__ void __launch_bounds__(128) twist_fft2_kernel(uint64_t *out, const double *in, int B,
                                                         const Fft1024Tables *T)
{
    __shared__ double2 xp_s[2][1024];
    const int pr = threadIdx.x >> 6, t = threadIdx.x & 63;
    const int p = blockIdx.x * 2 + pr;
    if (p >= B) return;
    const double *x = in + (size_t)p * N2;
    double2 v[16];
#pragma unroll
    for (int s = 0; s < 16; ++s) {
        const int idx = bitrev10(fft1024_freq(t, s));
        v[s] = make_double2(x[idx], x[idx + 1024]);
    }
    fft1024_inv(v, xp_s[pr], *T, t, 1 + pr);
    uint64_t *o = out + (size_t)p * N2;
#pragma unroll
    for (int m2 = 0; m2 < 16; ++m2) {
        const int m = t + 64 * m2;
        const double2 y = cmulc(v[m2], T->twist[m2 * 64 + t]);
        o[m] = f64_to_torus64(y.x * (1.0 / 1024.0));
        o[m + 1024] = f64_to_torus64(y.y * (1.0 / 1024.0));
    }
}

// one product per pair of warps; trgsw prepared: [8 rows][2 o][1024] complex
__global__ void __launch_bounds__(128) extprod2_kernel(ExtProd2Args a)
{
    __shared__ double2 xp_s[2][1024];
    const int pr = threadIdx.x >> 6, t = threadIdx.x & 63;
    const int p = blockIdx.x * 2 + pr;
    if (p >= a.B) return;
    const Fft1024Tables &T = *a.tables;
    const uint64_t *in = a.trlwe + (size_t)p * 2 * N2;
    const double2 *g = a.trgsw + (a.shared ? 0 : (size_t)p * 2 * L2 * 2 * 1024);
    double2 f0[16], f1[16];
#pragma unroll 1
    for (int r = 0; r < 2 * L2; ++r) {
        double2 v[16];
        digits2<false>(v, in + (r / L2) * N2, 0, r % L2, t, T);
        fft1024_fwd(v, xp_s[pr], T, t, 1 + pr);
        const double2 *g0 = g + ((size_t)r * 2) * 1024, *g1 = g0 + 1024;
        if (r == 0) {
#pragma unroll
            for (int s = 0; s < 16; ++s) {
                f0[s] = cmul(v[s], g0[s * 64 + t]);
                f1[s] = cmul(v[s], g1[s * 64 + t]);
            }
        } else {
#pragma unroll
            for (int s = 0; s < 16; ++s) {
                cfma(f0[s], v[s], g0[s * 64 + t]);
                cfma(f1[s], v[s], g1[s * 64 + t]);
            }
        }
    }
    uint64_t *o = a.out + (size_t)p * 2 * N2;
    fft1024_inv(f0, xp_s[pr], T, t, 1 + pr);
#pragma unroll
    for (int m2 = 0; m2 < 16; ++m2) {
        const int m = t + 64 * m2;
        const double2 y = cmulc(f0[m2], T.twist[m2 * 64 + t]);
        o[m] = f64_to_torus64(y.x * (1.0 / 1024.0));
        o[m + 1024] = f64_to_torus64(y.y * (1.0 / 1024.0));
    }
    fft1024_inv(f1, xp_s[pr], T, t, 1 + pr);
#pragma unroll
    for (int m2 = 0; m2 < 16; ++m2) {
        const int m = t + 64 * m2;
        const double2 y = cmulc(f1[m2], T.twist[m2 * 64 + t]);
        o[N2 + m] = f64_to_torus64(y.x * (1.0 / 1024.0));
        o[N2 + m + 1024] = f64_to_torus64(y.y * (1.0 / 1024.0));
    }
}

constexpr int PBS02_W = 6, PBS02_S = 2;

}  // namespace

cudaError_t launch_pbs02_f64(const Pbs02Args &a, int num_sms, cudaStream_t st)
{
    if (a.B <= 0) return cudaSuccess;
    using L = Pbs02Smem<PBS02_W, PBS02_S>;
    static_assert(L::TOTAL <= 227 * 1024, "shared memory budget");
    const int groups = (a.B + PBS02_W / 2 - 1) / (PBS02_W / 2);
    pbs02_f64_kernel<PBS02_W, PBS02_S>
        <<<groups < num_sms ? groups : num_sms, (PBS02_W + 1) * 32, L::TOTAL, st>>>(a);
    return cudaGetLastError();
}

cudaError_t init_pbs02_f64()
{
    return cudaFuncSetAttribute(pbs02_f64_kernel<PBS02_W, PBS02_S>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                Pbs02Smem<PBS02_W, PBS02_S>::TOTAL);
}

cudaError_t bk02_to_fft(double2 *dst, const uint64_t *src, int rows, const Fft1024Tables *T, cudaStream_t st)
{
    bk_fft2_kernel<<<rows, 128, 0, st>>>(dst, src, rows, T);
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
    twist_ifft2_kernel<<<(B + 1) / 2, 128, 0, st>>>(out, in, B, T);
    return cudaGetLastError();
}

cudaError_t launch_twist_fft2(uint64_t *out, const double *in, int B, const Fft1024Tables *T, cudaStream_t st)
{
    if (B <= 0) return cudaSuccess;
    twist_fft2_kernel<<<(B + 1) / 2, 128, 0, st>>>(out, in, B, T);
    return cudaGetLastError();
}

cudaError_t launch_extprod2(const ExtProd2Args &a, cudaStream_t st)
{
    if (a.B <= 0) return cudaSuccess;
    extprod2_kernel<<<(a.B + 1) / 2, 128, 0, st>>>(a);
    return cudaGetLastError();
}

}  // namespace cfdb
