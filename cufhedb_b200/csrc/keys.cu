// Key material on the device: deterministic key generation from a seed, and
// conversion of bootstrapping keys into the engine's FFT-domain layout.
//
// Key generation restates TFHEpp's bkgen / ikskgen (thirdparty/TFHEpp/src/
// cloudkey.cpp:7-20,53-69) with a counter-based generator in place of
// TFHEpp's randen/random_device source (include/utils.hpp:17-22), so a key set
// is reproducible from its seed: draw(seed, stream, ctr) is SplitMix64's
// finaliser applied to a per-stream key xor a scrambled counter, and the
// noise is an integer approximate Gaussian (the centred sum of four uniform
// 32-bit words, scaled).  These test/benchmark keys are not produced by a
// cryptographic generator; production keys come from TFHEpp and are loaded
// with the cufhedb_load_* entry points.
#include "keys.cuh"
#include "fft_f32.cuh"

namespace cfdb {

__host__ __device__ __forceinline__ uint64_t mix64(uint64_t z)
{
    z ^= z >> 30;
    z *= 0xBF58476D1CE4E5B9ull;
    z ^= z >> 27;
    z *= 0x94D049BB133111EBull;
    z ^= z >> 31;
    return z;
}

uint64_t stream_key(uint64_t seed, uint64_t stream) { return mix64(seed + stream * 0x9E3779B97F4A7C15ull); }

__host__ __device__ __forceinline__ uint64_t draw_k(uint64_t skey, uint64_t ctr)
{
    return mix64(skey ^ (ctr * 0xD1B54A32D192ED03ull + 0x632BE59BD9B4E019ull));
}

uint64_t host_draw(uint64_t seed, uint64_t stream, uint64_t ctr) { return draw_k(stream_key(seed, stream), ctr); }

__host__ __device__ __forceinline__ int64_t noise_k(uint64_t skey, uint64_t ctr, int64_t scale)
{
    const uint64_t u0 = draw_k(skey, ctr), u1 = draw_k(skey, ctr + 1);
    const int64_t s = (int64_t)((u0 & 0xFFFFFFFFull) + (u0 >> 32) + (u1 & 0xFFFFFFFFull) + (u1 >> 32)) -
                      (int64_t)(1ull << 33);
    return (s * scale) >> 32;
}

void host_secret_keys(uint64_t seed, uint32_t *s0, uint32_t *s1, uint64_t *s2)
{
    for (int i = 0; i < N0; ++i) s0[i] = 0;
    for (int i = 0; i < N1; ++i) s1[i] = 0;
    for (int i = 0; i < N2; ++i) s2[i] = 0;
    const uint64_t k0 = stream_key(seed, ST_SK0), k1 = stream_key(seed, ST_SK1), k2 = stream_key(seed, ST_SK2);
    for (int t = 0; t < 512; ++t) s0[draw_k(k0, t) % N0] = 1;
    for (int t = 0; t < 512; ++t) s1[draw_k(k1, t) % N1] = 1;
    for (int t = 0; t < 1024; ++t) s2[draw_k(k2, t) % N2] = 1;
}

namespace {

// one warp per key-switching-key row: TLWE of width n under `key` of message
// key_dom[i] * (k+1) * 2^(32 - (j+1) basebit)   (cloudkey.cpp:53-69)
template <bool WIDE_DOMAIN>
__global__ void ksk_rows_kernel(uint32_t *out, uint64_t nrows, int n, int t, int basebit, const void *key_dom,
                                const uint32_t *key_tgt, uint64_t skey, int64_t ns)
{
    const uint64_t row = (uint64_t)blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (row >= nrows) return;
    const uint32_t digits = (1u << basebit) - 1;
    const uint64_t ij = row / digits;
    const uint32_t k = (uint32_t)(row % digits);
    const uint32_t j = (uint32_t)(ij % t);
    const uint64_t i = ij / t;
    const uint64_t kd = WIDE_DOMAIN ? reinterpret_cast<const uint64_t *>(key_dom)[i]
                                    : reinterpret_cast<const uint32_t *>(key_dom)[i];
    const uint32_t m = (uint32_t)(kd * (uint64_t)(k + 1) * (1ull << (32 - (j + 1) * basebit)));
    const uint64_t base = row * CB_TLWE32;
    uint32_t *o = out + row * (uint64_t)ksk_pitch(n + 1);
    for (int x = n + 1 + lane; x < ksk_pitch(n + 1); x += 32) o[x] = 0u;   // row padding
    uint32_t part = 0;
    for (int x = lane; x < n; x += 32) {
        const uint32_t av = (uint32_t)draw_k(skey, base + x);
        o[x] = av;
        part += av * key_tgt[x];
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) part += __shfl_xor_sync(0xffffffffu, part, off);
    if (lane == 0) o[n] = m + (uint32_t)noise_k(skey, base + n, ns) + part;
}

// one CTA per TRLWE row of a bootstrapping key: b = a * s + e (negacyclic),
// plus m0 * h_d on polynomial k, coefficient 0 (trgsw.cpp:206-222)
template <typename T, int N, int L, int BGBIT>
__global__ void bk_rows_kernel(T *out, const uint32_t *s0, const int *spos, int nspos, uint64_t skey, int64_t ns)
{
    __shared__ T a_s[N];
    const int row = blockIdx.x;   // i * 2L + r
    const int i = row / (2 * L), r = row % (2 * L);
    const uint64_t base = (uint64_t)row * (4ull * N);
    T *pa = out + (size_t)row * 2 * N;
    T *pb = pa + N;
    for (int j = threadIdx.x; j < N; j += blockDim.x) {
        const T v = (T)draw_k(skey, base + j);
        a_s[j] = v;
        pa[j] = v;
    }
    __syncthreads();
    for (int j = threadIdx.x; j < N; j += blockDim.x) {
        T b = (T)noise_k(skey, base + N + 2 * j, ns);
        for (int p = 0; p < nspos; ++p) {
            const int t = spos[p];
            b += (j >= t) ? a_s[j - t] : (T)(T(0) - a_s[j - t + N]);
        }
        const int d = r % L, k = r / L;
        if (j == 0) {
            const T h = (T)1 << (sizeof(T) * 8 - (d + 1) * BGBIT);
            const T m0 = (T)s0[i] * h;
            if (k == 0) pa[0] += m0;   // poly 0 of row r is written above; adjust in place
            else b += m0;
        }
        pb[j] = b;
    }
}

// TLWE encryptions of B messages under `key` (n words), counter blocks idx0..idx0+B-1
template <typename T>
__global__ void tlwe_encrypt_kernel(T *out, const T *msg, int B, int n, const T *key, uint64_t skey, int64_t ns,
                                    uint64_t idx0, uint64_t cb)
{
    const int c = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (c >= B) return;
    const uint64_t base = (idx0 + c) * cb;
    T *o = out + (size_t)c * (n + 1);
    T part = 0;
    for (int x = lane; x < n; x += 32) {
        const T av = (T)draw_k(skey, base + x);
        o[x] = av;
        part += av * key[x];
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        if constexpr (sizeof(T) == 8) part += (T)__shfl_xor_sync(0xffffffffu, (unsigned long long)part, off);
        else part += __shfl_xor_sync(0xffffffffu, part, off);
    }
    if (lane == 0) o[n] = msg[c] + (T)noise_k(skey, base + n, ns) + part;
}

// n pseudo-random words (generator stream `stream` of `seed`), e.g. lvl0
// ciphertexts with uniform coefficients for timing runs
__global__ void fill_random_kernel(uint32_t *out, size_t n, uint64_t skey)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = (uint32_t)draw_k(skey, i);
}

// decryption phases b - <a, key> (mod 2^w) of B TLWEs of width n, one warp each
template <typename T>
__global__ void tlwe_phase_kernel(T *phase, const T *ct, int B, int n, const T *key)
{
    const int c = blockIdx.x * (blockDim.x / 32) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (c >= B) return;
    const T *x = ct + (size_t)c * (n + 1);
    T part = 0;
    for (int i = lane; i < n; i += 32) part += x[i] * key[i];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        if constexpr (sizeof(T) == 8) part += (T)__shfl_xor_sync(0xffffffffu, (unsigned long long)part, off);
        else part += __shfl_xor_sync(0xffffffffu, part, off);
    }
    if (lane == 0) phase[c] = x[n] - part;
}

// forward FFT of integer polynomials into the engine's chunk layout.
// src: [rows][2][1024] 32-bit torus; dst: [rows][16 s][2 o][32 lane] complex
__global__ void bk_fft1_kernel(double2 *dst, const uint32_t *src, int rows, const Fft512Tables *T)
{
    __shared__ double2 xp_s[4][FFT512_XP];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int poly = blockIdx.x * 4 + w;   // = row * 2 + o
    if (poly >= rows * 2) return;
    const int row = poly >> 1, o = poly & 1;
    const uint32_t *p = src + (size_t)poly * N1;
    double2 v[16];
#pragma unroll
    for (int m2 = 0; m2 < 16; ++m2) {
        const int m = lane + 32 * m2;
        v[m2] = cmul(make_double2((double)(int32_t)p[m], (double)(int32_t)p[m + 512]), T->twist[m2 * 32 + lane]);
    }
    fft512_fwd(v, xp_s[w], *T, lane);
    double2 *d = dst + (size_t)row * 1024;
#pragma unroll
    for (int s = 0; s < 16; ++s) d[(2 * s + o) * 32 + lane] = v[s];
}

__device__ __forceinline__ int bitrev9(int x) { return (int)(__brev((unsigned)x) >> 23); }

// TFHEpp BootstrappingKeyFFT<lvl01param> rows [rows][2][1024] (re | im halves,
// bit-reversed frequency order, spqlios-fft-impl.cpp:399-466) -> chunk layout
__global__ void bk_permute1_kernel(double2 *dst, const double *src, int rows)
{
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;   // (row, s, o, lane)
    if (e >= (size_t)rows * 1024) return;
    const int lane = (int)(e & 31), o = (int)((e >> 5) & 1), s = (int)((e >> 6) & 15);
    const size_t row = e >> 10;
    const int idx = bitrev9(fft512_freq(lane, s));
    const double *p = src + (row * 2 + o) * N1;
    dst[e] = make_double2(p[idx], p[idx + 512]);
}

// integer key polynomials [rows][2][1024] -> two limbs hi = round(b / 2^24),
// lo = b - hi * 2^24, each transformed in FP64 and stored as FP32 in the
// split-precision chunk layout [rows][16 s][2 o][32 lane]
// float4(hi.re, lo.re, hi.im, lo.im), the pairs the paired products read
__global__ void bk_split1_kernel(float4 *dst, const uint32_t *src, int rows, const Fft512Tables *T)
{
    __shared__ double2 xp_s[4][FFT512_XP];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int poly = blockIdx.x * 4 + w;
    if (poly >= rows * 2) return;
    const int row = poly >> 1, o = poly & 1;
    const uint32_t *p = src + (size_t)poly * N1;
    double2 vh[16], vl[16];
#pragma unroll
    for (int m2 = 0; m2 < 16; ++m2) {
        const int m = lane + 32 * m2;
        const int32_t b0 = (int32_t)p[m], b1 = (int32_t)p[m + 512];
        const int32_t h0 = (int32_t)(((int64_t)b0 + (1 << 23)) >> 24), h1 = (int32_t)(((int64_t)b1 + (1 << 23)) >> 24);
        const int32_t l0 = (int32_t)((int64_t)b0 - ((int64_t)h0 << 24)), l1 = (int32_t)((int64_t)b1 - ((int64_t)h1 << 24));
        vh[m2] = cmul(make_double2((double)h0, (double)h1), T->twist[m2 * 32 + lane]);
        vl[m2] = cmul(make_double2((double)l0, (double)l1), T->twist[m2 * 32 + lane]);
    }
    fft512_fwd(vh, xp_s[w], *T, lane);
    __syncwarp();
    fft512_fwd(vl, xp_s[w], *T, lane);
    float4 *d = dst + (size_t)row * 1024;
#pragma unroll
    for (int s = 0; s < 16; ++s)
        d[(2 * s + o) * 32 + lane] = make_float4((float)vh[s].x, (float)vl[s].x, (float)vh[s].y, (float)vl[s].y);
}

// FFT-domain key in the FP64 chunk layout -> integer polynomials (the inverse
// transform, rounded: exact for keys that are transforms of 32-bit integers)
__global__ void bk_fft1_to_int_kernel(uint32_t *dst, const double2 *src, int rows, const Fft512Tables *T)
{
    __shared__ double2 xp_s[4][FFT512_XP];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int poly = blockIdx.x * 4 + w;
    if (poly >= rows * 2) return;
    const int row = poly >> 1, o = poly & 1;
    double2 v[16];
#pragma unroll
    for (int s = 0; s < 16; ++s) v[s] = src[(size_t)row * 1024 + (2 * s + o) * 32 + lane];
    fft512_inv(v, xp_s[w], *T, lane);
    uint32_t *p = dst + (size_t)poly * N1;
#pragma unroll
    for (int m2 = 0; m2 < 16; ++m2) {
        const int m = lane + 32 * m2;
        const double2 y = cmulc(v[m2], T->twist[m2 * 32 + lane]);
        p[m] = (uint32_t)__double2ll_rn(y.x * (1.0 / 512.0));
        p[m + 512] = (uint32_t)__double2ll_rn(y.y * (1.0 / 512.0));
    }
}

}  // namespace

cudaError_t gen_ksk(uint32_t *out, int kind, uint64_t seed, const void *key_dom_d, const uint32_t *key_tgt_d,
                    cudaStream_t st)
{
    uint64_t rows;
    int n, t, basebit;
    int64_t ns;
    uint64_t stream;
    if (kind == 10) { rows = 1024ull * 2 * 1023; n = N0; t = 2; basebit = 10; ns = NS_LVL0; stream = ST_KSK10; }
    else if (kind == 20) { rows = 2048ull * 2 * 1023; n = N0; t = 2; basebit = 10; ns = NS_LVL0; stream = ST_KSK20; }
    else if (kind == 21) { rows = 2048ull * 10 * 7; n = N1; t = 10; basebit = 3; ns = NS_LVL1; stream = ST_KSK21; }
    else return cudaErrorInvalidValue;
    const uint64_t skey = stream_key(seed, stream);
    const int wpb = 8;
    const unsigned grid = (unsigned)((rows + wpb - 1) / wpb);
    if (kind == 10)
        ksk_rows_kernel<false><<<grid, wpb * 32, 0, st>>>(out, rows, n, t, basebit, key_dom_d, key_tgt_d, skey, ns);
    else
        ksk_rows_kernel<true><<<grid, wpb * 32, 0, st>>>(out, rows, n, t, basebit, key_dom_d, key_tgt_d, skey, ns);
    return cudaGetLastError();
}

cudaError_t gen_bk01(uint32_t *out, uint64_t seed, const uint32_t *s0_d, const int *s1pos_d, int ns1,
                     cudaStream_t st)
{
    bk_rows_kernel<uint32_t, N1, L1, BGBIT1><<<N0 * 2 * L1, 256, 0, st>>>(out, s0_d, s1pos_d, ns1,
                                                                          stream_key(seed, ST_BK01), NS_LVL1);
    return cudaGetLastError();
}

cudaError_t gen_bk02(uint64_t *out, uint64_t seed, const uint32_t *s0_d, const int *s2pos_d, int ns2,
                     cudaStream_t st)
{
    bk_rows_kernel<uint64_t, N2, L2, BGBIT2><<<N0 * 2 * L2, 256, 0, st>>>(out, s0_d, s2pos_d, ns2,
                                                                          stream_key(seed, ST_BK02), NS_LVL2);
    return cudaGetLastError();
}

cudaError_t encrypt_tlwe32(uint32_t *out, const uint32_t *msg_d, int B, int n, const uint32_t *key_d, int64_t ns,
                           uint64_t seed, uint64_t stream, uint64_t idx0, cudaStream_t st)
{
    if (B <= 0) return cudaSuccess;
    tlwe_encrypt_kernel<uint32_t><<<(B + 7) / 8, 256, 0, st>>>(out, msg_d, B, n, key_d, stream_key(seed, stream), ns,
                                                               idx0, CB_TLWE32);
    return cudaGetLastError();
}

cudaError_t fill_random32(uint32_t *out, size_t n, uint64_t seed, uint64_t stream, cudaStream_t st)
{
    if (n == 0) return cudaSuccess;
    fill_random_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(out, n, stream_key(seed, stream));
    return cudaGetLastError();
}

cudaError_t tlwe_phase32(uint32_t *phase, const uint32_t *ct, int B, int n, const uint32_t *key_d, cudaStream_t st)
{
    if (B <= 0) return cudaSuccess;
    tlwe_phase_kernel<uint32_t><<<(B + 7) / 8, 256, 0, st>>>(phase, ct, B, n, key_d);
    return cudaGetLastError();
}

cudaError_t tlwe_phase64(uint64_t *phase, const uint64_t *ct, int B, int n, const uint64_t *key_d, cudaStream_t st)
{
    if (B <= 0) return cudaSuccess;
    tlwe_phase_kernel<uint64_t><<<(B + 7) / 8, 256, 0, st>>>(phase, ct, B, n, key_d);
    return cudaGetLastError();
}

cudaError_t encrypt_tlwe64(uint64_t *out, const uint64_t *msg_d, int B, int n, const uint64_t *key_d, int64_t ns,
                           uint64_t seed, uint64_t stream, uint64_t idx0, cudaStream_t st)
{
    if (B <= 0) return cudaSuccess;
    tlwe_encrypt_kernel<uint64_t><<<(B + 7) / 8, 256, 0, st>>>(out, msg_d, B, n, key_d, stream_key(seed, stream), ns,
                                                               idx0, CB_TLWE64);
    return cudaGetLastError();
}

cudaError_t bk01_to_fft(double2 *dst, const uint32_t *src, int rows, const Fft512Tables *T, cudaStream_t st)
{
    bk_fft1_kernel<<<(rows * 2 + 3) / 4, 128, 0, st>>>(dst, src, rows, T);
    return cudaGetLastError();
}

cudaError_t bk01_to_split(float4 *dst, const uint32_t *src, int rows, const Fft512Tables *T, cudaStream_t st)
{
    bk_split1_kernel<<<(rows * 2 + 3) / 4, 128, 0, st>>>(dst, src, rows, T);
    return cudaGetLastError();
}

cudaError_t bk01_fft_to_int(uint32_t *dst, const double2 *src, int rows, const Fft512Tables *T, cudaStream_t st)
{
    bk_fft1_to_int_kernel<<<(rows * 2 + 3) / 4, 128, 0, st>>>(dst, src, rows, T);
    return cudaGetLastError();
}

cudaError_t bkfft01_permute(double2 *dst, const double *src, int rows, cudaStream_t st)
{
    const size_t n = (size_t)rows * 1024;
    bk_permute1_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(dst, src, rows);
    return cudaGetLastError();
}

}  // namespace cfdb
