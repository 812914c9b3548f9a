// Standalone batched negacyclic transforms in TFHEpp's frequency layout:
// TwistIFFT (torus -> frequency) and TwistFFT (frequency -> torus) for the
// 32-bit torus, N = 1024 (thirdparty/TFHEpp/include/mulfft.hpp:57-121).
// One warp per polynomial, using the same warp transform as the PBS kernel.
#include "fftops.cuh"

namespace cfdb {

namespace {

__device__ __forceinline__ int bitrev9(int x) { return (int)(__brev((unsigned)x) >> 23); }

__global__ void twist_ifft1_kernel(double *out, const uint32_t *in, int B, const Fft512Tables *T)
{
    __shared__ double2 xp_s[4][FFT512_XP];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int p = blockIdx.x * 4 + w;
    if (p >= B) return;
    const uint32_t *a = in + (size_t)p * N1;
    double2 v[16];
#pragma unroll
    for (int m2 = 0; m2 < 16; ++m2) {
        const int m = lane + 32 * m2;
        v[m2] = cmul(make_double2((double)(int32_t)a[m], (double)(int32_t)a[m + 512]), T->twist[m2 * 32 + lane]);
    }
    fft512_fwd(v, xp_s[w], *T, lane);
    double *o = out + (size_t)p * N1;
#pragma unroll
    for (int s = 0; s < 16; ++s) {
        const int idx = bitrev9(fft512_freq(lane, s));
        o[idx] = v[s].x;
        o[idx + 512] = v[s].y;
    }
}

__global__ void twist_fft1_kernel(uint32_t *out, const double *in, int B, const Fft512Tables *T)
{
    __shared__ double2 xp_s[4][FFT512_XP];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int p = blockIdx.x * 4 + w;
    if (p >= B) return;
    const double *x = in + (size_t)p * N1;
    double2 v[16];
#pragma unroll
    for (int s = 0; s < 16; ++s) {
        const int idx = bitrev9(fft512_freq(lane, s));
        v[s] = make_double2(x[idx], x[idx + 512]);
    }
    fft512_inv(v, xp_s[w], *T, lane);
    uint32_t *o = out + (size_t)p * N1;
#pragma unroll
    for (int m2 = 0; m2 < 16; ++m2) {
        const int m = lane + 32 * m2;
        const double2 y = cmulc(v[m2], T->twist[m2 * 32 + lane]);
        o[m] = f64_to_torus32(y.x * (1.0 / 512.0));
        o[m + 512] = f64_to_torus32(y.y * (1.0 / 512.0));
    }
}

}  // namespace

cudaError_t launch_twist_ifft1(double *out, const uint32_t *in, int B, const Fft512Tables *T, cudaStream_t st)
{
    if (B <= 0) return cudaSuccess;
    twist_ifft1_kernel<<<(B + 3) / 4, 128, 0, st>>>(out, in, B, T);
    return cudaGetLastError();
}

cudaError_t launch_twist_fft1(uint32_t *out, const double *in, int B, const Fft512Tables *T, cudaStream_t st)
{
    if (B <= 0) return cudaSuccess;
    twist_fft1_kernel<<<(B + 3) / 4, 128, 0, st>>>(out, in, B, T);
    return cudaGetLastError();
}

}  // namespace cfdb
