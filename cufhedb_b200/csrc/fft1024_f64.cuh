// FP64 negacyclic FFT for N = 2048 (1024 complex points, the lvl2 ring of the
// 64-bit torus): two warps (64 threads) per polynomial, 16 complex values per
// thread.  Same transform definition as fft_f64.cuh with w = exp(2 pi i/4096),
// W = exp(2 pi i/1024) (TFHEpp TwistIFFT/TwistFFT<lvl2param>,
// thirdparty/TFHEpp/include/mulfft.hpp:57-121).
//
// Factorisation 1024 = 16 x 64 with m = m1 + 64 m2, q = q2 + 16 q1:
//   1. thread m1 holds z_{m1+64 m2}: 16-point DFT over m2, twiddle W^{m1 q2};
//   2. one shared-memory transpose across the two warps (16 KB, swizzled);
//   3. thread (q2 = t >> 2, h = t & 3) holds the values with m1 = 4 m1' + h:
//      16-point DFT over m1', then the radix-4 over h as two radix-2 steps
//      through warp shuffles (partners t ^ 2, then t ^ 1).
// Thread t then owns the 16 frequencies
//   q(t, s) = (t >> 2) + 16 * (8 h1 + 4 h0 + (s & 3) + 16 * ((s >> 2) & 1) + 32 * (s >> 3)),
//   h0 = t & 1, h1 = (t >> 1) & 1.
#pragma once
#include "common.cuh"
#include "fft_f64.cuh"

namespace cfdb {

__host__ __device__ __forceinline__ int fft1024_freq(int t, int s)
{
    const int h0 = t & 1, h1 = (t >> 1) & 1;
    return (t >> 2) + 16 * (8 * h1 + 4 * h0 + (s & 3) + 16 * ((s >> 2) & 1) + 32 * (s >> 3));
}

// tw1024[q2 * 64 + m1] = W^{m1 q2}; twist[m2 * 64 + m1] = w^{m1 + 64 m2};
// w32[j] = exp(2 pi i j/32), w64[j] = exp(2 pi i j/64) for j < 16
struct Fft1024Tables {
    double2 tw1024[1024];
    double2 twist[1024];
    double2 w32[16];
    double2 w64[16];
};

__device__ __forceinline__ int xp2_index(int m1, int q2)
{
    return m1 * 16 + (q2 ^ (((m1 & 3) << 1) | ((m1 >> 2) & 1)));
}

// synchronises the two warps of one polynomial (named barrier `id`, 64 threads)
__device__ __forceinline__ void pair_sync(int id) { asm volatile("bar.sync %0, 64;" ::"r"(id) : "memory"); }

// multiply by i^b0 (b0 in {0,1}), S = +1, or by (-i)^b0, S = -1
template <int S>
__device__ __forceinline__ double2 mul_ipow(double2 a, int b0)
{
    if (!b0) return a;
    return (S > 0) ? make_double2(-a.y, a.x) : make_double2(a.y, -a.x);
}

// v[m2] = z_{t+64 m2} in; v[s] = V(fft1024_freq(t, s)) out.  xp: 1024-entry
// scratch shared by the two warps of the polynomial, bar: named barrier id.
__device__ __forceinline__ void fft1024_fwd(double2 v[16], double2 *xp, const Fft1024Tables &T, int t, int bar)
{
    dft16<1>(v);
#pragma unroll
    for (int q2 = 1; q2 < 16; ++q2) v[q2] = cmul(v[q2], T.tw1024[q2 * 64 + t]);
    pair_sync(bar);
#pragma unroll
    for (int q2 = 0; q2 < 16; ++q2) xp[xp2_index(t, q2)] = v[q2];
    pair_sync(bar);
    const int q2 = t >> 2, h = t & 3, h0 = t & 1, h1 = (t >> 1) & 1;
#pragma unroll
    for (int m1p = 0; m1p < 16; ++m1p) v[m1p] = xp[xp2_index(4 * m1p + h, q2)];
    dft16<1>(v);   // v[q1'] = G_h(q1')
    // radix-2 over h1 with partner t ^ 2: keep q1' = j + 8 h1, both b0
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        double2 send = h1 ? v[j] : v[8 + j];
        double2 recv = shfl_xor2(send, 2);
        double2 a = h1 ? recv : v[j];        // G_{h0}(q1')
        double2 b = h1 ? v[8 + j] : recv;    // G_{h0+2}(q1')
        double2 tb = cmul(b, T.w32[j + 8 * h1]);
        v[j] = cadd(a, tb);                  // H_{h0}(q1', b0 = 0)
        v[8 + j] = csub(a, tb);              // H_{h0}(q1', b0 = 1)
    }
    // radix-2 over h0 with partner t ^ 1: keep q1' = 8 h1 + 4 h0 + jj
    double2 r[16];
#pragma unroll
    for (int b0 = 0; b0 < 2; ++b0)
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) {
            const double2 lo = v[jj + 8 * b0], hi = v[4 + jj + 8 * b0];
            double2 send = h0 ? lo : hi;
            double2 recv = shfl_xor2(send, 1);
            double2 H0 = h0 ? recv : lo;
            double2 H1 = h0 ? hi : recv;
            double2 t1 = mul_ipow<1>(cmul(H1, T.w64[8 * h1 + 4 * h0 + jj]), b0);
            r[jj + 4 * b0] = cadd(H0, t1);       // b1 = 0
            r[jj + 4 * b0 + 8] = csub(H0, t1);   // b1 = 1
        }
#pragma unroll
    for (int s = 0; s < 16; ++s) v[s] = r[s];
}

// v[s] = V(fft1024_freq(t, s)) in; v[m2] = 1024 z_{t+64 m2} out
__device__ __forceinline__ void fft1024_inv(double2 v[16], double2 *xp, const Fft1024Tables &T, int t, int bar)
{
    const int q2 = t >> 2, h = t & 3, h0 = t & 1, h1 = (t >> 1) & 1;
    // inverse radix-2 over h0: thread h0 ends with H_{h0}(q1' = 8 h1 + jj', b0) for jj' < 8
    double2 r[16];
#pragma unroll
    for (int b0 = 0; b0 < 2; ++b0)
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) {
            const double2 p0 = v[jj + 4 * b0], p1 = v[jj + 4 * b0 + 8];
            double2 g0 = cadd(p0, p1);
            double2 g1 = cmulc(mul_ipow<-1>(csub(p0, p1), b0), T.w64[8 * h1 + 4 * h0 + jj]);
            double2 send = h0 ? g0 : g1;
            double2 recv = shfl_xor2(send, 1);
            // h0 = 0 keeps H_0 at q1' = 8h1 + jj (own) and 8h1 + 4 + jj (partner's)
            // h0 = 1 keeps H_1 at q1' = 8h1 + jj (partner's) and 8h1 + 4 + jj (own)
            r[jj + 8 * b0] = h0 ? recv : g0;
            r[4 + jj + 8 * b0] = h0 ? g1 : recv;
        }
    // inverse radix-2 over h1: thread h1 ends with G_{h0 + 2 h1}(q1') for all q1'
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const double2 a = r[j], b = r[8 + j];
        double2 g0 = cadd(a, b);
        double2 g1 = cmulc(csub(a, b), T.w32[j + 8 * h1]);
        double2 send = h1 ? g0 : g1;
        double2 recv = shfl_xor2(send, 2);
        v[j] = h1 ? recv : g0;
        v[8 + j] = h1 ? g1 : recv;
    }
    dft16<-1>(v);   // v[m1'] = Y[4 m1' + h][q2]
    pair_sync(bar);
#pragma unroll
    for (int m1p = 0; m1p < 16; ++m1p) xp[xp2_index(4 * m1p + h, q2)] = v[m1p];
    pair_sync(bar);
#pragma unroll
    for (int k = 0; k < 16; ++k) v[k] = xp[xp2_index(t, k)];
#pragma unroll
    for (int k = 1; k < 16; ++k) v[k] = cmulc(v[k], T.tw1024[k * 64 + t]);
    dft16<-1>(v);
}

// TFHEpp's torus64 conversion (spqlios fft_processor_spqlios.cpp:180-209):
// truncation toward zero, modulo 2^64 for |x| >= 2^63
__device__ __forceinline__ uint64_t f64_to_torus64(double x)
{
    if (fabs(x) < 9223372036854775808.0) return (uint64_t)__double2ll_rz(x);
    const unsigned long long bits = (unsigned long long)__double_as_longlong(x);
    const int e = (int)((bits >> 52) & 0x7FF) - 1075;
    const unsigned long long mant = (bits & ((1ull << 52) - 1)) | (1ull << 52);
    const unsigned long long mag = e >= 64 ? 0ull : (mant << e);
    return (bits >> 63) ? 0ull - mag : mag;
}

}  // namespace cfdb
