// FP64 negacyclic FFT for N = 1024 (512 complex points), one warp per
// polynomial, 16 complex values per lane, held in registers.
//
// Transform (the TwistIFFT/TwistFFT pair of TFHEpp, mulfft.hpp:57-121, whose
// spqlios layout is restated in oracle/tfhe_oracle.c):
//   forward  V(q) = sum_m z_m W^{mq},  z_m = (a_m + i a_{m+512}) w^m,
//            W = exp(2 pi i / 512), w = exp(2 pi i / 2048)
//   inverse  z_m = (1/512) sum_q V(q) W^{-mq}
//
// Factorisation 512 = 16 x 32 with m = m1 + 32 m2, q = q2 + 16 q1:
//   1. lane m1 holds z_{m1+32 m2}, m2 = 0..15: 16-point DFT over m2 in
//      registers, then twiddle W^{m1 q2};
//   2. one shared-memory transpose (per-warp 8.5 KB, rows padded so both the
//      write and the read are bank-conflict free);
//   3. lane (q2 = lane & 15, h = lane >> 4) holds the 16 values with m1 of
//      parity h: 16-point DFT in registers, then one radix-2 step with the
//      partner lane (lane ^ 16) through warp shuffles.
// After the forward transform lane L owns the 16 frequencies
//   q(L, s) = (L & 15) + 16 * ((s & 7) + 8 * (L >> 4) + 16 * (s >> 3)),
// which is also the layout the bootstrapping key is stored in, so the
// frequency-domain multiply-accumulate needs no data exchange, and the
// inverse transform starts from the same registers.
#pragma once
#include "common.cuh"

namespace cfdb {

// the frequency owned by slot s of lane L after the forward transform
__host__ __device__ __forceinline__ int fft512_freq(int lane, int s)
{
    return (lane & 15) + 16 * ((s & 7) + 8 * (lane >> 4) + 16 * (s >> 3));
}

// twiddle tables (built on the host in long double, see capi.cu):
//   tw512[q2 * 32 + m1] = W^{m1 q2}     (16 x 32)
//   twist[m2 * 32 + m1] = w^{m1 + 32 m2} (16 x 32)
//   w32[j]              = exp(2 pi i j / 32), j < 16
struct Fft512Tables {
    double2 tw512[512];
    double2 twist[512];
    double2 w32[16];
};

// y_k = sum_n a_n i^{S n k}
template <int S>
__device__ __forceinline__ void dft4(double2 &a0, double2 &a1, double2 &a2, double2 &a3)
{
    double2 s02 = cadd(a0, a2), d02 = csub(a0, a2);
    double2 s13 = cadd(a1, a3), d13 = csub(a1, a3);
    double2 t = (S > 0) ? make_double2(-d13.y, d13.x) : make_double2(d13.y, -d13.x);
    a0 = cadd(s02, s13);
    a2 = csub(s02, s13);
    a1 = cadd(d02, t);
    a3 = csub(d02, t);
}

// multiply by exp(S * 2 pi i e / 16) for the exponents the radix-4x4 DFT needs
template <int S, int E>
__device__ __forceinline__ double2 w16(double2 a)
{
    constexpr double C1 = 0.92387953251128673848;  // cos(pi/8)
    constexpr double S1 = 0.38268343236508978178;  // sin(pi/8)
    constexpr double R2 = 0.70710678118654752440;  // sqrt(2)/2
    if constexpr (E == 0) return a;
    else if constexpr (E == 4) return (S > 0) ? make_double2(-a.y, a.x) : make_double2(a.y, -a.x);
    else if constexpr (E == 2) {
        // (1 + S i) r
        return (S > 0) ? make_double2(R2 * (a.x - a.y), R2 * (a.x + a.y))
                       : make_double2(R2 * (a.x + a.y), R2 * (a.y - a.x));
    } else if constexpr (E == 6) {
        // (-1 + S i) r
        return (S > 0) ? make_double2(-R2 * (a.x + a.y), R2 * (a.x - a.y))
                       : make_double2(R2 * (a.y - a.x), -R2 * (a.x + a.y));
    } else {
        constexpr double c = (E == 1) ? C1 : (E == 3) ? S1 : -C1;   // E = 1, 3, 9
        constexpr double s0 = (E == 1) ? S1 : (E == 3) ? C1 : -S1;
        constexpr double s = (S > 0) ? s0 : -s0;
        return make_double2(fma(a.x, c, -a.y * s), fma(a.x, s, a.y * c));
    }
}

// in-place 16-point DFT, natural order in and out: X[k] = sum x[n] e^{S 2 pi i nk/16}
template <int S>
__device__ __forceinline__ void dft16(double2 v[16])
{
    // n = n1 + 4 n2, k = k2 + 4 k1
#pragma unroll
    for (int n1 = 0; n1 < 4; ++n1) dft4<S>(v[n1], v[n1 + 4], v[n1 + 8], v[n1 + 12]);
    // v[n1 + 4 k2] *= W16^{n1 k2}
    v[5] = w16<S, 1>(v[5]);
    v[6] = w16<S, 2>(v[6]);
    v[7] = w16<S, 3>(v[7]);
    v[9] = w16<S, 2>(v[9]);
    v[10] = w16<S, 4>(v[10]);
    v[11] = w16<S, 6>(v[11]);
    v[13] = w16<S, 3>(v[13]);
    v[14] = w16<S, 6>(v[14]);
    v[15] = w16<S, 9>(v[15]);
#pragma unroll
    for (int k2 = 0; k2 < 4; ++k2) dft4<S>(v[4 * k2], v[4 * k2 + 1], v[4 * k2 + 2], v[4 * k2 + 3]);
    // v[4 k2 + k1] holds X[k2 + 4 k1]: transpose the register names
    double2 t[16];
#pragma unroll
    for (int k2 = 0; k2 < 4; ++k2)
#pragma unroll
        for (int k1 = 0; k1 < 4; ++k1) t[k2 + 4 * k1] = v[4 * k2 + k1];
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = t[i];
}

// transpose scratch (FFT512_XP entries per warp): 32 rows of 16 values
// padded to 17, so that both the row-wise write and the column-wise read are
// free of bank conflicts and every address is a per-lane base plus a
// compile-time offset
__device__ __forceinline__ int xp_index(int m1, int q2) { return m1 * 17 + q2; }

// forward transform of the 16 values z_{lane+32 m2} held in v[m2]; on return
// v[s] = V(fft512_freq(lane, s)).  xp: this warp's FFT512_XP-entry scratch.
__device__ __forceinline__ void fft512_fwd(double2 v[16], double2 *xp, const Fft512Tables &T, int lane)
{
    dft16<1>(v);
#pragma unroll
    for (int q2 = 1; q2 < 16; ++q2) v[q2] = cmul(v[q2], T.tw512[q2 * 32 + lane]);
    __syncwarp();
#pragma unroll
    for (int q2 = 0; q2 < 16; ++q2) xp[xp_index(lane, q2)] = v[q2];
    __syncwarp();
    const int h = lane >> 4, q2 = lane & 15;
#pragma unroll
    for (int m1p = 0; m1p < 16; ++m1p) v[m1p] = xp[xp_index(2 * m1p + h, q2)];
    dft16<1>(v);
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        double2 send = h ? v[j] : v[8 + j];
        double2 recv = shfl_xor2(send, 16);
        double2 a = h ? recv : v[j];
        double2 b = h ? v[8 + j] : recv;
        double2 t = cmul(b, T.w32[j + 8 * h]);
        v[j] = cadd(a, t);
        v[8 + j] = csub(a, t);
    }
}

// inverse transform: v[s] = V(fft512_freq(lane, s)) in, v[m2] = 512 z_{lane+32 m2} out
__device__ __forceinline__ void fft512_inv(double2 v[16], double2 *xp, const Fft512Tables &T, int lane)
{
    const int h = lane >> 4, q2 = lane & 15;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        double2 a = v[j], b = v[8 + j];
        double2 g0 = cadd(a, b);
        double2 g1 = cmulc(csub(a, b), T.w32[j + 8 * h]);
        double2 send = h ? g0 : g1;
        double2 recv = shfl_xor2(send, 16);
        v[j] = h ? recv : g0;
        v[8 + j] = h ? g1 : recv;
    }
    dft16<-1>(v);
    __syncwarp();
#pragma unroll
    for (int m1p = 0; m1p < 16; ++m1p) xp[xp_index(2 * m1p + h, q2)] = v[m1p];
    __syncwarp();
#pragma unroll
    for (int k = 0; k < 16; ++k) v[k] = xp[xp_index(lane, k)];
#pragma unroll
    for (int k = 1; k < 16; ++k) v[k] = cmulc(v[k], T.tw512[k * 32 + lane]);
    dft16<-1>(v);
}

// TFHEpp's torus32 conversion: uint32_t(int64_t(x)), truncation toward zero
// (thirdparty/TFHEpp/thirdparties/spqlios/fft_processor_spqlios.cpp:121)
__device__ __forceinline__ uint32_t f64_to_torus32(double x) { return static_cast<uint32_t>(__double2ll_rz(x)); }

}  // namespace cfdb
