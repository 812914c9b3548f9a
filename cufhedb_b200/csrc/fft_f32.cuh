// FP32 negacyclic FFT for N = 1024 (512 complex points), one warp per
// polynomial, 16 complex values per lane: the same 16 x 32 factorisation and
// frequency ownership as the FP64 transform in fft_f64.cuh, in single
// precision.  Complex additions and subtractions use Blackwell's packed
// two-lane FP32 instructions (add/sub.rn.f32x2, one instruction per complex
// value).
#pragma once
#include "common.cuh"

namespace cfdb {

// Tables of the FP32 transforms.  The plain set: the twist, the stage-1 and
// radix-2 twiddles as (c, s), and for the paired inverse the same with each
// cosine and sine duplicated (c, c, s, s) plus the untwist (conj(twist) / 512).
struct Fft512TablesPlain {
    float2 tw512[512];
    float2 twist[512];
    float2 w32[16];
    float4 tw512p[512];
    float4 untwistp[512];   // conj(twist) / 512: inverse untwist and scaling in one product
    float4 w32p[16];
};
// The folded set: the lane's part of the twist rides on the forward stage-1
// twiddles and the lane's part of the untwist (with the 1/512 scale) on the
// inverse stage-1 twiddles; the per-register parts are compile-time constants
// (cw64, untwist_m2), and so are the forward radix-2 twiddles.
struct Fft512TablesFold {
    float2 tw512w[512];   // tw512w[q2 * 32 + m1] = W^{m1 q2} w^{m1}
    float4 tw512u[512];   // tw512u[k * 32 + m1] = W^{m1 k} w^{m1} / 512 (used conjugated)
    float4 w32p[16];
};
// both sets, as the context keeps them in global memory; a kernel copies the
// set it uses into shared memory.  tc_b: the two FP16 limbs of the constant
// matrix of the tensor-core stage 1 (tc_stage1.cuh), hi then lo.
struct Fft512TablesF {
    Fft512TablesPlain plain;
    Fft512TablesFold fold;
    uint16_t tc_b[2][32 * 32];
};
static_assert(sizeof(Fft512TablesPlain) % 16 == 0 && sizeof(Fft512TablesFold) % 16 == 0, "16-byte copies");

__device__ __forceinline__ unsigned long long f2_bits(float2 a)
{
    return *reinterpret_cast<unsigned long long *>(&a);
}
__device__ __forceinline__ float2 bits_f2(unsigned long long a) { return *reinterpret_cast<float2 *>(&a); }

__device__ __forceinline__ float2 fadd2(float2 a, float2 b)
{
    unsigned long long r;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(f2_bits(a)), "l"(f2_bits(b)));
    return bits_f2(r);
}
__device__ __forceinline__ float2 fsub2(float2 a, float2 b)
{
    unsigned long long r;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(f2_bits(a)), "l"(f2_bits(b)));
    return bits_f2(r);
}
__device__ __forceinline__ float2 fcmul(float2 a, float2 b)
{
    return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
// a * conj(b)
__device__ __forceinline__ float2 fcmulc(float2 a, float2 b)
{
    return make_float2(fmaf(a.x, b.x, a.y * b.y), fmaf(a.y, b.x, -a.x * b.y));
}
__device__ __forceinline__ void fcfma(float2 &acc, float2 a, float2 b)
{
    acc.x = fmaf(a.x, b.x, acc.x);
    acc.x = fmaf(-a.y, b.y, acc.x);
    acc.y = fmaf(a.x, b.y, acc.y);
    acc.y = fmaf(a.y, b.x, acc.y);
}
__device__ __forceinline__ float2 shfl_xor_f2(float2 v, int m)
{
    return make_float2(__shfl_xor_sync(0xffffffffu, v.x, m), __shfl_xor_sync(0xffffffffu, v.y, m));
}

template <int S>
__device__ __forceinline__ void fdft4(float2 &a0, float2 &a1, float2 &a2, float2 &a3)
{
    float2 s02 = fadd2(a0, a2), d02 = fsub2(a0, a2);
    float2 s13 = fadd2(a1, a3), d13 = fsub2(a1, a3);
    float2 t = (S > 0) ? make_float2(-d13.y, d13.x) : make_float2(d13.y, -d13.x);
    a0 = fadd2(s02, s13);
    a2 = fsub2(s02, s13);
    a1 = fadd2(d02, t);
    a3 = fsub2(d02, t);
}

template <int S, int E>
__device__ __forceinline__ float2 fw16(float2 a)
{
    constexpr float C1 = 0.92387953251128673848f;
    constexpr float S1 = 0.38268343236508978178f;
    constexpr float R2 = 0.70710678118654752440f;
    if constexpr (E == 0) return a;
    else if constexpr (E == 4) return (S > 0) ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
    else if constexpr (E == 2) {
        return (S > 0) ? make_float2(R2 * (a.x - a.y), R2 * (a.x + a.y))
                       : make_float2(R2 * (a.x + a.y), R2 * (a.y - a.x));
    } else if constexpr (E == 6) {
        return (S > 0) ? make_float2(-R2 * (a.x + a.y), R2 * (a.x - a.y))
                       : make_float2(R2 * (a.y - a.x), -R2 * (a.x + a.y));
    } else {
        constexpr float c = (E == 1) ? C1 : (E == 3) ? S1 : -C1;
        constexpr float s0 = (E == 1) ? S1 : (E == 3) ? C1 : -S1;
        constexpr float s = (S > 0) ? s0 : -s0;
        return make_float2(fmaf(a.x, c, -a.y * s), fmaf(a.x, s, a.y * c));
    }
}

template <int S>
__device__ __forceinline__ void fdft16(float2 v[16])
{
#pragma unroll
    for (int n1 = 0; n1 < 4; ++n1) fdft4<S>(v[n1], v[n1 + 4], v[n1 + 8], v[n1 + 12]);
    v[5] = fw16<S, 1>(v[5]);
    v[6] = fw16<S, 2>(v[6]);
    v[7] = fw16<S, 3>(v[7]);
    v[9] = fw16<S, 2>(v[9]);
    v[10] = fw16<S, 4>(v[10]);
    v[11] = fw16<S, 6>(v[11]);
    v[13] = fw16<S, 3>(v[13]);
    v[14] = fw16<S, 6>(v[14]);
    v[15] = fw16<S, 9>(v[15]);
#pragma unroll
    for (int k2 = 0; k2 < 4; ++k2) fdft4<S>(v[4 * k2], v[4 * k2 + 1], v[4 * k2 + 2], v[4 * k2 + 3]);
    float2 t[16];
#pragma unroll
    for (int k2 = 0; k2 < 4; ++k2)
#pragma unroll
        for (int k1 = 0; k1 < 4; ++k1) t[k2 + 4 * k1] = v[4 * k2 + k1];
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = t[i];
}

// 8-byte elements in rows padded to 17 (FFT512_XP entries per warp): each
// half-warp hits 16 distinct 8-byte bank pairs on both the row-wise write and
// the column-wise read, with compile-time offsets from a per-lane base
__device__ __forceinline__ int xpf_index(int m1, int q2) { return m1 * 17 + q2; }

// e^{2 pi i j / 32} for j < 8 as compile-time constants once unrolled
__device__ __forceinline__ float2 w32_const(int j)
{
    constexpr float C[9] = {1.000000000e+00f, 9.807852804e-01f, 9.238795325e-01f, 8.314696123e-01f,
                            7.071067812e-01f, 5.555702330e-01f, 3.826834324e-01f, 1.950903220e-01f, 0.0f};
    return make_float2(C[j], C[8 - j]);
}

template <class TT>
__device__ __forceinline__ void ffft512_fwd(float2 v[16], float2 *xp, const TT &T, int lane)
{
    fdft16<1>(v);
#pragma unroll
    for (int q2 = 1; q2 < 16; ++q2) v[q2] = fcmul(v[q2], T.tw512[q2 * 32 + lane]);
    __syncwarp();
#pragma unroll
    for (int q2 = 0; q2 < 16; ++q2) xp[xpf_index(lane, q2)] = v[q2];
    __syncwarp();
    const int h = lane >> 4, q2 = lane & 15;
#pragma unroll
    for (int m1p = 0; m1p < 16; ++m1p) v[m1p] = xp[xpf_index(2 * m1p + h, q2)];
    fdft16<1>(v);
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        float2 send = h ? v[j] : v[8 + j];
        float2 recv = shfl_xor_f2(send, 16);
        float2 a = h ? recv : v[j];
        float2 b = h ? v[8 + j] : recv;
        float2 t = fcmul(b, T.w32[j + 8 * h]);
        v[j] = fadd2(a, t);
        v[8 + j] = fsub2(a, t);
    }
}

// a * e^{2 pi i m2 / 64} = a * w^{32 m2} (compile-time constants once unrolled)
__device__ __forceinline__ float2 cw64(float2 a, int m2)
{
    constexpr float C[17] = {1.000000000e+00f, 9.951847267e-01f, 9.807852804e-01f, 9.569403357e-01f,
                             9.238795325e-01f, 8.819212643e-01f, 8.314696123e-01f, 7.730104534e-01f,
                             7.071067812e-01f, 6.343932842e-01f, 5.555702330e-01f, 4.713967368e-01f,
                             3.826834324e-01f, 2.902846773e-01f, 1.950903220e-01f, 9.801714033e-02f, 0.0f};
    if (m2 == 0) return a;
    const float c = C[m2], sn = C[16 - m2];
    return make_float2(fmaf(a.x, c, -a.y * sn), fmaf(a.x, sn, a.y * c));
}

// forward transform of inputs that carry only the per-register part of the
// twist, v[m2] = (a_m + i a_{m+512}) w^{32 m2} (cw64): the lane's part w^{lane}
// is applied with the stage-1 twiddles (tw512w, q2 = 0 included), the radix-2
// twiddles come from constants.  Same output as ffft512_fwd on fully twisted
// inputs.
__device__ __forceinline__ void ffft512_fwd_tw_rest(float2 v[16], float2 *xp, const Fft512TablesFold &T, int lane);
__device__ __forceinline__ void ffft512_fwd_tw(float2 v[16], float2 *xp, const Fft512TablesFold &T, int lane)
{
    fdft16<1>(v);
    ffft512_fwd_tw_rest(v, xp, T, lane);
}

// everything after the first 16-point DFT: v[q2] = X[q2] of this lane (the
// tensor-core path computes X on the tensor cores, tc_stage1.cuh)
__device__ __forceinline__ void ffft512_fwd_tw_rest(float2 v[16], float2 *xp, const Fft512TablesFold &T, int lane)
{
#pragma unroll
    for (int q2 = 0; q2 < 16; ++q2) v[q2] = fcmul(v[q2], T.tw512w[q2 * 32 + lane]);
    __syncwarp();
#pragma unroll
    for (int q2 = 0; q2 < 16; ++q2) xp[xpf_index(lane, q2)] = v[q2];
    __syncwarp();
    const int h = lane >> 4, q2 = lane & 15;
#pragma unroll
    for (int m1p = 0; m1p < 16; ++m1p) v[m1p] = xp[xpf_index(2 * m1p + h, q2)];
    fdft16<1>(v);
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        float2 send = h ? v[j] : v[8 + j];
        float2 recv = shfl_xor_f2(send, 16);
        float2 a = h ? recv : v[j];
        float2 b = h ? v[8 + j] : recv;
        float2 t = j == 0 ? b : fcmul(b, w32_const(j));
        if (h) t = make_float2(-t.y, t.x);
        v[j] = fadd2(a, t);
        v[8 + j] = fsub2(a, t);
    }
}

// ---- paired form: two polynomials transformed in lock step ----------------------
// A CP holds one complex value of each of two polynomials as (re_0, re_1),
// (im_0, im_1): every operation is one packed f32x2 instruction per
// component, the same for both.  Used for the hi and lo limb of one output.
struct CP {
    unsigned long long re, im;
};

__device__ __forceinline__ unsigned long long pk2(float a, float b)
{
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
    return r;
}
__device__ __forceinline__ float2 unpk2(unsigned long long v)
{
    float2 r;
    asm("mov.b64 {%0, %1}, %2;" : "=f"(r.x), "=f"(r.y) : "l"(v));
    return r;
}
__device__ __forceinline__ unsigned long long a2(unsigned long long a, unsigned long long b)
{
    unsigned long long r;
    asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ unsigned long long s2(unsigned long long a, unsigned long long b)
{
    unsigned long long r;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ unsigned long long m2(unsigned long long a, unsigned long long b)
{
    unsigned long long r;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ unsigned long long f2(unsigned long long a, unsigned long long b, unsigned long long c)
{
    unsigned long long r;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
    return r;
}

__device__ __forceinline__ CP padd(CP a, CP b) { return CP{a2(a.re, b.re), a2(a.im, b.im)}; }
__device__ __forceinline__ CP psub(CP a, CP b) { return CP{s2(a.re, b.re), s2(a.im, b.im)}; }
// a * (c + i s) for a twiddle stored (c, c, s, s)
__device__ __forceinline__ CP pmul_t(CP a, float4 w)
{
    const unsigned long long C = pk2(w.x, w.y), S = pk2(w.z, w.w);
    return CP{s2(m2(a.re, C), m2(a.im, S)), f2(a.re, S, m2(a.im, C))};
}
// a * conj(c + i s)
__device__ __forceinline__ CP pmulc_t(CP a, float4 w)
{
    const unsigned long long C = pk2(w.x, w.y), S = pk2(w.z, w.w);
    return CP{f2(a.re, C, m2(a.im, S)), s2(m2(a.im, C), m2(a.re, S))};
}
__device__ __forceinline__ CP pshfl_xor(CP v, int m)
{
    const float2 r = unpk2(v.re), i = unpk2(v.im);
    return CP{pk2(__shfl_xor_sync(0xffffffffu, r.x, m), __shfl_xor_sync(0xffffffffu, r.y, m)),
              pk2(__shfl_xor_sync(0xffffffffu, i.x, m), __shfl_xor_sync(0xffffffffu, i.y, m))};
}
__device__ __forceinline__ CP psel(bool c, CP a, CP b) { return c ? a : b; }

template <int S>
__device__ __forceinline__ void pdft4(CP &a0, CP &a1, CP &a2_, CP &a3)
{
    const CP s02 = padd(a0, a2_), d02 = psub(a0, a2_);
    const CP s13 = padd(a1, a3), d13 = psub(a1, a3);
    a0 = padd(s02, s13);
    a2_ = psub(s02, s13);
    // a1 = d02 + i^S d13, a3 = d02 - i^S d13 (i d = (-d.im, d.re))
    if constexpr (S > 0) {
        a1 = CP{s2(d02.re, d13.im), a2(d02.im, d13.re)};
        a3 = CP{a2(d02.re, d13.im), s2(d02.im, d13.re)};
    } else {
        a1 = CP{a2(d02.re, d13.im), s2(d02.im, d13.re)};
        a3 = CP{s2(d02.re, d13.im), a2(d02.im, d13.re)};
    }
}

template <int S, int E>
__device__ __forceinline__ CP pw16(CP a)
{
    constexpr float C1 = 0.92387953251128673848f;
    constexpr float S1 = 0.38268343236508978178f;
    constexpr float R2 = 0.70710678118654752440f;
    if constexpr (E == 0) return a;
    else if constexpr (E == 4) {
        const unsigned long long zero = pk2(0.0f, 0.0f);
        return (S > 0) ? CP{s2(zero, a.im), a.re} : CP{a.im, s2(zero, a.re)};
    } else if constexpr (E == 2) {
        const unsigned long long r = pk2(R2, R2);
        return (S > 0) ? CP{m2(s2(a.re, a.im), r), m2(a2(a.re, a.im), r)}
                       : CP{m2(a2(a.re, a.im), r), m2(s2(a.im, a.re), r)};
    } else if constexpr (E == 6) {
        const unsigned long long r = pk2(R2, R2), nr = pk2(-R2, -R2);
        return (S > 0) ? CP{m2(a2(a.re, a.im), nr), m2(s2(a.re, a.im), r)}
                       : CP{m2(s2(a.im, a.re), r), m2(a2(a.re, a.im), nr)};
    } else {
        constexpr float c = (E == 1) ? C1 : (E == 3) ? S1 : -C1;
        constexpr float s0 = (E == 1) ? S1 : (E == 3) ? C1 : -S1;
        constexpr float sn = (S > 0) ? s0 : -s0;
        const unsigned long long Cp = pk2(c, c), Sp = pk2(sn, sn), NSp = pk2(-sn, -sn);
        return CP{f2(a.re, Cp, m2(a.im, NSp)), f2(a.re, Sp, m2(a.im, Cp))};
    }
}

template <int S>
__device__ __forceinline__ void pdft16(CP v[16])
{
#pragma unroll
    for (int n1 = 0; n1 < 4; ++n1) pdft4<S>(v[n1], v[n1 + 4], v[n1 + 8], v[n1 + 12]);
    v[5] = pw16<S, 1>(v[5]);
    v[6] = pw16<S, 2>(v[6]);
    v[7] = pw16<S, 3>(v[7]);
    v[9] = pw16<S, 2>(v[9]);
    v[10] = pw16<S, 4>(v[10]);
    v[11] = pw16<S, 6>(v[11]);
    v[13] = pw16<S, 3>(v[13]);
    v[14] = pw16<S, 6>(v[14]);
    v[15] = pw16<S, 9>(v[15]);
#pragma unroll
    for (int k2 = 0; k2 < 4; ++k2) pdft4<S>(v[4 * k2], v[4 * k2 + 1], v[4 * k2 + 2], v[4 * k2 + 3]);
    CP t[16];
#pragma unroll
    for (int k2 = 0; k2 < 4; ++k2)
#pragma unroll
        for (int k1 = 0; k1 < 4; ++k1) t[k2 + 4 * k1] = v[4 * k2 + k1];
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = t[i];
}

// inverse transform of two polynomials at once (the forward steps in reverse
// with conjugate twiddles);
// xp: this warp's FFT512_XP 8-byte entries, through which the real and the
// imaginary parts are transposed one after the other.  Output v[m2] =
// 512 z_{lane + 32 m2} (multiply by untwistp to finish); with FOLD the stage-1
// twiddles (tw512u) also carry conj(w^{lane}) / 512, so the output is
// z_{lane + 32 m2} w^{32 m2}... times the rest of the twist only, which
// untwist_m2 removes with compile-time constants instead of a table read.
template <bool FOLD, class TT>
__device__ __forceinline__ void pfft512_inv(CP v[16], unsigned long long *xp, const TT &T, int lane)
{
    const int h = lane >> 4, q2 = lane & 15;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const CP a = v[j], b = v[8 + j];
        const CP g0 = padd(a, b);
        const CP g1 = pmulc_t(psub(a, b), T.w32p[j + 8 * h]);
        const CP recv = pshfl_xor(psel(h, g0, g1), 16);
        v[j] = psel(h, recv, g0);
        v[8 + j] = psel(h, g1, recv);
    }
    pdft16<-1>(v);
    __syncwarp();
#pragma unroll
    for (int m1p = 0; m1p < 16; ++m1p) xp[xpf_index(2 * m1p + h, q2)] = v[m1p].re;
    __syncwarp();
#pragma unroll
    for (int k = 0; k < 16; ++k) v[k].re = xp[xpf_index(lane, k)];
    __syncwarp();
#pragma unroll
    for (int m1p = 0; m1p < 16; ++m1p) xp[xpf_index(2 * m1p + h, q2)] = v[m1p].im;
    __syncwarp();
#pragma unroll
    for (int k = 0; k < 16; ++k) v[k].im = xp[xpf_index(lane, k)];
    if constexpr (FOLD) {
#pragma unroll
        for (int k = 0; k < 16; ++k) v[k] = pmulc_t(v[k], T.tw512u[k * 32 + lane]);
    } else {
#pragma unroll
        for (int k = 1; k < 16; ++k) v[k] = pmulc_t(v[k], T.tw512p[k * 32 + lane]);
    }
    pdft16<-1>(v);
}

// a * conj(e^{2 pi i m2 / 64}) = a * conj(w^{32 m2}): the per-register part of
// the untwist left after pfft512_inv (compile-time constants once unrolled)
__device__ __forceinline__ float2 untwist_m2(float2 a, int m2)
{
    constexpr float C[16] = {1.000000000e+00f, 9.951847267e-01f, 9.807852804e-01f, 9.569403357e-01f,
                             9.238795325e-01f, 8.819212643e-01f, 8.314696123e-01f, 7.730104534e-01f,
                             7.071067812e-01f, 6.343932842e-01f, 5.555702330e-01f, 4.713967368e-01f,
                             3.826834324e-01f, 2.902846773e-01f, 1.950903220e-01f, 9.801714033e-02f};
    if (m2 == 0) return a;
    const float c = C[m2], sn = C[16 - m2];
    return make_float2(fmaf(a.x, c, a.y * sn), fmaf(a.y, c, -a.x * sn));
}
__device__ __forceinline__ CP untwist_m2(CP a, int m2)
{
    constexpr float C[16] = {1.000000000e+00f, 9.951847267e-01f, 9.807852804e-01f, 9.569403357e-01f,
                             9.238795325e-01f, 8.819212643e-01f, 8.314696123e-01f, 7.730104534e-01f,
                             7.071067812e-01f, 6.343932842e-01f, 5.555702330e-01f, 4.713967368e-01f,
                             3.826834324e-01f, 2.902846773e-01f, 1.950903220e-01f, 9.801714033e-02f};
    if (m2 == 0) return a;
    return pmulc_t(a, make_float4(C[m2], C[m2], C[16 - m2], C[16 - m2]));
}


}  // namespace cfdb
