// FP32 negacyclic FFT for N = 1024 (512 complex points), one warp per
// polynomial, 16 complex values per lane: the same 16 x 32 factorisation and
// frequency ownership as the FP64 transform in fft_f64.cuh, in single
// precision.  Complex additions and subtractions use Blackwell's packed
// two-lane FP32 instructions (add/sub.rn.f32x2, one instruction per complex
// value).
#pragma once
#include "common.cuh"

namespace cfdb {

struct Fft512TablesF {
    float2 tw512[512];
    float2 twist[512];
    float2 untwist[512];   // conj(twist) / 512: inverse untwist and scaling in one product
    float2 w32[16];
};

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

__device__ __forceinline__ void ffft512_fwd(float2 v[16], float2 *xp, const Fft512TablesF &T, int lane)
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

__device__ __forceinline__ void ffft512_inv(float2 v[16], float2 *xp, const Fft512TablesF &T, int lane)
{
    const int h = lane >> 4, q2 = lane & 15;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        float2 a = v[j], b = v[8 + j];
        float2 g0 = fadd2(a, b);
        float2 g1 = fcmulc(fsub2(a, b), T.w32[j + 8 * h]);
        float2 send = h ? g0 : g1;
        float2 recv = shfl_xor_f2(send, 16);
        v[j] = h ? recv : g0;
        v[8 + j] = h ? g1 : recv;
    }
    fdft16<-1>(v);
    __syncwarp();
#pragma unroll
    for (int m1p = 0; m1p < 16; ++m1p) xp[xpf_index(2 * m1p + h, q2)] = v[m1p];
    __syncwarp();
#pragma unroll
    for (int k = 0; k < 16; ++k) v[k] = xp[xpf_index(lane, k)];
#pragma unroll
    for (int k = 1; k < 16; ++k) v[k] = fcmulc(v[k], T.tw512[k * 32 + lane]);
    fdft16<-1>(v);
}

}  // namespace cfdb
