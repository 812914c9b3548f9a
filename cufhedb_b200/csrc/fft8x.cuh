// Negacyclic FFT of M = 1024 complex points spread over T = 128 threads (8
// values per thread, four warps), FP64: the lvl2 ring (N = 2048).
//
// Transform (TFHEpp TwistIFFT / TwistFFT, thirdparty/TFHEpp/include/
// mulfft.hpp:57-121, spqlios layout restated in oracle/tfhe_oracle.c):
//   forward  V(q) = sum_m z_m W_M^{mq},  z_m = (a_m + i a_{m+M}) w^m,
//            W_P = exp(2 pi i / P), w = exp(2 pi i / 4M)
//   inverse  M z_m = sum_q V(q) W_M^{-mq}
//
// Factorisation M = 8 x 8 x 16 (L = 16 lanes per group):
//   A. thread t holds z_{t + T j}, j < 8: 8-point DFT over j in registers
//      (output k), twiddle W_M^{t k};
//   B. shared-memory transpose across the four warps: thread u = a + L k
//      (a < L) receives the values of threads t = a + L b, b < 8, for its k;
//      8-point DFT over b (output q1), twiddle W_T^{a q1};
//   C. the 16-point DFT over a, as 2 x 8: a second transpose, inside each warp
//      (the 16 values of a (k, q1) sit in the 16 lanes of one warp with that
//      k), gives thread u' = q1 + 8 a0 + 16 k the values a = a0 + 2 j, j < 8;
//      an 8-point DFT over j in registers (output r); then one radix-2 step
//      with the partner lane u' ^ 8 (the other a0): the pair trades half of
//      its registers, and thread a0 keeps r = rl + 4 a0, rl < 4, computing
//      Y0[r] +- W_16^r Y1[r] for q2 = r and r + 8.
// The frequency q = k + 8 (q1 + 8 q2) then sits in register slot s of thread
// u' as given by fft8x_freq() below; the bootstrapping key is stored in the
// same [s][u'] order, so the per-frequency products need no data exchange
// and the inverse transform (the same steps in reverse) starts from the same
// registers.
#pragma once
#include "common.cuh"

namespace cfdb {

// ---- complex arithmetic ---------------------------------------------------------
__device__ __forceinline__ double2 cx_add(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 cx_sub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cx_mul(double2 a, double2 b)
{
    return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ double2 cx_mulc(double2 a, double2 b)   // a * conj(b)
{
    return make_double2(fma(a.x, b.x, a.y * b.y), fma(a.y, b.x, -a.x * b.y));
}
__device__ __forceinline__ void cx_fma(double2 &acc, double2 a, double2 b)
{
    acc.x = fma(a.x, b.x, acc.x);
    acc.x = fma(-a.y, b.y, acc.x);
    acc.y = fma(a.x, b.y, acc.y);
    acc.y = fma(a.y, b.x, acc.y);
}
__device__ __forceinline__ double2 cx_shfl_xor(double2 v, int m)
{
    return make_double2(__shfl_xor_sync(0xffffffffu, v.x, m), __shfl_xor_sync(0xffffffffu, v.y, m));
}
__device__ __forceinline__ double2 cx_scale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }

template <typename C> struct cx_real;
template <> struct cx_real<double2> { using type = double; };

// multiply by i^S (S = +1) or (-i) (S = -1)
template <int S, typename C>
__device__ __forceinline__ C cx_mul_i(C a)
{
    C r;
    if constexpr (S > 0) { r.x = -a.y; r.y = a.x; }
    else { r.x = a.y; r.y = -a.x; }
    return r;
}

// multiply by exp(S 2 pi i e / 8), e = 1, 2, 3
template <int S, int E, typename C>
__device__ __forceinline__ C cx_w8(C a)
{
    using R = typename cx_real<C>::type;
    constexpr R H = (R)0.70710678118654752440;
    if constexpr (E == 2) {
        return cx_mul_i<S>(a);
    } else {
        C r;
        if constexpr (E == 1) {   // (1 + S i) / sqrt2
            if constexpr (S > 0) { r.x = H * (a.x - a.y); r.y = H * (a.x + a.y); }
            else { r.x = H * (a.x + a.y); r.y = H * (a.y - a.x); }
        } else {                  // (-1 + S i) / sqrt2
            if constexpr (S > 0) { r.x = -H * (a.x + a.y); r.y = H * (a.x - a.y); }
            else { r.x = H * (a.y - a.x); r.y = -H * (a.x + a.y); }
        }
        return r;
    }
}

// y_k = sum_n a_n i^{S n k}, natural order in and out
template <int S, typename C>
__device__ __forceinline__ void cx_dft4(C &a0, C &a1, C &a2, C &a3)
{
    const C s02 = cx_add(a0, a2), d02 = cx_sub(a0, a2);
    const C s13 = cx_add(a1, a3), d13 = cx_sub(a1, a3);
    const C t = cx_mul_i<S>(d13);
    a0 = cx_add(s02, s13);
    a2 = cx_sub(s02, s13);
    a1 = cx_add(d02, t);
    a3 = cx_sub(d02, t);
}

// in-place 8-point DFT X[k] = sum x[n] exp(S 2 pi i nk / 8), natural order
template <int S, typename C>
__device__ __forceinline__ void cx_dft8(C v[8])
{
    // n = n1 + 2 n2, k = k2 + 4 k1
    cx_dft4<S>(v[0], v[2], v[4], v[6]);
    cx_dft4<S>(v[1], v[3], v[5], v[7]);
    v[3] = cx_w8<S, 1>(v[3]);
    v[5] = cx_w8<S, 2>(v[5]);
    v[7] = cx_w8<S, 3>(v[7]);
    C x[8];
#pragma unroll
    for (int k2 = 0; k2 < 4; ++k2) {
        x[k2] = cx_add(v[2 * k2], v[2 * k2 + 1]);
        x[k2 + 4] = cx_sub(v[2 * k2], v[2 * k2 + 1]);
    }
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = x[i];
}

// ---- the negacyclic twist, split in two ------------------------------------------
// The twist factor of input m = t + T j is w^m = w^t * W_32^j (w = exp(2 pi i
// / 4M), 4M = 32 T).  W_32^j is a compile-time constant per register j, and
// w^t is common to the 8 values of thread t, so it commutes with stage A's
// 8-point DFT and is folded into that stage's twiddle table.  The kernels
// therefore multiply their inputs by W_32^j (cx_w32) and no twist table is
// read at all.
__host__ __device__ constexpr double w32_cos(int j)
{
    return j == 0 ? 1.0 : j == 1 ? 0.98078528040323044913 : j == 2 ? 0.92387953251128675613
         : j == 3 ? 0.83146961230254523708 : j == 4 ? 0.70710678118654752440 : j == 5 ? 0.55557023301960222474
         : j == 6 ? 0.38268343236508977173 : j == 7 ? 0.19509032201612826785 : 0.0;
}
__host__ __device__ constexpr double w32_sin(int j) { return w32_cos(8 - j); }

// a * W_32^j (S = +1) or a * conj(W_32^j) (S = -1); j < 8 known after unrolling
template <int S, typename C>
__device__ __forceinline__ C cx_w32(C a, int j)
{
    using R = typename cx_real<C>::type;
    if (j == 0) return a;
    const R c = (R)w32_cos(j), s = (R)(S > 0 ? w32_sin(j) : -w32_sin(j));
    C r;
    r.x = a.x * c - a.y * s;
    r.y = a.x * s + a.y * c;
    return r;
}

// ---- tables ---------------------------------------------------------------------
// Each thread's twiddles are powers of one step, so the tables hold the
// steps and the transforms form the powers by repeated multiplication (FP64:
// seven products add a few ulp, far inside the transform's error; the
// shared-memory reads they replace were a fifth of the kernel's traffic):
//   twA0[t] = w^t, twAs[t] = W_M^t     stage A twiddle w^t W_M^{t k} = twA0 twAs^k, k < 8
//   twB1[a] = W_T^a                    stage B twiddle W_T^{a q1} = twB1^q1, q1 < 8
// (stage C's twiddles W_16^r, r < 8, are compile-time constants)
template <typename C, int T>
struct Fft8xTables {
    static_assert(T == 128, "the transform is written for 128 threads (M = 1024)");
    static constexpr int M = 8 * T, L = T / 8;
    C twA0[T];
    C twAs[T];
    C twB1[L];
};

// host: the FP64 tables, computed in long double
template <int T>
inline void build_fft8x_tables(Fft8xTables<double2, T> &tab)
{
    constexpr int M = 8 * T, L = T / 8;
    const long double PI = 3.141592653589793238462643383279502884L;
    auto cis = [&](long long num, long long den) {
        const long double a = 2.0L * PI * (long double)num / (long double)den;
        return make_double2((double)cosl(a), (double)sinl(a));
    };
    for (int t = 0; t < T; ++t) {
        tab.twA0[t] = cis(t, 4 * M);
        tab.twAs[t] = cis(t, M);
    }
    for (int a = 0; a < L; ++a) tab.twB1[a] = cis(a, T);
}

// v[0..7] *= base * step^k (S = +1) or conj(base * step^k) (S = -1)
template <int S, typename C>
__device__ __forceinline__ void fft8x_twiddle_powers(C v[8], C base, C step)
{
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        if (k > 0) base = cx_mul(base, step);
        v[k] = S > 0 ? cx_mul(v[k], base) : cx_mulc(v[k], base);
    }
}

// v[1..7] *= step^k (S = +1) or conj(step^k) (S = -1); v[0] unchanged
template <int S, typename C>
__device__ __forceinline__ void fft8x_step_powers(C v[8], C step)
{
    C p = step;
#pragma unroll
    for (int k = 1; k < 8; ++k) {
        if (k > 1) p = cx_mul(p, step);
        v[k] = S > 0 ? cx_mul(v[k], p) : cx_mulc(v[k], p);
    }
}

// frequency held in register slot s of thread u after the forward transform:
// u = q1 + 8 a0 + 16 k, s = rl + 4 e, q2 = rl + 4 a0 + 8 e
template <int T>
__host__ __device__ __forceinline__ int fft8x_freq(int u, int s)
{
    static_assert(T == 128, "the transform is written for 128 threads (M = 1024)");
    const int q1 = u & 7, a0 = (u >> 3) & 1, k = u >> 4;
    const int q2 = (s & 3) + 4 * a0 + 8 * (s >> 2);
    return k + 8 * (q1 + 8 * q2);
}

// synchronises the T threads of one polynomial (named barrier `id`)
template <int T>
__device__ __forceinline__ void group_sync(int id)
{
    if constexpr (T == 32) __syncwarp();
    else asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(T) : "memory");
}

// transpose scratch: row t (the thread of stage A) holds its 8 values in a
// row padded to 9 entries (FFT8X_XP<T> entries in all), which keeps both the
// row-wise write and the column-wise read free of bank conflicts for 8- and
// 16-byte elements, with every address a per-thread base plus a compile-time
// offset
template <int T>
constexpr int FFT8X_XP = 9 * T;
template <typename C>
__device__ __forceinline__ int fft8x_xp(int t, int k)
{
    return t * 9 + k;
}

// Scratch discipline: both transforms end by reading only rows of xp that
// belong to the reading thread's own warp, and each starts by writing only
// such rows, so a __syncwarp() orders one transform after the previous one;
// the writes into other warps' rows (and the reads after them) are fenced by
// the group's named barrier.

// forward: v[j] = z_{t + T j} / w^t in (the inputs multiplied by W_32^j only),
// v[s] = V(fft8x_freq<T>(t, s)) out.  xp: FFT8X_XP<T>-entry scratch shared
// by the group; bar: its named barrier.
template <typename C, int T>
__device__ __forceinline__ void fft8x_fwd(C v[8], C *xp, const Fft8xTables<C, T> &tab, int t, int bar)
{
    constexpr int L = T / 8;
    cx_dft8<1>(v);
    fft8x_twiddle_powers<1>(v, tab.twA0[t], tab.twAs[t]);
    __syncwarp();
#pragma unroll
    for (int k = 0; k < 8; ++k) xp[fft8x_xp<C>(t, k)] = v[k];
    group_sync<T>(bar);
    const int a = t % L, k = t / L;
#pragma unroll
    for (int b = 0; b < 8; ++b) v[b] = xp[fft8x_xp<C>(a + L * b, k)];
    cx_dft8<1>(v);
    fft8x_step_powers<1>(v, tab.twB1[a]);
    // C: the second transpose stays inside the warp (rows t of this warp),
    // but other warps may still be reading these rows from the first one
    group_sync<T>(bar);
#pragma unroll
    for (int q1 = 0; q1 < 8; ++q1) xp[fft8x_xp<C>(t, q1)] = v[q1];
    __syncwarp();
    const int q1p = t & 7, a0 = (t >> 3) & 1, kp = t >> 4;
#pragma unroll
    for (int j = 0; j < 8; ++j) v[j] = xp[fft8x_xp<C>(a0 + 2 * j + L * kp, q1p)];
    cx_dft8<1>(v);
#pragma unroll
    for (int rl = 0; rl < 4; ++rl) {
        const C send = a0 ? v[rl] : v[rl + 4];
        const C recv = cx_shfl_xor(send, 8);
        const C p = a0 ? recv : v[rl];
        C q = cx_w32<1>(a0 ? v[rl + 4] : recv, 2 * rl);   // W_16^rl
        if (a0) q = cx_mul_i<1>(q);                        // W_16^4 = i
        v[rl] = cx_add(p, q);
        v[rl + 4] = cx_sub(p, q);
    }
}

// inverse: v[s] = V(fft8x_freq<T>(t, s)) in, v[j] = M z_{t + T j} / w^t out
// (callers multiply by conj(W_32^j) to finish the untwist)
template <typename C, int T>
__device__ __forceinline__ void fft8x_inv(C v[8], C *xp, const Fft8xTables<C, T> &tab, int t, int bar)
{
    constexpr int L = T / 8;
    const int a = t % L, k = t / L;
    const int q1p = t & 7, a0 = (t >> 3) & 1, kp = t >> 4;
    // C inverse: the radix-2 step (2 Y0[r], 2 W_16^r Y1[r] from X[r] +- X[r + 8]),
    // the pair's trade back, the 8-point inverse DFT over r, the transpose
    // back inside the warp
#pragma unroll
    for (int rl = 0; rl < 4; ++rl) {
        const C p = cx_add(v[rl], v[rl + 4]);
        C q = cx_w32<-1>(cx_sub(v[rl], v[rl + 4]), 2 * rl);   // conj(W_16^rl)
        if (a0) q = cx_mul_i<-1>(q);                           // conj(W_16^4) = -i
        const C recv = cx_shfl_xor(a0 ? p : q, 8);
        v[rl] = a0 ? recv : p;
        v[rl + 4] = a0 ? q : recv;
    }
    cx_dft8<-1>(v);
    __syncwarp();
#pragma unroll
    for (int j = 0; j < 8; ++j) xp[fft8x_xp<C>(a0 + 2 * j + L * kp, q1p)] = v[j];
    __syncwarp();
#pragma unroll
    for (int q1 = 0; q1 < 8; ++q1) v[q1] = xp[fft8x_xp<C>(t, q1)];
    fft8x_step_powers<-1>(v, tab.twB1[a]);
    cx_dft8<-1>(v);
    group_sync<T>(bar);
#pragma unroll
    for (int b = 0; b < 8; ++b) xp[fft8x_xp<C>(a + L * b, k)] = v[b];
    group_sync<T>(bar);
#pragma unroll
    for (int kk = 0; kk < 8; ++kk) v[kk] = xp[fft8x_xp<C>(t, kk)];
    fft8x_twiddle_powers<-1>(v, tab.twA0[t], tab.twAs[t]);
    cx_dft8<-1>(v);
}

}  // namespace cfdb
