// Batched lvl1 external products TRGSW (x) TRLWE, FP64 and split-precision
// FP32 paths, plus the conversion of integer TRGSWs into the engine's
// frequency-domain layout.
//
// Restates trgswfftExternalProduct<lvl1param> (thirdparty/TFHEpp/src/
// trgsw.cpp:77-103): res_o = sum_{k,d} IFFT(dec_d(trlwe_k)) * trgsw[k l + d][o],
// transformed back per output polynomial.  One warp per product; the TRGSW
// rows (one per TRGSW or one shared by the batch) are read straight from HBM
// in the per-lane chunk layout the PBS kernels use, so every load is a
// coalesced 16-byte access and each TRGSW byte is read once.  A warp's loads
// of TRGSW row r come after the transform of digit polynomial r, so lane 0
// asks L2 for the rows two ahead (a bulk prefetch) and the loads find them
// there instead of waiting on HBM.

#include "extprod.cuh"
#include "fft_f32.cuh"

namespace cfdb {

namespace {

// 16 KB per TRGSW row (1,024 complex FP64, or 1,024 (hi, lo) FP32 pairs)
constexpr uint32_t TRGSW_ROW_BYTES = 16384;

// rows r and r + 1 of this warp's own TRGSW into L2 (nothing to do when the
// batch shares one TRGSW: it stays in L2 anyway)
__device__ __forceinline__ void prefetch_rows(const void *g, int r, int n, const ExtProdArgs &a, int lane)
{
    if (a.shared || lane != 0) return;
    for (int k = r; k < r + n && k < 2 * L1; ++k)
        bulk_prefetch_l2(reinterpret_cast<const unsigned char *>(g) + (size_t)k * TRGSW_ROW_BYTES, TRGSW_ROW_BYTES);
}

__device__ __forceinline__ void digits_f64(double2 v[16], const uint32_t *poly, int d, int lane, const Fft512Tables &T)
{
    const int sh = 32 - BGBIT1 * (d + 1);
#pragma unroll
    for (int m2 = 0; m2 < 16; ++m2) {
        const int m = lane + 32 * m2;
        int d0 = (int)(((poly[m] + DEC1_OFFSET + DEC1_ROUND) >> sh) & 63u) - 32;
        int d1 = (int)(((poly[m + 512] + DEC1_OFFSET + DEC1_ROUND) >> sh) & 63u) - 32;
        v[m2] = cmul(make_double2((double)d0, (double)d1), T.twist[m2 * 32 + lane]);
    }
}

__device__ __forceinline__ void digits_f32(float2 v[16], const uint32_t *poly, int d, int lane,
                                           const Fft512TablesPlain &T)
{
    const int sh = 32 - BGBIT1 * (d + 1);
#pragma unroll
    for (int m2 = 0; m2 < 16; ++m2) {
        const int m = lane + 32 * m2;
        int d0 = (int)(((poly[m] + DEC1_OFFSET + DEC1_ROUND) >> sh) & 63u) - 32;
        int d1 = (int)(((poly[m + 512] + DEC1_OFFSET + DEC1_ROUND) >> sh) & 63u) - 32;
        v[m2] = fcmul(make_float2((float)d0, (float)d1), T.twist[m2 * 32 + lane]);
    }
}

__global__ void __launch_bounds__(128) extprod1_f64_kernel(ExtProdArgs a)
{
    __shared__ double2 xp_s[4][FFT512_XP];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int p = blockIdx.x * 4 + w;
    if (p >= a.B) return;
    const Fft512Tables &T = *reinterpret_cast<const Fft512Tables *>(a.tables);
    const uint32_t *in = a.trlwe + (size_t)p * 2 * N1;
    const double2 *g = reinterpret_cast<const double2 *>(a.trgsw) + (a.shared ? 0 : (size_t)p * 6 * 1024);
    double2 f0[16], f1[16];
    prefetch_rows(g, 0, 2, a, lane);
#pragma unroll 1
    for (int r = 0; r < 2 * L1; ++r) {
        double2 v[16];
        prefetch_rows(g, r + 2, 1, a, lane);
        digits_f64(v, in + (r / L1) * N1, r % L1, lane, T);
        fft512_fwd(v, xp_s[w], T, lane);
        const double2 *gc = g + (size_t)r * 1024;
        if (r == 0) {
#pragma unroll
            for (int s = 0; s < 16; ++s) {
                f0[s] = cmul(v[s], gc[(2 * s) * 32 + lane]);
                f1[s] = cmul(v[s], gc[(2 * s + 1) * 32 + lane]);
            }
        } else {
#pragma unroll
            for (int s = 0; s < 16; ++s) {
                cfma(f0[s], v[s], gc[(2 * s) * 32 + lane]);
                cfma(f1[s], v[s], gc[(2 * s + 1) * 32 + lane]);
            }
        }
    }
    uint32_t *o = a.out + (size_t)p * 2 * N1;
    fft512_inv(f0, xp_s[w], T, lane);
#pragma unroll
    for (int m2 = 0; m2 < 16; ++m2) {
        const int m = lane + 32 * m2;
        const double2 y = cmulc(f0[m2], T.twist[m2 * 32 + lane]);
        o[m] = f64_to_torus32(y.x * (1.0 / 512.0));
        o[m + 512] = f64_to_torus32(y.y * (1.0 / 512.0));
    }
    fft512_inv(f1, xp_s[w], T, lane);
#pragma unroll
    for (int m2 = 0; m2 < 16; ++m2) {
        const int m = lane + 32 * m2;
        const double2 y = cmulc(f1[m2], T.twist[m2 * 32 + lane]);
        o[N1 + m] = f64_to_torus32(y.x * (1.0 / 512.0));
        o[N1 + m + 512] = f64_to_torus32(y.y * (1.0 / 512.0));
    }
}

// o = the torus32 polynomial of the paired (hi, lo) frequency accumulator f:
// round(hi) * 2^24 + round(lo) (mod 2^32)
__device__ __forceinline__ void store_split(uint32_t *o, CP f[16], unsigned long long *xp, int lane,
                                            const Fft512TablesPlain &T)
{
    pfft512_inv<false>(f, xp, T, lane);
#pragma unroll
    for (int m2 = 0; m2 < 16; ++m2) {
        const int m = lane + 32 * m2;
        const CP y = pmul_t(f[m2], T.untwistp[m2 * 32 + lane]);
        const float2 re = unpk2(y.re), im = unpk2(y.im);
        o[m] = ((uint32_t)__float2int_rn(re.x) << 24) + (uint32_t)__float2ll_rn(re.y);
        o[m + 512] = ((uint32_t)__float2int_rn(im.x) << 24) + (uint32_t)__float2ll_rn(im.y);
    }
}

// both limbs of one output: f (+)= v * k, k = (hi.re, lo.re, hi.im, lo.im)
__device__ __forceinline__ void pmac_limbs(CP &f, float2 v, float4 k, bool first)
{
    const unsigned long long vr = pk2(v.x, v.x), vi = pk2(v.y, v.y), nvi = pk2(-v.y, -v.y);
    const unsigned long long kr = pk2(k.x, k.y), ki = pk2(k.z, k.w);
    if (first) {
        f.re = f2(nvi, ki, m2(vr, kr));
        f.im = f2(vi, kr, m2(vr, ki));
    } else {
        f.re = f2(nvi, ki, f2(vr, kr, f.re));
        f.im = f2(vi, kr, f2(vr, ki, f.im));
    }
}

__global__ void __launch_bounds__(128) extprod1_split_kernel(ExtProdArgs a)
{
    __shared__ unsigned long long xp_s[4][FFT512_XP];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int p = blockIdx.x * 4 + w;
    if (p >= a.B) return;
    const Fft512TablesPlain &T = reinterpret_cast<const Fft512TablesF *>(a.tables)->plain;
    const uint32_t *in = a.trlwe + (size_t)p * 2 * N1;
    const float4 *g = reinterpret_cast<const float4 *>(a.trgsw) + (a.shared ? 0 : (size_t)p * 6 * 1024);
    CP f0[16], f1[16];
    prefetch_rows(g, 0, 2, a, lane);
#pragma unroll 1
    for (int r = 0; r < 2 * L1; ++r) {
        float2 v[16];
        prefetch_rows(g, r + 2, 1, a, lane);
        digits_f32(v, in + (r / L1) * N1, r % L1, lane, T);
        ffft512_fwd(v, reinterpret_cast<float2 *>(xp_s[w]), T, lane);
        const float4 *gc = g + (size_t)r * 1024;
#pragma unroll
        for (int s = 0; s < 16; ++s) {
            pmac_limbs(f0[s], v[s], gc[(2 * s) * 32 + lane], r == 0);
            pmac_limbs(f1[s], v[s], gc[(2 * s + 1) * 32 + lane], r == 0);
        }
    }
    uint32_t *o = a.out + (size_t)p * 2 * N1;
    store_split(o, f0, xp_s[w], lane, T);
    store_split(o + N1, f1, xp_s[w], lane, T);
}

}  // namespace

cudaError_t launch_extprod1(const ExtProdArgs &a, int precision, cudaStream_t st)
{
    if (a.B <= 0) return cudaSuccess;
    if (precision == 0) extprod1_f64_kernel<<<(a.B + 3) / 4, 128, 0, st>>>(a);
    else extprod1_split_kernel<<<(a.B + 3) / 4, 128, 0, st>>>(a);
    return cudaGetLastError();
}

}  // namespace cfdb
