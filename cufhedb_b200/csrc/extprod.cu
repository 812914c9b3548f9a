// Batched lvl1 external products TRGSW (x) TRLWE, FP64 and split-precision
// FP32 paths, plus the conversion of integer TRGSWs into the engine's
// frequency-domain layout.
//
// Restates trgswfftExternalProduct<lvl1param> (thirdparty/TFHEpp/src/
// trgsw.cpp:77-103): res_o = sum_{k,d} IFFT(dec_d(trlwe_k)) * trgsw[k l + d][o],
// transformed back per output polynomial.  One warp per product; the TRGSW
// rows (one per TRGSW or one shared by the batch) are stored in the per-lane
// chunk layout the PBS kernels use, and each TRGSW byte is read once.  The
// FP64 kernel reads them straight from global memory.  In the split kernel
// every warp copies its product's TRGSW row by row into its own 16 KB of
// shared memory (a bulk copy completing on the warp's mbarrier), the copy of
// row r + 1 issued as soon as the products of row r are read out, so it runs
// under the transform of digit polynomial r + 1; lane 0 also asks L2 for the
// rows two ahead (a bulk prefetch), so each copy finds its row there.  Waits
// are bounded: a warp that gives up records DEV_TIMEOUT_ROW, issues no
// further copy and, before it exits, waits (bounded again) for the one it
// gave up on.

#include "extprod.cuh"
#include "fft_f32.cuh"

namespace cfdb {

namespace {

// 16 KB per TRGSW row (1,024 complex FP64, or 1,024 (hi, lo) FP32 pairs)
constexpr uint32_t TRGSW_ROW_BYTES = 16384;
constexpr int EP_WARPS = 4;   // products (warps) per CTA

// dynamic shared memory of a CTA: per warp a staged TRGSW row and its
// transpose scratch (XPB bytes), then one mbarrier per warp
template <int XPB>
constexpr int ep_smem_bytes()
{
    return EP_WARPS * (int)TRGSW_ROW_BYTES + EP_WARPS * XPB + EP_WARPS * 8;
}

// one warp's TRGSW row staged in shared memory (see the file comment)
struct RowStage {
    unsigned char *buf;   // TRGSW_ROW_BYTES, 128-byte aligned
    uint64_t *bar;
    uint32_t phase;
    bool ok;              // warp-uniform: no wait has given up

    __device__ __forceinline__ void init(int lane)
    {
        if (lane == 0) {
            mbar_init(bar, 1);
            fence_barrier_init();
        }
        __syncwarp();
    }
    // after every lane's last read of the buffer (callers __syncwarp first)
    __device__ __forceinline__ void issue(const unsigned char *row, int lane)
    {
        if (lane == 0 && ok) {
            fence_proxy_async_smem();
            mbar_arrive_expect_tx(bar, TRGSW_ROW_BYTES);
            bulk_g2s(buf, row, TRGSW_ROW_BYTES, bar);
        }
    }
    __device__ __forceinline__ void wait(int *err, int lane)
    {
        if (!ok) return;
        const bool done = __all_sync(0xffffffffu, mbar_wait(bar, phase));
        if (done) {
            phase ^= 1;
        } else {
            ok = false;
            if (lane == 0) report_error(err, DEV_TIMEOUT_ROW);
        }
    }
    // a copy given up on may still be in flight: wait for it (bounded)
    __device__ __forceinline__ void drain(int *err, int lane)
    {
        if (ok) return;
        const bool done = __all_sync(0xffffffffu, mbar_wait(bar, phase));
        if (!done && lane == 0) report_error(err, DEV_TIMEOUT_DRAIN);
    }
};

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

// The FP64 kernel reads its TRGSW rows straight from global memory: staged
// through shared memory like the split kernel it measured slower (4,096
// products 0.145 -> 0.190 ms).
__global__ void __launch_bounds__(EP_WARPS * 32) extprod1_f64_kernel(ExtProdArgs a)
{
    __shared__ double2 xp_s[EP_WARPS][FFT512_XP];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int p = blockIdx.x * EP_WARPS + w;
    if (p >= a.B) return;
    double2 *xp = xp_s[w];
    const Fft512Tables &T = *reinterpret_cast<const Fft512Tables *>(a.tables);
    const uint32_t *in = a.trlwe + (size_t)p * 2 * N1;
    if (lane == 0) bulk_prefetch_l2_if_aligned(in, 2 * N1 * sizeof(uint32_t));   // the TRLWE, read per digit
    const double2 *g = reinterpret_cast<const double2 *>(a.trgsw) + (a.shared ? 0 : (size_t)p * 6 * 1024);
    double2 f0[16], f1[16];
#pragma unroll 1
    for (int r = 0; r < 2 * L1; ++r) {
        double2 v[16];
        digits_f64(v, in + (r / L1) * N1, r % L1, lane, T);
        fft512_fwd(v, xp, T, lane);
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
    fft512_inv(f0, xp, T, lane);
#pragma unroll
    for (int m2 = 0; m2 < 16; ++m2) {
        const int m = lane + 32 * m2;
        const double2 y = cmulc(f0[m2], T.twist[m2 * 32 + lane]);
        o[m] = f64_to_torus32(y.x * (1.0 / 512.0));
        o[m + 512] = f64_to_torus32(y.y * (1.0 / 512.0));
    }
    fft512_inv(f1, xp, T, lane);
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

constexpr int XPB_SPLIT = FFT512_XP * (int)sizeof(unsigned long long);

__global__ void __launch_bounds__(EP_WARPS * 32) extprod1_split_kernel(ExtProdArgs a)
{
    extern __shared__ __align__(128) unsigned char smem[];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int p = blockIdx.x * EP_WARPS + w;
    if (p >= a.B) return;
    unsigned long long *xp =
        reinterpret_cast<unsigned long long *>(smem + EP_WARPS * TRGSW_ROW_BYTES + w * XPB_SPLIT);
    RowStage rs{smem + w * TRGSW_ROW_BYTES,
                reinterpret_cast<uint64_t *>(smem + EP_WARPS * (TRGSW_ROW_BYTES + XPB_SPLIT)) + w, 0u, true};
    rs.init(lane);
    const Fft512TablesPlain &T = reinterpret_cast<const Fft512TablesF *>(a.tables)->plain;
    const uint32_t *in = a.trlwe + (size_t)p * 2 * N1;
    if (lane == 0) bulk_prefetch_l2_if_aligned(in, 2 * N1 * sizeof(uint32_t));   // the TRLWE, read per digit
    const unsigned char *g = reinterpret_cast<const unsigned char *>(a.trgsw) +
                             (a.shared ? 0 : (size_t)p * 2 * L1 * TRGSW_ROW_BYTES);
    prefetch_rows(g, 1, 2, a, lane);
    rs.issue(g, lane);
    CP f0[16], f1[16];
#pragma unroll 1
    for (int r = 0; r < 2 * L1; ++r) {
        float2 v[16];
        prefetch_rows(g, r + 3, 1, a, lane);
        digits_f32(v, in + (r / L1) * N1, r % L1, lane, T);
        ffft512_fwd(v, reinterpret_cast<float2 *>(xp), T, lane);
        rs.wait(a.err, lane);
        const float4 *gc = reinterpret_cast<const float4 *>(rs.buf);
#pragma unroll
        for (int s = 0; s < 16; ++s) {
            pmac_limbs(f0[s], v[s], gc[(2 * s) * 32 + lane], r == 0);
            pmac_limbs(f1[s], v[s], gc[(2 * s + 1) * 32 + lane], r == 0);
        }
        __syncwarp();
        if (r + 1 < 2 * L1) rs.issue(g + (size_t)(r + 1) * TRGSW_ROW_BYTES, lane);
    }
    rs.drain(a.err, lane);
    uint32_t *o = a.out + (size_t)p * 2 * N1;
    store_split(o, f0, xp, lane, T);
    store_split(o + N1, f1, xp, lane, T);
}

}  // namespace

cudaError_t launch_extprod1(const ExtProdArgs &a, int precision, cudaStream_t st)
{
    if (a.B <= 0) return cudaSuccess;
    const unsigned grid = (unsigned)((a.B + EP_WARPS - 1) / EP_WARPS);
    if (precision == 0)
        extprod1_f64_kernel<<<grid, EP_WARPS * 32, 0, st>>>(a);
    else
        extprod1_split_kernel<<<grid, EP_WARPS * 32, ep_smem_bytes<XPB_SPLIT>(), st>>>(a);
    return cudaGetLastError();
}

cudaError_t init_extprod1()
{
    return cudaFuncSetAttribute(extprod1_split_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                ep_smem_bytes<XPB_SPLIT>());
}

}  // namespace cfdb
