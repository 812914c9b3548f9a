// Batched lvl0 -> lvl1 programmable bootstrapping, FP64 path.
//
// Restates GateBootstrappingTLWE2TLWEFFT<lvl01param>
// (thirdparty/TFHEpp/src/gatebootstrapping.cpp:14-23): BlindRotate
// (include/gatebootstrapping.hpp:15-43) = 672 x CMUXFFTwithPolynomialMulByXaiMinusOne
// (src/detwfa.cpp:20-35) followed by SampleExtractIndex(0) (src/trlwe.cpp:108-118).
//
// B200 layout: one CTA per group of W ciphertexts (one warp each) plus one
// producer warp.  Every accumulator TRLWE lives in shared memory for the whole
// blind rotation; the FFT-domain bootstrapping key streams through a ring of
// S 16 KB slots filled by bulk (TMA-engine) copies and shared by the W warps,
// so each key byte crosses L2->SM once per CTA instead of once per ciphertext.
// Per CMux each warp runs 6 forward transforms (decomposition fused into the
// load), a register-resident frequency-domain multiply-accumulate against the
// key chunk, and 2 inverse transforms whose output is added into the
// accumulator.  No grid-wide barrier: CTAs are independent.
#include "pbs_common.cuh"
#include "ring.cuh"

namespace cfdb {

template <int W, int S>
struct Pbs01Smem {
    static constexpr int RING_OFF = RING_HEADER_BYTES;
    static constexpr int CHUNK_BYTES = 16384;  // one TRGSW row: 2 outputs x 512 complex x 16 B
    static constexpr int TAB_OFF = RING_OFF + S * CHUNK_BYTES;
    static constexpr int WARP_OFF = TAB_OFF + ((int)sizeof(Fft512Tables) + 127) / 128 * 128;
    static constexpr int XP_BYTES = FFT512_XP * 16;
    static constexpr int ACC_BYTES = 2 * N1 * 4;
    static constexpr int ABAR_BYTES = ((N0 * 2) + 127) / 128 * 128;
    static constexpr int PER_WARP = XP_BYTES + ACC_BYTES + ABAR_BYTES;
    static constexpr int TOTAL = WARP_OFF + W * PER_WARP;
};

// digit d of (X^a - 1) * poly at coefficients m and m+512, twisted:
// v[m2] = (dig_d(m) + i dig_d(m+512)) * w^m,  m = lane + 32 m2.  The signed
// digit is the sign-extended field d of (t + offset + round) ^ DEC1_XOR.
__device__ __forceinline__ void load_digit_poly1(double2 v[16], const uint32_t *poly, uint32_t abar, int d, int lane,
                                        const Fft512Tables &T)
{
#pragma unroll
    for (int m2 = 0; m2 < 16; ++m2) {
        const int m = lane + 32 * m2;
        const uint32_t x0 = ((rot_coef<N1>(poly, m, abar) - poly[m]) + DEC1_OFFSET + DEC1_ROUND) ^ DEC1_XOR;
        const uint32_t x1 = ((rot_coef<N1>(poly, m + 512, abar) - poly[m + 512]) + DEC1_OFFSET + DEC1_ROUND) ^ DEC1_XOR;
        const int d0 = digit_field1(x0, d), d1 = digit_field1(x1, d);
        v[m2] = cmul(make_double2((double)d0, (double)d1), T.twist[m2 * 32 + lane]);
    }
}

// poly[m] += a_m, poly[m+512] += a_{m+512} from v[m2] = 512 z_m
__device__ __forceinline__ void add_inverse_poly1(uint32_t *poly, const double2 v[16], int lane,
                                                  const Fft512Tables &T)
{
#pragma unroll
    for (int m2 = 0; m2 < 16; ++m2) {
        const int m = lane + 32 * m2;
        double2 y = cmulc(v[m2], T.twist[m2 * 32 + lane]);
        poly[m] += f64_to_torus32(y.x * (1.0 / 512.0));
        poly[m + 512] += f64_to_torus32(y.y * (1.0 / 512.0));
    }
}

template <int W, int S>
__global__ void __launch_bounds__(W * 32, 1) pbs01_f64_kernel(Pbs01Args a)
{
    using L = Pbs01Smem<W, S>;
    extern __shared__ __align__(128) unsigned char smem[];
    Fft512Tables *T = reinterpret_cast<Fft512Tables *>(smem + L::TAB_OFF);
    const int ngroups = (a.B + W - 1) / W;
    constexpr int CHUNKS = N0 * 2 * L1;
    // key ring without a producer warp (ring.cuh)
    KeyRing<S, L::CHUNK_BYTES, W> ring{reinterpret_cast<RingHeader *>(smem), smem + L::RING_OFF,
                                    reinterpret_cast<const unsigned char *>(a.bk), (uint32_t)CHUNKS,
                                    (uint32_t)groups_of_block(ngroups, blockIdx.x, gridDim.x) * CHUNKS};

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) ring.init_by_thread0();
    {
        const float4 *src = reinterpret_cast<const float4 *>(a.tables);
        float4 *dst = reinterpret_cast<float4 *>(T);
        for (int i = threadIdx.x; i < (int)(sizeof(Fft512Tables) / 16); i += blockDim.x) dst[i] = src[i];
    }
    __syncthreads();
    if (threadIdx.x == 0) ring.prologue_by_thread0();

    unsigned char *wb = smem + L::WARP_OFF + warp * L::PER_WARP;
    double2 *xp = reinterpret_cast<double2 *>(wb);
    uint32_t *acc = reinterpret_cast<uint32_t *>(wb + L::XP_BYTES);
    uint16_t *abar_s = reinterpret_cast<uint16_t *>(wb + L::XP_BYTES + L::ACC_BYTES);

    uint32_t c = 0;
    for (int g = blockIdx.x; g < ngroups; g += gridDim.x) {
        const int ct = g * W + warp;
        const bool valid = ct < a.B;
        uint32_t bbar = 2 * N1;
        if (valid) {
            const uint32_t *in = a.in + (size_t)ct * (N0 + 1);
            for (int i = lane; i < N0; i += 32) abar_s[i] = (uint16_t)((in[i] + (1u << 20)) >> 21);
            bbar = 2 * N1 - (in[N0] >> 21);
        }
        for (int j = lane; j < N1; j += 32) {
            acc[j] = 0;
            acc[N1 + j] = testvec_rot1(a.tv, j, bbar);
        }
        __syncwarp();

        for (int i = 0; i < N0; ++i) {
            const uint32_t ab = valid ? abar_s[i] : 0u;
            const bool active = ab != 0;
            double2 f0[16], f1[16];
#pragma unroll 1
            for (int r = 0; r < 2 * L1; ++r, ++c) {
                double2 v[16];
                if (active) {
                    load_digit_poly1(v, acc + (r / L1) * N1, ab, r % L1, lane, *T);
                    fft512_fwd(v, xp, *T, lane);
                }
                const double2 *bkc = reinterpret_cast<const double2 *>(ring.acquire(c, a.err));
                if (active) {
                    if (r == 0) {
#pragma unroll
                        for (int s = 0; s < 16; ++s) {
                            f0[s] = cmul(v[s], bkc[(2 * s) * 32 + lane]);
                            f1[s] = cmul(v[s], bkc[(2 * s + 1) * 32 + lane]);
                        }
                    } else {
#pragma unroll
                        for (int s = 0; s < 16; ++s) {
                            cfma(f0[s], v[s], bkc[(2 * s) * 32 + lane]);
                            cfma(f1[s], v[s], bkc[(2 * s + 1) * 32 + lane]);
                        }
                    }
                }
                ring.release(c, lane);
            }
            if (active) {
                fft512_inv(f0, xp, *T, lane);
                add_inverse_poly1(acc, f0, lane, *T);
                fft512_inv(f1, xp, *T, lane);
                add_inverse_poly1(acc + N1, f1, lane, *T);
                __syncwarp();
            }
        }
        if (valid) {
            uint32_t *o = a.out + (size_t)ct * (N1 + 1);
            for (int j = lane; j < N1; j += 32) o[j] = j == 0 ? acc[0] : (uint32_t)(0u - acc[N1 - j]);
            if (lane == 0) o[N1] = acc[N1] + a.out_b_add;
        }
        __syncwarp();
    }
    __syncthreads();
    if (threadIdx.x == 0) ring.drain_by_thread0(a.err);
}

template <int W, int S>
static cudaError_t launch_pbs01_f64_t(const Pbs01Args &a, int grid, cudaStream_t st)
{
    using L = Pbs01Smem<W, S>;
    pbs01_f64_kernel<W, S><<<grid, W * 32, L::TOTAL, st>>>(a);
    return cudaGetLastError();
}

// Persistent grid: min(groups, SMs) CTAs of W warps (one ciphertext each, no
// producer warp), each looping over groups of W ciphertexts.  At most 8 warps
// keep 2 warps per SM sub-partition, so every thread may hold 255 registers
// (the 16 complex FFT values plus two 16-complex frequency accumulators per
// lane).  W = 7, 8 or 4 is chosen per launch (pbs01_choose_w); W = 4 puts one
// warp on each sub-partition, the shortest pass, with a deeper key ring in
// the shared memory the fewer warps leave.
template <int W>
constexpr int PBS01_S = W == 4 ? 6 : 4;

cudaError_t launch_pbs01_f64(const Pbs01Args &a, int num_sms, int w, cudaStream_t st)
{
    if (a.B <= 0) return cudaSuccess;
    static_assert(Pbs01Smem<8, PBS01_S<8>>::TOTAL <= 227 * 1024, "shared memory budget");
    static_assert(Pbs01Smem<4, PBS01_S<4>>::TOTAL <= 227 * 1024, "shared memory budget");
    const int groups = (a.B + w - 1) / w;
    const int grid = groups < num_sms ? groups : num_sms;
    if (w == 7) return launch_pbs01_f64_t<7, PBS01_S<7>>(a, grid, st);
    if (w == 8) return launch_pbs01_f64_t<8, PBS01_S<8>>(a, grid, st);
    if (w == 4) return launch_pbs01_f64_t<4, PBS01_S<4>>(a, grid, st);
    return cudaErrorInvalidValue;
}

// the dynamic shared-memory opt-in, set once per device when a context is
// created (so no attribute call happens inside a stream capture)
template <int W>
static cudaError_t init_pbs01_f64_t()
{
    return cudaFuncSetAttribute(pbs01_f64_kernel<W, PBS01_S<W>>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                Pbs01Smem<W, PBS01_S<W>>::TOTAL);
}

cudaError_t init_pbs01_f64()
{
    cudaError_t e = init_pbs01_f64_t<7>();
    if (e == cudaSuccess) e = init_pbs01_f64_t<8>();
    if (e == cudaSuccess) e = init_pbs01_f64_t<4>();
    return e;
}

}  // namespace cfdb
