// ArcEDB comparisons on the batched path: cuARCEDB::greater_than_tfhepp,
// less_than_tfhepp and equality_tfhepp (src/cuHEDB/comparable_gpu.cuh:52-168;
// CPU twins src/ARCEDB/comparison/comparable.cpp:506-729) over B rows at once.
//
// Encodings (src/ARCEDB/comparison/comparable.h:169-305): a value is split
// into radix-1024 digits; digit x_d of the left operand is the TRLWE of
// mu X^{x_d} (exponent_encrypt), digit y_d of the right operand the TRGSW of
// X^{-y_d} (exponent_encrypt_rgsw, is_negative).  Per digit the external
// product gives a TRLWE of mu X^{x_d - y_d}; multiplied by the all-ones
// polynomial sum_i X^i its constant coefficient is +mu when x_d <= y_d and -mu
// otherwise (the reference's PolyMul_st, cufft_gpu.cuh:214-226, computes that
// product through an FFT; here it is the exact negacyclic prefix sum), and the
// constant coefficient of the product itself is mu exactly when x_d == y_d.
// Digits combine from the least significant up: for order comparisons
//     r_d = PBS_mu(IKS10(eq_d + 2 hi_d + r_{d-1} + mu/2)),
// for equality r_d = HomAND(r_{d-1}, eq'_d) with the ArcEDB HomAND
// (comparable_gpu.cuh:30-40: a + b - mu, key switch, bootstrap to +-mu).
//
// The reference's less_than_tfhepp (GPU and CPU alike) tests x_d <= y_d per
// digit, so over several digits the combination above returns the complement
// of the lower digits' result whenever the top digits are equal; it is kept
// as op 1 for parity, and op 3 is the consistent strict form (x_d < y_d per
// digit: the all-ones polynomial with its constant term -1), which combines
// exactly like greater_than.
#include "ctx.cuh"
#include "extprod.cuh"
#include "fftops.cuh"
#include "lvl2.cuh"

namespace cfdb {

namespace {

constexpr uint32_t MU = 1u << 29;

// out (B lvl1 TLWEs) from t (B TRLWEs [2][1024]) by SampleExtractIndex(0)
// (TFHEpp src/trlwe.cpp:108-118) of
//   mode 0: t                                   (the equal term)
//   mode 1: t * sum_i X^i                        (less_than: +mu iff x <= y)
//   mode 2: -(t * sum_i X^i)                     (greater_than: +mu iff x > y)
//   mode 3: 2 t, b - mu                          (equality, single digit)
//   mode 4: t * (sum_i X^i - 2)                  (strict less than: +mu iff x < y)
// One 256-thread block per row; the negacyclic product with the all-ones
// polynomial is c_k = 2 P_k - S (P_k = a_0 + ... + a_k, S = P_{N-1}), and
// mode 4 subtracts 2 a_k.
__global__ void __launch_bounds__(256) arc_extract_kernel(uint32_t *out, const uint32_t *t, int mode)
{
    __shared__ uint32_t pre[N1];
    __shared__ uint32_t wsum[8], bsum[8];
    const int row = blockIdx.x, tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const uint32_t *a = t + (size_t)row * 2 * N1, *b = a + N1;
    uint32_t *o = out + (size_t)row * (N1 + 1);
    if (mode == 0 || mode == 3) {
        const uint32_t mul = mode == 3 ? 2u : 1u;
        for (int i = tid; i < N1; i += 256) o[i] = mul * (i == 0 ? a[0] : 0u - a[N1 - i]);
        if (tid == 0) o[N1] = mul * b[0] - (mode == 3 ? MU : 0u);
        return;
    }
    // inclusive prefix sums of a (4 consecutive values per thread), sum of b
    uint32_t v[4], run = 0, bs = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        run += a[4 * tid + k];
        v[k] = run;
        bs += b[4 * tid + k];
    }
    uint32_t x = run;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, off);
        if (lane >= off) x += y;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) bs += __shfl_xor_sync(0xffffffffu, bs, off);
    if (lane == 31) wsum[w] = x;
    if (lane == 0) bsum[w] = bs;
    __syncthreads();
    uint32_t base = x - run;   // exclusive within the warp
    for (int j = 0; j < w; ++j) base += wsum[j];
#pragma unroll
    for (int k = 0; k < 4; ++k) pre[4 * tid + k] = base + v[k];
    __syncthreads();
    uint32_t total = 0, btotal = 0;
    for (int j = 0; j < 8; ++j) {
        total += wsum[j];
        btotal += bsum[j];
    }
    const uint32_t sgn = mode == 2 ? 0u - 1u : 1u;
    const uint32_t corr = mode == 4 ? 2u : 0u;
    for (int i = tid; i < N1; i += 256) {
        const int k = i == 0 ? 0 : N1 - i;
        const uint32_t ck = 2u * pre[k] - total - corr * a[k];
        o[i] = sgn * (i == 0 ? ck : 0u - ck);
    }
    if (tid == 0) o[N1] = sgn * (2u * b[0] - btotal - corr * b[0]);
}

// out = eq + 2 hi + lo, b + mu/2 (the digit combination of greater/less than)
__global__ void arc_combine_kernel(uint32_t *out, const uint32_t *eq, const uint32_t *hi, const uint32_t *lo,
                                   size_t total)
{
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        uint32_t v = eq[e] + 2u * hi[e] + lo[e];
        if (e % (N1 + 1) == N1) v += MU >> 1;
        out[e] = v;
    }
}

// x_i <- x_i * m (pointwise, TFHEpp's frequency-domain layout: re in
// [0, N/2), im in [N/2, N); MulInFD, utils.hpp:83-93); m shared or per row
__global__ void fd_mul_kernel(double *x, const double *m, int half, size_t rows, int shared)
{
    const size_t total = rows * (size_t)half;
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const size_t r = e / half, k = e % half;
        double *xr = x + r * 2 * half;
        const double *mr = m + (shared ? 0 : r * 2 * half);
        const double ar = xr[k], ai = xr[k + half], br = mr[k], bi = mr[k + half];
        xr[k] = fma(ar, br, -(ai * bi));
        xr[k + half] = fma(ai, br, ar * bi);
    }
}

cudaError_t launch_fd_mul(double *x, const double *m, int half, int rows, int shared, cudaStream_t st)
{
    const size_t total = (size_t)rows * half;
    const unsigned grid = (unsigned)std::min<size_t>((total + 255) / 256, 4096);
    fd_mul_kernel<<<grid, 256, 0, st>>>(x, m, half, (size_t)rows, shared);
    return cudaGetLastError();
}

struct Arc {
    cufhedb_ctx *c;
    cudaStream_t st;
    int prec, B;

    int alloc(uint32_t **p, size_t words)
    {
        cudaError_t e = cudaMallocAsync((void **)p, words * 4, st);
        return e == cudaSuccess ? CUFHEDB_OK : cuda_error(e, "ArcEDB scratch");
    }
    int extprod(uint32_t *t, const uint32_t *trlwe, const void *trgsw)
    {
        ExtProdArgs a{};
        a.trlwe = trlwe;
        a.trgsw = trgsw;
        a.out = t;
        a.B = B;
        a.shared = 0;
        a.tables = prec == CUFHEDB_FP64 ? (const void *)c->tab512 : (const void *)c->tab512f;
        a.err = c->err;
        cudaError_t e = launch_extprod1(a, prec == CUFHEDB_FP64 ? 0 : 1, st);
        return e == cudaSuccess ? CUFHEDB_OK : cuda_error(e, "ArcEDB external product");
    }
    int extract(uint32_t *out, const uint32_t *t, int mode)
    {
        arc_extract_kernel<<<B, 256, 0, st>>>(out, t, mode);
        cudaError_t e = cudaGetLastError();
        return e == cudaSuccess ? CUFHEDB_OK : cuda_error(e, "ArcEDB sample extract");
    }
    // IKS10 of sa*a + sb*b + offset, then PBS01 to +-mu
    int bootstrap(uint32_t *out, const uint32_t *a, const uint32_t *b, int sb, uint32_t offset)
    {
        uint32_t *l0 = nullptr;
        int rc = alloc(&l0, (size_t)B * (N0 + 1));
        if (!rc) rc = iks_run(c, 10, a, b, 1, sb, offset, l0, B, st);
        if (!rc) rc = pbs01_run(c, l0, out, B, TestVec{0, 0, MU, nullptr}, 0u, prec, st);
        if (l0) cudaFreeAsync(l0, st);
        return rc;
    }
};

}  // namespace

}  // namespace cfdb

using namespace cfdb;

int cufhedb_arc_compare(cufhedb_ctx *ctx, int op, const uint32_t *trlwe, const void *trgsw, uint32_t *out, int B,
                        int D, int precision, cufhedb_stream_t stream)
{
    if (!aligned_to(trlwe, 4)) return cfdb::set_error(CUFHEDB_ERR_ARG, "trlwe must be 4-byte aligned");
    if (!aligned_to(trgsw, 16)) return cfdb::set_error(CUFHEDB_ERR_ARG, "trgsw must be 16-byte aligned");
    if (!aligned_to(out, 4)) return cfdb::set_error(CUFHEDB_ERR_ARG, "out must be 4-byte aligned");
    if (!ctx) return set_error(CUFHEDB_ERR_ARG, "ctx is null");
    if (op < 0 || op > 3) return set_error(CUFHEDB_ERR_ARG, "unknown ArcEDB comparison");
    if (B < 0 || D < 1) return set_error(CUFHEDB_ERR_ARG, "bad batch or digit count");
    if (B == 0) return CUFHEDB_OK;
    if (!trlwe || !trgsw || !out) return set_error(CUFHEDB_ERR_ARG, "null buffer");
    if (precision != CUFHEDB_FP64 && precision != CUFHEDB_SPLIT32 &&
        precision != CUFHEDB_SPLIT32_TC) return set_error(CUFHEDB_ERR_ARG, "unsupported precision");
    if (D > 1 && !ctx->ksk[0]) return set_error(CUFHEDB_ERR_NOKEY, "lvl10 key-switching key not loaded");
    if (D > 1 && !ctx->bk01) return set_error(CUFHEDB_ERR_NOKEY, "lvl01 bootstrapping key not loaded");
    DeviceGuard guard(ctx->device);
    Arc A{ctx, (cudaStream_t)stream, precision, B};
    const size_t trl = (size_t)B * 2 * N1, tlw = (size_t)B * (N1 + 1);
    const size_t gbytes = (size_t)B * 98304;   // prepared lvl1 TRGSW per row
    const unsigned char *g = static_cast<const unsigned char *>(trgsw);
    uint32_t *t = nullptr, *eq = nullptr, *hi = nullptr, *sum = nullptr;
    int rc = A.alloc(&t, trl);
    if (!rc) rc = A.alloc(&eq, tlw);
    if (!rc) rc = A.alloc(&hi, tlw);
    if (!rc) rc = A.alloc(&sum, tlw);
    const int single = op == 0 ? 2 : op == 1 ? 1 : op == 2 ? 3 : 4;
    // digit 0: the result so far goes straight to `out`
    if (!rc) rc = A.extprod(t, trlwe, g);
    if (!rc) rc = A.extract(out, t, single);
    for (int d = 1; d < D && !rc; ++d) {
        rc = A.extprod(t, trlwe + (size_t)d * trl, g + (size_t)d * gbytes);
        if (!rc) rc = A.extract(hi, t, single);
        if (op == 2) {
            // equality: r = HomAND(r, eq_d)  (a + b - mu, bootstrap)
            if (!rc) rc = A.bootstrap(out, out, hi, 1, 0u - MU);
        } else {
            if (!rc) rc = A.extract(eq, t, 0);
            if (!rc) {
                const unsigned grid = (unsigned)std::min<size_t>((tlw + 255) / 256, 4096);
                arc_combine_kernel<<<grid, 256, 0, A.st>>>(sum, eq, hi, out, tlw);
                cudaError_t e = cudaGetLastError();
                if (e != cudaSuccess) rc = cuda_error(e, "ArcEDB combine");
            }
            if (!rc) rc = A.bootstrap(out, sum, nullptr, 0, 0u);
        }
    }
    for (uint32_t *p : {t, eq, hi, sum})
        if (p) cudaFreeAsync(p, A.st);
    return rc;
}

// PolyMul_st (cufft_gpu.cuh:214-226): TwistFFT(TwistIFFT(a_i) * m) per row
int cufhedb_polymul_lvl1(cufhedb_ctx *ctx, const uint32_t *a, const double *m_fd, uint32_t *out, int B, int shared,
                         cufhedb_stream_t stream)
{
    if (!aligned_to(a, 4)) return cfdb::set_error(CUFHEDB_ERR_ARG, "a must be 4-byte aligned");
    if (!aligned_to(m_fd, 8)) return cfdb::set_error(CUFHEDB_ERR_ARG, "m_fd must be 8-byte aligned");
    if (!aligned_to(out, 4)) return cfdb::set_error(CUFHEDB_ERR_ARG, "out must be 4-byte aligned");
    if (!ctx || B < 0) return set_error(CUFHEDB_ERR_ARG, "bad argument");
    if (B == 0) return CUFHEDB_OK;
    if (!a || !m_fd || !out) return set_error(CUFHEDB_ERR_ARG, "null buffer");
    DeviceGuard guard(ctx->device);
    cudaStream_t st = (cudaStream_t)stream;
    double *fd = nullptr;
    cudaError_t e = cudaMallocAsync((void **)&fd, (size_t)B * N1 * sizeof(double), st);
    if (e == cudaSuccess) e = launch_twist_ifft1(fd, a, B, ctx->tab512, st);
    if (e == cudaSuccess) e = launch_fd_mul(fd, m_fd, N1 / 2, B, shared, st);
    if (e == cudaSuccess) e = launch_twist_fft1(out, fd, B, ctx->tab512, st);
    if (fd) cudaFreeAsync(fd, st);
    return e == cudaSuccess ? CUFHEDB_OK : cuda_error(e, "polynomial product (lvl1)");
}

int cufhedb_polymul_lvl2(cufhedb_ctx *ctx, const uint64_t *a, const double *m_fd, uint64_t *out, int B, int shared,
                         cufhedb_stream_t stream)
{
    if (!aligned_to(a, 8)) return cfdb::set_error(CUFHEDB_ERR_ARG, "a must be 8-byte aligned");
    if (!aligned_to(m_fd, 8)) return cfdb::set_error(CUFHEDB_ERR_ARG, "m_fd must be 8-byte aligned");
    if (!aligned_to(out, 8)) return cfdb::set_error(CUFHEDB_ERR_ARG, "out must be 8-byte aligned");
    if (!ctx || B < 0) return set_error(CUFHEDB_ERR_ARG, "bad argument");
    if (B == 0) return CUFHEDB_OK;
    if (!a || !m_fd || !out) return set_error(CUFHEDB_ERR_ARG, "null buffer");
    DeviceGuard guard(ctx->device);
    cudaStream_t st = (cudaStream_t)stream;
    double *fd = nullptr;
    cudaError_t e = cudaMallocAsync((void **)&fd, (size_t)B * N2 * sizeof(double), st);
    if (e == cudaSuccess) e = launch_twist_ifft2(fd, a, B, ctx->tab1024, st);
    if (e == cudaSuccess) e = launch_fd_mul(fd, m_fd, N2 / 2, B, shared, st);
    if (e == cudaSuccess) e = launch_twist_fft2(out, fd, B, ctx->tab1024, st);
    if (fd) cudaFreeAsync(fd, st);
    return e == cudaSuccess ? CUFHEDB_OK : cuda_error(e, "polynomial product (lvl2)");
}
