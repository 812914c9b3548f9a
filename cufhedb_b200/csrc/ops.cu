// Batched operator layer: cuHEDB's bootstrapped building blocks and the
// HomMSB / comparison chains, each applied to a whole column of rows at once.
//
// Restates (names as in the reference, each a batch here):
//   MSBGateBootstrapping x3, IdeGateBootstrapping x3, HomAND, HomOR,
//   LOG_to_ARI, log_rescale     src/cuHEDB/gatebootstrap_gpu.cuh:31-170
//   ExtractMSB5/9/10, HomMSB x2, ImExtractMSB5/9/14/19/24/29/33
//                               src/cuHEDB/msb_gpu.cuh:7-193
//   greater_than, greater_than_equal, less_than, less_than_equal, equal
//                               src/cuHEDB/HomCompare_gpu.cuh:13-76
// (CPU twins: src/HEDB/comparison/tfhepp_utils.cpp:8-120, operators.cpp:8-33,
// extract_msb.cpp, HomCompare.h.)  In the reference every step is one
// host-side key switch plus one single-ciphertext GPU launch per row; here
// every step is one batched key-switch kernel plus one batched bootstrap
// kernel for all rows, with the ciphertext arithmetic between steps done by
// small elementwise kernels, all enqueued on one stream (capturable into a
// CUDA graph with cufhedb_graph_begin / cufhedb_graph_end).
#include <string>

#include "ctx.cuh"

namespace cfdb {

namespace {

constexpr uint32_t MU1 = 1u << 29;
constexpr uint64_t MU2 = 1ull << 61;

// out = ((sa * a + sb * b) << shift), with badd added to the b word
template <typename T>
__global__ void lincomb_kernel(T *out, const T *a, T sa, const T *b, T sb, int shift, T badd, size_t total,
                               int width)
{
    for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        T v = sa * a[e];
        if (b) v += sb * b[e];
        v <<= shift;
        if ((int)(e % width) == width - 1) v += badd;
        out[e] = v;
    }
}

struct Ops {
    cufhedb_ctx *c;
    cudaStream_t st;
    int prec;
    int B;
    DeviceGuard guard;   // the context's device while the operator enqueues

    template <typename T>
    int alloc(T **p, size_t words)
    {
        cudaError_t e = cudaMallocAsync((void **)p, words * sizeof(T), st);
        return e == cudaSuccess ? CUFHEDB_OK : cuda_error(e, "operator scratch");
    }
    void release(void *p)
    {
        if (p) cudaFreeAsync(p, st);
    }

    template <typename T>
    int lin(T *out, const T *a, long long sa, const T *b, long long sb, int shift, T badd, int width)
    {
        const size_t total = (size_t)B * width;
        const unsigned grid = (unsigned)((total + 255) / 256 < 4096 ? (total + 255) / 256 : 4096);
        lincomb_kernel<T><<<grid, 256, 0, st>>>(out, a, (T)sa, b, (T)sb, shift, badd, total, width);
        cudaError_t e = cudaGetLastError();
        return e == cudaSuccess ? CUFHEDB_OK : cuda_error(e, "ciphertext arithmetic");
    }
    int lin1(uint32_t *out, const uint32_t *a, int sa, const uint32_t *b, int sb, int shift, uint32_t badd)
    {
        return lin<uint32_t>(out, a, sa, b, sb, shift, badd, N1 + 1);
    }
    int lin2(uint64_t *out, const uint64_t *a, long long sa, const uint64_t *b, long long sb, int shift,
             uint64_t badd)
    {
        return lin<uint64_t>(out, a, sa, b, sb, shift, badd, N2 + 1);
    }

    static TestVec tv_const(uint64_t v) { return TestVec{0, 0, v, nullptr}; }
    static TestVec tv_stair(uint32_t scale_bits) { return TestVec{1, 6, scale_bits, nullptr}; }

    // key switch of lvl1 rows (optionally sa*a + sb*b, b-offset) then PBS01
    int ks10_pbs01(uint32_t *out, const uint32_t *a, const uint32_t *b, int sa, int sb, uint32_t offset,
                   const TestVec &tv, uint32_t b_add)
    {
        uint32_t *l0 = nullptr;
        int rc = alloc(&l0, (size_t)B * (N0 + 1));
        if (!rc) rc = iks_run(c, 10, a, b, sa, sb, offset, l0, B, st);
        if (!rc) rc = pbs01_run(c, l0, out, B, tv, b_add, prec, st);
        release(l0);
        return rc;
    }
    int ks20_pbs01(uint32_t *out, const uint64_t *in, uint64_t offset, const TestVec &tv, uint32_t b_add)
    {
        uint32_t *l0 = nullptr;
        int rc = alloc(&l0, (size_t)B * (N0 + 1));
        if (!rc) rc = iks_run(c, 20, in, nullptr, 1, 0, offset, l0, B, st);
        if (!rc) rc = pbs01_run(c, l0, out, B, tv, b_add, prec, st);
        release(l0);
        return rc;
    }
    int ks20_pbs02(uint64_t *out, const uint64_t *in, uint64_t offset, const TestVec &tv, uint64_t b_add)
    {
        uint32_t *l0 = nullptr;
        int rc = alloc(&l0, (size_t)B * (N0 + 1));
        if (!rc) rc = iks_run(c, 20, in, nullptr, 1, 0, offset, l0, B, st);
        if (!rc) rc = pbs02_run(c, l0, out, B, tv, b_add, st);
        release(l0);
        return rc;
    }

    // ---- gatebootstrap_gpu.cuh building blocks --------------------------------
    int msb_11(uint32_t *out, const uint32_t *in, bool arith)
    {
        const uint32_t u = arith ? MU1 << 1 : MU1;
        return ks10_pbs01(out, in, nullptr, 1, 0, 1u << 26, tv_const((uint32_t)(0u - u)), arith ? u : 0u);
    }
    int msb_21(uint32_t *out, const uint64_t *in, bool arith)
    {
        const uint32_t u = arith ? MU1 << 1 : MU1;
        return ks20_pbs01(out, in, 1ull << 58, tv_const((uint32_t)(0u - u)), arith ? u : 0u);
    }
    int msb_22(uint64_t *out, const uint64_t *in, bool arith)
    {
        const uint64_t u = arith ? MU2 << 1 : MU2;
        return ks20_pbs02(out, in, 1ull << 57, tv_const(0ull - u), arith ? u : 0ull);
    }
    int ide_11(uint32_t *out, const uint32_t *in, uint32_t scale_bits)
    {
        return ks10_pbs01(out, in, nullptr, 1, 0, 1u << 26, tv_stair(scale_bits), 0u);
    }
    int ide_21(uint32_t *out, const uint64_t *in, uint32_t scale_bits)
    {
        return ks20_pbs01(out, in, 1ull << 58, tv_stair(scale_bits - 32), 0u);
    }
    int ide_22(uint64_t *out, const uint64_t *in, uint32_t scale_bits)
    {
        return ks20_pbs02(out, in, 1ull << 57, tv_stair(scale_bits), 0ull);
    }
    // LOG_to_ARI / log_rescale use the CPU twins' test vector, the constant
    // +2^30 (resp. +2^(scale_bits-1)) that mu_polygen(-mu) builds
    // (src/HEDB/comparison/tfhepp_utils.cpp:19-37), then add 2^29 (resp.
    // 2^(scale_bits-1)) to b: a logic 1 (phase ~ +1/8) ends at 3/8 and decodes to
    // 1, a logic 0 ends at -1/8 and decodes to 0.  The reference's GPU wrappers
    // (gatebootstrap_gpu.cuh:154-168) pass -2^30 instead, which inverts the result.
    int log_to_ari(uint32_t *out, const uint32_t *in)
    {
        return ks10_pbs01(out, in, nullptr, 1, 0, 0u, tv_const(MU1 << 1), MU1);
    }
    int log_rescale(uint32_t *out, const uint32_t *in, uint32_t scale_bits)
    {
        const uint32_t mu = 1u << (scale_bits - 1);
        return ks10_pbs01(out, in, nullptr, 1, 0, 0u, tv_const(mu), mu);
    }
    // c0 + c1 -/+ 1/8, bootstrapped to +-offset (HomAND / HomOR)
    int hom_andor(uint32_t *out, const uint32_t *ca, const uint32_t *cb, bool arith, bool is_or)
    {
        const uint32_t off = arith ? MU1 << 1 : MU1;
        const uint32_t shift = is_or ? (MU1 >> 1) : (uint32_t)(0u - (MU1 >> 1));
        return ks10_pbs01(out, ca, cb, 1, 1, shift, tv_const(off), arith ? off : 0u);
    }

    // ---- msb_gpu.cuh chains ---------------------------------------------------
    int extract_msb9(uint32_t *out, const uint32_t *in, uint32_t pb, bool arith)
    {
        uint32_t *sh = nullptr, *sg = nullptr;
        const size_t w = (size_t)B * (N1 + 1);
        int rc = alloc(&sh, w);
        if (!rc) rc = alloc(&sg, w);
        if (!rc) rc = lin1(sh, in, 1, nullptr, 0, (int)pb - 5, 0);
        if (!rc) rc = msb_11(sg, sh, true);
        if (!rc) rc = lin1(sh, sh, 1, sg, -1, 0, 0);
        if (!rc) rc = ide_11(sh, sh, 32 - pb);
        if (!rc) rc = lin1(out, in, 1, sh, -1, 0, 0);
        if (!rc) rc = msb_11(out, out, arith);
        release(sh);
        release(sg);
        return rc;
    }
    int extract_msb10(uint32_t *out, const uint32_t *in, uint32_t pb, bool arith)
    {
        uint32_t *sh = nullptr, *sg = nullptr;
        const size_t w = (size_t)B * (N1 + 1);
        int rc = alloc(&sh, w);
        if (!rc) rc = alloc(&sg, w);
        if (!rc) rc = lin1(sh, in, 1, nullptr, 0, (int)pb - 5, 0);
        if (!rc) rc = msb_11(sg, sh, true);
        if (!rc) rc = lin1(sh, sh, 1, sg, -1, 0, 0);
        if (!rc) rc = ide_11(sh, sh, 32 - pb);
        if (!rc) rc = lin1(out, in, 1, sh, -1, 0, 0);
        if (!rc) rc = extract_msb9(out, out, pb - 4, arith);
        release(sh);
        release(sg);
        return rc;
    }
    int hom_msb1(uint32_t *out, const uint32_t *in, uint32_t pb, bool arith)
    {
        if (pb <= 5) return msb_11(out, in, arith);
        if (pb <= 9) return extract_msb9(out, in, pb, arith);
        if (pb == 10) return extract_msb10(out, in, pb, arith);
        return set_error(CUFHEDB_ERR_ARG, "Plain bits out. (lvl1 HomMSB supports at most 10)");
    }
    // one lvl2 level of ImExtractMSB14/19/24/29/33: res = in - Ide(shift - MSB(shift))
    int lvl2_level(uint64_t *res, const uint64_t *in, uint32_t pb)
    {
        uint64_t *sh = nullptr, *sg = nullptr;
        const size_t w = (size_t)B * (N2 + 1);
        int rc = alloc(&sh, w);
        if (!rc) rc = alloc(&sg, w);
        if (!rc) rc = lin2(sh, in, 1, nullptr, 0, (int)pb - 6, 0);
        if (!rc) rc = msb_22(sg, sh, true);
        if (!rc) rc = lin2(sh, sh, 1, sg, -1, 0, 0);
        if (!rc) rc = ide_22(sh, sh, 64 - pb);
        if (!rc) rc = lin2(res, in, 1, sh, -1, 0, 0);
        release(sh);
        release(sg);
        return rc;
    }
    // ImExtractMSB{14,19,24,29,33}: lvl2 levels of 5 bits until <= 14 bits, then
    // lvl2 -> lvl1 key switch and the lvl1 ExtractMSB9
    int im_extract(uint32_t *out, const uint64_t *in, uint32_t pb, bool arith)
    {
        uint64_t *res = nullptr;
        int rc = alloc(&res, (size_t)B * (N2 + 1));
        if (!rc) rc = lvl2_level(res, in, pb);
        if (!rc) {
            if (pb <= 14) {
                rc = iks_run(c, 21, res, nullptr, 1, 0, 0, out, B, st);
                if (!rc) rc = extract_msb9(out, out, pb - 5, arith);
            } else {
                rc = im_extract(out, res, pb - 5, arith);
            }
        }
        release(res);
        return rc;
    }
    int hom_msb2(uint32_t *out, const uint64_t *in, uint32_t pb, bool arith)
    {
        if (pb <= 9) {
            int rc = iks_run(c, 21, in, nullptr, 1, 0, 0, out, B, st);
            if (rc) return rc;
            return pb <= 5 ? msb_11(out, out, arith) : extract_msb9(out, out, pb, arith);
        }
        if (pb <= 33) return im_extract(out, in, pb, arith);
        return set_error(CUFHEDB_ERR_ARG, "Plain bits out. (lvl2 HomMSB supports at most 33)");
    }

    // ---- HomCompare_gpu.cuh ----------------------------------------------------
    // op: 0 greater_than, 1 greater_than_equal, 2 less_than, 3 less_than_equal, 4 equal
    template <int LVL>
    int compare(int op, const void *c1, const void *c2, uint32_t *out, uint32_t pb, bool arith)
    {
        using T = typename std::conditional<LVL == 1, uint32_t, uint64_t>::type;
        const T *a = (const T *)c1, *b = (const T *)c2;
        if (op == 4) {
            uint32_t *ge = nullptr, *le = nullptr;
            const size_t w = (size_t)B * (N1 + 1);
            int rc = alloc(&ge, w);
            if (!rc) rc = alloc(&le, w);
            if (!rc) rc = compare<LVL>(1, c1, c2, ge, pb, false);
            if (!rc) rc = compare<LVL>(3, c1, c2, le, pb, false);
            if (!rc) rc = hom_andor(out, ge, le, arith, false);
            release(ge);
            release(le);
            return rc;
        }
        // greater_than: MSB(c2 - c1); greater_than_equal: NOT MSB(c1 - c2);
        // less_than: MSB(c1 - c2); less_than_equal: NOT MSB(c2 - c1)
        const bool swap = (op == 0 || op == 3);
        const bool negate = (op == 1 || op == 3);
        T *sub = nullptr;
        const int width = (LVL == 1 ? N1 : N2) + 1;
        int rc = alloc(&sub, (size_t)B * width);
        if (!rc) rc = lin<T>(sub, swap ? b : a, 1, swap ? a : b, -1, 0, 0, width);
        const bool msb_arith = negate ? false : arith;
        if (!rc) {
            if constexpr (LVL == 1) rc = hom_msb1(out, sub, pb + 1, msb_arith);
            else rc = hom_msb2(out, sub, pb + 1, msb_arith);
        }
        if (!rc && negate) {
            rc = lin1(out, out, -1, nullptr, 0, 0, 0);
            if (!rc && arith) rc = log_to_ari(out, out);
        }
        release(sub);
        return rc;
    }
};

int begin_ops(cufhedb_ctx *ctx, int B, int precision, Ops &o, cufhedb_stream_t stream)
{
    if (!ctx) return set_error(CUFHEDB_ERR_ARG, "ctx is null");
    if (B < 0) return set_error(CUFHEDB_ERR_ARG, "negative batch");
    if (precision != CUFHEDB_FP64 && precision != CUFHEDB_SPLIT32 &&
        precision != CUFHEDB_SPLIT32_TC)
        return set_error(CUFHEDB_ERR_ARG, "unsupported precision");
    if (o.guard.set(ctx->device) != cudaSuccess) return set_error(CUFHEDB_ERR_CUDA, "cudaSetDevice failed");
    o.c = ctx;
    o.st = (cudaStream_t)stream;
    o.prec = precision;
    o.B = B;
    return CUFHEDB_OK;
}

}  // namespace
}  // namespace cfdb

using cfdb::Ops;

extern "C" {

CUFHEDB_API int cufhedb_msb_bootstrap(cufhedb_ctx *ctx, int in_level, int out_level, const void *in, void *out,
                                      int B, int logic, int precision, cufhedb_stream_t stream)
{
    if (!aligned_to(in, in_level == 1 ? 4 : 8)) return cfdb::set_error(CUFHEDB_ERR_ARG, "in must be 4-byte (lvl1) or 8-byte (lvl2) aligned");
    if (!aligned_to(out, out_level == 1 ? 4 : 8)) return cfdb::set_error(CUFHEDB_ERR_ARG, "out must be 4-byte (lvl1) or 8-byte (lvl2) aligned");
    Ops o;
    int rc = cfdb::begin_ops(ctx, B, precision, o, stream);
    if (rc || B == 0) return rc;
    if (!in || !out) return cfdb::set_error(CUFHEDB_ERR_ARG, "null buffer");
    const bool arith = !logic;
    if (in_level == 1 && out_level == 1) return o.msb_11((uint32_t *)out, (const uint32_t *)in, arith);
    if (in_level == 2 && out_level == 1) return o.msb_21((uint32_t *)out, (const uint64_t *)in, arith);
    if (in_level == 2 && out_level == 2) return o.msb_22((uint64_t *)out, (const uint64_t *)in, arith);
    return cfdb::set_error(CUFHEDB_ERR_ARG, "unsupported level pair");
}

CUFHEDB_API int cufhedb_ide_bootstrap(cufhedb_ctx *ctx, int in_level, int out_level, const void *in, void *out,
                                      int B, uint32_t scale_bits, int precision, cufhedb_stream_t stream)
{
    if (!aligned_to(in, in_level == 1 ? 4 : 8)) return cfdb::set_error(CUFHEDB_ERR_ARG, "in must be 4-byte (lvl1) or 8-byte (lvl2) aligned");
    if (!aligned_to(out, out_level == 1 ? 4 : 8)) return cfdb::set_error(CUFHEDB_ERR_ARG, "out must be 4-byte (lvl1) or 8-byte (lvl2) aligned");
    Ops o;
    int rc = cfdb::begin_ops(ctx, B, precision, o, stream);
    if (rc || B == 0) return rc;
    if (!in || !out) return cfdb::set_error(CUFHEDB_ERR_ARG, "null buffer");
    if (in_level == 1 && out_level == 1 && scale_bits < 32)
        return o.ide_11((uint32_t *)out, (const uint32_t *)in, scale_bits);
    if (in_level == 2 && out_level == 1 && scale_bits >= 32 && scale_bits < 64)
        return o.ide_21((uint32_t *)out, (const uint64_t *)in, scale_bits);
    if (in_level == 2 && out_level == 2 && scale_bits < 64)
        return o.ide_22((uint64_t *)out, (const uint64_t *)in, scale_bits);
    return cfdb::set_error(CUFHEDB_ERR_ARG, "unsupported level pair or scale_bits");
}

CUFHEDB_API int cufhedb_log_to_ari(cufhedb_ctx *ctx, const uint32_t *in, uint32_t *out, int B, int precision,
                                   cufhedb_stream_t stream)
{
    if (!aligned_to(in, 4)) return cfdb::set_error(CUFHEDB_ERR_ARG, "in must be 4-byte aligned");
    if (!aligned_to(out, 4)) return cfdb::set_error(CUFHEDB_ERR_ARG, "out must be 4-byte aligned");
    Ops o;
    int rc = cfdb::begin_ops(ctx, B, precision, o, stream);
    if (rc || B == 0) return rc;
    if (!in || !out) return cfdb::set_error(CUFHEDB_ERR_ARG, "null buffer");
    return o.log_to_ari(out, in);
}

CUFHEDB_API int cufhedb_log_rescale(cufhedb_ctx *ctx, const uint32_t *in, uint32_t *out, int B, uint32_t scale_bits,
                                    int precision, cufhedb_stream_t stream)
{
    if (!aligned_to(in, 4)) return cfdb::set_error(CUFHEDB_ERR_ARG, "in must be 4-byte aligned");
    if (!aligned_to(out, 4)) return cfdb::set_error(CUFHEDB_ERR_ARG, "out must be 4-byte aligned");
    Ops o;
    int rc = cfdb::begin_ops(ctx, B, precision, o, stream);
    if (rc || B == 0) return rc;
    if (!in || !out) return cfdb::set_error(CUFHEDB_ERR_ARG, "null buffer");
    if (scale_bits < 1 || scale_bits > 31) return cfdb::set_error(CUFHEDB_ERR_ARG, "scale_bits out of range");
    return o.log_rescale(out, in, scale_bits);
}

CUFHEDB_API int cufhedb_hom_and(cufhedb_ctx *ctx, const uint32_t *ca, const uint32_t *cb, uint32_t *out, int B,
                                int logic, int precision, cufhedb_stream_t stream)
{
    if (!aligned_to(ca, 4)) return cfdb::set_error(CUFHEDB_ERR_ARG, "ca must be 4-byte aligned");
    if (!aligned_to(cb, 4)) return cfdb::set_error(CUFHEDB_ERR_ARG, "cb must be 4-byte aligned");
    if (!aligned_to(out, 4)) return cfdb::set_error(CUFHEDB_ERR_ARG, "out must be 4-byte aligned");
    Ops o;
    int rc = cfdb::begin_ops(ctx, B, precision, o, stream);
    if (rc || B == 0) return rc;
    if (!ca || !cb || !out) return cfdb::set_error(CUFHEDB_ERR_ARG, "null buffer");
    return o.hom_andor(out, ca, cb, !logic, false);
}

CUFHEDB_API int cufhedb_hom_or(cufhedb_ctx *ctx, const uint32_t *ca, const uint32_t *cb, uint32_t *out, int B,
                               int logic, int precision, cufhedb_stream_t stream)
{
    if (!aligned_to(ca, 4)) return cfdb::set_error(CUFHEDB_ERR_ARG, "ca must be 4-byte aligned");
    if (!aligned_to(cb, 4)) return cfdb::set_error(CUFHEDB_ERR_ARG, "cb must be 4-byte aligned");
    if (!aligned_to(out, 4)) return cfdb::set_error(CUFHEDB_ERR_ARG, "out must be 4-byte aligned");
    Ops o;
    int rc = cfdb::begin_ops(ctx, B, precision, o, stream);
    if (rc || B == 0) return rc;
    if (!ca || !cb || !out) return cfdb::set_error(CUFHEDB_ERR_ARG, "null buffer");
    return o.hom_andor(out, ca, cb, !logic, true);
}

CUFHEDB_API int cufhedb_hom_msb(cufhedb_ctx *ctx, int in_level, const void *in, uint32_t *out_lvl1, int B,
                                uint32_t plain_bits, int logic, int precision, cufhedb_stream_t stream)
{
    if (!aligned_to(in, in_level == 1 ? 4 : 8)) return cfdb::set_error(CUFHEDB_ERR_ARG, "in must be 4-byte (lvl1) or 8-byte (lvl2) aligned");
    if (!aligned_to(out_lvl1, 4)) return cfdb::set_error(CUFHEDB_ERR_ARG, "out_lvl1 must be 4-byte aligned");
    Ops o;
    int rc = cfdb::begin_ops(ctx, B, precision, o, stream);
    if (rc || B == 0) return rc;
    if (!in || !out_lvl1) return cfdb::set_error(CUFHEDB_ERR_ARG, "null buffer");
    if (plain_bits < 1) return cfdb::set_error(CUFHEDB_ERR_ARG, "Plain bits out.");
    if (in_level == 1) return o.hom_msb1(out_lvl1, (const uint32_t *)in, plain_bits, !logic);
    if (in_level == 2) return o.hom_msb2(out_lvl1, (const uint64_t *)in, plain_bits, !logic);
    return cfdb::set_error(CUFHEDB_ERR_ARG, "unsupported level");
}

CUFHEDB_API int cufhedb_compare(cufhedb_ctx *ctx, int op, int level, const void *c1, const void *c2,
                                uint32_t *out_lvl1, int B, uint32_t plain_bits, int logic, int precision,
                                cufhedb_stream_t stream)
{
    if (!aligned_to(c1, level == 1 ? 4 : 8)) return cfdb::set_error(CUFHEDB_ERR_ARG, "c1 must be 4-byte (lvl1) or 8-byte (lvl2) aligned");
    if (!aligned_to(c2, level == 1 ? 4 : 8)) return cfdb::set_error(CUFHEDB_ERR_ARG, "c2 must be 4-byte (lvl1) or 8-byte (lvl2) aligned");
    if (!aligned_to(out_lvl1, 4)) return cfdb::set_error(CUFHEDB_ERR_ARG, "out_lvl1 must be 4-byte aligned");
    Ops o;
    int rc = cfdb::begin_ops(ctx, B, precision, o, stream);
    if (rc || B == 0) return rc;
    if (!c1 || !c2 || !out_lvl1) return cfdb::set_error(CUFHEDB_ERR_ARG, "null buffer");
    if (op < 0 || op > 4) return cfdb::set_error(CUFHEDB_ERR_ARG, "unknown comparison");
    if (plain_bits < 1) return cfdb::set_error(CUFHEDB_ERR_ARG, "Plain bits out.");
    if (level == 1) return o.compare<1>(op, c1, c2, out_lvl1, plain_bits, !logic);
    if (level == 2) return o.compare<2>(op, c1, c2, out_lvl1, plain_bits, !logic);
    return cfdb::set_error(CUFHEDB_ERR_ARG, "unsupported level");
}

// ---- CUDA-graph capture of an operator DAG -----------------------------------

struct cufhedb_graph {
    cudaGraph_t g = nullptr;
    cudaGraphExec_t x = nullptr;
};

CUFHEDB_API int cufhedb_graph_begin(cufhedb_ctx *ctx, cufhedb_stream_t stream)
{
    if (!ctx || !stream) return cfdb::set_error(CUFHEDB_ERR_ARG, "capture needs a context and a non-default stream");
    cfdb::DeviceGuard g(ctx->device);
    cudaError_t e = cudaStreamBeginCapture((cudaStream_t)stream, cudaStreamCaptureModeThreadLocal);
    return e == cudaSuccess ? CUFHEDB_OK : cfdb::cuda_error(e, "cudaStreamBeginCapture");
}

CUFHEDB_API int cufhedb_graph_end(cufhedb_ctx *ctx, cufhedb_stream_t stream, cufhedb_graph **out)
{
    if (!ctx || !stream || !out) return cfdb::set_error(CUFHEDB_ERR_ARG, "bad argument");
    cfdb::DeviceGuard g(ctx->device);
    cufhedb_graph *gr = new cufhedb_graph();
    cudaError_t e = cudaStreamEndCapture((cudaStream_t)stream, &gr->g);
    if (e == cudaSuccess) e = cudaGraphInstantiate(&gr->x, gr->g, 0);
    if (e != cudaSuccess) {
        if (gr->g) cudaGraphDestroy(gr->g);
        delete gr;
        *out = nullptr;
        return cfdb::cuda_error(e, "graph capture");
    }
    *out = gr;
    return CUFHEDB_OK;
}

CUFHEDB_API int cufhedb_graph_launch(cufhedb_graph *graph, cufhedb_stream_t stream)
{
    if (!graph) return cfdb::set_error(CUFHEDB_ERR_ARG, "graph is null");
    cudaError_t e = cudaGraphLaunch(graph->x, (cudaStream_t)stream);
    return e == cudaSuccess ? CUFHEDB_OK : cfdb::cuda_error(e, "cudaGraphLaunch");
}

CUFHEDB_API int cufhedb_graph_destroy(cufhedb_graph *graph)
{
    if (!graph) return CUFHEDB_OK;
    if (graph->x) cudaGraphExecDestroy(graph->x);
    if (graph->g) cudaGraphDestroy(graph->g);
    delete graph;
    return CUFHEDB_OK;
}

}  // extern "C"
