// C ABI of the engine (include/cufhedb_b200.h): context, key material,
// batched operations and host-buffer entry points.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "cufhedb_b200.h"
#include "fft_f32.cuh"
#include "extprod.cuh"
#include "fftops.cuh"
#include "iks.cuh"
#include "keys.cuh"
#include "lvl2.cuh"
#include "pbs_common.cuh"
#include "tc_stage1.cuh"

using namespace cfdb;

#include "ctx.cuh"

namespace {

thread_local std::string g_err;

int fail(int code, const std::string &msg)
{
    g_err = msg;
    return code;
}

int cuda_fail(cudaError_t e, const char *what)
{
    const int code = (e == cudaErrorMemoryAllocation) ? CUFHEDB_ERR_OOM : CUFHEDB_ERR_CUDA;
    return fail(code, std::string(what) + ": " + cudaGetErrorString(e));
}

#define CK(call)                                                \
    do {                                                        \
        cudaError_t e_ = (call);                                \
        if (e_ != cudaSuccess) return cuda_fail(e_, #call);     \
    } while (0)

#define NEED(cond, msg)                                                 \
    do {                                                                \
        if (!(cond)) return fail(CUFHEDB_ERR_ARG, std::string(msg));    \
    } while (0)

constexpr size_t BK01_ROWS = (size_t)N0 * 2 * L1;   // TRGSW rows of the lvl01 key
constexpr size_t BK01_WORDS = BK01_ROWS * 2 * N1;
constexpr size_t BK02_ROWS = (size_t)N0 * 2 * L2;   // TRGSW rows of the lvl02 key
constexpr size_t BK02_WORDS = BK02_ROWS * 2 * N2;

// key-switching keys: rows (i, j, digit value) of a TLWE each; TFHEpp's
// layout (and the files') packs rows of row_words; the device layout pads
// every row to ksk_pitch(row_words) words
size_t ksk_rows(int kind)
{
    if (kind == 10) return (size_t)1024 * 2 * 1023;
    if (kind == 20) return (size_t)2048 * 2 * 1023;
    if (kind == 21) return (size_t)2048 * 10 * 7;
    return 0;
}
size_t ksk_row_words(int kind) { return kind == 21 ? N1 + 1 : N0 + 1; }
size_t ksk_words(int kind) { return ksk_rows(kind) * ksk_row_words(kind); }
size_t ksk_dev_bytes(int kind) { return ksk_rows(kind) * ksk_pitch((int)ksk_row_words(kind)) * sizeof(uint32_t); }

// rows [r0, r0 + n) from the packed host layout into the device layout, pad
// words zeroed
cudaError_t ksk_rows_to_device(uint32_t *dev, int kind, size_t r0, const void *host, size_t n)
{
    const size_t rw = ksk_row_words(kind), pw = (size_t)ksk_pitch((int)rw);
    cudaError_t e = cudaMemcpy2D(dev + r0 * pw, pw * 4, host, rw * 4, rw * 4, n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset2D(dev + r0 * pw + rw, pw * 4, 0, (pw - rw) * 4, n);
    return e;
}

int ksk_slot(int kind) { return kind == 10 ? 0 : kind == 20 ? 1 : kind == 21 ? 2 : -1; }

void build_tables(Fft512Tables &T)
{
    const long double PI = 3.141592653589793238462643383279502884L;
    for (int q2 = 0; q2 < 16; ++q2)
        for (int m1 = 0; m1 < 32; ++m1) {
            const long double a = 2.0L * PI * (long double)((m1 * q2) % 512) / 512.0L;
            T.tw512[q2 * 32 + m1] = make_double2((double)cosl(a), (double)sinl(a));
        }
    for (int m2 = 0; m2 < 16; ++m2)
        for (int m1 = 0; m1 < 32; ++m1) {
            const long double a = 2.0L * PI * (long double)(m1 + 32 * m2) / 2048.0L;
            T.twist[m2 * 32 + m1] = make_double2((double)cosl(a), (double)sinl(a));
        }
    for (int j = 0; j < 16; ++j) {
        const long double a = 2.0L * PI * (long double)j / 32.0L;
        T.w32[j] = make_double2((double)cosl(a), (double)sinl(a));
    }
}

void build_tables2(Fft1024Tables &T) { build_fft8x_tables<T2>(T); }

void build_tables_f(const Fft512Tables &D, Fft512TablesF &F)
{
    auto dup = [](double c, double s) { return make_float4((float)c, (float)c, (float)s, (float)s); };
    auto cx = [](double2 a, double2 b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); };
    Fft512TablesPlain &P = F.plain;
    Fft512TablesFold &Q = F.fold;
    for (int i = 0; i < 512; ++i) {
        P.tw512[i] = make_float2((float)D.tw512[i].x, (float)D.tw512[i].y);
        P.twist[i] = make_float2((float)D.twist[i].x, (float)D.twist[i].y);
        P.tw512p[i] = dup(D.tw512[i].x, D.tw512[i].y);
        P.untwistp[i] = dup(D.twist[i].x / 512.0, -D.twist[i].y / 512.0);
        const double2 t = cx(D.tw512[i], D.twist[i % 32]);   // W^{m1 q2} w^{m1}, m1 = i % 32
        Q.tw512w[i] = make_float2((float)t.x, (float)t.y);
        Q.tw512u[i] = dup(t.x / 512.0, t.y / 512.0);
    }
    for (int j = 0; j < 16; ++j) {
        P.w32[j] = make_float2((float)D.w32[j].x, (float)D.w32[j].y);
        P.w32p[j] = Q.w32p[j] = dup(D.w32[j].x, D.w32[j].y);
    }
    build_stage1_b(F.tc_b[0], F.tc_b[1]);
}

struct GateSpec {
    int sa, sb;
    uint32_t offset;
};

// thirdparty/TFHEpp/src/gate.cpp:60-181 (mu = lvl1param::mu = 2^29)
const GateSpec kGates[10] = {
    {-1, -1, 1u << 29},          {-1, -1, 0u - (1u << 29)}, {-2, -2, 0u - (2u << 29)}, {1, 1, 0u - (1u << 29)},
    {1, 1, 1u << 29},            {2, 2, 2u << 29},          {-1, 1, 0u - (1u << 29)},  {1, -1, 0u - (1u << 29)},
    {-1, 1, 1u << 29},           {1, -1, 1u << 29},
};

TestVec to_tv(const cufhedb_testvec *tv)
{
    TestVec t{};
    t.kind = tv->kind;
    t.pad = tv->pad_bits;
    t.value = tv->value;
    t.poly = tv->poly;
    return t;
}

int check_tv(const cufhedb_testvec *tv, int N)
{
    NEED(tv != nullptr, "test vector is null");
    NEED(tv->kind >= 0 && tv->kind <= 2, "unknown test-vector kind");
    if (tv->kind == CUFHEDB_TV_STAIRCASE) {
        NEED(tv->pad_bits >= 0 && tv->pad_bits < 31, "staircase pad_bits out of range");
        NEED(tv->value < 64, "staircase scale_bits out of range");
    }
    if (tv->kind == CUFHEDB_TV_POLY) NEED(tv->poly != nullptr, "test-vector polynomial is null");
    (void)N;
    return CUFHEDB_OK;
}

bool valid_precision(int p) { return p == CUFHEDB_FP64 || p == CUFHEDB_SPLIT32 || p == CUFHEDB_SPLIT32_TC; }

// the lvl01 PBS kernel of a precision, in the launch shape the context's
// table picks for the batch (key, tables and kernel set in `a` here)
int launch_pbs01_any(cufhedb_ctx *ctx, Pbs01Args &a, int precision, cudaStream_t st)
{
    // CUFHEDB_SPLIT32 lets the measured tables pick the stage-1 layout too;
    // CUFHEDB_SPLIT32_TC forces the tensor-core one
    int w = pbs01_choose_w(a.B, ctx->num_sms, ctx->pbs01_pass_ms[precision]);
    if (precision == CUFHEDB_SPLIT32) {
        const SplitLaunch c = pbs01_split_choose(a.B, ctx->num_sms, ctx->pbs01_pass_ms[CUFHEDB_SPLIT32],
                                                 ctx->pbs01_pass_ms[CUFHEDB_SPLIT32_TC]);
        w = c.w;
        if (c.tc) precision = CUFHEDB_SPLIT32_TC;
    }
    if (precision == CUFHEDB_FP64) {
        a.bk = ctx->bk01;
        a.tables = ctx->tab512;
        CK(launch_pbs01_f64(a, ctx->num_sms, w, st));
        return CUFHEDB_OK;
    }
    if (!ctx->bk01_split) return fail(CUFHEDB_ERR_NOKEY, "split-precision lvl01 key not prepared");
    a.bk = reinterpret_cast<const double2 *>(ctx->bk01_split);
    a.tables = ctx->tab512f;
    if (precision == CUFHEDB_SPLIT32_TC) CK(launch_pbs01_split_tc(a, ctx->num_sms, w, st));
    else CK(launch_pbs01_split(a, ctx->num_sms, w, st));
    return CUFHEDB_OK;
}

int pbs01_enqueue(cufhedb_ctx *ctx, const uint32_t *in, uint32_t *out, int B, const cufhedb_testvec *tv,
                  int precision, cudaStream_t st)
{
    if (!ctx->bk01) return fail(CUFHEDB_ERR_NOKEY, "lvl01 bootstrapping key not loaded");
    if (!valid_precision(precision)) return fail(CUFHEDB_ERR_ARG, "unsupported precision");
    Pbs01Args a{};
    a.in = in;
    a.out = out;
    a.B = B;
    a.tv = to_tv(tv);
    a.err = ctx->err;
    return launch_pbs01_any(ctx, a, precision, st);
}

int gate_enqueue(cufhedb_ctx *ctx, int gate, const uint32_t *ca, const uint32_t *cb, uint32_t *out, int B,
                 int precision, cudaStream_t st)
{
    NEED(gate >= 0 && gate < 10, "unknown gate");
    if (!ctx->ksk[0]) return fail(CUFHEDB_ERR_NOKEY, "lvl10 key-switching key not loaded");
    if (!ctx->bk01) return fail(CUFHEDB_ERR_NOKEY, "lvl01 bootstrapping key not loaded");
    uint32_t *mid = nullptr;
    CK(cudaMallocAsync((void **)&mid, (size_t)B * (N0 + 1) * sizeof(uint32_t), st));
    IksArgs k{};
    k.in32 = ca;
    k.in32b = cb;
    k.sa = kGates[gate].sa;
    k.sb = kGates[gate].sb;
    k.offset = kGates[gate].offset;
    k.out = mid;
    k.ksk = ctx->ksk[0];
    k.B = B;
    cudaError_t e = launch_iks(k, 10, st);
    cufhedb_testvec tv{CUFHEDB_TV_CONST, 0, 1u << 29, nullptr};
    int rc = (e == cudaSuccess) ? pbs01_enqueue(ctx, mid, out, B, &tv, precision, st) : cuda_fail(e, "iks10");
    cudaError_t ef = cudaFreeAsync(mid, st);
    if (rc != CUFHEDB_OK) return rc;
    CK(ef);
    return CUFHEDB_OK;
}

}  // namespace

// Internal entry points shared with other translation units of the library
// (not exported).
namespace cfdb {

int set_error(int code, const char *msg) { return fail(code, msg); }

int cuda_error(cudaError_t e, const char *what) { return cuda_fail(e, what); }

int pbs01_run(cufhedb_ctx *ctx, const uint32_t *in, uint32_t *out, int B, const TestVec &tv, uint32_t b_add,
              int precision, cudaStream_t st)
{
    if (B <= 0) return CUFHEDB_OK;
    if (!ctx->bk01) return fail(CUFHEDB_ERR_NOKEY, "lvl01 bootstrapping key not loaded");
    if (!valid_precision(precision)) return fail(CUFHEDB_ERR_ARG, "unsupported precision");
    Pbs01Args a{};
    a.in = in;
    a.out = out;
    a.B = B;
    a.tv = tv;
    a.out_b_add = b_add;
    a.err = ctx->err;
    return launch_pbs01_any(ctx, a, precision, st);
}

int pbs02_run(cufhedb_ctx *ctx, const uint32_t *in, uint64_t *out, int B, const TestVec &tv, uint64_t b_add,
              cudaStream_t st)
{
    if (B <= 0) return CUFHEDB_OK;
    if (!ctx->bk02) return fail(CUFHEDB_ERR_NOKEY, "lvl02 bootstrapping key not loaded");
    Pbs02Args a{};
    a.in = in;
    a.out = out;
    a.B = B;
    a.bk = ctx->bk02;
    a.tables = ctx->tab1024;
    a.tv = tv;
    a.out_b_add = b_add;
    a.err = ctx->err;
    CK(launch_pbs02_f64(a, ctx->num_sms, pbs02_choose_p(B, ctx->num_sms, ctx->pbs02_pass_ms), st));
    return CUFHEDB_OK;
}

int iks_run(cufhedb_ctx *ctx, int kind, const void *in, const uint32_t *in_b, int sa, int sb, uint64_t offset,
            uint32_t *out, int B, cudaStream_t st)
{
    if (B <= 0) return CUFHEDB_OK;
    const int slot = ksk_slot(kind);
    if (slot < 0) return fail(CUFHEDB_ERR_ARG, "unknown key-switching kind");
    if (!ctx->ksk[slot]) return fail(CUFHEDB_ERR_NOKEY, "key-switching key not loaded");
    IksArgs k{};
    if (kind == 10) {
        k.in32 = (const uint32_t *)in;
        k.in32b = in_b;
        k.sa = sa;
        k.sb = sb;
        k.offset = (uint32_t)offset;
    } else {
        k.in64 = (const uint64_t *)in;
        k.sa = 1;
        k.offset64 = offset;
    }
    k.out = out;
    k.ksk = ctx->ksk[slot];
    k.B = B;
    CK(launch_iks(k, kind, st));
    return CUFHEDB_OK;
}

int ctx_device(const cufhedb_ctx *ctx) { return ctx->device; }

// IKS10 of the combined gate input into the caller's lvl0 scratch (B x 673
// words, fully overwritten), then PBS01 into `out`; allocates nothing.
int gate_enqueue_into(cufhedb_ctx *ctx, int gate, const uint32_t *ca, const uint32_t *cb, uint32_t *out, int B,
                      int precision, cudaStream_t st, uint32_t *scratch_lvl0)
{
    NEED(gate >= 0 && gate < 10, "unknown gate");
    if (!ctx->ksk[0]) return fail(CUFHEDB_ERR_NOKEY, "lvl10 key-switching key not loaded");
    if (!ctx->bk01) return fail(CUFHEDB_ERR_NOKEY, "lvl01 bootstrapping key not loaded");
    IksArgs k{};
    k.in32 = ca;
    k.in32b = cb;
    k.sa = kGates[gate].sa;
    k.sb = kGates[gate].sb;
    k.offset = kGates[gate].offset;
    k.out = scratch_lvl0;
    k.ksk = ctx->ksk[0];
    k.B = B;
    CK(launch_iks(k, 10, st));
    cufhedb_testvec tv{CUFHEDB_TV_CONST, 0, 1u << 29, nullptr};
    return pbs01_enqueue(ctx, scratch_lvl0, out, B, &tv, precision, st);
}

}  // namespace cfdb

extern "C" {

int cufhedb_abi_version(void) { return CUFHEDB_ABI_VERSION; }

const char *cufhedb_last_error(void) { return g_err.c_str(); }

int cufhedb_ctx_create(cufhedb_ctx **out, int device)
{
    NEED(out != nullptr, "out is null");
    *out = nullptr;
    int ndev = 0;
    CK(cudaGetDeviceCount(&ndev));
    NEED(device >= 0 && device < ndev, "device index out of range");
    cudaDeviceProp prop;
    CK(cudaGetDeviceProperties(&prop, device));
    if (prop.major < 10)
        return fail(CUFHEDB_ERR_UNSUPPORTED, "cufhedb_b200 needs an sm_100 (Blackwell) device");
    DeviceGuard guard;
    CK(guard.set(device));
    cufhedb_ctx *ctx = new cufhedb_ctx();
    ctx->device = device;
    ctx->num_sms = prop.multiProcessorCount;
    Fft512Tables host_tab;
    build_tables(host_tab);
    Fft512TablesF host_tabf;
    build_tables_f(host_tab, host_tabf);
    cudaError_t e = cudaMalloc((void **)&ctx->tab512, sizeof(Fft512Tables));
    if (e == cudaSuccess) e = cudaMemcpy(ctx->tab512, &host_tab, sizeof(Fft512Tables), cudaMemcpyHostToDevice);
    Fft1024Tables *host_tab2 = new Fft1024Tables;
    build_tables2(*host_tab2);
    if (e == cudaSuccess) e = cudaMalloc((void **)&ctx->tab1024, sizeof(Fft1024Tables));
    if (e == cudaSuccess) e = cudaMemcpy(ctx->tab1024, host_tab2, sizeof(Fft1024Tables), cudaMemcpyHostToDevice);
    delete host_tab2;
    if (e == cudaSuccess) e = cudaMalloc((void **)&ctx->tab512f, sizeof(Fft512TablesF));
    if (e == cudaSuccess) e = cudaMemcpy(ctx->tab512f, &host_tabf, sizeof(Fft512TablesF), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMalloc((void **)&ctx->err, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(ctx->err, 0, sizeof(int));
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->io, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = init_pbs01_f64();
    if (e == cudaSuccess) e = init_pbs01_split();
    if (e == cudaSuccess) e = init_pbs02_f64();
    if (e == cudaSuccess) e = init_extprod1();
    if (e == cudaSuccess) e = noalloc_scratch_address(&ctx->noalloc_scratch);
    if (e == cudaSuccess) {
        // The entry points take their scratch from the device's stream-ordered
        // pool (cudaMallocAsync).  With the pool's default release threshold
        // of 0 every synchronisation hands its memory back to the driver, so
        // a synchronous call (the host-buffer entry points, the drop-in
        // header's batches) would map its scratch afresh each time; the pool
        // keeps what it has instead.
        cudaMemPool_t pool = nullptr;
        uint64_t keep = UINT64_MAX;
        e = cudaDeviceGetDefaultMemPool(&pool, device);
        if (e == cudaSuccess) e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    if (e != cudaSuccess) {
        cufhedb_ctx_destroy(ctx);
        return cuda_fail(e, "context set-up");
    }
    *out = ctx;
    return CUFHEDB_OK;
}

int cufhedb_ctx_destroy(cufhedb_ctx *ctx)
{
    if (!ctx) return CUFHEDB_OK;
    DeviceGuard g(ctx->device);
    if (ctx->io) cudaStreamSynchronize(ctx->io);
    cudaFree(ctx->tab512);
    cudaFree(ctx->tab512f);
    cudaFree(ctx->tab1024);
    cudaFree(ctx->bk02);
    cudaFree(ctx->bk02_int);
    cudaFree(ctx->bk01);
    cudaFree(ctx->bk01_split);
    cudaFree(ctx->bk01_int);
    for (auto p : ctx->ksk) cudaFree(p);
    cudaFree(ctx->err);
    cudaFree(ctx->s0_d);
    cudaFree(ctx->s1_d);
    cudaFree(ctx->s2_d);
    if (ctx->io) cudaStreamDestroy(ctx->io);
    delete ctx;
    return CUFHEDB_OK;
}

int cufhedb_ctx_num_sms(const cufhedb_ctx *ctx) { return ctx ? ctx->num_sms : 0; }

int cufhedb_sync(cufhedb_ctx *ctx, cufhedb_stream_t stream)
{
    NEED(ctx != nullptr, "ctx is null");
    DeviceGuard g(ctx->device);
    CK(cudaStreamSynchronize((cudaStream_t)stream));
    int flag = 0;
    CK(cudaMemcpy(&flag, ctx->err, sizeof(int), cudaMemcpyDeviceToHost));
    if (flag) {
        CK(cudaMemset(ctx->err, 0, sizeof(int)));
        return fail(CUFHEDB_ERR_DEVICE, "a kernel gave up a bounded wait (code " + std::to_string(flag) + ")");
    }
    return CUFHEDB_OK;
}

// ---- keys ----------------------------------------------------------------

int cufhedb_secret_keys(uint64_t seed, uint32_t *s0, uint32_t *s1, uint64_t *s2)
{
    NEED(s0 && s1 && s2, "null output");
    host_secret_keys(seed, s0, s1, s2);
    return CUFHEDB_OK;
}

static int ensure_alloc(void **p, size_t bytes)
{
    if (*p) return CUFHEDB_OK;
    CK(cudaMalloc(p, bytes));
    return CUFHEDB_OK;
}

// split-precision copy of the lvl01 key, from the integer key on the device
static int prepare_split01(cufhedb_ctx *ctx)
{
    int rc = ensure_alloc((void **)&ctx->bk01_split, BK01_ROWS * 1024 * sizeof(float4));
    if (rc) return rc;
    CK(bk01_to_split(ctx->bk01_split, ctx->bk01_int, (int)BK01_ROWS, ctx->tab512, 0));
    CK(cudaDeviceSynchronize());
    return CUFHEDB_OK;
}

int cufhedb_load_bkfft_lvl01(cufhedb_ctx *ctx, const double *bkfft)
{
    NEED(ctx && bkfft, "null argument");
    DeviceGuard g(ctx->device);
    int rc = ensure_alloc((void **)&ctx->bk01, BK01_ROWS * 1024 * sizeof(double2));
    if (rc) return rc;
    double *tmp = nullptr;
    CK(cudaMalloc((void **)&tmp, BK01_WORDS * sizeof(double)));
    cudaError_t e = cudaMemcpy(tmp, bkfft, BK01_WORDS * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = bkfft01_permute(ctx->bk01, tmp, (int)BK01_ROWS, 0);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    cudaFree(tmp);
    if (e != cudaSuccess) return cuda_fail(e, "load_bkfft_lvl01");
    // the integer key (inverse transform, rounded) feeds the split-precision limbs
    rc = ensure_alloc((void **)&ctx->bk01_int, BK01_WORDS * sizeof(uint32_t));
    if (rc) return rc;
    CK(bk01_fft_to_int(ctx->bk01_int, ctx->bk01, (int)BK01_ROWS, ctx->tab512, 0));
    return prepare_split01(ctx);
}

int cufhedb_load_bk_lvl01(cufhedb_ctx *ctx, const uint32_t *bk)
{
    NEED(ctx && bk, "null argument");
    DeviceGuard g(ctx->device);
    int rc = ensure_alloc((void **)&ctx->bk01, BK01_ROWS * 1024 * sizeof(double2));
    if (rc) return rc;
    rc = ensure_alloc((void **)&ctx->bk01_int, BK01_WORDS * sizeof(uint32_t));
    if (rc) return rc;
    CK(cudaMemcpy(ctx->bk01_int, bk, BK01_WORDS * sizeof(uint32_t), cudaMemcpyHostToDevice));
    CK(bk01_to_fft(ctx->bk01, ctx->bk01_int, (int)BK01_ROWS, ctx->tab512, 0));
    CK(cudaDeviceSynchronize());
    return prepare_split01(ctx);
}

int cufhedb_load_ksk(cufhedb_ctx *ctx, int kind, const uint32_t *ksk)
{
    NEED(ctx && ksk, "null argument");
    const int slot = ksk_slot(kind);
    NEED(slot >= 0, "unknown key-switching key kind");
    DeviceGuard g(ctx->device);
    int rc = ensure_alloc((void **)&ctx->ksk[slot], ksk_dev_bytes(kind));
    if (rc) return rc;
    CK(ksk_rows_to_device(ctx->ksk[slot], kind, 0, ksk, ksk_rows(kind)));
    return CUFHEDB_OK;
}

// ---- key files (the reference's raw layout, test/HE3_Query/fastR.h:6-74) -----

namespace {

// whole-file sizes of the three sections
constexpr size_t KF_SK_BYTES = (size_t)N1 * 4;
constexpr size_t KF_BK_BYTES = BK01_WORDS * sizeof(double);
constexpr size_t KF_KSK_BYTES = (size_t)1024 * 2 * 1023 * (N0 + 1) * 4;
constexpr size_t KF_CHUNK = (size_t)64 << 20;   // host staging for the key-switching key

struct FileCloser {
    FILE *f;
    ~FileCloser()
    {
        if (f) fclose(f);
    }
};

struct PinnedBuf {
    void *p = nullptr;
    ~PinnedBuf() { cudaFreeHost(p); }
};

// a whole key-switching key from a file (packed rows) into the device layout,
// through a pinned staging buffer of whole rows
int ksk_from_file(uint32_t *dev, int kind, FILE *f)
{
    const size_t rb = ksk_row_words(kind) * 4, rows = ksk_rows(kind), per = KF_CHUNK / rb;
    PinnedBuf buf;
    CK(cudaMallocHost(&buf.p, per * rb));
    for (size_t r0 = 0; r0 < rows; r0 += per) {
        const size_t m = std::min(per, rows - r0);
        if (fread(buf.p, 1, m * rb, f) != m * rb) return fail(CUFHEDB_ERR_ARG, "short read (key-switching key)");
        CK(ksk_rows_to_device(dev, kind, r0, buf.p, m));
    }
    return CUFHEDB_OK;
}

}  // namespace

int cufhedb_load_keyfile(cufhedb_ctx *ctx, const char *path, uint32_t *sk_out)
{
    NEED(ctx && path, "null argument");
    FileCloser fc{fopen(path, "rb")};
    if (!fc.f) return fail(CUFHEDB_ERR_ARG, std::string("cannot open key file ") + path);
    if (fseeko(fc.f, 0, SEEK_END) != 0) return fail(CUFHEDB_ERR_ARG, "cannot size key file");
    const off_t size = ftello(fc.f);
    if (size != (off_t)(KF_SK_BYTES + KF_BK_BYTES + KF_KSK_BYTES))
        return fail(CUFHEDB_ERR_ARG, "key file size is not secret key + BootstrappingKeyFFT<lvl01> + "
                                     "KeySwitchingKey<lvl10>");
    rewind(fc.f);
    std::vector<uint32_t> sk(N1);
    if (fread(sk.data(), 1, KF_SK_BYTES, fc.f) != KF_SK_BYTES) return fail(CUFHEDB_ERR_ARG, "short read (sk)");
    std::vector<double> bk(BK01_WORDS);
    if (fread(bk.data(), 1, KF_BK_BYTES, fc.f) != KF_BK_BYTES) return fail(CUFHEDB_ERR_ARG, "short read (bkfft)");
    int rc = cufhedb_load_bkfft_lvl01(ctx, bk.data());
    if (rc) return rc;
    DeviceGuard g(ctx->device);
    rc = ensure_alloc((void **)&ctx->ksk[0], ksk_dev_bytes(10));
    if (rc) return rc;
    rc = ksk_from_file(ctx->ksk[0], 10, fc.f);
    if (rc) return rc;
    if (sk_out) std::memcpy(sk_out, sk.data(), KF_SK_BYTES);
    return CUFHEDB_OK;
}

// ---- TFHEpp cereal key archives ---------------------------------------------
// The reference's key files (src/HEDB/utils/serialize.cpp:7-60,
// src/ARCEDB/utils/serialize.cpp) are cereal PortableBinary archives of
// EvalKey::serialize_<key>(ar) = ar(params, unique_ptr<key>)
// (thirdparty/TFHEpp/include/cloudkey.hpp:149-228): one endianness byte (1 =
// little endian), the parameter block, the pointer's valid byte (1), then the
// key's std::arrays of arithmetic values as one raw block, little endian, in
// TFHEpp's in-memory layout.  The key is therefore the file's last
// sizeof(key) bytes; the checks below pin the bytes around it.
static size_t cereal_key_bytes(int kind)
{
    switch (kind) {
    case CUFHEDB_CEREAL_BKFFT01: return BK01_WORDS * sizeof(double);
    case CUFHEDB_CEREAL_BKFFT02: return BK02_WORDS * sizeof(double);
    case CUFHEDB_CEREAL_KSK10: return ksk_words(10) * 4;
    case CUFHEDB_CEREAL_KSK20: return ksk_words(20) * 4;
    case CUFHEDB_CEREAL_KSK21: return ksk_words(21) * 4;
    default: return 0;
    }
}

int cufhedb_cereal_key_payload(const char *path, int kind, uint64_t *offset, uint64_t *bytes)
{
    NEED(path && offset && bytes, "null argument");
    const size_t n = cereal_key_bytes(kind);
    NEED(n > 0, "unknown cereal key kind");
    FileCloser fc{fopen(path, "rb")};
    if (!fc.f) return fail(CUFHEDB_ERR_ARG, std::string("cannot open ") + path);
    if (fseeko(fc.f, 0, SEEK_END) != 0) return fail(CUFHEDB_ERR_ARG, "cannot size the archive");
    const off_t size = ftello(fc.f);
    if (size < (off_t)(n + 2)) return fail(CUFHEDB_ERR_ARG, "archive smaller than the key it should hold");
    unsigned char endian = 0, valid = 0;
    rewind(fc.f);
    if (fread(&endian, 1, 1, fc.f) != 1) return fail(CUFHEDB_ERR_ARG, "short read");
    if (fseeko(fc.f, size - (off_t)n - 1, SEEK_SET) != 0 || fread(&valid, 1, 1, fc.f) != 1)
        return fail(CUFHEDB_ERR_ARG, "short read");
    if (endian != 1) return fail(CUFHEDB_ERR_ARG, "not a little-endian cereal portable binary archive");
    if (valid != 1) return fail(CUFHEDB_ERR_ARG, "the archive's key pointer is empty or of another key type");
    *offset = (uint64_t)(size - (off_t)n);
    *bytes = n;
    return CUFHEDB_OK;
}

int cufhedb_load_cereal_key(cufhedb_ctx *ctx, const char *path, int kind)
{
    NEED(ctx != nullptr, "ctx is null");
    uint64_t off = 0, n = 0;
    int rc = cufhedb_cereal_key_payload(path, kind, &off, &n);
    if (rc) return rc;
    FileCloser fc{fopen(path, "rb")};
    if (!fc.f || fseeko(fc.f, (off_t)off, SEEK_SET) != 0) return fail(CUFHEDB_ERR_ARG, "cannot seek in the archive");
    if (kind == CUFHEDB_CEREAL_BKFFT01 || kind == CUFHEDB_CEREAL_BKFFT02) {
        std::vector<double> bk(n / sizeof(double));
        if (fread(bk.data(), 1, n, fc.f) != n) return fail(CUFHEDB_ERR_ARG, "short read (bootstrapping key)");
        return kind == CUFHEDB_CEREAL_BKFFT01 ? cufhedb_load_bkfft_lvl01(ctx, bk.data())
                                              : cufhedb_load_bkfft_lvl02(ctx, bk.data());
    }
    const int ksk = kind == CUFHEDB_CEREAL_KSK10 ? 10 : kind == CUFHEDB_CEREAL_KSK20 ? 20 : 21;
    const int slot = ksk_slot(ksk);
    DeviceGuard g(ctx->device);
    rc = ensure_alloc((void **)&ctx->ksk[slot], ksk_dev_bytes(ksk));
    if (rc) return rc;
    return ksk_from_file(ctx->ksk[slot], ksk, fc.f);
}

int cufhedb_save_keyfile(cufhedb_ctx *ctx, const char *path, const uint32_t *sk)
{
    NEED(ctx && path, "null argument");
    if (!ctx->bk01_int) return fail(CUFHEDB_ERR_NOKEY, "lvl01 bootstrapping key not loaded");
    if (!ctx->ksk[0]) return fail(CUFHEDB_ERR_NOKEY, "lvl10 key-switching key not loaded");
    DeviceGuard g(ctx->device);
    std::vector<uint32_t> skw(N1, 0u);
    if (sk) std::memcpy(skw.data(), sk, KF_SK_BYTES);
    else if (ctx->have_sk) CK(cudaMemcpy(skw.data(), ctx->s1_d, KF_SK_BYTES, cudaMemcpyDeviceToHost));
    // TFHEpp's BootstrappingKeyFFT<lvl01param>: TwistIFFT of every key polynomial
    double *fd = nullptr;
    CK(cudaMalloc((void **)&fd, KF_BK_BYTES));
    std::vector<double> bk(BK01_WORDS);
    cudaError_t e = launch_twist_ifft1(fd, ctx->bk01_int, (int)(BK01_ROWS * 2), ctx->tab512, 0);
    if (e == cudaSuccess) e = cudaMemcpy(bk.data(), fd, KF_BK_BYTES, cudaMemcpyDeviceToHost);
    cudaFree(fd);
    if (e != cudaSuccess) return cuda_fail(e, "save_keyfile (bkfft)");
    FileCloser fc{fopen(path, "wb")};
    if (!fc.f) return fail(CUFHEDB_ERR_ARG, std::string("cannot create key file ") + path);
    if (fwrite(skw.data(), 1, KF_SK_BYTES, fc.f) != KF_SK_BYTES || fwrite(bk.data(), 1, KF_BK_BYTES, fc.f) != KF_BK_BYTES)
        return fail(CUFHEDB_ERR_ARG, "short write");
    const size_t rw = ksk_row_words(10), pw = (size_t)ksk_pitch((int)rw), rows = ksk_rows(10),
                 per = KF_CHUNK / (rw * 4);
    PinnedBuf buf;
    CK(cudaMallocHost(&buf.p, per * rw * 4));
    for (size_t r0 = 0; r0 < rows; r0 += per) {
        const size_t m = std::min(per, rows - r0);
        CK(cudaMemcpy2D(buf.p, rw * 4, ctx->ksk[0] + r0 * pw, pw * 4, rw * 4, m, cudaMemcpyDeviceToHost));
        if (fwrite(buf.p, 1, m * rw * 4, fc.f) != m * rw * 4)
            return fail(CUFHEDB_ERR_ARG, "short write (key-switching key)");
    }
    if (fflush(fc.f) != 0) return fail(CUFHEDB_ERR_ARG, "flush failed");
    return CUFHEDB_OK;
}

int cufhedb_keygen(cufhedb_ctx *ctx, uint64_t seed, unsigned flags)
{
    NEED(ctx != nullptr, "ctx is null");
    NEED((flags & ~31u) == 0, "unknown keygen flag");
    DeviceGuard g(ctx->device);
    std::vector<uint32_t> s0(N0), s1(N1);
    std::vector<uint64_t> s2(N2);
    host_secret_keys(seed, s0.data(), s1.data(), s2.data());
    int rc = ensure_alloc((void **)&ctx->s0_d, N0 * 4);
    if (!rc) rc = ensure_alloc((void **)&ctx->s1_d, N1 * 4);
    if (!rc) rc = ensure_alloc((void **)&ctx->s2_d, N2 * 8);
    if (rc) return rc;
    CK(cudaMemcpy(ctx->s0_d, s0.data(), N0 * 4, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(ctx->s1_d, s1.data(), N1 * 4, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(ctx->s2_d, s2.data(), N2 * 8, cudaMemcpyHostToDevice));
    ctx->have_sk = true;

    if (flags & CUFHEDB_GEN_BK01) {
        std::vector<int> pos;
        for (int i = 0; i < N1; ++i)
            if (s1[i]) pos.push_back(i);
        int *pos_d = nullptr;
        CK(cudaMalloc((void **)&pos_d, pos.size() * sizeof(int)));
        cudaError_t e = cudaMemcpy(pos_d, pos.data(), pos.size() * sizeof(int), cudaMemcpyHostToDevice);
        rc = ensure_alloc((void **)&ctx->bk01_int, BK01_WORDS * sizeof(uint32_t));
        if (!rc) rc = ensure_alloc((void **)&ctx->bk01, BK01_ROWS * 1024 * sizeof(double2));
        if (rc) {
            cudaFree(pos_d);
            return rc;
        }
        if (e == cudaSuccess) e = gen_bk01(ctx->bk01_int, seed, ctx->s0_d, pos_d, (int)pos.size(), 0);
        if (e == cudaSuccess) e = bk01_to_fft(ctx->bk01, ctx->bk01_int, (int)BK01_ROWS, ctx->tab512, 0);
        if (e == cudaSuccess) e = cudaDeviceSynchronize();
        cudaFree(pos_d);
        if (e != cudaSuccess) return cuda_fail(e, "keygen bk01");
        rc = prepare_split01(ctx);
        if (rc) return rc;
    }
    if (flags & CUFHEDB_GEN_BK02) {
        std::vector<int> pos;
        for (int i = 0; i < N2; ++i)
            if (s2[i]) pos.push_back(i);
        int *pos_d = nullptr;
        CK(cudaMalloc((void **)&pos_d, pos.size() * sizeof(int)));
        cudaError_t e = cudaMemcpy(pos_d, pos.data(), pos.size() * sizeof(int), cudaMemcpyHostToDevice);
        rc = ensure_alloc((void **)&ctx->bk02_int, BK02_WORDS * sizeof(uint64_t));
        if (!rc) rc = ensure_alloc((void **)&ctx->bk02, BK02_ROWS * 2 * 1024 * sizeof(double2));
        if (rc) {
            cudaFree(pos_d);
            return rc;
        }
        if (e == cudaSuccess) e = gen_bk02(ctx->bk02_int, seed, ctx->s0_d, pos_d, (int)pos.size(), 0);
        if (e == cudaSuccess) e = bk02_to_fft(ctx->bk02, ctx->bk02_int, (int)BK02_ROWS, ctx->tab1024, 0);
        if (e == cudaSuccess) e = cudaDeviceSynchronize();
        cudaFree(pos_d);
        if (e != cudaSuccess) return cuda_fail(e, "keygen bk02");
    }
    const int kinds[3] = {10, 20, 21};
    const unsigned kflags[3] = {CUFHEDB_GEN_KSK10, CUFHEDB_GEN_KSK20, CUFHEDB_GEN_KSK21};
    for (int t = 0; t < 3; ++t) {
        if (!(flags & kflags[t])) continue;
        rc = ensure_alloc((void **)&ctx->ksk[t], ksk_dev_bytes(kinds[t]));
        if (rc) return rc;
        const void *dom = kinds[t] == 10 ? (const void *)ctx->s1_d : (const void *)ctx->s2_d;
        const uint32_t *tgt = kinds[t] == 21 ? ctx->s1_d : ctx->s0_d;
        CK(gen_ksk(ctx->ksk[t], kinds[t], seed, dom, tgt, 0));
        CK(cudaDeviceSynchronize());
    }
    return CUFHEDB_OK;
}

int cufhedb_export_bk_lvl01(cufhedb_ctx *ctx, uint32_t *bk)
{
    NEED(ctx && bk, "null argument");
    if (!ctx->bk01_int) return fail(CUFHEDB_ERR_NOKEY, "no integer lvl01 key on the device");
    DeviceGuard g(ctx->device);
    CK(cudaMemcpy(bk, ctx->bk01_int, BK01_WORDS * sizeof(uint32_t), cudaMemcpyDeviceToHost));
    return CUFHEDB_OK;
}

int cufhedb_load_bk_lvl02(cufhedb_ctx *ctx, const uint64_t *bk)
{
    NEED(ctx && bk, "null argument");
    DeviceGuard g(ctx->device);
    int rc = ensure_alloc((void **)&ctx->bk02, BK02_ROWS * 2 * 1024 * sizeof(double2));
    if (!rc) rc = ensure_alloc((void **)&ctx->bk02_int, BK02_WORDS * sizeof(uint64_t));
    if (rc) return rc;
    CK(cudaMemcpy(ctx->bk02_int, bk, BK02_WORDS * sizeof(uint64_t), cudaMemcpyHostToDevice));
    CK(bk02_to_fft(ctx->bk02, ctx->bk02_int, (int)BK02_ROWS, ctx->tab1024, 0));
    CK(cudaDeviceSynchronize());
    return CUFHEDB_OK;
}

int cufhedb_load_bkfft_lvl02(cufhedb_ctx *ctx, const double *bkfft)
{
    NEED(ctx && bkfft, "null argument");
    DeviceGuard g(ctx->device);
    int rc = ensure_alloc((void **)&ctx->bk02, BK02_ROWS * 2 * 1024 * sizeof(double2));
    if (rc) return rc;
    double *tmp = nullptr;
    CK(cudaMalloc((void **)&tmp, BK02_WORDS * sizeof(double)));
    cudaError_t e = cudaMemcpy(tmp, bkfft, BK02_WORDS * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = bkfft02_permute(ctx->bk02, tmp, (int)BK02_ROWS, 0);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    cudaFree(tmp);
    if (e != cudaSuccess) return cuda_fail(e, "load_bkfft_lvl02");
    return CUFHEDB_OK;
}

int cufhedb_export_bk_lvl02(cufhedb_ctx *ctx, uint64_t *bk)
{
    NEED(ctx && bk, "null argument");
    if (!ctx->bk02_int) return fail(CUFHEDB_ERR_NOKEY, "no integer lvl02 key on the device");
    DeviceGuard g(ctx->device);
    CK(cudaMemcpy(bk, ctx->bk02_int, BK02_WORDS * sizeof(uint64_t), cudaMemcpyDeviceToHost));
    return CUFHEDB_OK;
}

int cufhedb_export_ksk_rows(cufhedb_ctx *ctx, int kind, const uint64_t *rows, int n, uint32_t *out)
{
    NEED(ctx && rows && out && n >= 0, "bad argument");
    const int slot = ksk_slot(kind);
    NEED(slot >= 0, "unknown key-switching key kind");
    if (!ctx->ksk[slot]) return fail(CUFHEDB_ERR_NOKEY, "key-switching key not loaded");
    DeviceGuard g(ctx->device);
    const size_t width = ksk_row_words(kind), pitch = (size_t)ksk_pitch((int)width);
    const size_t nrows = ksk_rows(kind);
    for (int r = 0; r < n; ++r) {
        NEED(rows[r] < nrows, "row index out of range");
        CK(cudaMemcpy(out + r * width, ctx->ksk[slot] + rows[r] * pitch, width * 4, cudaMemcpyDeviceToHost));
    }
    return CUFHEDB_OK;
}

int cufhedb_encrypt_lvl1(cufhedb_ctx *ctx, uint64_t seed, uint64_t stream_id, uint64_t idx0, const uint32_t *msg,
                         uint32_t *out, int B, cufhedb_stream_t stream)
{
    NEED(aligned_to(msg, 4), "msg must be 4-byte aligned");
    NEED(aligned_to(out, 4), "out must be 4-byte aligned");
    NEED(ctx && msg && out && B >= 0, "bad argument");
    if (!ctx->have_sk) return fail(CUFHEDB_ERR_NOKEY, "no deterministic key set (call cufhedb_keygen)");
    DeviceGuard g(ctx->device);
    CK(encrypt_tlwe32(out, msg, B, N1, ctx->s1_d, NS_LVL1, seed, stream_id, idx0, (cudaStream_t)stream));
    return CUFHEDB_OK;
}

int cufhedb_encrypt_lvl2(cufhedb_ctx *ctx, uint64_t seed, uint64_t stream_id, uint64_t idx0, const uint64_t *msg,
                         uint64_t *out, int B, cufhedb_stream_t stream)
{
    NEED(aligned_to(msg, 8), "msg must be 8-byte aligned");
    NEED(aligned_to(out, 8), "out must be 8-byte aligned");
    NEED(ctx && msg && out && B >= 0, "bad argument");
    if (!ctx->have_sk) return fail(CUFHEDB_ERR_NOKEY, "no deterministic key set (call cufhedb_keygen)");
    DeviceGuard g(ctx->device);
    CK(encrypt_tlwe64(out, msg, B, N2, ctx->s2_d, NS_LVL2, seed, stream_id, idx0, (cudaStream_t)stream));
    return CUFHEDB_OK;
}

int cufhedb_phase_lvl1(cufhedb_ctx *ctx, const uint32_t *ct, const uint32_t *key, uint32_t *phase, int B,
                       cufhedb_stream_t stream)
{
    NEED(aligned_to(ct, 4), "ct must be 4-byte aligned");
    NEED(aligned_to(key, 4), "key must be 4-byte aligned");
    NEED(aligned_to(phase, 4), "phase must be 4-byte aligned");
    NEED(ctx && ct && phase && B >= 0, "bad argument");
    if (!key && !ctx->have_sk) return fail(CUFHEDB_ERR_NOKEY, "no key given and no deterministic key set");
    DeviceGuard g(ctx->device);
    CK(tlwe_phase32(phase, ct, B, N1, key ? key : ctx->s1_d, (cudaStream_t)stream));
    return CUFHEDB_OK;
}

int cufhedb_phase_lvl2(cufhedb_ctx *ctx, const uint64_t *ct, const uint64_t *key, uint64_t *phase, int B,
                       cufhedb_stream_t stream)
{
    NEED(aligned_to(ct, 8), "ct must be 8-byte aligned");
    NEED(aligned_to(key, 8), "key must be 8-byte aligned");
    NEED(aligned_to(phase, 8), "phase must be 8-byte aligned");
    NEED(ctx && ct && phase && B >= 0, "bad argument");
    if (!key && !ctx->have_sk) return fail(CUFHEDB_ERR_NOKEY, "no key given and no deterministic key set");
    DeviceGuard g(ctx->device);
    CK(tlwe_phase64(phase, ct, B, N2, key ? key : ctx->s2_d, (cudaStream_t)stream));
    return CUFHEDB_OK;
}

// ---- batched operations --------------------------------------------------

int cufhedb_pbs_lvl01(cufhedb_ctx *ctx, const uint32_t *in_lvl0, uint32_t *out_lvl1, int B,
                      const cufhedb_testvec *tv, int precision, cufhedb_stream_t stream)
{
    NEED(aligned_to(in_lvl0, 4), "in_lvl0 must be 4-byte aligned");
    NEED(aligned_to(out_lvl1, 4), "out_lvl1 must be 4-byte aligned");
    NEED(aligned_to(tv && tv->kind == CUFHEDB_TV_POLY ? tv->poly : nullptr, 4), "poly : nullptr must be 4-byte aligned");
    NEED(ctx != nullptr, "ctx is null");
    NEED(B >= 0, "negative batch");
    if (B == 0) return CUFHEDB_OK;
    NEED(in_lvl0 && out_lvl1, "null buffer");
    int rc = check_tv(tv, N1);
    if (rc) return rc;
    DeviceGuard g(ctx->device);
    return pbs01_enqueue(ctx, in_lvl0, out_lvl1, B, tv, precision, (cudaStream_t)stream);
}

// One full pass (w ciphertexts on every SM) of each launch shape of a PBS
// kernel over uniform random lvl0 inputs: the best of two timed runs after
// one warm-up run.  level 1: precision FP64 or split; level 2: FP64.
static int autotune_level(cufhedb_ctx *ctx, int level, int precision, float out_ms[NSHAPES])
{
    const int *shapes = level == 1 ? PBS01_SHAPES : PBS02_SHAPES;
    int wmax = 0;
    for (int i = 0; i < NSHAPES; ++i) wmax = std::max(wmax, shapes[i]);
    const int Bmax = wmax * ctx->num_sms;
    const size_t out_words = (size_t)Bmax * (level == 1 ? (N1 + 1) : 2 * (N2 + 1));
    uint32_t *in = nullptr, *out = nullptr;
    cudaStream_t st = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int rc = CUFHEDB_OK;
    cudaError_t e = cudaMalloc((void **)&in, (size_t)Bmax * (N0 + 1) * 4);
    if (e == cudaSuccess) e = cudaMalloc((void **)&out, out_words * 4);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    if (e == cudaSuccess) e = fill_random32(in, (size_t)Bmax * (N0 + 1), 0x7A5E, 1, st);
    if (e != cudaSuccess) rc = cuda_fail(e, "autotune setup");
    for (int i = 0; i < NSHAPES && rc == CUFHEDB_OK; ++i) {
        const int w = shapes[i];
        float t_best = 0.0f;
        for (int it = 0; it < 3 && rc == CUFHEDB_OK; ++it) {
            e = cudaEventRecord(e0, st);
            if (e == cudaSuccess) {
                if (level == 1) {
                    const cufhedb_testvec tv{CUFHEDB_TV_CONST, 0, 1u << 29, nullptr};
                    Pbs01Args a{};
                    a.in = in;
                    a.out = out;
                    a.B = w * ctx->num_sms;
                    a.tv = to_tv(&tv);
                    a.err = ctx->err;
                    if (precision == CUFHEDB_FP64) {
                        a.bk = ctx->bk01;
                        a.tables = ctx->tab512;
                        e = launch_pbs01_f64(a, ctx->num_sms, w, st);
                    } else {
                        a.bk = reinterpret_cast<const double2 *>(ctx->bk01_split);
                        a.tables = ctx->tab512f;
                        e = precision == CUFHEDB_SPLIT32_TC ? launch_pbs01_split_tc(a, ctx->num_sms, w, st)
                                                            : launch_pbs01_split(a, ctx->num_sms, w, st);
                    }
                } else {
                    const cufhedb_testvec tv{CUFHEDB_TV_CONST, 0, 1ull << 61, nullptr};
                    Pbs02Args a{};
                    a.in = in;
                    a.out = reinterpret_cast<uint64_t *>(out);
                    a.B = w * ctx->num_sms;
                    a.bk = ctx->bk02;
                    a.tables = ctx->tab1024;
                    a.tv = to_tv(&tv);
                    a.err = ctx->err;
                    e = launch_pbs02_f64(a, ctx->num_sms, w, st);
                }
            }
            if (e == cudaSuccess) e = cudaEventRecord(e1, st);
            if (e == cudaSuccess) e = cudaEventSynchronize(e1);
            float ms = 0.0f;
            if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
            if (e != cudaSuccess) rc = cuda_fail(e, "autotune run");
            else if (it > 0 && (t_best == 0.0f || ms < t_best)) t_best = ms;   // the first run warms up
        }
        out_ms[i] = t_best;
    }
    if (rc == CUFHEDB_OK) rc = cufhedb_sync(ctx, st);
    if (st) cudaStreamDestroy(st);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(in);
    cudaFree(out);
    return rc;
}

int cufhedb_autotune_pbs01(cufhedb_ctx *ctx, int precision, float *ms_w7, float *ms_w8)
{
    NEED(ctx != nullptr, "ctx is null");
    NEED(valid_precision(precision), "unsupported precision");
    if (!ctx->bk01) return fail(CUFHEDB_ERR_NOKEY, "lvl01 bootstrapping key not loaded");
    if (precision != CUFHEDB_FP64 && !ctx->bk01_split)
        return fail(CUFHEDB_ERR_NOKEY, "split-precision lvl01 key not prepared");
    DeviceGuard g(ctx->device);
    float ms[NSHAPES];
    const int rc = autotune_level(ctx, 1, precision, ms);
    if (rc != CUFHEDB_OK) return rc;
    for (int i = 0; i < NSHAPES; ++i) ctx->pbs01_pass_ms[precision][i] = ms[i];
    if (ms_w7) *ms_w7 = ms[0];
    if (ms_w8) *ms_w8 = ms[1];
    return CUFHEDB_OK;
}

int cufhedb_autotune_pbs02(cufhedb_ctx *ctx, float *ms)
{
    NEED(ctx != nullptr, "ctx is null");
    if (!ctx->bk02) return fail(CUFHEDB_ERR_NOKEY, "lvl02 bootstrapping key not loaded");
    DeviceGuard g(ctx->device);
    float t[NSHAPES];
    const int rc = autotune_level(ctx, 2, CUFHEDB_FP64, t);
    if (rc != CUFHEDB_OK) return rc;
    for (int i = 0; i < NSHAPES; ++i) {
        ctx->pbs02_pass_ms[i] = t[i];
        if (ms) ms[i] = t[i];
    }
    return CUFHEDB_OK;
}

static float *shape_table(cufhedb_ctx *ctx, int level, int precision)
{
    if (level == 1 && valid_precision(precision)) return ctx->pbs01_pass_ms[precision];
    if (level == 2 && precision == CUFHEDB_FP64) return ctx->pbs02_pass_ms;
    return nullptr;
}

int cufhedb_autotune_table(cufhedb_ctx *ctx, int level, int precision, int *shapes, float *pass_ms)
{
    NEED(ctx != nullptr, "ctx is null");
    const float *t = shape_table(ctx, level, precision);
    NEED(t != nullptr, "no launch shapes for this level and precision");
    for (int i = 0; i < NSHAPES; ++i) {
        if (shapes) shapes[i] = level == 1 ? PBS01_SHAPES[i] : PBS02_SHAPES[i];
        if (pass_ms) pass_ms[i] = t[i];
    }
    return NSHAPES;
}

int cufhedb_launch_shape(cufhedb_ctx *ctx, int level, int precision, int B, int *shape)
{
    NEED(ctx != nullptr && shape != nullptr, "null argument");
    const float *t = shape_table(ctx, level, precision);
    NEED(t != nullptr && B > 0, "bad level, precision or batch");
    if (level == 1 && precision == CUFHEDB_SPLIT32)
        *shape = pbs01_split_choose(B, ctx->num_sms, t, ctx->pbs01_pass_ms[CUFHEDB_SPLIT32_TC]).w;
    else
        *shape = level == 1 ? pbs01_choose_w(B, ctx->num_sms, t) : pbs02_choose_p(B, ctx->num_sms, t);
    return CUFHEDB_OK;
}

int cufhedb_launch_layout(cufhedb_ctx *ctx, int B, int *tensor_core_stage1)
{
    NEED(ctx != nullptr && tensor_core_stage1 != nullptr && B > 0, "bad argument");
    *tensor_core_stage1 = pbs01_split_choose(B, ctx->num_sms, ctx->pbs01_pass_ms[CUFHEDB_SPLIT32],
                                             ctx->pbs01_pass_ms[CUFHEDB_SPLIT32_TC])
                              .tc
                              ? 1
                              : 0;
    return CUFHEDB_OK;
}

// A table is valid for one device model, SM count and parameter set: the
// hash covers the parameters the kernels are compiled for and the shape lists.
static uint64_t param_hash()
{
    char buf[160];
    std::snprintf(buf, sizeof buf, "n0=%d n1=%d l1=%d bg1=%d n2=%d l2=%d bg2=%d s1=%d,%d,%d s2=%d,%d,%d", N0, N1, L1,
                  BGBIT1, N2, L2, BGBIT2, PBS01_SHAPES[0], PBS01_SHAPES[1], PBS01_SHAPES[2], PBS02_SHAPES[0],
                  PBS02_SHAPES[1], PBS02_SHAPES[2]);
    uint64_t h = 1469598103934665603ull;   // FNV-1a
    for (const char *c = buf; *c; ++c) h = (h ^ (unsigned char)*c) * 1099511628211ull;
    return h;
}

static std::string device_tag(int device)
{
    cudaDeviceProp prop;
    std::string name = cudaGetDeviceProperties(&prop, device) == cudaSuccess ? prop.name : "unknown";
    for (char &c : name)
        if (c == ' ') c = '_';
    return name;
}

int cufhedb_autotune_save(cufhedb_ctx *ctx, const char *path)
{
    NEED(ctx && path, "null argument");
    FILE *f = std::fopen(path, "w");
    if (!f) return fail(CUFHEDB_ERR_ARG, std::string("cannot write ") + path);
    std::fprintf(f, "cufhedb_b200 autotune 1\ndevice %s sms %d params %016llx\n", device_tag(ctx->device).c_str(),
                 ctx->num_sms, (unsigned long long)param_hash());
    const char *names[3] = {"fp64", "split32", "split32tc"};
    for (int p = 0; p < 3; ++p) {
        std::fprintf(f, "pbs01 %s", names[p]);
        for (int i = 0; i < NSHAPES; ++i) std::fprintf(f, " %d %.6f", PBS01_SHAPES[i], ctx->pbs01_pass_ms[p][i]);
        std::fprintf(f, "\n");
    }
    std::fprintf(f, "pbs02 fp64");
    for (int i = 0; i < NSHAPES; ++i) std::fprintf(f, " %d %.6f", PBS02_SHAPES[i], ctx->pbs02_pass_ms[i]);
    std::fprintf(f, "\n");
    const bool ok = std::fclose(f) == 0;
    return ok ? CUFHEDB_OK : fail(CUFHEDB_ERR_ARG, std::string("cannot write ") + path);
}

int cufhedb_autotune_load(cufhedb_ctx *ctx, const char *path)
{
    NEED(ctx && path, "null argument");
    FILE *f = std::fopen(path, "r");
    if (!f) return fail(CUFHEDB_ERR_ARG, std::string("cannot read ") + path);
    char dev[256] = {0}, kind[16] = {0}, prec[16] = {0};
    int version = 0, sms = 0;
    unsigned long long hash = 0;
    bool ok = std::fscanf(f, "cufhedb_b200 autotune %d device %255s sms %d params %llx", &version, dev, &sms,
                          &hash) == 4 &&
              version == 1;
    const bool same = ok && device_tag(ctx->device) == dev && sms == ctx->num_sms && hash == param_hash();
    float t01[3][NSHAPES], t02[NSHAPES];
    int seen = 0;
    while (same && std::fscanf(f, "%15s %15s", kind, prec) == 2) {
        float *dst = nullptr;
        const int *shapes = nullptr;
        int bit = 0;
        if (!std::strcmp(kind, "pbs01") && !std::strcmp(prec, "fp64")) dst = t01[0], shapes = PBS01_SHAPES, bit = 1;
        else if (!std::strcmp(kind, "pbs01") && !std::strcmp(prec, "split32")) dst = t01[1], shapes = PBS01_SHAPES, bit = 2;
        else if (!std::strcmp(kind, "pbs01") && !std::strcmp(prec, "split32tc"))
            dst = t01[2], shapes = PBS01_SHAPES, bit = 4;
        else if (!std::strcmp(kind, "pbs02") && !std::strcmp(prec, "fp64")) dst = t02, shapes = PBS02_SHAPES, bit = 8;
        if (!dst) {
            ok = false;
            break;
        }
        for (int i = 0; i < NSHAPES && ok; ++i) {
            int w = 0;
            ok = std::fscanf(f, "%d %f", &w, &dst[i]) == 2 && w == shapes[i] && dst[i] > 0.0f;
        }
        seen |= bit;
    }
    std::fclose(f);
    if (!same) return fail(CUFHEDB_ERR_ARG, "autotune table is for another device, SM count or parameter set");
    if (!ok || seen != 15) return fail(CUFHEDB_ERR_ARG, "malformed autotune table");
    for (int i = 0; i < NSHAPES; ++i) {
        for (int p = 0; p < 3; ++p) ctx->pbs01_pass_ms[p][i] = t01[p][i];
        ctx->pbs02_pass_ms[i] = t02[i];
    }
    return CUFHEDB_OK;
}

int cufhedb_iks(cufhedb_ctx *ctx, int kind, const void *in, uint32_t *out, int B, cufhedb_stream_t stream)
{
    NEED(aligned_to(in, kind == 10 ? 4 : 8), "in must be 4-byte (kind 10) or 8-byte (kinds 20, 21) aligned");
    NEED(aligned_to(out, 4), "out must be 4-byte aligned");
    NEED(ctx != nullptr, "ctx is null");
    const int slot = ksk_slot(kind);
    NEED(slot >= 0, "unknown key-switching kind");
    NEED(B >= 0, "negative batch");
    if (B == 0) return CUFHEDB_OK;
    NEED(in && out, "null buffer");
    if (!ctx->ksk[slot]) return fail(CUFHEDB_ERR_NOKEY, "key-switching key not loaded");
    DeviceGuard g(ctx->device);
    IksArgs a{};
    if (kind == 10) a.in32 = (const uint32_t *)in;
    else a.in64 = (const uint64_t *)in;
    a.sa = 1;
    a.out = out;
    a.ksk = ctx->ksk[slot];
    a.B = B;
    CK(launch_iks(a, kind, (cudaStream_t)stream));
    return CUFHEDB_OK;
}

int cufhedb_gate_lvl1(cufhedb_ctx *ctx, int gate, const uint32_t *ca, const uint32_t *cb, uint32_t *out, int B,
                      int precision, cufhedb_stream_t stream)
{
    NEED(aligned_to(ca, 4), "ca must be 4-byte aligned");
    NEED(aligned_to(cb, 4), "cb must be 4-byte aligned");
    NEED(aligned_to(out, 4), "out must be 4-byte aligned");
    NEED(ctx != nullptr, "ctx is null");
    NEED(B >= 0, "negative batch");
    if (B == 0) return CUFHEDB_OK;
    NEED(ca && cb && out, "null buffer");
    DeviceGuard g(ctx->device);
    return gate_enqueue(ctx, gate, ca, cb, out, B, precision, (cudaStream_t)stream);
}

int cufhedb_twist_ifft_lvl1(cufhedb_ctx *ctx, const uint32_t *in, double *out, int B, cufhedb_stream_t stream)
{
    NEED(aligned_to(in, 4), "in must be 4-byte aligned");
    NEED(aligned_to(out, 8), "out must be 8-byte aligned");
    NEED(ctx && B >= 0, "bad argument");
    if (B == 0) return CUFHEDB_OK;
    NEED(in && out, "null buffer");
    DeviceGuard g(ctx->device);
    CK(launch_twist_ifft1(out, in, B, ctx->tab512, (cudaStream_t)stream));
    return CUFHEDB_OK;
}

int cufhedb_twist_fft_lvl1(cufhedb_ctx *ctx, const double *in, uint32_t *out, int B, cufhedb_stream_t stream)
{
    NEED(aligned_to(in, 8), "in must be 8-byte aligned");
    NEED(aligned_to(out, 4), "out must be 4-byte aligned");
    NEED(ctx && B >= 0, "bad argument");
    if (B == 0) return CUFHEDB_OK;
    NEED(in && out, "null buffer");
    DeviceGuard g(ctx->device);
    CK(launch_twist_fft1(out, in, B, ctx->tab512, (cudaStream_t)stream));
    return CUFHEDB_OK;
}

int cufhedb_trgsw_prepare_lvl1(cufhedb_ctx *ctx, const uint32_t *trgsw, void *out, int B, int precision,
                               cufhedb_stream_t stream)
{
    NEED(aligned_to(trgsw, 4), "trgsw must be 4-byte aligned");
    NEED(aligned_to(out, 16), "out must be 16-byte aligned");
    NEED(ctx && B >= 0, "bad argument");
    if (B == 0) return CUFHEDB_OK;
    NEED(trgsw && out, "null buffer");
    NEED(valid_precision(precision), "unsupported precision");
    DeviceGuard g(ctx->device);
    const int rows = B * 2 * L1;
    if (precision == CUFHEDB_FP64)
        CK(bk01_to_fft((double2 *)out, trgsw, rows, ctx->tab512, (cudaStream_t)stream));
    else
        CK(bk01_to_split((float4 *)out, trgsw, rows, ctx->tab512, (cudaStream_t)stream));
    return CUFHEDB_OK;
}

int cufhedb_trgswfft_prepare_lvl1(cufhedb_ctx *ctx, const double *trgswfft, void *out, int B,
                                  cufhedb_stream_t stream)
{
    NEED(aligned_to(trgswfft, 8), "trgswfft must be 8-byte aligned");
    NEED(aligned_to(out, 16), "out must be 16-byte aligned");
    NEED(ctx && B >= 0, "bad argument");
    if (B == 0) return CUFHEDB_OK;
    NEED(trgswfft && out, "null buffer");
    DeviceGuard g(ctx->device);
    CK(bkfft01_permute((double2 *)out, trgswfft, B * 2 * L1, (cudaStream_t)stream));
    return CUFHEDB_OK;
}

int cufhedb_extprod_lvl1(cufhedb_ctx *ctx, const uint32_t *trlwe, const void *trgsw, uint32_t *out, int B,
                         int shared, int precision, cufhedb_stream_t stream)
{
    NEED(aligned_to(trlwe, 4), "trlwe must be 4-byte aligned");
    NEED(aligned_to(trgsw, 16), "trgsw must be 16-byte aligned");
    NEED(aligned_to(out, 4), "out must be 4-byte aligned");
    NEED(ctx && B >= 0, "bad argument");
    if (B == 0) return CUFHEDB_OK;
    NEED(trlwe && trgsw && out, "null buffer");
    NEED(valid_precision(precision), "unsupported precision");
    DeviceGuard g(ctx->device);
    ExtProdArgs a{};
    a.trlwe = trlwe;
    a.trgsw = trgsw;
    a.out = out;
    a.B = B;
    a.shared = shared ? 1 : 0;
    a.tables = precision == CUFHEDB_FP64 ? (const void *)ctx->tab512 : (const void *)ctx->tab512f;
    a.err = ctx->err;
    CK(launch_extprod1(a, precision == CUFHEDB_FP64 ? 0 : 1, (cudaStream_t)stream));
    return CUFHEDB_OK;
}

static int pbs02_enqueue(cufhedb_ctx *ctx, const uint32_t *in, uint64_t *out, int B, const cufhedb_testvec *tv,
                         cudaStream_t st)
{
    if (!ctx->bk02) return fail(CUFHEDB_ERR_NOKEY, "lvl02 bootstrapping key not loaded");
    Pbs02Args a{};
    a.in = in;
    a.out = out;
    a.B = B;
    a.bk = ctx->bk02;
    a.tables = ctx->tab1024;
    a.tv = to_tv(tv);
    a.err = ctx->err;
    CK(launch_pbs02_f64(a, ctx->num_sms, pbs02_choose_p(B, ctx->num_sms, ctx->pbs02_pass_ms), st));
    return CUFHEDB_OK;
}

int cufhedb_pbs_lvl02(cufhedb_ctx *ctx, const uint32_t *in_lvl0, uint64_t *out_lvl2, int B, const cufhedb_testvec *tv,
                      cufhedb_stream_t stream)
{
    NEED(aligned_to(in_lvl0, 4), "in_lvl0 must be 4-byte aligned");
    NEED(aligned_to(out_lvl2, 8), "out_lvl2 must be 8-byte aligned");
    NEED(aligned_to(tv && tv->kind == CUFHEDB_TV_POLY ? tv->poly : nullptr, 8), "poly : nullptr must be 8-byte aligned");
    NEED(ctx != nullptr, "ctx is null");
    NEED(B >= 0, "negative batch");
    if (B == 0) return CUFHEDB_OK;
    NEED(in_lvl0 && out_lvl2, "null buffer");
    int rc = check_tv(tv, N2);
    if (rc) return rc;
    DeviceGuard g(ctx->device);
    return pbs02_enqueue(ctx, in_lvl0, out_lvl2, B, tv, (cudaStream_t)stream);
}

int cufhedb_trgsw_prepare_lvl2(cufhedb_ctx *ctx, const uint64_t *trgsw, void *out, int B, cufhedb_stream_t stream)
{
    NEED(aligned_to(trgsw, 8), "trgsw must be 8-byte aligned");
    NEED(aligned_to(out, 16), "out must be 16-byte aligned");
    NEED(ctx && B >= 0, "bad argument");
    if (B == 0) return CUFHEDB_OK;
    NEED(trgsw && out, "null buffer");
    DeviceGuard g(ctx->device);
    CK(bk02_to_fft((double2 *)out, trgsw, B * 2 * L2, ctx->tab1024, (cudaStream_t)stream));
    return CUFHEDB_OK;
}

int cufhedb_trgswfft_prepare_lvl2(cufhedb_ctx *ctx, const double *trgswfft, void *out, int B,
                                  cufhedb_stream_t stream)
{
    NEED(aligned_to(trgswfft, 8), "trgswfft must be 8-byte aligned");
    NEED(aligned_to(out, 16), "out must be 16-byte aligned");
    NEED(ctx && B >= 0, "bad argument");
    if (B == 0) return CUFHEDB_OK;
    NEED(trgswfft && out, "null buffer");
    DeviceGuard g(ctx->device);
    CK(bkfft02_permute((double2 *)out, trgswfft, B * 2 * L2, (cudaStream_t)stream));
    return CUFHEDB_OK;
}

int cufhedb_extprod_lvl2(cufhedb_ctx *ctx, const uint64_t *trlwe, const void *trgsw, uint64_t *out, int B,
                         int shared, cufhedb_stream_t stream)
{
    NEED(aligned_to(trlwe, 8), "trlwe must be 8-byte aligned");
    NEED(aligned_to(trgsw, 16), "trgsw must be 16-byte aligned");
    NEED(aligned_to(out, 8), "out must be 8-byte aligned");
    NEED(ctx && B >= 0, "bad argument");
    if (B == 0) return CUFHEDB_OK;
    NEED(trlwe && trgsw && out, "null buffer");
    DeviceGuard g(ctx->device);
    ExtProd2Args a{};
    a.trlwe = trlwe;
    a.trgsw = (const double2 *)trgsw;
    a.out = out;
    a.B = B;
    a.shared = shared ? 1 : 0;
    a.tables = ctx->tab1024;
    CK(launch_extprod2(a, (cudaStream_t)stream));
    return CUFHEDB_OK;
}

int cufhedb_twist_ifft_lvl2(cufhedb_ctx *ctx, const uint64_t *in, double *out, int B, cufhedb_stream_t stream)
{
    NEED(aligned_to(in, 8), "in must be 8-byte aligned");
    NEED(aligned_to(out, 8), "out must be 8-byte aligned");
    NEED(ctx && B >= 0, "bad argument");
    if (B == 0) return CUFHEDB_OK;
    NEED(in && out, "null buffer");
    DeviceGuard g(ctx->device);
    CK(launch_twist_ifft2(out, in, B, ctx->tab1024, (cudaStream_t)stream));
    return CUFHEDB_OK;
}

int cufhedb_twist_fft_lvl2(cufhedb_ctx *ctx, const double *in, uint64_t *out, int B, cufhedb_stream_t stream)
{
    NEED(aligned_to(in, 8), "in must be 8-byte aligned");
    NEED(aligned_to(out, 8), "out must be 8-byte aligned");
    NEED(ctx && B >= 0, "bad argument");
    if (B == 0) return CUFHEDB_OK;
    NEED(in && out, "null buffer");
    DeviceGuard g(ctx->device);
    CK(launch_twist_fft2(out, in, B, ctx->tab1024, (cudaStream_t)stream));
    return CUFHEDB_OK;
}

// ---- host-buffer entry points ----------------------------------------------

int cufhedb_pbs_lvl01_host(cufhedb_ctx *ctx, const uint32_t *in_lvl0, uint32_t *out_lvl1, int B,
                           const cufhedb_testvec *tv, int precision)
{
    NEED(ctx != nullptr, "ctx is null");
    NEED(B >= 0, "negative batch");
    if (B == 0) return CUFHEDB_OK;
    NEED(in_lvl0 && out_lvl1, "null buffer");
    int rc = check_tv(tv, N1);
    if (rc) return rc;
    DeviceGuard g(ctx->device);
    std::lock_guard<std::mutex> lk(ctx->io_mu);
    cudaStream_t st = ctx->io;
    const size_t ib = (size_t)B * (N0 + 1) * 4, ob = (size_t)B * (N1 + 1) * 4;
    uint32_t *din = nullptr, *dout = nullptr;
    CK(cudaMallocAsync((void **)&din, ib, st));
    CK(cudaMallocAsync((void **)&dout, ob, st));
    cudaError_t e = cudaMemcpyAsync(din, in_lvl0, ib, cudaMemcpyHostToDevice, st);
    rc = (e == cudaSuccess) ? pbs01_enqueue(ctx, din, dout, B, tv, precision, st) : cuda_fail(e, "h2d");
    if (rc == CUFHEDB_OK) {
        e = cudaMemcpyAsync(out_lvl1, dout, ob, cudaMemcpyDeviceToHost, st);
        if (e != cudaSuccess) rc = cuda_fail(e, "d2h");
    }
    cudaFreeAsync(din, st);
    cudaFreeAsync(dout, st);
    if (rc != CUFHEDB_OK) {
        cudaStreamSynchronize(st);
        return rc;
    }
    return cufhedb_sync(ctx, st);
}

int cufhedb_extprod_lvl1_host(cufhedb_ctx *ctx, const uint32_t *trlwe, const double *trgswfft, uint32_t *out, int B,
                              int shared)
{
    NEED(ctx != nullptr, "ctx is null");
    NEED(B >= 0, "negative batch");
    if (B == 0) return CUFHEDB_OK;
    NEED(trlwe && trgswfft && out, "null buffer");
    DeviceGuard g(ctx->device);
    std::lock_guard<std::mutex> lk(ctx->io_mu);
    cudaStream_t st = ctx->io;
    const int ng = shared ? 1 : B;
    const size_t tb = (size_t)B * 2 * N1 * 4, gb = (size_t)ng * 2 * L1 * 2 * N1 * 8;
    char *buf = nullptr;
    CK(cudaMallocAsync((void **)&buf, 2 * tb + 2 * gb, st));
    uint32_t *din = (uint32_t *)buf, *dout = (uint32_t *)(buf + tb);
    double *graw = (double *)(buf + 2 * tb);
    void *gprep = buf + 2 * tb + gb;
    int rc = CUFHEDB_OK;
    cudaError_t e = cudaMemcpyAsync(din, trlwe, tb, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(graw, trgswfft, gb, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = bkfft01_permute((double2 *)gprep, graw, ng * 2 * L1, st);
    if (e == cudaSuccess) {
        ExtProdArgs a{};
        a.trlwe = din;
        a.trgsw = gprep;
        a.out = dout;
        a.B = B;
        a.shared = shared ? 1 : 0;
        a.tables = ctx->tab512;
        a.err = ctx->err;
        e = launch_extprod1(a, 0, st);
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, dout, tb, cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) rc = cuda_fail(e, "extprod_lvl1_host");
    cudaFreeAsync(buf, st);
    if (rc != CUFHEDB_OK) {
        cudaStreamSynchronize(st);
        return rc;
    }
    return cufhedb_sync(ctx, st);
}

int cufhedb_gate_lvl1_host(cufhedb_ctx *ctx, int gate, const uint32_t *ca, const uint32_t *cb, uint32_t *out, int B,
                           int precision)
{
    NEED(ctx != nullptr, "ctx is null");
    NEED(B >= 0, "negative batch");
    if (B == 0) return CUFHEDB_OK;
    NEED(ca && cb && out, "null buffer");
    DeviceGuard g(ctx->device);
    std::lock_guard<std::mutex> lk(ctx->io_mu);
    cudaStream_t st = ctx->io;
    const size_t nb = (size_t)B * (N1 + 1) * 4;
    uint32_t *dbuf = nullptr;
    CK(cudaMallocAsync((void **)&dbuf, 3 * nb, st));
    uint32_t *da = dbuf, *db = dbuf + (size_t)B * (N1 + 1), *dout = dbuf + 2 * (size_t)B * (N1 + 1);
    int rc = CUFHEDB_OK;
    cudaError_t e = cudaMemcpyAsync(da, ca, nb, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(db, cb, nb, cudaMemcpyHostToDevice, st);
    rc = (e == cudaSuccess) ? gate_enqueue(ctx, gate, da, db, dout, B, precision, st) : cuda_fail(e, "h2d");
    if (rc == CUFHEDB_OK) {
        e = cudaMemcpyAsync(out, dout, nb, cudaMemcpyDeviceToHost, st);
        if (e != cudaSuccess) rc = cuda_fail(e, "d2h");
    }
    cudaFreeAsync(dbuf, st);
    if (rc != CUFHEDB_OK) {
        cudaStreamSynchronize(st);
        return rc;
    }
    return cufhedb_sync(ctx, st);
}

}  // extern "C"
