// Row sharding of host-buffer operator calls over several contexts, one per
// GPU (or several on one GPU).  Rows are independent in every operator of
// the path, so a column splits into contiguous slices, one per context, each
// run by its own host thread through that context's host-buffer call; no
// data crosses between devices, and nothing is exchanged but the caller's
// host buffers.  The reference binds one device only
// (src/cuHEDB/gatebootstrap_gpu.cuh:11-15).
#include <string>
#include <thread>
#include <vector>

#include "ctx.cuh"

namespace {

struct ShardResult {
    int rc = CUFHEDB_OK;
    std::string msg;
};

// runs fn(k, begin, count) for every non-empty slice of B rows over n
// shards on n host threads; the first failure is reported to the caller
template <typename F>
int run_shards(int n, int B, F &&fn)
{
    std::vector<ShardResult> res(n);
    std::vector<std::thread> th;
    for (int k = 0; k < n; ++k) {
        const int b0 = (int)((long)B * k / n), b1 = (int)((long)B * (k + 1) / n);
        if (b1 == b0) continue;
        th.emplace_back([&, k, b0, b1] {
            res[k].rc = fn(k, b0, b1 - b0);
            if (res[k].rc != CUFHEDB_OK) res[k].msg = cufhedb_last_error();
        });
    }
    for (auto &t : th) t.join();
    for (int k = 0; k < n; ++k)
        if (res[k].rc != CUFHEDB_OK)
            return cfdb::set_error(res[k].rc, ("shard " + std::to_string(k) + ": " + res[k].msg).c_str());
    return CUFHEDB_OK;
}

int check_ctxs(cufhedb_ctx *const *ctxs, int n)
{
    if (!ctxs || n < 1) return cfdb::set_error(CUFHEDB_ERR_ARG, "need at least one context");
    for (int k = 0; k < n; ++k)
        if (!ctxs[k]) return cfdb::set_error(CUFHEDB_ERR_ARG, "null context in the list");
    return CUFHEDB_OK;
}

}  // namespace

extern "C" {

CUFHEDB_API int cufhedb_compare_host(cufhedb_ctx *ctx, int op, int level, const void *c1, const void *c2,
                                     uint32_t *out_lvl1, int B, uint32_t plain_bits, int logic, int precision)
{
    if (!ctx) return cfdb::set_error(CUFHEDB_ERR_ARG, "ctx is null");
    if (B < 0) return cfdb::set_error(CUFHEDB_ERR_ARG, "negative batch");
    if (B == 0) return CUFHEDB_OK;
    if (!c1 || !c2 || !out_lvl1) return cfdb::set_error(CUFHEDB_ERR_ARG, "null buffer");
    if (level != 1 && level != 2) return cfdb::set_error(CUFHEDB_ERR_ARG, "unsupported level");
    cfdb::DeviceGuard guard;
    if (guard.set(ctx->device) != cudaSuccess) return cfdb::set_error(CUFHEDB_ERR_CUDA, "cudaSetDevice failed");
    std::lock_guard<std::mutex> lk(ctx->io_mu);
    cudaStream_t st = ctx->io;
    const size_t in_b = (size_t)B * (level == 1 ? (N1 + 1) * 4 : (N2 + 1) * 8), out_b = (size_t)B * (N1 + 1) * 4;
    auto up = [](size_t b) { return (b + 255) & ~(size_t)255; };
    unsigned char *d = nullptr;
    cudaError_t e = cudaMallocAsync((void **)&d, 2 * up(in_b) + out_b, st);
    if (e != cudaSuccess) return cfdb::cuda_error(e, "compare_host staging");
    unsigned char *d1 = d, *d2 = d + up(in_b);
    uint32_t *dout = reinterpret_cast<uint32_t *>(d + 2 * up(in_b));
    int rc = CUFHEDB_OK;
    e = cudaMemcpyAsync(d1, c1, in_b, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d2, c2, in_b, cudaMemcpyHostToDevice, st);
    rc = (e == cudaSuccess) ? cufhedb_compare(ctx, op, level, d1, d2, dout, B, plain_bits, logic, precision, st)
                            : cfdb::cuda_error(e, "h2d");
    if (rc == CUFHEDB_OK) {
        e = cudaMemcpyAsync(out_lvl1, dout, out_b, cudaMemcpyDeviceToHost, st);
        if (e != cudaSuccess) rc = cfdb::cuda_error(e, "d2h");
    }
    cudaFreeAsync(d, st);
    if (rc != CUFHEDB_OK) {
        cudaStreamSynchronize(st);
        return rc;
    }
    return cufhedb_sync(ctx, st);
}

CUFHEDB_API int cufhedb_gate_lvl1_host_multi(cufhedb_ctx *const *ctxs, int nctx, int gate, const uint32_t *ca,
                                             const uint32_t *cb, uint32_t *out, int B, int precision)
{
    int rc = check_ctxs(ctxs, nctx);
    if (rc) return rc;
    if (B < 0) return cfdb::set_error(CUFHEDB_ERR_ARG, "negative batch");
    if (B > 0 && (!ca || !cb || !out)) return cfdb::set_error(CUFHEDB_ERR_ARG, "null buffer");
    const size_t w = N1 + 1;
    return run_shards(nctx, B, [&](int k, int b0, int nb) {
        return cufhedb_gate_lvl1_host(ctxs[k], gate, ca + (size_t)b0 * w, cb + (size_t)b0 * w, out + (size_t)b0 * w, nb,
                                      precision);
    });
}

CUFHEDB_API int cufhedb_compare_host_multi(cufhedb_ctx *const *ctxs, int nctx, int op, int level, const void *c1,
                                           const void *c2, uint32_t *out_lvl1, int B, uint32_t plain_bits, int logic,
                                           int precision)
{
    int rc = check_ctxs(ctxs, nctx);
    if (rc) return rc;
    if (B < 0) return cfdb::set_error(CUFHEDB_ERR_ARG, "negative batch");
    if (B > 0 && (!c1 || !c2 || !out_lvl1)) return cfdb::set_error(CUFHEDB_ERR_ARG, "null buffer");
    if (level != 1 && level != 2) return cfdb::set_error(CUFHEDB_ERR_ARG, "unsupported level");
    const size_t in_w = level == 1 ? (N1 + 1) * 4 : (N2 + 1) * 8, out_w = (N1 + 1);
    const unsigned char *p1 = static_cast<const unsigned char *>(c1), *p2 = static_cast<const unsigned char *>(c2);
    return run_shards(nctx, B, [&](int k, int b0, int nb) {
        return cufhedb_compare_host(ctxs[k], op, level, p1 + (size_t)b0 * in_w, p2 + (size_t)b0 * in_w,
                                    out_lvl1 + (size_t)b0 * out_w, nb, plain_bits, logic, precision);
    });
}

}  // extern "C"
