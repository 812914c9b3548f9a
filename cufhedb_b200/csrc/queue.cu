// Scheduler for a queue of filter queries of uneven sizes and widths (the
// reference's query programs run one query at a time, each as an OpenMP row
// loop of one-row operator calls, test/HE3_Query/TPCH_Q6.cu:158-209).
//
// All queries are known when the queue starts.  The scheduler
//   1. estimates each query's cost: rows x (bootstraps per row of its
//      comparison chain, counted from the chain the operator layer runs, each
//      weighted by the per-ciphertext pass time of its level from the
//      launch-shape table);
//   2. packs queries that share one chain (level, comparison, plain bits,
//      result type) into batches of at most max_batch_rows rows, smallest
//      queries first, so one batched chain serves several queries;
//   3. orders the batches by cost per query they complete (the order that
//      minimises the sum of completion times of jobs that each finish with
//      their batch) and runs them on `nstreams` streams, each batch on the
//      stream that frees up first, so the lvl02 steps of one batch overlap the
//      lvl01 steps of another whenever SMs are free;
//   4. reports each query's completion time from the start of the queue
//      (CUDA events after its results are in place).
// A batch of several queries gathers their ciphertexts into contiguous
// device staging, runs the chain once and scatters the result rows back.
#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "ctx.cuh"

namespace {

// bootstraps per row of a comparison chain (ops.cu compare / hom_msb1 /
// hom_msb2): {lvl01, lvl02}
struct ChainCost {
    double n01, n02;
};

ChainCost msb_cost(int level, uint32_t p)
{
    if (level == 1) return {p <= 5 ? 1.0 : p <= 9 ? 3.0 : 5.0, 0.0};
    if (p <= 9) return {p <= 5 ? 1.0 : 3.0, 0.0};
    double levels = 1.0;
    for (uint32_t q = p; q > 14; q -= 5) levels += 1.0;
    return {3.0, 2.0 * levels};
}

ChainCost chain_cost(const cufhedb_query &q)
{
    ChainCost c = msb_cost(q.level, q.plain_bits + 1);
    const bool negate = q.op == 1 || q.op == 3;
    if (q.op == 4) return {2.0 * c.n01 + 1.0, 2.0 * c.n02};
    if (negate && !q.logic) c.n01 += 1.0;
    return c;
}

struct Batch {
    std::vector<int> members;
    long rows = 0;
    double cost = 0.0;
};

// Steps 1-3 of the scheduler (host only): the batches in run order and the
// stream each is queued on.  t01 / t02: per-ciphertext pass time of lvl01 /
// lvl02 bootstraps.
void plan_queue(const cufhedb_query *q, int nq, double t01, double t02, int max_batch_rows, int nstreams,
                std::vector<Batch> &batches, std::vector<int> &stream_of)
{
    std::vector<double> cost(nq);
    for (int i = 0; i < nq; ++i) {
        const ChainCost c = chain_cost(q[i]);
        cost[i] = (double)q[i].rows * (c.n01 * t01 + c.n02 * t02);
    }

    // batches: queries of one chain, smallest first, up to max_batch_rows
    std::vector<int> order(nq);
    for (int i = 0; i < nq; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost[a] < cost[b]; });
    auto same_chain = [&](int a, int b) {
        return q[a].level == q[b].level && q[a].op == q[b].op && q[a].plain_bits == q[b].plain_bits &&
               (q[a].logic != 0) == (q[b].logic != 0);
    };
    batches.clear();
    std::vector<int> open_of(nq, -1);   // open batch index per chain, keyed by its first query
    std::vector<int> chain_head;
    for (int i : order) {
        int head = -1;
        for (int h : chain_head)
            if (same_chain(h, i)) head = h;
        if (head < 0) {
            chain_head.push_back(i);
            head = i;
        }
        int &bi = open_of[head];
        if (bi >= 0 && batches[bi].rows + q[i].rows > max_batch_rows) bi = -1;
        if (bi < 0) {
            bi = (int)batches.size();
            batches.emplace_back();
        }
        batches[bi].members.push_back(i);
        batches[bi].rows += q[i].rows;
        batches[bi].cost += cost[i];
    }
    std::stable_sort(batches.begin(), batches.end(), [](const Batch &a, const Batch &b) {
        return a.cost / a.members.size() < b.cost / b.members.size();
    });

    // each batch on the stream with the least estimated work queued
    std::vector<double> busy(nstreams, 0.0);
    stream_of.assign(batches.size(), 0);
    for (size_t bi = 0; bi < batches.size(); ++bi) {
        const int s = (int)(std::min_element(busy.begin(), busy.end()) - busy.begin());
        busy[s] += batches[bi].cost;
        stream_of[bi] = s;
    }
}

bool query_shape_ok(const cufhedb_query &x)
{
    return (x.level == 1 || x.level == 2) && x.op >= 0 && x.op <= 4 && x.rows >= 0 && x.plain_bits >= 1;
}

}  // namespace

extern "C" CUFHEDB_API int cufhedb_queue_plan(const cufhedb_query *q, int nq, double t01_ms, double t02_ms,
                                              int max_batch_rows, int nstreams, int *batch_of,
                                              int *stream_of_batch, int *nbatches)
{
    using namespace cfdb;
    if (nq < 0 || (nq > 0 && (!q || !batch_of || !stream_of_batch)) || !nbatches)
        return set_error(CUFHEDB_ERR_ARG, "bad query list");
    if (max_batch_rows < 1 || nstreams < 1 || nstreams > 16)
        return set_error(CUFHEDB_ERR_ARG, "max_batch_rows >= 1 and 1 <= nstreams <= 16");
    if (!(t01_ms > 0.0) || !(t02_ms > 0.0)) return set_error(CUFHEDB_ERR_ARG, "pass times must be positive");
    for (int i = 0; i < nq; ++i)
        if (!query_shape_ok(q[i])) return set_error(CUFHEDB_ERR_ARG, ("bad query " + std::to_string(i)).c_str());
    std::vector<Batch> batches;
    std::vector<int> stream_of;
    plan_queue(q, nq, t01_ms, t02_ms, max_batch_rows, nstreams, batches, stream_of);
    for (size_t b = 0; b < batches.size(); ++b) {
        for (int m : batches[b].members) batch_of[m] = (int)b;
        stream_of_batch[b] = stream_of[b];
    }
    *nbatches = (int)batches.size();
    return CUFHEDB_OK;
}

extern "C" CUFHEDB_API int cufhedb_queue_run(cufhedb_ctx *ctx, const cufhedb_query *q, int nq, int precision,
                                             int max_batch_rows, int nstreams, float *latency_ms, float *total_ms)
{
    using namespace cfdb;
    if (!ctx) return set_error(CUFHEDB_ERR_ARG, "ctx is null");
    if (nq < 0 || (nq > 0 && (!q || !latency_ms))) return set_error(CUFHEDB_ERR_ARG, "bad query list");
    if (max_batch_rows < 1 || nstreams < 1 || nstreams > 16)
        return set_error(CUFHEDB_ERR_ARG, "max_batch_rows >= 1 and 1 <= nstreams <= 16");
    if (precision != CUFHEDB_FP64 && precision != CUFHEDB_SPLIT32 &&
        precision != CUFHEDB_SPLIT32_TC)
        return set_error(CUFHEDB_ERR_ARG, "unsupported precision");
    for (int i = 0; i < nq; ++i) {
        const cufhedb_query &x = q[i];
        if (!query_shape_ok(x) || (x.rows > 0 && (!x.c1 || !x.c2 || !x.out)) ||
            !aligned_to(x.c1, x.level == 1 ? 4 : 8) || !aligned_to(x.c2, x.level == 1 ? 4 : 8) ||
            !aligned_to(x.out, 4))
            return set_error(CUFHEDB_ERR_ARG, ("bad query " + std::to_string(i)).c_str());
    }
    if (total_ms) *total_ms = 0.0f;
    if (nq == 0) return CUFHEDB_OK;
    DeviceGuard guard;
    if (guard.set(ctx->device) != cudaSuccess) return set_error(CUFHEDB_ERR_CUDA, "cudaSetDevice failed");

    // per-ciphertext time of a full pass of the fastest shape, per level
    auto per_ct = [&](const float *t, const int *shapes) {
        double best = 1e30;
        for (int i = 0; i < NSHAPES; ++i) best = std::min(best, (double)t[i] / (shapes[i] * ctx->num_sms));
        return best;
    };
    const double t01 = per_ct(ctx->pbs01_pass_ms[precision], PBS01_SHAPES);
    const double t02 = per_ct(ctx->pbs02_pass_ms, PBS02_SHAPES);
    std::vector<Batch> batches;
    std::vector<int> stream_of;
    plan_queue(q, nq, t01, t02, max_batch_rows, nstreams, batches, stream_of);

    std::vector<cudaStream_t> streams(nstreams, nullptr);
    std::vector<cudaEvent_t> done(batches.size(), nullptr);
    cudaEvent_t start = nullptr;
    int rc = CUFHEDB_OK;
    cudaError_t e = cudaEventCreate(&start);
    for (int s = 0; s < nstreams && e == cudaSuccess; ++s) e = cudaStreamCreateWithFlags(&streams[s], cudaStreamNonBlocking);
    for (size_t b = 0; b < batches.size() && e == cudaSuccess; ++b) e = cudaEventCreate(&done[b]);
    if (e == cudaSuccess) e = cudaEventRecord(start, streams[0]);
    for (int s = 1; s < nstreams && e == cudaSuccess; ++s) e = cudaStreamWaitEvent(streams[s], start, 0);
    if (e != cudaSuccess) rc = cuda_error(e, "queue set-up");

    for (size_t bi = 0; bi < batches.size() && rc == CUFHEDB_OK; ++bi) {
        const Batch &B = batches[bi];
        cudaStream_t st = streams[stream_of[bi]];
        const cufhedb_query &h = q[B.members[0]];
        const size_t in_w = (size_t)(h.level == 1 ? N1 + 1 : N2 + 1) * (h.level == 1 ? 4 : 8);   // bytes per row
        const size_t out_w = (size_t)(N1 + 1) * 4;
        const void *c1 = h.c1, *c2 = h.c2;
        uint32_t *out = h.out;
        unsigned char *stage = nullptr;
        if (B.members.size() > 1) {
            // three regions, each on a 256-byte boundary
            auto up = [](size_t b) { return (b + 255) & ~(size_t)255; };
            const size_t c2_off = up((size_t)B.rows * in_w), out_off = c2_off + up((size_t)B.rows * in_w);
            e = cudaMallocAsync((void **)&stage, out_off + (size_t)B.rows * out_w, st);
            size_t off = 0;
            for (int m : B.members) {
                const size_t n = (size_t)q[m].rows;
                if (e == cudaSuccess && n)
                    e = cudaMemcpyAsync(stage + off * in_w, q[m].c1, n * in_w, cudaMemcpyDeviceToDevice, st);
                if (e == cudaSuccess && n)
                    e = cudaMemcpyAsync(stage + c2_off + off * in_w, q[m].c2, n * in_w, cudaMemcpyDeviceToDevice, st);
                off += n;
            }
            c1 = stage;
            c2 = stage + c2_off;
            out = reinterpret_cast<uint32_t *>(stage + out_off);
            if (e != cudaSuccess) rc = cuda_error(e, "queue gather");
        }
        if (rc == CUFHEDB_OK && B.rows > 0)
            rc = cufhedb_compare(ctx, h.op, h.level, c1, c2, out, (int)B.rows, h.plain_bits, h.logic, precision, st);
        if (rc == CUFHEDB_OK && stage) {
            size_t off = 0;
            for (int m : B.members) {
                const size_t n = (size_t)q[m].rows;
                if (e == cudaSuccess && n)
                    e = cudaMemcpyAsync(q[m].out, out + off * (N1 + 1), n * out_w, cudaMemcpyDeviceToDevice, st);
                off += n;
            }
            if (e == cudaSuccess) e = cudaFreeAsync(stage, st);
            if (e != cudaSuccess) rc = cuda_error(e, "queue scatter");
        }
        if (rc == CUFHEDB_OK) {
            e = cudaEventRecord(done[bi], st);
            if (e != cudaSuccess) rc = cuda_error(e, "queue event");
        }
    }
    for (int s = 0; s < nstreams; ++s)
        if (streams[s]) cudaStreamSynchronize(streams[s]);
    if (rc == CUFHEDB_OK) rc = cufhedb_sync(ctx, streams[0]);
    float tmax = 0.0f;
    for (size_t bi = 0; bi < batches.size() && rc == CUFHEDB_OK; ++bi) {
        float ms = 0.0f;
        e = cudaEventElapsedTime(&ms, start, done[bi]);
        if (e != cudaSuccess) {
            rc = cuda_error(e, "queue timing");
            break;
        }
        for (int m : batches[bi].members) latency_ms[m] = ms;
        tmax = std::max(tmax, ms);
    }
    if (rc == CUFHEDB_OK && total_ms) *total_ms = tmax;
    for (auto ev : done)
        if (ev) cudaEventDestroy(ev);
    if (start) cudaEventDestroy(start);
    for (auto s : streams)
        if (s) cudaStreamDestroy(s);
    return rc;
}
