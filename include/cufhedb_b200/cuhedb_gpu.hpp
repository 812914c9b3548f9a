// Drop-in replacement for cuFHEDB's GPU layer on top of the cufhedb_b200 C ABI.
//
// Include this header instead of the reference's src/cuHEDB/{gatebootstrap_gpu,
// msb_gpu,HomCompare_gpu}.cuh and fft_gpu/cufft_gpu.cuh.  It re-provides, with
// the same names, signatures and TFHEpp types:
//   * cufft::CuFFT_Torus<P> (cufft_gpu.cuh:10-451): the constructor, LoadBK,
//     ifft_st, fft_st, PolyMul_st, ExternalProduct_st,
//     GateBootstrappingTLWE2TLWEFFT_st, IdeGateBootstrappingTLWE2TLWEFFT_st
//     and the *_test timing loops (MoveBuf, a debug copy of the reference's
//     per-stream product buffer, has no counterpart: no such buffer exists);
//   * the globals cufftlvl1 / cufftlvl2 (gatebootstrap_gpu.cuh:24-25) and
//     warmupGPU() (cufft_gpu.cuh:462-470);
//   * cuHEDB::MSBGateBootstrapping x3, IdeGateBootstrapping x3, HomNOT, HomAND,
//     HomOR, LOG_to_ARI, log_rescale (gatebootstrap_gpu.cuh:31-170),
//     ExtractMSB5/9/10, ImExtractMSB5..33, HomMSB x2 (msb_gpu.cuh:7-193) and the
//     comparisons greater_than ... equal (HomCompare_gpu.cuh:13-76).
// The identity key switches these wrappers ran on the host
// (TFHEpp::IdentityKeySwitch) run on the GPU: the first call that passes a
// given TFHEEvalKey uploads its key-switching keys once.  Every call keeps the
// reference's synchronous, one-row semantics: it returns when its row's result
// is in the caller's memory.  Calls of the same operator with the same
// parameters that arrive together from several host threads (the reference's
// OpenMP row loops, test/HE3_Query/TPCH_Q6.cu:179-193) are coalesced into one
// batched launch (cufhedb_dropin::Coalescer); cuHEDB::batch:: takes whole
// columns at once.  The lvl0 -> lvl1 bootstraps run on the split-precision
// path unless CUFHEDB_PRECISION=fp64 is set in the environment or
// cufhedb_dropin::set_precision(CUFHEDB_FP64) is called; lvl2 is FP64.
//
// Needs TFHEpp's headers and the HEDB type aliases (HEDB/utils/types.h), the
// CUDA runtime, and libcufhedb_b200.so at link time.
#pragma once

#include <cuda_runtime.h>

#include <array>
#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "HEDB/comparison/tfhepp_utils.h"
#include "HEDB/utils/types.h"
#include "cufhedb_b200.h"

// the reference's header opens namespace HEDB for its includers
// (gatebootstrap_gpu.cuh:9); code written against it names TLWELvl1 etc.
// unqualified
using namespace HEDB;

namespace cufhedb_dropin {

inline void check(int rc)
{
    if (rc != CUFHEDB_OK) throw std::runtime_error(std::string("cufhedb: ") + cufhedb_last_error());
}

inline void check_cuda(cudaError_t e)
{
    if (e != cudaSuccess) throw std::runtime_error(std::string("cufhedb (CUDA): ") + cudaGetErrorString(e));
}

// one engine context per process on device 0 (the reference uses device 0 only,
// gatebootstrap_gpu.cuh:11-15)
inline cufhedb_ctx *engine()
{
    static cufhedb_ctx *ctx = [] {
        cufhedb_ctx *c = nullptr;
        check(cufhedb_ctx_create(&c, 0));
        return c;
    }();
    return ctx;
}

// key-switching keys of each TFHEEvalKey seen so far, uploaded once
inline void ensure_ksk(const HEDB::TFHEEvalKey &ek, int kind)
{
    static std::mutex mu;
    static std::map<std::pair<const void *, int>, bool> done;
    std::lock_guard<std::mutex> lk(mu);
    const void *src = kind == 10 ? (const void *)ek.iksklvl10.get()
                      : kind == 20 ? (const void *)ek.iksklvl20.get()
                                   : (const void *)ek.iksklvl21.get();
    if (!src) throw std::runtime_error("cufhedb: the evaluation key has no key-switching key of this kind");
    auto key = std::make_pair(src, kind);
    if (done.count(key)) return;
    check(cufhedb_load_ksk(engine(), kind, reinterpret_cast<const uint32_t *>(src)));
    done[key] = true;
}

// per-stream_id device staging (the reference's pitched per-stream buffers,
// cufft_gpu.cuh:138-151): one stream and one set of single-row buffers each
struct Slot {
    cudaStream_t st = nullptr;
    void *a = nullptr, *b = nullptr, *c = nullptr, *g = nullptr, *gp = nullptr;
};

class Slots {
  public:
    // bytes: sizes of the a/b/c row buffers and of the TRGSW staging
    Slots(size_t row_bytes, size_t trgsw_bytes) : row_(row_bytes), trgsw_(trgsw_bytes) {}
    ~Slots()
    {
        for (auto &s : slots_) {
            if (s.st) cudaStreamDestroy(s.st);
            cudaFree(s.a);
            cudaFree(s.b);
            cudaFree(s.c);
            cudaFree(s.g);
            cudaFree(s.gp);
        }
    }
    Slot &get(uint32_t id)
    {
        std::lock_guard<std::mutex> lk(mu_);
        if (id >= slots_.size()) slots_.resize(id + 1);
        Slot &s = slots_[id];
        if (!s.st) {
            engine();
            check_cuda(cudaStreamCreateWithFlags(&s.st, cudaStreamNonBlocking));
            check_cuda(cudaMalloc(&s.a, row_));
            check_cuda(cudaMalloc(&s.b, row_));
            check_cuda(cudaMalloc(&s.c, row_));
            check_cuda(cudaMalloc(&s.g, trgsw_));
            check_cuda(cudaMalloc(&s.gp, trgsw_));
        }
        return s;
    }

  private:
    size_t row_, trgsw_;
    std::mutex mu_;
    std::vector<Slot> slots_;
};

inline Slots &op_slots()
{
    // rows up to a lvl2 TRLWE (2 x 2048 x 8 bytes)
    static Slots s(2 * 2048 * 8, 8 * 2 * 2048 * 8);
    return s;
}

template <typename T>
inline void h2d(void *dst, const T &src, cudaStream_t st)
{
    check_cuda(cudaMemcpyAsync(dst, src.data(), sizeof(src), cudaMemcpyHostToDevice, st));
}

template <typename T>
inline void d2h(T &dst, const void *src, cudaStream_t st)
{
    check_cuda(cudaMemcpyAsync(dst.data(), src, sizeof(dst), cudaMemcpyDeviceToHost, st));
}

inline void finish(cudaStream_t st) { check(cufhedb_sync(engine(), st)); }

// precision of the lvl0 -> lvl1 bootstraps behind the one-row operators
inline int &precision_setting()
{
    static int p = [] {
        const char *e = std::getenv("CUFHEDB_PRECISION");
        const std::string v = e ? e : "";
        return v == "fp64" ? (int)CUFHEDB_FP64 : v == "split32tc" ? (int)CUFHEDB_SPLIT32_TC : (int)CUFHEDB_SPLIT32;
    }();
    return p;
}
inline int precision() { return precision_setting(); }
inline void set_precision(int p)
{
    if (p != CUFHEDB_FP64 && p != CUFHEDB_SPLIT32) throw std::invalid_argument("cufhedb: unknown precision");
    precision_setting() = p;
}

inline long env_long(const char *name, long dflt)
{
    const char *e = std::getenv(name);
    return e ? std::strtol(e, nullptr, 10) : dflt;
}

// Gathers concurrent one-row calls of one operator (same parameters) into one
// batched launch.  The first caller of a group is its leader: it keeps the
// group open while rows keep arriving (each arrival within gap_us of the
// previous one, at most window_us in all, at most max_rows rows), then closes
// it, copies every row's inputs to the device in one transfer through pinned
// staging, runs the batched operator once on its own stream, copies the
// results back and writes each caller's row.  Every other caller sleeps until
// its group is done; an error of the batched call is raised in every caller.
// Several groups (other operators, or the next group of the same operator)
// run at the same time on separate streams.  Limits come from the environment:
// CUFHEDB_COALESCE_ROWS (default 8192), CUFHEDB_COALESCE_GAP_US (200) and
// CUFHEDB_COALESCE_WINDOW_US (2000).
class Coalescer {
  public:
    using Key = std::array<uint64_t, 3>;
    // fn(in1, in2, out, rows, stream): the batched operator on device buffers
    using Fn = std::function<int(const void *, const void *, void *, int, cudaStream_t)>;

    static Coalescer &get()
    {
        static Coalescer c;
        return c;
    }

    void run(const Key &key, const void *in1, const void *in2, size_t in_bytes, void *out, size_t out_bytes,
             const Fn &fn)
    {
        std::unique_lock<std::mutex> lk(mu_);
        std::shared_ptr<Group> &slot = open_[key];
        const bool leader = !slot;
        if (leader) slot = std::make_shared<Group>();
        std::shared_ptr<Group> g = slot;
        g->rows.push_back({in1, in2, out});
        if (!leader) {
            g->lead_cv.notify_one();
            g->done_cv.wait(lk, [&] { return g->done; });
            if (!g->err.empty()) throw std::runtime_error(g->err);
            return;
        }
        using clk = std::chrono::steady_clock;
        const auto hard = clk::now() + std::chrono::microseconds(window_us_);
        auto last = clk::now();
        size_t seen = g->rows.size();
        while (g->rows.size() < max_rows_) {
            const auto until = std::min(hard, last + std::chrono::microseconds(gap_us_));
            g->lead_cv.wait_until(lk, until);
            const auto now = clk::now();
            if (g->rows.size() != seen) {
                seen = g->rows.size();
                last = now;
            } else if (now >= until) {
                break;
            }
            if (now >= hard) break;
        }
        auto it = open_.find(key);
        if (it != open_.end() && it->second == g) open_.erase(it);   // later arrivals start a new group
        Exec *x = take_exec();
        std::vector<Row> rows = g->rows;
        lk.unlock();
        std::string err = execute(*x, rows, in_bytes, out_bytes, fn);
        lk.lock();
        idle_.push_back(x);
        g->err = err;
        g->done = true;
        g->done_cv.notify_all();
        if (!err.empty()) throw std::runtime_error(err);
    }

    ~Coalescer()
    {
        for (Exec *x : idle_) {
            if (x->st) cudaStreamDestroy(x->st);
            cudaFreeHost(x->h);
            delete x;
        }
    }

  private:
    struct Row {
        const void *in1, *in2;
        void *out;
    };
    struct Group {
        std::vector<Row> rows;
        bool done = false;
        std::string err;
        std::condition_variable lead_cv, done_cv;
    };
    // a stream and pinned staging for one executing group
    struct Exec {
        cudaStream_t st = nullptr;
        unsigned char *h = nullptr;
        size_t cap = 0;
    };

    Coalescer()
        : max_rows_((size_t)env_long("CUFHEDB_COALESCE_ROWS", 8192)),
          gap_us_(env_long("CUFHEDB_COALESCE_GAP_US", 200)),
          window_us_(env_long("CUFHEDB_COALESCE_WINDOW_US", 2000))
    {
        if (max_rows_ < 1) max_rows_ = 1;
    }

    Exec *take_exec()
    {
        if (!idle_.empty()) {
            Exec *x = idle_.back();
            idle_.pop_back();
            return x;
        }
        return new Exec();
    }

    static std::string execute(Exec &x, const std::vector<Row> &rows, size_t in_bytes, size_t out_bytes,
                               const Fn &fn)
    {
        try {
            cufhedb_ctx *ctx = engine();
            if (!x.st) check_cuda(cudaStreamCreateWithFlags(&x.st, cudaStreamNonBlocking));
            const size_t n = rows.size();
            const bool two = rows[0].in2 != nullptr;
            // every region starts on a 256-byte boundary: the kernels read and
            // write 64-bit torus words, and n rows of lvl0 inputs (2,692 bytes
            // each) end on a 4-byte boundary only
            auto up = [](size_t b) { return (b + 255) & ~(size_t)255; };
            const size_t in2_off = up(n * in_bytes);
            const size_t out_off = up(in2_off + (two ? n * in_bytes : 0));
            const size_t total = out_off + n * out_bytes;
            if (x.cap < total) {
                cudaFreeHost(x.h);
                x.h = nullptr;
                x.cap = 0;
                check_cuda(cudaMallocHost((void **)&x.h, total));
                x.cap = total;
            }
            for (size_t i = 0; i < n; i++) {
                std::memcpy(x.h + i * in_bytes, rows[i].in1, in_bytes);
                if (two) std::memcpy(x.h + in2_off + i * in_bytes, rows[i].in2, in_bytes);
            }
            unsigned char *d = nullptr;
            check_cuda(cudaMallocAsync((void **)&d, total, x.st));
            int rc = CUFHEDB_OK;
            cudaError_t e = cudaMemcpyAsync(d, x.h, out_off, cudaMemcpyHostToDevice, x.st);
            if (e == cudaSuccess) rc = fn(d, two ? d + in2_off : nullptr, d + out_off, (int)n, x.st);
            std::string msg = rc == CUFHEDB_OK ? "" : std::string("cufhedb: ") + cufhedb_last_error();
            if (e == cudaSuccess && rc == CUFHEDB_OK)
                e = cudaMemcpyAsync(x.h + out_off, d + out_off, n * out_bytes, cudaMemcpyDeviceToHost, x.st);
            cudaFreeAsync(d, x.st);
            if (e != cudaSuccess) return std::string("cufhedb (CUDA): ") + cudaGetErrorString(e);
            if (!msg.empty()) {
                cudaStreamSynchronize(x.st);
                return msg;
            }
            if (cufhedb_sync(ctx, x.st) != CUFHEDB_OK) return std::string("cufhedb: ") + cufhedb_last_error();
            for (size_t i = 0; i < n; i++) std::memcpy(rows[i].out, x.h + out_off + i * out_bytes, out_bytes);
            return "";
        } catch (const std::exception &ex) {
            return ex.what();
        }
    }

    std::mutex mu_;
    std::map<Key, std::shared_ptr<Group>> open_;
    std::vector<Exec *> idle_;
    size_t max_rows_;
    long gap_us_, window_us_;
};

// one row through the coalescer: `in2` may be null (one-input operators)
template <typename In, typename Out>
inline void coalesced_row(const Coalescer::Key &key, Out &res, const In &in1, const In *in2, const Coalescer::Fn &fn)
{
    Coalescer::get().run(key, in1.data(), in2 ? in2->data() : nullptr, sizeof(In), res.data(), sizeof(Out), fn);
}

// operator codes of the coalescing keys
enum : uint64_t {
    OP_PBS = 1, OP_MSB, OP_IDE, OP_AND, OP_OR, OP_LOG2ARI, OP_RESCALE, OP_HOMMSB, OP_COMPARE, OP_GATE
};

}  // namespace cufhedb_dropin

namespace cufft {

template <class P>
class CuFFT_Torus {
  public:
    const int32_t _2N;
    const int32_t N;
    const int32_t Ns2;

    explicit CuFFT_Torus(const int num_stream = 20)
        : _2N(2 * P::n), N(P::n), Ns2(P::n / 2),
          slots_(sizeof(typename P::T) * 2 * P::n, sizeof(double) * (P::k + 1) * P::l * 2 * P::n)
    {
        (void)num_stream;   // streams are created on first use of each stream_id
    }

    // LoadBK (cufft_gpu.cuh:175-184): TFHEpp BootstrappingKeyFFT, host memory.
    // Then the launch shapes of this level's bootstraps are tuned once: read
    // from the table file CUFHEDB_AUTOTUNE_FILE names when that was made for
    // this device and parameter set, else measured (well under a second) and
    // written there.
    void LoadBK(const std::array<std::array<std::array<std::array<double, P::n>, 2>, (P::k + 1) * P::l>, 672> &bk)
    {
        cufhedb_ctx *ctx = cufhedb_dropin::engine();
        if constexpr (P::n == 1024)
            cufhedb_dropin::check(cufhedb_load_bkfft_lvl01(ctx, &bk[0][0][0][0]));
        else
            cufhedb_dropin::check(cufhedb_load_bkfft_lvl02(ctx, &bk[0][0][0][0]));
        const char *path = std::getenv("CUFHEDB_AUTOTUNE_FILE");
        if (path) cufhedb_autotune_load(ctx, path);   // refused when made elsewhere: tuned below
        float t[3] = {1.0f, 1.0f, 1.0f};
        cufhedb_autotune_table(ctx, P::n == 1024 ? 1 : 2, CUFHEDB_FP64, nullptr, t);
        if (!(t[0] == 1.0f && t[1] == 1.0f && t[2] == 1.0f)) return;   // this level is tuned already
        if constexpr (P::n == 1024) {
            cufhedb_dropin::check(cufhedb_autotune_pbs01(ctx, CUFHEDB_FP64, nullptr, nullptr));
            cufhedb_dropin::check(cufhedb_autotune_pbs01(ctx, CUFHEDB_SPLIT32, nullptr, nullptr));
            cufhedb_dropin::check(cufhedb_autotune_pbs01(ctx, CUFHEDB_SPLIT32_TC, nullptr, nullptr));
        } else {
            cufhedb_dropin::check(cufhedb_autotune_pbs02(ctx, nullptr));
        }
        if (path) cufhedb_autotune_save(ctx, path);
    }

    void ifft_st(std::array<double, P::n> &res, std::array<typename P::T, P::n> &a, const uint32_t stream_id)
    {
        auto &s = slots_.get(stream_id);
        cufhedb_dropin::h2d(s.a, a, s.st);
        if constexpr (P::n == 1024)
            cufhedb_dropin::check(cufhedb_twist_ifft_lvl1(cufhedb_dropin::engine(), (const uint32_t *)s.a,
                                                          (double *)s.g, 1, s.st));
        else
            cufhedb_dropin::check(cufhedb_twist_ifft_lvl2(cufhedb_dropin::engine(), (const uint64_t *)s.a,
                                                          (double *)s.g, 1, s.st));
        cufhedb_dropin::d2h(res, s.g, s.st);
        cufhedb_dropin::finish(s.st);
        set_multiplier(res);
    }

    void fft_st(std::array<typename P::T, P::n> &res, std::array<double, P::n> &a, const uint32_t stream_id)
    {
        auto &s = slots_.get(stream_id);
        cufhedb_dropin::h2d(s.g, a, s.st);
        if constexpr (P::n == 1024)
            cufhedb_dropin::check(cufhedb_twist_fft_lvl1(cufhedb_dropin::engine(), (const double *)s.g,
                                                         (uint32_t *)s.a, 1, s.st));
        else
            cufhedb_dropin::check(cufhedb_twist_fft_lvl2(cufhedb_dropin::engine(), (const double *)s.g,
                                                         (uint64_t *)s.a, 1, s.st));
        cufhedb_dropin::d2h(res, s.a, s.st);
        cufhedb_dropin::finish(s.st);
        set_multiplier(a);
    }

    // PolyMul_st (cufft_gpu.cuh:214-226): both polynomials of `trlwe` times the
    // engine's multiplier.  As in the reference that is the all-ones
    // polynomial its constructor transforms (cufft_gpu.cuh:116-127), replaced
    // by the result of the last ifft_st or the input of the last fft_st (both
    // write the buffer PolyMul reads there).
    void PolyMul_st(std::array<std::array<typename P::T, P::n>, 2> &res,
                    std::array<std::array<typename P::T, P::n>, 2> &trlwe, const uint32_t stream_id)
    {
        std::array<double, P::n> m;
        if (!get_multiplier(m)) {
            std::array<typename P::T, P::n> ones;
            ones.fill(1);
            ifft_st(m, ones, stream_id);
        }
        auto &s = slots_.get(stream_id);
        cufhedb_dropin::h2d(s.a, trlwe, s.st);
        cufhedb_dropin::h2d(s.g, m, s.st);
        if constexpr (P::n == 1024)
            cufhedb_dropin::check(cufhedb_polymul_lvl1(cufhedb_dropin::engine(), (const uint32_t *)s.a,
                                                       (const double *)s.g, (uint32_t *)s.b, 2, 1, s.st));
        else
            cufhedb_dropin::check(cufhedb_polymul_lvl2(cufhedb_dropin::engine(), (const uint64_t *)s.a,
                                                       (const double *)s.g, (uint64_t *)s.b, 2, 1, s.st));
        cufhedb_dropin::d2h(res, s.b, s.st);
        cufhedb_dropin::finish(s.st);
    }

    void ExternalProduct_st(std::array<std::array<typename P::T, P::n>, 2> &res,
                            std::array<std::array<typename P::T, P::n>, 2> &trlwe,
                            const std::array<std::array<std::array<double, P::n>, 2>, (P::k + 1) * P::l> &trgswfft,
                            const uint32_t stream_id)
    {
        auto &s = slots_.get(stream_id);
        cufhedb_dropin::h2d(s.a, trlwe, s.st);
        cufhedb_dropin::h2d(s.g, trgswfft, s.st);
        cufhedb_ctx *ctx = cufhedb_dropin::engine();
        if constexpr (P::n == 1024) {
            cufhedb_dropin::check(cufhedb_trgswfft_prepare_lvl1(ctx, (const double *)s.g, s.gp, 1, s.st));
            cufhedb_dropin::check(cufhedb_extprod_lvl1(ctx, (const uint32_t *)s.a, s.gp, (uint32_t *)s.b, 1, 0,
                                                       CUFHEDB_FP64, s.st));
        } else {
            cufhedb_dropin::check(cufhedb_trgswfft_prepare_lvl2(ctx, (const double *)s.g, s.gp, 1, s.st));
            cufhedb_dropin::check(
                cufhedb_extprod_lvl2(ctx, (const uint64_t *)s.a, s.gp, (uint64_t *)s.b, 1, 0, s.st));
        }
        cufhedb_dropin::d2h(res, s.b, s.st);
        cufhedb_dropin::finish(s.st);
    }

    // GateBootstrappingTLWE2TLWEFFT_st (cufft_gpu.cuh:250-271): constant test vector u
    void GateBootstrappingTLWE2TLWEFFT_st(std::array<typename P::T, P::n + 1> &tlwe, std::array<uint32_t, 673> &poly,
                                          const typename P::T u, const uint32_t stream_id)
    {
        cufhedb_testvec tv{CUFHEDB_TV_CONST, 0, (uint64_t)u, nullptr};
        pbs(tlwe, poly, tv, stream_id);
    }

    // IdeGateBootstrappingTLWE2TLWEFFT_st (cufft_gpu.cuh:273-294): the staircase
    // test vector 2^scale_bits * (i >> 6)
    void IdeGateBootstrappingTLWE2TLWEFFT_st(std::array<typename P::T, P::n + 1> &tlwe,
                                             std::array<uint32_t, 673> &poly, const uint32_t scale_bits,
                                             const uint32_t stream_id)
    {
        cufhedb_testvec tv{CUFHEDB_TV_STAIRCASE, 6, scale_bits, nullptr};
        pbs(tlwe, poly, tv, stream_id);
    }

    // timing loops of the reference's microbenchmarks (cost in microseconds)
    void ifft_test(std::array<double, P::n> &res, std::array<typename P::T, P::n> &a, uint32_t test_num, double &cost)
    {
        timed(cost, test_num, [&] { ifft_st(res, a, 0); });
    }
    void GateBootstrappingTLWE2TLWEFFT_test(std::array<typename P::T, P::n + 1> &tlwe,
                                            std::array<uint32_t, 673> &poly, const typename P::T u,
                                            uint32_t test_num, double &cost)
    {
        timed(cost, test_num, [&] { GateBootstrappingTLWE2TLWEFFT_st(tlwe, poly, u, 0); });
    }
    void ExternalProduct_test(std::array<std::array<typename P::T, P::n>, 2> &res,
                              std::array<std::array<typename P::T, P::n>, 2> &trlwe,
                              const std::array<std::array<std::array<double, P::n>, 2>, (P::k + 1) * P::l> &trgswfft,
                              uint32_t test_num, double &cost)
    {
        timed(cost, test_num, [&] { ExternalProduct_st(res, trlwe, trgswfft, 0); });
    }

    // batched bootstraps: B lvl0 inputs -> B outputs in one launch
    void GateBootstrappingTLWE2TLWEFFT_batch(std::vector<std::array<typename P::T, P::n + 1>> &out,
                                             const std::vector<std::array<uint32_t, 673>> &in, const typename P::T u,
                                             int precision = cufhedb_dropin::precision())
    {
        out.resize(in.size());
        if (in.empty()) return;
        cufhedb_testvec tv{CUFHEDB_TV_CONST, 0, (uint64_t)u, nullptr};
        cufhedb_ctx *ctx = cufhedb_dropin::engine();
        const int B = (int)in.size();
        void *din = nullptr, *dout = nullptr;
        cufhedb_dropin::check_cuda(cudaMalloc(&din, sizeof(in[0]) * B));
        cufhedb_dropin::check_cuda(cudaMalloc(&dout, sizeof(out[0]) * B));
        cufhedb_dropin::check_cuda(cudaMemcpy(din, in.data(), sizeof(in[0]) * B, cudaMemcpyHostToDevice));
        int rc;
        if constexpr (P::n == 1024)
            rc = cufhedb_pbs_lvl01(ctx, (const uint32_t *)din, (uint32_t *)dout, B, &tv, precision, nullptr);
        else
            rc = cufhedb_pbs_lvl02(ctx, (const uint32_t *)din, (uint64_t *)dout, B, &tv, nullptr);
        if (rc == CUFHEDB_OK) rc = cufhedb_sync(ctx, nullptr);
        if (rc == CUFHEDB_OK)
            cufhedb_dropin::check_cuda(cudaMemcpy(out.data(), dout, sizeof(out[0]) * B, cudaMemcpyDeviceToHost));
        cudaFree(din);
        cudaFree(dout);
        cufhedb_dropin::check(rc);
    }

  private:
    cufhedb_dropin::Slots slots_;
    std::mutex mul_mu_;
    bool mul_set_ = false;
    std::array<double, P::n> mul_{};

    void set_multiplier(const std::array<double, P::n> &m)
    {
        std::lock_guard<std::mutex> lk(mul_mu_);
        mul_ = m;
        mul_set_ = true;
    }
    bool get_multiplier(std::array<double, P::n> &m)
    {
        std::lock_guard<std::mutex> lk(mul_mu_);
        m = mul_;
        return mul_set_;
    }

    void pbs(std::array<typename P::T, P::n + 1> &tlwe, std::array<uint32_t, 673> &poly, const cufhedb_testvec &tv,
             uint32_t stream_id)
    {
        (void)stream_id;   // concurrent calls are coalesced; each returns with its own result
        const int prec = cufhedb_dropin::precision();
        const cufhedb_dropin::Coalescer::Key key{
            cufhedb_dropin::OP_PBS, ((uint64_t)P::n << 32) | ((uint64_t)tv.kind << 16) | ((uint64_t)tv.pad_bits << 8) |
                                        (uint64_t)prec,
            tv.value};
        cufhedb_dropin::coalesced_row(
            key, tlwe, poly, (const std::array<uint32_t, 673> *)nullptr,
            [&](const void *in, const void *, void *out, int B, cudaStream_t st) {
                if constexpr (P::n == 1024)
                    return cufhedb_pbs_lvl01(cufhedb_dropin::engine(), (const uint32_t *)in, (uint32_t *)out, B,
                                             &tv, prec, st);
                else
                    return cufhedb_pbs_lvl02(cufhedb_dropin::engine(), (const uint32_t *)in, (uint64_t *)out, B,
                                             &tv, st);
            });
    }

    template <typename F>
    static void timed(double &cost, uint32_t n, F &&f)
    {
        auto t0 = std::chrono::system_clock::now();
        for (uint32_t i = 0; i < n; ++i) f();
        cost = (double)std::chrono::duration_cast<std::chrono::microseconds>(std::chrono::system_clock::now() - t0)
                   .count();
    }
};

}  // namespace cufft

// the reference's globals (gatebootstrap_gpu.cuh:17-25)
inline cufft::CuFFT_Torus<HEDB::Lvl1> cufftlvl1(20);
inline cufft::CuFFT_Torus<HEDB::Lvl2> cufftlvl2(20);

inline void warmupGPU()
{
    cufhedb_dropin::engine();
    cudaDeviceSynchronize();
}

namespace cuHEDB {

using HEDB::Lvl1;
using HEDB::Lvl2;
using HEDB::TFHEEvalKey;
using HEDB::TLWELvl1;
using HEDB::TLWELvl2;

namespace detail {

using cufhedb_dropin::Coalescer;

// one row of a one-input operator, coalesced with concurrent calls of the same
// operator and parameters (the stream id orders nothing: the call is complete
// when it returns, as in the reference)
template <typename In, typename Out, typename F>
inline void one_row(const Coalescer::Key &key, Out &res, const In &in, F &&op)
{
    cufhedb_dropin::coalesced_row(key, res, in, (const In *)nullptr,
                                  [&](const void *a, const void *, void *o, int B, cudaStream_t st) {
                                      return op(a, o, B, st);
                                  });
}

// one row of a two-input operator
template <typename In, typename Out, typename F>
inline void two_rows(const Coalescer::Key &key, Out &res, const In &a, const In &b, F &&op)
{
    cufhedb_dropin::coalesced_row(key, res, a, &b,
                                  [&](const void *x, const void *y, void *o, int B, cudaStream_t st) {
                                      return op(x, y, o, B, st);
                                  });
}

inline Coalescer::Key key(uint64_t op, uint64_t a, uint64_t b = 0)
{
    return {op, a, (b << 1) | (uint64_t)cufhedb_dropin::precision()};
}

template <typename P>
constexpr int level()
{
    return P::n == 1024 ? 1 : 2;
}

}  // namespace detail

// ---- gatebootstrap_gpu.cuh ---------------------------------------------------
#define CUFHEDB_MSB_ROW(RES, IN, LIN, LOUT, KSK)                                                              \
    inline void MSBGateBootstrapping(RES &res, const IN &tlwe, const TFHEEvalKey &ek, bool result_type,       \
                                     uint32_t stream_id)                                                      \
    {                                                                                                         \
        (void)stream_id;                                                                                      \
        cufhedb_dropin::ensure_ksk(ek, KSK);                                                                  \
        const int prec = cufhedb_dropin::precision();                                                         \
        detail::one_row(detail::key(cufhedb_dropin::OP_MSB, LIN * 16 + LOUT, result_type), res, tlwe,        \
                        [&](const void *in, void *out, int B, cudaStream_t st) {                              \
                            return cufhedb_msb_bootstrap(cufhedb_dropin::engine(), LIN, LOUT, in, out, B,     \
                                                         result_type, prec, st);                              \
                        });                                                                                   \
    }
CUFHEDB_MSB_ROW(TLWELvl1, TLWELvl1, 1, 1, 10)
CUFHEDB_MSB_ROW(TLWELvl1, TLWELvl2, 2, 1, 20)
CUFHEDB_MSB_ROW(TLWELvl2, TLWELvl2, 2, 2, 20)
#undef CUFHEDB_MSB_ROW

#define CUFHEDB_IDE_ROW(RES, IN, LIN, LOUT, KSK)                                                              \
    inline void IdeGateBootstrapping(RES &res, const IN &tlwe, uint32_t scale_bits, const TFHEEvalKey &ek,    \
                                     uint32_t stream_id)                                                      \
    {                                                                                                         \
        (void)stream_id;                                                                                      \
        cufhedb_dropin::ensure_ksk(ek, KSK);                                                                  \
        const int prec = cufhedb_dropin::precision();                                                         \
        detail::one_row(detail::key(cufhedb_dropin::OP_IDE, LIN * 16 + LOUT, scale_bits), res, tlwe,         \
                        [&](const void *in, void *out, int B, cudaStream_t st) {                              \
                            return cufhedb_ide_bootstrap(cufhedb_dropin::engine(), LIN, LOUT, in, out, B,     \
                                                         scale_bits, prec, st);                               \
                        });                                                                                   \
    }
CUFHEDB_IDE_ROW(TLWELvl1, TLWELvl1, 1, 1, 10)
CUFHEDB_IDE_ROW(TLWELvl1, TLWELvl2, 2, 1, 20)
CUFHEDB_IDE_ROW(TLWELvl2, TLWELvl2, 2, 2, 20)
#undef CUFHEDB_IDE_ROW

template <typename P>
inline void HomNOT(TFHEpp::TLWE<P> &res, const TFHEpp::TLWE<P> &tlwe)
{
    for (int i = 0; i <= P::k * P::n; i++) res[i] = -tlwe[i];
}

inline void HomAND(TLWELvl1 &res, const TLWELvl1 &ca, const TLWELvl1 &cb, const TFHEEvalKey &ek, bool result_type,
                   uint32_t stream_id)
{
    (void)stream_id;
    cufhedb_dropin::ensure_ksk(ek, 10);
    const int prec = cufhedb_dropin::precision();
    detail::two_rows(detail::key(cufhedb_dropin::OP_AND, 0, result_type), res, ca, cb,
                     [&](const void *a, const void *b, void *out, int B, cudaStream_t st) {
                         return cufhedb_hom_and(cufhedb_dropin::engine(), (const uint32_t *)a, (const uint32_t *)b,
                                                (uint32_t *)out, B, result_type, prec, st);
                     });
}

inline void HomOR(TLWELvl1 &res, const TLWELvl1 &ca, const TLWELvl1 &cb, const TFHEEvalKey &ek, bool result_type,
                  uint32_t stream_id)
{
    (void)stream_id;
    cufhedb_dropin::ensure_ksk(ek, 10);
    const int prec = cufhedb_dropin::precision();
    detail::two_rows(detail::key(cufhedb_dropin::OP_OR, 0, result_type), res, ca, cb,
                     [&](const void *a, const void *b, void *out, int B, cudaStream_t st) {
                         return cufhedb_hom_or(cufhedb_dropin::engine(), (const uint32_t *)a, (const uint32_t *)b,
                                               (uint32_t *)out, B, result_type, prec, st);
                     });
}

inline void LOG_to_ARI(TLWELvl1 &res, const TLWELvl1 &tlwe, const TFHEEvalKey &ek, uint32_t stream_id)
{
    (void)stream_id;
    cufhedb_dropin::ensure_ksk(ek, 10);
    const int prec = cufhedb_dropin::precision();
    detail::one_row(detail::key(cufhedb_dropin::OP_LOG2ARI, 0), res, tlwe,
                    [&](const void *in, void *out, int B, cudaStream_t st) {
                        return cufhedb_log_to_ari(cufhedb_dropin::engine(), (const uint32_t *)in, (uint32_t *)out,
                                                  B, prec, st);
                    });
}

inline void log_rescale(TLWELvl1 &res, const TLWELvl1 &tlwe, uint32_t scale_bits, const TFHEEvalKey &ek,
                        uint32_t stream_id)
{
    (void)stream_id;
    cufhedb_dropin::ensure_ksk(ek, 10);
    const int prec = cufhedb_dropin::precision();
    detail::one_row(detail::key(cufhedb_dropin::OP_RESCALE, 0, scale_bits), res, tlwe,
                    [&](const void *in, void *out, int B, cudaStream_t st) {
                        return cufhedb_log_rescale(cufhedb_dropin::engine(), (const uint32_t *)in, (uint32_t *)out,
                                                   B, scale_bits, prec, st);
                    });
}

// ---- msb_gpu.cuh ---------------------------------------------------------------
inline void HomMSB(TLWELvl1 &res, const TLWELvl1 &tlwe, uint32_t plain_bits, const TFHEEvalKey &ek,
                   bool result_type, uint32_t stream_id)
{
    (void)stream_id;
    if (plain_bits > 10) throw std::invalid_argument("Plain bits out. ");
    cufhedb_dropin::ensure_ksk(ek, 10);
    const int prec = cufhedb_dropin::precision();
    detail::one_row(detail::key(cufhedb_dropin::OP_HOMMSB, 1, plain_bits * 2 + result_type), res, tlwe,
                    [&](const void *in, void *out, int B, cudaStream_t st) {
                        return cufhedb_hom_msb(cufhedb_dropin::engine(), 1, in, (uint32_t *)out, B, plain_bits,
                                               result_type, prec, st);
                    });
}

inline void HomMSB(TLWELvl1 &res, const TLWELvl2 &tlwe, uint32_t plain_bits, const TFHEEvalKey &ek,
                   bool result_type, uint32_t stream_id)
{
    (void)stream_id;
    if (plain_bits > 33) throw std::invalid_argument("Plain bits out. ");
    cufhedb_dropin::ensure_ksk(ek, 10);
    cufhedb_dropin::ensure_ksk(ek, 20);
    cufhedb_dropin::ensure_ksk(ek, 21);
    const int prec = cufhedb_dropin::precision();
    detail::one_row(detail::key(cufhedb_dropin::OP_HOMMSB, 2, plain_bits * 2 + result_type), res, tlwe,
                    [&](const void *in, void *out, int B, cudaStream_t st) {
                        return cufhedb_hom_msb(cufhedb_dropin::engine(), 2, in, (uint32_t *)out, B, plain_bits,
                                               result_type, prec, st);
                    });
}

inline void ExtractMSB5(TLWELvl1 &res, const TLWELvl1 &tlwe, const TFHEEvalKey &ek, bool result_type,
                        uint32_t stream_id = 0)
{
    MSBGateBootstrapping(res, tlwe, ek, result_type, stream_id);
}

namespace detail {
// the reference reaches each ExtractMSB / ImExtractMSB stage only for the
// plain_bits range its HomMSB dispatches to it; the GPU chain is entered
// at the top, so other values are refused instead of being re-dispatched
inline void msb_range(uint32_t plain_bits, uint32_t lo, uint32_t hi)
{
    if (plain_bits < lo || plain_bits > hi)
        throw std::invalid_argument("cufhedb: plain_bits outside this MSB stage's range");
}
}  // namespace detail

inline void ExtractMSB9(TLWELvl1 &res, const TLWELvl1 &tlwe, uint32_t plain_bits, const TFHEEvalKey &ek,
                        bool result_type, uint32_t stream_id = 0)
{
    detail::msb_range(plain_bits, 6, 9);
    HomMSB(res, tlwe, plain_bits, ek, result_type, stream_id);
}

inline void ExtractMSB10(TLWELvl1 &res, const TLWELvl1 &tlwe, uint32_t plain_bits, const TFHEEvalKey &ek,
                         bool result_type, uint32_t stream_id = 0)
{
    detail::msb_range(plain_bits, 10, 10);
    HomMSB(res, tlwe, plain_bits, ek, result_type, stream_id);
}

inline void ImExtractMSB5(TLWELvl1 &res, const TLWELvl2 &tlwe, uint32_t plain_bits, const TFHEEvalKey &ek,
                          bool result_type, uint32_t stream_id)
{
    (void)plain_bits;   // the 5-bit stage ignores it (msb_gpu.cuh:64-69)
    HomMSB(res, tlwe, 5, ek, result_type, stream_id);
}

#define CUFHEDB_IMEXTRACT(NAME, LO, HI)                                                                    \
    inline void NAME(TLWELvl1 &res, const TLWELvl2 &tlwe, uint32_t plain_bits, const TFHEEvalKey &ek,     \
                     bool result_type, uint32_t stream_id)                                                \
    {                                                                                                     \
        detail::msb_range(plain_bits, LO, HI);                                                            \
        HomMSB(res, tlwe, plain_bits, ek, result_type, stream_id);                                        \
    }
CUFHEDB_IMEXTRACT(ImExtractMSB9, 6, 9)
CUFHEDB_IMEXTRACT(ImExtractMSB14, 10, 14)
CUFHEDB_IMEXTRACT(ImExtractMSB19, 15, 19)
CUFHEDB_IMEXTRACT(ImExtractMSB24, 20, 24)
CUFHEDB_IMEXTRACT(ImExtractMSB29, 25, 29)
CUFHEDB_IMEXTRACT(ImExtractMSB33, 30, 33)
#undef CUFHEDB_IMEXTRACT

// ---- HomCompare_gpu.cuh ----------------------------------------------------------
namespace detail {
template <typename P>
inline void compare(int op, TFHEpp::TLWE<P> &c1, TFHEpp::TLWE<P> &c2, TLWELvl1 &res, uint32_t plain_bits,
                    const TFHEEvalKey &ek, bool result_type, uint32_t stream_id)
{
    (void)stream_id;
    cufhedb_dropin::ensure_ksk(ek, 10);
    if (level<P>() == 2) {
        cufhedb_dropin::ensure_ksk(ek, 20);
        cufhedb_dropin::ensure_ksk(ek, 21);
    }
    const int prec = cufhedb_dropin::precision();
    two_rows(key(cufhedb_dropin::OP_COMPARE, (uint64_t)op * 16 + level<P>(), plain_bits * 2 + result_type), res, c1,
             c2, [&](const void *a, const void *b, void *out, int B, cudaStream_t st) {
                 return cufhedb_compare(cufhedb_dropin::engine(), op, level<P>(), a, b, (uint32_t *)out, B,
                                        plain_bits, result_type, prec, st);
             });
}
}  // namespace detail

template <typename P>
void greater_than(TFHEpp::TLWE<P> &cipher1, TFHEpp::TLWE<P> &cipher2, TLWELvl1 &res, uint32_t plain_bits,
                  TFHEEvalKey &ek, bool result_type, uint32_t stream_id)
{
    detail::compare<P>(0, cipher1, cipher2, res, plain_bits, ek, result_type, stream_id);
}

template <typename P>
void greater_than_equal(TFHEpp::TLWE<P> &cipher1, TFHEpp::TLWE<P> &cipher2, TLWELvl1 &res, uint32_t plain_bits,
                        TFHEEvalKey &ek, bool result_type, uint32_t stream_id)
{
    detail::compare<P>(1, cipher1, cipher2, res, plain_bits, ek, result_type, stream_id);
}

template <typename P>
void less_than(TFHEpp::TLWE<P> &cipher1, TFHEpp::TLWE<P> &cipher2, TLWELvl1 &res, uint32_t plain_bits,
               TFHEEvalKey &ek, bool result_type, uint32_t stream_id)
{
    detail::compare<P>(2, cipher1, cipher2, res, plain_bits, ek, result_type, stream_id);
}

template <typename P>
void less_than_equal(TFHEpp::TLWE<P> &cipher1, TFHEpp::TLWE<P> &cipher2, TLWELvl1 &res, uint32_t plain_bits,
                     TFHEEvalKey &ek, bool result_type, uint32_t stream_id)
{
    detail::compare<P>(3, cipher1, cipher2, res, plain_bits, ek, result_type, stream_id);
}

template <typename P>
void equal(TFHEpp::TLWE<P> &cipher1, TFHEpp::TLWE<P> &cipher2, TLWELvl1 &res, uint32_t plain_bits, TFHEEvalKey &ek,
           bool result_type, uint32_t stream_id)
{
    detail::compare<P>(4, cipher1, cipher2, res, plain_bits, ek, result_type, stream_id);
}

// ---- batched operators: the same semantics over vectors of rows ---------------------
namespace batch {

// op: 0 greater_than, 1 greater_than_equal, 2 less_than, 3 less_than_equal, 4 equal
template <typename P>
void compare(int op, const std::vector<TFHEpp::TLWE<P>> &c1, const std::vector<TFHEpp::TLWE<P>> &c2,
             std::vector<TLWELvl1> &res, uint32_t plain_bits, const TFHEEvalKey &ek, bool result_type,
             int precision = cufhedb_dropin::precision())
{
    if (c1.size() != c2.size()) throw std::invalid_argument("cufhedb: column sizes differ");
    res.resize(c1.size());
    if (c1.empty()) return;
    cufhedb_dropin::ensure_ksk(ek, 10);
    if (detail::level<P>() == 2) {
        cufhedb_dropin::ensure_ksk(ek, 20);
        cufhedb_dropin::ensure_ksk(ek, 21);
    }
    const int B = (int)c1.size();
    void *d1 = nullptr, *d2 = nullptr, *dr = nullptr;
    cufhedb_dropin::check_cuda(cudaMalloc(&d1, sizeof(c1[0]) * B));
    cufhedb_dropin::check_cuda(cudaMalloc(&d2, sizeof(c2[0]) * B));
    cufhedb_dropin::check_cuda(cudaMalloc(&dr, sizeof(res[0]) * B));
    cufhedb_dropin::check_cuda(cudaMemcpy(d1, c1.data(), sizeof(c1[0]) * B, cudaMemcpyHostToDevice));
    cufhedb_dropin::check_cuda(cudaMemcpy(d2, c2.data(), sizeof(c2[0]) * B, cudaMemcpyHostToDevice));
    cufhedb_ctx *ctx = cufhedb_dropin::engine();
    int rc = cufhedb_compare(ctx, op, detail::level<P>(), d1, d2, (uint32_t *)dr, B, plain_bits, result_type,
                             precision, nullptr);
    if (rc == CUFHEDB_OK) rc = cufhedb_sync(ctx, nullptr);
    if (rc == CUFHEDB_OK)
        cufhedb_dropin::check_cuda(cudaMemcpy(res.data(), dr, sizeof(res[0]) * B, cudaMemcpyDeviceToHost));
    cudaFree(d1);
    cudaFree(d2);
    cudaFree(dr);
    cufhedb_dropin::check(rc);
}

inline void HomAND(std::vector<TLWELvl1> &res, const std::vector<TLWELvl1> &ca, const std::vector<TLWELvl1> &cb,
                   const TFHEEvalKey &ek, bool result_type, int precision = cufhedb_dropin::precision())
{
    if (ca.size() != cb.size()) throw std::invalid_argument("cufhedb: column sizes differ");
    res.resize(ca.size());
    if (ca.empty()) return;
    cufhedb_dropin::ensure_ksk(ek, 10);
    const int B = (int)ca.size();
    void *da = nullptr, *db = nullptr, *dr = nullptr;
    cufhedb_dropin::check_cuda(cudaMalloc(&da, sizeof(ca[0]) * B));
    cufhedb_dropin::check_cuda(cudaMalloc(&db, sizeof(cb[0]) * B));
    cufhedb_dropin::check_cuda(cudaMalloc(&dr, sizeof(res[0]) * B));
    cufhedb_dropin::check_cuda(cudaMemcpy(da, ca.data(), sizeof(ca[0]) * B, cudaMemcpyHostToDevice));
    cufhedb_dropin::check_cuda(cudaMemcpy(db, cb.data(), sizeof(cb[0]) * B, cudaMemcpyHostToDevice));
    cufhedb_ctx *ctx = cufhedb_dropin::engine();
    int rc = cufhedb_hom_and(ctx, (const uint32_t *)da, (const uint32_t *)db, (uint32_t *)dr, B, result_type,
                             precision, nullptr);
    if (rc == CUFHEDB_OK) rc = cufhedb_sync(ctx, nullptr);
    if (rc == CUFHEDB_OK)
        cufhedb_dropin::check_cuda(cudaMemcpy(res.data(), dr, sizeof(res[0]) * B, cudaMemcpyDeviceToHost));
    cudaFree(da);
    cudaFree(db);
    cudaFree(dr);
    cufhedb_dropin::check(rc);
}

}  // namespace batch

}  // namespace cuHEDB
