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
// reference's synchronous, one-row semantics; cuHEDB::batch:: adds the same
// operators over vectors of rows, which is where the throughput is.
//
// Needs TFHEpp's headers and the HEDB type aliases (HEDB/utils/types.h), the
// CUDA runtime, and libcufhedb_b200.so at link time.
#pragma once

#include <cuda_runtime.h>

#include <array>
#include <chrono>
#include <cstdint>
#include <cstring>
#include <map>
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

    // LoadBK (cufft_gpu.cuh:175-184): TFHEpp BootstrappingKeyFFT, host memory
    void LoadBK(const std::array<std::array<std::array<std::array<double, P::n>, 2>, (P::k + 1) * P::l>, 672> &bk)
    {
        if constexpr (P::n == 1024)
            cufhedb_dropin::check(cufhedb_load_bkfft_lvl01(cufhedb_dropin::engine(), &bk[0][0][0][0]));
        else
            cufhedb_dropin::check(cufhedb_load_bkfft_lvl02(cufhedb_dropin::engine(), &bk[0][0][0][0]));
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
                                             int precision = CUFHEDB_FP64)
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
        auto &s = slots_.get(stream_id);
        cufhedb_dropin::h2d(s.a, poly, s.st);
        if constexpr (P::n == 1024)
            cufhedb_dropin::check(cufhedb_pbs_lvl01(cufhedb_dropin::engine(), (const uint32_t *)s.a,
                                                    (uint32_t *)s.b, 1, &tv, CUFHEDB_FP64, s.st));
        else
            cufhedb_dropin::check(cufhedb_pbs_lvl02(cufhedb_dropin::engine(), (const uint32_t *)s.a,
                                                    (uint64_t *)s.b, 1, &tv, s.st));
        cufhedb_dropin::d2h(tlwe, s.b, s.st);
        cufhedb_dropin::finish(s.st);
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

// runs one operator on one row through the per-stream_id staging
template <typename In, typename Out, typename F>
inline void one_row(Out &res, const In &in, uint32_t stream_id, F &&op)
{
    auto &s = cufhedb_dropin::op_slots().get(stream_id);
    cufhedb_dropin::h2d(s.a, in, s.st);
    cufhedb_dropin::check(op(s.a, s.b, s.st));
    cufhedb_dropin::d2h(res, s.b, s.st);
    cufhedb_dropin::finish(s.st);
}

template <typename P>
constexpr int level()
{
    return P::n == 1024 ? 1 : 2;
}

}  // namespace detail

// ---- gatebootstrap_gpu.cuh ---------------------------------------------------
inline void MSBGateBootstrapping(TLWELvl1 &res, const TLWELvl1 &tlwe, const TFHEEvalKey &ek, bool result_type,
                                 uint32_t stream_id)
{
    cufhedb_dropin::ensure_ksk(ek, 10);
    detail::one_row(res, tlwe, stream_id, [&](void *in, void *out, cudaStream_t st) {
        return cufhedb_msb_bootstrap(cufhedb_dropin::engine(), 1, 1, in, out, 1, result_type, CUFHEDB_FP64, st);
    });
}

inline void MSBGateBootstrapping(TLWELvl1 &res, const TLWELvl2 &tlwe, const TFHEEvalKey &ek, bool result_type,
                                 uint32_t stream_id)
{
    cufhedb_dropin::ensure_ksk(ek, 20);
    detail::one_row(res, tlwe, stream_id, [&](void *in, void *out, cudaStream_t st) {
        return cufhedb_msb_bootstrap(cufhedb_dropin::engine(), 2, 1, in, out, 1, result_type, CUFHEDB_FP64, st);
    });
}

inline void MSBGateBootstrapping(TLWELvl2 &res, const TLWELvl2 &tlwe, const TFHEEvalKey &ek, bool result_type,
                                 uint32_t stream_id)
{
    cufhedb_dropin::ensure_ksk(ek, 20);
    detail::one_row(res, tlwe, stream_id, [&](void *in, void *out, cudaStream_t st) {
        return cufhedb_msb_bootstrap(cufhedb_dropin::engine(), 2, 2, in, out, 1, result_type, CUFHEDB_FP64, st);
    });
}

inline void IdeGateBootstrapping(TLWELvl1 &res, const TLWELvl1 &tlwe, uint32_t scale_bits, const TFHEEvalKey &ek,
                                 uint32_t stream_id)
{
    cufhedb_dropin::ensure_ksk(ek, 10);
    detail::one_row(res, tlwe, stream_id, [&](void *in, void *out, cudaStream_t st) {
        return cufhedb_ide_bootstrap(cufhedb_dropin::engine(), 1, 1, in, out, 1, scale_bits, CUFHEDB_FP64, st);
    });
}

inline void IdeGateBootstrapping(TLWELvl1 &res, const TLWELvl2 &tlwe, uint32_t scale_bits, const TFHEEvalKey &ek,
                                 uint32_t stream_id)
{
    cufhedb_dropin::ensure_ksk(ek, 20);
    detail::one_row(res, tlwe, stream_id, [&](void *in, void *out, cudaStream_t st) {
        return cufhedb_ide_bootstrap(cufhedb_dropin::engine(), 2, 1, in, out, 1, scale_bits, CUFHEDB_FP64, st);
    });
}

inline void IdeGateBootstrapping(TLWELvl2 &res, const TLWELvl2 &tlwe, uint32_t scale_bits, const TFHEEvalKey &ek,
                                 uint32_t stream_id)
{
    cufhedb_dropin::ensure_ksk(ek, 20);
    detail::one_row(res, tlwe, stream_id, [&](void *in, void *out, cudaStream_t st) {
        return cufhedb_ide_bootstrap(cufhedb_dropin::engine(), 2, 2, in, out, 1, scale_bits, CUFHEDB_FP64, st);
    });
}

template <typename P>
inline void HomNOT(TFHEpp::TLWE<P> &res, const TFHEpp::TLWE<P> &tlwe)
{
    for (int i = 0; i <= P::k * P::n; i++) res[i] = -tlwe[i];
}

inline void HomAND(TLWELvl1 &res, const TLWELvl1 &ca, const TLWELvl1 &cb, const TFHEEvalKey &ek, bool result_type,
                   uint32_t stream_id)
{
    cufhedb_dropin::ensure_ksk(ek, 10);
    auto &s = cufhedb_dropin::op_slots().get(stream_id);
    cufhedb_dropin::h2d(s.a, ca, s.st);
    cufhedb_dropin::h2d(s.c, cb, s.st);
    cufhedb_dropin::check(cufhedb_hom_and(cufhedb_dropin::engine(), (const uint32_t *)s.a, (const uint32_t *)s.c,
                                          (uint32_t *)s.b, 1, result_type, CUFHEDB_FP64, s.st));
    cufhedb_dropin::d2h(res, s.b, s.st);
    cufhedb_dropin::finish(s.st);
}

inline void HomOR(TLWELvl1 &res, const TLWELvl1 &ca, const TLWELvl1 &cb, const TFHEEvalKey &ek, bool result_type,
                  uint32_t stream_id)
{
    cufhedb_dropin::ensure_ksk(ek, 10);
    auto &s = cufhedb_dropin::op_slots().get(stream_id);
    cufhedb_dropin::h2d(s.a, ca, s.st);
    cufhedb_dropin::h2d(s.c, cb, s.st);
    cufhedb_dropin::check(cufhedb_hom_or(cufhedb_dropin::engine(), (const uint32_t *)s.a, (const uint32_t *)s.c,
                                         (uint32_t *)s.b, 1, result_type, CUFHEDB_FP64, s.st));
    cufhedb_dropin::d2h(res, s.b, s.st);
    cufhedb_dropin::finish(s.st);
}

inline void LOG_to_ARI(TLWELvl1 &res, const TLWELvl1 &tlwe, const TFHEEvalKey &ek, uint32_t stream_id)
{
    cufhedb_dropin::ensure_ksk(ek, 10);
    detail::one_row(res, tlwe, stream_id, [&](void *in, void *out, cudaStream_t st) {
        return cufhedb_log_to_ari(cufhedb_dropin::engine(), (const uint32_t *)in, (uint32_t *)out, 1, CUFHEDB_FP64,
                                  st);
    });
}

inline void log_rescale(TLWELvl1 &res, const TLWELvl1 &tlwe, uint32_t scale_bits, const TFHEEvalKey &ek,
                        uint32_t stream_id)
{
    cufhedb_dropin::ensure_ksk(ek, 10);
    detail::one_row(res, tlwe, stream_id, [&](void *in, void *out, cudaStream_t st) {
        return cufhedb_log_rescale(cufhedb_dropin::engine(), (const uint32_t *)in, (uint32_t *)out, 1, scale_bits,
                                   CUFHEDB_FP64, st);
    });
}

// ---- msb_gpu.cuh ---------------------------------------------------------------
inline void HomMSB(TLWELvl1 &res, const TLWELvl1 &tlwe, uint32_t plain_bits, const TFHEEvalKey &ek,
                   bool result_type, uint32_t stream_id)
{
    if (plain_bits > 10) throw std::invalid_argument("Plain bits out. ");
    cufhedb_dropin::ensure_ksk(ek, 10);
    detail::one_row(res, tlwe, stream_id, [&](void *in, void *out, cudaStream_t st) {
        return cufhedb_hom_msb(cufhedb_dropin::engine(), 1, in, (uint32_t *)out, 1, plain_bits, result_type,
                               CUFHEDB_FP64, st);
    });
}

inline void HomMSB(TLWELvl1 &res, const TLWELvl2 &tlwe, uint32_t plain_bits, const TFHEEvalKey &ek,
                   bool result_type, uint32_t stream_id)
{
    if (plain_bits > 33) throw std::invalid_argument("Plain bits out. ");
    cufhedb_dropin::ensure_ksk(ek, 10);
    cufhedb_dropin::ensure_ksk(ek, 20);
    cufhedb_dropin::ensure_ksk(ek, 21);
    detail::one_row(res, tlwe, stream_id, [&](void *in, void *out, cudaStream_t st) {
        return cufhedb_hom_msb(cufhedb_dropin::engine(), 2, in, (uint32_t *)out, 1, plain_bits, result_type,
                               CUFHEDB_FP64, st);
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
    cufhedb_dropin::ensure_ksk(ek, 10);
    if (level<P>() == 2) {
        cufhedb_dropin::ensure_ksk(ek, 20);
        cufhedb_dropin::ensure_ksk(ek, 21);
    }
    auto &s = cufhedb_dropin::op_slots().get(stream_id);
    cufhedb_dropin::h2d(s.a, c1, s.st);
    cufhedb_dropin::h2d(s.c, c2, s.st);
    cufhedb_dropin::check(cufhedb_compare(cufhedb_dropin::engine(), op, level<P>(), s.a, s.c, (uint32_t *)s.b, 1,
                                          plain_bits, result_type, CUFHEDB_FP64, s.st));
    cufhedb_dropin::d2h(res, s.b, s.st);
    cufhedb_dropin::finish(s.st);
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
             int precision = CUFHEDB_FP64)
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
                   const TFHEEvalKey &ek, bool result_type, int precision = CUFHEDB_FP64)
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
