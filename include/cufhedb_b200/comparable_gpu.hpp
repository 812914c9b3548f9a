// Drop-in replacement for cuFHEDB's src/cuHEDB/comparable_gpu.cuh (the ArcEDB
// comparisons) on top of the cufhedb_b200 C ABI.
//
// Include this header instead of the reference's comparable_gpu.cuh.  It
// re-provides, with the same names, signatures and TFHEpp types:
//   * the globals cufftplvl1 / cufftplvl2 (comparable_gpu.cuh:23-24);
//   * cuARCEDB::HomAND, HomOR (30-50), greater_than_tfhepp x2 (52-97),
//     equality_tfhepp x2 (99-127), less_than_tfhepp x2 (129-168) and
//     lift_and_and x2 (170-196).
// Where the reference ran the external product and the key switch on the host
// (TFHEpp::trgswfftExternalProduct, TFHEpp::IdentityKeySwitch) and only the
// polynomial product and the bootstrap on the GPU, every step here runs on the
// GPU, one cufhedb_arc_compare call per comparison (all digits).  Results
// decrypt the same; less_than_tfhepp keeps the reference's digit semantics
// (x_d <= y_d per digit, see cufhedb_arc_compare).  cuARCEDB::batch::compare
// takes whole columns, which is where the throughput is.
//
// Needs TFHEpp's headers and the ArcEDB / HEDB type aliases
// (ARCEDB/utils/types.h, HEDB/utils/types.h), the CUDA runtime, and
// libcufhedb_b200.so at link time.
#pragma once

#include <vector>

#include "ARCEDB/utils/types.h"
#include "cufhedb_b200/cuhedb_gpu.hpp"

// the reference's header opens namespace arcedb for its includers
// (comparable_gpu.cuh:8)
using namespace arcedb;

inline cufft::CuFFT_Torus<arcedb::Lvl1> cufftplvl1(20);
inline cufft::CuFFT_Torus<arcedb::Lvl2> cufftplvl2(20);

namespace cufhedb_dropin {

// device memory for one call
struct DevBuf {
    void *p = nullptr;
    explicit DevBuf(size_t bytes) { check_cuda(cudaMalloc(&p, bytes ? bytes : 1)); }
    ~DevBuf() { cudaFree(p); }
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
};

constexpr size_t kPreparedTrgswLvl1 = 98304;

// rows x digits -> cufhedb_arc_compare; x / y digit-major host arrays
inline void arc_compare(int op, const arcedb::TRLWELvl1 *x, const arcedb::TRGSWLvl1 *y, arcedb::TLWELvl1 *out,
                        int rows, int digits, const arcedb::TFHEEvalKey *ek, cudaStream_t st, int precision)
{
    if (digits > 1) ensure_ksk(*ek, 10);
    cufhedb_ctx *ctx = engine();
    const size_t n = (size_t)rows * digits;
    DevBuf dx(sizeof(*x) * n), dy(sizeof(*y) * n), dp(kPreparedTrgswLvl1 * n), dout(sizeof(*out) * rows);
    check_cuda(cudaMemcpyAsync(dx.p, x, sizeof(*x) * n, cudaMemcpyHostToDevice, st));
    check_cuda(cudaMemcpyAsync(dy.p, y, sizeof(*y) * n, cudaMemcpyHostToDevice, st));
    check(cufhedb_trgswfft_prepare_lvl1(ctx, (const double *)dy.p, dp.p, (int)n, st));
    check(cufhedb_arc_compare(ctx, op, (const uint32_t *)dx.p, dp.p, (uint32_t *)dout.p, rows, digits, precision,
                              st));
    check_cuda(cudaMemcpyAsync(out, dout.p, sizeof(*out) * rows, cudaMemcpyDeviceToHost, st));
    finish(st);
}

inline void arc_one(int op, std::vector<arcedb::TRLWELvl1> &x, std::vector<arcedb::TRGSWLvl1> &y, size_t digits,
                    arcedb::TLWELvl1 &res, const arcedb::TFHEEvalKey *ek, uint32_t stream_id)
{
    if (digits == 0 || x.size() < digits || y.size() < digits)
        throw std::invalid_argument("cufhedb: fewer digit ciphertexts than cipher_size");
    auto &s = op_slots().get(stream_id);
    arc_compare(op, x.data(), y.data(), &res, 1, (int)digits, ek, s.st, CUFHEDB_FP64);
}

// lvl1 gate a + b + offset through IKS10 and PBS01 with the constant mu test vector
inline void arc_gate(int gate, arcedb::TLWELvl1 &res, const arcedb::TLWELvl1 &ca, const arcedb::TLWELvl1 &cb,
                     const arcedb::TFHEEvalKey &ek, uint32_t stream_id)
{
    (void)stream_id;   // concurrent calls are coalesced into one batched gate launch
    ensure_ksk(ek, 10);
    const int prec = precision();
    coalesced_row(Coalescer::Key{OP_GATE, (uint64_t)gate, (uint64_t)prec}, res, ca, &cb,
                  [&](const void *a, const void *b, void *out, int B, cudaStream_t st) {
                      return cufhedb_gate_lvl1(engine(), gate, (const uint32_t *)a, (const uint32_t *)b,
                                               (uint32_t *)out, B, prec, st);
                  });
}

// lift_and_and: (c1 + c2 - mu) key-switched to lvl0, bootstrapped with the
// constant -c test vector, then +c
template <class Out>
inline void lift_and_and(const arcedb::TLWELvl1 &c1, const arcedb::TLWELvl1 &c2, Out &res, uint32_t scale_bits,
                         const arcedb::TFHEEvalKey &ek, uint32_t stream_id)
{
    using T = typename Out::value_type;
    ensure_ksk(ek, 10);
    arcedb::TLWELvl1 temp;
    for (int i = 0; i <= arcedb::Lvl1::k * arcedb::Lvl1::n; i++) temp[i] = c1[i] + c2[i];
    temp[arcedb::Lvl1::k * arcedb::Lvl1::n] -= arcedb::Lvl1::μ;
    const T c = (T)(1ULL << (scale_bits - 1));
    auto &s = op_slots().get(stream_id);
    cufhedb_ctx *ctx = engine();
    h2d(s.a, temp, s.st);
    check(cufhedb_iks(ctx, 10, s.a, (uint32_t *)s.c, 1, s.st));
    cufhedb_testvec tv{CUFHEDB_TV_CONST, 0, (uint64_t)(T)(0 - c), nullptr};
    if constexpr (sizeof(T) == 4)
        check(cufhedb_pbs_lvl01(ctx, (const uint32_t *)s.c, (uint32_t *)s.b, 1, &tv, CUFHEDB_FP64, s.st));
    else
        check(cufhedb_pbs_lvl02(ctx, (const uint32_t *)s.c, (uint64_t *)s.b, 1, &tv, s.st));
    d2h(res, s.b, s.st);
    finish(s.st);
    res[res.size() - 1] += c;
}

}  // namespace cufhedb_dropin

namespace cuARCEDB {

using arcedb::TFHEEvalKey;
using arcedb::TFHESecretKey;
using arcedb::TLWELvl1;
using arcedb::TLWELvl2;
using arcedb::TRGSWLvl1;
using arcedb::TRLWELvl1;

// comparable_gpu.cuh:30-39 (a + b - mu) and 41-50 (a + b + mu)
inline void HomAND(TLWELvl1 &res, const TLWELvl1 &ca, const TLWELvl1 &cb, const TFHEEvalKey &ek, uint32_t stream_id)
{
    cufhedb_dropin::arc_gate(CUFHEDB_AND, res, ca, cb, ek, stream_id);
}

inline void HomOR(TLWELvl1 &res, const TLWELvl1 &ca, const TLWELvl1 &cb, const TFHEEvalKey &ek, uint32_t stream_id)
{
    cufhedb_dropin::arc_gate(CUFHEDB_OR, res, ca, cb, ek, stream_id);
}

// one digit: +mu iff x > y
inline void greater_than_tfhepp(TRLWELvl1 &cipher1, TRGSWLvl1 &cipher2, TLWELvl1 &res, TFHESecretKey &sk,
                                uint32_t stream_id)
{
    (void)sk;
    auto &s = cufhedb_dropin::op_slots().get(stream_id);
    cufhedb_dropin::arc_compare(0, &cipher1, &cipher2, &res, 1, 1, nullptr, s.st, CUFHEDB_FP64);
}

inline void greater_than_tfhepp(std::vector<TRLWELvl1> &ciphers1, std::vector<TRGSWLvl1> &ciphers2,
                                size_t cipher_size, TLWELvl1 &res, TFHEEvalKey &ek, TFHESecretKey &sk,
                                uint32_t stream_id)
{
    (void)sk;
    cufhedb_dropin::arc_one(0, ciphers1, ciphers2, cipher_size, res, &ek, stream_id);
}

// one digit: 2 * SampleExtract - mu (+mu iff x == y)
inline void equality_tfhepp(TRLWELvl1 &cipher1, TRGSWLvl1 &cipher2, TLWELvl1 &res, TFHESecretKey &sk,
                            uint32_t stream_id)
{
    (void)sk;
    auto &s = cufhedb_dropin::op_slots().get(stream_id);
    cufhedb_dropin::arc_compare(2, &cipher1, &cipher2, &res, 1, 1, nullptr, s.st, CUFHEDB_FP64);
}

inline void equality_tfhepp(std::vector<TRLWELvl1> &ciphers1, std::vector<TRGSWLvl1> &ciphers2, size_t cipher_size,
                            TLWELvl1 &res, TFHEEvalKey &ek, TFHESecretKey &sk, uint32_t stream_id)
{
    (void)sk;
    cufhedb_dropin::arc_one(2, ciphers1, ciphers2, cipher_size, res, &ek, stream_id);
}

// one digit: +mu iff x <= y (the reference's test polynomial)
inline void less_than_tfhepp(TRLWELvl1 &cipher1, TRGSWLvl1 &cipher2, TLWELvl1 &res, TFHESecretKey &sk,
                             uint32_t stream_id)
{
    (void)sk;
    auto &s = cufhedb_dropin::op_slots().get(stream_id);
    cufhedb_dropin::arc_compare(1, &cipher1, &cipher2, &res, 1, 1, nullptr, s.st, CUFHEDB_FP64);
}

inline void less_than_tfhepp(std::vector<TRLWELvl1> &ciphers1, std::vector<TRGSWLvl1> &ciphers2, size_t cipher_size,
                             TLWELvl1 &res, TFHEEvalKey &ek, TFHESecretKey &sk, uint32_t stream_id)
{
    (void)sk;
    cufhedb_dropin::arc_one(1, ciphers1, ciphers2, cipher_size, res, &ek, stream_id);
}

inline void lift_and_and(TLWELvl1 &cipher1, TLWELvl1 &cipher2, TLWELvl1 &res, uint32_t scale_bits,
                         TFHEpp::EvalKey &ek, TFHEpp::SecretKey &sk, uint32_t stream_id)
{
    (void)sk;
    cufhedb_dropin::lift_and_and(cipher1, cipher2, res, scale_bits, ek, stream_id);
}

inline void lift_and_and(TLWELvl1 &cipher1, TLWELvl1 &cipher2, TLWELvl2 &res, uint32_t scale_bits,
                         TFHEpp::EvalKey &ek, TFHEpp::SecretKey &sk, uint32_t stream_id)
{
    (void)sk;
    cufhedb_dropin::lift_and_and(cipher1, cipher2, res, scale_bits, ek, stream_id);
}

namespace batch {

// A whole column in one call: x[r] / y[r] hold row r's digits (least
// significant first, as exponent_encrypt writes them); op 0 greater_than,
// 1 less_than (the reference's semantics), 2 equality, 3 strict less_than.
inline void compare(int op, const std::vector<std::vector<TRLWELvl1>> &x, const std::vector<std::vector<TRGSWLvl1>> &y,
                    size_t cipher_size, std::vector<TLWELvl1> &res, const TFHEEvalKey &ek,
                    int precision = CUFHEDB_FP64)
{
    const size_t rows = x.size();
    if (y.size() != rows) throw std::invalid_argument("cufhedb: operand columns differ in length");
    res.resize(rows);
    if (rows == 0) return;
    std::vector<TRLWELvl1> xd(rows * cipher_size);
    std::vector<TRGSWLvl1> yd(rows * cipher_size);
    for (size_t r = 0; r < rows; ++r) {
        if (x[r].size() < cipher_size || y[r].size() < cipher_size)
            throw std::invalid_argument("cufhedb: fewer digit ciphertexts than cipher_size");
        for (size_t d = 0; d < cipher_size; ++d) {
            xd[d * rows + r] = x[r][d];
            yd[d * rows + r] = y[r][d];
        }
    }
    cudaStream_t st = cufhedb_dropin::op_slots().get(0).st;
    cufhedb_dropin::arc_compare(op, xd.data(), yd.data(), res.data(), (int)rows, (int)cipher_size, &ek, st,
                                precision);
}

}  // namespace batch

}  // namespace cuARCEDB
