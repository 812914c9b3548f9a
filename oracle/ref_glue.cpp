// Test-oracle glue: a C entry layer over the reference's own TFHEpp and HEDB
// CPU code, compiled from the reference sources by oracle/Makefile (target
// `ref`).  Used only by tests/ and by bench.py's CPU-baseline leg, as the
// checker and as the timed CPU reference; never by the product library.
//
// Key material comes from the caller (the deterministic generator in
// tfhe_oracle.c), so the reference runs on exactly the keys the GPU path uses.
// TFHEpp's own generator (thirdparty/TFHEpp/src/cloudkey.cpp:22-74) draws from
// std::random_device and cannot be seeded.

#include <cstdlib>
#include <cstring>
#include <fstream>
#include <thread>
#include <vector>
#include <atomic>

#include <tfhe++.hpp>
#include "HEDB/comparison/comparison.h"

using namespace TFHEpp;
using HEDB::TLWELvl1;

namespace {
struct RefCtx {
    SecretKey sk;
    EvalKey ek;
    // key-switching keys are allocated with calloc so that rows never written
    // stay untouched zero pages; they are released with free().
    KeySwitchingKey<lvl10param> *ksk10 = nullptr;
    KeySwitchingKey<lvl20param> *ksk20 = nullptr;
    KeySwitchingKey<lvl21param> *ksk21 = nullptr;
};

template <class T>
T *calloc_obj()
{
    return reinterpret_cast<T *>(std::calloc(1, sizeof(T)));
}
}  // namespace

extern "C" {

void *tref_new() { return new RefCtx(); }

void tref_free(void *p)
{
    RefCtx *c = static_cast<RefCtx *>(p);
    c->ek.iksklvl10.release();
    c->ek.iksklvl20.release();
    c->ek.iksklvl21.release();
    std::free(c->ksk10);
    std::free(c->ksk20);
    std::free(c->ksk21);
    delete c;
}

void tref_set_secret(void *p, const uint32_t *s0, const uint32_t *s1,
                     const uint64_t *s2)
{
    RefCtx *c = static_cast<RefCtx *>(p);
    for (uint32_t i = 0; i < lvl0param::n; i++) c->sk.key.lvl0[i] = s0[i];
    for (uint32_t i = 0; i < lvl1param::n; i++) c->sk.key.lvl1[i] = s1[i];
    for (uint32_t i = 0; i < lvl2param::n; i++) c->sk.key.lvl2[i] = s2[i];
}

// Integer bootstrapping key [672][(k+1)l][2][N] -> BootstrappingKeyFFT via
// TFHEpp's own ApplyFFT2trgsw (thirdparty/TFHEpp/src/trgsw.cpp:183-193), which
// is what bkfftgen does after trgswSymEncrypt (cloudkey.cpp:22-33).
void tref_set_bk01_int(void *p, const uint32_t *bk)
{
    RefCtx *c = static_cast<RefCtx *>(p);
    if (!c->ek.bkfftlvl01)
        c->ek.bkfftlvl01 = std::make_unique<BootstrappingKeyFFT<lvl01param>>();
    const size_t per = sizeof(TRGSW<lvl1param>) / sizeof(uint32_t);
    for (uint32_t i = 0; i < lvl0param::n; i++) {
        TRGSW<lvl1param> t;
        std::memcpy(t.data(), bk + i * per, sizeof(t));
        (*c->ek.bkfftlvl01)[i] = ApplyFFT2trgsw<lvl1param>(t);
    }
}

void tref_set_bk02_int(void *p, const uint64_t *bk)
{
    RefCtx *c = static_cast<RefCtx *>(p);
    if (!c->ek.bkfftlvl02)
        c->ek.bkfftlvl02 = std::make_unique<BootstrappingKeyFFT<lvl02param>>();
    const size_t per = sizeof(TRGSW<lvl2param>) / sizeof(uint64_t);
    for (uint32_t i = 0; i < lvl0param::n; i++) {
        TRGSW<lvl2param> t;
        std::memcpy(t.data(), bk + i * per, sizeof(t));
        (*c->ek.bkfftlvl02)[i] = ApplyFFT2trgsw<lvl2param>(t);
    }
}

void tref_get_bkfft01(void *p, double *out)
{
    RefCtx *c = static_cast<RefCtx *>(p);
    std::memcpy(out, c->ek.bkfftlvl01->data(), sizeof(BootstrappingKeyFFT<lvl01param>));
}

void tref_get_bkfft02(void *p, double *out)
{
    RefCtx *c = static_cast<RefCtx *>(p);
    std::memcpy(out, c->ek.bkfftlvl02->data(), sizeof(BootstrappingKeyFFT<lvl02param>));
}

// kind: 10, 20, 21.  Returns the base of a zero-initialised full-size key the
// caller fills (all rows, or only the rows a given input will touch).
void *tref_ksk_alloc(void *p, int kind)
{
    RefCtx *c = static_cast<RefCtx *>(p);
    if (kind == 10) {
        if (!c->ksk10) {
            c->ksk10 = calloc_obj<KeySwitchingKey<lvl10param>>();
            c->ek.iksklvl10.reset(c->ksk10);
        }
        return c->ksk10;
    }
    if (kind == 20) {
        if (!c->ksk20) {
            c->ksk20 = calloc_obj<KeySwitchingKey<lvl20param>>();
            c->ek.iksklvl20.reset(c->ksk20);
        }
        return c->ksk20;
    }
    if (kind == 21) {
        if (!c->ksk21) {
            c->ksk21 = calloc_obj<KeySwitchingKey<lvl21param>>();
            c->ek.iksklvl21.reset(c->ksk21);
        }
        return c->ksk21;
    }
    return nullptr;
}

size_t tref_ksk_bytes(int kind)
{
    if (kind == 10) return sizeof(KeySwitchingKey<lvl10param>);
    if (kind == 20) return sizeof(KeySwitchingKey<lvl20param>);
    if (kind == 21) return sizeof(KeySwitchingKey<lvl21param>);
    return 0;
}

// Writes one key of the context as the reference's key tools do
// (src/HEDB/utils/serialize.cpp:7-60): a cereal PortableBinary archive of
// EvalKey::serialize_<key> (thirdparty/TFHEpp/include/cloudkey.hpp:149-228).
// kind: 1 bkfftlvl01, 2 bkfftlvl02, 10 iksklvl10, 20 iksklvl20, 21 iksklvl21.
// Returns 0, or -1 for an unknown kind or an unset key.
int tref_save_cereal(void *p, int kind, const char *path)
{
    RefCtx *c = static_cast<RefCtx *>(p);
    std::ofstream ofs{path, std::ios::binary};
    cereal::PortableBinaryOutputArchive ar(ofs);
    switch (kind) {
    case 1: if (!c->ek.bkfftlvl01) return -1; c->ek.serialize_bkfftlvl01(ar); break;
    case 2: if (!c->ek.bkfftlvl02) return -1; c->ek.serialize_bkfftlvl02(ar); break;
    case 10: if (!c->ek.iksklvl10) return -1; c->ek.serialize_iksklvl10(ar); break;
    case 20: if (!c->ek.iksklvl20) return -1; c->ek.serialize_iksklvl20(ar); break;
    case 21: if (!c->ek.iksklvl21) return -1; c->ek.serialize_iksklvl21(ar); break;
    default: return -1;
    }
    return 0;
}

// ---- primitives (mulfft.hpp:57-121, trgsw.cpp:20-39,77-103) -----------------
void tref_twist_ifft_lvl1(double *out, const uint32_t *a)
{
    PolynomialInFD<lvl1param> r;
    Polynomial<lvl1param> x;
    std::memcpy(x.data(), a, sizeof(x));
    TwistIFFT<lvl1param>(r, x);
    std::memcpy(out, r.data(), sizeof(r));
}

void tref_twist_fft_lvl1(uint32_t *out, const double *a)
{
    PolynomialInFD<lvl1param> x;
    Polynomial<lvl1param> r;
    std::memcpy(x.data(), a, sizeof(x));
    TwistFFT<lvl1param>(r, x);
    std::memcpy(out, r.data(), sizeof(r));
}

void tref_twist_ifft_lvl2(double *out, const uint64_t *a)
{
    PolynomialInFD<lvl2param> r;
    Polynomial<lvl2param> x;
    std::memcpy(x.data(), a, sizeof(x));
    TwistIFFT<lvl2param>(r, x);
    std::memcpy(out, r.data(), sizeof(r));
}

void tref_twist_fft_lvl2(uint64_t *out, const double *a)
{
    PolynomialInFD<lvl2param> x;
    Polynomial<lvl2param> r;
    std::memcpy(x.data(), a, sizeof(x));
    TwistFFT<lvl2param>(r, x);
    std::memcpy(out, r.data(), sizeof(r));
}

void tref_decomp_lvl1(uint32_t *out, const uint32_t *poly, int digit)
{
    Polynomial<lvl1param> x;
    DecomposedPolynomial<lvl1param> d;
    std::memcpy(x.data(), poly, sizeof(x));
    DecompositionPolynomial<lvl1param>(d, x, digit);
    std::memcpy(out, d.data(), sizeof(d));
}

void tref_decomp_lvl2(uint64_t *out, const uint64_t *poly, int digit)
{
    Polynomial<lvl2param> x;
    DecomposedPolynomial<lvl2param> d;
    std::memcpy(x.data(), poly, sizeof(x));
    DecompositionPolynomial<lvl2param>(d, x, digit);
    std::memcpy(out, d.data(), sizeof(d));
}

void tref_extprod_lvl1(uint32_t *res, const uint32_t *trlwe, const double *trgswfft)
{
    TRLWE<lvl1param> in, out;
    auto *g = new TRGSWFFT<lvl1param>;
    std::memcpy(in.data(), trlwe, sizeof(in));
    std::memcpy(g->data(), trgswfft, sizeof(*g));
    trgswfftExternalProduct<lvl1param>(out, in, *g);
    std::memcpy(res, out.data(), sizeof(out));
    delete g;
}

void tref_extprod_lvl2(uint64_t *res, const uint64_t *trlwe, const double *trgswfft)
{
    TRLWE<lvl2param> in, out;
    auto *g = new TRGSWFFT<lvl2param>;
    std::memcpy(in.data(), trlwe, sizeof(in));
    std::memcpy(g->data(), trgswfft, sizeof(*g));
    trgswfftExternalProduct<lvl2param>(out, in, *g);
    std::memcpy(res, out.data(), sizeof(out));
    delete g;
}

// One digit of the ArcEDB comparisons exactly as src/ARCEDB/comparison/
// comparable.cpp runs it with TFHEpp (that file itself needs SEAL, so its
// TFHEpp steps are repeated here): op 0 greater_than_tfhepp (506-523),
// 1 less_than_tfhepp (652-666), 2 equality_tfhepp (623-633), 3 the equal
// term of the multi-digit order comparisons (537-538).
void tref_arc_digit_lvl1(uint32_t *res, int op, const uint32_t *trlwe, const double *trgswfft)
{
    using P = lvl1param;
    TRLWE<P> in, prod, mul;
    TLWE<P> r;
    auto *g = new TRGSWFFT<P>;
    std::memcpy(in.data(), trlwe, sizeof(in));
    std::memcpy(g->data(), trgswfft, sizeof(*g));
    trgswfftExternalProduct<P>(prod, in, *g);
    delete g;
    if (op == 2 || op == 3) {
        SampleExtractIndex<P>(r, prod, 0);
        if (op == 2) {
            for (size_t i = 0; i <= P::n; i++) r[i] = 2 * r[i];
            r[P::n] -= P::μ;
        }
    } else {
        Polynomial<P> test_plaintext;
        for (size_t i = 0; i < P::n; i++) test_plaintext[i] = 1;
        if (op == 1) test_plaintext[0] = P::plain_modulus - 1;
        PolyMul<P>(mul[0], prod[0], test_plaintext);
        PolyMul<P>(mul[1], prod[1], test_plaintext);
        SampleExtractIndex<P>(r, mul, 0);
        if (op == 0)
            for (size_t i = 0; i <= P::n; i++) r[i] = -r[i];
    }
    std::memcpy(res, r.data(), sizeof(r));
}

// ---- PBS / IKS / gates ------------------------------------------------------
void tref_pbs01(void *p, uint32_t *out, const uint32_t *in0, const uint32_t *tv)
{
    RefCtx *c = static_cast<RefCtx *>(p);
    TLWE<lvl0param> x;
    TLWE<lvl1param> r;
    Polynomial<lvl1param> t;
    std::memcpy(x.data(), in0, sizeof(x));
    std::memcpy(t.data(), tv, sizeof(t));
    GateBootstrappingTLWE2TLWEFFT<lvl01param>(r, x, *c->ek.bkfftlvl01, t);
    std::memcpy(out, r.data(), sizeof(r));
}

void tref_pbs02(void *p, uint64_t *out, const uint32_t *in0, const uint64_t *tv)
{
    RefCtx *c = static_cast<RefCtx *>(p);
    TLWE<lvl0param> x;
    TLWE<lvl2param> r;
    Polynomial<lvl2param> t;
    std::memcpy(x.data(), in0, sizeof(x));
    std::memcpy(t.data(), tv, sizeof(t));
    GateBootstrappingTLWE2TLWEFFT<lvl02param>(r, x, *c->ek.bkfftlvl02, t);
    std::memcpy(out, r.data(), sizeof(r));
}

void tref_iks10(void *p, uint32_t *out, const uint32_t *in)
{
    RefCtx *c = static_cast<RefCtx *>(p);
    TLWE<lvl1param> x;
    TLWE<lvl0param> r;
    std::memcpy(x.data(), in, sizeof(x));
    IdentityKeySwitch<lvl10param>(r, x, *c->ksk10);
    std::memcpy(out, r.data(), sizeof(r));
}

void tref_iks20(void *p, uint32_t *out, const uint64_t *in)
{
    RefCtx *c = static_cast<RefCtx *>(p);
    TLWE<lvl2param> x;
    TLWE<lvl0param> r;
    std::memcpy(x.data(), in, sizeof(x));
    IdentityKeySwitch<lvl20param>(r, x, *c->ksk20);
    std::memcpy(out, r.data(), sizeof(r));
}

void tref_iks21(void *p, uint32_t *out, const uint64_t *in)
{
    RefCtx *c = static_cast<RefCtx *>(p);
    TLWE<lvl2param> x;
    TLWE<lvl1param> r;
    std::memcpy(x.data(), in, sizeof(x));
    IdentityKeySwitch<lvl21param>(r, x, *c->ksk21);
    std::memcpy(out, r.data(), sizeof(r));
}

// HomNAND over lvl1 ciphertexts (thirdparty/TFHEpp/src/gate.cpp:50-65 with
// GateBootstrapping<lvl1> at gatebootstrapping.hpp:150-158: IKS10 then PBS01).
void tref_homnand(void *p, uint32_t *out, const uint32_t *ca, const uint32_t *cb)
{
    RefCtx *c = static_cast<RefCtx *>(p);
    TLWE<lvl1param> a, b, r;
    std::memcpy(a.data(), ca, sizeof(a));
    std::memcpy(b.data(), cb, sizeof(b));
    HomNAND<lvl1param>(r, a, b, c->ek);
    std::memcpy(out, r.data(), sizeof(r));
}

// n independent HomNANDs on `nthreads` host threads (row-parallel, as the
// reference's query drivers run them under `omp parallel for`).
void tref_homnand_batch(void *p, uint32_t *out, const uint32_t *ca, const uint32_t *cb,
                        int n, int nthreads)
{
    const size_t w = lvl1param::n + 1;
    std::atomic<int> next(0);
    auto work = [&]() {
        for (;;) {
            int i = next.fetch_add(1);
            if (i >= n) break;
            tref_homnand(p, out + i * w, ca + i * w, cb + i * w);
        }
    };
    if (nthreads <= 1) { work(); return; }
    std::vector<std::thread> th;
    for (int t = 0; t < nthreads; t++) th.emplace_back(work);
    for (auto &t : th) t.join();
}

void tref_pbs01_batch(void *p, uint32_t *out, const uint32_t *in0, const uint32_t *tv,
                      int n, int nthreads)
{
    std::atomic<int> next(0);
    auto work = [&]() {
        for (;;) {
            int i = next.fetch_add(1);
            if (i >= n) break;
            tref_pbs01(p, out + (size_t)i * (lvl1param::n + 1),
                       in0 + (size_t)i * (lvl0param::n + 1), tv);
        }
    };
    if (nthreads <= 1) { work(); return; }
    std::vector<std::thread> th;
    for (int t = 0; t < nthreads; t++) th.emplace_back(work);
    for (auto &t : th) t.join();
}

// ---- HEDB CPU operators (src/HEDB/comparison/HomCompare.h:14-75) -------------
// op: 0 greater_than, 1 greater_than_equal, 2 less_than, 3 less_than_equal, 4 equal
void tref_compare_lvl1(void *p, uint32_t *res, const uint32_t *c1, const uint32_t *c2,
                       int op, uint32_t plain_bits, int logic)
{
    RefCtx *c = static_cast<RefCtx *>(p);
    TLWE<lvl1param> a, b;
    TLWELvl1 r;
    std::memcpy(a.data(), c1, sizeof(a));
    std::memcpy(b.data(), c2, sizeof(b));
    bool rt = logic != 0;
    switch (op) {
    case 0: HEDB::greater_than<lvl1param>(a, b, r, plain_bits, c->ek, rt); break;
    case 1: HEDB::greater_than_equal<lvl1param>(a, b, r, plain_bits, c->ek, rt); break;
    case 2: HEDB::less_than<lvl1param>(a, b, r, plain_bits, c->ek, rt); break;
    case 3: HEDB::less_than_equal<lvl1param>(a, b, r, plain_bits, c->ek, rt); break;
    default: HEDB::equal<lvl1param>(a, b, r, plain_bits, c->ek, rt); break;
    }
    std::memcpy(res, r.data(), sizeof(r));
}

void tref_compare_lvl2(void *p, uint32_t *res, const uint64_t *c1, const uint64_t *c2,
                       int op, uint32_t plain_bits, int logic)
{
    RefCtx *c = static_cast<RefCtx *>(p);
    TLWE<lvl2param> a, b;
    TLWELvl1 r;
    std::memcpy(a.data(), c1, sizeof(a));
    std::memcpy(b.data(), c2, sizeof(b));
    bool rt = logic != 0;
    switch (op) {
    case 0: HEDB::greater_than<lvl2param>(a, b, r, plain_bits, c->ek, rt); break;
    case 1: HEDB::greater_than_equal<lvl2param>(a, b, r, plain_bits, c->ek, rt); break;
    case 2: HEDB::less_than<lvl2param>(a, b, r, plain_bits, c->ek, rt); break;
    case 3: HEDB::less_than_equal<lvl2param>(a, b, r, plain_bits, c->ek, rt); break;
    default: HEDB::equal<lvl2param>(a, b, r, plain_bits, c->ek, rt); break;
    }
    std::memcpy(res, r.data(), sizeof(r));
}

// n rows of tref_compare_lvl1 / tref_compare_lvl2 on `nthreads` host threads
// (row-parallel, as the reference's query drivers run the HEDB operators under
// `omp parallel for`); rows are back to back in c1, c2 and res.
void tref_compare_lvl1_batch(void *p, uint32_t *res, const uint32_t *c1, const uint32_t *c2, int n,
                             int op, uint32_t plain_bits, int logic, int nthreads)
{
    const size_t w = lvl1param::n + 1;
    std::atomic<int> next(0);
    auto work = [&]() {
        for (;;) {
            const int i = next.fetch_add(1);
            if (i >= n) break;
            tref_compare_lvl1(p, res + i * w, c1 + i * w, c2 + i * w, op, plain_bits, logic);
        }
    };
    if (nthreads <= 1) { work(); return; }
    std::vector<std::thread> th;
    for (int t = 0; t < nthreads; t++) th.emplace_back(work);
    for (auto &t : th) t.join();
}

void tref_compare_lvl2_batch(void *p, uint32_t *res, const uint64_t *c1, const uint64_t *c2, int n,
                             int op, uint32_t plain_bits, int logic, int nthreads)
{
    const size_t w2 = lvl2param::n + 1, w1 = lvl1param::n + 1;
    std::atomic<int> next(0);
    auto work = [&]() {
        for (;;) {
            const int i = next.fetch_add(1);
            if (i >= n) break;
            tref_compare_lvl2(p, res + i * w1, c1 + i * w2, c2 + i * w2, op, plain_bits, logic);
        }
    };
    if (nthreads <= 1) { work(); return; }
    std::vector<std::thread> th;
    for (int t = 0; t < nthreads; t++) th.emplace_back(work);
    for (auto &t : th) t.join();
}

void tref_homand(void *p, uint32_t *res, const uint32_t *ca, const uint32_t *cb, int logic)
{
    RefCtx *c = static_cast<RefCtx *>(p);
    TLWELvl1 a, b, r;
    std::memcpy(a.data(), ca, sizeof(a));
    std::memcpy(b.data(), cb, sizeof(b));
    HEDB::HomAND(r, a, b, c->ek, logic != 0);
    std::memcpy(res, r.data(), sizeof(r));
}

// Whole ArcEDB comparisons of n rows of D digits on `nthreads` host threads,
// as comparable.cpp composes them from the single-digit functions (order
// comparisons 525-557 / 668-698: equal term, doubled high digit, lower
// result, mu/2, IdentityKeySwitch<lvl10>, GateBootstrappingTLWE2TLWEFFT<lvl01>
// with mu; equality 635-650: TFHEpp::HomAND).  The top digit's external
// product runs twice per digit, as there.  trlwe: D x n x [2][1024];
// trgswfft: D x n TRGSWFFT<lvl1param>; op 0 gt, 1 lt, 2 eq.
void tref_arc_compare_batch(void *p, uint32_t *res, int op, const uint32_t *trlwe, const double *trgswfft,
                            int n, int D, int nthreads)
{
    using P = lvl1param;
    RefCtx *c = static_cast<RefCtx *>(p);
    const size_t tw = 2 * P::n, gw = sizeof(TRGSWFFT<P>) / sizeof(double), w = P::n + 1;
    std::atomic<int> next(0);
    auto work = [&]() {
        for (;;) {
            const int i = next.fetch_add(1);
            if (i >= n) break;
            auto x = [&](int d) { return trlwe + ((size_t)d * n + i) * tw; };
            auto g = [&](int d) { return trgswfft + ((size_t)d * n + i) * gw; };
            TLWE<P> r, hi, eq, sum;
            TLWE<lvl0param> l0;
            tref_arc_digit_lvl1(r.data(), op, x(0), g(0));
            for (int d = 1; d < D; ++d) {
                tref_arc_digit_lvl1(hi.data(), op, x(d), g(d));
                if (op == 2) {
                    HomAND<P>(sum, r, hi, c->ek);
                    r = sum;
                    continue;
                }
                tref_arc_digit_lvl1(eq.data(), 3, x(d), g(d));
                for (size_t k = 0; k <= P::n; k++) sum[k] = eq[k] + 2 * hi[k] + r[k];
                sum[P::n] += P::μ >> 1;
                IdentityKeySwitch<lvl10param>(l0, sum, *c->ek.iksklvl10);
                GateBootstrappingTLWE2TLWEFFT<lvl01param>(r, l0, *c->ek.bkfftlvl01, μpolygen<P, P::μ>());
            }
            std::memcpy(res + (size_t)i * w, r.data(), sizeof(r));
        }
    };
    if (nthreads <= 1) { work(); return; }
    std::vector<std::thread> th;
    for (int t = 0; t < nthreads; t++) th.emplace_back(work);
    for (auto &t : th) t.join();
}

}  // extern "C"
