// Drop-in check of include/cufhedb_b200/cuhedb_gpu.hpp.
//
// The flow of the reference's own GPU programs (test/HE3_Query/HomComp.cu,
// test/Bootstrapping.cu): TFHEpp generates the keys, cufftlvl1 / cufftlvl2
// .LoadBK upload the bootstrapping keys, and the cuHEDB:: operators run with
// TFHEpp ciphertexts and stream ids.  Only the include differs.  Every GPU
// result is decrypted and checked against the plaintext and against the
// reference's CPU operators (HEDB::greater_than etc., TFHEpp's bootstrap and
// external product) on the same ciphertexts.
//
//   dropin_check           lvl1 keys: transforms, external product, PBS01,
//                          gates, LOG_to_ARI / log_rescale, HomMSB, compares
//   dropin_check --lvl2    also lvl2 keys (about 17 GB of host memory for the
//                          TFHEpp key-switching keys): PBS02, lvl2 compares
//
// Exit status 0 means every check passed.
#include "HEDB/comparison/comparison.h"
#include "HEDB/utils/types.h"
#include "cufhedb_b200/cuhedb_gpu.hpp"

#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <random>
#include <string>
#include <thread>
#include <vector>

namespace {

int g_failed = 0;

void report(const char *what, bool ok, const std::string &detail = "")
{
    std::printf("%-58s %s %s\n", what, ok ? "PASS" : "FAIL", detail.c_str());
    if (!ok) ++g_failed;
}

double seconds_since(std::chrono::steady_clock::time_point t0)
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

template <typename T>
int64_t torus_diff(T a, T b)
{
    using S = std::make_signed_t<T>;
    return (int64_t)(S)(a - b);
}

template <class P>
TFHEpp::TLWE<P> enc_int(typename P::T v, uint32_t bits, const TFHESecretKey &sk)
{
    const uint32_t scale_bits = std::numeric_limits<typename P::T>::digits - bits - 1;
    return TFHEpp::tlweSymInt32Encrypt<P>(v, P::α, std::pow(2., scale_bits), sk.key.get<P>());
}

bool dec_logic(const TLWELvl1 &c, const TFHESecretKey &sk)
{
    return TFHEpp::tlweSymDecrypt<Lvl1>(c, sk.key.get<Lvl1>());
}

uint32_t dec_arith(const TLWELvl1 &c, const TFHESecretKey &sk)
{
    return TFHEpp::tlweSymInt32Decrypt<Lvl1>(c, std::pow(2., 31), sk.key.get<Lvl1>()) & 1u;
}

void check_transforms(std::mt19937_64 &rng)
{
    TFHEpp::Polynomial<Lvl1> a;
    for (auto &x : a) x = (uint32_t)rng();
    TFHEpp::PolynomialInFD<Lvl1> ref_fd, gpu_fd;
    TFHEpp::TwistIFFT<Lvl1>(ref_fd, a);
    cufftlvl1.ifft_st(gpu_fd, a, 0);
    double err = 0, mag = 0;
    for (int i = 0; i < Lvl1::n; i++) {
        err = std::max(err, std::fabs(ref_fd[i] - gpu_fd[i]));
        mag = std::max(mag, std::fabs(ref_fd[i]));
    }
    report("cufftlvl1.ifft_st vs TFHEpp::TwistIFFT<Lvl1>", err <= 1e-13 * mag);
    TFHEpp::Polynomial<Lvl1> back_gpu, back_ref;
    cufftlvl1.fft_st(back_gpu, ref_fd, 1);
    TFHEpp::TwistFFT<Lvl1>(back_ref, ref_fd);
    int64_t d_ref = 0, d_in = 0;
    for (int i = 0; i < Lvl1::n; i++) {
        d_ref = std::max(d_ref, std::abs(torus_diff(back_gpu[i], back_ref[i])));
        d_in = std::max(d_in, std::abs(torus_diff(back_gpu[i], a[i])));
    }
    report("cufftlvl1.fft_st vs TFHEpp::TwistFFT<Lvl1> (+-1)", d_ref <= 1 && d_in <= 1);
}

void check_extprod(std::mt19937_64 &rng, const TFHESecretKey &sk)
{
    int64_t worst = 0;
    for (int t = 0; t < 3; t++) {
        TFHEpp::Polynomial<Lvl1> m{};
        m[0] = (uint32_t)(rng() & 1);
        auto g = TFHEpp::trgswSymEncrypt<Lvl1>(m, Lvl1::α, sk.key.get<Lvl1>());
        auto gfft = TFHEpp::ApplyFFT2trgsw<Lvl1>(g);
        TRLWELvl1 c, ref, gpu;
        for (auto &row : c)
            for (auto &x : row) x = (uint32_t)rng();
        TFHEpp::trgswfftExternalProduct<Lvl1>(ref, c, gfft);
        cufftlvl1.ExternalProduct_st(gpu, c, gfft, (uint32_t)t);
        for (int k = 0; k < 2; k++)
            for (int i = 0; i < Lvl1::n; i++) worst = std::max(worst, std::abs(torus_diff(gpu[k][i], ref[k][i])));
    }
    report("cufftlvl1.ExternalProduct_st vs trgswfftExternalProduct (+-1)", worst <= 1,
           "max |diff| " + std::to_string(worst));
}

void check_pbs01(std::mt19937_64 &rng, const TFHESecretKey &sk, const TFHEEvalKey &ek)
{
    const uint32_t mu = Lvl1::μ;
    int bad = 0, disagree = 0;
    int64_t worst = 0;
    for (int t = 0; t < 24; t++) {
        const bool bit = rng() & 1;
        auto in = TFHEpp::tlweSymEncrypt<TFHEpp::lvl0param>(bit ? TFHEpp::lvl0param::μ : -TFHEpp::lvl0param::μ,
                                                            TFHEpp::lvl0param::α, sk.key.get<TFHEpp::lvl0param>());
        TLWELvl1 gpu, cpu;
        cufftlvl1.GateBootstrappingTLWE2TLWEFFT_st(gpu, in, mu, (uint32_t)(t % 4));
        TFHEpp::GateBootstrappingTLWE2TLWEFFT<TFHEpp::lvl01param>(cpu, in, *ek.bkfftlvl01,
                                                                  TFHEpp::μpolygen<Lvl1, Lvl1::μ>());
        bad += dec_logic(gpu, sk) != bit;
        disagree += dec_logic(cpu, sk) != dec_logic(gpu, sk);
        // same keys, same input: the two phases differ only by transform rounding
        uint32_t pg = gpu[Lvl1::n], pc = cpu[Lvl1::n];
        for (int i = 0; i < Lvl1::n; i++) {
            pg -= gpu[i] * sk.key.get<Lvl1>()[i];
            pc -= cpu[i] * sk.key.get<Lvl1>()[i];
        }
        worst = std::max(worst, std::abs(torus_diff(pg, pc)));
    }
    report("cufftlvl1.GateBootstrappingTLWE2TLWEFFT_st decrypts (24 bits)", bad == 0 && disagree == 0);
    report("  phase vs TFHEpp::GateBootstrappingTLWE2TLWEFFT < 2^25", worst < (1 << 25),
           "max |diff| " + std::to_string(worst));
}

void check_gates(std::mt19937_64 &rng, const TFHESecretKey &sk, const TFHEEvalKey &ek)
{
    int bad_and = 0, bad_or = 0, bad_l2a = 0, bad_resc = 0;
    for (int t = 0; t < 16; t++) {
        const bool a = rng() & 1, b = rng() & 1;
        // LOGIC encodings: +-2^29
        auto ca = TFHEpp::tlweSymEncrypt<Lvl1>(a ? Lvl1::μ : -Lvl1::μ, Lvl1::α, sk.key.get<Lvl1>());
        auto cb = TFHEpp::tlweSymEncrypt<Lvl1>(b ? Lvl1::μ : -Lvl1::μ, Lvl1::α, sk.key.get<Lvl1>());
        TLWELvl1 r, rc;
        cuHEDB::HomAND(r, ca, cb, ek, LOGIC, 0);
        bad_and += dec_logic(r, sk) != (a && b);
        cuHEDB::HomOR(r, ca, cb, ek, LOGIC, 1);
        bad_or += dec_logic(r, sk) != (a || b);
        cuHEDB::LOG_to_ARI(r, ca, ek, 2);
        TFHEpp::LOG_to_ARI(rc, ca, ek);
        bad_l2a += dec_arith(r, sk) != (uint32_t)a || dec_arith(rc, sk) != (uint32_t)a;
        // the result is the bit at scale 2^scale_bits; scale_bits = 28 keeps it
        // far above the output noise (rms ~2^22), so both decrypt exactly
        cuHEDB::log_rescale(r, ca, 28, ek, 3);
        TFHEpp::log_rescale(rc, ca, 28, ek);
        const uint32_t vg = TFHEpp::tlweSymInt32Decrypt<Lvl1>(r, std::pow(2., 28), sk.key.get<Lvl1>());
        const uint32_t vc = TFHEpp::tlweSymInt32Decrypt<Lvl1>(rc, std::pow(2., 28), sk.key.get<Lvl1>());
        bad_resc += vg != vc || vg != (uint32_t)a;
    }
    report("cuHEDB::HomAND (LOGIC, 16 pairs)", bad_and == 0);
    report("cuHEDB::HomOR (LOGIC, 16 pairs)", bad_or == 0);
    report("cuHEDB::LOG_to_ARI == TFHEpp::LOG_to_ARI == plaintext", bad_l2a == 0);
    report("cuHEDB::log_rescale(28) == TFHEpp::log_rescale(28) == plaintext", bad_resc == 0);
}

void check_msb_lvl1(std::mt19937_64 &rng, const TFHESecretKey &sk, const TFHEEvalKey &ek)
{
    for (uint32_t bits : {5u, 8u, 10u}) {
        int bad = 0;
        for (int t = 0; t < 8; t++) {
            // a value of `bits` bits whose sign bit is the MSB
            const uint32_t v = (uint32_t)(rng() & ((1u << bits) - 1));
            const uint32_t scale_bits = 32 - bits;
            auto c = TFHEpp::tlweSymInt32Encrypt<Lvl1>(v, Lvl1::α, std::pow(2., scale_bits), sk.key.get<Lvl1>());
            TLWELvl1 r, rc;
            cuHEDB::HomMSB(r, c, bits, ek, LOGIC, (uint32_t)t);
            HEDB::HomMSB(rc, c, bits, ek, LOGIC);
            bad += dec_logic(r, sk) != dec_logic(rc, sk) || dec_logic(r, sk) != (bool)(v >> (bits - 1));
        }
        report(("cuHEDB::HomMSB<lvl1> " + std::to_string(bits) + " bits == HEDB::HomMSB == MSB").c_str(), bad == 0);
    }
    bool threw = false;
    try {
        TLWELvl1 r{}, c{};
        cuHEDB::HomMSB(r, c, 11, ek, LOGIC, 0);
    } catch (const std::invalid_argument &) {
        threw = true;
    }
    report("cuHEDB::HomMSB<lvl1> 11 bits throws invalid_argument", threw);
}

bool plain_cmp(int op, uint64_t x, uint64_t y)
{
    switch (op) {
    case 0: return x > y;
    case 1: return x >= y;
    case 2: return x < y;
    case 3: return x <= y;
    default: return x == y;
    }
}

template <class P>
void gpu_cmp(int op, TFHEpp::TLWE<P> &a, TFHEpp::TLWE<P> &b, TLWELvl1 &r, uint32_t bits, TFHEEvalKey &ek,
             bool rt, uint32_t sid)
{
    switch (op) {
    case 0: cuHEDB::greater_than<P>(a, b, r, bits, ek, rt, sid); break;
    case 1: cuHEDB::greater_than_equal<P>(a, b, r, bits, ek, rt, sid); break;
    case 2: cuHEDB::less_than<P>(a, b, r, bits, ek, rt, sid); break;
    case 3: cuHEDB::less_than_equal<P>(a, b, r, bits, ek, rt, sid); break;
    default: cuHEDB::equal<P>(a, b, r, bits, ek, rt, sid); break;
    }
}

template <class P>
void cpu_cmp(int op, TFHEpp::TLWE<P> &a, TFHEpp::TLWE<P> &b, TLWELvl1 &r, uint32_t bits, TFHEEvalKey &ek, bool rt)
{
    switch (op) {
    case 0: HEDB::greater_than<P>(a, b, r, bits, ek, rt); break;
    case 1: HEDB::greater_than_equal<P>(a, b, r, bits, ek, rt); break;
    case 2: HEDB::less_than<P>(a, b, r, bits, ek, rt); break;
    case 3: HEDB::less_than_equal<P>(a, b, r, bits, ek, rt); break;
    default: HEDB::equal<P>(a, b, r, bits, ek, rt); break;
    }
}

const char *OPS[] = {"greater_than", "greater_than_equal", "less_than", "less_than_equal", "equal"};

template <class P>
void check_compare(std::mt19937_64 &rng, const TFHESecretKey &sk, TFHEEvalKey &ek, uint32_t bits, int pairs,
                   int cpu_pairs)
{
    const uint64_t mask = (bits >= 64 ? ~0ull : (1ull << bits) - 1);
    for (int op = 0; op < 5; op++)
        for (bool rt : {LOGIC, ARITHMETIC}) {
            int bad = 0, bad_cpu = 0;
            for (int t = 0; t < pairs; t++) {
                const uint64_t x = rng() & mask;
                const uint64_t y = (t % 4 == 0) ? x : (rng() & mask);
                auto cx = enc_int<P>((typename P::T)x, bits, sk);
                auto cy = enc_int<P>((typename P::T)y, bits, sk);
                TLWELvl1 r;
                gpu_cmp<P>(op, cx, cy, r, bits, ek, rt, (uint32_t)t);
                const bool got = rt == LOGIC ? dec_logic(r, sk) : dec_arith(r, sk);
                bad += got != plain_cmp(op, x, y);
                if (t < cpu_pairs) {
                    TLWELvl1 rc;
                    cpu_cmp<P>(op, cx, cy, rc, bits, ek, rt);
                    const bool want = rt == LOGIC ? dec_logic(rc, sk) : dec_arith(rc, sk);
                    bad_cpu += want != got;
                }
            }
            std::string what = std::string("cuHEDB::") + OPS[op] + "<Lvl" + (P::n == 1024 ? "1" : "2") + "> " +
                               std::to_string(bits) + " bits " + (rt == LOGIC ? "LOGIC" : "ARITH");
            report(what.c_str(), bad == 0 && bad_cpu == 0,
                   std::to_string(pairs) + " pairs, " + std::to_string(cpu_pairs) + " vs HEDB CPU");
        }
}

template <class P>
void check_batch_compare(std::mt19937_64 &rng, const TFHESecretKey &sk, const TFHEEvalKey &ek, uint32_t bits,
                         int rows, int precision)
{
    const uint64_t mask = (1ull << bits) - 1;
    std::vector<TFHEpp::TLWE<P>> col(rows), thr(rows);
    std::vector<uint64_t> x(rows);
    const uint64_t c = rng() & mask;
    auto cthr = enc_int<P>((typename P::T)c, bits, sk);
    for (int i = 0; i < rows; i++) {
        x[i] = rng() & mask;
        col[i] = enc_int<P>((typename P::T)x[i], bits, sk);
        thr[i] = cthr;
    }
    std::vector<TLWELvl1> res;
    cuHEDB::batch::compare<P>(3, col, thr, res, bits, ek, LOGIC, precision);   // warm-up
    auto t0 = std::chrono::steady_clock::now();
    cuHEDB::batch::compare<P>(3, col, thr, res, bits, ek, LOGIC, precision);
    const double s = seconds_since(t0);
    int bad = 0;
    for (int i = 0; i < rows; i++) bad += dec_logic(res[i], sk) != (x[i] <= c);
    char buf[96];
    std::snprintf(buf, sizeof buf, "%d rows, %.0f rows/s incl. copies", rows, rows / s);
    std::string what = std::string("cuHEDB::batch::compare<Lvl") + (P::n == 1024 ? "1" : "2") + "> le " +
                       std::to_string(bits) + " bits " + (precision == CUFHEDB_SPLIT32 ? "split32" : "fp64");
    report(what.c_str(), bad == 0, buf);
}

// The reference's query programs' row loop (test/HE3_Query/TPCH_Q6.cu:179-193):
// `omp parallel for num_threads(T)`, every thread calling the one-row
// operator with its own stream id, each call returning with its row's result.
// parallel_rows() is that loop's static schedule on T host threads (thread t
// takes the t-th contiguous block of rows, stream id t).
// Concurrent calls are coalesced into batched launches; here the rows per
// second through that unchanged API are set beside cuHEDB::batch::compare on
// the same rows, and every result of both is decrypted against plaintext.
template <typename F>
void parallel_rows(int rows, int threads, F &&f)
{
    std::vector<std::thread> th;
    for (int t = 0; t < threads; t++)
        th.emplace_back([&, t] {
            const int lo = (int)((long)rows * t / threads), hi = (int)((long)rows * (t + 1) / threads);
            for (int i = lo; i < hi; i++) f(i, (uint32_t)t);
        });
    for (auto &x : th) x.join();
}

template <class P>
void check_row_loop(std::mt19937_64 &rng, const TFHESecretKey &sk, TFHEEvalKey &ek, uint32_t bits, int rows,
                    int threads)
{
    const uint64_t mask = (1ull << bits) - 1;
    const uint64_t c = rng() & mask;
    auto cthr = enc_int<P>((typename P::T)c, bits, sk);
    std::vector<TFHEpp::TLWE<P>> col(rows), thr(rows, cthr);
    std::vector<uint64_t> x(rows);
    for (int i = 0; i < rows; i++) {
        x[i] = rng() & mask;
        col[i] = enc_int<P>((typename P::T)x[i], bits, sk);
    }
    std::vector<TLWELvl1> res(rows);
    // warm-up: one round of `threads` rows
    parallel_rows(std::min(threads, rows), threads, [&](int i, uint32_t sid) {
        cuHEDB::less_than_equal<P>(col[i], thr[i], res[i], bits, ek, LOGIC, sid);
    });
    auto t0 = std::chrono::steady_clock::now();
    parallel_rows(rows, threads, [&](int i, uint32_t sid) {
        cuHEDB::less_than_equal<P>(col[i], thr[i], res[i], bits, ek, LOGIC, sid);
    });
    const double s_rows = seconds_since(t0);
    int bad = 0;
    for (int i = 0; i < rows; i++) bad += dec_logic(res[i], sk) != (x[i] <= c);
    std::vector<TLWELvl1> bres;
    t0 = std::chrono::steady_clock::now();
    cuHEDB::batch::compare<P>(3, col, thr, bres, bits, ek, LOGIC);
    const double s_batch = seconds_since(t0);
    int bad_batch = 0;
    for (int i = 0; i < rows; i++) bad_batch += dec_logic(bres[i], sk) != (x[i] <= c);
    char buf[160];
    std::snprintf(buf, sizeof buf, "%.0f rows/s one-row calls, %.0f rows/s batch (ratio %.2f)", rows / s_rows,
                  rows / s_batch, s_rows / s_batch);
    std::string what = std::string("row loop: ") + std::to_string(threads) + " threads x " + std::to_string(rows) +
                       " less_than_equal<Lvl" + (P::n == 1024 ? "1" : "2") + "> " + std::to_string(bits) + " bits";
    report(what.c_str(), bad == 0 && bad_batch == 0, buf);
}

void check_pbs02(std::mt19937_64 &rng, const TFHESecretKey &sk)
{
    int bad = 0;
    for (int t = 0; t < 8; t++) {
        const bool bit = rng() & 1;
        auto in = TFHEpp::tlweSymEncrypt<TFHEpp::lvl0param>(bit ? TFHEpp::lvl0param::μ : -TFHEpp::lvl0param::μ,
                                                            TFHEpp::lvl0param::α, sk.key.get<TFHEpp::lvl0param>());
        TLWELvl2 out;
        cufftlvl2.GateBootstrappingTLWE2TLWEFFT_st(out, in, Lvl2::μ, (uint32_t)t);
        bad += TFHEpp::tlweSymDecrypt<Lvl2>(out, sk.key.get<Lvl2>()) != bit;
    }
    report("cufftlvl2.GateBootstrappingTLWE2TLWEFFT_st decrypts (8 bits)", bad == 0);
}

}  // namespace

// The reference's query programs call the per-row operators from an OpenMP
// row loop, each thread with its own stream id (test/HE3_Query/TPCH_Q6.cu:
// 179-181).  Here: 8 host threads, each running a mix of operators on its own
// stream id at the same time, every result decrypted against the plaintext.
void check_threads(const TFHESecretKey &sk, TFHEEvalKey &ek)
{
    constexpr int NT = 8, ROWS = 12;
    std::atomic<int> bad{0};
    std::vector<std::thread> th;
    for (int t = 0; t < NT; t++)
        th.emplace_back([&, t] {
            std::mt19937_64 r(1000 + t);
            const uint32_t sid = 4 + (uint32_t)t;
            for (int i = 0; i < ROWS; i++) {
                const bool a = r() & 1, b = r() & 1;
                auto ca = TFHEpp::tlweSymEncrypt<Lvl1>(a ? Lvl1::μ : -Lvl1::μ, Lvl1::α, sk.key.get<Lvl1>());
                auto cb = TFHEpp::tlweSymEncrypt<Lvl1>(b ? Lvl1::μ : -Lvl1::μ, Lvl1::α, sk.key.get<Lvl1>());
                TLWELvl1 res;
                cuHEDB::HomAND(res, ca, cb, ek, LOGIC, sid);
                bad += dec_logic(res, sk) != (a && b);
                const uint32_t x = r() % 64, y = r() % 64;
                auto cx = enc_int<Lvl1>(x, 6, sk), cy = enc_int<Lvl1>(y, 6, sk);
                cuHEDB::less_than_equal<Lvl1>(cx, cy, res, 6, ek, LOGIC, sid);
                bad += dec_logic(res, sk) != (x <= y);
                auto in = TFHEpp::tlweSymEncrypt<TFHEpp::lvl0param>(a ? TFHEpp::lvl0param::μ : -TFHEpp::lvl0param::μ,
                                                                    TFHEpp::lvl0param::α,
                                                                    sk.key.get<TFHEpp::lvl0param>());
                cufftlvl1.GateBootstrappingTLWE2TLWEFFT_st(res, in, Lvl1::μ, sid);
                bad += dec_logic(res, sk) != a;
            }
        });
    for (auto &x : th) x.join();
    report("8 host threads x 12 rows, own stream ids (AND, <=, PBS)", bad == 0,
           "wrong " + std::to_string(bad.load()));
}

int main(int argc, char **argv)
{
    const bool lvl2 = argc > 1 && std::strcmp(argv[1], "--lvl2") == 0;
    warmupGPU();
    std::mt19937_64 rng(20240611);

    auto t0 = std::chrono::steady_clock::now();
    auto sk = std::make_unique<TFHESecretKey>();
    auto ek = std::make_unique<TFHEEvalKey>();
    ek->emplacebkfft<Lvl01>(*sk);
    ek->emplaceiksk<Lvl10>(*sk);
    if (lvl2) {
        ek->emplacebkfft<Lvl02>(*sk);
        ek->emplaceiksk<Lvl20>(*sk);
        ek->emplaceiksk<Lvl21>(*sk);
    }
    std::printf("TFHEpp key generation: %.1f s\n", seconds_since(t0));

    t0 = std::chrono::steady_clock::now();
    cufftlvl1.LoadBK(*ek->bkfftlvl01);
    if (lvl2) cufftlvl2.LoadBK(*ek->bkfftlvl02);
    std::printf("LoadBK: %.2f s\n", seconds_since(t0));

    try {
        check_transforms(rng);
        check_extprod(rng, *sk);
        check_pbs01(rng, *sk, *ek);
        check_gates(rng, *sk, *ek);
        check_msb_lvl1(rng, *sk, *ek);
        check_compare<Lvl1>(rng, *sk, *ek, 6, 8, 2);
        check_batch_compare<Lvl1>(rng, *sk, *ek, 6, 512, CUFHEDB_FP64);
        check_batch_compare<Lvl1>(rng, *sk, *ek, 6, 512, CUFHEDB_SPLIT32);
        check_threads(*sk, *ek);
        check_row_loop<Lvl1>(rng, *sk, *ek, 6, 16384, 48);
        check_row_loop<Lvl1>(rng, *sk, *ek, 6, 16384, 1024);
        if (lvl2) {
            check_pbs02(rng, *sk);
            check_compare<Lvl2>(rng, *sk, *ek, 20, 3, 1);
            // 26 bits: the ImExtractMSB29 chain; near 30 bits a compare sits at
            // the noise floor of the lvl2 parameters with randomly drawn keys
            check_compare<Lvl2>(rng, *sk, *ek, 26, 2, 0);
            check_batch_compare<Lvl2>(rng, *sk, *ek, 20, 256, CUFHEDB_FP64);
            check_row_loop<Lvl2>(rng, *sk, *ek, 20, 4096, 48);
            check_row_loop<Lvl2>(rng, *sk, *ek, 20, 4096, 1024);
        }
    } catch (const std::exception &e) {
        std::printf("exception: %s\n", e.what());
        return 2;
    }
    std::printf("%s: %d failed\n", g_failed ? "FAILED" : "OK", g_failed);
    return g_failed ? 1 : 0;
}
