/*
 * TEST ORACLE -- not part of the product.
 *
 * A plain-C restatement of the TFHE programmable-bootstrapping path of
 * cuFHEDB / TFHEpp, used only by tests/, by __graft_entry__.smoke() as the
 * checker, and by bench.py's CPU-baseline leg.  The product library
 * (cufhedb_b200) never links or calls it.
 *
 * Parity pin: every restated function is checked in tests/ against the
 * reference's own TFHEpp compiled from its sources (oracle/_ref, see
 * oracle/Makefile) and against committed golden vectors (tests/golden/).
 *
 * Parameter set: thirdparty/TFHEpp/include/params/128bit.hpp:7-83
 *   lvl0 n=672, alpha=2^-16, u32 torus
 *   lvl1 N=1024, k=1, l=3, Bgbit=6, alpha=2^-25, u32 torus
 *   lvl2 N=2048, k=1, l=4, Bgbit=9, alpha=2^-52, u64 torus
 *   lvl10 IKS basebit=10 t=2; lvl20 basebit=10 t=2; lvl21 basebit=3 t=10
 *
 * Deterministic key material (not in the reference, whose generator is
 * seeded from std::random_device, thirdparty/TFHEpp/include/utils.hpp:17-22):
 * a counter-based generator draw(seed, stream, ctr) and an integer-only
 * approximate Gaussian (sum of four uniform 32-bit words, scaled), so that the
 * CPU oracle and the GPU key generator produce bit-identical keys.
 */
#ifndef CUFHEDB_B200_TFHE_ORACLE_H
#define CUFHEDB_B200_TFHE_ORACLE_H
#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    ORC_N0 = 672,
    ORC_N1 = 1024, ORC_L1 = 3, ORC_BG1 = 6,
    ORC_N2 = 2048, ORC_L2 = 4, ORC_BG2 = 9,
};

/* generator ---------------------------------------------------------------*/
uint64_t orc_draw(uint64_t seed, uint64_t stream, uint64_t ctr);
int64_t orc_noise(uint64_t seed, uint64_t stream, uint64_t ctr, int64_t scale);

/* secret keys: hamming-weight keys as thirdparty/TFHEpp/src/key.cpp:8-17
 * (512, 512, 1024 draws with replacement). */
void orc_secret_keys(uint64_t seed, uint32_t *s0, uint32_t *s1, uint64_t *s2);

/* encryption under a key; idx selects the counter block within `stream` */
void orc_tlwe32_encrypt(uint32_t *c, int n, uint32_t m, const uint32_t *key,
                        int64_t noise_scale, uint64_t seed, uint64_t stream, uint64_t idx);
void orc_tlwe64_encrypt(uint64_t *c, int n, uint64_t m, const uint64_t *key,
                        int64_t noise_scale, uint64_t seed, uint64_t stream, uint64_t idx);
uint32_t orc_tlwe32_phase(const uint32_t *c, int n, const uint32_t *key);
uint64_t orc_tlwe64_phase(const uint64_t *c, int n, const uint64_t *key);

/* bootstrapping keys (integer TRGSW form, [672][(k+1)l][2][N]) */
void orc_bk01(uint64_t seed, const uint32_t *s0, const uint32_t *s1, uint32_t *bk, int nthreads);
void orc_bk02(uint64_t seed, const uint32_t *s0, const uint64_t *s2, uint64_t *bk, int nthreads);
/* a lvl1 TRLWE of the plaintext polynomial `plain` (trlwe.cpp:30-37) */
void orc_trlwe32_encrypt(uint32_t *out, const uint32_t *plain, const uint32_t *s1, uint64_t seed,
                         uint64_t stream, uint64_t idx);
/* one TRGSW of the monomial-0 message m0 (cloudkey.cpp:11-20, trgsw.cpp:206-222) */
void orc_trgsw32(uint32_t *out, uint32_t m0, const uint32_t *s1, uint64_t seed,
                 uint64_t stream, uint64_t idx);
void orc_trgsw64(uint64_t *out, uint64_t m0, const uint64_t *s2, uint64_t seed,
                 uint64_t stream, uint64_t idx);

/* key-switching keys: one row (a TLWE of the target level) or the full key */
void orc_ksk10_row(uint64_t seed, const uint32_t *s1, const uint32_t *s0, int i, int j, int k, uint32_t *row);
void orc_ksk20_row(uint64_t seed, const uint64_t *s2, const uint32_t *s0, int i, int j, int k, uint32_t *row);
void orc_ksk21_row(uint64_t seed, const uint64_t *s2, const uint32_t *s1, int i, int j, int k, uint32_t *row);
void orc_ksk_full(int kind, uint64_t seed, const uint32_t *s0, const uint32_t *s1,
                  const uint64_t *s2, uint32_t *ksk, int nthreads);
size_t orc_ksk_words(int kind);

/* negacyclic FFT with TFHEpp/spqlios conventions (mulfft.hpp:57-121) */
void orc_twist_ifft32(double *out, const uint32_t *a, int N);
void orc_twist_fft32(uint32_t *out, const double *in, int N);
void orc_twist_ifft64(double *out, const uint64_t *a, int N);
void orc_twist_fft64(uint64_t *out, const double *in, int N);

/* gadget decomposition (trgsw.cpp:9-39) */
void orc_decomp32(uint32_t *out, const uint32_t *poly, int digit);
void orc_decomp64(uint64_t *out, const uint64_t *poly, int digit);

/* external product: FFT form (trgsw.cpp:77-103) and exact integer form */
void orc_extprod32_fft(uint32_t *res, const uint32_t *trlwe, const double *trgswfft);
void orc_extprod64_fft(uint64_t *res, const uint64_t *trlwe, const double *trgswfft);
void orc_extprod32_exact(uint32_t *res, const uint32_t *trlwe, const uint32_t *trgsw);
void orc_extprod64_exact(uint64_t *res, const uint64_t *trlwe, const uint64_t *trgsw);
void orc_trgsw32_fft(double *out, const uint32_t *trgsw);
void orc_trgsw64_fft(double *out, const uint64_t *trgsw);

/* PBS = BlindRotate + SampleExtractIndex(0) (gatebootstrapping.cpp:14-23) */
void orc_blind_rotate01(uint32_t *acc, const uint32_t *in0, const double *bkfft, const uint32_t *tv);
void orc_pbs01(uint32_t *out, const uint32_t *in0, const double *bkfft, const uint32_t *tv);
void orc_pbs02(uint64_t *out, const uint32_t *in0, const double *bkfft, const uint64_t *tv);
void orc_pbs01_exact(uint32_t *out, const uint32_t *in0, const uint32_t *bk, const uint32_t *tv);
/* the exact PBS at FFT speed: key prepared once ([672][6][2 outputs][2 limbs][1024]
 * doubles, 132 MB), n bootstraps on nthreads threads; *max_dev is the largest
 * distance of an FFT product from its nearest integer (< 1/4: all exact) */
void orc_bk01_exact_prepare(double *prep, const uint32_t *bk);
void orc_extprod32_exact_split(uint32_t *res, const uint32_t *trlwe, const double *prep_trgsw, double *max_dev);
void orc_pbs01_exact_batch(uint32_t *out, const uint32_t *in0, int n, const double *prep, const uint32_t *tv,
                           int nthreads, double *max_dev);
void orc_sample_extract32(uint32_t *out, const uint32_t *acc, int N);
void orc_sample_extract64(uint64_t *out, const uint64_t *acc, int N);

/* identity key switching (keyswitch.cpp:11-48); rows generated on the fly
 * from the seed, or read from a full key when ksk != NULL */
void orc_iks10(uint32_t *out, const uint32_t *in, uint64_t seed, const uint32_t *s1,
               const uint32_t *s0, const uint32_t *ksk);
void orc_iks20(uint32_t *out, const uint64_t *in, uint64_t seed, const uint64_t *s2,
               const uint32_t *s0, const uint32_t *ksk);
void orc_iks21(uint32_t *out, const uint64_t *in, uint64_t seed, const uint64_t *s2,
               const uint32_t *s1, const uint32_t *ksk);
/* marks the rows an input touches: used[(i*t + j)*(2^basebit-1) + k] = 1 */
void orc_iks_rows(int kind, const void *in, uint8_t *used);

/* test vectors (gatebootstrapping.hpp:132-138, tfhepp_utils.h:105-120) */
void orc_tv_const32(uint32_t *tv, uint32_t mu);
void orc_tv_const64(uint64_t *tv, uint64_t mu);
void orc_tv_gpoly32(uint32_t *tv, uint32_t plain_bits, uint32_t scale_bits);
void orc_tv_gpoly64(uint64_t *tv, uint32_t plain_bits, uint32_t scale_bits);

/* HomNAND on lvl1 ciphertexts (gate.cpp:50-65): IKS10 then PBS01 */
void orc_homnand(uint32_t *out, const uint32_t *ca, const uint32_t *cb, const double *bkfft01,
                 uint64_t seed, const uint32_t *s1, const uint32_t *s0, const uint32_t *ksk10);

#ifdef __cplusplus
}
#endif
#endif
