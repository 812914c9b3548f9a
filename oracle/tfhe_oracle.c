/*
 * TEST ORACLE -- not part of the product.  See tfhe_oracle.h.
 *
 * Plain-C restatement of TFHEpp's PBS path (paths relative to the
 * reference's thirdparty/TFHEpp/).  Every function cites what it restates.
 */
#define _GNU_SOURCE
#include "tfhe_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ */
/* deterministic generator (not in the reference)                            */
/* ------------------------------------------------------------------------ */

static uint64_t mix64(uint64_t z)
{
    z ^= z >> 30;
    z *= 0xBF58476D1CE4E5B9ULL;
    z ^= z >> 27;
    z *= 0x94D049BB133111EBULL;
    z ^= z >> 31;
    return z;
}

uint64_t orc_draw(uint64_t seed, uint64_t stream, uint64_t ctr)
{
    uint64_t k = mix64(seed + stream * 0x9E3779B97F4A7C15ULL);
    return mix64(k ^ (ctr * 0xD1B54A32D192ED03ULL + 0x632BE59BD9B4E019ULL));
}

/* Integer approximate Gaussian: S = sum of four uniform 32-bit words minus
 * its mean (variance 2^64/3), scaled by `scale`/2^32, floor.  With
 * scale = round(sigma*sqrt(3)) the result has standard deviation ~sigma. */
int64_t orc_noise(uint64_t seed, uint64_t stream, uint64_t ctr, int64_t scale)
{
    uint64_t u0 = orc_draw(seed, stream, ctr);
    uint64_t u1 = orc_draw(seed, stream, ctr + 1);
    int64_t s = (int64_t)((u0 & 0xFFFFFFFFULL) + (u0 >> 32) + (u1 & 0xFFFFFFFFULL) + (u1 >> 32)) -
                (int64_t)(1ULL << 33);
    return (s * scale) >> 32;
}

enum {
    ST_SK0 = 1, ST_SK1 = 2, ST_SK2 = 3,
    ST_KSK10 = 0x10, ST_KSK20 = 0x11, ST_KSK21 = 0x12,
    ST_BK01 = 0x20, ST_BK02 = 0x21,
};
/* noise scales round(alpha * 2^w * sqrt(3)) for params/128bit.hpp alphas */
#define NS_LVL0 113512  /* alpha 2^-16, 32-bit torus */
#define NS_LVL1 222     /* alpha 2^-25, 32-bit torus */
#define NS_LVL2 7094    /* alpha 2^-52, 64-bit torus */

/* counter-block sizes per ciphertext */
#define CB_TLWE32 2048ULL
#define CB_TLWE64 4096ULL

/* key.cpp:8-17 + key.hpp:38-49: hwt positions drawn with replacement */
void orc_secret_keys(uint64_t seed, uint32_t *s0, uint32_t *s1, uint64_t *s2)
{
    memset(s0, 0, ORC_N0 * sizeof(uint32_t));
    memset(s1, 0, ORC_N1 * sizeof(uint32_t));
    memset(s2, 0, ORC_N2 * sizeof(uint64_t));
    for (int t = 0; t < 512; t++) s0[orc_draw(seed, ST_SK0, t) % ORC_N0] = 1;
    for (int t = 0; t < 512; t++) s1[orc_draw(seed, ST_SK1, t) % ORC_N1] = 1;
    for (int t = 0; t < 1024; t++) s2[orc_draw(seed, ST_SK2, t) % ORC_N2] = 1;
}

/* tlwe.cpp:16-31 (tlweSymEncrypt) */
void orc_tlwe32_encrypt(uint32_t *c, int n, uint32_t m, const uint32_t *key,
                        int64_t noise_scale, uint64_t seed, uint64_t stream, uint64_t idx)
{
    uint64_t base = idx * CB_TLWE32;
    uint32_t b = m + (uint32_t)orc_noise(seed, stream, base + n, noise_scale);
    for (int i = 0; i < n; i++) {
        c[i] = (uint32_t)orc_draw(seed, stream, base + i);
        b += c[i] * key[i];
    }
    c[n] = b;
}

void orc_tlwe64_encrypt(uint64_t *c, int n, uint64_t m, const uint64_t *key,
                        int64_t noise_scale, uint64_t seed, uint64_t stream, uint64_t idx)
{
    uint64_t base = idx * CB_TLWE64;
    uint64_t b = m + (uint64_t)orc_noise(seed, stream, base + n, noise_scale);
    for (int i = 0; i < n; i++) {
        c[i] = orc_draw(seed, stream, base + i);
        b += c[i] * key[i];
    }
    c[n] = b;
}

uint32_t orc_tlwe32_phase(const uint32_t *c, int n, const uint32_t *key)
{
    uint32_t p = c[n];
    for (int i = 0; i < n; i++) p -= c[i] * key[i];
    return p;
}

uint64_t orc_tlwe64_phase(const uint64_t *c, int n, const uint64_t *key)
{
    uint64_t p = c[n];
    for (int i = 0; i < n; i++) p -= c[i] * key[i];
    return p;
}

/* trlwe.cpp:8-24 (trlweSymEncryptZero, k=1): b = a*s + e, negacyclic */
static void trlwe32_zero(uint32_t *c, int N, const uint32_t *key, int64_t ns,
                         uint64_t seed, uint64_t stream, uint64_t idx)
{
    uint64_t base = idx * (4ULL * N);
    uint32_t *a = c, *b = c + N;
    for (int j = 0; j < N; j++) a[j] = (uint32_t)orc_draw(seed, stream, base + j);
    for (int j = 0; j < N; j++) b[j] = (uint32_t)orc_noise(seed, stream, base + N + 2 * j, ns);
    for (int t = 0; t < N; t++) {
        if (!key[t]) continue;
        uint32_t kt = key[t];
        for (int j = 0; j < N; j++) {
            int src = j - t;
            if (src >= 0) b[j] += a[src] * kt;
            else b[j] -= a[src + N] * kt;
        }
    }
}

static void trlwe64_zero(uint64_t *c, int N, const uint64_t *key, int64_t ns,
                         uint64_t seed, uint64_t stream, uint64_t idx)
{
    uint64_t base = idx * (4ULL * N);
    uint64_t *a = c, *b = c + N;
    for (int j = 0; j < N; j++) a[j] = orc_draw(seed, stream, base + j);
    for (int j = 0; j < N; j++) b[j] = (uint64_t)orc_noise(seed, stream, base + N + 2 * j, ns);
    for (int t = 0; t < N; t++) {
        if (!key[t]) continue;
        uint64_t kt = key[t];
        for (int j = 0; j < N; j++) {
            int src = j - t;
            if (src >= 0) b[j] += a[src] * kt;
            else b[j] -= a[src + N] * kt;
        }
    }
}

/* trlwe.cpp:30-37 (trlweSymEncrypt<lvl1param>): a TRLWE of zero with the
 * plaintext polynomial added to b. */
void orc_trlwe32_encrypt(uint32_t *out, const uint32_t *plain, const uint32_t *s1, uint64_t seed,
                         uint64_t stream, uint64_t idx)
{
    trlwe32_zero(out, ORC_N1, s1, NS_LVL1, seed, stream, idx);
    for (int j = 0; j < ORC_N1; j++) out[ORC_N1 + j] += plain[j];
}

/* trgsw.cpp:206-222 (trgswSymEncrypt) with plainpoly = {m0} as bkgen uses
 * (cloudkey.cpp:11-20): row r = i + k*l gets m0*h_i on poly k, coeff 0. */
void orc_trgsw32(uint32_t *out, uint32_t m0, const uint32_t *s1, uint64_t seed,
                 uint64_t stream, uint64_t idx)
{
    const int rows = 2 * ORC_L1;
    for (int r = 0; r < rows; r++)
        trlwe32_zero(out + (size_t)r * 2 * ORC_N1, ORC_N1, s1, NS_LVL1, seed, stream,
                     idx * rows + r);
    for (int i = 0; i < ORC_L1; i++)
        for (int k = 0; k < 2; k++) {
            uint32_t h = 1U << (32 - (i + 1) * ORC_BG1);
            out[((size_t)(i + k * ORC_L1) * 2 + k) * ORC_N1] += m0 * h;
        }
}

void orc_trgsw64(uint64_t *out, uint64_t m0, const uint64_t *s2, uint64_t seed,
                 uint64_t stream, uint64_t idx)
{
    const int rows = 2 * ORC_L2;
    for (int r = 0; r < rows; r++)
        trlwe64_zero(out + (size_t)r * 2 * ORC_N2, ORC_N2, s2, NS_LVL2, seed, stream,
                     idx * rows + r);
    for (int i = 0; i < ORC_L2; i++)
        for (int k = 0; k < 2; k++) {
            uint64_t h = 1ULL << (64 - (i + 1) * ORC_BG2);
            out[((size_t)(i + k * ORC_L2) * 2 + k) * ORC_N2] += m0 * h;
        }
}

typedef struct {
    int kind, t0, t1;
    uint64_t seed;
    const uint32_t *s0, *s1;
    const uint64_t *s2;
    void *out;
} job_t;

static void *bk_job(void *p)
{
    job_t *j = (job_t *)p;
    for (int i = j->t0; i < j->t1; i++) {
        if (j->kind == 1)
            orc_trgsw32((uint32_t *)j->out + (size_t)i * 2 * ORC_L1 * 2 * ORC_N1, j->s0[i], j->s1,
                        j->seed, ST_BK01, i);
        else
            orc_trgsw64((uint64_t *)j->out + (size_t)i * 2 * ORC_L2 * 2 * ORC_N2, j->s0[i], j->s2,
                        j->seed, ST_BK02, i);
    }
    return NULL;
}

static void run_jobs(job_t *proto, int total, int nthreads, void *(*fn)(void *))
{
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    pthread_t th[256];
    job_t jobs[256];
    for (int t = 0; t < nthreads; t++) {
        jobs[t] = *proto;
        jobs[t].t0 = (int)((long)total * t / nthreads);
        jobs[t].t1 = (int)((long)total * (t + 1) / nthreads);
        pthread_create(&th[t], NULL, fn, &jobs[t]);
    }
    for (int t = 0; t < nthreads; t++) pthread_join(th[t], NULL);
}

/* cloudkey.cpp:7-20 (bkgen) */
void orc_bk01(uint64_t seed, const uint32_t *s0, const uint32_t *s1, uint32_t *bk, int nthreads)
{
    job_t j = {1, 0, 0, seed, s0, s1, NULL, bk};
    run_jobs(&j, ORC_N0, nthreads, bk_job);
}

void orc_bk02(uint64_t seed, const uint32_t *s0, const uint64_t *s2, uint64_t *bk, int nthreads)
{
    job_t j = {2, 0, 0, seed, s0, NULL, s2, bk};
    run_jobs(&j, ORC_N0, nthreads, bk_job);
}

/* cloudkey.cpp:53-69 (ikskgen): row (i,j,k) encrypts key[i]*(k+1)*2^(w-(j+1)*basebit) */
void orc_ksk10_row(uint64_t seed, const uint32_t *s1, const uint32_t *s0, int i, int j, int k, uint32_t *row)
{
    uint32_t m = s1[i] * (uint32_t)(k + 1) * (uint32_t)(1ULL << (32 - (j + 1) * 10));
    orc_tlwe32_encrypt(row, ORC_N0, m, s0, NS_LVL0, seed, ST_KSK10, ((uint64_t)i * 2 + j) * 1023 + k);
}

void orc_ksk20_row(uint64_t seed, const uint64_t *s2, const uint32_t *s0, int i, int j, int k, uint32_t *row)
{
    uint32_t m = (uint32_t)(s2[i] * (uint64_t)(k + 1) * (1ULL << (32 - (j + 1) * 10)));
    orc_tlwe32_encrypt(row, ORC_N0, m, s0, NS_LVL0, seed, ST_KSK20, ((uint64_t)i * 2 + j) * 1023 + k);
}

void orc_ksk21_row(uint64_t seed, const uint64_t *s2, const uint32_t *s1, int i, int j, int k, uint32_t *row)
{
    uint32_t m = (uint32_t)(s2[i] * (uint64_t)(k + 1) * (1ULL << (32 - (j + 1) * 3)));
    orc_tlwe32_encrypt(row, ORC_N1, m, s1, NS_LVL1, seed, ST_KSK21, ((uint64_t)i * 10 + j) * 7 + k);
}

size_t orc_ksk_words(int kind)
{
    if (kind == 10) return (size_t)1024 * 2 * 1023 * (ORC_N0 + 1);
    if (kind == 20) return (size_t)2048 * 2 * 1023 * (ORC_N0 + 1);
    if (kind == 21) return (size_t)2048 * 10 * 7 * (ORC_N1 + 1);
    return 0;
}

static void *ksk_job(void *p)
{
    job_t *jb = (job_t *)p;
    uint32_t *out = (uint32_t *)jb->out;
    for (int i = jb->t0; i < jb->t1; i++) {
        if (jb->kind == 10) {
            for (int j = 0; j < 2; j++)
                for (int k = 0; k < 1023; k++)
                    orc_ksk10_row(jb->seed, jb->s1, jb->s0, i, j, k,
                                  out + (((size_t)i * 2 + j) * 1023 + k) * (ORC_N0 + 1));
        } else if (jb->kind == 20) {
            for (int j = 0; j < 2; j++)
                for (int k = 0; k < 1023; k++)
                    orc_ksk20_row(jb->seed, jb->s2, jb->s0, i, j, k,
                                  out + (((size_t)i * 2 + j) * 1023 + k) * (ORC_N0 + 1));
        } else {
            for (int j = 0; j < 10; j++)
                for (int k = 0; k < 7; k++)
                    orc_ksk21_row(jb->seed, jb->s2, jb->s1, i, j, k,
                                  out + (((size_t)i * 10 + j) * 7 + k) * (ORC_N1 + 1));
        }
    }
    return NULL;
}

void orc_ksk_full(int kind, uint64_t seed, const uint32_t *s0, const uint32_t *s1,
                  const uint64_t *s2, uint32_t *ksk, int nthreads)
{
    job_t j = {kind, 0, 0, seed, s0, s1, s2, ksk};
    run_jobs(&j, kind == 10 ? 1024 : 2048, nthreads, ksk_job);
}

/* ------------------------------------------------------------------------ */
/* negacyclic FFT, spqlios conventions                                       */
/* ------------------------------------------------------------------------ */
/*
 * TwistIFFT (torus -> frequency, fft_processor_spqlios.cpp:41-93 with the
 * ifft tables of spqlios-fft-impl.cpp:399-466): for M = N/2,
 *   z_m = (a_m + i a_{m+M}) * w^m,      w = exp(2 pi i / 2N)
 *   V(q) = sum_m z_m W^{mq},            W = exp(2 pi i / M)
 *   out[idx] = Re V(rev(idx)), out[idx+M] = Im V(rev(idx)),  rev = log2(M)-bit reversal.
 * TwistFFT (frequency -> torus, fft_processor_spqlios.cpp:95-215): the
 * inverse, z_m = (1/M) sum_q V(q) W^{-mq}, a_m + i a_{m+M} = z_m w^{-m},
 * converted with truncation toward zero (uint32_t(int64_t(x)) for the 32-bit
 * torus, mantissa shifting modulo 2^64 for the 64-bit torus).
 */
typedef struct { double re, im; } cpx;
static const long double PI_L = 3.141592653589793238462643383279502884L;

static int ilog2(int x) { int r = 0; while ((1 << r) < x) r++; return r; }

static int bitrev(int x, int bits)
{
    int r = 0;
    for (int b = 0; b < bits; b++) r |= ((x >> b) & 1) << (bits - 1 - b);
    return r;
}

/* twiddle tables, computed once in long double: rt[M][k] = exp(2 pi i k / M)
 * for k < M (M = 512 or 1024), tw[N][m] = exp(pi i m / N) for m < N/2 */
static cpx *rt_tab[2], *tw_tab[2];
static int *rev_tab[2];
static pthread_once_t tab_once = PTHREAD_ONCE_INIT;

static void build_tables(void)
{
    for (int t = 0; t < 2; t++) {
        int N = t == 0 ? ORC_N1 : ORC_N2, M = N / 2;
        rt_tab[t] = (cpx *)malloc(sizeof(cpx) * M);
        tw_tab[t] = (cpx *)malloc(sizeof(cpx) * M);
        rev_tab[t] = (int *)malloc(sizeof(int) * M);
        for (int k = 0; k < M; k++) rev_tab[t][k] = bitrev(k, ilog2(M));
        for (int k = 0; k < M; k++) {
            long double a = 2.0L * PI_L * (long double)k / (long double)M;
            rt_tab[t][k].re = (double)cosl(a);
            rt_tab[t][k].im = (double)sinl(a);
            long double b = PI_L * (long double)k / (long double)N;
            tw_tab[t][k].re = (double)cosl(b);
            tw_tab[t][k].im = (double)sinl(b);
        }
    }
}

static int tab_id(int N)
{
    pthread_once(&tab_once, build_tables);
    return N == ORC_N1 ? 0 : 1;
}

/* in-place radix-2 DIT; X[q] = sum x[m] exp(sign*2 pi i m q / M) */
static void fft_inplace(cpx *x, int M, int sign, const cpx *rt)
{
    const int *rev = rev_tab[M == ORC_N1 / 2 ? 0 : 1];
    for (int i = 0; i < M; i++) {
        int j = rev[i];
        if (i < j) { cpx t = x[i]; x[i] = x[j]; x[j] = t; }
    }
    for (int len = 2; len <= M; len <<= 1) {
        int half = len / 2, stride = M / len;
        for (int k = 0; k < half; k++) {
            double wr = rt[k * stride].re, wi = sign * rt[k * stride].im;
            for (int i = 0; i < M; i += len) {
                cpx u = x[i + k], v = x[i + k + half];
                cpx t = {v.re * wr - v.im * wi, v.re * wi + v.im * wr};
                x[i + k].re = u.re + t.re; x[i + k].im = u.im + t.im;
                x[i + k + half].re = u.re - t.re; x[i + k + half].im = u.im - t.im;
            }
        }
    }
}

static void twist_fwd(double *out, const double *ar, int N)
{
    int M = N / 2, t = tab_id(N);
    cpx z[ORC_N2 / 2];
    for (int m = 0; m < M; m++) {
        double c = tw_tab[t][m].re, s = tw_tab[t][m].im;
        double re = ar[m], im = ar[m + M];
        z[m].re = re * c - im * s;
        z[m].im = re * s + im * c;
    }
    fft_inplace(z, M, +1, rt_tab[t]);
    for (int idx = 0; idx < M; idx++) {
        int q = rev_tab[t][idx];
        out[idx] = z[q].re;
        out[idx + M] = z[q].im;
    }
}

/* returns the real coefficient values a_0..a_{N-1} (before torus conversion) */
static void twist_inv(double *ar, const double *in, int N)
{
    int M = N / 2, t = tab_id(N);
    cpx z[ORC_N2 / 2];
    for (int idx = 0; idx < M; idx++) {
        int q = rev_tab[t][idx];
        z[q].re = in[idx];
        z[q].im = in[idx + M];
    }
    fft_inplace(z, M, -1, rt_tab[t]);
    double inv = 1.0 / (double)M;
    for (int m = 0; m < M; m++) {
        double c = tw_tab[t][m].re, s = -tw_tab[t][m].im;
        double re = z[m].re * inv, im = z[m].im * inv;
        ar[m] = re * c - im * s;
        ar[m + M] = re * s + im * c;
    }
}

void orc_twist_ifft32(double *out, const uint32_t *a, int N)
{
    double *ar = (double *)malloc(sizeof(double) * N);
    for (int i = 0; i < N; i++) ar[i] = (double)(int32_t)a[i];
    twist_fwd(out, ar, N);
    free(ar);
}

void orc_twist_ifft64(double *out, const uint64_t *a, int N)
{
    double *ar = (double *)malloc(sizeof(double) * N);
    for (int i = 0; i < N; i++) ar[i] = (double)(int64_t)a[i];
    twist_fwd(out, ar, N);
    free(ar);
}

void orc_twist_fft32(uint32_t *out, const double *in, int N)
{
    double *ar = (double *)malloc(sizeof(double) * N);
    twist_inv(ar, in, N);
    for (int i = 0; i < N; i++) out[i] = (uint32_t)(int64_t)ar[i];
    free(ar);
}

/* fft_processor_spqlios.cpp:180-209: truncation toward zero, modulo 2^64 */
static uint64_t d2t64(double x)
{
    double a = fabs(x);
    uint64_t mag;
    if (a < 1.0) mag = 0;
    else {
        int e;
        double f = frexp(a, &e);                 /* a = f * 2^e, f in [0.5,1) */
        uint64_t mant = (uint64_t)ldexp(f, 53);  /* exact 53-bit integer */
        int sh = e - 53;
        if (sh >= 64) mag = 0;
        else if (sh >= 0) mag = mant << sh;
        else mag = mant >> (-sh);
    }
    return x < 0 ? (uint64_t)0 - mag : mag;
}

void orc_twist_fft64(uint64_t *out, const double *in, int N)
{
    double *ar = (double *)malloc(sizeof(double) * N);
    twist_inv(ar, in, N);
    for (int i = 0; i < N; i++) out[i] = d2t64(ar[i]);
    free(ar);
}

/* ------------------------------------------------------------------------ */
/* decomposition and external product                                        */
/* ------------------------------------------------------------------------ */

/* trgsw.cpp:9-39 */
void orc_decomp32(uint32_t *out, const uint32_t *poly, int digit)
{
    uint32_t offset = 0;
    for (int i = 1; i <= ORC_L1; i++) offset += (1U << (ORC_BG1 - 1)) * (1U << (32 - i * ORC_BG1));
    const uint32_t round = 1U << (32 - ORC_L1 * ORC_BG1 - 1);
    const int sh = 32 - (digit + 1) * ORC_BG1;
    for (int i = 0; i < ORC_N1; i++)
        out[i] = (((poly[i] + offset + round) >> sh) & ((1U << ORC_BG1) - 1)) - (1U << (ORC_BG1 - 1));
}

void orc_decomp64(uint64_t *out, const uint64_t *poly, int digit)
{
    uint64_t offset = 0;
    for (int i = 1; i <= ORC_L2; i++) offset += (1ULL << (ORC_BG2 - 1)) * (1ULL << (64 - i * ORC_BG2));
    const uint64_t round = 1ULL << (64 - ORC_L2 * ORC_BG2 - 1);
    const int sh = 64 - (digit + 1) * ORC_BG2;
    for (int i = 0; i < ORC_N2; i++)
        out[i] = (((poly[i] + offset + round) >> sh) & ((1ULL << ORC_BG2) - 1)) - (1ULL << (ORC_BG2 - 1));
}

/* utils.hpp:83-108 MulInFD / FMAInFD on the [re | im] split layout */
static void fma_fd(double *res, const double *a, const double *b, int N, int first)
{
    int M = N / 2;
    for (int i = 0; i < M; i++) {
        double re = a[i] * b[i] - a[i + M] * b[i + M];
        double im = a[i] * b[i + M] + a[i + M] * b[i];
        if (first) { res[i] = re; res[i + M] = im; }
        else { res[i] += re; res[i + M] += im; }
    }
}

/* trgsw.cpp:77-103; trgswfft layout [(k+1)l][2][N] doubles */
void orc_extprod32_fft(uint32_t *res, const uint32_t *trlwe, const double *trgswfft)
{
    const int N = ORC_N1, L = ORC_L1;
    double dfd[ORC_N1], acc[2][ORC_N1];
    uint32_t dec[ORC_N1];
    int first = 1;
    for (int k = 0; k < 2; k++)
        for (int d = 0; d < L; d++) {
            orc_decomp32(dec, trlwe + k * N, d);
            orc_twist_ifft32(dfd, dec, N);
            for (int m = 0; m < 2; m++)
                fma_fd(acc[m], dfd, trgswfft + ((size_t)(k * L + d) * 2 + m) * N, N, first);
            first = 0;
        }
    for (int m = 0; m < 2; m++) orc_twist_fft32(res + m * N, acc[m], N);
}

void orc_extprod64_fft(uint64_t *res, const uint64_t *trlwe, const double *trgswfft)
{
    const int N = ORC_N2, L = ORC_L2;
    static __thread double dfd[ORC_N2], acc[2][ORC_N2];
    static __thread uint64_t dec[ORC_N2];
    int first = 1;
    for (int k = 0; k < 2; k++)
        for (int d = 0; d < L; d++) {
            orc_decomp64(dec, trlwe + k * N, d);
            orc_twist_ifft64(dfd, dec, N);
            for (int m = 0; m < 2; m++)
                fma_fd(acc[m], dfd, trgswfft + ((size_t)(k * L + d) * 2 + m) * N, N, first);
            first = 0;
        }
    for (int m = 0; m < 2; m++) orc_twist_fft64(res + m * N, acc[m], N);
}

/* exact: sum_{k,d} dec_d(trlwe_k) * trgsw[k l + d][m] in Z[X]/(X^N+1) mod 2^w */
void orc_extprod32_exact(uint32_t *res, const uint32_t *trlwe, const uint32_t *trgsw)
{
    const int N = ORC_N1, L = ORC_L1;
    uint32_t dec[ORC_N1];
    memset(res, 0, 2 * N * sizeof(uint32_t));
    for (int k = 0; k < 2; k++)
        for (int d = 0; d < L; d++) {
            orc_decomp32(dec, trlwe + k * N, d);
            for (int m = 0; m < 2; m++) {
                const uint32_t *g = trgsw + ((size_t)(k * L + d) * 2 + m) * N;
                uint32_t *r = res + m * N;
                for (int t = 0; t < N; t++) {
                    uint32_t dt = dec[t];
                    if (!dt) continue;
                    for (int j = 0; j < t; j++) r[j] -= dt * g[j - t + N];
                    for (int j = t; j < N; j++) r[j] += dt * g[j - t];
                }
            }
        }
}

void orc_extprod64_exact(uint64_t *res, const uint64_t *trlwe, const uint64_t *trgsw)
{
    const int N = ORC_N2, L = ORC_L2;
    static __thread uint64_t dec[ORC_N2];
    memset(res, 0, 2 * N * sizeof(uint64_t));
    for (int k = 0; k < 2; k++)
        for (int d = 0; d < L; d++) {
            orc_decomp64(dec, trlwe + k * N, d);
            for (int m = 0; m < 2; m++) {
                const uint64_t *g = trgsw + ((size_t)(k * L + d) * 2 + m) * N;
                uint64_t *r = res + m * N;
                for (int t = 0; t < N; t++) {
                    uint64_t dt = dec[t];
                    if (!dt) continue;
                    for (int j = 0; j < t; j++) r[j] -= dt * g[j - t + N];
                    for (int j = t; j < N; j++) r[j] += dt * g[j - t];
                }
            }
        }
}

/* trgsw.cpp:183-193 ApplyFFT2trgsw */
void orc_trgsw32_fft(double *out, const uint32_t *trgsw)
{
    for (int r = 0; r < 2 * ORC_L1 * 2; r++)
        orc_twist_ifft32(out + (size_t)r * ORC_N1, trgsw + (size_t)r * ORC_N1, ORC_N1);
}

void orc_trgsw64_fft(double *out, const uint64_t *trgsw)
{
    for (int r = 0; r < 2 * ORC_L2 * 2; r++)
        orc_twist_ifft64(out + (size_t)r * ORC_N2, trgsw + (size_t)r * ORC_N2, ORC_N2);
}

/* ------------------------------------------------------------------------ */
/* blind rotation, sample extraction, PBS                                    */
/* ------------------------------------------------------------------------ */

/* utils.hpp:110-125 PolynomialMulByXai, a in [0, 2N] */
static void mulxai32(uint32_t *res, const uint32_t *p, uint32_t a, int N)
{
    if (a == 0 || a == 2u * N) { memcpy(res, p, N * sizeof(uint32_t)); return; }
    if (a < (uint32_t)N) {
        for (uint32_t i = 0; i < a; i++) res[i] = -p[i - a + N];
        for (uint32_t i = a; i < (uint32_t)N; i++) res[i] = p[i - a];
    } else {
        uint32_t aa = a - N;
        for (uint32_t i = 0; i < aa; i++) res[i] = p[i - aa + N];
        for (uint32_t i = aa; i < (uint32_t)N; i++) res[i] = -p[i - aa];
    }
}

static void mulxai64(uint64_t *res, const uint64_t *p, uint32_t a, int N)
{
    if (a == 0 || a == 2u * N) { memcpy(res, p, N * sizeof(uint64_t)); return; }
    if (a < (uint32_t)N) {
        for (uint32_t i = 0; i < a; i++) res[i] = -p[i - a + N];
        for (uint32_t i = a; i < (uint32_t)N; i++) res[i] = p[i - a];
    } else {
        uint32_t aa = a - N;
        for (uint32_t i = 0; i < aa; i++) res[i] = p[i - aa + N];
        for (uint32_t i = aa; i < (uint32_t)N; i++) res[i] = -p[i - aa];
    }
}

/* utils.hpp:127-141 PolynomialMulByXaiMinusOne, a in [1, 2N) */
static void mulxai_minus1_32(uint32_t *res, const uint32_t *p, uint32_t a, int N)
{
    if (a < (uint32_t)N) {
        for (uint32_t i = 0; i < a; i++) res[i] = -p[i - a + N] - p[i];
        for (uint32_t i = a; i < (uint32_t)N; i++) res[i] = p[i - a] - p[i];
    } else {
        uint32_t aa = a - N;
        for (uint32_t i = 0; i < aa; i++) res[i] = p[i - aa + N] - p[i];
        for (uint32_t i = aa; i < (uint32_t)N; i++) res[i] = -p[i - aa] - p[i];
    }
}

static void mulxai_minus1_64(uint64_t *res, const uint64_t *p, uint32_t a, int N)
{
    if (a < (uint32_t)N) {
        for (uint32_t i = 0; i < a; i++) res[i] = -p[i - a + N] - p[i];
        for (uint32_t i = a; i < (uint32_t)N; i++) res[i] = p[i - a] - p[i];
    } else {
        uint32_t aa = a - N;
        for (uint32_t i = 0; i < aa; i++) res[i] = p[i - aa + N] - p[i];
        for (uint32_t i = aa; i < (uint32_t)N; i++) res[i] = -p[i - aa] - p[i];
    }
}

/* trlwe.cpp:108-118 SampleExtractIndex(index 0) */
void orc_sample_extract32(uint32_t *out, const uint32_t *acc, int N)
{
    out[0] = acc[0];
    for (int i = 1; i < N; i++) out[i] = -acc[N - i];
    out[N] = acc[N];
}

void orc_sample_extract64(uint64_t *out, const uint64_t *acc, int N)
{
    out[0] = acc[0];
    for (int i = 1; i < N; i++) out[i] = -acc[N - i];
    out[N] = acc[N];
}

/* gatebootstrapping.hpp:15-43 (BlindRotate, num_out = 1) + detwfa.cpp:20-35 */
void orc_blind_rotate01(uint32_t *acc, const uint32_t *in0, const double *bkfft, const uint32_t *tv)
{
    const int N = ORC_N1;
    const size_t trgsw_len = (size_t)2 * ORC_L1 * 2 * N;
    uint32_t bbar = 2 * N - (in0[ORC_N0] >> 21);
    uint32_t tmp[2 * ORC_N1], prod[2 * ORC_N1];
    memset(acc, 0, N * sizeof(uint32_t));
    mulxai32(acc + N, tv, bbar, N);
    for (int i = 0; i < ORC_N0; i++) {
        uint32_t abar = (in0[i] + (1U << 20)) >> 21;
        if (abar == 0) continue;
        for (int k = 0; k < 2; k++) mulxai_minus1_32(tmp + k * N, acc + k * N, abar, N);
        orc_extprod32_fft(prod, tmp, bkfft + i * trgsw_len);
        for (int j = 0; j < 2 * N; j++) acc[j] += prod[j];
    }
}

void orc_pbs01(uint32_t *out, const uint32_t *in0, const double *bkfft, const uint32_t *tv)
{
    uint32_t acc[2 * ORC_N1];
    orc_blind_rotate01(acc, in0, bkfft, tv);
    orc_sample_extract32(out, acc, ORC_N1);
}

void orc_pbs01_exact(uint32_t *out, const uint32_t *in0, const uint32_t *bk, const uint32_t *tv)
{
    const int N = ORC_N1;
    const size_t trgsw_len = (size_t)2 * ORC_L1 * 2 * N;
    uint32_t acc[2 * ORC_N1], tmp[2 * ORC_N1], prod[2 * ORC_N1];
    uint32_t bbar = 2 * N - (in0[ORC_N0] >> 21);
    memset(acc, 0, N * sizeof(uint32_t));
    mulxai32(acc + N, tv, bbar, N);
    for (int i = 0; i < ORC_N0; i++) {
        uint32_t abar = (in0[i] + (1U << 20)) >> 21;
        if (abar == 0) continue;
        for (int k = 0; k < 2; k++) mulxai_minus1_32(tmp + k * N, acc + k * N, abar, N);
        orc_extprod32_exact(prod, tmp, bk + i * trgsw_len);
        for (int j = 0; j < 2 * N; j++) acc[j] += prod[j];
    }
    orc_sample_extract32(out, acc, N);
}

/*
 * Exact lvl01 PBS at FFT speed, for noise measurements over thousands of
 * bootstraps (the schoolbook orc_pbs01_exact takes seconds per bootstrap).
 * The external product is the same integer sum as orc_extprod32_exact,
 * sum_{k,d} dec_d(acc_k) * trgsw[k l + d][m] in Z[X]/(X^N+1) mod 2^32, with
 * every key polynomial g split into signed 16-bit limbs g = g1 * 2^16 + g0
 * (g0 in [-2^15, 2^15), g1 in [-2^15, 2^15]).  Each limb product sum is an
 * integer below 6 * 1024 * 32 * 2^15 = 2^32.6 in magnitude, so the FP64
 * negacyclic FFT computes it to far better than 1/2 and rounding recovers it
 * exactly; the result is v0 + v1 * 2^16 mod 2^32.  Every rounding is checked:
 * the largest distance of an FFT output from its nearest integer is reported
 * (a value below 1/4 certifies that every product was exact).
 */
#define PREP_ROW ((size_t)2 * 2 * ORC_N1)   /* per TRGSW row: [m][limb][N] doubles */

void orc_bk01_exact_prepare(double *prep, const uint32_t *bk)
{
    double ar[ORC_N1];
    for (size_t r = 0; r < (size_t)ORC_N0 * 2 * ORC_L1; r++)
        for (int m = 0; m < 2; m++) {
            const uint32_t *g = bk + (r * 2 + m) * ORC_N1;
            for (int limb = 0; limb < 2; limb++) {
                for (int j = 0; j < ORC_N1; j++) {
                    int32_t v = (int32_t)g[j];
                    int32_t g0 = (int32_t)(((uint32_t)v + 0x8000u) & 0xFFFFu) - 0x8000;
                    ar[j] = limb == 0 ? (double)g0 : (double)(((int64_t)v - g0) >> 16);
                }
                twist_fwd(prep + r * PREP_ROW + ((size_t)m * 2 + limb) * ORC_N1, ar, ORC_N1);
            }
        }
}

static void extprod32_exact_split(uint32_t *res, const uint32_t *trlwe, const double *prep, double *max_dev)
{
    const int N = ORC_N1, L = ORC_L1;
    double dfd[2 * ORC_L1][ORC_N1], acc[ORC_N1];
    uint32_t dec[ORC_N1];
    int64_t v[2][ORC_N1];
    for (int k = 0; k < 2; k++)
        for (int d = 0; d < L; d++) {
            orc_decomp32(dec, trlwe + k * N, d);
            double x[ORC_N1];
            for (int j = 0; j < N; j++) x[j] = (double)(int32_t)dec[j];
            twist_fwd(dfd[k * L + d], x, N);
        }
    for (int m = 0; m < 2; m++) {
        for (int limb = 0; limb < 2; limb++) {
            for (int r = 0; r < 2 * L; r++)
                fma_fd(acc, dfd[r], prep + (size_t)r * PREP_ROW + ((size_t)m * 2 + limb) * N, N, r == 0);
            double a[ORC_N1];
            twist_inv(a, acc, N);
            for (int j = 0; j < N; j++) {
                double rj = nearbyint(a[j]);
                double dev = fabs(a[j] - rj);
                if (dev > *max_dev) *max_dev = dev;
                v[limb][j] = (int64_t)rj;
            }
        }
        for (int j = 0; j < N; j++) res[m * N + j] = (uint32_t)(uint64_t)(v[0][j] + v[1][j] * 65536);
    }
}

void orc_extprod32_exact_split(uint32_t *res, const uint32_t *trlwe, const double *prep_trgsw, double *max_dev)
{
    *max_dev = 0.0;
    extprod32_exact_split(res, trlwe, prep_trgsw, max_dev);
}

static void pbs01_exact_split(uint32_t *out, const uint32_t *in0, const double *prep, const uint32_t *tv,
                              double *max_dev)
{
    const int N = ORC_N1;
    uint32_t acc[2 * ORC_N1], tmp[2 * ORC_N1], prod[2 * ORC_N1];
    uint32_t bbar = 2 * N - (in0[ORC_N0] >> 21);
    memset(acc, 0, N * sizeof(uint32_t));
    mulxai32(acc + N, tv, bbar, N);
    for (int i = 0; i < ORC_N0; i++) {
        uint32_t abar = (in0[i] + (1U << 20)) >> 21;
        if (abar == 0) continue;
        for (int k = 0; k < 2; k++) mulxai_minus1_32(tmp + k * N, acc + k * N, abar, N);
        extprod32_exact_split(prod, tmp, prep + (size_t)i * 2 * ORC_L1 * PREP_ROW, max_dev);
        for (int j = 0; j < 2 * N; j++) acc[j] += prod[j];
    }
    orc_sample_extract32(out, acc, N);
}

typedef struct {
    uint32_t *out;
    const uint32_t *in0, *tv;
    const double *prep;
    int t0, t1;
    double max_dev;
} pbsx_job_t;

static void *pbsx_job(void *arg)
{
    pbsx_job_t *j = (pbsx_job_t *)arg;
    for (int b = j->t0; b < j->t1; b++)
        pbs01_exact_split(j->out + (size_t)b * (ORC_N1 + 1), j->in0 + (size_t)b * (ORC_N0 + 1), j->prep, j->tv,
                          &j->max_dev);
    return NULL;
}

void orc_pbs01_exact_batch(uint32_t *out, const uint32_t *in0, int n, const double *prep, const uint32_t *tv,
                           int nthreads, double *max_dev)
{
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    pthread_t th[256];
    pbsx_job_t jobs[256];
    for (int t = 0; t < nthreads; t++) {
        jobs[t] = (pbsx_job_t){out, in0, tv, prep, (int)((long)n * t / nthreads), (int)((long)n * (t + 1) / nthreads), 0.0};
        pthread_create(&th[t], NULL, pbsx_job, &jobs[t]);
    }
    *max_dev = 0.0;
    for (int t = 0; t < nthreads; t++) {
        pthread_join(th[t], NULL);
        if (jobs[t].max_dev > *max_dev) *max_dev = jobs[t].max_dev;
    }
}

void orc_pbs02(uint64_t *out, const uint32_t *in0, const double *bkfft, const uint64_t *tv)
{
    const int N = ORC_N2;
    const size_t trgsw_len = (size_t)2 * ORC_L2 * 2 * N;
    uint64_t *acc = (uint64_t *)malloc(sizeof(uint64_t) * 2 * N * 3);
    uint64_t *tmp = acc + 2 * N, *prod = acc + 4 * N;
    uint32_t bbar = 2 * N - (in0[ORC_N0] >> 20);
    memset(acc, 0, N * sizeof(uint64_t));
    mulxai64(acc + N, tv, bbar, N);
    for (int i = 0; i < ORC_N0; i++) {
        uint32_t abar = (in0[i] + (1U << 19)) >> 20;
        if (abar == 0) continue;
        for (int k = 0; k < 2; k++) mulxai_minus1_64(tmp + k * N, acc + k * N, abar, N);
        orc_extprod64_fft(prod, tmp, bkfft + i * trgsw_len);
        for (int j = 0; j < 2 * N; j++) acc[j] += prod[j];
    }
    orc_sample_extract64(out, acc, N);
    free(acc);
}

/* ------------------------------------------------------------------------ */
/* identity key switching (keyswitch.cpp:11-48)                              */
/* ------------------------------------------------------------------------ */

void orc_iks10(uint32_t *out, const uint32_t *in, uint64_t seed, const uint32_t *s1,
               const uint32_t *s0, const uint32_t *ksk)
{
    const uint32_t prec = 1U << (32 - (1 + 10 * 2));
    uint32_t row[ORC_N0 + 1];
    memset(out, 0, (ORC_N0 + 1) * sizeof(uint32_t));
    out[ORC_N0] = in[ORC_N1];
    for (int i = 0; i < ORC_N1; i++) {
        uint32_t abar = in[i] + prec;
        for (int j = 0; j < 2; j++) {
            uint32_t aij = (abar >> (32 - (j + 1) * 10)) & 1023;
            if (!aij) continue;
            const uint32_t *r;
            if (ksk) r = ksk + (((size_t)i * 2 + j) * 1023 + aij - 1) * (ORC_N0 + 1);
            else { orc_ksk10_row(seed, s1, s0, i, j, aij - 1, row); r = row; }
            for (int k = 0; k <= ORC_N0; k++) out[k] -= r[k];
        }
    }
}

void orc_iks20(uint32_t *out, const uint64_t *in, uint64_t seed, const uint64_t *s2,
               const uint32_t *s0, const uint32_t *ksk)
{
    const uint64_t prec = 1ULL << (64 - (1 + 10 * 2));
    uint32_t row[ORC_N0 + 1];
    memset(out, 0, (ORC_N0 + 1) * sizeof(uint32_t));
    out[ORC_N0] = (uint32_t)((in[ORC_N2] + (1ULL << 31)) >> 32);
    for (int i = 0; i < ORC_N2; i++) {
        uint64_t abar = in[i] + prec;
        for (int j = 0; j < 2; j++) {
            uint32_t aij = (uint32_t)((abar >> (64 - (j + 1) * 10)) & 1023);
            if (!aij) continue;
            const uint32_t *r;
            if (ksk) r = ksk + (((size_t)i * 2 + j) * 1023 + aij - 1) * (ORC_N0 + 1);
            else { orc_ksk20_row(seed, s2, s0, i, j, aij - 1, row); r = row; }
            for (int k = 0; k <= ORC_N0; k++) out[k] -= r[k];
        }
    }
}

void orc_iks21(uint32_t *out, const uint64_t *in, uint64_t seed, const uint64_t *s2,
               const uint32_t *s1, const uint32_t *ksk)
{
    const uint64_t prec = 1ULL << (64 - (1 + 3 * 10));
    uint32_t row[ORC_N1 + 1];
    memset(out, 0, (ORC_N1 + 1) * sizeof(uint32_t));
    out[ORC_N1] = (uint32_t)((in[ORC_N2] + (1ULL << 31)) >> 32);
    for (int i = 0; i < ORC_N2; i++) {
        uint64_t abar = in[i] + prec;
        for (int j = 0; j < 10; j++) {
            uint32_t aij = (uint32_t)((abar >> (64 - (j + 1) * 3)) & 7);
            if (!aij) continue;
            const uint32_t *r;
            if (ksk) r = ksk + (((size_t)i * 10 + j) * 7 + aij - 1) * (ORC_N1 + 1);
            else { orc_ksk21_row(seed, s2, s1, i, j, aij - 1, row); r = row; }
            for (int k = 0; k <= ORC_N1; k++) out[k] -= r[k];
        }
    }
}

void orc_iks_rows(int kind, const void *in, uint8_t *used)
{
    if (kind == 10) {
        const uint32_t *x = (const uint32_t *)in;
        for (int i = 0; i < ORC_N1; i++) {
            uint32_t abar = x[i] + (1U << 11);
            for (int j = 0; j < 2; j++) {
                uint32_t aij = (abar >> (32 - (j + 1) * 10)) & 1023;
                if (aij) used[((size_t)i * 2 + j) * 1023 + aij - 1] = 1;
            }
        }
    } else if (kind == 20) {
        const uint64_t *x = (const uint64_t *)in;
        for (int i = 0; i < ORC_N2; i++) {
            uint64_t abar = x[i] + (1ULL << 43);
            for (int j = 0; j < 2; j++) {
                uint32_t aij = (uint32_t)((abar >> (64 - (j + 1) * 10)) & 1023);
                if (aij) used[((size_t)i * 2 + j) * 1023 + aij - 1] = 1;
            }
        }
    } else {
        const uint64_t *x = (const uint64_t *)in;
        for (int i = 0; i < ORC_N2; i++) {
            uint64_t abar = x[i] + (1ULL << 33);
            for (int j = 0; j < 10; j++) {
                uint32_t aij = (uint32_t)((abar >> (64 - (j + 1) * 3)) & 7);
                if (aij) used[((size_t)i * 10 + j) * 7 + aij - 1] = 1;
            }
        }
    }
}

/* ------------------------------------------------------------------------ */
/* test vectors and gates                                                    */
/* ------------------------------------------------------------------------ */

void orc_tv_const32(uint32_t *tv, uint32_t mu) { for (int i = 0; i < ORC_N1; i++) tv[i] = mu; }
void orc_tv_const64(uint64_t *tv, uint64_t mu) { for (int i = 0; i < ORC_N2; i++) tv[i] = mu; }

/* src/HEDB/comparison/tfhepp_utils.h:113-120 gpolygen */
void orc_tv_gpoly32(uint32_t *tv, uint32_t plain_bits, uint32_t scale_bits)
{
    uint32_t pad = 10 - plain_bits;
    for (int i = 0; i < ORC_N1; i++) tv[i] = (uint32_t)((1ULL << scale_bits) * (uint64_t)(i >> pad));
}

void orc_tv_gpoly64(uint64_t *tv, uint32_t plain_bits, uint32_t scale_bits)
{
    uint32_t pad = 11 - plain_bits;
    for (int i = 0; i < ORC_N2; i++) tv[i] = (1ULL << scale_bits) * (uint64_t)(i >> pad);
}

/* gate.cpp:50-65 + gatebootstrapping.hpp:150-158 */
void orc_homnand(uint32_t *out, const uint32_t *ca, const uint32_t *cb, const double *bkfft01,
                 uint64_t seed, const uint32_t *s1, const uint32_t *s0, const uint32_t *ksk10)
{
    uint32_t x[ORC_N1 + 1], l0[ORC_N0 + 1], tv[ORC_N1];
    for (int i = 0; i <= ORC_N1; i++) x[i] = -ca[i] - cb[i];
    x[ORC_N1] += 1U << 29;
    orc_iks10(l0, x, seed, s1, s0, ksk10);
    orc_tv_const32(tv, 1U << 29);
    orc_pbs01(out, l0, bkfft01, tv);
}
