/*
 * cufhedb_b200 -- B200-native (sm_100a) TFHE programmable-bootstrapping engine.
 *
 * C ABI of the engine that replaces cuFHEDB's GPU layer (src/cuHEDB/, header-
 * only CUDA: fft_gpu/cufft_gpu.cuh, BlindRotate_gpu.cuh, ExternalProduct_gpu.cuh,
 * fft_gpu.cuh) and the host-side TFHEpp::IdentityKeySwitch calls its operator
 * wrappers make (src/cuHEDB/gatebootstrap_gpu.cuh:42,59,76,90,101,113,133,149,
 * 159,167; msb_gpu.cuh:67,75,95).  Plain pointers and sizes only; every call
 * returns an int status (CUFHEDB_OK = 0) and cufhedb_last_error() gives the
 * message of the calling thread's last failure.
 *
 * Data layouts are TFHEpp's (thirdparty/TFHEpp/include/params.hpp:31-91),
 * parameter set params/128bit.hpp:7-83:
 *   TLWE<lvl0param>  673 x uint32   (a[672], b)
 *   TLWE<lvl1param>  1025 x uint32  (a[1024], b)
 *   TLWE<lvl2param>  2049 x uint64  (a[2048], b)
 *   BootstrappingKey<lvl01param>     [672][6][2][1024] uint32
 *   BootstrappingKeyFFT<lvl01param>  [672][6][2][1024] double (spqlios layout)
 *   BootstrappingKey<lvl02param>     [672][8][2][2048] uint64
 *   BootstrappingKeyFFT<lvl02param>  [672][8][2][2048] double
 *   KeySwitchingKey<lvl10param>      [1024][2][1023][673] uint32
 *   KeySwitchingKey<lvl20param>      [2048][2][1023][673] uint32
 *   KeySwitchingKey<lvl21param>      [2048][10][7][1025] uint32
 * Batches are arrays of B such objects, back to back.
 *
 * Entry points taking a stream enqueue work and return; device-side failures
 * (a bounded wait inside a kernel that expired) are reported by the next
 * cufhedb_sync() on that context.  *_host entry points take host buffers,
 * copy in and out on an internal stream and return when the results are in
 * the caller's memory.
 */
#ifndef CUFHEDB_B200_H
#define CUFHEDB_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CUFHEDB_ABI_VERSION 1

#if defined(__GNUC__)
#define CUFHEDB_API __attribute__((visibility("default")))
#else
#define CUFHEDB_API
#endif

typedef struct cufhedb_ctx cufhedb_ctx;
typedef void *cufhedb_stream_t; /* a cudaStream_t; NULL is the legacy default stream */

enum cufhedb_status {
    CUFHEDB_OK = 0,
    CUFHEDB_ERR_ARG = 1,         /* null pointer, negative size, unknown kind */
    CUFHEDB_ERR_NOKEY = 2,       /* the key this call needs was never loaded or generated */
    CUFHEDB_ERR_CUDA = 3,        /* CUDA runtime error */
    CUFHEDB_ERR_OOM = 4,         /* device or pinned allocation failed */
    CUFHEDB_ERR_DEVICE = 5,      /* a kernel gave up a bounded wait and flagged the context */
    CUFHEDB_ERR_UNSUPPORTED = 6  /* no usable sm_100 device */
};

enum cufhedb_precision {
    CUFHEDB_FP64 = 0,      /* FP64 FFT and FP64 frequency-domain products */
    CUFHEDB_SPLIT32 = 1,   /* FP32 transforms, two-limb key, exact top-limb rounding */
    CUFHEDB_SPLIT32_TC = 2 /* SPLIT32 with the first step of every digit transform on the tensor
                              cores (tcgen05, FP16 two-limb constants, FP32 accumulation) */
};

enum cufhedb_ksk_kind { CUFHEDB_KSK10 = 10, CUFHEDB_KSK20 = 20, CUFHEDB_KSK21 = 21 };

enum cufhedb_keygen_flags {
    CUFHEDB_GEN_BK01 = 1,
    CUFHEDB_GEN_BK02 = 2,
    CUFHEDB_GEN_KSK10 = 4,
    CUFHEDB_GEN_KSK20 = 8,
    CUFHEDB_GEN_KSK21 = 16,
    CUFHEDB_GEN_ALL = 31
};

/* test vector of a bootstrap: the accumulator starts as (0, X^bbar * tv) */
enum cufhedb_tv_kind {
    CUFHEDB_TV_CONST = 0,     /* tv[i] = value (TFHEpp mu-polygen) */
    CUFHEDB_TV_STAIRCASE = 1, /* tv[i] = 2^value * (i >> pad_bits) (HEDB gpolygen) */
    CUFHEDB_TV_POLY = 2       /* tv = poly, N words of device memory */
};

typedef struct {
    int kind;
    int pad_bits;
    uint64_t value;
    const void *poly;
} cufhedb_testvec;

/* two-input lvl1 gates of TFHEpp (thirdparty/TFHEpp/src/gate.cpp:60-181):
 * out = PBS(IKS10(sa*ca + sb*cb + offset)) with a constant mu test vector */
enum cufhedb_gate {
    CUFHEDB_NAND = 0,
    CUFHEDB_NOR = 1,
    CUFHEDB_XNOR = 2,
    CUFHEDB_AND = 3,
    CUFHEDB_OR = 4,
    CUFHEDB_XOR = 5,
    CUFHEDB_ANDNY = 6,
    CUFHEDB_ANDYN = 7,
    CUFHEDB_ORNY = 8,
    CUFHEDB_ORYN = 9
};

/* ---- context ------------------------------------------------------------ */
CUFHEDB_API int cufhedb_abi_version(void);
CUFHEDB_API const char *cufhedb_last_error(void);
/* replaces the CuFFT_Torus constructor (src/cuHEDB/fft_gpu/cufft_gpu.cuh:135-163):
 * binds a device, builds the twiddle tables; keys are loaded separately.
 * Entry points take transient scratch from the device's default stream-ordered
 * memory pool; this call sets that pool's release threshold to its maximum,
 * so memory freed into it stays mapped across synchronisations (a process-
 * wide attribute of the default pool; nothing outlasts the process). */
CUFHEDB_API int cufhedb_ctx_create(cufhedb_ctx **out, int device);
CUFHEDB_API int cufhedb_ctx_destroy(cufhedb_ctx *ctx);
CUFHEDB_API int cufhedb_ctx_num_sms(const cufhedb_ctx *ctx);
/* waits for `stream`, then reports (and clears) any device-side failure flag */
CUFHEDB_API int cufhedb_sync(cufhedb_ctx *ctx, cufhedb_stream_t stream);

/* ---- key material ----------------------------------------------------------- */
/* LoadBK (cufft_gpu.cuh:175-184): TFHEpp BootstrappingKeyFFT<lvl01param>, host memory */
CUFHEDB_API int cufhedb_load_bkfft_lvl01(cufhedb_ctx *ctx, const double *bkfft);
/* integer BootstrappingKey<lvl01param> (TFHEpp bkgen output), host memory */
CUFHEDB_API int cufhedb_load_bk_lvl01(cufhedb_ctx *ctx, const uint32_t *bk);
/* the lvl02 key: integer BootstrappingKey<lvl02param> or TFHEpp
 * BootstrappingKeyFFT<lvl02param> (cufftlvl2.LoadBK), host memory */
CUFHEDB_API int cufhedb_load_bk_lvl02(cufhedb_ctx *ctx, const uint64_t *bk);
CUFHEDB_API int cufhedb_load_bkfft_lvl02(cufhedb_ctx *ctx, const double *bkfft);
/* KeySwitchingKey<lvl10/20/21param>, host memory in TFHEpp's packed layout
 * (rows of n+1 words); kind is cufhedb_ksk_kind.  On the device every row is
 * padded to a multiple of 16 bytes (673 -> 676, 1025 -> 1028 words; the
 * export and save functions below return the packed layout).  Replaces the
 * host-resident key TFHEpp::IdentityKeySwitch reads (EvalKey::iksklvl*). */
CUFHEDB_API int cufhedb_load_ksk(cufhedb_ctx *ctx, int kind, const uint32_t *ksk);
/* Deterministic key set from `seed`, generated on the device (restates
 * TFHEpp bkgen / ikskgen, thirdparty/TFHEpp/src/cloudkey.cpp:7-69, with a
 * counter-based generator).  For tests and benchmarks: not a cryptographic
 * generator. */
CUFHEDB_API int cufhedb_keygen(cufhedb_ctx *ctx, uint64_t seed, unsigned flags);
/* copies of device-resident key material, for checking and serialisation:
 * the integer lvl01 key (when loaded with cufhedb_load_bk_lvl01 or generated),
 * and n rows of a key-switching key (row = (i*t + j)*(2^basebit-1) + k) */
CUFHEDB_API int cufhedb_export_bk_lvl01(cufhedb_ctx *ctx, uint32_t *bk);
CUFHEDB_API int cufhedb_export_bk_lvl02(cufhedb_ctx *ctx, uint64_t *bk);
CUFHEDB_API int cufhedb_export_ksk_rows(cufhedb_ctx *ctx, int kind, const uint64_t *rows, int n, uint32_t *out);
/* the secret keys of the deterministic key set (host-only computation) */
CUFHEDB_API int cufhedb_secret_keys(uint64_t seed, uint32_t *s0, uint32_t *s1, uint64_t *s2);
/* Key files in the raw layout of the reference's query programs
 * (test/HE3_Query/fastR.h:6-74): the lvl1 secret key (1024 x uint32), TFHEpp's
 * BootstrappingKeyFFT<lvl01param> (672 x 6 x 2 x 1024 doubles) and
 * KeySwitchingKey<lvl10param> (1024 x 2 x 1023 x 673 uint32), in that order,
 * 5.71 GB.  load: uploads both keys (the key-switching key in pieces of whole
 * rows, about 64 MB each)
 * and copies the secret key to sk_out when it is not NULL; save: writes this
 * context's lvl01 and lvl10 keys, with `sk` (1024 words), or the
 * deterministic key set's lvl1 key when sk is NULL, or zeros. */
CUFHEDB_API int cufhedb_load_keyfile(cufhedb_ctx *ctx, const char *path, uint32_t *sk_out);
CUFHEDB_API int cufhedb_save_keyfile(cufhedb_ctx *ctx, const char *path, const uint32_t *sk);
/* TFHEpp cereal key archives, as the reference's key tools write them
 * (src/HEDB/utils/serialize.cpp:7-60: cereal::PortableBinaryOutputArchive of
 * EvalKey::serialize_bkfftlvl01 / _bkfftlvl02 / _iksklvl10 / _iksklvl20 /
 * _iksklvl21, thirdparty/TFHEpp/include/cloudkey.hpp:149-228).  payload:
 * host-only, locates and checks the key inside the archive (the last
 * sizeof(key) bytes, after the parameter block and the pointer's valid byte);
 * load: reads it into the context like cufhedb_load_bkfft_lvl01/02 /
 * cufhedb_load_ksk (key-switching keys streamed in pieces of whole rows). */
enum cufhedb_cereal_kind {
    CUFHEDB_CEREAL_BKFFT01 = 1,
    CUFHEDB_CEREAL_BKFFT02 = 2,
    CUFHEDB_CEREAL_KSK10 = 10,
    CUFHEDB_CEREAL_KSK20 = 20,
    CUFHEDB_CEREAL_KSK21 = 21
};
CUFHEDB_API int cufhedb_cereal_key_payload(const char *path, int kind, uint64_t *offset, uint64_t *bytes);
CUFHEDB_API int cufhedb_load_cereal_key(cufhedb_ctx *ctx, const char *path, int kind);
/* deterministic lvl1 TLWE encryptions of B messages (device arrays), counter
 * blocks idx0.. of generator stream `stream_id` (test/benchmark inputs) */
CUFHEDB_API int cufhedb_encrypt_lvl1(cufhedb_ctx *ctx, uint64_t seed, uint64_t stream_id, uint64_t idx0, const uint32_t *msg,
                         uint32_t *out, int B, cufhedb_stream_t stream);
/* the same for lvl2 TLWEs (2049 x uint64) under the lvl2 key */
CUFHEDB_API int cufhedb_encrypt_lvl2(cufhedb_ctx *ctx, uint64_t seed, uint64_t stream_id, uint64_t idx0,
                                     const uint64_t *msg, uint64_t *out, int B, cufhedb_stream_t stream);

/* decryption phases b - <a, key> (mod 2^32 / 2^64) of B lvl1 / lvl2 TLWEs, the
 * quantity tlweSymDecrypt / tlweSymInt32Decrypt round (TFHEpp src/tlwe.cpp:
 * 18-91, src/HEDB/comparison/tfhepp_utils.h:32-45); `key` is a device array of
 * 1024 (lvl1) / 2048 (lvl2) key words, or NULL for the deterministic key set's */
CUFHEDB_API int cufhedb_phase_lvl1(cufhedb_ctx *ctx, const uint32_t *ct, const uint32_t *key, uint32_t *phase, int B,
                                   cufhedb_stream_t stream);
CUFHEDB_API int cufhedb_phase_lvl2(cufhedb_ctx *ctx, const uint64_t *ct, const uint64_t *key, uint64_t *phase, int B,
                                   cufhedb_stream_t stream);

/* ---- batched operations on device memory ------------------------------------- */
/* B x GateBootstrappingTLWE2TLWEFFT<lvl01param> (cufft_gpu.cuh:250-294;
 * TFHEpp src/gatebootstrapping.cpp:14-23): lvl0 TLWE in, lvl1 TLWE out */
CUFHEDB_API int cufhedb_pbs_lvl01(cufhedb_ctx *ctx, const uint32_t *in_lvl0, uint32_t *out_lvl1, int B,
                      const cufhedb_testvec *tv, int precision, cufhedb_stream_t stream);
/* B x GateBootstrappingTLWE2TLWEFFT<lvl02param> (FP64): lvl0 TLWE in, lvl2
 * TLWE (2049 x uint64) out; test vectors of 2048 64-bit words */
CUFHEDB_API int cufhedb_pbs_lvl02(cufhedb_ctx *ctx, const uint32_t *in_lvl0, uint64_t *out_lvl2, int B,
                                  const cufhedb_testvec *tv, cufhedb_stream_t stream);
/* B x IdentityKeySwitch<lvl10/20/21param> (TFHEpp src/keyswitch.cpp:11-48).
 * kind 10: in = B x 1025 uint32; kinds 20, 21: in = B x 2049 uint64.
 * out = B x 673 (10, 20) or B x 1025 (21) uint32. */
CUFHEDB_API int cufhedb_iks(cufhedb_ctx *ctx, int kind, const void *in, uint32_t *out, int B, cufhedb_stream_t stream);
/* B two-input lvl1 gates (TFHEpp HomNAND etc., src/gate.cpp:50-181):
 * IKS10 of the combined input, then PBS01 with the constant mu = 2^29 test vector */
CUFHEDB_API int cufhedb_gate_lvl1(cufhedb_ctx *ctx, int gate, const uint32_t *ca, const uint32_t *cb, uint32_t *out, int B,
                      int precision, cufhedb_stream_t stream);
/* cufhedb_gate_lvl1 without any allocation, for callers that cannot let a
 * library allocate device memory while they run (an engine that reserves all
 * device memory up front, or an allocator that owns the device).  No
 * counterpart in the reference.  The key-switched intermediate lives in a
 * fixed per-device array inside the library (2.63 MiB, held by every GPU that
 * loads the library until exit; reserved by cufhedb_ctx_create, which looks
 * up its address, so no call of this entry point allocates): B <= 1024 gates
 * per call, larger batches are rejected with CUFHEDB_ERR_ARG.  All calls on a
 * device share that array, so calls that overlap on the GPU race; order them
 * on one stream.  The caller's current device is left as it was. */
CUFHEDB_API int cufhedb_gate_lvl1_noalloc(cufhedb_ctx *ctx, int gate, const uint32_t *ca, const uint32_t *cb,
                                          uint32_t *out, int B, int precision, cufhedb_stream_t stream);
/* Prepared (frequency-domain) TRGSWs for the external product: 98,304 bytes
 * each, in the engine's layout for the given precision.  From integer
 * TRGSW<lvl1param> ([6][2][1024] uint32, device memory), or (FP64 only) from
 * TFHEpp's TRGSWFFT<lvl1param> ([6][2][1024] double, device memory). */
CUFHEDB_API int cufhedb_trgsw_prepare_lvl1(cufhedb_ctx *ctx, const uint32_t *trgsw, void *out, int B, int precision,
                                           cufhedb_stream_t stream);
CUFHEDB_API int cufhedb_trgswfft_prepare_lvl1(cufhedb_ctx *ctx, const double *trgswfft, void *out, int B,
                                              cufhedb_stream_t stream);
/* B x trgswfftExternalProduct<lvl1param> (TFHEpp src/trgsw.cpp:77-103; the
 * reference's ExternalProduct_st, cufft_gpu.cuh:228-248): out_i = trgsw_i (x) trlwe_i,
 * trlwe / out = B x [2][1024] uint32; `shared` != 0 uses one TRGSW for all. */
CUFHEDB_API int cufhedb_extprod_lvl1(cufhedb_ctx *ctx, const uint32_t *trlwe, const void *trgsw, uint32_t *out,
                                     int B, int shared, int precision, cufhedb_stream_t stream);
/* lvl2 external products (FP64): prepared TRGSWs are 262,144 bytes each,
 * from integer TRGSW<lvl2param> ([8][2][2048] uint64) or TFHEpp's
 * TRGSWFFT<lvl2param> ([8][2][2048] double); trlwe / out = B x [2][2048] uint64 */
CUFHEDB_API int cufhedb_trgsw_prepare_lvl2(cufhedb_ctx *ctx, const uint64_t *trgsw, void *out, int B,
                                           cufhedb_stream_t stream);
CUFHEDB_API int cufhedb_trgswfft_prepare_lvl2(cufhedb_ctx *ctx, const double *trgswfft, void *out, int B,
                                              cufhedb_stream_t stream);
CUFHEDB_API int cufhedb_extprod_lvl2(cufhedb_ctx *ctx, const uint64_t *trlwe, const void *trgsw, uint64_t *out,
                                     int B, int shared, cufhedb_stream_t stream);
/* B TwistIFFT<lvl2param> / TwistFFT<lvl2param>, TFHEpp layout */
CUFHEDB_API int cufhedb_twist_ifft_lvl2(cufhedb_ctx *ctx, const uint64_t *in, double *out, int B,
                                        cufhedb_stream_t stream);
CUFHEDB_API int cufhedb_twist_fft_lvl2(cufhedb_ctx *ctx, const double *in, uint64_t *out, int B,
                                       cufhedb_stream_t stream);
/* B TwistIFFT<lvl1param> / TwistFFT<lvl1param> in TFHEpp's frequency layout
 * (include/mulfft.hpp:57-121; the reference's ifft_st / fft_st, cufft_gpu.cuh:187-211) */
CUFHEDB_API int cufhedb_twist_ifft_lvl1(cufhedb_ctx *ctx, const uint32_t *in, double *out, int B, cufhedb_stream_t stream);
CUFHEDB_API int cufhedb_twist_fft_lvl1(cufhedb_ctx *ctx, const double *in, uint32_t *out, int B, cufhedb_stream_t stream);

/* ---- batched operator layer (cuHEDB, src/cuHEDB/gatebootstrap_gpu.cuh,
 *      msb_gpu.cuh, HomCompare_gpu.cuh): every call applies the operator to B
 *      rows; lvl1 ciphertexts are 1025 x uint32, lvl2 ciphertexts 2049 x uint64;
 *      `logic` != 0 is the reference's LOGIC result type (+-1/8), 0 ARITHMETIC;
 *      `precision` selects the lvl0 -> lvl1 bootstraps' path (lvl2 is FP64). */
/* MSBGateBootstrapping (gatebootstrap_gpu.cuh:31-78): level pairs 1->1, 2->1, 2->2 */
CUFHEDB_API int cufhedb_msb_bootstrap(cufhedb_ctx *ctx, int in_level, int out_level, const void *in, void *out,
                                      int B, int logic, int precision, cufhedb_stream_t stream);
/* IdeGateBootstrapping (gatebootstrap_gpu.cuh:80-117): level pairs 1->1, 2->1, 2->2 */
CUFHEDB_API int cufhedb_ide_bootstrap(cufhedb_ctx *ctx, int in_level, int out_level, const void *in, void *out,
                                      int B, uint32_t scale_bits, int precision, cufhedb_stream_t stream);
/* LOG_to_ARI and log_rescale (gatebootstrap_gpu.cuh:154-168) */
CUFHEDB_API int cufhedb_log_to_ari(cufhedb_ctx *ctx, const uint32_t *in, uint32_t *out, int B, int precision,
                                   cufhedb_stream_t stream);
CUFHEDB_API int cufhedb_log_rescale(cufhedb_ctx *ctx, const uint32_t *in, uint32_t *out, int B,
                                    uint32_t scale_bits, int precision, cufhedb_stream_t stream);
/* HomAND / HomOR of LOGIC inputs (gatebootstrap_gpu.cuh:124-152) */
CUFHEDB_API int cufhedb_hom_and(cufhedb_ctx *ctx, const uint32_t *ca, const uint32_t *cb, uint32_t *out, int B,
                                int logic, int precision, cufhedb_stream_t stream);
CUFHEDB_API int cufhedb_hom_or(cufhedb_ctx *ctx, const uint32_t *ca, const uint32_t *cb, uint32_t *out, int B,
                               int logic, int precision, cufhedb_stream_t stream);
/* HomMSB (msb_gpu.cuh:57-62 for lvl1 input, :175-193 for lvl2 input); plain_bits
 * beyond 10 (lvl1) or 33 (lvl2) fail with CUFHEDB_ERR_ARG ("Plain bits out.") */
CUFHEDB_API int cufhedb_hom_msb(cufhedb_ctx *ctx, int in_level, const void *in, uint32_t *out_lvl1, int B,
                                uint32_t plain_bits, int logic, int precision, cufhedb_stream_t stream);
/* greater_than (op 0), greater_than_equal (1), less_than (2), less_than_equal (3),
 * equal (4) of level-`level` ciphertexts c1, c2 (HomCompare_gpu.cuh:13-76) */
CUFHEDB_API int cufhedb_compare(cufhedb_ctx *ctx, int op, int level, const void *c1, const void *c2,
                                uint32_t *out_lvl1, int B, uint32_t plain_bits, int logic, int precision,
                                cufhedb_stream_t stream);

/* One filter query of a queue: `rows` comparisons c1[i] op c2[i] of level-
 * `level` ciphertexts (device memory), results to `out` (rows lvl1 TLWEs). */
typedef struct {
    int level;           /* 1 or 2 */
    int op;              /* as cufhedb_compare: 0 gt, 1 ge, 2 lt, 3 le, 4 eq */
    uint32_t plain_bits;
    int logic;
    int rows;
    const void *c1, *c2;
    uint32_t *out;
} cufhedb_query;
/* Runs a whole queue of such queries (the reference's query programs run one
 * query at a time as a row loop of one-row operator calls,
 * test/HE3_Query/TPCH_Q6.cu:158-209): queries that share a comparison chain
 * are packed into batches of at most max_batch_rows rows, smallest first; the
 * batches run in order of cost per completed query on `nstreams` streams
 * (1..16), so different levels' bootstraps overlap.  latency_ms[i] receives
 * query i's completion time from the start of the queue and total_ms (may be
 * NULL) the whole queue's; returns when every result is in place. */
CUFHEDB_API int cufhedb_queue_run(cufhedb_ctx *ctx, const cufhedb_query *q, int nq, int precision,
                                  int max_batch_rows, int nstreams, float *latency_ms, float *total_ms);
/* The plan cufhedb_queue_run follows, host only (no device, no context):
 * t01_ms / t02_ms are the per-ciphertext times of lvl01 / lvl02 bootstraps
 * (queue_run takes them from the context's launch-shape table).  Batches are
 * numbered in run order; batch_of[i] (nq entries) receives query i's batch,
 * stream_of_batch[b] (up to nq entries) the stream batch b is queued on, and
 * *nbatches their count.  The query pointers are not read. */
CUFHEDB_API int cufhedb_queue_plan(const cufhedb_query *q, int nq, double t01_ms, double t02_ms,
                                   int max_batch_rows, int nstreams, int *batch_of, int *stream_of_batch,
                                   int *nbatches);

/* B negacyclic products out_i = a_i * m (the reference's PolyMul_st,
 * src/cuHEDB/fft_gpu/cufft_gpu.cuh:214-226, which multiplies by the
 * polynomial its engine last transformed): TwistFFT(TwistIFFT(a_i) x m) in
 * FP64.  a / out: B polynomials (1024 uint32 or 2048 uint64); m_fd: the
 * multiplier in TFHEpp's frequency-domain layout (TwistIFFT output, N doubles),
 * one for all rows when `shared` != 0, else B of them.  Device memory. */
CUFHEDB_API int cufhedb_polymul_lvl1(cufhedb_ctx *ctx, const uint32_t *a, const double *m_fd, uint32_t *out, int B,
                                     int shared, cufhedb_stream_t stream);
CUFHEDB_API int cufhedb_polymul_lvl2(cufhedb_ctx *ctx, const uint64_t *a, const double *m_fd, uint64_t *out, int B,
                                     int shared, cufhedb_stream_t stream);

/* ArcEDB comparisons (cuARCEDB::greater_than_tfhepp / less_than_tfhepp /
 * equality_tfhepp, src/cuHEDB/comparable_gpu.cuh:52-168; CPU twins
 * src/ARCEDB/comparison/comparable.cpp:506-729) of B rows of D radix-1024
 * digits.  trlwe: D x B x [2][1024] uint32, the TRLWE of mu X^{x_d}
 * (exponent_encrypt); trgsw: D x B prepared TRGSWs (98,304 bytes each, from
 * cufhedb_trgsw_prepare_lvl1 / cufhedb_trgswfft_prepare_lvl1) of X^{-y_d}
 * (exponent_encrypt_rgsw with is_negative); digit 0 least significant.
 * op 0: greater_than (+mu iff x > y), 1: less_than exactly as the reference
 * computes it (x_d <= y_d per digit; over several digits the lower digits'
 * result is complemented when the top digits are equal), 2: equality,
 * 3: strict less_than (x < y, combining like greater_than; no counterpart in
 * the reference).  out: B lvl1 TLWEs (+-mu); D > 1 needs the lvl10 and lvl01 keys. */
CUFHEDB_API int cufhedb_arc_compare(cufhedb_ctx *ctx, int op, const uint32_t *trlwe, const void *trgsw,
                                    uint32_t *out, int B, int D, int precision, cufhedb_stream_t stream);

/* ---- CUDA-graph capture of an operator DAG: everything enqueued on `stream`
 *      between begin and end (which must be a non-default stream) becomes one
 *      graph, replayed by cufhedb_graph_launch. */
typedef struct cufhedb_graph cufhedb_graph;
CUFHEDB_API int cufhedb_graph_begin(cufhedb_ctx *ctx, cufhedb_stream_t stream);
CUFHEDB_API int cufhedb_graph_end(cufhedb_ctx *ctx, cufhedb_stream_t stream, cufhedb_graph **out);
CUFHEDB_API int cufhedb_graph_launch(cufhedb_graph *graph, cufhedb_stream_t stream);
CUFHEDB_API int cufhedb_graph_destroy(cufhedb_graph *graph);

/* ---- host-buffer entry points (synchronous; the _st calls of cufft_gpu.cuh) ---- */
CUFHEDB_API int cufhedb_pbs_lvl01_host(cufhedb_ctx *ctx, const uint32_t *in_lvl0, uint32_t *out_lvl1, int B,
                           const cufhedb_testvec *tv, int precision);
/* host-memory external products with TFHEpp TRGSWFFT<lvl1param> operands (FP64) */
CUFHEDB_API int cufhedb_extprod_lvl1_host(cufhedb_ctx *ctx, const uint32_t *trlwe, const double *trgswfft,
                                          uint32_t *out, int B, int shared);
CUFHEDB_API int cufhedb_gate_lvl1_host(cufhedb_ctx *ctx, int gate, const uint32_t *ca, const uint32_t *cb, uint32_t *out, int B,
                           int precision);

/* cufhedb_compare on host buffers (c1, c2: B ciphertexts of `level`; out: B
 * lvl1 TLWEs), synchronous like the other *_host calls */
CUFHEDB_API int cufhedb_compare_host(cufhedb_ctx *ctx, int op, int level, const void *c1, const void *c2,
                                     uint32_t *out_lvl1, int B, uint32_t plain_bits, int logic, int precision);
/* Row sharding over several contexts (one per GPU; the reference binds device
 * 0 only, src/cuHEDB/gatebootstrap_gpu.cuh:11-15): the B rows split into
 * nctx contiguous slices, each run by its own host thread through that
 * context's host-buffer call; results land in `out` in row order.  Every
 * context needs the keys the operator uses.  No data crosses between
 * devices. */
CUFHEDB_API int cufhedb_gate_lvl1_host_multi(cufhedb_ctx *const *ctxs, int nctx, int gate, const uint32_t *ca,
                                             const uint32_t *cb, uint32_t *out, int B, int precision);
CUFHEDB_API int cufhedb_compare_host_multi(cufhedb_ctx *const *ctxs, int nctx, int op, int level, const void *c1,
                                           const void *c2, uint32_t *out_lvl1, int B, uint32_t plain_bits, int logic,
                                           int precision);

/* Self-test of the kernels' bounded waits (no counterpart in the reference,
 * which has none): one block waits `polls` times (1 .. 2^20) for a key-ring
 * chunk that is never issued, gives up, records the failure and returns.
 * Returns what cufhedb_sync then reports: CUFHEDB_ERR_DEVICE with the wait's
 * code when the path works; the context stays usable afterwards. */
CUFHEDB_API int cufhedb_selftest_wait_timeout(cufhedb_ctx *ctx, uint32_t polls);

/* ---- launch-shape autotuner --------------------------------------------------- */
/* The persistent PBS kernels come in three launch shapes each (ciphertexts
 * per CTA): lvl01 7, 8 and 4, lvl02 3, 2 and 1.  A launch of B ciphertexts
 * takes ceil(ceil(B / shape) / SMs) passes; every launch (PBS, gates,
 * operator chains) picks the shape with the least passes x measured pass
 * time, ties to the earlier shape; without measurements all pass times count
 * as equal.  CUFHEDB_SPLIT32 launches also pick the layout of the first
 * transform step, on the CUDA cores or on the tensor cores (the
 * CUFHEDB_SPLIT32_TC kernel), by the same rule over both tables once both
 * are measured, ties to the CUDA cores.  No counterpart in the reference,
 * which runs one ciphertext per launch.  The tuning calls are synchronous;
 * call them outside stream capture. */
/* times one full pass of each lvl01 shape for `precision` (uniform random lvl0
 * inputs, the loaded key) and keeps them in the context; ms_w7 / ms_w8 (may be
 * NULL) receive the 7- and 8-per-CTA pass times */
CUFHEDB_API int cufhedb_autotune_pbs01(cufhedb_ctx *ctx, int precision, float *ms_w7, float *ms_w8);
/* the same for the lvl02 shapes; ms (may be NULL) receives the 3 pass times */
CUFHEDB_API int cufhedb_autotune_pbs02(cufhedb_ctx *ctx, float *ms);
/* the context's table for a level (1 with FP64 or SPLIT32, 2 with FP64):
 * shapes[3] and pass_ms[3] (either may be NULL); returns 3 */
CUFHEDB_API int cufhedb_autotune_table(cufhedb_ctx *ctx, int level, int precision, int *shapes, float *pass_ms);
/* the shape (ciphertexts per CTA) a launch of B ciphertexts would use now */
CUFHEDB_API int cufhedb_launch_shape(cufhedb_ctx *ctx, int level, int precision, int B, int *shape);
/* the stage-1 layout a CUFHEDB_SPLIT32 launch of B ciphertexts would use now:
 * *tensor_core_stage1 = 1 (tensor cores) or 0 (CUDA cores) */
CUFHEDB_API int cufhedb_launch_layout(cufhedb_ctx *ctx, int B, int *tensor_core_stage1);
/* persist / restore the context's pass times: a text file keyed by the device
 * name, the SM count and a hash of the parameter set and shape lists; load
 * refuses a table made for anything else (CUFHEDB_ERR_ARG), after which the
 * caller tunes again */
CUFHEDB_API int cufhedb_autotune_save(cufhedb_ctx *ctx, const char *path);
CUFHEDB_API int cufhedb_autotune_load(cufhedb_ctx *ctx, const char *path);

/* ---- diagnostics ------------------------------------------------------------ */
/* measured CUDA-core FMA throughput (TFLOP/s) of `device`, FP64 (fp64 != 0) or
 * FP32: the roofline denominator of the bootstrapping kernels */
CUFHEDB_API int cufhedb_measure_fma_peak(int device, int fp64, double *tflops);

#ifdef __cplusplus
}
#endif
#endif /* CUFHEDB_B200_H */
