#pragma once
#include "common.cuh"
#include "fft_f64.cuh"

namespace cfdb {

// generator streams and counter-block sizes of the deterministic key set
enum : uint64_t {
    ST_SK0 = 1, ST_SK1 = 2, ST_SK2 = 3,
    ST_KSK10 = 0x10, ST_KSK20 = 0x11, ST_KSK21 = 0x12,
    ST_BK01 = 0x20, ST_BK02 = 0x21,
};
constexpr uint64_t CB_TLWE32 = 2048, CB_TLWE64 = 4096;
// noise scales round(alpha * 2^w * sqrt(3)) for the params/128bit.hpp alphas
constexpr int64_t NS_LVL0 = 113512;   // alpha 2^-16, 32-bit torus
constexpr int64_t NS_LVL1 = 222;      // alpha 2^-25, 32-bit torus
constexpr int64_t NS_LVL2 = 7094;     // alpha 2^-52, 64-bit torus

uint64_t stream_key(uint64_t seed, uint64_t stream);
uint64_t host_draw(uint64_t seed, uint64_t stream, uint64_t ctr);
void host_secret_keys(uint64_t seed, uint32_t *s0, uint32_t *s1, uint64_t *s2);

// rows of ksk_pitch(width) words (common.cuh), pad words zero
cudaError_t gen_ksk(uint32_t *out, int kind, uint64_t seed, const void *key_dom_d, const uint32_t *key_tgt_d,
                    cudaStream_t st);
cudaError_t gen_bk01(uint32_t *out, uint64_t seed, const uint32_t *s0_d, const int *s1pos_d, int ns1,
                     cudaStream_t st);
cudaError_t gen_bk02(uint64_t *out, uint64_t seed, const uint32_t *s0_d, const int *s2pos_d, int ns2,
                     cudaStream_t st);
cudaError_t encrypt_tlwe32(uint32_t *out, const uint32_t *msg_d, int B, int n, const uint32_t *key_d, int64_t ns,
                           uint64_t seed, uint64_t stream, uint64_t idx0, cudaStream_t st);
cudaError_t encrypt_tlwe64(uint64_t *out, const uint64_t *msg_d, int B, int n, const uint64_t *key_d, int64_t ns,
                           uint64_t seed, uint64_t stream, uint64_t idx0, cudaStream_t st);
cudaError_t fill_random32(uint32_t *out, size_t n, uint64_t seed, uint64_t stream, cudaStream_t st);
cudaError_t tlwe_phase32(uint32_t *phase, const uint32_t *ct, int B, int n, const uint32_t *key_d, cudaStream_t st);
cudaError_t tlwe_phase64(uint64_t *phase, const uint64_t *ct, int B, int n, const uint64_t *key_d, cudaStream_t st);
cudaError_t bk01_to_fft(double2 *dst, const uint32_t *src, int rows, const Fft512Tables *T, cudaStream_t st);
cudaError_t bkfft01_permute(double2 *dst, const double *src, int rows, cudaStream_t st);
cudaError_t bk01_to_split(float4 *dst, const uint32_t *src, int rows, const Fft512Tables *T, cudaStream_t st);
cudaError_t bk01_fft_to_int(uint32_t *dst, const double2 *src, int rows, const Fft512Tables *T, cudaStream_t st);

}  // namespace cfdb
