#pragma once
#include "common.cuh"
#include "fft1024_f64.cuh"
#include "pbs_common.cuh"

namespace cfdb {

struct Pbs02Args {
    const uint32_t *in;      // B x (N0+1) lvl0 TLWE
    uint64_t *out;           // B x (N2+1) lvl2 TLWE
    int B;
    const double2 *bk;       // N0 x 8 rows x 2 outputs x 1024 complex (chunk layout [s][t])
    const void *tables;      // Fft1024Tables in global memory
    TestVec tv;
    uint64_t out_b_add;      // added to the b word of every output
    int *err;
};

struct ExtProd2Args {
    const uint64_t *trlwe;   // B x 2 x 2048
    const double2 *trgsw;    // prepared: B (or 1) x 8 rows x 2 outputs x 1024 complex
    uint64_t *out;           // B x 2 x 2048
    int B;
    int shared;
    const Fft1024Tables *tables;
};

// p: ciphertexts per CTA, one of PBS02_SHAPES
cudaError_t launch_pbs02_f64(const Pbs02Args &a, int num_sms, int p, cudaStream_t st);
cudaError_t init_pbs02_f64();
cudaError_t launch_extprod2(const ExtProd2Args &a, cudaStream_t st);
cudaError_t bk02_to_fft(double2 *dst, const uint64_t *src, int rows, const Fft1024Tables *T, cudaStream_t st);
cudaError_t bkfft02_permute(double2 *dst, const double *src, int rows, cudaStream_t st);
cudaError_t launch_twist_ifft2(double *out, const uint64_t *in, int B, const Fft1024Tables *T, cudaStream_t st);
cudaError_t launch_twist_fft2(uint64_t *out, const double *in, int B, const Fft1024Tables *T, cudaStream_t st);

}  // namespace cfdb
