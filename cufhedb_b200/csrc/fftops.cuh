#pragma once
#include "common.cuh"
#include "fft_f64.cuh"

namespace cfdb {

cudaError_t launch_twist_ifft1(double *out, const uint32_t *in, int B, const Fft512Tables *T, cudaStream_t st);
cudaError_t launch_twist_fft1(uint32_t *out, const double *in, int B, const Fft512Tables *T, cudaStream_t st);

}  // namespace cfdb
