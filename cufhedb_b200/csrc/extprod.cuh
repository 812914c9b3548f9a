#pragma once
#include "common.cuh"
#include "fft_f64.cuh"

namespace cfdb {

struct ExtProdArgs {
    const uint32_t *trlwe;   // B x 2 x 1024
    const void *trgsw;       // prepared TRGSWs: B (or 1 when shared) x 6 rows x 1024 x 16 bytes
    uint32_t *out;           // B x 2 x 1024
    int B;
    int shared;              // 1: one TRGSW for the whole batch
    const void *tables;      // Fft512Tables (FP64 path) or Fft512TablesF (split path)
    int *err;                // device error word (bounded waits that gave up)
};

// precision 0: FP64, 1: split-precision FP32
cudaError_t launch_extprod1(const ExtProdArgs &a, int precision, cudaStream_t st);
// once per process and device, before the first launch (dynamic shared memory)
cudaError_t init_extprod1();

}  // namespace cfdb
