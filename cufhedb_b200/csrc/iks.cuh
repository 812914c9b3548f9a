#pragma once
#include "common.cuh"

namespace cfdb {

// kind 10: in32 = B x 1025 lvl1 TLWE (optionally sa*in32 + sb*in32b, b += offset)
// kind 20/21: in64 = B x 2049 lvl2 TLWE
// out: B x 673 (kinds 10, 20) or B x 1025 (kind 21)
struct IksArgs {
    const uint32_t *in32;
    const uint32_t *in32b;
    const uint64_t *in64;
    int sa, sb;
    uint32_t offset;     // added to b of the 32-bit input (gate / MSB offsets)
    uint64_t offset64;   // added to b of the 64-bit input before rescaling
    uint32_t *out;
    const uint32_t *ksk;   // rows of ksk_pitch(out width) words, 16-byte aligned
    int B;
};

cudaError_t launch_iks(const IksArgs &a, int kind, cudaStream_t st);

}  // namespace cfdb
