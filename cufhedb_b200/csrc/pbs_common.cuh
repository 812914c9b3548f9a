// Kernel-argument structs and helpers shared by the PBS / external-product
// kernels.
#pragma once
#include "common.cuh"
#include "fft_f64.cuh"

namespace cfdb {

// Test-vector descriptor.  The accumulator starts as (0, X^bbar * tv).
//   kind 0: constant tv[i] = value (TFHEpp mu-polygen, gatebootstrapping.hpp:132-138;
//           the GPU reference's upolygen, cuHEDB fft_gpu/BlindRotate_gpu.cuh:92-124)
//   kind 1: staircase tv[i] = 2^value * (i >> pad) (HEDB gpolygen,
//           src/HEDB/comparison/tfhepp_utils.h:113-120)
//   kind 2: an arbitrary polynomial `poly` (device memory, N words)
struct TestVec {
    int kind;
    int pad;
    uint64_t value;
    const void *poly;
};

// coefficient j of X^a * poly, a in [0, 2N]  (utils.hpp:110-125)
template <int N, typename T>
__device__ __forceinline__ T rot_coef(const T *poly, int j, uint32_t a)
{
    const uint32_t idx = (uint32_t)(j - (int)a) & (2 * N - 1);
    T v = poly[idx & (N - 1)];
    return (idx & N) ? (T)(T(0) - v) : v;
}

__device__ __forceinline__ uint32_t testvec_coef1(const TestVec &tv, uint32_t i)
{
    if (tv.kind == 0) return (uint32_t)tv.value;
    if (tv.kind == 1) return (uint32_t)((1ull << tv.value) * (uint64_t)(i >> tv.pad));
    return reinterpret_cast<const uint32_t *>(tv.poly)[i];
}

__device__ __forceinline__ uint64_t testvec_coef2(const TestVec &tv, uint32_t i)
{
    if (tv.kind == 0) return tv.value;
    if (tv.kind == 1) return (1ull << tv.value) * (uint64_t)(i >> tv.pad);
    return reinterpret_cast<const uint64_t *>(tv.poly)[i];
}

// coefficient j of X^bbar * tv for the lvl1 ring
__device__ __forceinline__ uint32_t testvec_rot1(const TestVec &tv, int j, uint32_t bbar)
{
    const uint32_t idx = (uint32_t)(j - (int)bbar) & (2 * N1 - 1);
    const uint32_t v = testvec_coef1(tv, idx & (N1 - 1));
    return (idx & N1) ? 0u - v : v;
}

__device__ __forceinline__ uint64_t testvec_rot2(const TestVec &tv, int j, uint32_t bbar)
{
    const uint32_t idx = (uint32_t)(j - (int)bbar) & (2 * N2 - 1);
    const uint64_t v = testvec_coef2(tv, idx & (N2 - 1));
    return (idx & N2) ? 0ull - v : v;
}

struct Pbs01Args {
    const uint32_t *in;      // B x (N0+1) lvl0 TLWE
    uint32_t *out;           // B x (N1+1) lvl1 TLWE
    int B;
    const double2 *bk;       // N0 x 6 chunks x 1024 complex, chunk layout [s][o][lane]
    const void *tables;      // Fft512Tables in global memory
    TestVec tv;
    uint32_t out_b_add;      // added to the b word of every output (the "+ u" of MSB/gate bootstraps)
    int *err;
};

// w: ciphertexts (warps) per CTA, one of PBS01_SHAPES
cudaError_t launch_pbs01_f64(const Pbs01Args &a, int num_sms, int w, cudaStream_t st);
// bk: split-precision key (float4 hi/lo chunk layout), tables: Fft512TablesF
cudaError_t launch_pbs01_split(const Pbs01Args &a, int num_sms, int w, cudaStream_t st);
// the same with the first step of every digit transform on the tensor cores
cudaError_t launch_pbs01_split_tc(const Pbs01Args &a, int num_sms, int w, cudaStream_t st);

// Launch shapes of the persistent PBS kernels, as ciphertexts per CTA: lvl01
// 7 (with a producer warp on the split path), 8 and 4 (one warp per SM
// sub-partition: the shortest pass, for batches that leave SMs idle); lvl02
// 3, 2 and 1 (four warps per ciphertext).  Each CTA works through
// ceil(ceil(B / w) / SMs) passes of w ciphertexts; the autotuner measures
// one full pass of every shape, and a launch takes the shape with the least
// passes x pass time.  Ties go to the earlier shape in the list, so with no
// measurement (all pass times equal) the fewest passes win and a one-pass
// batch runs 7 (lvl01) or 3 (lvl02) per CTA.
constexpr int NSHAPES = 3;
constexpr int PBS01_SHAPES[NSHAPES] = {7, 8, 4};
constexpr int PBS02_SHAPES[NSHAPES] = {3, 2, 1};

inline int choose_shape(int B, int num_sms, const int shapes[NSHAPES], const float pass_ms[NSHAPES])
{
    int best = 0;
    float best_cost = 0.0f;
    for (int i = 0; i < NSHAPES; ++i) {
        const int w = shapes[i];
        const int groups = (B + w - 1) / w;
        const float cost = (float)((groups + num_sms - 1) / num_sms) * pass_ms[i];
        if (i == 0 || cost < best_cost) {
            best = i;
            best_cost = cost;
        }
    }
    return shapes[best];
}
inline int pbs01_choose_w(int B, int num_sms, const float pass_ms[NSHAPES])
{
    return choose_shape(B, num_sms, PBS01_SHAPES, pass_ms);
}
// a pass-time table still at the context's untuned default (every entry
// exactly 1.0; no measured pass takes exactly 1 ms)
inline bool shape_table_measured(const float pass_ms[NSHAPES])
{
    for (int i = 0; i < NSHAPES; ++i)
        if (pass_ms[i] != 1.0f) return true;
    return false;
}
// The split path's launch: the shape and the stage-1 layout (CUDA cores, or
// tensor cores when both tables are measured) with the least passes x pass
// time; ties go to the CUDA-core layout, then to the earlier shape.
struct SplitLaunch {
    int w;
    bool tc;
};
inline SplitLaunch pbs01_split_choose(int B, int num_sms, const float cc_ms[NSHAPES], const float tc_ms[NSHAPES])
{
    auto cost = [&](int i, const float *t) {
        const int groups = (B + PBS01_SHAPES[i] - 1) / PBS01_SHAPES[i];
        return (float)((groups + num_sms - 1) / num_sms) * t[i];
    };
    SplitLaunch best{PBS01_SHAPES[0], false};
    float best_cost = cost(0, cc_ms);
    for (int i = 1; i < NSHAPES; ++i)
        if (cost(i, cc_ms) < best_cost) best = {PBS01_SHAPES[i], false}, best_cost = cost(i, cc_ms);
    if (shape_table_measured(cc_ms) && shape_table_measured(tc_ms))
        for (int i = 0; i < NSHAPES; ++i)
            if (cost(i, tc_ms) < best_cost) best = {PBS01_SHAPES[i], true}, best_cost = cost(i, tc_ms);
    return best;
}
inline int pbs02_choose_p(int B, int num_sms, const float pass_ms[NSHAPES])
{
    return choose_shape(B, num_sms, PBS02_SHAPES, pass_ms);
}
cudaError_t init_pbs01_f64();
cudaError_t init_pbs01_split();

}  // namespace cfdb
