// Batched identity key switching, lvl1->lvl0, lvl2->lvl0, lvl2->lvl1.
//
// Restates IdentityKeySwitch<P> (thirdparty/TFHEpp/src/keyswitch.cpp:11-48):
//   b' = b (same width) or round(b / 2^32) (64 -> 32 bit),
//   for each input coefficient i and digit j < t:
//     a_ij = ((a_i + prec_offset) >> (w - (j+1) basebit)) & (2^basebit - 1)
//     if a_ij != 0: res -= ksk[i][j][a_ij - 1]
// The reference runs this on the host for every GPU bootstrap
// (src/cuHEDB/gatebootstrap_gpu.cuh:42,133).  Here it is an HBM-bound gather:
// one CTA per ciphertext walks the input coefficients in chunks of NT; each
// chunk's digits are decoded into a shared list of selected key rows (in key
// order), then
// every thread accumulates a fixed set of output words over those rows with
// several rows' loads in flight.  All CTAs of a batch walk the key in the same
// order, so concurrently running CTAs that select the same row share it in L2.
#include "common.cuh"
#include "iks.cuh"

namespace cfdb {

namespace {

template <int NOUT, int NT>
__device__ __forceinline__ void gather_rows(const uint32_t *__restrict__ ksk, const uint32_t *rowid, int nrows,
                                            uint32_t *acc)
{
    constexpr int PER = (NOUT + NT - 1) / NT;
    constexpr int U = 4;
    const int t = threadIdx.x;
    int r = 0;
    for (; r + U <= nrows; r += U) {
        uint32_t v[U][PER];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const uint32_t *row = ksk + (size_t)rowid[r + u] * NOUT;
#pragma unroll
            for (int p = 0; p < PER; ++p) {
                const int k = t + p * NT;
                v[u][p] = (k < NOUT) ? __ldg(row + k) : 0u;
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
            for (int p = 0; p < PER; ++p) acc[p] -= v[u][p];
    }
    for (; r < nrows; ++r) {
        const uint32_t *row = ksk + (size_t)rowid[r] * NOUT;
#pragma unroll
        for (int p = 0; p < PER; ++p) {
            const int k = t + p * NT;
            if (k < NOUT) acc[p] -= __ldg(row + k);
        }
    }
}

// input coefficient k of ciphertext `ct`; for the lvl1 gate form the input is
// sa*ca + sb*cb (TFHEpp HomGate, src/gate.cpp:50-58)
template <bool WIDE>
__device__ __forceinline__ uint64_t iks_input(const IksArgs &a, size_t base, int k)
{
    if constexpr (WIDE) {
        return a.in64[base + k];
    } else {
        uint32_t x = a.in32[base + k];
        if (a.in32b) x = (uint32_t)a.sa * x + (uint32_t)a.sb * a.in32b[base + k];
        else x = (uint32_t)a.sa * x;
        return x;
    }
}

template <int NT, bool WIDE, int NIN, int BASEBIT, int TT, int NOUT>
__global__ void __launch_bounds__(NT) iks_kernel(IksArgs a)
{
    static_assert(NT % 32 == 0, "whole warps");
    constexpr int NW = NT / 32;
    __shared__ uint32_t rowid[NT * TT];
    __shared__ int wsum[NW];
    constexpr int W = WIDE ? 64 : 32;
    constexpr uint64_t prec = 1ull << (W - (1 + BASEBIT * TT));
    constexpr uint32_t mask = (1u << BASEBIT) - 1;
    constexpr int PER = (NOUT + NT - 1) / NT;
    const int ct = blockIdx.x;
    const size_t base = (size_t)ct * (NIN + 1);
    uint32_t acc[PER];
#pragma unroll
    for (int p = 0; p < PER; ++p) acc[p] = 0;

    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int i0 = 0; i0 < NIN; i0 += NT) {
        // the chunk's selected rows, compacted in key order (ascending i, j)
        // so that every CTA of the batch walks the key the same way and rows
        // that several ciphertexts select are fetched close together in time
        const int i = i0 + threadIdx.x;
        uint32_t ids[TT];
        int n = 0;
        if (i < NIN) {
            const uint64_t abar = iks_input<WIDE>(a, base, i) + prec;
#pragma unroll
            for (int j = 0; j < TT; ++j) {
                const uint32_t d = (uint32_t)((WIDE ? abar : (uint32_t)abar) >> (W - (j + 1) * BASEBIT)) & mask;
                if (d) ids[n++] = ((uint32_t)i * TT + j) * mask + d - 1;
            }
        }
        int incl = n;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, incl, off);
            if (lane >= off) incl += y;
        }
        if (lane == 31) wsum[wid] = incl;
        __syncthreads();
        int pos = incl - n, total = 0;
#pragma unroll
        for (int w = 0; w < NW; ++w) {
            const int c = wsum[w];
            if (w < wid) pos += c;
            total += c;
        }
#pragma unroll
        for (int j = 0; j < TT; ++j)
            if (j < n) rowid[pos + j] = ids[j];
        __syncthreads();
        gather_rows<NOUT, NT>(a.ksk, rowid, total, acc);
        __syncthreads();
    }

    uint32_t bnew;
    if constexpr (WIDE) bnew = (uint32_t)((a.in64[base + NIN] + a.offset64 + (1ull << 31)) >> 32);
    else bnew = (uint32_t)iks_input<false>(a, base, NIN) + a.offset;
    uint32_t *o = a.out + (size_t)ct * NOUT;
#pragma unroll
    for (int p = 0; p < PER; ++p) {
        const int k = threadIdx.x + p * NT;
        if (k < NOUT - 1) o[k] = acc[p];
        else if (k == NOUT - 1) o[k] = acc[p] + bnew;
    }
}

}  // namespace

cudaError_t launch_iks(const IksArgs &a, int kind, cudaStream_t st)
{
    if (a.B <= 0) return cudaSuccess;
    if (kind == 10)
        iks_kernel<256, false, N1, KS10_BASEBIT, KS10_T, N0 + 1><<<a.B, 256, 0, st>>>(a);
    else if (kind == 20)
        iks_kernel<256, true, N2, KS20_BASEBIT, KS20_T, N0 + 1><<<a.B, 256, 0, st>>>(a);
    else if (kind == 21)
        iks_kernel<352, true, N2, KS21_BASEBIT, KS21_T, N1 + 1><<<a.B, 352, 0, st>>>(a);
    else
        return cudaErrorInvalidValue;
    return cudaGetLastError();
}

}  // namespace cfdb
