// Batched identity key switching, lvl1->lvl0, lvl2->lvl0, lvl2->lvl1.
//
// Restates IdentityKeySwitch<P> (thirdparty/TFHEpp/src/keyswitch.cpp:11-48):
//   b' = b (same width) or round(b / 2^32) (64 -> 32 bit),
//   for each input coefficient i and digit j < t:
//     a_ij = ((a_i + prec_offset) >> (w - (j+1) basebit)) & (2^basebit - 1)
//     if a_ij != 0: res -= ksk[i][j][a_ij - 1]
// The reference runs this on the host for every GPU bootstrap
// (src/cuHEDB/gatebootstrap_gpu.cuh:42,133).  Here it is an HBM-bound gather
// over key rows padded to 16-byte multiples (ksk_pitch), read as uint4:
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

// a 16-byte read-only load, issued where it stands (volatile: the U loads of
// a group are all in flight before the first subtraction)
__device__ __forceinline__ uint4 ldg_v4(const uint4 *p)
{
    uint4 v;
    asm volatile("ld.global.nc.v4.u32 {%0, %1, %2, %3}, [%4];"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                 : "l"(p));
    return v;
}

// a -= x, placed after the group's loads (volatile, like them)
__device__ __forceinline__ void sub_v4(uint4 &a, const uint4 &x)
{
    asm volatile("sub.u32 %0, %0, %4;\n\tsub.u32 %1, %1, %5;\n\tsub.u32 %2, %2, %6;\n\tsub.u32 %3, %3, %7;"
                 : "+r"(a.x), "+r"(a.y), "+r"(a.z), "+r"(a.w)
                 : "r"(x.x), "r"(x.y), "r"(x.z), "r"(x.w));
}

// acc[p] -= row[t + p NT] (16-byte words of the padded rows) over the listed
// rows, U rows' loads in flight per thread
template <int NP4, int NT>
__device__ __forceinline__ void gather_rows(const uint4 *__restrict__ ksk, const uint32_t *rowid, int nrows,
                                            uint4 *acc)
{
    constexpr int PER = (NP4 + NT - 1) / NT;
    constexpr int U = 8;
    const int t = threadIdx.x;
    int r = 0;
    for (; r + U <= nrows; r += U) {
        uint4 v[U][PER];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const uint4 *row = ksk + (size_t)rowid[r + u] * NP4;
#pragma unroll
            for (int p = 0; p < PER; ++p) {
                const int k = t + p * NT;
                v[u][p] = (k < NP4) ? ldg_v4(row + k) : make_uint4(0u, 0u, 0u, 0u);
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u)
#pragma unroll
            for (int p = 0; p < PER; ++p) sub_v4(acc[p], v[u][p]);
    }
    for (; r < nrows; ++r) {
        const uint4 *row = ksk + (size_t)rowid[r] * NP4;
#pragma unroll
        for (int p = 0; p < PER; ++p) {
            const int k = t + p * NT;
            if (k < NP4) {
                const uint4 x = ldg_v4(row + k);
                acc[p].x -= x.x;
                acc[p].y -= x.y;
                acc[p].z -= x.z;
                acc[p].w -= x.w;
            }
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
    constexpr int NP4 = ksk_pitch(NOUT) / 4;
    constexpr int PER = (NP4 + NT - 1) / NT;
    const int ct = blockIdx.x;
    const size_t base = (size_t)ct * (NIN + 1);
    uint4 acc[PER];
#pragma unroll
    for (int p = 0; p < PER; ++p) acc[p] = make_uint4(0u, 0u, 0u, 0u);

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
        gather_rows<NP4, NT>(reinterpret_cast<const uint4 *>(a.ksk), rowid, total, acc);
        __syncthreads();
    }

    uint32_t bnew;
    if constexpr (WIDE) bnew = (uint32_t)((a.in64[base + NIN] + a.offset64 + (1ull << 31)) >> 32);
    else bnew = (uint32_t)iks_input<false>(a, base, NIN) + a.offset;
    uint32_t *o = a.out + (size_t)ct * NOUT;
#pragma unroll
    for (int p = 0; p < PER; ++p) {
        const int k0 = 4 * (threadIdx.x + p * NT);
        const uint32_t v[4] = {acc[p].x, acc[p].y, acc[p].z, acc[p].w};
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            if (k0 + c < NOUT - 1) o[k0 + c] = v[c];
            else if (k0 + c == NOUT - 1) o[k0 + c] = v[c] + bnew;
        }
    }
}

}  // namespace

cudaError_t launch_iks(const IksArgs &a, int kind, cudaStream_t st)
{
    if (a.B <= 0) return cudaSuccess;
    // one 16-byte word of a padded row per thread: 169 of 192 (lvl0 rows),
    // 257 of 288 (lvl1 rows)
    if (kind == 10)
        iks_kernel<192, false, N1, KS10_BASEBIT, KS10_T, N0 + 1><<<a.B, 192, 0, st>>>(a);
    else if (kind == 20)
        iks_kernel<192, true, N2, KS20_BASEBIT, KS20_T, N0 + 1><<<a.B, 192, 0, st>>>(a);
    else if (kind == 21)
        iks_kernel<288, true, N2, KS21_BASEBIT, KS21_T, N1 + 1><<<a.B, 288, 0, st>>>(a);
    else
        return cudaErrorInvalidValue;
    return cudaGetLastError();
}

}  // namespace cfdb
