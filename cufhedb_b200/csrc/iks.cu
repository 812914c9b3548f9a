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

// ---- key-stationary lvl2 -> lvl1 switch (large batches) ------------------------
// The gather above reads each selected 4,100-byte key row once per ciphertext:
// 75 GB per 1,024 ciphertexts, served from L2 (the 0.59 GB key stays there).
// Turned around, each CTA owns 8 output words of 256 ciphertexts and walks
// the whole key once, staging those 8 words of every key row in shared
// memory (2.4 GB of L2 reads per 1,024 ciphertexts), and each thread, one
// ciphertext, subtracts the staged words of the rows its digits select.  The
// subtractions are the gather's, in the same order per word (ascending i,
// j), so the results are identical.  Eight words per CTA (129 word blocks)
// give 28 warps per SM at 1,024 ciphertexts; the staged rows are padded to
// 48 bytes, so the eight digit values of a quarter-warp's 16-byte reads fall
// in eight distinct bank groups.
constexpr int KS_TILE = 256;                          // ciphertexts per CTA, one per thread
constexpr int KS_WB = 8;                              // output words per CTA
constexpr int KS_NB = (N1 + 1 + KS_WB - 1) / KS_WB;   // word blocks: 129
constexpr int KS_IC = 2;                              // input coefficients per staged chunk
constexpr int KS_DIG = 1 << KS21_BASEBIT;             // digit values 0..7 (row 0: zeros)
constexpr int KS_ROWS = KS_IC * KS21_T * KS_DIG;      // staged rows per chunk: 160
constexpr int KS_RW4 = 3;                             // uint4 per staged row: 8 words + 4 pad
constexpr int KS_P4 = ksk_pitch(N1 + 1) / 4;          // uint4 per key row in HBM: 257
constexpr int KS_LOADS = KS_IC * KS21_T * (KS_DIG - 1) * (KS_WB / 4);   // uint4 per chunk: 280
constexpr int KS_PER = (KS_LOADS + KS_TILE - 1) / KS_TILE;              // per thread: 2
constexpr uint64_t KS_PREC = 1ull << (64 - (1 + KS21_BASEBIT * KS21_T));
constexpr int KS_SHIFT = 64 - KS21_BASEBIT * KS21_T;                    // the digits' 30 bits

// X[i][b] = the top 30 bits of a_i + prec_offset (ciphertext b's ten digits
// of coefficient i), 0 for the padding b >= B
__global__ void ks21_prep_kernel(const uint64_t *__restrict__ in, uint32_t *X, int B, int Bp)
{
    const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (size_t)N2 * Bp) return;
    const int i = (int)(idx / Bp), b = (int)(idx % Bp);
    X[idx] = b < B ? (uint32_t)((in[(size_t)b * (N2 + 1) + i] + KS_PREC) >> KS_SHIFT) : 0u;
}

__global__ void __launch_bounds__(KS_TILE, 4) ks21_kernel(const uint32_t *__restrict__ X, int Bp,
                                                       const uint4 *__restrict__ ksk, const uint64_t *in,
                                                       uint32_t *out, int B, uint64_t offset64)
{
    __shared__ uint4 stage[2][KS_ROWS * KS_RW4];
    const int t = threadIdx.x, s = blockIdx.x, ct = blockIdx.y * KS_TILE + t;
    // digit-0 rows are zero in both buffers (never written again)
    for (int e = t; e < 2 * KS_IC * KS21_T * KS_RW4; e += KS_TILE) {
        const int buf = e / (KS_IC * KS21_T * KS_RW4), rem = e % (KS_IC * KS21_T * KS_RW4);
        stage[buf][(rem / KS_RW4) * KS_DIG * KS_RW4 + rem % KS_RW4] = make_uint4(0u, 0u, 0u, 0u);
    }
    // this thread's share of chunk c: key row (i, j, d) words 16 s + 4 q .. + 3,
    // where they exist (the last word block holds only the padded row's word
    // 1024 and its pad: q = 0)
    uint4 r[KS_PER];
    auto load = [&](int c) {
#pragma unroll
        for (int k = 0; k < KS_PER; ++k) {
            const int e = t + k * KS_TILE;
            r[k] = make_uint4(0u, 0u, 0u, 0u);
            if (e < KS_LOADS) {
                const int q = e % (KS_WB / 4), row = e / (KS_WB / 4);   // row = (ii T + j) (2^b - 1) + d - 1
                const int w4 = (KS_WB / 4) * s + q;
                if (w4 < KS_P4) {
                    const size_t g = (size_t)c * KS_IC * KS21_T * (KS_DIG - 1) + row;
                    r[k] = __ldg(ksk + g * KS_P4 + w4);
                }
            }
        }
    };
    auto store = [&](int buf) {
#pragma unroll
        for (int k = 0; k < KS_PER; ++k) {
            const int e = t + k * KS_TILE;
            if (e < KS_LOADS) {
                const int q = e % (KS_WB / 4), row = e / (KS_WB / 4), ij = row / (KS_DIG - 1),
                          d = row % (KS_DIG - 1) + 1;
                stage[buf][(ij * KS_DIG + d) * KS_RW4 + q] = r[k];
            }
        }
    };
    uint32_t acc[KS_WB];
#pragma unroll
    for (int k = 0; k < KS_WB; ++k) acc[k] = 0u;
    constexpr int NCHUNK = N2 / KS_IC;
    load(0);
    store(0);
    __syncthreads();
#pragma unroll 1
    for (int c = 0; c < NCHUNK; ++c) {
        if (c + 1 < NCHUNK) load(c + 1);
        const uint4 *buf = stage[c & 1];
#pragma unroll
        for (int ii = 0; ii < KS_IC; ++ii) {
            const uint32_t x = X[(size_t)(c * KS_IC + ii) * Bp + (size_t)blockIdx.y * KS_TILE + t];
#pragma unroll
            for (int j = 0; j < KS21_T; ++j) {
                const uint32_t d = (x >> (KS21_BASEBIT * (KS21_T - 1 - j))) & (KS_DIG - 1);
                const uint4 *row = buf + ((ii * KS21_T + j) * KS_DIG + d) * KS_RW4;
#pragma unroll
                for (int q = 0; q < KS_WB / 4; ++q) {
                    const uint4 v = row[q];
                    acc[4 * q] -= v.x;
                    acc[4 * q + 1] -= v.y;
                    acc[4 * q + 2] -= v.z;
                    acc[4 * q + 3] -= v.w;
                }
            }
        }
        if (c + 1 < NCHUNK) store((c + 1) & 1);
        __syncthreads();
    }
    if (ct >= B) return;
    const uint32_t bnew = (uint32_t)((in[(size_t)ct * (N2 + 1) + N2] + offset64 + (1ull << 31)) >> 32);
    uint32_t *o = out + (size_t)ct * (N1 + 1);
#pragma unroll
    for (int k = 0; k < KS_WB; ++k) {
        const int w = KS_WB * s + k;
        if (w < N1) o[w] = acc[k];
        else if (w == N1) o[w] = acc[k] + bnew;
    }
}

// batches from this size on take the key-stationary lvl2 -> lvl1 switch
constexpr int KS21_MIN_BATCH = 512;

}  // namespace

cudaError_t launch_iks(const IksArgs &a, int kind, cudaStream_t st)
{
    if (a.B <= 0) return cudaSuccess;
    if (kind == 21 && a.B >= KS21_MIN_BATCH) {
        const int tiles = (a.B + KS_TILE - 1) / KS_TILE, Bp = tiles * KS_TILE;
        uint32_t *X = nullptr;
        cudaError_t e = cudaMallocAsync((void **)&X, (size_t)N2 * Bp * sizeof(uint32_t), st);
        if (e != cudaSuccess) return e;
        const size_t n = (size_t)N2 * Bp;
        ks21_prep_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(a.in64, X, a.B, Bp);
        e = cudaGetLastError();
        if (e == cudaSuccess) {
            ks21_kernel<<<dim3(KS_NB, tiles), KS_TILE, 0, st>>>(X, Bp, reinterpret_cast<const uint4 *>(a.ksk),
                                                                 a.in64, a.out, a.B, a.offset64);
            e = cudaGetLastError();
        }
        const cudaError_t ef = cudaFreeAsync(X, st);
        return e != cudaSuccess ? e : ef;
    }
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
