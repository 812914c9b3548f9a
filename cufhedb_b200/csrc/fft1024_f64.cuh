// FP64 negacyclic FFT for N = 2048 (1024 complex points, the lvl2 ring of the
// 64-bit torus): the fft8x transform with T = 128 threads (four warps) per
// polynomial, 8 complex values per thread (TFHEpp TwistIFFT/TwistFFT
// <lvl2param>, thirdparty/TFHEpp/include/mulfft.hpp:57-121).
#pragma once
#include "common.cuh"
#include "fft8x.cuh"

namespace cfdb {

constexpr int T2 = 128;   // threads per lvl2 polynomial
using Fft1024Tables = Fft8xTables<double2, T2>;

__host__ __device__ __forceinline__ int fft1024_freq(int t, int s) { return fft8x_freq<T2>(t, s); }

// TFHEpp's torus64 conversion (spqlios fft_processor_spqlios.cpp:180-209):
// truncation toward zero, modulo 2^64 for |x| >= 2^63.  Branch-free from the
// bit pattern x = +-mant 2^e: mant << e for e >= 0 (0 once e >= 64), mant >> -e
// (truncation) for e < 0; zero and subnormals shift out to 0.
__device__ __forceinline__ uint64_t f64_to_torus64(double x)
{
    const unsigned long long bits = (unsigned long long)__double_as_longlong(x);
    const int e = (int)((bits >> 52) & 0x7FF) - 1075;
    const unsigned long long mant = (bits & ((1ull << 52) - 1)) | (1ull << 52);
    const unsigned long long left = e >= 64 ? 0ull : mant << (e & 63);
    const unsigned long long right = mant >> (-e < 63 ? -e : 63);
    const unsigned long long mag = e >= 0 ? left : right;
    return (bits >> 63) ? 0ull - mag : mag;
}

}  // namespace cfdb
