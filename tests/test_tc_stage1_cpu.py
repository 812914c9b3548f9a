"""The tensor-core stage 1 of the split-precision lvl01 transform
(csrc/tc_stage1.cuh), checked without a GPU.

Per digit polynomial and lane, the CUDA-core forward transform starts with the
per-register twist (cw64) and a 16-point DFT (fdft16<1>, fft_f32.cuh); the
tensor-core path replaces both with one product of the lane's 32 real inputs
(16 real then 16 imaginary parts) by a constant 32 x 32 real matrix B, split
into two FP16 limbs.  Here the header's B builder is compiled for the host and
its limbs are checked: (1) a line-by-line port of the CUDA-core steps (the
butterflies and twiddles of fdft4 / fw16 / fdft16 and the cw64 constants)
equals the matrix formula in float64; (2) the limbs sum to B within 2^-23 and
sit in the canonical K-major layout the MMA reads; (3) random exact digits
times the limbs, accumulated in FP32, match the float64 stage to FP32
accuracy.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "cufhedb_b200", "csrc")

PROG = r"""
#include "tc_stage1.cuh"
#include <cstdio>
int main()
{
    static uint16_t hi[cfdb::TC_B_HALVES], lo[cfdb::TC_B_HALVES];
    cfdb::build_stage1_b(hi, lo);
    for (int n = 0; n < 32; ++n)
        for (int k = 0; k < 32; ++k)
            std::printf("%d %d %d %u %u\n", n, k, cfdb::tc_b_index(n, k), hi[cfdb::tc_b_index(n, k)],
                        lo[cfdb::tc_b_index(n, k)]);
    std::printf("idesc %u\n", cfdb::TC_IDESC);
    return 0;
}
"""


def _nvcc():
    for c in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and os.path.exists(c):
            return c
    return None


@pytest.fixture(scope="module")
def limbs(tmp_path_factory):
    nvcc = _nvcc()
    if nvcc is None:
        pytest.skip("nvcc not available")
    d = tmp_path_factory.mktemp("tc")
    src, exe = d / "tc.cu", d / "tc"
    src.write_text(PROG)
    r = subprocess.run([nvcc, "-std=c++17", "-I", CSRC, "-I", os.path.join(ROOT, "include"), "-o", str(exe),
                        str(src)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60).stdout.splitlines()
    hi = np.zeros((32, 32), np.float64)
    lo = np.zeros((32, 32), np.float64)
    idx = np.zeros((32, 32), np.int64)
    for ln in out[:-1]:
        n, k, i, h, l = map(int, ln.split())
        hi[k, n] = np.array([h], np.uint16).view(np.float16)[0]
        lo[k, n] = np.array([l], np.uint16).view(np.float16)[0]
        idx[n, k] = i
    return hi, lo, idx, int(out[-1].split()[1])


def _fdft4(a0, a1, a2, a3):
    s02, d02, s13, d13 = a0 + a2, a0 - a2, a1 + a3, a1 - a3
    t = 1j * d13                      # fdft4<1>: t = (-d13.y, d13.x)
    return s02 + s13, d02 + t, s02 - s13, d02 - t


def _stage_cuda_cores(x):
    """cw64 then fdft16<1> as fft_f32.cuh writes them, in float64"""
    v = [x[m2] * np.exp(2j * np.pi * m2 / 64) for m2 in range(16)]
    for n1 in range(4):
        v[n1], v[n1 + 4], v[n1 + 8], v[n1 + 12] = _fdft4(v[n1], v[n1 + 4], v[n1 + 8], v[n1 + 12])
    for pos, e in ((5, 1), (6, 2), (7, 3), (9, 2), (10, 4), (11, 6), (13, 3), (14, 6), (15, 9)):
        v[pos] = v[pos] * np.exp(2j * np.pi * e / 16)
    for k2 in range(4):
        v[4 * k2], v[4 * k2 + 1], v[4 * k2 + 2], v[4 * k2 + 3] = _fdft4(*v[4 * k2:4 * k2 + 4])
    t = [0j] * 16
    for k2 in range(4):
        for k1 in range(4):
            t[k2 + 4 * k1] = v[4 * k2 + k1]
    return np.array(t)


def _b_exact():
    b = np.zeros((32, 32))
    for m in range(16):
        for q in range(16):
            w = np.exp(2j * np.pi * m * (1 + 4 * q) / 64)
            b[m, q], b[m, 16 + q], b[16 + m, q], b[16 + m, 16 + q] = w.real, w.imag, -w.imag, w.real
    return b


def test_matrix_equals_the_cuda_core_stage():
    rng = np.random.default_rng(1)
    b = _b_exact()
    for _ in range(20):
        x = rng.integers(-32, 32, 16) + 1j * rng.integers(-32, 32, 16)
        want = _stage_cuda_cores(x)
        got = np.concatenate([x.real, x.imag]) @ b
        assert np.max(np.abs(got[:16] + 1j * got[16:] - want)) < 1e-9


def test_limbs_and_layout(limbs):
    hi, lo, idx, idesc = limbs
    assert np.max(np.abs(hi + lo - _b_exact())) <= 2.0 ** -23
    # canonical K-major, no swizzle: (n, k) -> (n/8)*256 + (k/8)*64 + (n%8)*8 + k%8 halves
    n, k = np.meshgrid(np.arange(32), np.arange(32), indexing="ij")
    assert np.array_equal(idx, (n // 8) * 256 + (k // 8) * 64 + (n % 8) * 8 + (k % 8))
    assert sorted(idx.ravel()) == list(range(1024))
    # D F32 (bit 4), A / B FP16 and K-major (0), N = 32 (4 << 17), M = 128 (8 << 24)
    assert idesc == (1 << 4) | (4 << 17) | (8 << 24)


def test_exact_digits_times_limbs_in_fp32(limbs):
    hi, lo, _, _ = limbs
    rng = np.random.default_rng(2)
    b = _b_exact()
    a = rng.integers(-32, 32, (256, 32)).astype(np.float32)
    acc = np.zeros((256, 32), np.float32)
    for limb in (hi, lo):
        for kk in range(32):                    # FP32 accumulation, product by product
            acc = (acc + a[:, kk:kk + 1] * limb[kk].astype(np.float32)).astype(np.float32)
    want = a.astype(np.float64) @ b
    err = np.abs(acc.astype(np.float64) - want)
    scale = np.abs(a).sum(axis=1, keepdims=True)
    assert np.max(err / scale) < 2.0 ** -21
