"""The transforms' frequency layouts, checked without a GPU.

After a forward transform each thread holds a fixed set of frequencies in its
register slots; the bootstrapping keys are stored in that [slot][thread]
order, and reference-format keys are permuted by the same maps
(keys.cu / fftops.cu for lvl1, bk_permute2_kernel for lvl2), so each map is a
contract between a transform and its key layout.  The header functions
fft512_freq (csrc/fft_f64.cuh, lvl1: 512 points, one warp, 16 values per
lane; the FP64 and split kernels share it) and fft8x_freq<128>
(csrc/fft8x.cuh, lvl2: 1024 points, four warps, 8 values per thread) are
compiled for the host with nvcc, and their tables compared with numpy models
of the factorisations, which are themselves checked against a direct DFT:
  lvl1  512 = 16 x 32: 16-point DFT over m2 in registers, twiddle W^{m1 q2},
        transpose, 16-point DFT over m1 = h + 2 m1', one radix-2 step between
        the lanes L and L ^ 16;
  lvl2  1024 = 8 x 8 x 16: 8-point DFT over j, twiddle w^t W_M^{tk};
        transpose, 8-point DFT over b, twiddle W_T^{a q1}; in-warp transpose
        to a = a0 + 2 j, 8-point DFT over j, one radix-2 step between the
        lanes u and u ^ 8.
The GPU tests (test_gpu_lvl1.py, test_gpu_lvl2.py) check the kernels'
numbers; this pins the layouts.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "cufhedb_b200", "csrc")
T, M, L = 128, 1024, 16

PROG = r"""
#include "fft8x.cuh"
#include "fft_f64.cuh"
#include <cstdio>
int main()
{
    for (int u = 0; u < 128; ++u)
        for (int s = 0; s < 8; ++s) std::printf("%d\n", cfdb::fft8x_freq<128>(u, s));
    for (int lane = 0; lane < 32; ++lane)
        for (int s = 0; s < 16; ++s) std::printf("%d\n", cfdb::fft512_freq(lane, s));
    return 0;
}
"""


def _nvcc():
    for c in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and os.path.exists(c):
            return c
    return None


@pytest.fixture(scope="module")
def freq_tables(tmp_path_factory):
    nvcc = _nvcc()
    if nvcc is None:
        pytest.skip("nvcc not available")
    d = tmp_path_factory.mktemp("fft8x")
    src, exe = d / "freq.cu", d / "freq"
    src.write_text(PROG)
    r = subprocess.run([nvcc, "-std=c++17", "-I", CSRC, "-o", str(exe), str(src)], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    out = np.array([int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True,
                                                    timeout=60).stdout.split()])
    return {"lvl2": out[:T * 8].reshape(T, 8), "lvl1": out[T * 8:].reshape(32, 16)}


@pytest.fixture(scope="module")
def freq_table(freq_tables):
    return freq_tables["lvl2"]


def _dft8(x, sign):
    """x[..., n] -> X[..., k] = sum_n x[n] exp(sign 2 pi i n k / 8)."""
    n = np.arange(8)
    return x @ np.exp(sign * 2j * np.pi * np.outer(n, n) / 8)


def _dft16(x, sign):
    n = np.arange(16)
    return x @ np.exp(sign * 2j * np.pi * np.outer(n, n) / 16)


def _forward_model_512(z):
    """The lvl1 factorised forward transform: V[lane, s] for input z[m], m < 512."""
    lanes = np.arange(32)
    w = lambda num, den: np.exp(2j * np.pi * num / den)
    # lane m1 holds z_{m1 + 32 m2}: 16-point DFT over m2 (output q2), twiddle W^{m1 q2}
    v1 = _dft16(np.stack([z[lanes + 32 * m2] for m2 in range(16)], axis=1), 1)
    v1 = v1 * w(np.outer(lanes, np.arange(16)) % 512, 512)
    # lane (q2 = L & 15, h = L >> 4) gets m1' -> v1[2 m1' + h, q2]; 16-point DFT over m1'
    h, q2 = lanes >> 4, lanes & 15
    y = _dft16(np.stack([v1[2 * m + h, q2] for m in range(16)], axis=1), 1)
    out = np.empty((32, 16), complex)
    partner = lanes ^ 16
    for j in range(8):
        # lane h keeps q1 = j + 8 h and j + 8 h + 16: Y0 from the h = 0 lane, Y1 from the h = 1 lane
        a = np.where(h == 1, y[partner, 8 + j], y[lanes, j])
        b = np.where(h == 1, y[lanes, 8 + j], y[partner, j])
        t = b * w(j + 8 * h, 32)
        out[:, j] = a + t
        out[:, 8 + j] = a - t
    return out


def _forward_model(z):
    """The factorised forward transform: returns V[u, s] for input z[m], m < M."""
    t = np.arange(T)
    k8 = np.arange(8)
    w = lambda num, den: np.exp(2j * np.pi * num / den)
    # stage A: thread t holds z_{t + T j} / w^t; DFT over j, twiddle w^t W_M^{t k}
    va = _dft8(np.stack([z[t + T * j] / w(t, 4 * M) for j in range(8)], axis=1), 1)
    va = va * w(np.outer(t, 1 + 4 * k8) % (4 * M), 4 * M)
    # stage B: thread u = a + L k gets b -> va[a + L b, k]; DFT over b, twiddle W_T^{a q1}
    a, k = t % L, t // L
    vb = _dft8(np.stack([va[a + L * b, k] for b in range(8)], axis=1), 1)
    vb = vb * w(np.outer(a, k8) % T, T)
    # stage C: thread u' = q1 + 8 a0 + 16 k' gets j -> vb[a0 + 2 j + L k', q1]
    q1p, a0, kp = t & 7, (t >> 3) & 1, t >> 4
    y = _dft8(np.stack([vb[a0 + 2 * j + L * kp, q1p] for j in range(8)], axis=1), 1)
    out = np.empty((T, 8), complex)
    partner = t ^ 8
    for rl in range(4):
        # thread a0 keeps r = rl + 4 a0: Y0[r] from the a0 = 0 lane, Y1[r] from the a0 = 1 lane
        p = np.where(a0 == 1, y[partner, rl + 4], y[t, rl])
        q = np.where(a0 == 1, y[t, rl + 4], y[partner, rl])
        q = q * w(2 * rl, 32) * np.where(a0 == 1, 1j, 1.0)        # W_16^r
        out[:, rl] = p + q
        out[:, rl + 4] = p - q
    return out


def test_lvl2_frequency_map_is_a_permutation(freq_table):
    assert sorted(freq_table.ravel().tolist()) == list(range(M))


def test_lvl2_factorisation_lands_each_frequency_where_the_map_says(freq_table):
    rng = np.random.default_rng(7)
    z = rng.normal(size=M) + 1j * rng.normal(size=M)
    v = _forward_model(z)
    m = np.arange(M)
    direct = np.exp(2j * np.pi * np.outer(np.arange(M), m) / M) @ z
    err = np.max(np.abs(v - direct[freq_table]))
    assert err <= 1e-11 * np.max(np.abs(direct))


def test_lvl1_frequency_map_is_a_permutation(freq_tables):
    assert sorted(freq_tables["lvl1"].ravel().tolist()) == list(range(512))


def test_lvl1_factorisation_lands_each_frequency_where_the_map_says(freq_tables):
    rng = np.random.default_rng(11)
    z = rng.normal(size=512) + 1j * rng.normal(size=512)
    v = _forward_model_512(z)
    direct = np.exp(2j * np.pi * np.outer(np.arange(512), np.arange(512)) / 512) @ z
    err = np.max(np.abs(v - direct[freq_tables["lvl1"]]))
    assert err <= 1e-11 * np.max(np.abs(direct))
