"""The lvl2 transform's frequency layout (csrc/fft8x.cuh), checked without a GPU.

fft8x_freq<128>(u, s) names the frequency that register slot s of thread u
holds after the forward transform; the bootstrapping key is stored in that
[s][u] order and reference-format keys are permuted by it
(bk_permute2_kernel), so it is a contract between the transform and the key
layout.  The header function is compiled for the host with nvcc and its
table compared with a numpy model of the transform's factorisation
M = 8 x 8 x 16 (stage A: 8-point DFT over j, twiddle w^t W_M^{tk}; stage B:
transpose, 8-point DFT over b, twiddle W_T^{a q1}; stage C: in-warp
transpose to a = a0 + 2 j, 8-point DFT over j, one radix-2 step between the
lanes u and u ^ 8), which is itself checked against a direct DFT.  The GPU
tests (test_gpu_lvl2.py) check the kernels' numbers; this pins the layout.
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
#include <cstdio>
int main()
{
    for (int u = 0; u < 128; ++u)
        for (int s = 0; s < 8; ++s) std::printf("%d\n", cfdb::fft8x_freq<128>(u, s));
    return 0;
}
"""


def _nvcc():
    for c in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and os.path.exists(c):
            return c
    return None


@pytest.fixture(scope="module")
def freq_table(tmp_path_factory):
    nvcc = _nvcc()
    if nvcc is None:
        pytest.skip("nvcc not available")
    d = tmp_path_factory.mktemp("fft8x")
    src, exe = d / "freq.cu", d / "freq"
    src.write_text(PROG)
    r = subprocess.run([nvcc, "-std=c++17", "-I", CSRC, "-o", str(exe), str(src)], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60).stdout.split()
    return np.array([int(x) for x in out]).reshape(T, 8)


def _dft8(x, sign):
    """x[..., n] -> X[..., k] = sum_n x[n] exp(sign 2 pi i n k / 8)."""
    n = np.arange(8)
    return x @ np.exp(sign * 2j * np.pi * np.outer(n, n) / 8)


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


def test_frequency_map_is_a_permutation(freq_table):
    assert sorted(freq_table.ravel().tolist()) == list(range(M))


def test_factorisation_lands_each_frequency_where_the_map_says(freq_table):
    rng = np.random.default_rng(7)
    z = rng.normal(size=M) + 1j * rng.normal(size=M)
    v = _forward_model(z)
    m = np.arange(M)
    direct = np.exp(2j * np.pi * np.outer(np.arange(M), m) / M) @ z
    err = np.max(np.abs(v - direct[freq_table]))
    assert err <= 1e-11 * np.max(np.abs(direct))
