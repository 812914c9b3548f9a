"""Launch-shape choice of the lvl01 PBS (pbs01_choose_w in csrc/pbs_common.cuh),
checked without a GPU.

Each CTA works through ceil(B / w / SMs) passes of w ciphertexts (w = 7 with a
producer warp, w = 8 without); the autotuner measures one pass of each shape,
and the launch picks the shape with the smaller passes x pass time, ties to
w = 7.  The header function is compiled for the host with nvcc and its
choices compared with that rule and with hand-worked cases on 148 SMs.
"""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "cufhedb_b200", "csrc")
SMS = 148
PASS = {"untuned": (0.0, 0.0), "split": (9.40, 10.50), "fp64": (14.28, 14.54), "w8_faster": (10.0, 9.0)}
BMAX = 20000

PROG = r"""
#include "pbs_common.cuh"
#include <cstdio>
int main(int argc, char **argv)
{
    const float pass_ms[2] = {(float)atof(argv[1]), (float)atof(argv[2])};
    for (int B = 1; B <= %d; ++B) std::printf("%%d\n", cfdb::pbs01_choose_w(B, %d, pass_ms));
    return 0;
}
""" % (BMAX, SMS)


def _nvcc():
    for c in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and os.path.exists(c):
            return c
    return None


@pytest.fixture(scope="module")
def choices(tmp_path_factory):
    nvcc = _nvcc()
    if nvcc is None:
        pytest.skip("nvcc not available")
    d = tmp_path_factory.mktemp("shape")
    src, exe = d / "shape.cu", d / "shape"
    src.write_text(PROG)
    r = subprocess.run([nvcc, "-std=c++17", "-I", CSRC, "-I", os.path.join(ROOT, "include"), "-o", str(exe),
                        str(src)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    out = {}
    for name, (p7, p8) in PASS.items():
        res = subprocess.run([str(exe), repr(p7), repr(p8)], capture_output=True, text=True, timeout=60)
        out[name] = [int(x) for x in res.stdout.split()]
        assert len(out[name]) == BMAX
    return out


def _rule(B, p7, p8):
    cost = lambda w, p: -(-(-(-B // w)) // SMS) * p   # ceil(ceil(B / w) / SMS) passes x pass time
    return 8 if cost(8, p8) < cost(7, p7) else 7


def test_choice_follows_the_rule_for_every_batch(choices):
    for name, (p7, p8) in PASS.items():
        want = [_rule(B, p7, p8) for B in range(1, BMAX + 1)]
        got = choices[name]
        bad = [B for B in range(1, BMAX + 1) if got[B - 1] != want[B - 1]]
        assert not bad, (name, bad[:10])


def test_hand_worked_cases(choices):
    c = lambda name, B: choices[name][B - 1]
    assert all(w == 7 for w in choices["untuned"])      # no measurement yet: ties go to 7
    assert c("split", 1) == 7                            # one pass either way: the lighter one
    assert c("split", 1024) == 7                         # 147 CTAs of 7: one pass
    assert c("split", 7 * SMS) == 7                      # 1,036: still one pass of 7
    assert c("split", 7 * SMS + 1) == 8                  # 1,037: two passes of 7 or one of 8
    assert c("split", 8 * SMS) == 8                      # 1,184
    assert c("split", 4736) == 8                         # 5 passes of 7 (47.0) vs 4 of 8 (42.0)
    assert c("split", 16384) == 8                        # 16 x 9.40 = 150.4 vs 14 x 10.50 = 147.0
    assert c("fp64", 16384) == 8                         # 16 x 14.28 = 228.5 vs 14 x 14.54 = 203.6
    assert c("w8_faster", 1024) == 8                     # a faster 8-per-CTA pass wins at equal passes
