"""Launch-shape choice of the persistent PBS kernels (choose_shape in
csrc/pbs_common.cuh), checked without a GPU.

A kernel runs in one of three shapes, w ciphertexts per CTA (lvl01: 7, 8, 4;
lvl02: 3, 2, 1).  Each CTA works through ceil(ceil(B / w) / SMs) passes of w
ciphertexts; the autotuner measures one full pass of each shape, and a launch
picks the shape with the least passes x pass time, ties to the earlier shape
in the list.  The header functions are compiled for the host with nvcc and
their choices compared with that rule for every batch up to 20,000 and with
hand-worked cases on 148 SMs.
"""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "cufhedb_b200", "csrc")
SMS = 148
SHAPES = {1: (7, 8, 4), 2: (3, 2, 1)}
# pass times (ms) per shape, in list order: the context's untuned default,
# figures of the order measured on B200, and a case where the wide shape wins
PASS = {
    1: {"untuned": (1.0, 1.0, 1.0), "split": (9.40, 10.50, 6.0), "fp64": (14.28, 14.54, 9.0),
        "w8_faster": (10.0, 9.0, 9.5)},
    2: {"untuned": (1.0, 1.0, 1.0), "f64": (17.7, 13.5, 8.0)},
}
BMAX = 20000

PROG = r"""
#include "pbs_common.cuh"
#include <cstdio>
#include <cstdlib>
int main(int argc, char **argv)
{
    const int level = atoi(argv[1]);
    const float pass_ms[3] = {(float)atof(argv[2]), (float)atof(argv[3]), (float)atof(argv[4])};
    for (int B = 1; B <= %d; ++B)
        std::printf("%%d\n", level == 1 ? cfdb::pbs01_choose_w(B, %d, pass_ms) : cfdb::pbs02_choose_p(B, %d, pass_ms));
    return 0;
}
""" % (BMAX, SMS, SMS)


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
    for level, cases in PASS.items():
        for name, t in cases.items():
            res = subprocess.run([str(exe), str(level), *map(repr, t)], capture_output=True, text=True, timeout=60)
            out[level, name] = [int(x) for x in res.stdout.split()]
            assert len(out[level, name]) == BMAX
    return out


def _rule(B, shapes, t):
    costs = [-(-(-(-B // w)) // SMS) * p for w, p in zip(shapes, t)]   # passes x pass time
    return shapes[costs.index(min(costs))]                             # first minimum: ties to the earlier


def test_choice_follows_the_rule_for_every_batch(choices):
    for level, cases in PASS.items():
        for name, t in cases.items():
            want = [_rule(B, SHAPES[level], t) for B in range(1, BMAX + 1)]
            got = choices[level, name]
            bad = [B for B in range(1, BMAX + 1) if got[B - 1] != want[B - 1]]
            assert not bad, (level, name, bad[:10])


def test_hand_worked_cases(choices):
    c = lambda level, name, B: choices[level, name][B - 1]
    # untuned: the fewest passes, ties to the first shape
    assert all(c(1, "untuned", B) == 7 for B in range(1, 7 * SMS + 1))
    assert c(1, "untuned", 7 * SMS + 1) == 8                # 2 passes of 7 or 1 of 8
    assert all(c(2, "untuned", B) == 3 for B in (1, 100, 444, 10000))
    # lvl01 split, measured
    assert c(1, "split", 1) == 4                            # one pass either way: the shortest
    assert c(1, "split", 4 * SMS) == 4                      # 592: one pass of 4
    assert c(1, "split", 4 * SMS + 1) == 7                  # 2 x 6.0 = 12.0 vs one pass of 7
    assert c(1, "split", 1024) == 7                         # 147 CTAs of 7: one pass
    assert c(1, "split", 7 * SMS + 1) == 8                  # 1,037: two passes of 7 or one of 8
    assert c(1, "split", 8 * SMS) == 8                      # 1,184
    assert c(1, "split", 4736) == 8                         # 5 passes of 7 (47.0) vs 4 of 8 (42.0)
    assert c(1, "split", 16384) == 8                        # 16 x 9.40 = 150.4 vs 14 x 10.50 = 147.0
    assert c(1, "fp64", 16384) == 8                         # 16 x 14.28 = 228.5 vs 14 x 14.54 = 203.6
    assert c(1, "w8_faster", 1024) == 8                     # a faster 8-per-CTA pass wins at equal passes
    # lvl02, measured
    assert c(2, "f64", 48) == 1                             # 48 CTAs of 1: the shortest pass
    assert c(2, "f64", SMS + 1) == 2                        # 2 x 8.0 = 16.0 vs one pass of 2 (13.5)
    assert c(2, "f64", 2 * SMS + 1) == 3                    # 297: one pass of 3 (17.7) vs 2 of 2 (27.0)
    assert c(2, "f64", 16384) == 3                          # 37 x 17.7 = 654.9 vs 56 x 13.5 = 756.0


SPLIT_PROG = r"""
#include "pbs_common.cuh"
#include <cstdio>
#include <cstdlib>
int main(int argc, char **argv)
{
    float cc[3], tc[3];
    for (int i = 0; i < 3; ++i) cc[i] = (float)atof(argv[1 + i]), tc[i] = (float)atof(argv[4 + i]);
    for (int B = 1; B <= %d; ++B) {
        const cfdb::SplitLaunch c = cfdb::pbs01_split_choose(B, %d, cc, tc);
        std::printf("%%d %%d\n", c.w, c.tc ? 1 : 0);
    }
    return 0;
}
""" % (BMAX, SMS)


def _split_rule(B, cc, tc):
    """the split launch: least passes x pass time over the CUDA-core table,
    then the tensor-core one (only when both are measured); ties to the
    CUDA-core layout and the earlier shape"""
    measured = lambda t: any(x != 1.0 for x in t)
    cost = lambda i, t: -(-(-(-B // SHAPES[1][i])) // SMS) * t[i]
    best, best_cost = (SHAPES[1][0], 0), cost(0, cc)
    for i in range(1, 3):
        if cost(i, cc) < best_cost:
            best, best_cost = (SHAPES[1][i], 0), cost(i, cc)
    if measured(cc) and measured(tc):
        for i in range(3):
            if cost(i, tc) < best_cost:
                best, best_cost = (SHAPES[1][i], 1), cost(i, tc)
    return best


@pytest.mark.parametrize("cc, tc", [
    ((9.40, 10.30, 7.50), (13.06, 13.12, 9.93)),   # as measured on B200: the CUDA cores everywhere
    ((9.40, 10.30, 7.50), (1.0, 1.0, 1.0)),        # tensor-core table unmeasured: never chosen
    ((9.40, 10.30, 7.50), (9.0, 10.30, 7.50)),     # tensor cores faster at 7 per CTA only
    ((1.0, 1.0, 1.0), (0.5, 0.5, 0.5)),            # CUDA-core table unmeasured: CUDA cores
])
def test_split_layout_choice_matches_rule(tmp_path, cc, tc):
    nvcc = _nvcc()
    if nvcc is None:
        pytest.skip("nvcc not available")
    src, exe = tmp_path / "split.cu", tmp_path / "split"
    src.write_text(SPLIT_PROG)
    subprocess.run([nvcc, "-std=c++17", "-I", CSRC, "-o", str(exe), str(src)], check=True, capture_output=True)
    out = subprocess.run([str(exe), *map(str, cc), *map(str, tc)], check=True, capture_output=True,
                         text=True).stdout.split("\n")
    got = [tuple(int(x) for x in line.split()) for line in out if line]
    assert len(got) == BMAX
    for B in range(1, BMAX + 1):
        assert got[B - 1] == _split_rule(B, [float(x) for x in cc], [float(x) for x in tc]), B
