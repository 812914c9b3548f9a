"""GPU: the launch-shape autotuner and its persisted table.

Every shape of both persistent PBS kernels (lvl01: 7, 8, 4 ciphertexts per
CTA on both precisions; lvl02: 3, 2, 1) is forced in turn through a table
file whose pass times make that shape the cheapest, and a ragged multi-pass
batch through it must decrypt to the right bits; the measured table survives
a save / load round trip into a new context, and a table made for another
device or parameter set is refused.
"""
from __future__ import annotations

import numpy as np
import pytest

from conftest import SEED

pytestmark = pytest.mark.gpu
N0, N1, N2 = 672, 1024, 2048
MU1, MU2 = 1 << 29, 1 << 61


@pytest.fixture(scope="module")
def eng2():
    from cufhedb_b200 import GEN_BK01, GEN_BK02, GEN_KSK10, Engine
    eng = Engine(0)
    eng.keygen(SEED, GEN_BK01 | GEN_BK02 | GEN_KSK10)
    yield eng
    eng.close()


def _force(eng, tmp_path, level, precision, shape):
    """load a table in which `shape` has the only short pass for this level"""
    from cufhedb_b200 import FP64, SPLIT32, SPLIT32_TC
    path = str(tmp_path / "real.tbl")
    eng.autotune_save(path)
    lines = open(path).read().splitlines()
    key = {1: {FP64: "pbs01 fp64 ", SPLIT32: "pbs01 split32 ", SPLIT32_TC: "pbs01 split32tc "},
           2: {FP64: "pbs02 fp64 "}}[level][precision]
    for i, ln in enumerate(lines):
        if ln.startswith(key):
            f = ln.split()
            for j in range(2, len(f), 2):
                f[j + 1] = "0.001" if int(f[j]) == shape else "1000.0"
            lines[i] = " ".join(f)
    forced = str(tmp_path / f"forced_{level}_{precision}_{shape}.tbl")
    open(forced, "w").write("\n".join(lines) + "\n")
    assert eng.autotune_load(forced)
    return path


@pytest.mark.parametrize("precision", ["split32", "fp64", "split32tc"])
@pytest.mark.parametrize("shape", [7, 8, 4])
def test_every_lvl01_shape_bootstraps_correctly(eng2, tmp_path, precision, shape):
    import torch
    from cufhedb_b200 import FP64, SPLIT32, SPLIT32_TC
    prec = {"split32": SPLIT32, "fp64": FP64, "split32tc": SPLIT32_TC}[precision]
    real = _force(eng2, tmp_path, 1, prec, shape)
    try:
        B = 2 * shape * eng2.num_sms + 5          # two full passes and a ragged third
        assert eng2.launch_shape(1, prec, B) == shape
        bits = torch.randint(0, 2, (2, B), generator=torch.Generator().manual_seed(shape))
        msg = torch.where(bits == 1, MU1, -MU1).to(torch.int32).cuda()
        ca = torch.empty(B * (N1 + 1), dtype=torch.int32, device="cuda")
        cb = torch.empty_like(ca)
        eng2.encrypt_lvl1(SEED, 0xC1, 0, msg[0].contiguous(), ca)
        eng2.encrypt_lvl1(SEED, 0xC1, B, msg[1].contiguous(), cb)
        out = torch.empty_like(ca)
        eng2.gate_lvl1("NAND", ca, cb, out, prec)
        ph = torch.empty(B, dtype=torch.int32, device="cuda")
        eng2.phase_lvl1(out, ph)
        eng2.sync()
        got = (ph > 0).cpu().numpy().astype(int)
        assert np.array_equal(got, 1 - (bits[0] & bits[1]).numpy().astype(int))
    finally:
        assert eng2.autotune_load(real)


def test_split_launch_picks_the_stage1_layout_from_the_tables(eng2, tmp_path):
    """CUFHEDB_SPLIT32 launches take the tensor-core stage 1 only when its
    measured pass time is the shortest: with this GPU's measured tables the
    CUDA-core layout (as on B200), with a table in which the tensor-core
    7-per-CTA pass is the only short one the tensor-core layout, and the
    gates decrypt either way."""
    import torch
    from cufhedb_b200 import SPLIT32, SPLIT32_TC
    B = 1000
    eng2.autotune()
    measured = eng2.autotune_table(1, SPLIT32)
    measured_tc = eng2.autotune_table(1, SPLIT32_TC)
    cc_best = min(-(-(-(-B // w)) // eng2.num_sms) * t for w, t in measured.items())
    tc_best = min(-(-(-(-B // w)) // eng2.num_sms) * t for w, t in measured_tc.items())
    assert eng2.launch_layout(B) == ("tensor-core" if tc_best < cc_best else "cuda-core")
    real = _force(eng2, tmp_path, 1, SPLIT32_TC, 7)
    try:
        assert eng2.launch_layout(B) == "tensor-core"
        assert eng2.launch_shape(1, SPLIT32, B) == 7
        bits = torch.randint(0, 2, (2, B), generator=torch.Generator().manual_seed(77))
        msg = torch.where(bits == 1, MU1, -MU1).to(torch.int32).cuda()
        ca = torch.empty(B * (N1 + 1), dtype=torch.int32, device="cuda")
        cb = torch.empty_like(ca)
        eng2.encrypt_lvl1(SEED, 0xC7, 0, msg[0].contiguous(), ca)
        eng2.encrypt_lvl1(SEED, 0xC7, B, msg[1].contiguous(), cb)
        out = torch.empty_like(ca)
        eng2.gate_lvl1("NAND", ca, cb, out, SPLIT32)
        ph = torch.empty(B, dtype=torch.int32, device="cuda")
        eng2.phase_lvl1(out, ph)
        eng2.sync()
        got = (ph > 0).cpu().numpy().astype(int)
        assert np.array_equal(got, 1 - (bits[0] & bits[1]).numpy().astype(int))
    finally:
        assert eng2.autotune_load(real)


@pytest.mark.parametrize("shape", [3, 2, 1])
def test_every_lvl02_shape_bootstraps_correctly(eng2, oracle, keys, tmp_path, shape):
    import torch
    from cufhedb_b200 import FP64, testvec_const
    from oracle.oracle import NS_LVL0
    real = _force(eng2, tmp_path, 2, FP64, shape)
    try:
        s0, _, s2 = keys
        B = shape * eng2.num_sms + 3 if shape > 1 else 2 * eng2.num_sms + 1
        assert eng2.launch_shape(2, FP64, B) == shape
        bits = np.random.default_rng(shape).integers(0, 2, B)
        x = np.stack([oracle.tlwe32(MU1 if b else (-MU1) & 0xFFFFFFFF, s0, NS_LVL0, SEED, 0xC2, i)
                      for i, b in enumerate(bits)])
        out = torch.empty(B * (N2 + 1), dtype=torch.int64, device="cuda")
        eng2.pbs_lvl02(torch.from_numpy(x.view(np.int32).copy()).cuda(), out, testvec_const(MU2))
        ph = torch.empty(B, dtype=torch.int64, device="cuda")
        eng2.phase_lvl2(out, ph)
        eng2.sync()
        got = (ph > 0).cpu().numpy().astype(int)
        assert np.array_equal(got, bits)
    finally:
        assert eng2.autotune_load(real)


def test_table_persists_and_is_refused_elsewhere(eng2, tmp_path):
    from cufhedb_b200 import Engine, FP64, GEN_BK01, SPLIT32
    path = str(tmp_path / "tuned.tbl")
    t = eng2.autotune(path)
    assert not t["loaded"]
    for name in ("pbs01_fp64", "pbs01_split32", "pbs01_split32tc", "pbs02"):
        assert all(ms > 0 for ms in t[name].values()), t
    fresh = Engine(0)
    fresh.keygen(SEED, GEN_BK01)
    again = fresh.autotune(path)
    assert again["loaded"] and again == {**t, "loaded": True}
    for B in (1, 48, 1024, 5000):
        for prec in (FP64, SPLIT32):
            assert fresh.launch_shape(1, prec, B) == eng2.launch_shape(1, prec, B)
    lines = open(path).read().splitlines()
    f = lines[1].split()
    f[-1] = f[-1][:-1] + ("0" if f[-1][-1] != "0" else "1")   # another parameter set's hash
    lines[1] = " ".join(f)
    other = str(tmp_path / "other.tbl")
    open(other, "w").write("\n".join(lines) + "\n")
    assert not fresh.autotune_load(other)
    fresh.close()
