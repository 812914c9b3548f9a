"""GPU parity against the reference's own CPU implementation on the same keys
and inputs, for every lvl01 path (FP64, split32, and split32 with the
first transform step on the tensor cores):

* GateBootstrappingTLWE2TLWEFFT<lvl01param> (TFHEpp src/gatebootstrapping.cpp:
  14-23) over whole batches that land on each lvl01 launch shape (1,024
  ciphertexts: 7 per CTA; 8 x #SMs: 8 per CTA): every output decrypts like
  TFHEpp's, and output phases agree within 2^25 (the bootstrapping noise is
  about 2^18.5; 2^25 is 1/16 of mu);
* HomNAND (TFHEpp src/gate.cpp:50-65: IKS10 + PBS01);
* GateBootstrappingTLWE2TLWEFFT<lvl02param> on a two-pass batch (phases
  within 2^56 of the 64-bit torus, mu = 2^61);
* the HEDB comparison chains greater_than / greater_than_equal / less_than /
  less_than_equal / equal (src/HEDB/comparison/HomCompare.h:14-75, MSB
  extraction src/HEDB/comparison/extract_msb.cpp) at lvl1 widths 4, 8, 9
  (ExtractMSB5 / 9 / 10; width 9 runs ExtractMSB10, whose inner call passes
  plain_bits - 4, extract_msb.cpp:55) and lvl2 widths 16, 20, 24, 32, with
  LOGIC and ARITHMETIC results: 32 rows per width and op, each row's decrypted
  result equal to the reference operator's and to plaintext.  At 31 and 32
  bits (32 / 33 plain bits, the top of the reference's range) the reference's
  own chain decides rows with |x - y| <= 1 by the sign of the accumulated
  noise (measured on its CPU operators: 1 of 48 near-equal rows wrong at 31
  bits, 8 of 48 at 32, none up to 30), so there those rows are excluded from
  the comparison and every other row must match.
"""
from __future__ import annotations

import os

import numpy as np
import pytest

from conftest import SEED, signed_diff

from oracle.oracle import N0, N1, N2, NS_LVL0, NS_LVL1, NS_LVL2

pytestmark = pytest.mark.gpu
MU = 1 << 29
THREADS = os.cpu_count() or 1
OPS = {"gt": 0, "ge": 1, "lt": 2, "le": 3, "eq": 4}
TRUTH = {"gt": lambda x, y: x > y, "ge": lambda x, y: x >= y, "lt": lambda x, y: x < y,
         "le": lambda x, y: x <= y, "eq": lambda x, y: x == y}


def _dev(a):
    import torch
    a = np.ascontiguousarray(a)
    v = a.view(np.int64) if a.dtype == np.uint64 else a.view(np.int32)
    return torch.from_numpy(v.copy()).cuda()


def _phases(oracle, cts, s1):
    s1u = s1.astype(np.uint64)
    c = np.asarray(cts).reshape(-1, N1 + 1).astype(np.uint64)
    ph = (c[:, N1] - (c[:, :N1] @ s1u)) & 0xFFFFFFFF
    return np.where(ph >= 2 ** 31, ph.astype(np.int64) - 2 ** 32, ph.astype(np.int64))


@pytest.fixture(scope="module")
def eng_all():
    from cufhedb_b200 import GEN_ALL, Engine
    eng = Engine(0)
    eng.keygen(SEED, GEN_ALL)
    yield eng
    eng.close()


PRECISIONS = ["split32", "fp64", "split32tc"]


def _prec(name):
    from cufhedb_b200 import FP64, SPLIT32, SPLIT32_TC
    return {"split32": SPLIT32, "fp64": FP64, "split32tc": SPLIT32_TC}[name]


@pytest.mark.parametrize("precision", PRECISIONS)
def test_pbs01_matches_reference_on_both_launch_shapes(engine, oracle, ref_keyed, keys, precision):
    import torch
    from cufhedb_b200 import testvec_const
    prec = _prec(precision)
    s0, s1, _ = keys
    tv = np.full(N1, MU, np.uint32)
    for B, stream_id in ((1024, 0xA1), (8 * engine.num_sms, 0xA2)):
        bits = np.random.default_rng(B).integers(0, 2, B)
        x = np.stack([oracle.tlwe32(MU if b else (-MU) & 0xFFFFFFFF, s0, NS_LVL0, SEED, stream_id, i)
                      for i, b in enumerate(bits)])
        out = torch.zeros(B * (N1 + 1), dtype=torch.int32, device="cuda")
        engine.pbs_lvl01(_dev(x), out, testvec_const(MU), prec)
        engine.sync()
        pg = _phases(oracle, out.cpu().numpy().view(np.uint32), s1)
        pr = _phases(oracle, ref_keyed.pbs01_batch(x, tv, THREADS), s1)
        assert np.array_equal((pg > 0).astype(int), bits), B
        assert np.array_equal((pr > 0).astype(int), bits), B
        d = np.abs(pg - pr)
        assert np.max(d) < 2 ** 25, (B, int(np.max(d)))


def test_pbs02_matches_reference_on_a_two_pass_batch(eng_all, oracle, ref_all, keys):
    """GateBootstrappingTLWE2TLWEFFT<lvl02param> on 3 x #SMs + 7 ciphertexts
    (one full pass of the 3-per-CTA shape and a ragged second): every output
    decrypts to its bit, and 40 sampled outputs agree with TFHEpp's on the
    same keys and inputs within 2^56 of the 64-bit torus (mu = 2^61)."""
    import torch
    from cufhedb_b200 import testvec_const
    s0, _, s2 = keys
    MU2 = 1 << 61
    B = 3 * eng_all.num_sms + 7
    bits = np.random.default_rng(0xA5).integers(0, 2, B)
    x = np.stack([oracle.tlwe32(MU if b else (-MU) & 0xFFFFFFFF, s0, NS_LVL0, SEED, 0xA5, i)
                  for i, b in enumerate(bits)])
    out = torch.zeros(B * (N2 + 1), dtype=torch.int64, device="cuda")
    eng_all.pbs_lvl02(_dev(x), out, testvec_const(MU2))
    eng_all.sync()
    got = out.cpu().numpy().view(np.uint64).reshape(B, -1)
    pg = np.array([int(signed_diff(oracle.phase64(o, s2), 0, 64)) for o in got], dtype=object)
    assert np.array_equal(np.array([int(p > 0) for p in pg]), bits)
    tv = np.full(N2, MU2, np.uint64)
    for i in np.random.default_rng(0xA6).choice(B, 40, replace=False):
        pr = int(signed_diff(oracle.phase64(ref_all.pbs02(x[i], tv), s2), 0, 64))
        assert (pr > 0) == bool(bits[i]) and abs(pr - int(pg[i])) < 2 ** 56, int(i)


@pytest.mark.parametrize("precision", PRECISIONS)
def test_homnand_matches_reference_batch(eng_all, oracle, ref_all, keys, precision):
    prec = _prec(precision)
    _, s1, _ = keys
    B = 96
    rng = np.random.default_rng(0xA3)
    a, b = rng.integers(0, 2, B), rng.integers(0, 2, B)
    enc = lambda bits, base: np.stack([oracle.tlwe32(MU if t else (-MU) & 0xFFFFFFFF, s1, NS_LVL1, SEED, 0xA3,
                                                     base + i) for i, t in enumerate(bits)])
    ca, cb = enc(a, 0), enc(b, B)
    import torch
    out = torch.zeros(B * (N1 + 1), dtype=torch.int32, device="cuda")
    eng_all.gate_lvl1("NAND", _dev(ca), _dev(cb), out, prec)
    eng_all.sync()
    pg = _phases(oracle, out.cpu().numpy().view(np.uint32), s1)
    pr = _phases(oracle, ref_all.homnand_batch(ca, cb, THREADS), s1)
    truth = 1 - (a & b)
    assert np.array_equal((pg > 0).astype(int), truth)
    assert np.array_equal((pr > 0).astype(int), truth)
    assert np.max(np.abs(pg - pr)) < 2 ** 25


def _encrypt(oracle, keys, level, vals, pb, base):
    _, s1, s2 = keys
    if level == 1:
        return np.stack([oracle.tlwe32(int(v) << (32 - pb - 1), s1, NS_LVL1, SEED, 0xA4, base + i)
                         for i, v in enumerate(vals)])
    return np.stack([oracle.tlwe64(int(v) << (64 - pb - 1), s2, NS_LVL2, SEED, 0xA5, base + i)
                     for i, v in enumerate(vals)])


def _decode(oracle, cts, s1, logic):
    ph = _phases(oracle, cts, s1)
    if logic:
        return (ph > 0).astype(int)
    # ARITHMETIC results encode 1 as 2^31 (HEDB tfhepp_utils.h:32-45 with 1 plain bit)
    u = ph & 0xFFFFFFFF
    return (((u + 2 ** 30) >> 31) & 1).astype(int)


@pytest.mark.parametrize("level,pb", [(1, 4), (1, 8), (1, 9), (2, 16), (2, 20), (2, 24), (2, 32)])
def test_compare_chains_match_reference_operators(eng_all, oracle, ref_all, keys, level, pb):
    import torch
    from cufhedb_b200 import FP64, SPLIT32
    _, s1, _ = keys
    B = 32
    rng = np.random.default_rng(1000 * level + pb)
    x = rng.integers(0, 2 ** pb, B, dtype=np.uint64)
    y = rng.integers(0, 2 ** pb, B, dtype=np.uint64)
    y[:6] = x[:6]                                        # equal values
    y[6:9] = np.minimum(x[6:9] + 1, 2 ** pb - 1)         # neighbours
    y[9:12] = np.where(x[9:12] > 0, x[9:12] - 1, 0)
    x[12], y[12] = 0, 2 ** pb - 1                        # extremes
    x[13], y[13] = 2 ** pb - 1, 0
    c1 = _encrypt(oracle, keys, level, x, pb, 0)
    c2 = _encrypt(oracle, keys, level, y, pb, B)
    d1, d2 = _dev(c1), _dev(c2)
    out = torch.zeros(B * (N1 + 1), dtype=torch.int32, device="cuda")
    gap = np.abs(x.astype(np.int64) - y.astype(np.int64))
    decided = gap >= 2 if pb >= 31 else np.ones(B, bool)
    for op, opi in OPS.items():
        truth = TRUTH[op](x, y).astype(int)
        for logic in (True, False) if op in ("ge", "lt") else (True,):
            theirs = _decode(oracle, ref_all.compare_batch(level, c1, c2, opi, pb, logic, THREADS), s1, logic)
            assert np.array_equal(theirs[decided], truth[decided]), (op, logic)
            for prec in (SPLIT32, FP64):
                out.zero_()
                eng_all.compare(op, level, d1, d2, out, pb, logic=logic, precision=prec)
                eng_all.sync()
                got = _decode(oracle, out.cpu().numpy().view(np.uint32), s1, logic)
                bad = np.nonzero(got[decided] != theirs[decided])
                assert np.array_equal(got[decided], theirs[decided]), (op, logic, prec, bad)
