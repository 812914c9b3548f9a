"""GPU parity: ArcEDB comparisons (cuARCEDB greater_than_tfhepp /
less_than_tfhepp / equality_tfhepp, src/cuHEDB/comparable_gpu.cuh:52-168)
over radix-1024 digits through the C ABI.  One digit: against the oracle's
exact restatement (within the rounding of the external product) and the
plaintext truth.  Several digits: against a plaintext model of the
reference's digit combination and, for a few rows, against the reference's
own TFHEpp steps run on the CPU with the same keys."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import SEED, fill_ref_ksk, signed_diff

from oracle.oracle import L1, N1

pytestmark = pytest.mark.gpu
MU = 1 << 29
DIGIT = 1024


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a).view(np.int32).copy()).cuda()


def _digit_truth(op, x, y):
    return {"gt": x > y, "lt": x <= y, "lt_strict": x < y, "eq": x == y}[op]


def model(op, xd, yd):
    """The reference's combination (comparable_gpu.cuh:65-97, 137-168) on
    plaintext digits: order comparisons bootstrap eq + 2 hi + lo + mu/2, whose
    phase in units of mu/2 is positive on the torus (16 units) for 1..7."""
    r = _digit_truth(op, xd[0], yd[0])
    for x, y in zip(xd[1:], yd[1:]):
        if op == "eq":
            r = r and x == y
        else:
            units = (2 if x == y else 0) + (4 if _digit_truth(op, x, y) else -4) + (2 if r else -2) + 1
            r = 1 <= units % 16 <= 7
    return r


def _digits(v, D):
    return [(v >> (10 * d)) & (DIGIT - 1) for d in range(D)]


def _case(oracle, keys, D, B, seed):
    """B value pairs of D digits: random, equal top digits, equal values, extremes"""
    _, s1, _ = keys
    rng = np.random.default_rng(seed)
    top = DIGIT ** D
    xs = rng.integers(0, top, B).astype(np.int64)
    ys = rng.integers(0, top, B).astype(np.int64)
    for i in range(0, B, 4):
        ys[i] = xs[i]                                          # equal values
    for i in range(1, B, 4):
        low = DIGIT ** (D - 1) if D > 1 else 1
        ys[i] = (xs[i] // low) * low + rng.integers(0, low)    # equal top digit
    xs[2], ys[2] = top - 1, 0
    xs[3], ys[3] = 0, top - 1
    trl = np.zeros((D, B, 2, N1), np.uint32)
    g = np.zeros((D, B, 2 * L1, 2, N1), np.uint32)
    for d in range(D):
        for i in range(B):
            trl[d, i] = oracle.arc_trlwe(_digits(int(xs[i]), D)[d], s1, SEED, 0xA3, d * B + i)
            g[d, i] = oracle.arc_trgsw(_digits(int(ys[i]), D)[d], s1, SEED, 0xA4, d * B + i)
    return xs, ys, trl, g


def _run(engine, op, trl, g, D, B, prec):
    import torch
    prep = torch.empty(D * B * 2 * L1 * N1 * 2, dtype=torch.float64, device="cuda")
    engine.trgsw_prepare_lvl1(_dev(g), prep, prec)
    out = torch.zeros(B * (N1 + 1), dtype=torch.int32, device="cuda")
    engine.arc_compare(op, _dev(trl), prep, out, D, precision=prec)
    engine.sync()
    return out.cpu().numpy().view(np.uint32).reshape(B, N1 + 1)


def _signs(oracle, s1, out):
    return np.array([signed_diff(oracle.phase32(c, s1), 0) > 0 for c in out])


@pytest.mark.parametrize("precision", ["fp64", "split32"])
def test_arc_single_digit(engine, oracle, keys, precision):
    from cufhedb_b200 import FP64, SPLIT32
    prec = FP64 if precision == "fp64" else SPLIT32
    _, s1, _ = keys
    B = 32
    xs, ys, trl, g = _case(oracle, keys, 1, B, 5)
    for op in ("gt", "lt", "eq", "lt_strict"):
        got = _run(engine, op, trl, g, 1, B, prec)
        truth = np.array([_digit_truth(op, int(x), int(y)) for x, y in zip(xs, ys)])
        assert np.array_equal(_signs(oracle, s1, got), truth), op
        # FP64: the external product is within 1 of the exact one per
        # coefficient and the product with the test polynomial sums 1024 of
        # them; split FP32: its lo limb adds < 2^16 per coefficient
        tol = 1 << 12 if prec == FP64 else 1 << 23
        for i in range(0, B, 5):
            want = oracle.arc_single(op, trl[0, i], g[0, i])
            assert np.max(np.abs(signed_diff(got[i], want))) <= tol, (op, i)


@pytest.mark.parametrize("D", [2, 3])
@pytest.mark.parametrize("precision", ["fp64", "split32"])
def test_arc_multi_digit(engine, oracle, keys, D, precision):
    from cufhedb_b200 import FP64, SPLIT32
    prec = FP64 if precision == "fp64" else SPLIT32
    _, s1, _ = keys
    B = 48
    xs, ys, trl, g = _case(oracle, keys, D, B, 10 + D)
    res = {}
    for op in ("gt", "lt", "eq", "lt_strict"):
        got = _signs(oracle, s1, _run(engine, op, trl, g, D, B, prec))
        want = np.array([model(op, _digits(int(x), D), _digits(int(y), D)) for x, y in zip(xs, ys)])
        assert np.array_equal(got, want), op
        if op != "lt":
            plain = {"gt": xs > ys, "eq": xs == ys, "lt_strict": xs < ys}[op]
            assert np.array_equal(got, plain), op
        res[op] = got
    # the reference's less_than over several digits: where the top digits
    # differ it is x < y; where they are equal it is the complement of the
    # lower digits' less_than
    top = DIGIT ** (D - 1)
    tied = (xs // top) == (ys // top)
    assert tied.any() and (~tied).any()
    assert np.array_equal(res["lt"][~tied], (xs < ys)[~tied])
    lower = np.array([model("lt", _digits(int(x), D - 1), _digits(int(y), D - 1)) for x, y in zip(xs, ys)])
    assert np.array_equal(res["lt"][tied], ~lower[tied])


def test_arc_multi_digit_against_reference(engine, oracle, ref_keyed, keys, bkfft01):
    """Two digits, the reference's TFHEpp steps on the CPU (external product,
    PolyMul, SampleExtractIndex, IdentityKeySwitch<lvl10>, GateBootstrapping
    TLWE2TLWEFFT<lvl01>, HomAND) with the same keys: same decrypted results."""
    from cufhedb_b200 import FP64
    ref = ref_keyed
    _, s1, _ = keys
    B, D = 6, 2
    xs, ys, trl, g = _case(oracle, keys, D, B, 31)
    tv = np.full(N1, MU, np.uint32)

    def boot(x):
        fill_ref_ksk(ref, oracle, keys, 10, [x])
        return ref.pbs01(ref.iks(10, x), tv)

    for op in ("gt", "lt", "eq"):
        got = _signs(oracle, s1, _run(engine, op, trl, g, D, B, FP64))
        want = np.array([model(op, _digits(int(x), D), _digits(int(y), D)) for x, y in zip(xs, ys)])
        assert np.array_equal(got, want), op
        for i in range(B):
            gf = [oracle.trgsw32_fft(g[d, i]) for d in range(D)]
            r = ref.arc_digit(op, trl[0, i], gf[0])
            hi = ref.arc_digit(op, trl[1, i], gf[1])
            if op == "eq":
                x = r + hi
                x[N1] = np.uint32((int(x[N1]) - MU) % 2 ** 32)
            else:
                x = ref.arc_digit("equal_term", trl[1, i], gf[1]) + np.uint32(2) * hi + r
                x[N1] = np.uint32((int(x[N1]) + (MU >> 1)) % 2 ** 32)
            r = boot(x)
            assert got[i] == (signed_diff(oracle.phase32(r, s1), 0) > 0), (op, i)


def test_polymul_lvl1_and_lvl2(engine, oracle):
    """cufhedb_polymul_lvl1/2 (the reference's PolyMul_st) against the exact
    negacyclic product: the all-ones multiplier (the reference's default)
    shared by the batch, and one small multiplier per row."""
    import torch
    from oracle.oracle import N2, polymul32
    rng = np.random.default_rng(8)
    B = 6
    a = rng.integers(0, 2 ** 32, (B, N1), dtype=np.uint64).astype(np.uint32)
    ones = np.ones(N1, np.uint32)
    m = torch.from_numpy(oracle.twist_ifft32(ones)).cuda()
    out = torch.zeros(B * N1, dtype=torch.int32, device="cuda")
    engine.polymul_lvl1(_dev(a), m, out, shared=True)
    engine.sync()
    got = out.cpu().numpy().view(np.uint32).reshape(B, N1)
    for i in range(B):
        assert np.max(np.abs(signed_diff(got[i], polymul32(a[i], ones)))) <= 4
    p = rng.integers(-2, 3, (B, N1)).astype(np.int64).astype(np.uint32)
    mp = torch.from_numpy(np.stack([oracle.twist_ifft32(x) for x in p])).cuda()
    engine.polymul_lvl1(_dev(a), mp, out, shared=False)
    engine.sync()
    got = out.cpu().numpy().view(np.uint32).reshape(B, N1)
    for i in range(B):
        assert np.max(np.abs(signed_diff(got[i], polymul32(a[i], p[i])))) <= 4
    # lvl2: 64-bit torus through the FP64 transform keeps the top ~2^-45 of
    # the product, as the reference's GPU kernel does
    a2 = rng.integers(0, 2 ** 64, (2, N2), dtype=np.uint64)
    m2 = torch.from_numpy(oracle.twist_ifft64(np.ones(N2, np.uint64))).cuda()
    out2 = torch.zeros(2 * N2, dtype=torch.int64, device="cuda")
    engine.polymul_lvl2(torch.from_numpy(a2.view(np.int64).copy()).cuda(), m2, out2, shared=True)
    engine.sync()
    got2 = out2.cpu().numpy().view(np.uint64).reshape(2, N2)
    for i in range(2):
        s = np.cumsum(a2[i].astype(object)) % 2 ** 64
        want = np.array([(2 * int(s[k]) - int(s[-1])) % 2 ** 64 for k in range(N2)], dtype=object)
        d = (got2[i].astype(object) - want) % 2 ** 64
        d = np.array([int(x) - 2 ** 64 if x >= 2 ** 63 else int(x) for x in d])
        assert np.max(np.abs(d)) < 2 ** 30


@pytest.mark.parametrize("precision", ["fp64", "split32"])
def test_arc_single_digit_golden(engine, oracle, keys, precision):
    """The GPU comparison against the reference's own outputs stored in
    tests/golden/arcedb_lvl1.npz (inputs regenerated by the oracle)."""
    import os
    from cufhedb_b200 import FP64, SPLIT32
    prec = FP64 if precision == "fp64" else SPLIT32
    g = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "arcedb_lvl1.npz"))
    _, s1, _ = keys
    pairs = g["pairs"]
    B = len(pairs)
    trl = np.stack([oracle.arc_trlwe(int(x), s1, SEED, 0xA5, i) for i, (x, _) in enumerate(pairs)])[None]
    gg = np.stack([oracle.arc_trgsw(int(y), s1, SEED, 0xA6, i) for i, (_, y) in enumerate(pairs)])[None]
    tol = 1 << 12 if prec == FP64 else 1 << 23
    for k, op in enumerate(("gt", "lt", "eq")):
        got = _run(engine, op, trl, gg, 1, B, prec)
        for i in range(B):
            assert np.max(np.abs(signed_diff(got[i], g["out"][i, k]))) <= tol, (op, i)
