"""CPU: the C restatement (oracle/) against the reference's own TFHEpp built
from its sources (oracle/_ref) and against the committed golden vectors."""
from __future__ import annotations

import os

import numpy as np
import pytest

from conftest import SEED, fill_ref_ksk, signed_diff

from oracle.oracle import N0, N1, N2, NS_LVL0, NS_LVL1, NS_LVL2

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_generator_is_deterministic(oracle):
    a = [oracle.draw(1, 2, i) for i in range(4)]
    b = [oracle.draw(1, 2, i) for i in range(4)]
    assert a == b and len(set(a)) == 4
    ns = np.array([oracle.noise(7, 3, 2 * i, NS_LVL0) for i in range(20000)], np.float64)
    assert abs(ns.mean()) < 0.05 * 2 ** 16 and 0.9 < ns.std() / 2 ** 16 < 1.1


def test_secret_keys_hamming(oracle, keys):
    s0, s1, s2 = keys
    for s, n, h in ((s0, N0, 512), (s1, N1, 512), (s2, N2, 1024)):
        assert set(np.unique(s)) <= {0, 1}
        assert 0.3 * n < s.sum() <= h


def test_fft_matches_reference(oracle, ref):
    rng = np.random.default_rng(11)
    for _ in range(4):
        a = rng.integers(0, 2 ** 32, N1, dtype=np.uint64).astype(np.uint32)
        vo, vr = oracle.twist_ifft32(a), ref.twist_ifft32(a)
        assert np.max(np.abs(vo - vr)) <= 1e-13 * np.max(np.abs(vr))
        d = signed_diff(oracle.twist_fft32(vr), ref.twist_fft32(vr))
        assert np.max(np.abs(d)) <= 1
        assert np.max(np.abs(signed_diff(oracle.twist_fft32(vo), a))) <= 1
        a2 = rng.integers(0, 2 ** 64, N2, dtype=np.uint64)
        wo, wr = oracle.twist_ifft64(a2), ref.twist_ifft64(a2)
        assert np.max(np.abs(wo - wr)) <= 1e-13 * np.max(np.abs(wr))
        # lvl2 round trip error is intrinsic to FP64 (TFHEpp test/polymul.cpp:57-68 allows 2^14)
        d2 = signed_diff(oracle.twist_fft64(wr), ref.twist_fft64(wr), 64)
        assert max(abs(int(x)) for x in d2) <= 2 ** 14


def test_decomposition_bit_exact(oracle, ref):
    rng = np.random.default_rng(12)
    a = rng.integers(0, 2 ** 32, N1, dtype=np.uint64).astype(np.uint32)
    a[:4] = [0, 0xFFFFFFFF, 0x80000000, 0x7FFFFFFF]
    for d in range(3):
        assert np.array_equal(oracle.decomp32(a, d), ref.decomp32(a, d))
    a2 = rng.integers(0, 2 ** 64, N2, dtype=np.uint64)
    a2[:3] = [0, 2 ** 64 - 1, 2 ** 63]
    for d in range(4):
        assert np.array_equal(oracle.decomp64(a2, d), ref.decomp64(a2, d))


def test_external_product_lvl1(oracle, ref, keys):
    _, s1, _ = keys
    rng = np.random.default_rng(13)
    for m in (0, 1):
        g = oracle.trgsw32(m, s1, SEED, 0x30, m)
        gfft = oracle.trgsw32_fft(g)
        trl = rng.integers(0, 2 ** 32, (2, N1), dtype=np.uint64).astype(np.uint32)
        r_ref = ref.extprod32(trl, gfft)
        r_fft = oracle.extprod32_fft(trl, gfft)
        r_ex = oracle.extprod32_exact(trl, g)
        assert np.max(np.abs(signed_diff(r_ref, r_fft))) <= 1
        assert np.max(np.abs(signed_diff(r_ref, r_ex))) <= 1


def test_external_product_lvl2(oracle, ref, keys):
    _, _, s2 = keys
    rng = np.random.default_rng(14)
    g = oracle.trgsw64(1, s2, SEED, 0x31, 0)
    gfft = oracle.trgsw64_fft(g)
    trl = rng.integers(0, 2 ** 64, (2, N2), dtype=np.uint64)
    r_ref = ref.extprod64(trl, gfft)
    r_ex = oracle.extprod64_exact(trl, g)
    # FP64 on the 64-bit torus loses the low bits (TFHEpp FFT round-off), far below the noise
    d = signed_diff(r_ref, r_ex, 64)
    assert max(abs(int(x)) for x in d.ravel()) < 2 ** 30


@pytest.mark.parametrize("kind", [10, 20, 21])
def test_identity_key_switch_bit_exact(oracle, ref, keys, kind):
    s0, s1, s2 = keys
    rng = np.random.default_rng(15 + kind)
    if kind == 10:
        xs = [oracle.tlwe32(int(m) << 29, s1, NS_LVL1, SEED, 0x41, i)
              for i, m in enumerate(rng.integers(0, 8, 3))]
    else:
        xs = [oracle.tlwe64(int(m) << 61, s2, NS_LVL2, SEED, 0x42, i)
              for i, m in enumerate(rng.integers(0, 8, 3))]
    ref.set_secret(s0, s1, s2)
    fill_ref_ksk(ref, oracle, keys, kind, xs)
    for x in xs:
        assert np.array_equal(oracle.iks(kind, x, SEED, keys), ref.iks(kind, x))


def test_pbs01_decrypts_like_reference(oracle, ref_keyed, keys, bkfft01):
    s0, s1, _ = keys
    tv = np.full(N1, 1 << 29, np.uint32)
    for t in range(6):
        m = (1 << 29) if t % 2 else (-(1 << 29)) & 0xFFFFFFFF
        x0 = oracle.tlwe32(m, s0, NS_LVL0, SEED, 0x40, t)
        r = ref_keyed.pbs01(x0, tv)
        o = oracle.pbs01(x0, bkfft01, tv)
        pr = int(signed_diff(oracle.phase32(r, s1), 0))
        po = int(signed_diff(oracle.phase32(o, s1), 0))
        expect = 1 << 29 if t % 2 else -(1 << 29)
        assert abs(pr - expect) < 2 ** 26 and abs(po - expect) < 2 ** 26


def test_fast_exact_pbs_equals_schoolbook(oracle, keys, bk01):
    """The exact PBS used for noise measurements (16-bit key limbs through the
    FP64 FFT, every product rounded to its integer) equals the schoolbook
    integer product bit for bit: external products on random accumulators,
    and a whole bootstrap against orc_pbs01_exact; its exactness certificate
    (largest distance of an FFT product from an integer) stays far below 1/4."""
    s0, _, _ = keys
    prep = oracle.bk01_exact_prepare(bk01)
    rng = np.random.default_rng(0x5C)
    for i in (0, 1, 671):
        trl = rng.integers(0, 2 ** 32, (2, N1), dtype=np.uint64).astype(np.uint32)
        got, dev = oracle.extprod32_exact_split(trl, prep[i])
        assert np.array_equal(got, oracle.extprod32_exact(trl, bk01[i])) and dev < 1e-3
    x = np.stack([oracle.tlwe32((1 << 29) if i else (-(1 << 29)) & 0xFFFFFFFF, s0, NS_LVL0, SEED, 0x5D, i)
                  for i in range(2)])
    tv = np.full(N1, 1 << 29, np.uint32)
    out, dev = oracle.pbs01_exact_batch(x, prep, tv)
    assert dev < 1e-3
    assert np.array_equal(out[0], oracle.pbs01_exact(x[0], bk01, tv))
    ph = [int(signed_diff(oracle.phase32(o, keys[1]), 0)) for o in out]
    assert ph[0] < 0 < ph[1]


def test_golden_vectors(oracle, keys):
    """Fixtures produced by the reference's TFHEpp (tests/golden/make_golden.py)."""
    g = np.load(os.path.join(GOLD, "tfhepp_lvl1.npz"))
    assert int(g["seed"]) == SEED
    for a, v, back in zip(g["fft_in"], g["fft_out"], g["fft_back"]):
        assert np.max(np.abs(oracle.twist_ifft32(a) - v)) <= 1e-13 * np.max(np.abs(v))
        assert np.max(np.abs(signed_diff(oracle.twist_fft32(v), back))) <= 1
    for a, d0, d1, d2 in zip(g["fft_in"], g["dec0"], g["dec1"], g["dec2"]):
        assert np.array_equal(oracle.decomp32(a, 0), d0)
        assert np.array_equal(oracle.decomp32(a, 1), d1)
        assert np.array_equal(oracle.decomp32(a, 2), d2)
    s0, s1, _ = keys
    for q, row in zip(g["ksk_rows"], g["ksk_sample"]):
        q = int(q)
        assert np.array_equal(oracle.ksk_row(10, SEED, keys, q // 2046, (q % 2046) // 1023, q % 1023), row)
    for x, out in zip(g["iks_in"], g["iks_out"]):
        assert np.array_equal(oracle.iks(10, x, SEED, keys), out)
    bk = oracle.bk01(SEED, s0, s1)
    assert np.array_equal(bk[3, 4, 1, :8], g["bk_sample"])
    tv = np.full(N1, 1 << 29, np.uint32)
    bkf = oracle.bkfft01(bk)
    for x0, bit, out in zip(g["pbs_in"], g["pbs_bit"], g["pbs_out"]):
        assert int(signed_diff(oracle.phase32(x0, s0), 0) > 0) == int(bit)
        assert int(signed_diff(oracle.phase32(out, s1), 0) > 0) == int(bit)
    for x0, out in zip(g["pbs_in"][:2], g["pbs_out"][:2]):
        mine = oracle.pbs01(x0, bkf, tv)
        assert (signed_diff(oracle.phase32(mine, s1), 0) > 0) == (signed_diff(oracle.phase32(out, s1), 0) > 0)


def test_golden_vectors_lvl2(oracle, keys):
    """lvl2 fixtures produced by the reference's TFHEpp (tests/golden/make_golden.py):
    transforms, decomposition, both lvl2 key switches and the lvl02 PBS."""
    g = np.load(os.path.join(GOLD, "tfhepp_lvl2.npz"))
    assert int(g["seed"]) == SEED
    for a, v, back in zip(g["fft_in"], g["fft_out"], g["fft_back"]):
        assert np.max(np.abs(oracle.twist_ifft64(a) - v)) <= 1e-13 * np.max(np.abs(v))
        # lvl2 round trip error is intrinsic to FP64 (TFHEpp test/polymul.cpp:57-68 allows 2^14)
        assert max(abs(int(x)) for x in signed_diff(oracle.twist_fft64(v), back, 64)) <= 2 ** 14
    for a, digits in zip(g["fft_in"], g["dec"]):
        for d in range(4):
            assert np.array_equal(oracle.decomp64(a, d), digits[d])
    for kind in (20, 21):
        for x, out in zip(g[f"iks{kind}_in"], g[f"iks{kind}_out"]):
            assert np.array_equal(oracle.iks(kind, x, SEED, keys), out)
    s0, _, s2 = keys
    bk = oracle.bk02(SEED, s0, s2)
    assert np.array_equal(bk[5, 6, 1, :8], g["bk_sample"])
    bkf = np.stack([oracle.trgsw64_fft(row) for row in bk])
    tv = np.full(N2, 1 << 61, np.uint64)
    for x0, bit, out in zip(g["pbs_in"], g["pbs_bit"], g["pbs_out"]):
        theirs = int(signed_diff(oracle.phase64(out, s2), 0, 64))
        mine = int(signed_diff(oracle.phase64(oracle.pbs02(x0, bkf, tv), s2), 0, 64))
        expect = (1 << 61) if bit else -(1 << 61)
        assert abs(theirs - expect) < 2 ** 56 and abs(mine - theirs) < 2 ** 56


def test_arcedb_digit_matches_reference(oracle, ref, keys):
    """The oracle's ArcEDB encodings and single-digit comparisons against the
    reference's own TFHEpp steps (FFT external product and FFT PolyMul, so a
    few torus units of rounding apart from the exact oracle)."""
    _, s1, _ = keys
    rng = np.random.default_rng(77)
    pairs = [(0, 0), (0, 1), (1, 0), (5, 5), (1023, 0), (0, 1023), (512, 511), (1023, 1023)]
    pairs += [tuple(int(v) for v in rng.integers(0, 1024, 2)) for _ in range(4)]
    for i, (x, y) in enumerate(pairs):
        trl = oracle.arc_trlwe(x, s1, SEED, 0xA1, i)
        g = oracle.arc_trgsw(y, s1, SEED, 0xA2, i)
        gfft = oracle.trgsw32_fft(g)
        for op, truth in (("gt", x > y), ("lt", x <= y), ("eq", x == y)):
            mine = oracle.arc_single(op, trl, g)
            theirs = ref.arc_digit(op, trl, gfft)
            assert np.max(np.abs(signed_diff(mine, theirs))) <= 256, (op, x, y)
            assert (signed_diff(oracle.phase32(mine, s1), 0) > 0) == truth, (op, x, y)
        strict = oracle.arc_single("lt_strict", trl, g)
        assert (signed_diff(oracle.phase32(strict, s1), 0) > 0) == (x < y)
        eq_term = signed_diff(oracle.phase32(ref.arc_digit("equal_term", trl, gfft), s1), 0)
        assert abs(eq_term - (1 << 29 if x == y else 0)) < 1 << 26


def test_arcedb_golden_vectors(oracle, keys):
    """tests/golden/arcedb_lvl1.npz: the reference's own single-digit ArcEDB
    outputs (tests/golden/make_golden.py) on encryptions the oracle
    regenerates deterministically; no compiled reference needed."""
    g = np.load(os.path.join(GOLD, "arcedb_lvl1.npz"))
    assert int(g["seed"]) == SEED
    _, s1, _ = keys
    ops = ("gt", "lt", "eq")
    for i, (x, y) in enumerate(g["pairs"]):
        trl = oracle.arc_trlwe(int(x), s1, SEED, 0xA5, i)
        gi = oracle.arc_trgsw(int(y), s1, SEED, 0xA6, i)
        for k, op in enumerate(ops):
            mine = oracle.arc_single(op, trl, gi)
            assert np.max(np.abs(signed_diff(mine, g["out"][i, k]))) <= 256, (op, x, y)
        truth = (x > y, x <= y, x == y)
        for k in range(3):
            assert (signed_diff(oracle.phase32(g["out"][i, k], s1), 0) > 0) == truth[k]
