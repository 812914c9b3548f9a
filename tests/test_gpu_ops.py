"""GPU parity: the batched operator layer (cuHEDB MSB / identity bootstraps,
HomMSB chains, comparisons, HomAND / HomOR, graph capture) against plaintext
evaluation and, for a few rows, against the reference's own CPU operators
(HEDB::less_than_equal etc. compiled in oracle/_ref) on the same keys."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import SEED, signed_diff

from oracle.oracle import N1, N2, NS_LVL1, NS_LVL2

pytestmark = pytest.mark.gpu
MU1 = 1 << 29


def _dev(a):
    import torch
    a = np.ascontiguousarray(a)
    v = a.view(np.int64) if a.dtype == np.uint64 else a.view(np.int32)
    return torch.from_numpy(v.copy()).cuda()


def _empty1(B):
    import torch
    return torch.zeros(B * (N1 + 1), dtype=torch.int32, device="cuda")


@pytest.fixture(scope="module")
def eng_all():
    from cufhedb_b200 import GEN_ALL, Engine
    eng = Engine(0)
    eng.keygen(SEED, GEN_ALL)
    yield eng
    eng.close()


def enc1(oracle, s1, vals, pb, base):
    return np.stack([oracle.tlwe32(int(v) << (32 - pb - 1), s1, NS_LVL1, SEED, 0x71, base + i)
                     for i, v in enumerate(vals)])


def enc2(oracle, s2, vals, pb, base):
    return np.stack([oracle.tlwe64(int(v) << (64 - pb - 1), s2, NS_LVL2, SEED, 0x72, base + i)
                     for i, v in enumerate(vals)])


def logic_bits(oracle, out, s1, B):
    o = out.cpu().numpy().view(np.uint32).reshape(B, N1 + 1)
    return np.array([int(signed_diff(oracle.phase32(x, s1), 0)) > 0 for x in o]).astype(int)


def arith_bits(oracle, out, s1, B):
    o = out.cpu().numpy().view(np.uint32).reshape(B, N1 + 1)
    return np.array([int(round(oracle.phase32(x, s1) / 2 ** 31)) % 2 for x in o]).astype(int)


TRUTH = {"gt": lambda x, y: x > y, "ge": lambda x, y: x >= y, "lt": lambda x, y: x < y,
         "le": lambda x, y: x <= y, "eq": lambda x, y: x == y}


@pytest.mark.parametrize("op", ["gt", "ge", "lt", "le", "eq"])
def test_compare_lvl1_6bit(eng_all, oracle, keys, op):
    _, s1, _ = keys
    pb, B = 6, 40
    rng = np.random.default_rng(61)
    x = rng.integers(0, 2 ** pb, B); y = rng.integers(0, 2 ** pb, B)
    y[:5] = x[:5]
    c1, c2 = enc1(oracle, s1, x, pb, 0), enc1(oracle, s1, y, pb, 500)
    out = _empty1(B)
    eng_all.compare(op, 1, _dev(c1), _dev(c2), out, pb, logic=True)
    eng_all.sync()
    assert np.array_equal(logic_bits(oracle, out, s1, B), TRUTH[op](x, y).astype(int))


@pytest.mark.parametrize("op", ["le", "gt"])
def test_compare_lvl2_20bit_range_filter(eng_all, oracle, keys, op):
    """The range-filter shape: 20-bit values encrypted at lvl2 against an
    encrypted threshold (6 lvl02 + 3 lvl01 bootstraps per row)."""
    _, s1, s2 = keys
    pb, B = 20, 24
    rng = np.random.default_rng(62)
    x = rng.integers(0, 2 ** pb, B)
    c = int(np.percentile(x, 30))
    x[:3] = [c, c - 1, c + 1]
    c1, c2 = enc2(oracle, s2, x, pb, 0), enc2(oracle, s2, np.full(B, c), pb, 1000)
    out = _empty1(B)
    eng_all.compare(op, 2, _dev(c1), _dev(c2), out, pb, logic=True)
    eng_all.sync()
    assert np.array_equal(logic_bits(oracle, out, s1, B), TRUTH[op](x, np.full(B, c)).astype(int))


@pytest.mark.parametrize("logic", [True, False])
def test_compare_lvl2_30bit(eng_all, oracle, keys, logic):
    """30-bit values (the reference's HomComp width): the longest MSB chain
    (ImExtractMSB33), LOGIC and ARITHMETIC results."""
    _, s1, s2 = keys
    pb, B = 30, 32
    rng = np.random.default_rng(65)
    x = rng.integers(0, 2 ** pb, B); y = rng.integers(0, 2 ** pb, B)
    y[:4] = x[:4]
    c1, c2 = enc2(oracle, s2, x, pb, 2000), enc2(oracle, s2, y, pb, 3000)
    out = _empty1(B)
    eng_all.compare("ge", 2, _dev(c1), _dev(c2), out, pb, logic=logic)
    eng_all.sync()
    got = logic_bits(oracle, out, s1, B) if logic else arith_bits(oracle, out, s1, B)
    assert np.array_equal(got, (x >= y).astype(int))


def test_compare_arithmetic_result_and_gates(eng_all, oracle, keys):
    _, s1, _ = keys
    pb, B = 5, 32
    rng = np.random.default_rng(63)
    x = rng.integers(0, 2 ** pb, B); y = rng.integers(0, 2 ** pb, B)
    c1, c2 = enc1(oracle, s1, x, pb, 0), enc1(oracle, s1, y, pb, 100)
    out = _empty1(B)
    eng_all.compare("ge", 1, _dev(c1), _dev(c2), out, pb, logic=False)
    eng_all.sync()
    assert np.array_equal(arith_bits(oracle, out, s1, B), (x >= y).astype(int))
    # HomAND / HomOR of LOGIC inputs
    a = rng.integers(0, 2, B); b = rng.integers(0, 2, B)
    enc = lambda bits, base: np.stack([oracle.tlwe32(MU1 if t else (-MU1) & 0xFFFFFFFF, s1, NS_LVL1, SEED, 0x73,
                                                     base + i) for i, t in enumerate(bits)])
    ca, cb = _dev(enc(a, 0)), _dev(enc(b, 100))
    o_and, o_or = _empty1(B), _empty1(B)
    eng_all.hom_and(ca, cb, o_and)
    eng_all.hom_or(ca, cb, o_or)
    eng_all.sync()
    assert np.array_equal(logic_bits(oracle, o_and, s1, B), a & b)
    assert np.array_equal(logic_bits(oracle, o_or, s1, B), a | b)


def test_hom_msb_plain_bits_out_of_range(eng_all):
    from cufhedb_b200 import CufhedbError
    import torch
    x = torch.zeros(2 * (N1 + 1), dtype=torch.int32, device="cuda")
    with pytest.raises(CufhedbError) as e:
        eng_all.hom_msb(1, x, _empty1(2), 11)
    assert e.value.code == 1 and "Plain bits out" in str(e.value)
    y = torch.zeros(2 * (N2 + 1), dtype=torch.int64, device="cuda")
    with pytest.raises(CufhedbError):
        eng_all.hom_msb(2, y, _empty1(2), 34)


def test_compare_graph_capture_replays(eng_all, oracle, keys):
    import torch
    _, s1, s2 = keys
    pb, B = 16, 16
    rng = np.random.default_rng(64)
    x = rng.integers(0, 2 ** pb, B); c = 2 ** 15
    c1, c2 = _dev(enc2(oracle, s2, x, pb, 0)), _dev(enc2(oracle, s2, np.full(B, c), pb, 200))
    out = _empty1(B)
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        eng_all.graph_begin(s)
        eng_all.compare("lt", 2, c1, c2, out, pb, stream=s)
        g = eng_all.graph_end(s)
        for _ in range(2):
            out.zero_()
            eng_all.graph_launch(g, s)
            s.synchronize()
            assert np.array_equal(logic_bits(oracle, out, s1, B), (x < c).astype(int))
        eng_all.graph_destroy(g)
    eng_all.sync(s)


def test_compare_lvl2_matches_reference_cpu_operators(eng_all, oracle, ref, keys, bk01):
    """Same keys, same ciphertexts: HEDB::less_than_equal<Lvl2> on the CPU
    (the reference's own operator chain) decrypts to the same bits."""
    s0, s1, s2 = keys
    ref.set_secret(s0, s1, s2)
    ref.set_bk01(bk01)
    ref.set_bk02(oracle.bk02(SEED, s0, s2))
    for kind in (10, 20, 21):
        ptr, _ = ref.ksk_view(kind)
        oracle.ksk_full_into(kind, SEED, keys, ptr)
    pb, B = 12, 2
    x = np.array([1000, 3000]); c = 2048
    c1, c2 = enc2(oracle, s2, x, pb, 0), enc2(oracle, s2, np.full(B, c), pb, 300)
    out = _empty1(B)
    eng_all.compare("le", 2, _dev(c1), _dev(c2), out, pb, logic=True)
    eng_all.sync()
    got = logic_bits(oracle, out, s1, B)
    theirs = np.array([int(signed_diff(oracle.phase32(ref.compare_lvl2(c1[i], c2[i], 3, pb, True), s1), 0)) > 0
                       for i in range(B)]).astype(int)
    assert np.array_equal(got, (x <= c).astype(int))
    assert np.array_equal(theirs, got)
