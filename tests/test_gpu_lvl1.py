"""GPU parity: the lvl1 path (keys, transforms, IKS10, PBS01, gates) through
the C ABI against the oracle and the reference's own TFHEpp."""
from __future__ import annotations

import os

import numpy as np
import pytest

from conftest import SEED, fill_ref_ksk, signed_diff

from oracle.oracle import N0, N1, NS_LVL0, NS_LVL1

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
MU = 1 << 29


def dev(a):
    import torch
    a = np.ascontiguousarray(a)
    view = a.view(np.int32) if a.dtype == np.uint32 else a.view(np.int64) if a.dtype == np.uint64 else a
    return torch.from_numpy(view.copy()).cuda()


def host(t, dtype=np.uint32):
    return t.cpu().numpy().view(dtype)


def empty_dev(n, dtype="i32"):
    import torch
    return torch.zeros(n, dtype={"i32": torch.int32, "i64": torch.int64, "f64": torch.float64}[dtype], device="cuda")


def phase(oracle, c, key):
    return int(signed_diff(oracle.phase32(c, key), 0))


def test_keygen_matches_oracle(engine, oracle, keys, bk01):
    assert np.array_equal(engine.export_bk_lvl01(), bk01)
    rows = np.array([0, 1, 777_777, 1024 * 2 * 1023 - 1], np.uint64)
    got = engine.export_ksk_rows(10, rows)
    for q, row in zip(rows, got):
        q = int(q)
        assert np.array_equal(oracle.ksk_row(10, SEED, keys, q // 2046, (q % 2046) // 1023, q % 1023), row)


def test_twist_transforms_match_reference(engine, ref):
    rng = np.random.default_rng(21)
    B = 37
    a = rng.integers(0, 2 ** 32, (B, N1), dtype=np.uint64).astype(np.uint32)
    out = empty_dev(B * N1, "f64")
    engine.twist_ifft_lvl1(dev(a), out)
    engine.sync()
    got = out.cpu().numpy().reshape(B, N1)
    want = np.stack([ref.twist_ifft32(x) for x in a])
    assert np.max(np.abs(got - want)) <= 1e-13 * np.max(np.abs(want))
    back = empty_dev(B * N1)
    import torch
    engine.twist_fft_lvl1(torch.from_numpy(want.copy()).cuda(), back)
    engine.sync()
    back = host(back).reshape(B, N1)
    want_back = np.stack([ref.twist_fft32(v) for v in want])
    d = signed_diff(back, want_back)
    assert np.max(np.abs(d)) <= 1
    assert np.max(np.abs(signed_diff(back, a))) <= 1
    g = np.load(os.path.join(GOLD, "tfhepp_lvl1.npz"))
    out = empty_dev(4 * N1, "f64")
    engine.twist_ifft_lvl1(dev(g["fft_in"]), out)
    engine.sync()
    assert np.max(np.abs(out.cpu().numpy().reshape(4, N1) - g["fft_out"])) <= 1e-13 * np.max(np.abs(g["fft_out"]))


def test_iks10_bit_exact(engine, oracle, keys):
    s0, s1, _ = keys
    B = 37
    xs = np.stack([oracle.tlwe32((i % 8) << 29, s1, NS_LVL1, SEED, 0x41, i) for i in range(B)])
    xs[0, :] = 0
    xs[1, :N1] = 0xFFFFFFFF
    out = empty_dev(B * (N0 + 1))
    engine.iks(10, dev(xs), out)
    engine.sync()
    got = host(out).reshape(B, N0 + 1)
    for x, o in zip(xs, got):
        assert np.array_equal(oracle.iks(10, x, SEED, keys), o)
    g = np.load(os.path.join(GOLD, "tfhepp_lvl1.npz"))
    out = empty_dev(4 * (N0 + 1))
    engine.iks(10, dev(g["iks_in"]), out)
    engine.sync()
    assert np.array_equal(host(out).reshape(4, N0 + 1), g["iks_out"])


@pytest.mark.parametrize("tvkind", ["const", "staircase", "poly"])
def test_pbs01_trivial_inputs_exact(engine, oracle, tvkind):
    """a = 0 makes every rotation index 0, so the PBS is exactly X^bbar * tv,
    sample-extracted: bit-exact, including bbar = 2N (b < 2^21)."""
    from cufhedb_b200 import testvec_const, testvec_poly, testvec_staircase
    B = 9
    x = np.zeros((B, N0 + 1), np.uint32)
    x[:, N0] = np.array([0, 1, (1 << 21) - 1, 1 << 21, 0x80000000, 0xFFFFFFFF, 1234 << 21, 3 << 30, 7], np.uint32)
    if tvkind == "const":
        tv = testvec_const(MU); tvp = np.full(N1, MU, np.uint32)
    elif tvkind == "staircase":
        tv = testvec_staircase(24, 6); tvp = oracle.gpoly32(4, 24)
    else:
        tvp = np.random.default_rng(5).integers(0, 2 ** 32, N1, dtype=np.uint64).astype(np.uint32)
        tvd = dev(tvp)
        tv = testvec_poly(tvd)
    out = empty_dev(B * (N1 + 1))
    engine.pbs_lvl01(dev(x), out, tv)
    engine.sync()
    got = host(out).reshape(B, N1 + 1)
    dummy_bkf = np.zeros((N0, 6, 2, N1), np.float64)
    for xi, o in zip(x, got):
        assert np.array_equal(oracle.pbs01(xi, dummy_bkf, tvp), o)


def test_pbs01_decrypts_batch(engine, oracle, keys):
    s0, s1, _ = keys
    B = 7 * 20 + 3
    bits = np.random.default_rng(22).integers(0, 2, B)
    x = np.stack([oracle.tlwe32(MU if b else (-MU) & 0xFFFFFFFF, s0, NS_LVL0, SEED, 0x50, i) for i, b in enumerate(bits)])
    from cufhedb_b200 import testvec_const
    out = empty_dev(B * (N1 + 1))
    engine.pbs_lvl01(dev(x), out, testvec_const(MU))
    engine.sync()
    got = host(out).reshape(B, N1 + 1)
    ph = np.array([phase(oracle, o, s1) for o in got])
    assert np.array_equal((ph > 0).astype(int), bits)
    err = np.abs(ph) - MU
    assert np.max(np.abs(err)) < 2 ** 26, np.max(np.abs(err))


def test_pbs01_matches_reference(engine, oracle, ref_keyed, keys, bkfft01):
    """Same keys and inputs through the reference's TFHEpp: same decryptions,
    output phases within the bootstrapping noise of each other."""
    s0, s1, _ = keys
    B = 6
    from cufhedb_b200 import testvec_const
    x = np.stack([oracle.tlwe32(MU if i % 2 else (-MU) & 0xFFFFFFFF, s0, NS_LVL0, SEED, 0x51, i) for i in range(B)])
    out = empty_dev(B * (N1 + 1))
    engine.pbs_lvl01(dev(x), out, testvec_const(MU))
    engine.sync()
    got = host(out).reshape(B, N1 + 1)
    tv = np.full(N1, MU, np.uint32)
    for xi, o in zip(x, got):
        r = ref_keyed.pbs01(xi, tv)
        pr, pg = phase(oracle, r, s1), phase(oracle, o, s1)
        assert (pr > 0) == (pg > 0)
        assert abs(pr - pg) < 2 ** 25
    g = np.load(os.path.join(GOLD, "tfhepp_lvl1.npz"))
    out = empty_dev(4 * (N1 + 1))
    engine.pbs_lvl01(dev(g["pbs_in"]), out, testvec_const(MU))
    engine.sync()
    for o, bit in zip(host(out).reshape(4, N1 + 1), g["pbs_bit"]):
        assert int(phase(oracle, o, s1) > 0) == int(bit)


@pytest.mark.parametrize("gate", ["NAND", "AND", "OR", "NOR", "XOR", "XNOR", "ANDNY", "ANDYN", "ORNY", "ORYN"])
def test_gates_truth_table(engine, oracle, keys, gate):
    s0, s1, _ = keys
    B = 64
    from cufhedb_b200 import GATES
    rng = np.random.default_rng(100 + GATES[gate])
    a = rng.integers(0, 2, B); b = rng.integers(0, 2, B)
    enc = lambda bits, base: np.stack([oracle.tlwe32(MU if t else (-MU) & 0xFFFFFFFF, s1, NS_LVL1, SEED, 0x60, base + i)
                                       for i, t in enumerate(bits)])
    ca, cb = enc(a, 0), enc(b, 1000)
    out = empty_dev(B * (N1 + 1))
    engine.gate_lvl1(gate, dev(ca), dev(cb), out)
    engine.sync()
    got = np.array([phase(oracle, o, s1) > 0 for o in host(out).reshape(B, N1 + 1)]).astype(int)
    truth = {"NAND": 1 - (a & b), "AND": a & b, "OR": a | b, "NOR": 1 - (a | b), "XOR": a ^ b, "XNOR": 1 - (a ^ b),
             "ANDNY": (1 - a) & b, "ANDYN": a & (1 - b), "ORNY": (1 - a) | b, "ORYN": a | (1 - b)}[gate]
    assert np.array_equal(got, truth)


def test_homnand_matches_reference(engine, oracle, ref_keyed, keys):
    s0, s1, _ = keys
    B = 4
    a, b = np.array([0, 0, 1, 1]), np.array([0, 1, 0, 1])
    enc = lambda bits, base: np.stack([oracle.tlwe32(MU if t else (-MU) & 0xFFFFFFFF, s1, NS_LVL1, SEED, 0x61, base + i)
                                       for i, t in enumerate(bits)])
    ca, cb = enc(a, 0), enc(b, 100)
    gate_in = [((0 - ca[i].astype(np.uint64) - cb[i].astype(np.uint64)) & 0xFFFFFFFF).astype(np.uint32) for i in range(B)]
    for g_ in gate_in:
        g_[N1] = (int(g_[N1]) + MU) & 0xFFFFFFFF
    fill_ref_ksk(ref_keyed, oracle, keys, 10, gate_in)
    got = engine.gate_lvl1_host("NAND", ca, cb)
    for i in range(B):
        r = ref_keyed.homnand(ca[i], cb[i])
        pr, pg = phase(oracle, r, s1), phase(oracle, got[i], s1)
        assert (pr > 0) == (pg > 0) == bool(1 - (a[i] & b[i]))
        assert abs(pr - pg) < 2 ** 25


def test_api_errors(engine):
    from cufhedb_b200 import CufhedbError, Engine, testvec_const
    import torch
    x = empty_dev(N0 + 1)
    out = empty_dev(N1 + 1)
    engine.pbs_lvl01(x[:0], out[:0], testvec_const(MU))  # B = 0 is a no-op
    with pytest.raises(CufhedbError) as e:
        engine.pbs_lvl01(x, out, testvec_const(MU), precision=7)
    assert e.value.code == 1
    fresh = Engine(0)
    with pytest.raises(CufhedbError) as e:
        fresh.pbs_lvl01(x, out, testvec_const(MU))
    assert e.value.code == 2
    fresh.close()
    engine.sync()


@pytest.mark.parametrize("path", ["split32", "split32tc"])
def test_split32_pbs_decrypts_with_fp64_noise_level(engine, oracle, keys, path):
    """Split-precision FP32 path: every output decrypts, and its output noise
    (phase minus the encoded +-mu) has the variance of the FP64 path's.  The
    two paths' outputs are not compared with each other: a few-unit difference
    in the accumulator changes which way the gadget decomposition rounds, so
    two correct runs carry independent rounding noise.  With 1,029 samples per
    path the variance ratio of two equal-variance noises lies within
    [0.88, 1.13] at 95 %; the bound 1.25 leaves room for that spread."""
    from cufhedb_b200 import FP64, SPLIT32, SPLIT32_TC, testvec_const
    SPLIT = SPLIT32 if path == "split32" else SPLIT32_TC
    s0, s1, _ = keys
    B = 7 * 147
    bits = np.random.default_rng(31).integers(0, 2, B)
    x = np.stack([oracle.tlwe32(MU if b else (-MU) & 0xFFFFFFFF, s0, NS_LVL0, SEED, 0x52, i) for i, b in enumerate(bits)])
    xd = dev(x)
    o64, o32 = empty_dev(B * (N1 + 1)), empty_dev(B * (N1 + 1))
    engine.pbs_lvl01(xd, o64, testvec_const(MU), FP64)
    engine.pbs_lvl01(xd, o32, testvec_const(MU), SPLIT)
    engine.sync()
    s1u = s1.astype(np.uint64)

    def phases(o):
        o = host(o).reshape(B, N1 + 1).astype(np.uint64)
        ph = (o[:, N1] - (o[:, :N1] @ s1u)) & 0xFFFFFFFF
        return np.where(ph >= 2 ** 31, ph.astype(np.float64) - 2 ** 32, ph.astype(np.float64))

    p64, p32 = phases(o64), phases(o32)
    sign = np.where(bits == 1, 1.0, -1.0)
    assert np.array_equal((p32 > 0).astype(int), bits)
    assert np.array_equal((p64 > 0).astype(int), bits)
    n64, n32 = p64 - sign * MU, p32 - sign * MU
    ratio = np.var(n32) / np.var(n64)
    assert ratio < 1.25, ratio
    assert abs(np.mean(n32)) < 4 * np.std(n32) / np.sqrt(B)


def test_split32_gates(engine, oracle, keys):
    from cufhedb_b200 import SPLIT32
    _, s1, _ = keys
    B = 96
    rng = np.random.default_rng(41)
    a = rng.integers(0, 2, B); b = rng.integers(0, 2, B)
    enc = lambda bits, base: np.stack([oracle.tlwe32(MU if t else (-MU) & 0xFFFFFFFF, s1, NS_LVL1, SEED, 0x62, base + i)
                                       for i, t in enumerate(bits)])
    ca, cb = enc(a, 0), enc(b, 1000)
    out = empty_dev(B * (N1 + 1))
    engine.gate_lvl1("NAND", dev(ca), dev(cb), out, SPLIT32)
    engine.sync()
    got = np.array([phase(oracle, o, s1) > 0 for o in host(out).reshape(B, N1 + 1)]).astype(int)
    assert np.array_equal(got, 1 - (a & b))


def test_split_key_from_tfhepp_fft_layout(oracle, keys, bkfft01, bk01):
    """Loading TFHEpp's FFT-domain key recovers the integer key exactly (the
    split limbs are derived from it) and gives the same PBS as keygen."""
    from cufhedb_b200 import Engine
    eng = Engine(0)
    eng.load_bkfft_lvl01(bkfft01)
    assert np.array_equal(eng.export_bk_lvl01(), bk01)
    eng.close()


@pytest.mark.parametrize("precision", ["fp64", "split32"])
def test_autotuned_launch_shapes_decrypt(engine, oracle, keys, precision):
    """The autotuner times both launch shapes; batches that land on either
    shape (1,024 -> 7 per CTA, one pass of 8 per CTA on every SM -> 8) still
    decrypt to the gate's truth table."""
    import torch
    from cufhedb_b200 import FP64, SPLIT32
    prec = FP64 if precision == "fp64" else SPLIT32
    ms7, ms8 = engine.autotune_pbs01(prec)
    assert ms7 > 0 and ms8 > 0
    _, s1, _ = keys
    for B in (1024, 8 * engine.num_sms):
        bits = torch.randint(0, 2, (2, B), generator=torch.Generator().manual_seed(B))
        msg = torch.where(bits == 1, MU, -MU).to(torch.int32).cuda()
        ca, cb = empty_dev(B * (N1 + 1)), empty_dev(B * (N1 + 1))
        engine.encrypt_lvl1(SEED, 0x64, 0, msg[0].contiguous(), ca)
        engine.encrypt_lvl1(SEED, 0x64, B, msg[1].contiguous(), cb)
        out = empty_dev(B * (N1 + 1))
        engine.gate_lvl1("AND", ca, cb, out, prec)
        ph = empty_dev(B)
        engine.phase_lvl1(out, ph)
        engine.sync()
        got = (ph > 0).cpu().numpy().astype(int)
        assert np.array_equal(got, (bits[0] & bits[1]).numpy().astype(int))


def test_bounded_wait_expires_reports_and_context_survives(engine, oracle, keys):
    """A key-ring wait that can never complete (no chunk is issued) gives up
    after its poll limit, the failure is reported by cufhedb_sync, and the
    same context then bootstraps correctly."""
    from cufhedb_b200 import _lib
    rc = engine.selftest_wait_timeout(4096)
    assert rc == _lib.ERR_DEVICE
    assert b"bounded wait" in _lib.load().cufhedb_last_error()
    # reported once, then cleared
    engine.sync()
    _, s1, _ = keys
    B = 16
    bits = np.arange(B) % 2
    ca = np.stack([oracle.tlwe32(MU if b else (-MU) & 0xFFFFFFFF, s1, NS_LVL1, SEED, 0x45, i) for i, b in enumerate(bits)])
    cb = np.stack([oracle.tlwe32(MU, s1, NS_LVL1, SEED, 0x46, i) for i in range(B)])
    out = empty_dev(B * (N1 + 1))
    engine.gate_lvl1("NAND", dev(ca), dev(cb), out)
    engine.sync()
    got = host(out).reshape(B, N1 + 1)
    for i in range(B):
        assert (phase(oracle, got[i], s1) > 0) == (not (bits[i] and 1))


@pytest.mark.parametrize("precision", ["fp64", "split32"])
def test_ragged_and_multi_pass_batches(engine, precision):
    """One ciphertext, and a batch of two full passes over every SM plus a
    ragged remainder (the persistent grid loops over groups, the last group
    partly empty): every gate output decrypts to NAND."""
    import torch
    from cufhedb_b200 import FP64, SPLIT32
    prec = FP64 if precision == "fp64" else SPLIT32
    for B in (1, 2 * 7 * engine.num_sms + 5):
        bits = torch.randint(0, 2, (2, B), generator=torch.Generator().manual_seed(B + 7))
        msg = torch.where(bits == 1, MU, -MU).to(torch.int32).cuda()
        ca, cb = empty_dev(B * (N1 + 1)), empty_dev(B * (N1 + 1))
        engine.encrypt_lvl1(SEED, 0x66, 0, msg[0].contiguous(), ca)
        engine.encrypt_lvl1(SEED, 0x66, B, msg[1].contiguous(), cb)
        out = empty_dev(B * (N1 + 1))
        engine.gate_lvl1("NAND", ca, cb, out, prec)
        ph = empty_dev(B)
        engine.phase_lvl1(out, ph)
        engine.sync()
        got = (ph > 0).cpu().numpy().astype(int)
        assert np.array_equal(got, 1 - (bits[0] & bits[1]).numpy().astype(int)), B
