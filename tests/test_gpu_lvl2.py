"""GPU parity: the lvl2 ring (N = 2048, 64-bit torus) -- transforms, external
products, PBS02, and the lvl2 -> lvl0 / lvl2 -> lvl1 key switches -- against
the oracle and the reference's TFHEpp."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import SEED, fill_ref_ksk, signed_diff

from oracle.oracle import L2, N0, N1, N2, NS_LVL0, NS_LVL2

pytestmark = pytest.mark.gpu
MU2 = 1 << 61


def _dev(a):
    import torch
    a = np.ascontiguousarray(a)
    v = a.view(np.int64) if a.dtype == np.uint64 else a.view(np.int32) if a.dtype == np.uint32 else a
    return torch.from_numpy(v.copy()).cuda()


def _maxabs64(d):
    return max(abs(int(x)) for x in np.asarray(d).ravel())


@pytest.fixture(scope="module")
def engine2():
    from cufhedb_b200 import GEN_BK02, GEN_KSK20, GEN_KSK21, Engine
    eng = Engine(0)
    eng.keygen(SEED, GEN_BK02 | GEN_KSK20 | GEN_KSK21)
    yield eng
    eng.close()


@pytest.fixture(scope="module")
def bk02(oracle, keys):
    s0, _, s2 = keys
    return oracle.bk02(SEED, s0, s2)


def test_keygen_lvl2_matches_oracle(engine2, bk02, oracle, keys):
    assert np.array_equal(engine2.export_bk_lvl02(), bk02)
    for kind, rows in ((20, [0, 4_000_000, 2048 * 2 * 1023 - 1]), (21, [0, 77_777, 2048 * 10 * 7 - 1])):
        got = engine2.export_ksk_rows(kind, np.array(rows, np.uint64))
        per = 2 * 1023 if kind == 20 else 70
        dig = 1023 if kind == 20 else 7
        for q, row in zip(rows, got):
            assert np.array_equal(oracle.ksk_row(kind, SEED, keys, q // per, (q % per) // dig, q % dig), row)


def test_twist_transforms_lvl2(engine2, ref):
    import torch
    rng = np.random.default_rng(51)
    B = 9
    a = rng.integers(0, 2 ** 64, (B, N2), dtype=np.uint64)
    out = torch.empty(B * N2, dtype=torch.float64, device="cuda")
    engine2.twist_ifft_lvl2(_dev(a), out)
    engine2.sync()
    got = out.cpu().numpy().reshape(B, N2)
    want = np.stack([ref.twist_ifft64(x) for x in a])
    assert np.max(np.abs(got - want)) <= 1e-13 * np.max(np.abs(want))
    back = torch.empty(B * N2, dtype=torch.int64, device="cuda")
    engine2.twist_fft_lvl2(torch.from_numpy(want.copy()).cuda(), back)
    engine2.sync()
    back = back.cpu().numpy().view(np.uint64).reshape(B, N2)
    for i in range(B):
        assert _maxabs64(signed_diff(back[i], ref.twist_fft64(want[i]), 64)) <= 2 ** 14
        assert _maxabs64(signed_diff(back[i], a[i], 64)) <= 2 ** 14


def test_extprod_lvl2_vs_exact_and_reference(engine2, oracle, ref, keys):
    import torch
    _, _, s2 = keys
    rng = np.random.default_rng(52)
    B = 4
    trl = rng.integers(0, 2 ** 64, (B, 2, N2), dtype=np.uint64)
    g = np.stack([oracle.trgsw64(int(m), s2, SEED, 0x34, i) for i, m in enumerate(rng.integers(0, 2, B))])
    prep = torch.empty(B * 2 * L2 * 2 * 1024 * 2, dtype=torch.float64, device="cuda")
    engine2.trgsw_prepare_lvl2(_dev(g), prep)
    out = torch.empty(B * 2 * N2, dtype=torch.int64, device="cuda")
    engine2.extprod_lvl2(_dev(trl), prep, out)
    engine2.sync()
    got = out.cpu().numpy().view(np.uint64).reshape(B, 2, N2)
    for i in range(B):
        exact = oracle.extprod64_exact(trl[i], g[i])
        theirs = ref.extprod64(trl[i], oracle.trgsw64_fft(g[i]))
        # FP64 keeps ~53 of 64 bits: both the reference and this path are
        # within a few 2^24 of the exact product, far below the lvl2 message
        assert _maxabs64(signed_diff(got[i], exact, 64)) < 2 ** 30
        assert _maxabs64(signed_diff(theirs, exact, 64)) < 2 ** 30


def test_pbs02_trivial_inputs_exact(engine2, oracle):
    from cufhedb_b200 import testvec_const
    B = 5
    x = np.zeros((B, N0 + 1), np.uint32)
    x[:, N0] = np.array([0, 1, (1 << 20) - 1, 0x80000000, 0xFFFFFFFF], np.uint32)
    import torch
    out = torch.empty(B * (N2 + 1), dtype=torch.int64, device="cuda")
    engine2.pbs_lvl02(_dev(x), out, testvec_const(MU2))
    engine2.sync()
    got = out.cpu().numpy().view(np.uint64).reshape(B, N2 + 1)
    dummy = np.zeros((N0, 2 * L2, 2, N2), np.float64)
    tv = np.full(N2, MU2, np.uint64)
    for xi, o in zip(x, got):
        assert np.array_equal(oracle.pbs02(xi, dummy, tv), o)


def test_pbs02_decrypts_like_reference(engine2, oracle, ref, keys, bk02):
    from cufhedb_b200 import testvec_const
    import torch
    s0, s1, s2 = keys
    ref.set_secret(s0, s1, s2)
    ref.set_bk02(bk02)
    B = 12
    bits = np.random.default_rng(53).integers(0, 2, B)
    mu0 = 1 << 29
    x = np.stack([oracle.tlwe32(mu0 if b else (-mu0) & 0xFFFFFFFF, s0, NS_LVL0, SEED, 0x53, i)
                  for i, b in enumerate(bits)])
    out = torch.empty(B * (N2 + 1), dtype=torch.int64, device="cuda")
    engine2.pbs_lvl02(_dev(x), out, testvec_const(MU2))
    engine2.sync()
    got = out.cpu().numpy().view(np.uint64).reshape(B, N2 + 1)
    tv = np.full(N2, MU2, np.uint64)
    for i in range(B):
        pg = int(signed_diff(oracle.phase64(got[i], s2), 0, 64))
        assert (pg > 0) == bool(bits[i])
        assert abs(abs(pg) - MU2) < 2 ** 56
        if i < 3:
            pr = int(signed_diff(oracle.phase64(ref.pbs02(x[i], tv), s2), 0, 64))
            assert (pr > 0) == (pg > 0) and abs(pr - pg) < 2 ** 56


@pytest.mark.parametrize("kind", [20, 21])
def test_iks_from_lvl2_bit_exact(engine2, oracle, keys, kind):
    import torch
    _, _, s2 = keys
    B = 6
    xs = np.stack([oracle.tlwe64((i % 8) << 61, s2, NS_LVL2, SEED, 0x42, i) for i in range(B)])
    xs[0, :] = 0
    width = N0 + 1 if kind == 20 else N1 + 1
    out = torch.empty(B * width, dtype=torch.int32, device="cuda")
    engine2.iks(kind, _dev(xs), out)
    engine2.sync()
    got = out.cpu().numpy().view(np.uint32).reshape(B, width)
    for x, o in zip(xs, got):
        assert np.array_equal(oracle.iks(kind, x, SEED, keys), o)


def test_iks21_key_stationary_batch_equals_gather(engine2, oracle, keys):
    """Batches of 512 and more take the key-stationary lvl2 -> lvl1 switch; on
    600 ciphertexts (a ragged third tile of 256) it gives bit for bit what
    the per-ciphertext gather gives on the same inputs in batches of 8, and
    sampled rows equal the oracle's key switch."""
    import torch
    _, _, s2 = keys
    B, width = 600, N1 + 1
    rng = np.random.default_rng(71)
    xs = rng.integers(0, 2 ** 64, (B, N2 + 1), dtype=np.uint64)
    xs[0, :] = 0
    xs[1, :N2] = 0
    x_d = _dev(xs).reshape(-1)
    big = torch.empty(B * width, dtype=torch.int32, device="cuda")
    engine2.iks(21, x_d, big)
    small = torch.empty_like(big)
    per = N2 + 1
    for b0 in range(0, B, 8):
        engine2.iks(21, x_d[b0 * per:(b0 + 8) * per], small[b0 * width:(b0 + 8) * width])
    engine2.sync()
    assert torch.equal(big, small)
    got = big.cpu().numpy().view(np.uint32).reshape(B, width)
    for i in (0, 1, 2, 255, 256, 511, 512, B - 1):
        assert np.array_equal(oracle.iks(21, xs[i], SEED, keys), got[i]), i


def test_host_ksk21_loads_into_the_padded_device_layout(engine2, oracle, keys):
    """A whole lvl21 key-switching key handed over as a host array in TFHEpp's
    packed row layout (cufhedb_load_ksk) lands in the device layout (rows
    padded to 16-byte multiples): the rows read back equal the host rows and
    the key switch of the loaded key equals the one of the generated key."""
    import torch
    from cufhedb_b200 import Engine
    _, _, s2 = keys
    rows, width = 2048 * 10 * 7, N1 + 1
    host = np.zeros(rows * width, np.uint32)
    oracle.ksk_full_into(21, SEED, keys, host.ctypes.data)
    eng = Engine(0)
    eng.load_ksk(21, host)
    q = np.array([0, 1, 2, 3, 70_001, rows - 1], np.uint64)
    got = eng.export_ksk_rows(21, q)
    host = host.reshape(rows, width)
    for r, row in zip(q, got):
        assert np.array_equal(host[int(r)], row)
    del host
    B = 5
    xs = np.stack([oracle.tlwe64((i % 8) << 61, s2, NS_LVL2, SEED, 0x43, i) for i in range(B)])
    o1 = torch.empty(B * width, dtype=torch.int32, device="cuda")
    o2 = torch.empty_like(o1)
    engine2.iks(21, _dev(xs), o1)
    eng.iks(21, _dev(xs), o2)
    engine2.sync()
    eng.sync()
    assert torch.equal(o1, o2)
    eng.close()


def test_pbs02_ragged_multi_pass_batch(engine2, oracle, keys):
    """Two full passes of three ciphertexts per SM plus a ragged remainder of
    two: every output decrypts to its input bit at +-mu."""
    from cufhedb_b200 import testvec_const
    import torch
    s0, _, _ = keys
    B = 2 * 3 * engine2.num_sms + 2
    bits = np.random.default_rng(54).integers(0, 2, B)
    mu0 = 1 << 29
    x = np.stack([oracle.tlwe32(mu0 if b else (-mu0) & 0xFFFFFFFF, s0, NS_LVL0, SEED, 0x54, i)
                  for i, b in enumerate(bits)])
    out = torch.empty(B * (N2 + 1), dtype=torch.int64, device="cuda")
    engine2.pbs_lvl02(_dev(x), out, testvec_const(MU2))
    ph = torch.empty(B, dtype=torch.int64, device="cuda")
    engine2.phase_lvl2(out, ph)
    engine2.sync()
    p = ph.cpu().numpy()
    assert np.array_equal((p > 0).astype(int), bits)
    assert np.max(np.abs(np.abs(p.astype(np.float64)) - MU2)) < 2.0 ** 56


def test_misaligned_buffers_are_refused(engine2):
    """A 64-bit torus buffer that does not start on an 8-byte boundary is
    refused with CUFHEDB_ERR_ARG before anything is enqueued (a misaligned
    word access would be a device fault)."""
    import torch
    from cufhedb_b200 import CufhedbError, testvec_const
    x = torch.zeros(2 * (N0 + 1), dtype=torch.int32, device="cuda")
    raw = torch.zeros(2 * (N2 + 1) + 1, dtype=torch.int64, device="cuda")
    odd = raw.view(torch.int32)[1:1 + 2 * 2 * (N2 + 1)]       # starts 4 bytes into the buffer
    import ctypes
    from cufhedb_b200 import _lib
    tv = testvec_const(1 << 61)
    rc = engine2.lib.cufhedb_pbs_lvl02(engine2.ctx, x.data_ptr(), odd.data_ptr(), 2, ctypes.byref(tv), None)
    assert rc == _lib.ERR_ARG and b"8-byte aligned" in _lib.load().cufhedb_last_error()
    rc = engine2.lib.cufhedb_iks(engine2.ctx, 20, odd.data_ptr(), x.data_ptr(), 1, None)
    assert rc == _lib.ERR_ARG
    engine2.sync()
