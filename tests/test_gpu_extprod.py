"""GPU parity: batched lvl1 external products against the exact integer
product (oracle) and the reference's TFHEpp trgswfftExternalProduct."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import SEED, signed_diff

from oracle.oracle import L1, N1

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch
    a = np.ascontiguousarray(a)
    v = a.view(np.int32) if a.dtype == np.uint32 else a
    return torch.from_numpy(v.copy()).cuda()


def _case(oracle, keys, B, seed):
    _, s1, _ = keys
    rng = np.random.default_rng(seed)
    trl = rng.integers(0, 2 ** 32, (B, 2, N1), dtype=np.uint64).astype(np.uint32)
    msgs = rng.integers(0, 2, B)
    g = np.stack([oracle.trgsw32(int(m), s1, SEED, 0x33, i) for i, m in enumerate(msgs)])
    return trl, g


@pytest.mark.parametrize("precision", ["fp64", "split32"])
def test_extprod_vs_exact(engine, oracle, keys, precision):
    import torch
    from cufhedb_b200 import FP64, SPLIT32
    prec = FP64 if precision == "fp64" else SPLIT32
    B = 24
    trl, g = _case(oracle, keys, B, 7)
    prep = torch.empty(B * 2 * L1 * 1024 * 2, dtype=torch.float64, device="cuda")
    engine.trgsw_prepare_lvl1(_dev(g), prep, prec)
    out = torch.empty(B * 2 * N1, dtype=torch.int32, device="cuda")
    engine.extprod_lvl1(_dev(trl), prep, out, precision=prec)
    engine.sync()
    got = out.cpu().numpy().view(np.uint32).reshape(B, 2, N1)
    err = np.stack([signed_diff(got[i], oracle.extprod32_exact(trl[i], g[i])) for i in range(B)])
    if prec == FP64:
        assert np.max(np.abs(err)) <= 1
    else:
        # hi limb exact, lo limb FP32: a few thousand torus units, far below the
        # ~2^17.8 standard deviation one external product adds as key noise
        assert np.max(np.abs(err)) < 2 ** 16
        assert np.std(err.astype(np.float64)) < 2 ** 14


def test_extprod_shared_trgsw_and_reference_layout(engine, oracle, ref, keys):
    import torch
    B = 8
    trl, g = _case(oracle, keys, B, 8)
    gfft = oracle.trgsw32_fft(g[0])
    # TFHEpp layout, one TRGSW shared by the batch, host-memory entry point
    got = engine.extprod_lvl1_host(trl, gfft, shared=True)
    for i in range(B):
        want = ref.extprod32(trl[i], gfft)
        assert np.max(np.abs(signed_diff(got[i], want))) <= 1
    # the same through device memory and the TFHEpp-layout preparation
    prep = torch.empty(2 * L1 * 1024 * 2, dtype=torch.float64, device="cuda")
    engine.trgswfft_prepare_lvl1(torch.from_numpy(gfft.copy()).cuda(), prep)
    out = torch.empty(B * 2 * N1, dtype=torch.int32, device="cuda")
    engine.extprod_lvl1(_dev(trl), prep, out, shared=True)
    engine.sync()
    assert np.array_equal(out.cpu().numpy().view(np.uint32).reshape(B, 2, N1), got)
