"""GPU: the allocation-free gate entry point (cufhedb_gate_lvl1_noalloc).

It exists for callers that cannot let a library allocate device memory while
they run (an engine that reserves all device memory at start-up, or a host
whose allocator owns the device).  Through the C ABI, two calls in a row must
give exactly what the allocating entry point (cufhedb_gate_lvl1) gives on the
same inputs -- the second call with a smaller batch, so nothing left in the
shared intermediate from the first call can leak into it --, a call must
leave free device memory and the stream-ordered pool's used bytes unchanged
and the caller's current device as it was, and a batch above the 1,024-gate
limit must be refused.

This file is collected last so that a run that stops at the first failure has
already run every other test; it also passes on its own in a fresh process.
"""
from __future__ import annotations

import ctypes

import numpy as np
import pytest

from conftest import SEED

pytestmark = pytest.mark.gpu
N1, MU = 1024, 1 << 29
POOL_USED_MEM_CURRENT = 7   # cudaMemPoolAttrUsedMemCurrent


def _pairs(engine, B, base):
    import torch
    g = torch.Generator().manual_seed(base)
    bits = torch.randint(0, 2, (2, B), generator=g).numpy()
    msg = np.where(bits == 1, MU, (-MU) & 0xFFFFFFFF).astype(np.uint32).view(np.int32)
    msg_d = torch.from_numpy(msg.copy()).cuda()
    ca = torch.empty(B * (N1 + 1), dtype=torch.int32, device="cuda")
    cb = torch.empty_like(ca)
    engine.encrypt_lvl1(SEED, 0x90, base, msg_d[0].contiguous(), ca)
    engine.encrypt_lvl1(SEED, 0x90, base + B, msg_d[1].contiguous(), cb)
    return ca, cb, bits


def _device_memory_state(device: int):
    """(free device bytes, used bytes of the device's default stream-ordered pool)"""
    rt = ctypes.CDLL("libcudart.so.12")
    free, total = ctypes.c_size_t(0), ctypes.c_size_t(0)
    assert rt.cudaMemGetInfo(ctypes.byref(free), ctypes.byref(total)) == 0
    pool = ctypes.c_void_p(0)
    assert rt.cudaDeviceGetDefaultMemPool(ctypes.byref(pool), device) == 0
    used = ctypes.c_uint64(0)
    assert rt.cudaMemPoolGetAttribute(pool, POOL_USED_MEM_CURRENT, ctypes.byref(used)) == 0
    return free.value, used.value


def test_noalloc_gate_matches_allocating_entry_point(engine):
    import torch
    _, s1, _ = engine.secret_keys(SEED)
    cases = [(B, base, gate) + _pairs(engine, B, base) for B, base, gate in ((1000, 0, "NAND"), (37, 5000, "AND"))]
    wants = []
    for B, _, gate, ca, cb, _ in cases:
        want = torch.zeros_like(ca)
        engine.gate_lvl1(gate, ca, cb, want)
        wants.append(want)
    gots = [torch.full_like(c[3], -1) for c in cases]
    engine.sync()
    torch.cuda.synchronize()
    before = _device_memory_state(torch.cuda.current_device())
    for (B, _, gate, ca, cb, _), got in zip(cases, gots):
        engine.gate_lvl1_noalloc(gate, ca, cb, got)
    engine.sync()
    torch.cuda.synchronize()
    assert _device_memory_state(torch.cuda.current_device()) == before
    for (B, _, gate, ca, cb, bits), want, got in zip(cases, wants, gots):
        assert torch.equal(got, want)
        o = got.cpu().numpy().view(np.uint32).reshape(B, N1 + 1).astype(np.uint64)
        ph = (o[:, N1] - (o[:, :N1] @ s1.astype(np.uint64))) & 0xFFFFFFFF
        dec = ((ph > 0) & (ph < 2 ** 31)).astype(int)
        truth = 1 - (bits[0] & bits[1]) if gate == "NAND" else bits[0] & bits[1]
        assert np.array_equal(dec, truth)
    assert torch.cuda.current_device() == 0


def test_noalloc_gate_rejects_batches_above_limit(engine):
    import torch
    from cufhedb_b200 import CufhedbError
    ca = torch.zeros(1025 * (N1 + 1), dtype=torch.int32, device="cuda")
    with pytest.raises(CufhedbError) as e:
        engine.gate_lvl1_noalloc("NAND", ca, ca, ca)
    assert e.value.code == 1 and "1024" in str(e.value)
