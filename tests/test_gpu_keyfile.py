"""GPU: key files in the reference's raw layout (test/HE3_Query/fastR.h:
secret key, BootstrappingKeyFFT<lvl01param>, KeySwitchingKey<lvl10param>) --
a context that loads a saved file computes bit-identical gates."""
from __future__ import annotations

import os

import numpy as np
import pytest

from conftest import SEED

pytestmark = pytest.mark.gpu
N1, N0 = 1024, 672
MU = 1 << 29


def test_keyfile_round_trip_gives_identical_gates(tmp_path):
    import torch
    from cufhedb_b200 import FP64, GEN_BK01, GEN_KSK10, SPLIT32, Engine
    path = str(tmp_path / "key.bin")
    a = Engine(0)
    a.keygen(SEED, GEN_BK01 | GEN_KSK10)
    a.save_keyfile(path)
    expect = 1024 * 4 + 672 * 6 * 2 * 1024 * 8 + 1024 * 2 * 1023 * 673 * 4
    assert os.path.getsize(path) == expect
    _, s1, _ = Engine.secret_keys(SEED)
    b = Engine(0)
    sk = b.load_keyfile(path)
    os.remove(path)
    assert np.array_equal(sk, s1)
    B = 64
    bits = torch.randint(0, 2, (2, B), generator=torch.Generator().manual_seed(9))
    msg = torch.where(bits == 1, MU, -MU).to(torch.int32).cuda()
    ca = torch.empty(B * (N1 + 1), dtype=torch.int32, device="cuda")
    cb = torch.empty_like(ca)
    a.encrypt_lvl1(SEED, 0x66, 0, msg[0].contiguous(), ca)
    a.encrypt_lvl1(SEED, 0x66, B, msg[1].contiguous(), cb)
    for prec in (FP64, SPLIT32):
        oa, ob = torch.empty_like(ca), torch.empty_like(ca)
        a.gate_lvl1("NAND", ca, cb, oa, prec)
        b.gate_lvl1("NAND", ca, cb, ob, prec)
        a.sync()
        b.sync()
        assert torch.equal(oa, ob)
    a.close()
    b.close()


def test_keyfile_rejects_wrong_size(tmp_path):
    from cufhedb_b200 import CufhedbError, Engine
    path = tmp_path / "short.bin"
    path.write_bytes(b"\\0" * 4096)
    e = Engine(0)
    with pytest.raises(CufhedbError) as err:
        e.load_keyfile(str(path))
    assert err.value.code == 1
    e.close()
