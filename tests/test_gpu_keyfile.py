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


def test_cereal_archives_load_into_a_context(ref_keyed, oracle, keys, bk01, tmp_path):
    """The reference's cereal key archives (src/HEDB/utils/serialize.cpp) load
    into a fresh context: the lvl01 bootstrapping key recovers the integer key
    exactly, and with the lvl10 key-switching key from its archive the
    context's gates decrypt."""
    import torch
    from cufhedb_b200 import Engine
    from oracle.oracle import N1, NS_LVL1
    s0, s1, _ = keys
    p_bk = str(tmp_path / "bkfftlvl01.key")
    ref_keyed.save_cereal("bkfft01", p_bk)
    ptr, _ = ref_keyed.ksk_view(10)
    oracle.ksk_full_into(10, SEED, keys, ptr)
    p_ks = str(tmp_path / "iksklvl10.key")
    ref_keyed.save_cereal("ksk10", p_ks)
    eng = Engine(0)
    eng.load_cereal_key(p_bk, "bkfft01")
    eng.load_cereal_key(p_ks, "ksk10")
    os.unlink(p_ks)
    assert np.array_equal(eng.export_bk_lvl01(), bk01)
    B = 32
    rng = np.random.default_rng(8)
    a, b = rng.integers(0, 2, B), rng.integers(0, 2, B)
    enc = lambda bits, base: np.stack([oracle.tlwe32((1 << 29) if t else (-(1 << 29)) & 0xFFFFFFFF, s1, NS_LVL1,
                                                     SEED, 0xE1, base + i) for i, t in enumerate(bits)])
    out = eng.gate_lvl1_host("NAND", enc(a, 0), enc(b, B))
    ph = [(int(oracle.phase32(o, s1)) + 2 ** 31) % 2 ** 32 - 2 ** 31 for o in out]
    assert np.array_equal((np.array(ph) > 0).astype(int), 1 - (a & b))
    eng.close()
