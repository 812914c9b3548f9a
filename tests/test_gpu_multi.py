"""GPU: row sharding over several contexts (cufhedb_gate_lvl1_host_multi,
cufhedb_compare_host_multi).  Each context owns one device; here two and
three contexts share device 0, which exercises the slicing, the per-shard
host threads and the row-order gather (the kernels of different contexts do
not wait on one another).  The bootstraps are deterministic, so a sharded
call must return exactly what one context returns for the whole column,
including columns shorter than the number of contexts."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import SEED

pytestmark = pytest.mark.gpu
N1, MU = 1024, 1 << 29


@pytest.fixture(scope="module")
def engines():
    from cufhedb_b200 import GEN_BK01, GEN_BK02, GEN_KSK10, GEN_KSK20, GEN_KSK21, Engine
    es = [Engine(0) for _ in range(3)]
    for e in es:
        e.keygen(SEED, GEN_BK01 | GEN_BK02 | GEN_KSK10 | GEN_KSK20 | GEN_KSK21)
    yield es
    for e in es:
        e.close()


@pytest.mark.parametrize("nctx", [2, 3])
def test_sharded_gates_equal_one_context(engines, oracle, keys, nctx):
    from cufhedb_b200 import SPLIT32
    from cufhedb_b200.engine import gate_lvl1_host_multi
    from oracle.oracle import NS_LVL1
    _, s1, _ = keys
    for B in (1, 2, 301):
        rng = np.random.default_rng(B)
        a, b = rng.integers(0, 2, B), rng.integers(0, 2, B)
        enc = lambda bits, base: np.stack([oracle.tlwe32(MU if t else (-MU) & 0xFFFFFFFF, s1, NS_LVL1, SEED, 0xF1,
                                                         base + i) for i, t in enumerate(bits)])
        ca, cb = enc(a, 0), enc(b, B)
        want = engines[0].gate_lvl1_host("AND", ca, cb, SPLIT32)
        got = gate_lvl1_host_multi(engines[:nctx], "AND", ca, cb, SPLIT32)
        assert np.array_equal(got, want), B
        ph = [(int(oracle.phase32(o, s1)) + 2 ** 31) % 2 ** 32 - 2 ** 31 for o in got]
        assert np.array_equal((np.array(ph) > 0).astype(int), a & b)


def test_sharded_lvl2_compare_equals_one_context(engines, oracle, keys):
    from cufhedb_b200 import SPLIT32
    from cufhedb_b200.engine import compare_host, compare_host_multi
    from oracle.oracle import NS_LVL2
    _, s1, s2 = keys
    pb, B = 16, 50
    rng = np.random.default_rng(77)
    x, y = rng.integers(0, 2 ** pb, B), rng.integers(0, 2 ** pb, B)
    enc = lambda v, base: np.stack([oracle.tlwe64(int(t) << (64 - pb - 1), s2, NS_LVL2, SEED, 0xF2, base + i)
                                    for i, t in enumerate(v)])
    c1, c2 = enc(x, 0), enc(y, B)
    want = compare_host(engines[0], "le", 2, c1, c2, pb, True, SPLIT32)
    got = compare_host_multi(engines, "le", 2, c1, c2, pb, True, SPLIT32)
    assert np.array_equal(got, want)
    ph = [(int(oracle.phase32(o, s1)) + 2 ** 31) % 2 ** 32 - 2 ** 31 for o in got]
    assert np.array_equal((np.array(ph) > 0).astype(int), (x <= y).astype(int))
