"""GPU: the query shapes on the batched operator layer -- the filter +
grouped aggregate (3 range predicates, 3 x 2 groups, SUM and COUNT after
decryption, DAG replayed as a CUDA graph) and an uneven queue of filter
queries, run by the native scheduler and as width groups -- against
plaintext evaluation."""
from __future__ import annotations

import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng_q():
    from cufhedb_b200 import GEN_ALL, Engine
    from conftest import SEED
    eng = Engine(0)
    eng.keygen(SEED, GEN_ALL)
    yield eng
    eng.close()


@pytest.mark.parametrize("precision", ["split32", "fp64"])
def test_filter_group_aggregate_matches_plaintext(eng_q, precision):
    from cufhedb_b200 import FP64, SPLIT32
    from cufhedb_b200.queries import filter_group_aggregate
    r = filter_group_aggregate(eng_q, 96, SPLIT32 if precision == "split32" else FP64, steps=2)
    assert r["aggregates_match"], r
    assert r["count_errors"] == 0


def test_uneven_queue_packed_by_width(eng_q):
    from cufhedb_b200 import SPLIT32
    from cufhedb_b200.queries import run_queue
    queries = [(20, 8), (33, 16), (7, 8), (12, 24), (9, 32), (16, 16)]
    r = run_queue(eng_q, queries, SPLIT32, mode="width_groups")
    assert r["decrypt_errors"] == 0, r
    assert r["rows"] == sum(n for n, _ in queries)
    assert r["width_groups"] == {8: 27, 16: 49, 24: 12, 32: 9}


@pytest.mark.parametrize("max_batch_rows,nstreams", [(16384, 2), (24, 3), (1, 1)])
def test_uneven_queue_native_scheduler(eng_q, max_batch_rows, nstreams):
    """Every query decrypts bit-exact whether the scheduler packs queries into
    shared batches (gather / scatter through staging), splits them into
    single-query batches (batch cap below every query) or runs them on one
    stream; each query has its own latency, no later than the whole queue."""
    from cufhedb_b200 import SPLIT32
    from cufhedb_b200.queries import run_queue
    queries = [(20, 8), (33, 16), (7, 8), (12, 24), (9, 32), (16, 16), (5, 8), (40, 16), (3, 32)]
    r = run_queue(eng_q, queries, SPLIT32, mode="scheduled", max_batch_rows=max_batch_rows, nstreams=nstreams)
    assert r["decrypt_errors"] == 0, r
    assert r["rows"] == sum(n for n, _ in queries)
    lat = r["latency_ms"]
    assert 0 < lat["min"] <= lat["median"] <= lat["max"] <= r["ms"] + 1e-3
