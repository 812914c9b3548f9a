"""CPU: the native queue scheduler's plan (cufhedb_queue_plan, host only) --
queries that share a comparison chain are packed into batches of at most
max_batch_rows rows, smallest first; batches run in order of estimated cost
per completed query (Smith's rule); each batch goes to the stream with the
least estimated work queued.  The rules are restated here from the chain
lengths the operator layer runs (msb_gpu.cuh / HomCompare_gpu.cuh chains)."""
from __future__ import annotations

import numpy as np
import pytest

T01, T02 = 9.4 / 1036, 17.7 / 444   # ms per ciphertext of a full pass, lvl01 / lvl02


def _chain(level, op, pb, logic):
    """(lvl01, lvl02) bootstraps per row of cufhedb_compare's chain"""
    p = pb + 1
    if level == 1:
        n01, n02 = (1 if p <= 5 else 3 if p <= 9 else 5), 0
    elif p <= 9:
        n01, n02 = (1 if p <= 5 else 3), 0
    else:
        levels, q = 1, p
        while q > 14:
            levels, q = levels + 1, q - 5
        n01, n02 = 3, 2 * levels
    if op == "eq":
        return 2 * n01 + 1, 2 * n02
    if op in ("ge", "le") and not logic:
        n01 += 1
    return n01, n02


def _cost(q):
    op, level, rows, pb, logic = q
    n01, n02 = _chain(level, op, pb, logic)
    return rows * (n01 * T01 + n02 * T02)


def _queue(seed=11, n=64):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        width = int(rng.choice([8, 16, 24, 32]))
        rows = int(np.exp(rng.uniform(np.log(2 ** 8), np.log(2 ** 16))))
        out.append(("le", 1 if width == 8 else 2, rows, width, True))
    return out


def test_plan_rules_on_an_uneven_queue():
    from cufhedb_b200.engine import queue_plan
    qs = _queue()
    cap = 16384
    batch_of, stream_of = queue_plan(qs, T01, T02, max_batch_rows=cap, nstreams=2)
    nb = len(stream_of)
    assert sorted(set(batch_of)) == list(range(nb))
    members = [[i for i, b in enumerate(batch_of) if b == k] for k in range(nb)]
    key = lambda q: (q[1], q[0], q[3], q[4])
    for m in members:
        # one chain per batch; over the row cap only as a single query
        assert len({key(qs[i]) for i in m}) == 1
        rows = sum(qs[i][2] for i in m)
        assert rows <= cap or len(m) == 1
    # smallest first within a chain: a batch never holds a query cheaper than
    # one of an earlier-opened batch of the same chain that it could have joined
    # (packing in ascending cost order fills batches with consecutive queries)
    for k in {key(q) for q in qs}:
        chain = sorted((i for i, q in enumerate(qs) if key(q) == k), key=lambda i: (_cost(qs[i]), i))
        seen, last = [], None
        for i in chain:
            if batch_of[i] != last:
                assert batch_of[i] not in seen
                seen.append(batch_of[i])
                last = batch_of[i]
    # run order: ascending cost per completed query
    per = [sum(_cost(qs[i]) for i in m) / len(m) for m in members]
    assert all(per[k] <= per[k + 1] * (1 + 1e-12) for k in range(nb - 1))
    # list scheduling on the estimated work of each stream
    busy = [0.0, 0.0]
    for k in range(nb):
        s = int(np.argmin(busy))
        assert stream_of[k] == s
        busy[s] += sum(_cost(qs[i]) for i in members[k])


def test_plan_edge_cases():
    from cufhedb_b200 import CufhedbError
    from cufhedb_b200.engine import queue_plan
    assert queue_plan([], T01, T02) == ([], [])
    # one query above the row cap is a batch of its own
    b, s = queue_plan([("lt", 2, 70000, 20, True), ("lt", 2, 10, 20, True)], T01, T02, max_batch_rows=65536)
    assert b[0] != b[1] and len(s) == 2
    # different chains never share a batch, even when tiny
    b, _ = queue_plan([("lt", 2, 5, 20, True), ("le", 2, 5, 20, True), ("lt", 2, 5, 24, True),
                       ("lt", 2, 5, 20, False), ("lt", 1, 5, 6, True)], T01, T02)
    assert len(set(b)) == 5
    # the same chain merges up to the cap
    b, _ = queue_plan([("eq", 1, 100, 6, True)] * 5, T01, T02, max_batch_rows=300)
    assert sorted(np.bincount(b).tolist()) == [2, 3]
    for bad in ([("lt", 3, 5, 20, True)], [("lt", 2, -1, 20, True)], [("lt", 2, 5, 0, True)]):
        with pytest.raises(CufhedbError):
            queue_plan(bad, T01, T02)
    with pytest.raises(CufhedbError):
        queue_plan([("lt", 2, 5, 20, True)], T01, T02, nstreams=0)
    with pytest.raises(CufhedbError):
        queue_plan([("lt", 2, 5, 20, True)], 0.0, T02)
