"""Encrypted query shapes on the batched operator layer.

The reference runs its TPC-H style queries as OpenMP row loops that call one
cuHEDB operator per row (test/HE3_Query/TPCH_Q6.cu:158-209,
TPCH_Q1.cu:246-262): compare each column against an encrypted constant,
combine the predicate bits with HomAND, build group masks, decrypt the
bitmap, and aggregate in plaintext (the CKKS aggregation path is compiled out,
TPCH_Q6.cu:424).  Here every operator runs over a whole column in one batched
call, and the operator DAG of a query can be captured once as a CUDA graph and
replayed.

* ``filter_group_aggregate`` -- a conjunction of three range predicates over
  a synthetic lineitem-like table (a 16-bit day-number date at lvl2, a 4-bit
  discount and a 6-bit quantity at lvl1), split into 3 x 2 groups by a
  3-valued flag and a 2-valued status, then SUM(price * (1 - discount)) and
  COUNT per group after decryption.
* ``run_queue`` -- many filter queries of uneven row counts and widths, run by
  the engine's native queue scheduler (cufhedb_queue_run: smallest queries
  first, queries of one comparison chain packed into shared batches, batches
  on two streams), or, for comparison, as one batch per width run back to
  back.

Decryption for the checks uses the deterministic key set (``Engine.keygen``).
"""
from __future__ import annotations

import numpy as np

from .engine import N1, N2, Engine

LVL1_MAX_BITS = 9   # compare adds a sign bit; lvl1 HomMSB handles up to 10 (msb_gpu.cuh:57-62)


def _level(bits: int) -> int:
    return 1 if bits <= LVL1_MAX_BITS else 2


def encrypt_column(eng: Engine, values, bits: int, seed: int, stream_id: int, idx0: int, level: int | None = None):
    """values (< 2^bits) encrypted as HEDB's tlweSymInt32Encrypt does (message
    v * 2^(w - bits - 1), src/HEDB/comparison/tfhepp_utils.h:15-30), at lvl1
    for widths up to 9 bits, else at lvl2.  Returns a device tensor."""
    import torch
    level = level or _level(bits)
    v = np.ascontiguousarray(values, np.uint64)
    if level == 1:
        msg = torch.from_numpy((v << np.uint64(32 - bits - 1)).astype(np.uint32).view(np.int32)).cuda()
        out = torch.empty(v.size * (N1 + 1), dtype=torch.int32, device="cuda")
        eng.encrypt_lvl1(seed, stream_id, idx0, msg, out)
    else:
        msg = torch.from_numpy((v << np.uint64(64 - bits - 1)).view(np.int64)).cuda()
        out = torch.empty(v.size * (N2 + 1), dtype=torch.int64, device="cuda")
        eng.encrypt_lvl2(seed, stream_id, idx0, msg, out)
    return out


def decrypt_bits(eng: Engine, ct_lvl1, rows: int) -> np.ndarray:
    """LOGIC lvl1 results -> 0/1 (phase > 0), with the deterministic key set"""
    import torch
    ph = torch.empty(rows, dtype=torch.int32, device="cuda")
    eng.phase_lvl1(ct_lvl1, ph)
    eng.sync()
    return (ph > 0).cpu().numpy().astype(np.int64)


def synthetic_lineitem(rows: int, seed: int = 2026):
    """Synthetic table with the reference generators' shapes
    (TPCH_Q6.cu:41-74, TPCH_Q1.cu:50-82): day-number dates uniform over seven
    years, discount 0..10 (percent), quantity 1..50, price a 24-bit fixed-point
    value log-uniform over [1, 2^24), a 3-valued flag and a 2-valued status."""
    rng = np.random.default_rng(seed)
    return {
        "date": rng.integers(0, 7 * 365, rows).astype(np.uint64),
        "discount": rng.integers(0, 11, rows).astype(np.uint64),
        "quantity": rng.integers(1, 51, rows).astype(np.uint64),
        "price": np.exp(rng.uniform(0.0, np.log(2.0 ** 24 - 1), rows)).astype(np.uint64),
        "flag": rng.integers(0, 3, rows).astype(np.uint64),
        "status": rng.integers(0, 2, rows).astype(np.uint64),
    }


# predicate constants: date in [D0, D1), discount in [5, 7], quantity < 24
D0, D1 = 365, 2 * 365
WIDTH = {"date": 16, "discount": 4, "quantity": 6, "flag": 2, "status": 1}


def plaintext_filter_group_aggregate(t):
    pred = (t["date"] >= D0) & (t["date"] < D1) & (t["discount"] >= 5) & (t["discount"] <= 7) & (t["quantity"] < 24)
    out = {}
    for f in range(3):
        for s in range(2):
            m = pred & (t["flag"] == f) & (t["status"] == s)
            rev = (t["price"][m].astype(np.int64) * (100 - t["discount"][m].astype(np.int64))).sum()
            out[(f, s)] = (int(m.sum()), int(rev))
    return out


class FilterGroupAggregate:
    """The encrypted DAG of one filter + group query over a whole table: 5
    comparisons against encrypted constants, 5 equality tests for the group
    keys, and 13 HomANDs, every one a batched call over all rows."""

    def __init__(self, eng: Engine, table: dict, precision: int, seed: int = 0x5EED_B200):
        import torch
        self.eng, self.precision, self.rows = eng, precision, len(table["date"])
        n = self.rows
        self.cols = {k: encrypt_column(eng, table[k], WIDTH[k], seed, 0xA0 + i, 0)
                     for i, k in enumerate(WIDTH)}
        const = lambda v, k, sid: encrypt_column(eng, np.full(n, v, np.uint64), WIDTH[k], seed, sid, 0)
        self.consts = {"d0": const(D0, "date", 0xB0), "d1": const(D1, "date", 0xB1),
                       "c5": const(5, "discount", 0xB2), "c7": const(7, "discount", 0xB3),
                       "q24": const(24, "quantity", 0xB4)}
        self.consts.update({f"f{f}": const(f, "flag", 0xB8 + f) for f in range(3)})
        self.consts.update({f"s{s}": const(s, "status", 0xBC + s) for s in range(2)})
        mk = lambda: torch.empty(n * (N1 + 1), dtype=torch.int32, device="cuda")
        self.tmp = [mk() for _ in range(6)]
        self.flag_eq = [mk() for _ in range(3)]
        self.status_eq = [mk() for _ in range(2)]
        self.masks = {(f, s): mk() for f in range(3) for s in range(2)}
        self.graph = None
        eng.sync()   # the encryptions ran on the current stream; the DAG may run on another

    def enqueue(self, stream=None):
        e, p, c, k, tmp = self.eng, self.precision, self.cols, self.consts, self.tmp
        cmp = lambda op, col, const, out: e.compare(op, 2 if col == "date" else 1, c[col], k[const], out,
                                                    WIDTH[col], True, p, stream)
        cmp("ge", "date", "d0", tmp[0])
        cmp("lt", "date", "d1", tmp[1])
        cmp("ge", "discount", "c5", tmp[2])
        cmp("le", "discount", "c7", tmp[3])
        cmp("lt", "quantity", "q24", tmp[4])
        e.hom_and(tmp[0], tmp[1], tmp[5], True, p, stream)
        e.hom_and(tmp[5], tmp[2], tmp[0], True, p, stream)
        e.hom_and(tmp[0], tmp[3], tmp[1], True, p, stream)
        e.hom_and(tmp[1], tmp[4], tmp[5], True, p, stream)          # tmp[5] = predicate
        for f in range(3):
            cmp("eq", "flag", f"f{f}", self.flag_eq[f])
        for s in range(2):
            cmp("eq", "status", f"s{s}", self.status_eq[s])
        for f in range(3):
            e.hom_and(tmp[5], self.flag_eq[f], tmp[f], True, p, stream)
            for s in range(2):
                e.hom_and(tmp[f], self.status_eq[s], self.masks[(f, s)], True, p, stream)

    def capture(self, stream):
        """record the whole DAG as one CUDA graph on `stream` (non-default)"""
        self.eng.graph_begin(stream)
        self.enqueue(stream)
        self.graph = self.eng.graph_end(stream)

    def replay(self, stream):
        self.eng.graph_launch(self.graph, stream)

    def close(self):
        if self.graph is not None:
            self.eng.graph_destroy(self.graph)
            self.graph = None

    def results(self, table) -> dict:
        """decrypt the six group masks and aggregate in plaintext, as the
        reference's GPU queries do after decryption (TPCH_Q6.cu:146-156)"""
        out = {}
        price = table["price"].astype(np.int64)
        disc = table["discount"].astype(np.int64)
        for key, m in self.masks.items():
            bits = decrypt_bits(self.eng, m, self.rows).astype(bool)
            out[key] = (int(bits.sum()), int((price[bits] * (100 - disc[bits])).sum()))
        return out


def filter_group_aggregate(eng: Engine, rows: int, precision: int, steps: int = 1, seed: int = 2026):
    """Build, capture and time the query; returns a result dict with rows/s,
    the mask decrypt errors and whether every group's SUM and COUNT match the
    plaintext evaluation."""
    import torch
    table = synthetic_lineitem(rows, seed)
    q = FilterGroupAggregate(eng, table, precision)
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        q.enqueue(stream)                 # warm-up (pool growth) outside the graph
        eng.sync(stream)
        q.capture(stream)
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        for e0, e1 in ev:
            e0.record(stream)
            q.replay(stream)
            e1.record(stream)
        eng.sync(stream)
    ms = min(e0.elapsed_time(e1) for e0, e1 in ev)
    got = q.results(table)
    want = plaintext_filter_group_aggregate(table)
    q.close()
    return {"rows": rows, "ms": ms, "rows_per_s": rows / (ms / 1000.0), "groups": len(want),
            "aggregates_match": got == want,
            "count_errors": int(sum(abs(got[k][0] - want[k][0]) for k in want)),
            "selected_rows": int(sum(v[0] for v in want.values())),
            "bootstraps_per_row": {"lvl02": 8, "lvl01": 39}}


def run_queue(eng: Engine, queries: list, precision: int, seed: int = 0x5EED_B200, mode: str = "scheduled",
              max_batch_rows: int = 16384, nstreams: int = 2):
    """Uneven queue of filter queries x <= c.  `queries` is a list of
    (rows, bits).  mode "scheduled": the native scheduler (cufhedb_queue_run)
    with each query's own ciphertexts; mode "width_groups": queries of equal
    width concatenated and each width's chain run once, the widths back to
    back.  Returns per-query latency (completion from the start of the
    queue), aggregate rows/s and decrypt errors."""
    import torch
    rng = np.random.default_rng(seed)
    data = []
    for qi, (rows, bits) in enumerate(queries):
        x = rng.integers(0, 2 ** bits, rows).astype(np.uint64)
        c = int(rng.integers(0, 2 ** bits))
        data.append((x, c, bits))
    total_rows = sum(r for r, _ in queries)
    latency = [0.0] * len(queries)
    errors = 0
    if mode == "scheduled":
        cts = []
        for qi, (x, c, bits) in enumerate(data):
            c1 = encrypt_column(eng, x, bits, seed, 0xC0 + bits, 1_000_000 * qi)
            c2 = encrypt_column(eng, np.full(x.size, c, np.uint64), bits, seed, 0xD0 + bits, 1_000_000 * qi)
            out = torch.empty(x.size * (N1 + 1), dtype=torch.int32, device="cuda")
            cts.append(("le", _level(bits), c1, c2, out, bits, True))
        eng.sync()
        latency, total_ms = eng.queue_run(cts, precision, max_batch_rows, nstreams)
        for (x, c, bits), q in zip(data, cts):
            errors += int(np.sum(decrypt_bits(eng, q[4], x.size) != (x <= c).astype(np.int64)))
        extra = {"scheduler": {"max_batch_rows": max_batch_rows, "streams": nstreams}}
    else:
        widths = sorted({b for _, b in queries})
        groups = {}
        for w in widths:
            idx = [i for i, (_, _, b) in enumerate(data) if b == w]
            xs = np.concatenate([data[i][0] for i in idx])
            cs = np.concatenate([np.full(data[i][0].size, data[i][1], np.uint64) for i in idx])
            c1 = encrypt_column(eng, xs, w, seed, 0xC0 + w, 0)
            c2 = encrypt_column(eng, cs, w, seed, 0xD0 + w, 0)
            out = torch.empty(xs.size * (N1 + 1), dtype=torch.int32, device="cuda")
            groups[w] = (idx, xs, cs, c1, c2, out)
        eng.sync()
        stream = torch.cuda.current_stream()
        start = torch.cuda.Event(enable_timing=True)
        done = {w: torch.cuda.Event(enable_timing=True) for w in widths}
        start.record(stream)
        for w in widths:
            idx, xs, cs, c1, c2, out = groups[w]
            eng.compare("le", _level(w), c1, c2, out, w, True, precision, stream)
            done[w].record(stream)
        eng.sync(stream)
        for w in widths:
            idx, xs, cs, c1, c2, out = groups[w]
            t = start.elapsed_time(done[w])
            for i in idx:
                latency[i] = t
            errors += int(np.sum(decrypt_bits(eng, out, xs.size) != (xs <= cs).astype(np.int64)))
        total_ms = max(start.elapsed_time(done[w]) for w in widths)
        extra = {"width_groups": {int(w): int(groups[w][1].size) for w in widths}}
    return {"queries": len(queries), "rows": total_rows, "ms": total_ms, "mode": mode,
            "rows_per_s": total_rows / (total_ms / 1000.0), "decrypt_errors": errors,
            "latency_ms": {"min": min(latency), "median": float(np.median(latency)), "max": max(latency),
                           "mean": float(np.mean(latency))}, **extra}
