#!/usr/bin/env python
"""Benchmark: lvl1 gate bootstraps per second on B200 (one process per GPU).

Workload (one step): 1,024 independent lvl1 HomNAND gates over pairs of
uniformly random bits -- per gate one lvl1->lvl0 identity key switch and one
lvl0->lvl1 programmable bootstrap (TFHEpp HomNAND, thirdparty/TFHEpp/src/
gate.cpp:50-65) -- with the reference's default parameters
(params/128bit.hpp: n=672, N=1024, l=3, Bg=2^6, IKS basebit 10, t=2).
Keys and inputs come from the deterministic generator; inputs are encrypted
on the device, so `value` is measured with inputs resident in HBM.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun each rank runs its own 1,024-gate batch on its own GPU
(independent rows: weak scaling, no data-path collective); the reported time
is the max over ranks.  `--impl reference` times the reference's own TFHEpp
CPU HomNAND (oracle/_ref) on this host's cores instead.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SEED = 0x5EED_B200
N0, N1 = 672, 1024
MU = 1 << 29
F1 = 156_893_184            # algorithmic flop per lvl01 PBS (672 CMux x 233,472)
METRIC = "lvl1 PBS/s (HomNAND gate bootstraps: IKS10 + PBS01), 1 B200"
WORKLOAD = ("1,024 lvl1 HomNAND gate bootstraps over uniform random bit pairs, TFHEpp 128-bit "
            "params (n=672, N=1024, l=3, Bg=2^6, IKS10 basebit 10 t 2)")


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--batch", type=int, default=1024)
    p.add_argument("--precision", choices=["fp64", "split32"], default="fp64")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--filter-rows", type=int, default=0,
                   help="also time the encrypted range filter (20-bit lvl2 column, x <= c at the 30th "
                        "percentile) over this many rows and report filter rows/s")
    p.add_argument("--filter-only", action="store_true", help="run only the range-filter measurement")
    p.add_argument("--profile-pbs", action="store_true",
                   help="run only the lvl01 PBS kernel on `--batch` random lvl0 inputs (lvl01 key only, "
                        "~0.1 GB on the device): the small case for ncu captures")
    return p.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", str(rank)))
    return rank, world, local


class ClockSampler:
    """nvidia-smi clock / throttle samples during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.idx = gpu_index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        time.sleep(0.25)
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        rows = []
        with open(self.f.name) as fh:
            for line in fh:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.f.name)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].strip() == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


class CpuReference:
    """The reference's TFHEpp HomNAND (oracle/_ref) on host threads over the
    deterministic key set: keys are set up once, each run() is one bounded
    sample."""

    def __init__(self, nthreads: int):
        from oracle.oracle import Oracle, RefTFHEpp
        self.nthreads = nthreads
        self.o, self.r = Oracle(), RefTFHEpp()
        s0, s1, s2 = self.o.secret_keys(SEED)
        self.s1 = s1
        self.r.set_secret(s0, s1, s2)
        self.r.set_bk01(self.o.bk01(SEED, s0, s1, nthreads))
        ptr, _ = self.r.ksk_view(10)
        self.o.ksk_full_into(10, SEED, (s0, s1, s2), ptr, nthreads)

    def inputs(self, n: int):
        import numpy as np
        from oracle.oracle import NS_LVL1
        bits = np.random.default_rng(7).integers(0, 2, (2, n))
        enc = lambda b, base: np.stack([self.o.tlwe32(MU if t else (-MU) & 0xFFFFFFFF, self.s1, NS_LVL1, SEED, 0x70,
                                                      base + i) for i, t in enumerate(b)])
        return enc(bits[0], 0), enc(bits[1], n)

    def run(self, ca, cb) -> float:
        """gates per second over the given pairs"""
        t0 = time.perf_counter()
        self.r.homnand_batch(ca, cb, self.nthreads)
        return ca.shape[0] / (time.perf_counter() - t0)

    def close(self):
        self.r.close()


def cpu_sample_size(nthreads: int) -> int:
    # ~20 CPU-seconds of TFHEpp HomNAND at ~25 ms per gate, at least 4 per thread
    return max(800, 4 * nthreads)


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    nthreads = os.cpu_count() or 1
    n = cpu_sample_size(nthreads)
    ref = CpuReference(nthreads)
    ca, cb = ref.inputs(n)
    for _ in range(max(1, args.warmup)):
        ref.run(ca[:nthreads], cb[:nthreads])
    rates = [ref.run(ca, cb) for _ in range(args.steps)]
    ref.close()
    value = statistics.median(rates)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "PBS/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * args.batch / value,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "batch": args.batch, "l2": "n/a (host)"},
        "cpu_baseline": {"value": value, "unit": "PBS/s", "cores": nthreads, "kind": "reference",
                         "sample": f"{n} HomNANDs per step on {nthreads} host threads (TFHEpp from oracle/_ref)"},
        "e2e": {"value": value, "unit": "PBS/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args):
    import numpy as np
    import torch

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=180))
    from cufhedb_b200 import FP64, GEN_BK01, GEN_KSK10, SPLIT32, Engine, _lib

    prec = FP64 if args.precision == "fp64" else SPLIT32
    B = args.batch
    eng = Engine(local)
    seed = SEED + rank
    eng.keygen(seed, GEN_BK01 | GEN_KSK10)
    g = torch.Generator().manual_seed(1234 + rank)
    bits = torch.randint(0, 2, (2, B), generator=g)
    msg = np.where(bits.numpy() == 1, MU, (-MU) & 0xFFFFFFFF).astype(np.uint32).view(np.int32)
    msg_d = torch.from_numpy(msg.copy()).cuda()
    ca = torch.empty(B * (N1 + 1), dtype=torch.int32, device="cuda")
    cb = torch.empty_like(ca)
    eng.encrypt_lvl1(seed, 0x70, 0, msg_d[0].contiguous(), ca)
    eng.encrypt_lvl1(seed, 0x70, B, msg_d[1].contiguous(), cb)
    out = torch.empty_like(ca)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream()

    def step():
        eng.gate_lvl1("NAND", ca, cb, out, prec, stream)

    for _ in range(max(3, args.warmup)):
        step()
    eng.sync(stream)

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
        torch.cuda.synchronize()

    clocks = ClockSampler(local)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    barrier()
    clocks.start()
    for e0, e1 in ev:
        flush.zero_()                 # evict L2 between timed steps (untimed)
        e0.record(stream)
        step()
        e1.record(stream)
    barrier()
    clk = clocks.stop()
    eng.sync(stream)
    total_ms = sum(e0.elapsed_time(e1) for e0, e1 in ev)

    # correctness of the last step: decrypt every output with the lvl1 secret key
    _, s1, _ = Engine.secret_keys(seed)
    o = out.cpu().numpy().view(np.uint32).reshape(B, N1 + 1).astype(np.uint64)
    ph = (o[:, N1] - (o[:, :N1] @ s1.astype(np.uint64))) & 0xFFFFFFFF
    dec = (ph.astype(np.int64) - ((ph >= 2 ** 31) * 2 ** 32) > 0).astype(int)
    want = 1 - (bits[0].numpy() & bits[1].numpy())
    errors = int(np.sum(dec != want))

    # dominant kernel alone: the PBS over the key-switched batch
    lvl0 = torch.empty(B * (N0 + 1), dtype=torch.int32, device="cuda")
    from cufhedb_b200 import testvec_const
    eng.iks(10, ca, lvl0)
    tv = testvec_const(MU)
    k_ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(5)]
    for e0, e1 in k_ev:
        flush.zero_()
        e0.record(stream)
        eng.pbs_lvl01(lvl0, out, tv, prec, stream)
        e1.record(stream)
    torch.cuda.synchronize()
    pbs_ms = statistics.median(e0.elapsed_time(e1) for e0, e1 in k_ev)
    iks_ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(5)]
    for e0, e1 in iks_ev:
        flush.zero_()
        e0.record(stream)
        eng.iks(10, ca, lvl0, stream)
        e1.record(stream)
    torch.cuda.synchronize()
    iks_ms = statistics.median(e0.elapsed_time(e1) for e0, e1 in iks_ev)

    # end to end through the C ABI with host buffers: pinned H2D + gate + D2H
    ca_h = ca.cpu().pin_memory()
    cb_h = cb.cpu().pin_memory()
    out_h = torch.empty_like(ca_h).pin_memory()
    ca2, cb2, out2 = torch.empty_like(ca), torch.empty_like(cb), torch.empty_like(out)
    e2e_ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
              for _ in range(args.steps)]
    barrier()
    for e0, e1 in e2e_ev:
        flush.zero_()
        e0.record(stream)
        ca2.copy_(ca_h, non_blocking=True)
        cb2.copy_(cb_h, non_blocking=True)
        eng.gate_lvl1("NAND", ca2, cb2, out2, prec, stream)
        out_h.copy_(out2, non_blocking=True)
        e1.record(stream)
    barrier()
    eng.sync(stream)
    e2e_ms = sum(e0.elapsed_time(e1) for e0, e1 in e2e_ev)

    import ctypes
    pk = ctypes.c_double(0.0)
    _lib.check(eng.lib.cufhedb_measure_fma_peak(local, 1 if prec == FP64 else 0, ctypes.byref(pk)))

    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([total_ms, e2e_ms, float(errors)], device="cuda")
        dist.all_reduce(t[:2], op=dist.ReduceOp.MAX)
        dist.all_reduce(t[2:], op=dist.ReduceOp.SUM)
        total_ms, e2e_ms, errors = float(t[0]), float(t[1]), int(t[2])

    if rank == 0:
        value = world * B * args.steps / (total_ms / 1000.0)
        e2e_value = world * B * args.steps / (e2e_ms / 1000.0)
        achieved = B * F1 / (pbs_ms / 1000.0) / 1e12
        line = {
            "metric": METRIC, "value": value, "unit": "PBS/s", "n_gpus": world, "steps": args.steps,
            "warmup": max(3, args.warmup), "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if prec == FP64 else "f32",
            "data": "synthetic (deterministic keys and encryptions of uniform random bits)",
            "config": {"workload": WORKLOAD, "batch_per_gpu": B, "precision": args.precision,
                       "l2": "flushed (256 MB write, untimed) before every timed step",
                       "parallelism": f"independent rows, {world} GPU(s)"},
            "decrypt_errors": errors,
            "pbs_kernel_ms": pbs_ms, "iks_kernel_ms": iks_ms,
            "roofline": {"bound": "fp64" if prec == FP64 else "fp32", "kernel": "pbs01",
                         "achieved": achieved, "peak": pk.value, "unit": "TFLOP/s",
                         "frac": achieved / pk.value if pk.value else None, "traffic": None,
                         "peak_source": "measured CUDA-core FMA microbenchmark (cufhedb_measure_fma_peak), "
                                        "this GPU, this run",
                         "algorithmic_flop_per_launch": B * F1},
            "gpu_launches": 2 * args.steps,
            "clocks": clk,
            "e2e": {"value": e2e_value, "unit": "PBS/s",
                    "h2d_bytes_per_step": 2 * B * (N1 + 1) * 4, "d2h_bytes_per_step": B * (N1 + 1) * 4},
        }
        if world == 1 and not args.no_cpu_baseline:
            try:
                nthreads = os.cpu_count() or 1
                n = cpu_sample_size(nthreads)
                c_a = ca.cpu().numpy().view(np.uint32).reshape(B, N1 + 1)
                c_b = cb.cpu().numpy().view(np.uint32).reshape(B, N1 + 1)
                reps = -(-n // B)
                c_a, c_b = np.tile(c_a, (reps, 1))[:n], np.tile(c_b, (reps, 1))[:n]
                cref = CpuReference(nthreads)
                cref.run(c_a[:nthreads], c_b[:nthreads])
                rate = cref.run(c_a, c_b)
                cref.close()
                line["cpu_baseline"] = {"value": rate, "unit": "PBS/s", "cores": nthreads, "kind": "reference",
                                        "sample": f"{n} HomNANDs (TFHEpp from oracle/_ref) on {nthreads} host threads"}
            except Exception as exc:  # the GPU number stands without it
                line["cpu_baseline"] = {"value": None, "unit": "PBS/s", "cores": None, "kind": "reference",
                                        "sample": f"unavailable: {exc}"}
        print(json.dumps(line), flush=True)
    eng.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def range_filter(eng, rows: int, precision: int, steps: int = 1):
    """Encrypted range filter x <= c over a synthetic 20-bit column at lvl2
    (the reference's HomComp / TPC-H filter shape: less_than_equal<Lvl2>, 6 lvl02
    + 3 lvl01 bootstraps and 10 key switches per row).  Returns (rows/s, ms per
    pass, decrypt errors, bootstraps per row)."""
    import numpy as np
    import torch
    from cufhedb_b200 import Engine
    pb = 20
    g = torch.Generator().manual_seed(77)
    x = torch.randint(0, 2 ** pb, (rows,), generator=g).numpy().astype(np.uint64)
    c = int(np.percentile(x, 30))
    shift = np.uint64(64 - pb - 1)
    msg = torch.from_numpy((x << shift).view(np.int64)).cuda()
    thr = torch.from_numpy((np.full(rows, c, np.uint64) << shift).view(np.int64)).cuda()
    c1 = torch.empty(rows * 2049, dtype=torch.int64, device="cuda")
    c2 = torch.empty_like(c1)
    eng.encrypt_lvl2(SEED, 0x7A, 0, msg, c1)
    eng.encrypt_lvl2(SEED, 0x7A, rows, thr, c2)
    out = torch.empty(rows * (N1 + 1), dtype=torch.int32, device="cuda")
    eng.compare("le", 2, c1, c2, out, pb, True, precision)   # warm-up (and pool growth)
    eng.sync()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    for e0, e1 in ev:
        e0.record()
        eng.compare("le", 2, c1, c2, out, pb, True, precision)
        e1.record()
    eng.sync()
    ms = statistics.median(e0.elapsed_time(e1) for e0, e1 in ev)
    _, s1, _ = Engine.secret_keys(SEED)
    o = out.cpu().numpy().view(np.uint32).reshape(rows, N1 + 1).astype(np.uint64)
    ph = (o[:, N1] - (o[:, :N1] @ s1.astype(np.uint64))) & 0xFFFFFFFF
    dec = ((ph > 0) & (ph < 2 ** 31)).astype(int)
    errors = int(np.sum(dec != (x <= c).astype(int)))
    return rows / (ms / 1000.0), ms, errors


def run_filter_only(args):
    from cufhedb_b200 import FP64, GEN_ALL, SPLIT32, Engine
    prec = FP64 if args.precision == "fp64" else SPLIT32
    eng = Engine(0)
    eng.keygen(SEED, GEN_ALL)
    rows = args.filter_rows or 16384
    rate, ms, errors = range_filter(eng, rows, prec, max(1, args.steps))
    print(json.dumps({"workload": "range filter x <= c, 20-bit lvl2 column", "rows": rows,
                      "precision": args.precision, "rows_per_s": rate, "ms": ms, "decrypt_errors": errors,
                      "pbs_per_row": {"lvl02": 6, "lvl01": 3}}))
    eng.close()


def run_profile_pbs(args):
    """--steps launches of the PBS kernel alone, no key-switching key."""
    import torch
    from cufhedb_b200 import FP64, GEN_BK01, SPLIT32, Engine, testvec_const
    prec = FP64 if args.precision == "fp64" else SPLIT32
    eng = Engine(0)
    eng.keygen(SEED, GEN_BK01)
    g = torch.Generator(device="cuda").manual_seed(99)
    x = torch.randint(-2 ** 31, 2 ** 31, (args.batch * (N0 + 1),), generator=g, device="cuda", dtype=torch.int64)
    x = x.to(torch.int32)
    out = torch.empty(args.batch * (N1 + 1), dtype=torch.int32, device="cuda")
    tv = testvec_const(MU)
    for _ in range(args.warmup):
        eng.pbs_lvl01(x, out, tv, prec)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    for e0, e1 in ev:
        e0.record()
        eng.pbs_lvl01(x, out, tv, prec)
        e1.record()
    eng.sync()
    ms = [e0.elapsed_time(e1) for e0, e1 in ev]
    print(json.dumps({"profile": "pbs01", "batch": args.batch, "precision": args.precision,
                      "ms": ms, "pbs_per_s": args.batch / (statistics.median(ms) / 1000.0) if ms else None}))
    eng.close()


def main():
    args = parse()
    if args.profile_pbs:
        run_profile_pbs(args)
    elif args.filter_only:
        run_filter_only(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
