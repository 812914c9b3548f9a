#!/usr/bin/env python
"""Benchmark: lvl1 bootstraps per second on B200, split-FP32 vs FP64 path,
plus encrypted-filter rows per second (one process per GPU).

Gate workload (one step): 1,024 independent lvl1 HomNAND gates over pairs of
uniformly random bits -- per gate one lvl1->lvl0 identity key switch and one
lvl0->lvl1 programmable bootstrap (TFHEpp HomNAND, thirdparty/TFHEpp/src/
gate.cpp:50-65) -- with the reference's default parameters
(params/128bit.hpp: n=672, N=1024, l=3, Bg=2^6, IKS basebit 10, t=2).  Keys
and inputs come from the deterministic generator; inputs are encrypted on the
device, so `value` is measured with inputs resident in HBM.  `value` is the
split-precision path; the same steps are timed on the FP64 path (`fp64`).

Filter workload (1 GPU): the 20-bit range filter x <= c at the 30th
percentile over 16,384 rows encrypted at lvl2 (less_than_equal<Lvl2>, 6 lvl02
+ 3 lvl01 bootstraps and 10 key switches per row).  Error-rate workload (1
GPU): HomNAND over fresh encryptions on both paths, every output decrypted.

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
N0, N1, N2 = 672, 1024, 2048
MU = 1 << 29
F1 = 156_893_184            # algorithmic flop per lvl01 PBS (672 CMux x 233,472)
F2 = 432_144_384            # algorithmic flop per lvl02 PBS (672 CMux x 643,072)
METRIC = "lvl1 PBS/s, 1 B200: split-FP32 vs FP64 path at 0 decrypt errors; filter rows/s"
WORKLOAD = ("1,024 lvl1 HomNAND gate bootstraps (IKS10 + PBS01 each) over uniform random bit pairs, "
            "TFHEpp 128-bit params (n=672, N=1024, l=3, Bg=2^6, IKS10 basebit 10 t 2)")
# DRAM bytes (read + write) of one 1,024-ciphertext PBS launch, from the ncu
# captures summarised under profiles/ (pbs01_*_batch1024.md)
TRAFFIC = {"split32": 68_939_264 + 3_732_480, "fp64": 69_385_472 + 3_819_008}


def parse(argv=None):
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--batch", type=int, default=1024)
    p.add_argument("--precision", choices=["fp64", "split32", "split32tc"], default="split32",
                   help="headline path (the other one is timed alongside)")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--filter-rows", type=int, default=16384,
                   help="rows of the encrypted range filter timed at N=1 (0: skip)")
    p.add_argument("--noise-samples", type=int, default=2048,
                   help="lvl01 bootstraps compared with the FP64 (TFHEpp) and exact CPU oracles at N=1 (0: skip)")
    p.add_argument("--error-bootstraps", type=int, default=1048576,
                   help="HomNAND bootstraps per path decrypted for the error rate at N=1 (0: skip)")
    p.add_argument("--filter-only", action="store_true", help="run only the range-filter measurement")
    p.add_argument("--error-only", action="store_true", help="run only the error-rate / noise measurement")
    p.add_argument("--extprod", action="store_true",
                   help="external-product microbenchmark: 4,096 products at lvl1 (both paths) and lvl2")
    p.add_argument("--profile-pbs", action="store_true",
                   help="run only the PBS kernel on `--batch` random lvl0 inputs (bootstrapping key only, "
                        "a few hundred MB on the device): the small case for ncu captures")
    p.add_argument("--level", type=int, choices=[1, 2], default=1, help="PBS level for --profile-pbs")
    p.add_argument("--agg-leg-rows", type=int, default=65536,
                   help="rows of the filter + grouped aggregate query timed at N=1 beside the gate steps (0: skip)")
    p.add_argument("--agg-rows", type=int, default=0,
                   help="run only the filter + grouped aggregate query (3 range predicates, 6 groups) over this "
                        "many rows, its operator DAG captured as one CUDA graph")
    p.add_argument("--queue", type=int, default=0,
                   help="run only a queue of this many filter queries, rows log-uniform in [2^8, --queue-max-rows], "
                        "widths uniform in {8, 16, 24, 32}")
    p.add_argument("--queue-max-rows", type=int, default=65536)
    p.add_argument("--queue-mode", choices=["scheduled", "width_groups"], default="scheduled",
                   help="native queue scheduler, or one batch per width run back to back")
    p.add_argument("--arc-rows", type=int, default=0,
                   help="run only the ArcEDB comparison measurement over this many rows")
    p.add_argument("--arc-digits", type=int, default=2, help="radix-1024 digits per value for --arc-rows")
    p.add_argument("--profile-iks", type=int, choices=[10, 20, 21], default=0,
                   help="run only the identity key switch of this kind on `--batch` random inputs (its key only)")
    return p.parse_args(argv)


def tensor_peak():
    """(dense bf16 tensor-core TFLOP/s of this pool's B200s, source): the
    measured burst figure of MEASURED_PEAKS.json when present, else the
    earlier measurement on this pool (1,590 TFLOP/s)."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            return float(json.load(fh)["bf16_tflops"]), "measured (MEASURED_PEAKS.json bf16_tflops, burst)"
    except Exception:
        return 1590.0, "fallback (earlier measurement on this pool)"


def _prec(name: str) -> int:
    from cufhedb_b200 import FP64, SPLIT32, SPLIT32_TC
    return {"fp64": FP64, "split32": SPLIT32, "split32tc": SPLIT32_TC}[name]


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", str(rank)))
    return rank, world, local


def reduce_over_ranks(max_vals, sum_vals, device):
    """Max of the timings and sum of the counters over all ranks (identity
    without a process group).  Works on gloo (CPU tensors) and nccl."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return list(max_vals), list(sum_vals)
    t = torch.tensor(list(max_vals) + list(sum_vals), dtype=torch.float64, device=device)
    m = t[:len(max_vals)].clone()
    s = t[len(max_vals):].clone()
    dist.all_reduce(m, op=dist.ReduceOp.MAX)
    dist.all_reduce(s, op=dist.ReduceOp.SUM)
    return [float(x) for x in m], [float(x) for x in s]


def whole_job_rate(world: int, units_per_rank: int, steps: int, max_total_ms: float) -> float:
    """units per second over all ranks, timed by the slowest rank"""
    return world * units_per_rank * steps / (max_total_ms / 1000.0)


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
    """The reference's TFHEpp / HEDB CPU code (oracle/_ref) on host threads
    over the deterministic key set: keys are set up once, each run() is one
    bounded sample."""

    def __init__(self, nthreads: int):
        from oracle.oracle import Oracle, RefTFHEpp
        self.nthreads = nthreads
        self.o, self.r = Oracle(), RefTFHEpp()
        self.keys = self.o.secret_keys(SEED)
        s0, s1, s2 = self.keys
        self.s1 = s1
        self.r.set_secret(s0, s1, s2)
        self.bk01 = self.o.bk01(SEED, s0, s1, nthreads)
        self.r.set_bk01(self.bk01)
        ptr, _ = self.r.ksk_view(10)
        self.o.ksk_full_into(10, SEED, self.keys, ptr, nthreads)
        self.lvl2 = False

    def load_lvl2(self):
        """the lvl02 bootstrapping key and the lvl20 / lvl21 key-switching keys
        (the HEDB lvl2 comparison chains need them)"""
        if self.lvl2:
            return
        s0, _, s2 = self.keys
        self.r.set_bk02(self.o.bk02(SEED, s0, s2, self.nthreads))
        for kind in (20, 21):
            ptr, _ = self.r.ksk_view(kind)
            self.o.ksk_full_into(kind, SEED, self.keys, ptr, self.nthreads)
        self.lvl2 = True

    def inputs(self, n: int):
        import numpy as np
        from oracle.oracle import NS_LVL1
        bits = np.random.default_rng(7).integers(0, 2, (2, n))
        enc = lambda b, base: np.stack([self.o.tlwe32(MU if t else (-MU) & 0xFFFFFFFF, self.s1, NS_LVL1, SEED, 0x70,
                                                      base + i) for i, t in enumerate(b)])
        return enc(bits[0], 0), enc(bits[1], n)

    def run(self, ca, cb, nthreads: int | None = None) -> float:
        """HomNANDs per second over the given pairs"""
        t0 = time.perf_counter()
        self.r.homnand_batch(ca, cb, nthreads or self.nthreads)
        return ca.shape[0] / (time.perf_counter() - t0)

    def close(self):
        self.r.close()


def run_reference(args):
    """The reference's own TFHEpp HomNAND (oracle/_ref) on all host threads:
    each step is one batch of the workload (--batch gates, 1,024 by default),
    timed by the host clock."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    nthreads = os.cpu_count() or 1
    n = args.batch
    ref = CpuReference(nthreads)
    ca, cb = ref.inputs(n)
    for _ in range(max(1, args.warmup)):
        ref.run(ca, cb)
    step_ms = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        ref.r.homnand_batch(ca, cb, nthreads)
        step_ms.append(1000.0 * (time.perf_counter() - t0))
    ref.close()
    total_ms = sum(step_ms)
    value = n * args.steps / (total_ms / 1000.0)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "PBS/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "batch_per_gpu": n, "precision": "fp64 (TFHEpp spqlios FFT)",
                   "l2": "n/a (host)", "parallelism": f"{nthreads} host threads, row-parallel"},
        "cpu_baseline": {"value": value, "unit": "PBS/s", "cores": nthreads, "kind": "reference",
                         "sample": f"{n} HomNANDs per step (the whole batch) on {nthreads} host threads "
                                   "(TFHEpp from oracle/_ref)"},
        "e2e": {"value": value, "unit": "PBS/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def _events(n):
    import torch
    return [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(n)]


def _timed(fn, steps, flush, stream):
    """CUDA-event time (ms) of each of `steps` calls of fn, L2 flushed (untimed) before each"""
    ev = _events(steps)
    for e0, e1 in ev:
        flush.zero_()
        e0.record(stream)
        fn()
        e1.record(stream)
    stream.synchronize()
    return [e0.elapsed_time(e1) for e0, e1 in ev]


def _timed_sync_call(fn, steps, flush, stream):
    """time (ms) of each of `steps` synchronous host calls, L2 flushed (untimed,
    finished) before each; CUDA events on the idle stream bracket the call"""
    ev = _events(steps)
    for e0, e1 in ev:
        flush.zero_()
        stream.synchronize()
        e0.record(stream)
        fn()
        e1.record(stream)
    stream.synchronize()
    return [e0.elapsed_time(e1) for e0, e1 in ev]


def _gate_errors(eng, out, want_bits, stream):
    """decrypt every HomNAND output on the device: (errors, noise sum, noise sum of squares)"""
    import torch
    B = want_bits.numel()
    ph = torch.empty(B, dtype=torch.int32, device="cuda")
    eng.phase_lvl1(out, ph, stream=stream)
    sign = (ph > 0).to(torch.int64)
    errors = int((sign != want_bits).sum())
    noise = ph.to(torch.float64) - torch.where(want_bits == 1, float(MU), float(-MU)).to(torch.float64)
    return errors, float(noise.sum()), float((noise * noise).sum())


def error_rate(eng, nboot: int, stream, chunk: int = 8192):
    """HomNAND over fresh encryptions on both paths, same inputs; every output
    decrypted.  Returns per path: bootstraps, decrypt errors, output noise
    variance (torus units^2 of 2^32), and the split / fp64 variance ratio."""
    import torch
    from cufhedb_b200 import FP64, SPLIT32
    g = torch.Generator(device="cuda").manual_seed(4242)
    ca = torch.empty(chunk * (N1 + 1), dtype=torch.int32, device="cuda")
    cb = torch.empty_like(ca)
    out = torch.empty_like(ca)
    res = {p: {"bootstraps": 0, "errors": 0, "s1": 0.0, "s2": 0.0} for p in ("split32", "fp64")}
    done = 0
    while done < nboot:
        B = min(chunk, nboot - done)
        bits = torch.randint(0, 2, (2, B), generator=g, device="cuda")
        msg = torch.where(bits == 1, MU, -MU).to(torch.int32)
        eng.encrypt_lvl1(SEED, 0x7E, 2 * done, msg[0].contiguous(), ca[:B * (N1 + 1)], stream)
        eng.encrypt_lvl1(SEED, 0x7E, 2 * done + B, msg[1].contiguous(), cb[:B * (N1 + 1)], stream)
        want = (1 - bits[0] * bits[1]).to(torch.int64)
        for name, prec in (("split32", SPLIT32), ("fp64", FP64)):
            eng.gate_lvl1("NAND", ca[:B * (N1 + 1)], cb[:B * (N1 + 1)], out[:B * (N1 + 1)], prec, stream)
            e, s1, s2 = _gate_errors(eng, out[:B * (N1 + 1)], want, stream)
            r = res[name]
            r["bootstraps"] += B
            r["errors"] += e
            r["s1"] += s1
            r["s2"] += s2
        done += B
    outd = {}
    for name, r in res.items():
        n = r["bootstraps"]
        mean = r["s1"] / n
        outd[name] = {"bootstraps": n, "decrypt_errors": r["errors"], "noise_var": r["s2"] / n - mean * mean,
                      "noise_mean": mean}
    outd["split_over_fp64_noise_var"] = outd["split32"]["noise_var"] / outd["fp64"]["noise_var"]
    return outd


def noise_vs_oracles(eng, cref, n: int, stream):
    """Per-bootstrap output noise of the GPU lvl01 PBS on both paths against
    two CPU oracles, on the same keys and lvl0 inputs: the reference's own
    TFHEpp GateBootstrappingTLWE2TLWEFFT<lvl01param> (FP64 FFT) and the exact
    integer PBS (orc_pbs01_exact_batch: every negacyclic product exact).
    Inputs are HomNAND gate inputs of fresh encryptions, key-switched on the
    GPU (bit-exact with TFHEpp's IdentityKeySwitch).  Reported per path
    (split32, fp64 on the GPU; tfhepp on the CPU): the output noise variance
    (phase minus the encoded +-mu, torus units of 2^-32), its ratio to the
    exact oracle's, the variance and largest size of the phase difference from
    each oracle, and decryption errors."""
    import numpy as np
    import torch
    from cufhedb_b200 import FP64, SPLIT32, testvec_const
    rng = np.random.default_rng(4343)
    bits = rng.integers(0, 2, (2, n))
    s1 = cref.s1
    from oracle.oracle import NS_LVL1
    enc = lambda b, base: np.stack([cref.o.tlwe32(MU if t else (-MU) & 0xFFFFFFFF, s1, NS_LVL1, SEED, 0x7F, base + i)
                                    for i, t in enumerate(b)])
    ca, cb = enc(bits[0], 0), enc(bits[1], n)
    x = ((0 - ca.astype(np.uint64) - cb.astype(np.uint64)) & 0xFFFFFFFF).astype(np.uint32)
    x[:, N1] = (x[:, N1].astype(np.uint64) + MU).astype(np.uint32)   # HomNAND: (0, mu) - ca - cb
    xd = torch.from_numpy(x.view(np.int32).copy()).cuda()
    lvl0 = torch.empty(n * (N0 + 1), dtype=torch.int32, device="cuda")
    eng.iks(10, xd, lvl0, stream)
    outs = {}
    for name, prec in (("split32", SPLIT32), ("fp64", FP64)):
        o = torch.empty(n * (N1 + 1), dtype=torch.int32, device="cuda")
        eng.pbs_lvl01(lvl0, o, testvec_const(MU), prec, stream)
        outs[name] = o
    stream.synchronize()
    eng.sync(stream)
    l0h = lvl0.cpu().numpy().view(np.uint32).reshape(n, N0 + 1)
    tv = np.full(N1, MU, np.uint32)
    t0 = time.perf_counter()
    outs_h = {k: v.cpu().numpy().view(np.uint32).reshape(n, N1 + 1) for k, v in outs.items()}
    outs_h["tfhepp"] = cref.r.pbs01_batch(l0h, tv, cref.nthreads)
    t_ref = time.perf_counter() - t0
    prep = cref.o.bk01_exact_prepare(cref.bk01)
    t0 = time.perf_counter()
    exact, max_dev = cref.o.pbs01_exact_batch(l0h, prep, tv, cref.nthreads)
    t_exact = time.perf_counter() - t0
    s1u = s1.astype(np.uint64)

    def phase(c):
        c = c.astype(np.uint64)
        p = (c[:, N1] - (c[:, :N1] @ s1u)) & 0xFFFFFFFF
        return np.where(p >= 2 ** 31, p.astype(np.float64) - 2 ** 32, p.astype(np.float64))

    want = 1 - (bits[0] & bits[1])
    expect = np.where(want == 1, float(MU), float(-MU))
    p_exact = phase(exact)
    p_ref = phase(outs_h["tfhepp"])
    res = {"samples": n, "workload": "HomNAND inputs key-switched on the GPU, lvl01 PBS with mu = 2^29",
           "exact": {"noise_var": float(np.var(p_exact - expect)), "decrypt_errors": int(np.sum((p_exact > 0) != want)),
                     "max_fft_rounding_distance": max_dev, "cpu_s": t_exact,
                     "oracle": "orc_pbs01_exact_batch (16-bit key limbs, FP64 FFT, every product rounded to its "
                               "integer; equal to the schoolbook product)"},
           "tfhepp_cpu_s": t_ref, "threads": cref.nthreads}
    for name in ("split32", "fp64", "tfhepp"):
        p = phase(outs_h[name])
        nv = float(np.var(p - expect))
        res[name] = {"noise_var": nv, "noise_var_over_exact": nv / res["exact"]["noise_var"],
                     "decrypt_errors": int(np.sum((p > 0) != want)),
                     "diff_vs_exact": {"var": float(np.var(p - p_exact)), "max_abs": float(np.max(np.abs(p - p_exact)))}}
        if name != "tfhepp":
            res[name]["noise_var_over_tfhepp"] = nv / float(np.var(p_ref - expect))
            res[name]["diff_vs_tfhepp"] = {"var": float(np.var(p - p_ref)), "max_abs": float(np.max(np.abs(p - p_ref)))}
    return res


def range_filter(eng, rows: int, precision: int, steps: int = 1):
    """Encrypted range filter x <= c over a synthetic 20-bit column at lvl2
    (the reference's HomComp / TPC-H filter shape: less_than_equal<Lvl2>, 6 lvl02
    + 3 lvl01 bootstraps and 10 key switches per row).  Returns (rows/s, ms per
    pass, decrypt errors)."""
    import numpy as np
    import torch
    pb = 20
    g = torch.Generator().manual_seed(77)
    x = torch.randint(0, 2 ** pb, (rows,), generator=g).numpy().astype(np.uint64)
    c = int(np.percentile(x, 30))
    shift = np.uint64(64 - pb - 1)
    msg = torch.from_numpy((x << shift).view(np.int64)).cuda()
    thr = torch.from_numpy((np.full(rows, c, np.uint64) << shift).view(np.int64)).cuda()
    c1 = torch.empty(rows * (N2 + 1), dtype=torch.int64, device="cuda")
    c2 = torch.empty_like(c1)
    eng.encrypt_lvl2(SEED, 0x7A, 0, msg, c1)
    eng.encrypt_lvl2(SEED, 0x7A, rows, thr, c2)
    out = torch.empty(rows * (N1 + 1), dtype=torch.int32, device="cuda")
    eng.compare("le", 2, c1, c2, out, pb, True, precision)   # warm-up (and pool growth)
    eng.sync()
    ev = _events(steps)
    for e0, e1 in ev:
        e0.record()
        eng.compare("le", 2, c1, c2, out, pb, True, precision)
        e1.record()
    eng.sync()
    ms = statistics.median(e0.elapsed_time(e1) for e0, e1 in ev)
    ph = torch.empty(rows, dtype=torch.int32, device="cuda")
    eng.phase_lvl1(out, ph)
    got = (ph > 0).cpu().numpy().astype(int)
    errors = int(np.sum(got != (x <= c).astype(int)))
    return rows / (ms / 1000.0), ms, errors, (c1, c2, x, c)


def filter_cpu_baseline(cref, c1, c2, x, c, rows: int):
    """The reference's HEDB less_than_equal<Lvl2> (src/HEDB/comparison/
    HomCompare.h:55-66) on all host threads over the first `rows` rows of the
    filter's own ciphertexts: (rows/s, decrypt errors)."""
    import numpy as np
    cref.load_lvl2()
    a = c1[:rows * (N2 + 1)].cpu().numpy().view(np.uint64).reshape(rows, N2 + 1)
    b = c2[:rows * (N2 + 1)].cpu().numpy().view(np.uint64).reshape(rows, N2 + 1)
    t0 = time.perf_counter()
    out = cref.r.compare_batch(2, a, b, 3, 20, True, cref.nthreads)
    rate = rows / (time.perf_counter() - t0)
    s1u = cref.s1.astype(np.uint64)
    o = out.astype(np.uint64)
    ph = (o[:, N1] - (o[:, :N1] @ s1u)) & 0xFFFFFFFF
    got = ((ph > 0) & (ph < 2 ** 31)).astype(int)
    return rate, int(np.sum(got != (x[:rows] <= c).astype(int)))


def run_ours(args):
    import numpy as np
    import torch

    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=180))
    from cufhedb_b200 import FP64, GEN_ALL, GEN_BK01, GEN_KSK10, SPLIT32, SPLIT32_TC, Engine, _lib, testvec_const

    head = args.precision
    other = "fp64" if head != "fp64" else "split32"
    PREC = {"fp64": FP64, "split32": SPLIT32, "split32tc": SPLIT32_TC}
    B = args.batch
    single = world == 1
    eng = Engine(local)
    seed = SEED + rank
    eng.keygen(seed, GEN_ALL if (single and args.filter_rows) else GEN_BK01 | GEN_KSK10)
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
    want = (1 - bits[0] * bits[1]).to(torch.int64).cuda()
    W = max(3, args.warmup)

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
        torch.cuda.synchronize()

    # ---- launch-shape autotuning (untimed): one full pass of every shape ----------
    tuned = eng.autotune(levels=(1, 2) if (single and args.filter_rows) else (1,))
    tune = {f"pbs01_{name}": {"pass_ms_by_shape": tuned[f"pbs01_{name}"],
                              "ciphertexts_per_cta": eng.launch_shape(1, PREC[name], B)}
            for name in ("split32", "fp64", "split32tc")}
    tune["pbs01_split32"]["stage1_layout"] = eng.launch_layout(B)   # chosen over both split tables
    if single and args.filter_rows:
        tune["pbs02"] = {"pass_ms_by_shape": tuned["pbs02"],
                         "ciphertexts_per_cta_filter": eng.launch_shape(2, FP64, args.filter_rows)}

    # ---- the timed gate steps, headline path then the other path ----------------
    res = {}
    clk = None
    for name in (head, other):
        prec = PREC[name]
        step = lambda: eng.gate_lvl1("NAND", ca, cb, out, prec, stream)
        for _ in range(W):
            step()
        barrier()
        clocks = ClockSampler(local) if name == head else None
        if clocks:
            clocks.start()
        ms = _timed(step, args.steps, flush, stream)
        barrier()
        if clocks:
            clk = clocks.stop()
        errors, _, _ = _gate_errors(eng, out, want, stream)
        res[name] = {"total_ms": sum(ms), "errors": errors}

    # ---- dominant kernel alone: the PBS over the key-switched batch -------------
    lvl0 = torch.empty(B * (N0 + 1), dtype=torch.int32, device="cuda")
    eng.iks(10, ca, lvl0)
    tv = testvec_const(MU)
    for name in (head, other):
        prec = PREC[name]
        res[name]["pbs_ms"] = statistics.median(
            _timed(lambda: eng.pbs_lvl01(lvl0, out, tv, prec, stream), 5, flush, stream))
    iks_ms = statistics.median(_timed(lambda: eng.iks(10, ca, lvl0, stream), 5, flush, stream))
    # the split path with its first transform step on the tensor cores, kernel alone
    tc_name = "split32tc" if head != "split32tc" else "split32"
    tc_ms = statistics.median(_timed(lambda: eng.pbs_lvl01(lvl0, out, tv, PREC[tc_name], stream), 5, flush, stream))
    eng.gate_lvl1("NAND", ca, cb, out, PREC[tc_name], stream)
    tc_errors, _, _ = _gate_errors(eng, out, want, stream)

    # ---- end to end through the C ABI with host buffers: cufhedb_gate_lvl1_host
    # (pinned host inputs and output; H2D, key switch, PBS and D2H inside the
    # synchronous call, as the reference's one-call-per-batch operators are)
    import numpy as np
    ca_h = ca.cpu().pin_memory()
    cb_h = cb.cpu().pin_memory()
    out_h = torch.empty_like(ca_h).pin_memory()
    ca_n, cb_n, out_n = (t.numpy().view(np.uint32) for t in (ca_h, cb_h, out_h))

    def e2e_step():
        eng.gate_lvl1_host("NAND", ca_n, cb_n, PREC[head], out=out_n)

    barrier()
    e2e_ms = sum(_timed_sync_call(e2e_step, args.steps, flush, stream))

    import ctypes
    peaks = {}
    for name, fp64 in (("fp64", 1), ("split32", 0)):
        pk = ctypes.c_double(0.0)
        _lib.check(eng.lib.cufhedb_measure_fma_peak(local, fp64, ctypes.byref(pk)))
        peaks[name] = pk.value

    (t_head, t_other, t_e2e), (err_head, err_other) = reduce_over_ranks(
        [res[head]["total_ms"], res[other]["total_ms"], e2e_ms], [res[head]["errors"], res[other]["errors"]],
        "cuda")

    extra = {}
    cref = None
    if single and rank == 0 and not args.no_cpu_baseline:
        cref = CpuReference(os.cpu_count() or 1)
    if single and rank == 0:
        if args.filter_rows:
            rate, ms, ferr, finputs = range_filter(eng, args.filter_rows, PREC[head])
            extra["filter"] = {"rows": args.filter_rows, "rows_per_s": rate, "ms": ms, "decrypt_errors": ferr,
                               "workload": "x <= c (30th percentile), 20-bit column at lvl2, less_than_equal<Lvl2>",
                               "bootstraps_per_row": {"lvl02": 6, "lvl01": 3},
                               "lvl01_path": head}
            if cref is not None:
                nrows = min(args.filter_rows, max(64, 4 * cref.nthreads))
                crate, cerr = filter_cpu_baseline(cref, *finputs, nrows)
                extra["filter"]["cpu_baseline"] = {
                    "value": crate, "unit": "rows/s", "cores": cref.nthreads, "kind": "reference",
                    "decrypt_errors": cerr,
                    "sample": f"first {nrows} rows of the same ciphertexts, HEDB less_than_equal<Lvl2> "
                              "(oracle/_ref) on all host threads"}
            del finputs
        if args.filter_rows and args.agg_leg_rows:
            from cufhedb_b200.queries import filter_group_aggregate
            extra["aggregate"] = {
                "workload": "filter (date range at lvl2, discount range, quantity bound) + 3 x 2 groups, "
                            "SUM(price * (1 - discount)) and COUNT after decryption; DAG replayed as a CUDA graph",
                "precision": head, **filter_group_aggregate(eng, args.agg_leg_rows, PREC[head], steps=1)}
        if args.error_bootstraps:
            extra["error_rate"] = error_rate(eng, args.error_bootstraps, stream)
        if cref is not None and args.noise_samples:
            extra["noise_vs_oracles"] = noise_vs_oracles(eng, cref, args.noise_samples, stream)

    if rank == 0:
        value = whole_job_rate(world, B, args.steps, t_head)
        v_other = whole_job_rate(world, B, args.steps, t_other)
        e2e_value = whole_job_rate(world, B, args.steps, t_e2e)
        bf16, bf16_src = tensor_peak()

        def roof(name):
            # peak: the dense bf16 tensor-core figure of MEASURED_PEAKS.json; the
            # path computes on the CUDA cores, so the figure that bounds the kernel
            # is the CUDA-core FMA throughput measured alongside
            ach = B * F1 / (res[name]["pbs_ms"] / 1000.0) / 1e12
            core = "FP64" if name == "fp64" else "FP32"
            return {"bound": "tensor", "kernel": f"pbs01 ({name})", "achieved": ach,
                    "peak": bf16, "unit": "TFLOP/s", "frac": ach / bf16, "peak_source": bf16_src,
                    "traffic": TRAFFIC[name], "algorithmic_bytes": 66_060_288 + B * (2692 + 4100),
                    "algorithmic_flop_per_launch": B * F1,
                    "cuda_core_fma_peak": peaks[name],
                    "frac_of_cuda_core_fma_peak": ach / peaks[name] if peaks[name] else None,
                    "cuda_core_fma_peak_source": f"measured {core} CUDA-core FMA throughput "
                                                 "(cufhedb_measure_fma_peak), this GPU, this run",
                    "compute_units": f"{core} CUDA cores (transforms and products); the tensor-core "
                                     "stage-1 variant is timed beside it"}

        line = {
            "metric": METRIC, "value": value, "unit": "PBS/s", "n_gpus": world, "steps": args.steps,
            "warmup": W, "ms_per_step": t_head / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32" if head == "split32" else "f64",
            "data": "synthetic (deterministic keys and encryptions of uniform random bits)",
            "config": {"workload": WORKLOAD, "batch_per_gpu": B, "precision": head,
                       "l2": "flushed (256 MB write, untimed) before every timed step",
                       "parallelism": f"independent rows, {world} GPU(s)"},
            "decrypt_errors": int(err_head),
            other: {"value": v_other, "unit": "PBS/s", "ms_per_step": t_other / args.steps,
                    "decrypt_errors": int(err_other), "pbs_kernel_ms": res[other]["pbs_ms"],
                    "roofline": roof(other)},
            "split_over_fp64": (value / v_other) if head == "split32" else (v_other / value),
            "split_over_fp64_kernel": (res["fp64"]["pbs_ms"] / res["split32"]["pbs_ms"]),
            "pbs_kernel_ms": res[head]["pbs_ms"], "iks_kernel_ms": iks_ms,
            tc_name: {"pbs_kernel_ms": tc_ms, "pbs_per_s_kernel": B / (tc_ms / 1000.0),
                      "decrypt_errors_one_step": int(tc_errors),
                      "shape": eng.launch_shape(1, PREC[tc_name], B),
                      "what": "split32 with the first step of every digit transform on the tensor cores "
                              "(tcgen05 MMA, FP16 two-limb constants, FP32 accumulation in tensor memory)"},
            "autotune": tune,
            "roofline": roof(head),
            "gpu_launches": 2 * args.steps,
            "clocks": clk,
            "e2e": {"value": e2e_value, "unit": "PBS/s",
                    "h2d_bytes_per_step": 2 * B * (N1 + 1) * 4, "d2h_bytes_per_step": B * (N1 + 1) * 4},
        }
        line.update(extra)
        if cref is not None:
            try:
                nthreads = cref.nthreads
                c_a = ca.cpu().numpy().view(np.uint32).reshape(B, N1 + 1)
                c_b = cb.cpu().numpy().view(np.uint32).reshape(B, N1 + 1)
                cref.run(c_a[:nthreads], c_b[:nthreads])
                rate = cref.run(c_a, c_b)
                n1 = 16
                rate1 = cref.run(c_a[:n1], c_b[:n1], 1)
                line["cpu_baseline"] = {"value": rate, "unit": "PBS/s", "cores": nthreads, "kind": "reference",
                                        "sample": f"the step's {B} HomNANDs (TFHEpp from oracle/_ref) on {nthreads} "
                                                  "host threads",
                                        "one_core": {"value": rate1, "unit": "PBS/s", "cores": 1,
                                                     "sample": f"{n1} of the same HomNANDs on one thread"}}
            except Exception as exc:  # the GPU number stands without it
                line["cpu_baseline"] = {"value": None, "unit": "PBS/s", "cores": None, "kind": "reference",
                                        "sample": f"unavailable: {exc}"}
            cref.close()
        print(json.dumps(line), flush=True)
    eng.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


def run_filter_only(args):
    from cufhedb_b200 import GEN_ALL, Engine
    prec = _prec(args.precision)
    eng = Engine(0)
    eng.keygen(SEED, GEN_ALL)
    rows = args.filter_rows or 16384
    rate, ms, errors, _ = range_filter(eng, rows, prec, max(1, args.steps))
    print(json.dumps({"workload": "range filter x <= c, 20-bit lvl2 column", "rows": rows,
                      "precision": args.precision, "rows_per_s": rate, "ms": ms, "decrypt_errors": errors,
                      "pbs_per_row": {"lvl02": 6, "lvl01": 3}}))
    eng.close()


def run_error_only(args):
    import torch
    from cufhedb_b200 import GEN_BK01, GEN_KSK10, Engine
    eng = Engine(0)
    eng.keygen(SEED, GEN_BK01 | GEN_KSK10)
    r = error_rate(eng, args.error_bootstraps, torch.cuda.current_stream())
    print(json.dumps({"workload": "HomNAND over fresh encryptions of uniform random bits, every output decrypted",
                      **r}))
    eng.close()


def run_extprod(args):
    """4,096 external products TRGSW(random bit) x TRLWE(uniform) at lvl1 (FP64
    and split) and lvl2 (FP64), one TRGSW per product; computation error
    against the exact integer product (oracle) on a sample."""
    import numpy as np
    import torch
    from cufhedb_b200 import FP64, GEN_BK01, SPLIT32, Engine
    from oracle.oracle import Oracle
    B = 4096
    eng = Engine(0)
    eng.keygen(SEED, GEN_BK01)
    o = Oracle()
    _, s1, s2 = o.secret_keys(SEED)
    stream = torch.cuda.current_stream()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.int32, device="cuda")
    rng = np.random.default_rng(5)
    out = {}
    # lvl1: TRGSWs are encryptions of random bits (oracle, a sample) tiled to B
    nsamp = 16
    g1 = np.stack([o.trgsw32(int(m), s1, SEED, 0x35, i) for i, m in enumerate(rng.integers(0, 2, nsamp))])
    g1_all = np.tile(g1, (B // nsamp, 1, 1, 1))
    trl1 = rng.integers(0, 2 ** 32, (B, 2, N1), dtype=np.uint64).astype(np.uint32)
    g_d = torch.from_numpy(g1_all.view(np.int32).copy()).cuda()
    t_d = torch.from_numpy(trl1.view(np.int32).copy()).cuda()
    o_d = torch.empty(B * 2 * N1, dtype=torch.int32, device="cuda")
    for name, prec in (("fp64", FP64), ("split32", SPLIT32)):
        prep = torch.empty(B * 98304 // 8, dtype=torch.float64, device="cuda")
        eng.trgsw_prepare_lvl1(g_d, prep, prec)
        fn = lambda: eng.extprod_lvl1(t_d, prep, o_d, precision=prec, stream=stream)
        for _ in range(3):
            fn()
        ms = statistics.median(_timed(fn, max(3, args.steps), flush, stream))
        got = o_d.cpu().numpy().view(np.uint32).reshape(B, 2, N1)
        err = np.concatenate([((got[i].astype(np.int64) - o.extprod32_exact(trl1[i], g1_all[i]).astype(np.int64)
                                + 2 ** 31) % 2 ** 32 - 2 ** 31).ravel() for i in range(nsamp)])
        out[f"lvl1_{name}"] = {"products": B, "ms": ms, "products_per_s": B / (ms / 1000.0),
                               "achieved_tflops": B * 233_472 / (ms / 1000.0) / 1e12,
                               "algorithmic_bytes": B * (98_304 + 2 * 8192),
                               "err_vs_exact": {"samples": int(err.size), "max_abs": int(np.max(np.abs(err))),
                                                "var": float(np.var(err.astype(np.float64)))}}
        del prep
    # lvl2
    nsamp2 = 4
    g2 = np.stack([o.trgsw64(int(m), s2, SEED, 0x36, i) for i, m in enumerate(rng.integers(0, 2, nsamp2))])
    g2_all = np.tile(g2, (B // nsamp2, 1, 1, 1))
    trl2 = rng.integers(0, 2 ** 64, (B, 2, N2), dtype=np.uint64)
    g_d = torch.from_numpy(g2_all.view(np.int64).copy()).cuda()
    t_d = torch.from_numpy(trl2.view(np.int64).copy()).cuda()
    o_d = torch.empty(B * 2 * N2, dtype=torch.int64, device="cuda")
    prep = torch.empty(B * 262144 // 8, dtype=torch.float64, device="cuda")
    eng.trgsw_prepare_lvl2(g_d, prep)
    fn = lambda: eng.extprod_lvl2(t_d, prep, o_d, stream=stream)
    for _ in range(3):
        fn()
    ms = statistics.median(_timed(fn, max(3, args.steps), flush, stream))
    got = o_d.cpu().numpy().view(np.uint64).reshape(B, 2, N2)
    errs = []
    for i in range(nsamp2):
        d = (got[i] - o.extprod64_exact(trl2[i], g2_all[i])).view(np.int64)
        errs.append(d.astype(np.float64).ravel())
    err = np.concatenate(errs)
    out["lvl2_fp64"] = {"products": B, "ms": ms, "products_per_s": B / (ms / 1000.0),
                        "achieved_tflops": B * 643_072 / (ms / 1000.0) / 1e12,
                        "algorithmic_bytes": B * (262_144 + 2 * 32768),
                        "err_vs_exact": {"samples": int(err.size), "max_abs": float(np.max(np.abs(err))),
                                         "var": float(np.var(err))}}
    print(json.dumps({"workload": "external products, 4,096 per level, one TRGSW(random bit) per product", **out}))
    eng.close()


def run_profile_pbs(args):
    """--steps launches of the PBS kernel alone, no key-switching key."""
    import torch
    from cufhedb_b200 import FP64, GEN_BK01, GEN_BK02, SPLIT32, SPLIT32_TC, Engine, testvec_const
    prec = {"fp64": FP64, "split32": SPLIT32, "split32tc": SPLIT32_TC}[args.precision]
    eng = Engine(0)
    eng.keygen(SEED, GEN_BK01 if args.level == 1 else GEN_BK02)
    g = torch.Generator(device="cuda").manual_seed(99)
    x = torch.randint(-2 ** 31, 2 ** 31, (args.batch * (N0 + 1),), generator=g, device="cuda", dtype=torch.int64)
    x = x.to(torch.int32)
    if args.level == 1:
        out = torch.empty(args.batch * (N1 + 1), dtype=torch.int32, device="cuda")
        tv = testvec_const(MU)
        fn = lambda: eng.pbs_lvl01(x, out, tv, prec)
    else:
        out = torch.empty(args.batch * (N2 + 1), dtype=torch.int64, device="cuda")
        tv = testvec_const(1 << 61)
        fn = lambda: eng.pbs_lvl02(x, out, tv)
    for _ in range(args.warmup):
        fn()
    ev = _events(args.steps)
    for e0, e1 in ev:
        e0.record()
        fn()
        e1.record()
    eng.sync()
    ms = [e0.elapsed_time(e1) for e0, e1 in ev]
    rate = args.batch / (statistics.median(ms) / 1000.0) if ms else None
    print(json.dumps({"profile": f"pbs0{args.level}", "batch": args.batch,
                      "precision": args.precision if args.level == 1 else "fp64", "ms": ms, "pbs_per_s": rate,
                      "achieved_tflops": rate * (F1 if args.level == 1 else F2) / 1e12 if rate else None}))
    eng.close()


def run_profile_iks(args):
    """--steps launches of one identity key switch alone (lvl10: 5.6 GB key,
    lvl20: 11.3 GB, lvl21: 0.59 GB)."""
    import torch
    from cufhedb_b200 import GEN_KSK10, GEN_KSK20, GEN_KSK21, Engine
    flags = {10: GEN_KSK10, 20: GEN_KSK20, 21: GEN_KSK21}[args.profile_iks]
    eng = Engine(0)
    eng.keygen(SEED, flags)
    g = torch.Generator(device="cuda").manual_seed(98)
    if args.profile_iks == 10:
        x = torch.randint(-2 ** 31, 2 ** 31, (args.batch * (N1 + 1),), generator=g, device="cuda",
                          dtype=torch.int64).to(torch.int32)
        rows, width = 2 * N1, N0 + 1
    else:
        x = torch.randint(-2 ** 62, 2 ** 62, (args.batch * (N2 + 1),), generator=g, device="cuda", dtype=torch.int64)
        rows, width = (2 * N2, N0 + 1) if args.profile_iks == 20 else (10 * N2, N1 + 1)
    out = torch.empty(args.batch * width, dtype=torch.int32, device="cuda")
    fn = lambda: eng.iks(args.profile_iks, x, out)
    for _ in range(args.warmup):
        fn()
    ev = _events(args.steps)
    for e0, e1 in ev:
        e0.record()
        fn()
        e1.record()
    eng.sync()
    ms = [e0.elapsed_time(e1) for e0, e1 in ev]
    # algorithmic bytes: every selected key row (uniform inputs select a non-zero digit
    # with probability 1 - 2^-basebit) of `width` words, per ciphertext
    row_bytes = width * 4
    print(json.dumps({"profile": f"iks{args.profile_iks}", "batch": args.batch, "ms": ms,
                      "algorithmic_bytes_per_ct_max": rows * row_bytes,
                      "gbs_at_max_rows": args.batch * rows * row_bytes / (statistics.median(ms) / 1000.0) / 1e9}))
    eng.close()


def _engine_all_keys_tuned():
    from cufhedb_b200 import GEN_ALL, Engine
    eng = Engine(0)
    eng.keygen(SEED, GEN_ALL)
    return eng, eng.autotune()


def run_agg(args):
    from cufhedb_b200.queries import filter_group_aggregate
    eng, tune = _engine_all_keys_tuned()
    prec = _prec(args.precision)
    r = filter_group_aggregate(eng, args.agg_rows, prec, steps=max(1, min(args.steps, 3)))
    print(json.dumps({"workload": "filter (date range at lvl2, discount range, quantity bound) + 3 x 2 groups, "
                                  "SUM(price * (1 - discount)) and COUNT after decryption; DAG replayed as a CUDA graph",
                      "precision": args.precision, "autotune_pass_ms": tune, **r}))
    eng.close()


def run_queue_bench(args):
    import numpy as np
    from cufhedb_b200.queries import run_queue
    eng, tune = _engine_all_keys_tuned()
    prec = _prec(args.precision)
    rng = np.random.default_rng(64)
    lo, hi = np.log(2.0 ** 8), np.log(float(args.queue_max_rows))
    queries = [(int(round(np.exp(rng.uniform(lo, hi)))), int(rng.choice([8, 16, 24, 32]))) for _ in range(args.queue)]
    r = run_queue(eng, queries, prec, mode=args.queue_mode)
    print(json.dumps({"workload": f"{args.queue} filter queries x <= c, rows log-uniform in [2^8, {args.queue_max_rows}], "
                                  "widths uniform in {8, 16, 24, 32}",
                      "precision": args.precision, "autotune_pass_ms": tune, **r}))
    eng.close()


def _arc_model(op, xd, yd):
    """plaintext result of the ArcEDB digit combination (the same rule the
    GPU path and the reference compute): +mu iff true"""
    def single(x, y):
        return {"gt": x > y, "lt": x <= y, "eq": x == y}[op]
    r = single(xd[0], yd[0])
    for x, y in zip(xd[1:], yd[1:]):
        if op == "eq":
            r = r and x == y
        else:
            units = (2 if x == y else 0) + (4 if single(x, y) else -4) + (2 if r else -2) + 1
            r = 1 <= units % 16 <= 7
    return r


def run_arc(args):
    """ArcEDB comparisons (greater_than / less_than / equality over radix-1024
    digits: TRLWE of mu X^x_d against TRGSW of X^-y_d) of --arc-rows rows,
    FP64 and split; every output decrypted on the GPU and checked against the
    plaintext model; the reference's TFHEpp composition (oracle/_ref) timed on
    the host threads over a bounded sample."""
    import numpy as np
    import torch
    from cufhedb_b200 import FP64, GEN_BK01, GEN_KSK10, SPLIT32, Engine
    from oracle.oracle import Oracle, RefTFHEpp
    rows, D = args.arc_rows, args.arc_digits
    eng = Engine(0)
    eng.keygen(SEED, GEN_BK01 | GEN_KSK10)
    tune = eng.autotune(levels=(1,))
    o = Oracle()
    s0, s1, s2 = o.secret_keys(SEED)
    # 256 distinct encrypted rows (a quarter equal values, a quarter equal top
    # digits), tiled to `rows`
    nsamp = min(256, rows)
    rng = np.random.default_rng(99)
    xs = rng.integers(0, 1024 ** D, nsamp)
    ys = rng.integers(0, 1024 ** D, nsamp)
    ys[::4] = xs[::4]
    top = 1024 ** (D - 1)
    ys[1::4] = (xs[1::4] // top) * top + rng.integers(0, top, len(ys[1::4]))
    dig = lambda v, d: (int(v) >> (10 * d)) & 1023
    trl = np.stack([np.stack([o.arc_trlwe(dig(xs[i], d), s1, SEED, 0xB1, d * nsamp + i) for i in range(nsamp)])
                    for d in range(D)])
    g = np.stack([np.stack([o.arc_trgsw(dig(ys[i], d), s1, SEED, 0xB2, d * nsamp + i) for i in range(nsamp)])
                  for d in range(D)])
    idx = np.arange(rows) % nsamp
    trl_d = torch.from_numpy(np.ascontiguousarray(trl[:, idx]).view(np.int32)).cuda()
    g_d = torch.from_numpy(np.ascontiguousarray(g[:, idx]).view(np.int32)).cuda()
    stream = torch.cuda.current_stream()
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.int32, device="cuda")
    out = torch.empty(rows * (N1 + 1), dtype=torch.int32, device="cuda")
    ph = torch.empty(rows, dtype=torch.int32, device="cuda")
    res = {}
    for name, prec in (("split32", SPLIT32), ("fp64", FP64)):
        prep = torch.empty(D * rows * 98304 // 8, dtype=torch.float64, device="cuda")
        eng.trgsw_prepare_lvl1(g_d, prep, prec)
        for op in ("gt", "lt", "eq"):
            fn = lambda: eng.arc_compare(op, trl_d, prep, out, D, precision=prec, stream=stream)
            for _ in range(max(3, args.warmup)):
                fn()
            ms = statistics.median(_timed(fn, max(3, min(args.steps, 10)), flush, stream))
            eng.phase_lvl1(out, ph, stream=stream)
            got = (ph > 0).cpu().numpy()
            want = np.array([_arc_model(op, [dig(xs[i], d) for d in range(D)], [dig(ys[i], d) for d in range(D)])
                             for i in range(nsamp)])[idx]
            res[f"{op}_{name}"] = {"ms": ms, "rows_per_s": rows / (ms / 1000.0),
                                   "decrypt_errors": int((got != want).sum())}
        del prep
    eng.close()
    # the reference's composition on the host (TFHEpp from oracle/_ref)
    nthreads = os.cpu_count() or 1
    r = RefTFHEpp()
    r.set_secret(s0, s1, s2)
    r.set_bk01(o.bk01(SEED, s0, s1, nthreads))
    ptr, _ = r.ksk_view(10)
    o.ksk_full_into(10, SEED, (s0, s1, s2), ptr, nthreads)
    ncpu = min(nsamp, max(2 * nthreads, 64))
    gf = np.stack([np.stack([o.trgsw32_fft(g[d, i]) for i in range(ncpu)]) for d in range(D)])
    t0 = time.perf_counter()
    cout = r.arc_compare_batch("gt", np.ascontiguousarray(trl[:, :ncpu]), gf, nthreads)
    cpu_rate = ncpu / (time.perf_counter() - t0)
    cpu_sign = [(int(o.phase32(c, s1)) + 2 ** 31) % 2 ** 32 - 2 ** 31 > 0 for c in cout]
    cpu_err = sum(int(sg != _arc_model("gt", [dig(xs[i], d) for d in range(D)], [dig(ys[i], d) for d in range(D)]))
                  for i, sg in enumerate(cpu_sign))
    r.close()
    print(json.dumps({"workload": f"ArcEDB comparisons, {rows} rows x {D} radix-1024 digits "
                                  f"({nsamp} distinct encrypted rows tiled), lvl1 TRLWE vs TRGSW",
                      "per_row": {"external_products": D, "lvl01_bootstraps": D - 1, "iks10": D - 1},
                      "autotune_pass_ms": tune, **res,
                      "cpu_baseline": {"value": cpu_rate, "unit": "rows/s", "cores": nthreads, "kind": "reference",
                                       "sample": f"{ncpu} greater_than rows, TFHEpp composition of "
                                                 "comparable.cpp from oracle/_ref", "decrypt_errors": cpu_err}}))


def main():
    args = parse()
    if args.arc_rows:
        run_arc(args)
    elif args.agg_rows:
        run_agg(args)
    elif args.queue:
        run_queue_bench(args)
    elif args.profile_iks:
        run_profile_iks(args)
    elif args.profile_pbs:
        run_profile_pbs(args)
    elif args.filter_only:
        run_filter_only(args)
    elif args.error_only:
        run_error_only(args)
    elif args.extprod:
        run_extprod(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
