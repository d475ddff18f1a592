"""Benchmark: mine() seconds and bitset-AND GB/s on the B200 engine.

Default workload: the planted-pattern database (100,000 transactions over
1,000 items, 2,000 planted Zipf(1.1) patterns + Zipf(1.1) noise, mean length
10, seed 7) mined at minSup 0.005 by cuEclat and cuApriori; one step mines it
with both.  ``--workload`` selects another synthetic database.

* ``value``: seconds per step with the transaction tidsets already resident in
  HBM (cpm_mine on a loaded database), timed with CUDA events on the library's
  stream, max over ranks.
* ``e2e``: the same step through the public Python API from host arrays --
  ``cuEclat(csr, minSup).mine()`` and ``cuApriori(...).mine()`` -- including
  the host->device copy of the CSR, packing, mining and the device->host copy
  of the patterns (the reference's own ``getMiningTime()`` definition).
* ``roofline``: the dominant kernel of the step against MEASURED_PEAKS.json.
* ``cpu_baseline``: the reference's host path (NumPy in place of CuPy,
  ``oracle.numpy_port``) on one core, one full step.

``--impl reference`` times that host path alone on this box's cores.
Multi-GPU runs (torchrun) give every rank its own database of the same shape
(seed + rank): weak scaling, no collective on the data path.
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
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

import numpy as np  # noqa: E402

WORKLOADS = {
    # name: (generator kwargs builder, minSup, algorithms)
    "planted-100k": ("planted_zipf", 0.005, ("eclat", "apriori")),
    "uniform-10k": ("uniform_poisson", 0.01, ("eclat",)),
    "dense-bernoulli-64k": ("dense_bernoulli", 0.6, ("eclat",)),
    "dense-fixed-64k": ("dense_fixed_length", 0.6, ("eclat",)),
    "sparse-zipf-1m": ("sparse_zipf", 0.001, ("eclat",)),
}


def make_workload(name, rank):
    from cupami_b200 import datasets

    gen, minsup, algos = WORKLOADS[name]
    fn = getattr(datasets, gen)
    import inspect

    seed = inspect.signature(fn).parameters["seed"].default + rank
    return fn(seed=seed), minsup, algos, seed


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d.get("hbm_gbs", 6650.0), d.get("bf16_tflops", 1590.0), "measured"
    return 6650.0, 1590.0, "fallback"


class ClockSampler:
    """nvidia-smi samples during the timed region."""

    def __init__(self, index):
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.file, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait(timeout=10)
        self.file.seek(0)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.file.read().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.file.name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "samples": len(sm), "reasons": sorted(reasons)}


def flush_l2(buf):
    buf.add_(1)


def int8_peak_tops():
    import torch

    a = torch.randint(-8, 8, (8192, 8192), dtype=torch.int8, device="cuda")
    b = torch.randint(-8, 8, (8192, 8192), dtype=torch.int8, device="cuda")
    best = 1e9
    for _ in range(12):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch._int_mm(a, b)
        e.record()
        torch.cuda.synchronize()
        best = min(best, s.elapsed_time(e))
    return 2 * 8192 ** 3 / (best * 1e-3) / 1e12


def cpu_baseline(csr, minsup, algos, budget_s=30.0):
    """The reference's host path (NumPy kernels) on one core, whole steps."""
    import oracle
    from oracle import numpy_port

    labels, rows, cols, n_tx = numpy_port.device_pairs_from_csr(csr.offsets, csr.items)
    ms = oracle.support_count(minsup, n_tx)
    times = []
    t_end = time.perf_counter() + budget_s
    while not times or (time.perf_counter() < t_end and len(times) < 3):
        t0 = time.perf_counter()
        labels, rows, cols, n_tx = numpy_port.device_pairs_from_csr(csr.offsets, csr.items)
        for a in algos:
            (numpy_port.eclat if a == "eclat" else numpy_port.apriori)(labels, rows, cols, n_tx, ms)
        times.append(time.perf_counter() - t0)
    return statistics.median(times), len(times)


def run_reference(args, world, rank):
    if rank != 0:
        return
    csr, minsup, algos, seed = make_workload(args.workload, 0)
    cores = 1
    times = []
    import oracle
    from oracle import numpy_port

    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        labels, rows, cols, n_tx = numpy_port.device_pairs_from_csr(csr.offsets, csr.items)
        ms = oracle.support_count(minsup, n_tx)
        for a in algos:
            (numpy_port.eclat if a == "eclat" else numpy_port.apriori)(labels, rows, cols, n_tx, ms)
        if i >= args.warmup:
            times.append(time.perf_counter() - t0)
    v = statistics.mean(times)
    line = {
        "impl": "reference", "metric": "mine() seconds per step (" + "+".join(algos) + ")",
        "value": v, "unit": "s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": v * 1e3, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "u64", "data": "synthetic",
        "config": {"workload": args.workload, "seed": seed, "minSup": minsup, "algorithms": list(algos)},
        "cpu_baseline": {"value": v, "unit": "s", "cores": cores, "kind": "port",
                         "sample": f"whole {args.workload} step (NumPy restatement of the reference host path)"},
        "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="planted-100k", choices=sorted(WORKLOADS))
    ap.add_argument("--scheduler", default="plain", choices=["plain", "learned"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    world, rank, local = dist_setup()
    if args.impl == "reference":
        return run_reference(args, world, rank)

    import torch

    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
        pg = dist
    import cupami_b200
    from cupami_b200 import _native

    csr, minsup, algos, seed = make_workload(args.workload, rank)
    n_tx = int(np.count_nonzero(np.diff(csr.offsets.astype(np.int64)) > 0))
    ms_count = cupami_b200.cuApriori._getSupportCount(minsup, n_tx)
    ctx = _native.context(local)
    db = _native.Database.from_ids(ctx, csr.offsets, csr.items)
    opts = _native.Opts()
    _native.library().cpm_default_opts(opts)
    opts.scheduler = _native.CPM_SCHED_LEARNED if args.scheduler == "learned" else _native.CPM_SCHED_PLAIN
    algo_code = {"eclat": (_native.CPM_ECLAT, _native.CPM_ORDER_ECLAT),
                 "apriori": (_native.CPM_APRIORI, _native.CPM_ORDER_APRIORI)}
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MB > L2

    def device_step():
        stats = []
        for a in algos:
            code, order = algo_code[a]
            res = db.mine(ms_count, code, opts, order)
            stats.append(res.stats)
        return stats

    def barrier():
        torch.cuda.synchronize()
        if pg:
            pg.barrier()

    for _ in range(args.warmup):
        device_step()
    barrier()
    sampler = ClockSampler(local)
    step_ms, per_kernel = [], []
    launches = 0
    for _ in range(args.steps):
        flush_l2(flush)
        torch.cuda.synchronize()
        stats = device_step()
        step_ms.append(sum(s["ms_total"] for s in stats))
        per_kernel.append(stats)
        launches += sum(int(s["kernel_launches"]) for s in stats)
    barrier()
    clocks = sampler.stop()
    # e2e through the public API from host arrays.
    for _ in range(args.warmup):
        for a in algos:
            (cupami_b200.cuEclat if a == "eclat" else cupami_b200.cuApriori)(csr, minsup).mine()
    barrier()
    e2e = []
    d2h = 0
    for _ in range(args.steps):
        flush_l2(flush)
        torch.cuda.synchronize()
        t = 0.0
        for a in algos:
            m = (cupami_b200.cuEclat if a == "eclat" else cupami_b200.cuApriori)(csr, minsup)
            m.mine()
            t += m.getMiningTime()
            off, it, sup, _ = m.getPatternArrays()
            d2h = max(d2h, it.nbytes + sup.nbytes // 2 * 3)
        e2e.append(t)
    barrier()
    value = statistics.mean(step_ms) / 1e3
    e2e_v = statistics.mean(e2e)
    if pg:
        t = torch.tensor([value, e2e_v], device="cuda", dtype=torch.float64)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        value, e2e_v = t.tolist()
    # Roofline of the dominant kernel, averaged over the timed steps.
    deep_ms = statistics.mean(sum(s["ms_deep"] for s in st) for st in per_kernel)
    pair_ms = statistics.mean(sum(s["ms_pairs"] for s in st) for st in per_kernel)
    deep_bytes = statistics.mean(sum(s["bytes_alg"] for s in st) for st in per_kernel)
    pair_ops = statistics.mean(sum(s["pair_ops"] for s in st) for st in per_kernel)
    hbm, bf16, src = peaks()
    if deep_ms >= pair_ms:
        achieved = deep_bytes / (deep_ms * 1e-3) / 1e9 if deep_ms else 0.0
        roof = {"kernel": "deep-level intersection (k_deep)", "bound": "hbm", "achieved": achieved,
                "peak": hbm, "unit": "GB/s", "frac": achieved / hbm, "traffic": None,
                "peak_source": src, "ms_per_step": deep_ms, "alg_bytes_per_step": deep_bytes}
    else:
        i8 = int8_peak_tops()
        achieved = pair_ops / (pair_ms * 1e-3) / 1e12 if pair_ms else 0.0
        roof = {"kernel": "pair Gram", "bound": "tensor", "achieved": achieved, "peak": i8,
                "unit": "TOPS", "frac": achieved / i8, "traffic": None,
                "peak_source": "torch._int_mm int8 8192^3 best of 12 on this box",
                "ms_per_step": pair_ms, "alg_ops_per_step": pair_ops}
    if rank != 0:
        if pg:
            pg.barrier()
            pg.destroy_process_group()
        return
    cpu = None
    if not args.no_cpu_baseline:
        v, n = cpu_baseline(csr, minsup, algos)
        cpu = {"value": v, "unit": "s", "cores": 1, "kind": "port",
               "sample": f"whole step, median of {n} (NumPy restatement of the reference host path)"}
    h2d = int(csr.offsets.nbytes + csr.items.nbytes) * len(algos)
    last = per_kernel[-1]
    line = {
        "metric": "mine() seconds per step (" + "+".join(algos) + ")",
        "value": value, "unit": "s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": value * 1e3, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "u64", "data": "synthetic",
        "config": {"workload": args.workload, "seed": seed, "minSup": minsup, "algorithms": list(algos),
                   "transactions": n_tx, "scheduler": args.scheduler,
                   "l2": "256 MB buffer rewritten before every timed step",
                   "parallelism": f"replicas{world}" if world > 1 else "single"},
        "e2e": {"value": e2e_v, "unit": "s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "roofline": roof,
        "cpu_baseline": cpu,
        "gpu_launches": launches,
        "clocks": clocks,
        "patterns": [int(s["n_patterns"]) for s in last],
        "kernel_stats": last,
    }
    print(json.dumps(line), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
