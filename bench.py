"""Benchmark: mine() seconds and bitset-AND GB/s on the B200 engine.

Default workload: the large sparse database (1,000,000 transactions over
20,000 items, Poisson(40) lengths, Zipf(1.0) items, seed 3) mined by cuEclat
at minSup 0.001 (6,280,597 patterns); one step mines it once.  The
planted-pattern database (100,000 x 1,000, cuEclat + cuApriori) and the 512
batched databases are measured after it and reported under ``others``.
``--workload`` selects another synthetic database as the headline.

* ``value``: seconds per step with the transaction tidsets already resident in
  HBM (cpm_mine on a loaded database), timed with CUDA events on the library's
  stream, max over ranks.
* ``e2e``: the same step through the public Python API from host arrays --
  ``cuEclat(csr, minSup).mine()`` and ``cuApriori(...).mine()`` -- including
  the host->device copy of the CSR, packing, mining and the device->host copy
  of the patterns (the reference's own ``getMiningTime()`` definition).
* ``roofline``: the dominant kernel of the step against MEASURED_PEAKS.json.
* ``cpu_baseline``: the reference's host path (NumPy in place of CuPy,
  ``oracle.numpy_port``) on one core: one full step where that takes seconds;
  on the 1M x 20k workload (hours on one core) an estimate from timed samples
  of every operation the reference's driver runs, times the exact number of
  times it runs them (``estimate_reference_cpu``).

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
    # the reference's quickstart dataset, whose mining times it publishes
    "quickstart-10k": ("quickstart", 0.01, ("eclat", "apriori")),
    "dense-bernoulli-64k": ("dense_bernoulli", 0.6, ("eclat",)),
    "dense-fixed-64k": ("dense_fixed_length", 0.6, ("eclat",)),
    "sparse-zipf-1m": ("sparse_zipf", 0.001, ("eclat",)),
    # the same generator at a quarter of the transactions (profiling-sized)
    "sparse-zipf-250k": ("sparse_zipf_250k", 0.001, ("eclat",)),
    # 512 independent databases mined in one pass (cuEclat.mineBatch)
    "batched-zipf-512": ("batched_zipf", 0.01, ("eclat-batch",)),
    # temporal database (100,000 rows, 200 items) mined by cuPFEclat and cuPFApriori
    "temporal-100k": ("temporal_planted", 0.005, ("pf-eclat", "pf-apriori")),
}

# Periodicity limits (timestamp units) of the temporal workloads.
MAX_PER = {"temporal-100k": 2500}


# Published mine() seconds of the reference on a workload (cuEclat + cuApriori
# on the quickstart dataset: 0.2545 s + 0.7180 s, quickstart.ipynb).
PUBLISHED = {"quickstart-10k": 0.2545 + 0.7180}


def make_workload(name, rank):
    from cupami_b200 import datasets

    gen, minsup, algos = WORKLOADS[name]
    seed = rank_seed(name, rank)
    return getattr(datasets, gen)(seed=seed), minsup, algos, seed


def n_transactions(csr):
    if isinstance(csr, list):
        return sum(n_transactions(c) for c in csr)
    return int(np.count_nonzero(np.diff(csr.offsets.astype(np.int64)) > 0))


def max_over_ranks(values, device):
    """Element-wise max of per-rank timings (the only collective: no data-path exchange)."""
    import torch
    import torch.distributed as dist

    t = torch.tensor(values, device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()


def rank_seed(name, rank):
    """Seed of this rank's database: the workload's own seed plus the rank (weak scaling)."""
    import inspect

    from cupami_b200 import datasets

    fn = getattr(datasets, WORKLOADS[name][0])
    return inspect.signature(fn).parameters["seed"].default + rank


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


# Exact counts of the reference driver's operations on a workload's answer
# (frames, positions, intersections, copied rows), from the oracle's summary.
SEARCH_COUNTS = {"sparse-zipf-1m": ROOT / "tests" / "golden" / "sparse_zipf_1m_summary.json"}


def search_counts(workload):
    p = SEARCH_COUNTS.get(workload)
    if p is None or not p.exists():
        return None
    d = json.loads(p.read_text())
    return (d["reference_search"], d["patterns"]) if "reference_search" in d else None


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


def deep_traffic(workload, tidsets, arena_mb):
    """The committed ncu record of one k_deep launch of this workload (DRAM
    bytes per launch, L2 throughput), or None if there is none."""
    p = ROOT / "profiles" / "k_deep_traffic.json"
    if not p.exists() or arena_mb:
        return None
    d = json.loads(p.read_text()).get(workload)
    if not d or d.get("tidsets", 0) != tidsets:
        return None
    return d


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


def _port_step(csr, minsup, algos):
    import oracle
    from oracle import numpy_port

    labels, rows, cols, n_tx = numpy_port.device_pairs_from_csr(csr.offsets, csr.items)
    ms = oracle.support_count(minsup, n_tx)
    for a in algos:
        (numpy_port.apriori if a == "apriori" else numpy_port.eclat)(labels, rows, cols, n_tx, ms)


def cpu_step_seconds(csr, minsup, algos, budget_s=30.0):
    """The reference's host path (NumPy kernels) on one core for one step.

    Batched workloads run a sample of databases (first ones, up to the time
    budget) and scale by transactions; returns (seconds, sample description)."""
    if isinstance(csr, list):
        t0 = time.perf_counter()
        done_tx = 0
        k = 0
        for c in csr:
            _port_step(c, minsup, algos)
            done_tx += n_transactions(c)
            k += 1
            if time.perf_counter() - t0 > budget_s:
                break
        spent = time.perf_counter() - t0
        total = n_transactions(csr)
        return spent * total / max(1, done_tx), f"{k} of {len(csr)} databases ({done_tx} of {total} transactions), scaled by transactions"
    times = []
    t_end = time.perf_counter() + budget_s
    while not times or (time.perf_counter() < t_end and len(times) < 3):
        t0 = time.perf_counter()
        _port_step(csr, minsup, algos)
        times.append(time.perf_counter() - t0)
    return statistics.median(times), f"whole step, median of {len(times)}"


class ReferenceCpuModel:
    """Seconds the reference's Eclat driver takes on one core with NumPy kernels
    (``oracle.numpy_port``), for a database too large to mine that way in a
    benchmark: the label mapping, packing and singleton counts run in full;
    every other operation of the driver (cuEclat.py:168-245) is timed on
    samples of the real tidsets and multiplied by how often the driver runs it
    on this database (``counts``: pair candidates, top-level class members,
    positions, intersected rows, copied child rows, patterns).

    The model is per operation, not per pattern: ``count_supports`` of a pair
    (two gathered rows, AND, popcount), ``intersect_extensions`` per call and per
    row, ``take`` per copied row, the top-level vertical gather per member, and
    one dict insertion per pattern.  NumPy's costs here do not depend on the
    bits' values, only on the row width, which is the same for every tidset
    (the reference keeps every tidset as a full-width bitset)."""

    def __init__(self, csr, counts, patterns):
        from oracle import numpy_port

        self.np = numpy_port
        self.counts, self.patterns = counts, patterns
        t0 = time.perf_counter()
        labels, rows, cols, n_tx = numpy_port.device_pairs_from_csr(csr.offsets, csr.items)
        self.bits = numpy_port.pack(rows, cols, n_tx, len(labels))
        sup = numpy_port.supports_of(self.bits, [[i] for i in range(len(labels))])
        self.fixed_s = time.perf_counter() - t0
        self.n_tx = n_tx
        self.frequent = np.array([i for i, v in enumerate(sup) if v >= 1], dtype=np.int64)

    @staticmethod
    def _slope(fn, sizes, reps=2):
        """(per-call, per-unit) seconds from the best of ``reps`` timings at each size (least squares)."""
        xs, ys = [], []
        for n in sizes:
            best = min(fn(n) for _ in range(reps))
            xs.append(n)
            ys.append(best)
        b, a = np.polyfit(np.asarray(xs, float), np.asarray(ys, float), 1)
        return max(a, 0.0), max(b, 0.0)

    def sample(self, seed):
        """One estimate (seconds) from a fresh sample; returns (seconds, detail)."""
        rng = np.random.default_rng(seed)
        k, bits, fr = self.np, self.bits, self.frequent
        pick = lambda n: fr[rng.integers(0, fr.size, n)]

        def t_pairs(n):
            batch = np.stack([pick(n), pick(n)], axis=1).tolist()
            t0 = time.perf_counter()
            k.supports_of(bits, batch)
            return time.perf_counter() - t0

        def t_vertical(n):
            members, left = pick(n), int(pick(1)[0])
            t0 = time.perf_counter()
            k.NUMPY.vertical(bits, members, left)
            return time.perf_counter() - t0

        rows = bits[pick(513)]

        def t_frame(m):
            # The driver's own search loop over one frame of m members whose
            # children all fail: m - 1 positions, m(m - 1)/2 intersected rows.
            t0 = time.perf_counter()
            k._search({}, ("p",), [str(i) for i in range(m)], rows[:m], self.n_tx + 1)
            return time.perf_counter() - t0

        child = rows[1:]

        def t_take(n):
            keep = sorted(rng.choice(child.shape[0], n, replace=False).tolist())
            t0 = time.perf_counter()
            k.NUMPY.take(child, keep)
            return time.perf_counter() - t0

        names = [str(i) for i in range(1024)]
        big = {(names[i & 1023], names[i >> 10], "x"): i for i in range(1 << 20)}  # a dict of realistic size

        def t_dict(n):
            head = ("a", "b")
            t0 = time.perf_counter()
            for i in range(n):
                big[head + (names[i & 1023], names[(i >> 10) & 1023])] = int(i)
            return time.perf_counter() - t0

        c = self.counts
        # Pair batches large enough that the gathered rows (two per pair) leave
        # the caches, as the driver's 65,536-pair batches do: up to 1 GB each.
        width = bits.shape[1] * 4
        top = int(min(c["pair_candidates"], max(256, (1 << 30) // width)))
        _, pair = self._slope(t_pairs, sorted({max(1, top // 4), max(1, top // 2), top}))
        _, vert = self._slope(t_vertical, (64, 128, 256))
        ms = (2, 4, 16, 64)
        tf = [min(t_frame(m) for _ in range(2)) for m in ms]
        (call, row), *_ = np.linalg.lstsq(np.array([[m - 1, m * (m - 1) / 2] for m in ms], float),
                                          np.array(tf), rcond=None)
        call, row = max(float(call), 0.0), max(float(row), 0.0)
        _, take = self._slope(t_take, (8, 64, 256))
        _, ins = self._slope(t_dict, (20_000, 100_000))
        positions = c["top_positions"] + c["deep_positions"]
        intersections = c["top_intersections"] + c["deep_intersections"]
        parts = {"fixed": self.fixed_s, "pairs": pair * c["pair_candidates"], "vertical": vert * c["top_members"],
                 "intersect_calls": call * positions, "intersect_rows": row * intersections,
                 "take": take * c["copied_children"], "dict": ins * self.patterns}
        return sum(parts.values()), parts


def reference_gpu_seconds(csr, minsup, algos, ours, device, budget_s=60.0):
    """The reference's GPU path on this GPU for one step, warm (``oracle.ref_gpu``:
    its own three kernels compiled from its source, its driver loops, torch
    standing in for CuPy).  ``ours`` holds this engine's pattern dicts of the
    same step, to check that both paths agree.

    Batched workloads run the first databases up to the time budget and scale
    by transactions; a single database that runs past the budget is scaled by
    the patterns found by then (an estimate, and labelled as one)."""
    from oracle import ref_gpu

    if not ref_gpu.available():
        return {"unavailable": "oracle/_ref/libref_bitsets.so not built"}
    csrs = csr if isinstance(csr, list) else [csr]
    algos = ["eclat" if a == "eclat-batch" else a for a in algos]
    uploads = [ref_gpu.upload(c.offsets, c.items, device) for c in csrs]
    k = ref_gpu.RefKernels(device)
    # first call: module load and allocator warm-up (the reference's would also include NVRTC)
    first = None
    if n_transactions(csrs[0]) <= 200_000:
        t0 = time.perf_counter()
        for a in algos:
            ref_gpu.mine(*uploads[0], minsup, a, k)
        first = time.perf_counter() - t0
    t0 = time.perf_counter()
    k.deadline = t0 + budget_s
    done_tx, done_db, same, partial = 0, 0, True, None
    try:
        for i, (c, up) in enumerate(zip(csrs, uploads)):
            for j, a in enumerate(algos):
                out = {}
                try:
                    ref_gpu.mine(*up, minsup, a, k, out)
                except TimeoutError:
                    partial = (len(out), len(ours[i][j]))
                    raise
                got = [("\t".join(key), v) for key, v in out.items()]
                same &= got == list(ours[i][j].items())
            done_tx += n_transactions(c)
            done_db += 1
    except TimeoutError:
        pass
    spent = time.perf_counter() - t0
    kind = ("reference kernels (cupami _bitsets source, nvcc sm_100a) + reference driver loops; "
            "torch tensors in place of CuPy arrays")
    if partial is not None and done_db == 0:
        found, want = partial
        return {"value": spent * want / max(1, found), "unit": "s", "first_call_s": first, "estimated": True,
                "sample": f"stopped after {spent:.1f} s with {found} of {want} patterns; scaled by patterns",
                "identical_output": None, "kind": kind}
    total = n_transactions(csrs)
    return {"value": spent * total / max(1, done_tx), "unit": "s", "first_call_s": first,
            "estimated": done_db < len(csrs),
            "sample": (f"{done_db} of {len(csrs)} databases, scaled by transactions" if len(csrs) > 1
                       else "whole step, warm"),
            "identical_output": bool(same), "kind": kind}


def run_reference(args, world, rank):
    if rank != 0:
        return
    csr, minsup, algos, seed = make_workload(args.workload, 0)
    budget = 20.0 if isinstance(csr, list) else 60.0
    times, sample, estimated = [], "", False
    counts = search_counts(args.workload)
    model = ReferenceCpuModel(csr, *counts) if counts and algos == ("eclat",) else None
    for i in range(args.warmup + args.steps):
        if model is not None:
            v, parts = model.sample(seed=i)
            sample = ("estimate: label mapping, packing and singletons run in full (%.1f s); pair counts, "
                      "vertical gathers, intersect calls and rows, child copies and dict inserts timed on "
                      "samples of the real tidsets and scaled by the driver's exact operation counts on this "
                      "database; last step's parts (s): %s" % (model.fixed_s, json.dumps(
                          {key: round(val, 1) for key, val in parts.items()})))
            estimated = True
        else:
            v, sample = cpu_step_seconds(csr, minsup, algos, budget_s=budget if isinstance(csr, list) else 0.0)
        if i >= args.warmup:
            times.append(v)
    v = statistics.mean(times)
    line = {
        "impl": "reference", "metric": "mine() seconds per step (" + "+".join(algos) + ")",
        "value": v, "unit": "s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": v * 1e3, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "u64", "data": "synthetic",
        "config": {"workload": args.workload, "seed": seed, "minSup": minsup, "algorithms": list(algos)},
        "cpu_baseline": {"value": v, "unit": "s", "cores": 1, "kind": "port", "estimated": estimated,
                         "sample": f"{sample} (NumPy restatement of the reference host path)"},
        "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def periodic_workload(name, rank):
    """(csr, timestamps, transactions as label tuples, minSup, maxPer, seed) of a temporal workload."""
    from cupami_b200 import datasets

    gen, minsup, _ = WORKLOADS[name]
    seed = rank_seed(name, rank)
    csr, ts = getattr(datasets, gen)(seed=seed)
    o, it = csr.offsets.tolist(), [str(v) for v in csr.items.tolist()]
    baskets = [tuple(it[o[i]:o[i + 1]]) for i in range(len(o) - 1)]
    return csr, ts, baskets, minsup, MAX_PER[name], seed


def periodic_cpu_seconds(baskets, ts, minsup, maxper):
    """The reference's periodic miners restated on one core (oracle.periodic), one full step."""
    from oracle import periodic

    t0 = time.perf_counter()
    rows = [[int(t), *b] for t, b in zip(ts.tolist(), baskets)]
    labels, bits, timestamps, end = periodic.prepare(rows)
    count, limit = periodic.thresholds(minsup, maxper, len(timestamps), end)
    for fn in (periodic.pf_eclat, periodic.pf_apriori):
        fn(labels, bits, timestamps, end, count, limit)
    return time.perf_counter() - t0


def run_periodic_reference(args, world, rank, local):
    if rank != 0:
        return
    csr, ts, baskets, minsup, maxper, seed = periodic_workload(args.workload, 0)
    times = [periodic_cpu_seconds(baskets, ts, minsup, maxper) for _ in range(args.warmup + args.steps)]
    v = statistics.mean(times[args.warmup:])
    line = {
        "impl": "reference", "metric": "mine() seconds per step (pf-eclat+pf-apriori)",
        "value": v, "unit": "s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": v * 1e3, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "i64", "data": "synthetic",
        "config": {"workload": args.workload, "seed": seed, "minSup": minsup, "maxPer": maxper},
        "cpu_baseline": {"value": v, "unit": "s", "cores": 1, "kind": "port",
                         "sample": "whole step (NumPy restatement of the reference periodic miners)"},
        "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_periodic(args, world, rank, local):
    """cuPFEclat + cuPFApriori on a temporal database: device time with resident
    tidsets, the drop-in API from host rows, the periodic_counts kernel against
    the roofline, and the reference's kernels and host path beside them."""
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
    from cupami_b200.frequentPattern import _bitsets
    from cupami_b200.periodicFrequentPattern import _temporal

    csr, ts, baskets, minsup, maxper, seed = periodic_workload(args.workload, rank)
    n = len(baskets)
    end = int(ts[-1])
    labels = sorted({x for b in baskets for x in b})
    index = {label: i for i, label in enumerate(labels)}
    cols = np.fromiter((index[x] for b in baskets for x in b), dtype=np.uint32, count=csr.nnz)
    ctx = _native.context(local)
    db = _native.Database.from_temporal(ctx, csr.offsets, cols, len(labels), ts, end)
    ms_count = cupami_b200.cuApriori._getSupportCount(minsup, n)
    codes = [("pf-eclat", _native.CPM_ECLAT, _native.CPM_ORDER_DEPTH_FIRST),
             ("pf-apriori", _native.CPM_APRIORI, _native.CPM_ORDER_APRIORI)]
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MB > L2

    def device_step():
        return [(a, db.mine_periodic(ms_count, maxper, code, order)) for a, code, order in codes]

    for _ in range(args.warmup):
        device_step()
    torch.cuda.synchronize()
    if pg:
        pg.barrier()
    sampler = ClockSampler(local)
    step_ms, launches, last = [], 0, None
    for _ in range(args.steps):
        flush_l2(flush)
        torch.cuda.synchronize()
        last = device_step()
        step_ms.append(sum(r.stats["ms_total"] for _, r in last))
        launches += sum(int(r.stats["kernel_launches"]) for _, r in last)
    clocks = sampler.stop()
    torch.cuda.synchronize()
    if pg:
        pg.barrier()

    from cupami_b200.datasets import TemporalCSR

    def api_step():
        t, d2h = 0.0, 0
        for cls in (cupami_b200.cuPFEclat, cupami_b200.cuPFApriori):
            m = cls(TemporalCSR(csr.offsets, csr.items, ts), minsup, maxper)
            m.mine()
            t += m.getMiningTime()
            d2h += 20 * len(m._result)  # parent, item, support (4 bytes each) and periodicity (8) per pattern
        return t, d2h

    for _ in range(args.warmup):
        api_step()
    e2e, d2h = [], 0
    for _ in range(args.steps):
        flush_l2(flush)
        torch.cuda.synchronize()
        t, d2h = api_step()
        e2e.append(t)
    value = statistics.mean(step_ms) / 1e3
    e2e_v = statistics.mean(e2e)
    if pg:
        value, e2e_v = max_over_ranks([value, e2e_v], "cuda")
        pg.destroy_process_group()
    # The counting kernel alone (k_periodic through cpm_periodic_counts, no early
    # stop) on every pair of the kept items, timed with CUDA events on the
    # library's stream.  Algorithmic bytes per candidate: its two rows of 32-bit
    # words, a timestamp per set row, the two column ids and the two results.
    rows_idx = torch.from_numpy(np.repeat(np.arange(n, dtype=np.int64),
                                          np.diff(csr.offsets.astype(np.int64))).copy()).cuda()
    # rows padded to a multiple of 4 words (16-byte aligned rows); the kernel scans the first n rows
    bits32 = _bitsets.build_bitsets(None, rows_idx, torch.from_numpy(cols.view(np.int32).copy()).cuda(),
                                    (n + 127) // 128 * 128, len(labels))
    d_ts = torch.from_numpy(ts.copy()).cuda()
    apriori = dict(last)["pf-apriori"]  # by length: the kept single items come first
    singles = int(np.count_nonzero(np.diff(apriori.offsets.astype(np.int64)) == 1))
    kept = sorted(int(c) for c in apriori.items[:singles])
    pairs = np.array([(a, b) for i, a in enumerate(kept) for b in kept[i + 1:]], dtype=np.uint32).reshape(-1, 2)
    d_pairs = torch.from_numpy(pairs.view(np.int32).copy()).cuda()
    sup = torch.zeros(len(pairs), dtype=torch.int64, device="cuda")
    per = torch.zeros(len(pairs), dtype=torch.int64, device="cuda")
    stream = torch.cuda.ExternalStream(ctx.stream())
    lib = _native.library()

    def launch():
        ctx.check(lib.cpm_periodic_counts(ctx.handle, bits32.data_ptr(), bits32.shape[1], d_pairs.data_ptr(),
                                          len(pairs), 2, d_ts.data_ptr(), n, end, sup.data_ptr(), per.data_ptr()))

    for _ in range(3):
        launch()
    ctx.check(lib.cpm_synchronize(ctx.handle))
    kms = []
    for _ in range(args.steps):
        flush_l2(flush)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        launch()
        e1.record(stream)
        e1.synchronize()
        kms.append(e0.elapsed_time(e1))
    k_ms = statistics.mean(kms)
    alg_bytes = len(pairs) * (2 * ((n + 31) // 32) * 4 + 8 + 16) + 8 * int(sup.sum().item())
    achieved = alg_bytes / (k_ms * 1e-3) / 1e9
    hbm, _, src = peaks()
    roof = {"kernel": "k_periodic (cpm_periodic_counts, every pair of the kept items)", "bound": "hbm",
            "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm, "traffic": None,
            "peak_source": src, "ms_per_launch": k_ms, "alg_bytes_per_launch": alg_bytes, "candidates": len(pairs),
            "alg_bytes": "per candidate: 2 rows x words32 x 4 + 8 per set row (timestamps) + 24 (ids, results); "
                         "the bitsets (items x rows / 8 bytes) stay in L2 between candidates"}
    if rank != 0:
        return
    ours = {a: [("\t".join(labels[c] for c in r.items[int(r.offsets[k]):int(r.offsets[k + 1])].tolist()),
                 int(r.supports[k]), int(r.periods[k])) for k in range(len(r))] for a, r in last}
    ref_leg = None
    if not args.no_ref_gpu:
        from oracle import ref_gpu

        if ref_gpu.available():
            k = ref_gpu.RefKernels(local)
            limit = min(int(np.floor(maxper)), np.iinfo(np.int64).max)
            got = {}
            for warm in (True, False):
                t0 = time.perf_counter()
                for a in ("pf-eclat", "pf-apriori"):
                    found = ref_gpu.periodic_mine(baskets, ts.tolist(), end, ms_count, limit,
                                                  "eclat" if a == "pf-eclat" else "apriori", k)
                    got[a] = [("\t".join(p), s_, p_) for p, s_, p_ in found]
                spent = time.perf_counter() - t0
                if warm:
                    first = spent
            ref_leg = {"value": spent, "unit": "s", "first_call_s": first, "sample": "whole step, warm",
                       "identical_output": got == ours,
                       "kind": "reference periodic_counts and build_bitsets (cupami sources, nvcc sm_100a) "
                               "+ reference driver loops; torch tensors in place of CuPy arrays"}
        else:
            ref_leg = {"unavailable": "oracle/_ref/libref_bitsets.so not built"}
    cpu = None
    if not args.no_cpu_baseline:
        cpu = {"value": periodic_cpu_seconds(baskets, ts, minsup, maxper), "unit": "s", "cores": 1,
               "kind": "port", "sample": "whole step (NumPy restatement of the reference periodic miners)"}
    line = {
        "metric": "mine() seconds per step (pf-eclat+pf-apriori)",
        "value": value, "unit": "s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": value * 1e3, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "i64", "data": "synthetic",
        "config": {"workload": args.workload, "seed": seed, "minSup": minsup, "maxPer": maxper,
                   "transactions": n, "items": len(labels), "l2": "256 MB buffer rewritten before every timed step",
                   "parallelism": f"replicas{world}" if world > 1 else "single"},
        "e2e": {"value": e2e_v, "unit": "s", "h2d_bytes_per_step": 2 * (csr.offsets.nbytes + csr.nnz * 4 + ts.nbytes),
                "d2h_bytes_per_step": d2h},
        "roofline": roof,
        "cpu_baseline": cpu,
        "reference_gpu": ref_leg,
        "gpu_launches": launches,
        "clocks": clocks,
        "patterns": [len(r) for _, r in last],
        "kernel_stats": [r.stats for _, r in last],
    }
    print(json.dumps(line), flush=True)


def device_options(sched, args):
    from cupami_b200 import _native

    o = _native.Opts()
    _native.library().cpm_default_opts(o)
    o.scheduler = _native.CPM_SCHED_LEARNED if sched == "learned" else _native.CPM_SCHED_PLAIN
    o.arena_bytes = args.arena_mb << 20
    o.tidsets = args.tidsets
    return o


def deep_bound(traffic, alg_bytes):
    """What serves the deep kernel's bytes: DRAM when ncu saw at least half of
    the algorithmic bytes there, else the L2 (the working set stays on chip)."""
    if traffic is None or not alg_bytes:
        return "unmeasured"
    return "hbm" if traffic >= 0.5 * alg_bytes else "l2"


class Workload:
    """One synthetic database (or batch of databases) loaded on the device,
    with the device step, the public-API step and their timings."""

    def __init__(self, name, rank, local, args):
        import cupami_b200
        from cupami_b200 import _native

        self.name, self.args, self.local = name, args, local
        self.csr, self.minsup, self.algos, self.seed = make_workload(name, rank)
        self.batched = isinstance(self.csr, list)
        self.csrs = self.csr if self.batched else [self.csr]
        self.n_tx = n_transactions(self.csr)
        # The first public-API mine() of the process: library load, context,
        # module loading and allocator warm-up, then the step itself.
        self.first_call_s, _ = self.api_step(args.scheduler, materialise=False)
        self.ctx = _native.context(local)
        self.dbs = [_native.Database.from_ids(self.ctx, c.offsets, c.items) for c in self.csrs]
        self.ms_counts = [cupami_b200.cuApriori._getSupportCount(self.minsup, n_transactions(c)) for c in self.csrs]

    def close(self):
        for db in self.dbs:
            db.close()
        self.dbs = []

    def device_step(self, sched):
        """[(algorithm, stats, results)] of one step with resident tidsets."""
        from cupami_b200 import _native

        codes = {"eclat": (_native.CPM_ECLAT, _native.CPM_ORDER_ECLAT),
                 "apriori": (_native.CPM_APRIORI, _native.CPM_ORDER_APRIORI)}
        out = []
        for a in self.algos:
            if a == "eclat-batch":
                res = _native.mine_batch(self.ctx, self.dbs, self.ms_counts, device_options(sched, self.args))
                out.append((a, res[0].stats, res))
            else:
                code, order = codes[a]
                res = self.dbs[0].mine(self.ms_counts[0], code, device_options(sched, self.args), order)
                out.append((a, res.stats, [res]))
        return out

    def api_step(self, sched, materialise):
        """(seconds, d2h bytes) of one step through the public Python API from
        host arrays; with ``materialise`` the seconds also cover building the
        pattern dict of every miner (what the reference's mine() builds)."""
        import cupami_b200

        t, d2h = 0.0, 0
        for a in self.algos:
            if a == "eclat-batch":
                t0 = time.perf_counter()
                miners = cupami_b200.cuEclat.mineBatch(self.csrs, self.minsup)
                if materialise:
                    for m in miners:
                        m.getPatterns()
                t += time.perf_counter() - t0
                for m in miners:
                    off, it, sup, _ = m.getPatternArrays()
                    d2h += it.nbytes + sup.nbytes // 2 * 3
            else:
                m = (cupami_b200.cuEclat if a == "eclat" else cupami_b200.cuApriori)(self.csr, self.minsup)
                m.scheduler = sched
                m.mine()
                t += m.getMiningTime()
                if materialise:
                    t0 = time.perf_counter()
                    m.getPatterns()
                    t += time.perf_counter() - t0
                off, it, sup, _ = m.getPatternArrays()
                d2h += it.nbytes + sup.nbytes // 2 * 3
        return t, d2h

    def h2d_bytes(self):
        return sum(int(c.offsets.nbytes + c.items.nbytes) for c in self.csrs) * len(self.algos)


def timed_device(w, sched, steps, warmup, flush, barrier):
    for _ in range(warmup):
        w.device_step(sched)
    barrier()
    ms, kst, launches, last = [], [], 0, None
    for _ in range(steps):
        flush_l2(flush)
        torch_sync()
        out = w.device_step(sched)
        ms.append(sum(st["ms_total"] for _, st, _ in out))
        kst.append(out)
        launches += sum(int(st["kernel_launches"]) for _, st, _ in out)
        last = out
    barrier()
    return ms, kst, launches, last


def timed_api(w, sched, steps, warmup, flush, barrier, materialise=False):
    for _ in range(warmup):
        w.api_step(sched, materialise)
    barrier()
    e2e, d2h = [], 0
    for _ in range(steps):
        flush_l2(flush)
        torch_sync()
        t, d2h = w.api_step(sched, materialise)
        e2e.append(t)
    barrier()
    return e2e, d2h


def torch_sync():
    import torch

    torch.cuda.synchronize()


def other_workload(name, args, local, flush, steps=5, warmup=3):
    """value and e2e of a secondary workload (single rank), same definitions as the headline."""
    w = Workload(name, 0, local, args)
    try:
        ms, kst, launches, last = timed_device(w, args.scheduler, steps, warmup, flush, torch_sync)
        e2e, _ = timed_api(w, args.scheduler, steps, 1, flush, torch_sync)
        deep_ms = statistics.mean(sum(st["ms_deep"] for a, st, _ in out if a != "apriori") for out in kst)
        deep_bytes = statistics.mean(sum(st["bytes_alg"] for a, st, _ in out if a != "apriori") for out in kst)
        return {"value": statistics.mean(ms) / 1e3, "unit": "s", "e2e": statistics.mean(e2e),
                "first_call_s": w.first_call_s, "steps": steps, "seed": w.seed, "minSup": w.minsup,
                "algorithms": list(w.algos), "databases": len(w.csrs), "transactions": w.n_tx,
                "patterns": [int(st["n_patterns"]) for _, st, _ in last],
                "deep_ms": deep_ms, "deep_alg_gbs": deep_bytes / (deep_ms * 1e-3) / 1e9 if deep_ms else None,
                "apriori_ms": statistics.mean(sum(st["ms_total"] for a, st, _ in out if a == "apriori")
                                              for out in kst) if "apriori" in w.algos else None}
    finally:
        w.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="sparse-zipf-1m", choices=sorted(WORKLOADS))
    ap.add_argument("--scheduler", default="plain", choices=["plain", "learned"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-ab", action="store_true", help="skip the learned-vs-plain scheduler comparison")
    ap.add_argument("--no-ref-gpu", action="store_true", help="skip the reference-GPU-path leg")
    ap.add_argument("--no-others", action="store_true", help="skip the secondary workloads")
    ap.add_argument("--others", default="planted-100k,batched-zipf-512",
                    help="secondary workloads measured after the headline (comma separated)")
    ap.add_argument("--arena-mb", type=int, default=0,
                    help="deep-level arena size (memory-bounded rounds past it); 0 = automatic")
    ap.add_argument("--tidsets", type=int, default=0, choices=[0, 1, 2],
                    help="deep-level tidset forms: 0 automatic, 1 bitsets only, 2 lists wherever possible")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    world, rank, local = dist_setup()
    if args.workload in MAX_PER:
        return (run_periodic_reference if args.impl == "reference" else run_periodic)(args, world, rank, local)
    if args.impl == "reference":
        return run_reference(args, world, rank)
    run_ours(args, world, rank, local)


def run_ours(args, world, rank, local):
    import torch

    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
        pg = dist
    from cupami_b200 import _native, costmodel

    w = Workload(args.workload, rank, local, args)
    have_model = costmodel.ensure_default(w.ctx)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")  # 256 MB > L2

    def barrier():
        torch.cuda.synchronize()
        if pg:
            pg.barrier()

    sampler = ClockSampler(local)
    step_ms, per_kernel, launches, last = timed_device(w, args.scheduler, args.steps, args.warmup, flush, barrier)
    clocks = sampler.stop()
    # Scheduler A/B on the same resident data (Eclat deep phase only).
    ab = None
    if not args.no_ab and have_model and any(a != "apriori" for a in w.algos):
        other = "learned" if args.scheduler == "plain" else "plain"
        o_ms, o_kst, _, o_last = timed_device(w, other, args.steps, args.warmup, flush, barrier)
        deep = lambda kst: statistics.mean(sum(st["ms_deep"] for a, st, _ in out if a != "apriori") for out in kst)
        same = all(np.array_equal(r1.supports, r2.supports) and np.array_equal(r1.items, r2.items)
                   for (_, _, a1), (_, _, a2) in zip(last, o_last) for r1, r2 in zip(a1, a2))
        times = {args.scheduler: (statistics.mean(step_ms), deep(per_kernel)), other: (statistics.mean(o_ms), deep(o_kst))}
        ab = {"plain_ms": times["plain"][0], "learned_ms": times["learned"][0],
              "plain_deep_ms": times["plain"][1], "learned_deep_ms": times["learned"][1],
              "speedup_step": times["plain"][0] / times["learned"][0],
              "speedup_deep": times["plain"][1] / times["learned"][1] if times["learned"][1] else None,
              "identical_output": bool(same)}
    # e2e through the public API from host arrays: arrays only (the headline),
    # then with the pattern dict built as the reference's mine() does.
    e2e, d2h = timed_api(w, args.scheduler, args.steps, args.warmup, flush, barrier)
    e2e_dict, _ = timed_api(w, args.scheduler, max(1, min(3, args.steps)), 0, flush, barrier, materialise=True)
    value = statistics.mean(step_ms) / 1e3
    e2e_v = statistics.mean(e2e)
    e2e_dict_v = statistics.mean(e2e_dict)
    if pg:
        value, e2e_v, e2e_dict_v = max_over_ranks([value, e2e_v, e2e_dict_v], "cuda")
        # The last collective: rank 0's baselines below run on its own, so no
        # rank waits on a barrier while they do.
        pg.destroy_process_group()
    # Roofline of the deep phase (k_deep, then k_local for the units below
    # projected prefixes), the step's dominant part on Eclat workloads, from
    # its own CUDA events.
    hbm, bf16, src = peaks()
    eclat_stats = [[st for a, st, _ in out if a != "apriori"] for out in per_kernel]
    roof = None
    if eclat_stats and eclat_stats[0]:
        deep_ms = statistics.mean(sum(s["ms_deep"] for s in st) for st in eclat_stats)
        deep_bytes = statistics.mean(sum(s["bytes_alg"] for s in st) for st in eclat_stats)
        local_ms = statistics.mean(sum(s.get("ms_local", 0.0) for s in st) for st in eclat_stats)
        proj_units = statistics.mean(sum(s.get("projected_units", 0) for s in st) for st in eclat_stats)
        row_units = statistics.mean(sum(s.get("row_units", 0) for s in st) for st in eclat_stats)
        units = statistics.mean(sum(s.get("work_items", 0) for s in st) for st in eclat_stats)
        achieved = deep_bytes / (deep_ms * 1e-3) / 1e9 if deep_ms else 0.0
        tr = deep_traffic(args.workload, args.tidsets, args.arena_mb)
        traffic = tr["dram_bytes_per_launch"] if tr else None
        roof = {"kernel": "deep phase: k_deep (persistent, a CTA per unit) then k_local (a warp per projected unit)",
                "bound": deep_bound(traffic, deep_bytes),
                "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm, "traffic": traffic,
                "peak_source": src, "frac_of": "HBM copy bandwidth (" + src + "); algorithmic bytes / kernel time",
                "frac_of_8tbs_spec": achieved / 8000.0,
                "dram_share_of_alg_bytes": traffic / deep_bytes if traffic and deep_bytes else None,
                "l2_bytes_per_launch": tr.get("l2_bytes_per_launch") if tr else None,
                # per kernel: DRAM and L2 bytes, L2 bytes/s and the L2 throughput % of peak (ncu)
                "by_kernel": tr.get("kernels") if tr else None,
                "traffic_source": ("profiles/k_deep_traffic.json (ncu dram__bytes_read.sum + dram__bytes_write.sum "
                                   "of one launch of each kernel): " + tr["profile"]) if tr else None,
                "ms_per_launch": deep_ms, "ms_k_local": local_ms, "alg_bytes_per_launch": deep_bytes,
                "units": units, "projected_units": proj_units, "row_units": row_units,
                "alg_bytes": "sum over units of the prefix, every sibling and every child written, each at its "
                             "own form's size (bitset 8*W, list 16 + 4*ids, projected bitset 16*ceil(n/128)); "
                             "row-wise units count their prefix's rows instead of the siblings (12 B per row "
                             "+ 2 B per frequent index)"}
    pair_ms = statistics.mean(sum(st["ms_pairs"] for _, st, _ in out) for out in per_kernel)
    pair_ops = statistics.mean(sum(st["pair_ops"] for _, st, _ in out) for out in per_kernel)
    int8_peak = int8_peak_tops()
    gram_tops = pair_ops / (pair_ms * 1e-3) / 1e12 if pair_ms else 0.0
    gram = {"kernel": "pair Gram (k_gram_tc when the tensor-core engine runs)", "ms_per_step": pair_ms,
            "ops_per_step": pair_ops, "tops": gram_tops, "peak_int8_tops": int8_peak,
            "peak_source": "torch._int_mm int8 8192^3, best of 12, measured in this run",
            "frac": gram_tops / int8_peak if int8_peak else None,
            "ops": "2*128*256*K per issued tile (full tiles of the upper triangle)"}
    if rank != 0:
        w.close()
        return
    ref_gpu_leg = None
    if not args.no_ref_gpu:
        ours = [[r.patterns(db.labels) for r in res] for db, res in
                zip(w.dbs, zip(*[res for _, _, res in last]))]
        ref_gpu_leg = reference_gpu_seconds(w.csr, w.minsup, w.algos, ours, local)
        del ours
    last_stats = [st for _, st, _ in last]
    w.close()
    cpu = None
    if not args.no_cpu_baseline:
        counts = search_counts(args.workload)
        if counts and w.algos == ("eclat",):
            model = ReferenceCpuModel(w.csr, *counts)
            v, parts = model.sample(seed=0)
            cpu = {"value": v, "unit": "s", "cores": 1, "kind": "port", "estimated": True,
                   "sample": "estimate of the NumPy restatement of the reference host path: label mapping, "
                             "packing and singletons run in full; every other driver operation timed on samples "
                             "of the real tidsets and scaled by its exact count on this database",
                   "parts_s": {k: round(x, 2) for k, x in parts.items()}}
        else:
            v, sample = cpu_step_seconds(w.csr, w.minsup, w.algos)
            cpu = {"value": v, "unit": "s", "cores": 1, "kind": "port", "estimated": False,
                   "sample": f"{sample} (NumPy restatement of the reference host path)"}
    others = None
    if not args.no_others and world == 1:
        others = {}
        for name in [x for x in args.others.split(",") if x and x != args.workload]:
            others[name] = other_workload(name, args, local, flush)
    line = {
        "metric": "mine() seconds per step (" + "+".join(w.algos) + ")",
        "value": value, "unit": "s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": value * 1e3, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": value / PUBLISHED[args.workload] if args.workload in PUBLISHED else None,
        "dtype": "u64", "data": "synthetic",
        "config": {"workload": args.workload, "seed": w.seed, "minSup": w.minsup, "algorithms": list(w.algos),
                   "databases": len(w.csrs), "transactions": w.n_tx, "scheduler": args.scheduler,
                   "l2": "256 MB buffer rewritten before every timed step",
                   "parallelism": f"replicas{world}" if world > 1 else "single"},
        "e2e": {"value": e2e_v, "unit": "s", "h2d_bytes_per_step": w.h2d_bytes(), "d2h_bytes_per_step": d2h,
                "with_pattern_dict_s": e2e_dict_v, "first_call_s": w.first_call_s,
                "api": "cuEclat/cuApriori(TransactionCSR, minSup).mine() + getPatternArrays(); "
                       "with_pattern_dict_s adds getPatterns() (the dict the reference's mine() builds); "
                       "first_call_s is the process's first mine(), library and context set-up included"},
        "roofline": roof,
        "pair_gram": gram,
        "cpu_baseline": cpu,
        "reference_gpu": ref_gpu_leg,
        "scheduler_ab": ab,
        "gpu_launches": launches,
        "clocks": clocks,
        "patterns": [int(st["n_patterns"]) for st in last_stats],
        "kernel_stats": last_stats,
        "others": others,
    }
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
