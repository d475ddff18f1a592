"""GPU: the kernel-module drop-in, the hook-driven search and bounded waits."""
from itertools import combinations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rows(seed=3, n=600, n_items=12):
    rng = np.random.default_rng(seed)
    p = rng.uniform(0.2, 0.7, n_items)
    return [[int(i) for i in np.nonzero(rng.random(n_items) < p)[0]] for _ in range(n)]


def test_bitsets_module_matches_numpy():
    import torch

    from cupami_b200.frequentPattern import _bitsets

    rng = np.random.default_rng(0)
    n_tx, n_items, nnz = 1000, 37, 9000
    rows = rng.integers(0, n_tx, nnz).astype(np.uint64)
    cols = rng.integers(0, n_items, nnz).astype(np.uint32)
    xp = _bitsets.array_module()
    bits = _bitsets.build_bitsets(xp, xp.asarray(rows, dtype=xp.uint64), xp.asarray(cols, dtype=xp.uint32),
                                  n_tx, n_items)
    ref = np.zeros((n_items, (n_tx + 31) // 32), dtype=np.uint32)
    np.bitwise_or.at(ref, (cols.astype(np.int64), (rows // 32).astype(np.int64)),
                     np.left_shift(np.uint32(1), (rows % 32).astype(np.uint32)))
    got = bits.cpu().numpy().view(np.uint32)
    assert np.array_equal(got, ref)
    cands = [[int(a), int(b), int(c)] for a, b, c in rng.integers(0, n_items, (500, 3))]
    sup = _bitsets.count_supports(xp, bits, cands)
    want = np.bitwise_count(ref[[c[0] for c in cands]] & ref[[c[1] for c in cands]]
                            & ref[[c[2] for c in cands]]).sum(axis=1).tolist()
    assert sup == want
    children, sup = _bitsets.intersect_extensions(xp, bits[3], bits[5:20])
    want_children = ref[5:20] & ref[3]
    assert np.array_equal(children.cpu().numpy().view(np.uint32), want_children)
    assert sup == np.bitwise_count(want_children).sum(axis=1).tolist()
    assert _bitsets.count_supports(xp, bits, []) == []
    assert isinstance(torch.cuda.current_device(), int)


def test_hook_overrides_run_the_constrained_search(oracle_lib):
    """A cuSpatialEclat-style subclass: only pairwise 'neighbour' itemsets."""
    import cupami_b200

    rows = _rows()
    neighbours = {str(i): {str(j) for j in range(12) if abs(i - j) <= 3 and i != j} for i in range(12)}

    class Constrained(cupami_b200.cuEclat):
        def _candidatePairs(self, frequent, items):
            for k, left in enumerate(frequent):
                for right in frequent[k + 1:]:
                    if items[right] in neighbours[items[left]]:
                        yield left, right

        def _extensionBatch(self, cp, prefix, labels, bitsets, start, stop):
            allowed = set(neighbours[prefix[0]])
            for item in prefix[1:]:
                allowed &= neighbours[item]
            keep = [i for i in range(start, stop) if labels[i] in allowed]
            if not keep:
                return [], None
            return [labels[i] for i in keep], bitsets[cp.asarray(keep, dtype=cp.int64)]

    miner = Constrained(rows, 30)
    miner._PAIR_BATCH_SIZE = 7
    miner._INTERSECTION_BATCH_BYTES = 64
    miner.mine()
    full = oracle_lib.mine_rows(rows, 30)
    want = {k: v for k, v in full.items()
            if all(b in neighbours[a] for a, b in combinations(k.split("\t"), 2))}
    assert miner.getPatterns() == want
    assert any(k.count("\t") >= 2 for k in want)


def test_spin_limit_runs_out_and_context_survives(oracle_lib):
    import cupami_b200
    from cupami_b200._native import CPM_ETIMEOUT, NativeError

    rows = _rows(seed=9, n=3000, n_items=18)
    miner = cupami_b200.cuEclat(rows, 0.05)
    miner._SPIN_LIMIT = 1
    with pytest.raises(NativeError) as err:
        miner.mine()
    assert err.value.code == CPM_ETIMEOUT
    miner._SPIN_LIMIT = 0
    miner.mine()
    assert miner.getPatterns() == oracle_lib.mine_rows(rows, 0.05)


def test_cli_writes_reference_format(tmp_path):
    import subprocess
    import sys
    from pathlib import Path

    src = tmp_path / "t.csv"
    out = tmp_path / "p.txt"
    src.write_text("1,2\n1\n2\n")
    root = Path(__file__).resolve().parents[1]
    res = subprocess.run([sys.executable, "-m", "cupami_b200.frequentPattern.cuEclat", str(src), str(out), "2"],
                         capture_output=True, text=True, timeout=120, cwd=root)
    assert res.returncode == 0, res.stderr
    assert out.read_text() == "1 : 2\n2 : 2\n"


@pytest.mark.parametrize("arena_kb,project", [(64, 65408), (64, 1), (512, 1)])
def test_memory_bounded_rounds_are_exact(oracle_lib, arena_kb, project):
    """A small child-tidset arena forces bounded rounds, halving and shallow
    splits (with projected levels, whose children are smaller, and without)."""
    import cupami_b200
    from cupami_b200 import TransactionCSR

    rng = np.random.default_rng(21)
    p = rng.uniform(0.3, 0.85, 20)
    rows = [[int(i) for i in np.nonzero(rng.random(20) < p)[0]] for _ in range(4000)]
    csr = TransactionCSR.from_rows(rows, universe=20)
    m = cupami_b200.cuEclat(csr, 0.2)
    m._ARENA_BYTES = arena_kb * 1024
    m._DEEP_PROJECT = project
    m.mine()
    stats = m.getKernelStats()
    assert stats["deep_rounds"] > 1
    labels, arrays = oracle_lib.mine_csr(csr.offsets, csr.items, 0.2)
    assert list(m.getPatterns().items()) == list(oracle_lib.to_dict(labels, arrays).items())


def test_launch_shapes_and_autotuner_keep_output():
    """Every deep-level launch shape, and the autotuner's pick, mine the same patterns."""
    import cupami_b200
    from cupami_b200 import _native, datasets

    csr = datasets.dense_bernoulli(n=16384, n_items=96, seed=3)
    base = cupami_b200.cuEclat(csr, 0.6)
    base.mine()
    want = list(base.getPatterns().items())
    assert len(want) > 1000
    for block in (128, 256, 512, 1024):
        for ctas in (1, 2, 4):
            m = cupami_b200.cuEclat(csr, 0.6)
            m._DEEP_BLOCK, m._DEEP_CTAS_PER_SM = block, ctas
            m.mine()
            assert list(m.getPatterns().items()) == want, (block, ctas)
    tuned = cupami_b200.cuEclat(csr, 0.6).autotune()
    assert tuned["block"] in (128, 256, 512, 1024) and 1 <= tuned["ctas_per_sm"] <= 4 and tuned["ms_deep"] > 0
    assert tuned["list_div"] in (0, 1, 2, 4, 8)
    m = cupami_b200.cuEclat(csr, 0.6)
    m.mine()
    assert list(m.getPatterns().items()) == want
    bad = cupami_b200.cuEclat(csr, 0.6)
    bad._DEEP_BLOCK = 96
    with pytest.raises(_native.NativeError):
        bad.mine()


@pytest.mark.parametrize("name,minsup", [("planted_zipf", 0.005), ("uniform_poisson", 0.01),
                                         ("dense_bernoulli", 0.6)])
def test_list_and_bitset_tidsets_agree(oracle_lib, name, minsup):
    """Deep levels with transaction-id lists for sparse tidsets and with bitsets
    only give the same patterns, in order, as the oracle."""
    import cupami_b200
    from cupami_b200 import datasets

    csr = getattr(datasets, name)()
    out = []
    for tidsets in (2, 1):
        for balance in (1, 2):  # a warp per sibling, or siblings split over warps by size
            m = cupami_b200.cuEclat(csr, minsup)
            m._TIDSETS = tidsets
            m._DEEP_BALANCE = balance
            m.mine()
            out.append((list(m.getPatterns().items()), m.getKernelStats()))
    assert all(o[0] == out[0][0] for o in out)
    out = out[::2]
    labels, arrays = oracle_lib.mine_csr(csr.offsets, csr.items, minsup)
    assert dict(out[0][0]) == oracle_lib.to_dict(labels, arrays)
    if name == "planted_zipf":  # sparse deep levels: the lists move fewer bytes
        assert out[0][1]["bytes_alg"] < out[1][1]["bytes_alg"]


def test_lists_in_memory_bounded_rounds_and_batches(oracle_lib):
    from cupami_b200 import _native, cuEclat, datasets

    from cupami_b200 import TransactionCSR

    # Sparse items (p up to 0.3) at a low threshold: the deeper children are
    # held by under 1/32 of the 4000 transactions, so they become lists.
    rng = np.random.default_rng(22)
    p = rng.uniform(0.02, 0.3, 30)
    rows = [[int(i) for i in np.nonzero(rng.random(30) < p)[0]] for _ in range(4000)]
    csr = TransactionCSR.from_rows(rows, universe=30)
    labels, arrays = oracle_lib.mine_csr(csr.offsets, csr.items, 0.005)
    want = oracle_lib.to_dict(labels, arrays)
    for arena in (64 << 10, 0):
        m = cuEclat(csr, 0.005)
        m._ARENA_BYTES = arena
        m._TIDSETS = 2
        m._DEEP_PROJECT = 1  # child lists, not projected bitsets
        m.mine()
        assert m.getPatterns() == want
        if arena:
            assert m.getKernelStats()["deep_rounds"] > 1
    csrs = datasets.batched_zipf(limit=12)
    for tidsets in (2, 1):
        cls = type("E", (cuEclat,), {"_TIDSETS": tidsets})
        for csr, m in zip(csrs, cls.mineBatch(csrs, 0.01)):
            labels, arrays = oracle_lib.mine_csr(csr.offsets, csr.items, 0.01)
            assert m.getPatterns() == oracle_lib.to_dict(labels, arrays)


def test_interpreter_exit_with_live_databases():
    """A process that ends with databases still alive (a global, a traceback)
    exits cleanly: the context frees its databases before itself."""
    import subprocess
    import sys
    from pathlib import Path

    code = (
        "import numpy as np, cupami_b200._native as n\n"
        "ctx = n.context(0)\n"
        "off = np.array([0, 2, 3], np.uint64); ids = np.array([1, 2, 2], np.uint32)\n"
        "KEEP = n.Database.from_ids(ctx, off, ids)\n"
        "def f():\n"
        "    db = n.Database.from_ids(ctx, off, ids)\n"
        "    raise RuntimeError('left with a live database')\n"
        "f()\n"
    )
    root = Path(__file__).resolve().parents[1]
    r = subprocess.run([sys.executable, "-c", code], cwd=root, capture_output=True, text=True, timeout=240)
    assert r.returncode == 1, (r.returncode, r.stderr[-2000:])
    assert "left with a live database" in r.stderr


@pytest.mark.parametrize("name,minsup", [("planted_zipf", 0.005), ("uniform_poisson", 0.01),
                                         ("dense_bernoulli", 0.6), ("sparse_zipf_small", 0.003)])
def test_projected_levels_agree(oracle_lib, name, minsup):
    """Children of small prefixes numbered by rank within them (mined by the
    warp-per-unit kernel) give the same patterns, in order, as the deep kernel
    alone and as the oracle, with bitsets only and with lists."""
    import cupami_b200
    from cupami_b200 import datasets

    if name == "sparse_zipf_small":
        csr = datasets.sparse_zipf(n=50_000, n_items=2_000, mean=20, seed=5)
    else:
        csr = getattr(datasets, name)()
    out = {}
    # automatic, off, and prefixes of at most 1,000 / 16,384 / 65,408 transactions
    for project in (0, 1, 1000, 16384, 65408):
        for tidsets in (0, 1, 2):
            m = cupami_b200.cuEclat(csr, minsup)
            m._DEEP_PROJECT, m._TIDSETS = project, tidsets
            m.mine()
            out[project, tidsets] = (list(m.getPatterns().items()), m.getKernelStats())
    # Row-wise counting of small prefixes (one database, projection on), off and on.
    for rows in (0, 1):
        for tidsets in (0, 2):
            m = cupami_b200.cuEclat(csr, minsup)
            m._DEEP_PROJECT, m._TIDSETS, m._DEEP_ROWS = 65408, tidsets, rows
            m.mine()
            out["rows", rows, tidsets] = (list(m.getPatterns().items()), m.getKernelStats())
    want = out[1, 0][0]
    assert all(v[0] == want for v in out.values())
    assert out["rows", 1, 0][1]["row_units"] == 0
    if name == "sparse_zipf_small":  # list prefixes with many long list siblings
        assert out["rows", 0, 2][1]["row_units"] > 0
    labels, arrays = oracle_lib.mine_csr(csr.offsets, csr.items, minsup)
    assert dict(want) == oracle_lib.to_dict(labels, arrays)
    # Projection moved units to the warp-per-unit kernel; without it none.
    # (uniform_poisson has no frequent 3-itemset, and every dense_bernoulli
    # prefix holds over 39,000 transactions: nothing is projected there.)
    if name in ("planted_zipf", "sparse_zipf_small"):
        assert out[16384, 0][1]["projected_units"] > 0
        assert out[65408, 0][1]["projected_units"] >= out[16384, 0][1]["projected_units"]
    assert out[1, 0][1]["projected_units"] == 0


def test_projected_levels_in_rounds_and_batches(oracle_lib):
    """Projection inside memory-bounded rounds and batched launches stays exact."""
    from cupami_b200 import TransactionCSR, cuEclat, datasets

    rng = np.random.default_rng(23)
    p = rng.uniform(0.02, 0.4, 40)
    rows = [[int(i) for i in np.nonzero(rng.random(40) < p)[0]] for _ in range(6000)]
    csr = TransactionCSR.from_rows(rows, universe=40)
    labels, arrays = oracle_lib.mine_csr(csr.offsets, csr.items, 0.004)
    want = oracle_lib.to_dict(labels, arrays)
    for arena in (64 << 10, 512 << 10, 0):
        m = cuEclat(csr, 0.004)
        m._ARENA_BYTES = arena
        m._DEEP_PROJECT = 65408  # a small search: projected only when asked
        m.mine()
        assert m.getKernelStats()["projected_units"] > 0
        assert m.getPatterns() == want, arena
        if arena:
            assert m.getKernelStats()["deep_rounds"] > 1
    csrs = datasets.batched_zipf(limit=16)
    for project in (0, 1, 65408):
        cls = type("E", (cuEclat,), {"_DEEP_PROJECT": project})
        for c, m in zip(csrs, cls.mineBatch(csrs, 0.01)):
            labels, arrays = oracle_lib.mine_csr(c.offsets, c.items, 0.01)
            assert m.getPatterns() == oracle_lib.to_dict(labels, arrays)
