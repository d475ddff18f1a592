"""Periodic-frequent miners (cuPFEclat / cuPFApriori) and the periodic_counts kernel.

CPU part: the oracle (oracle/periodic.py) against the reference miners' own
outputs (golden/periodic_patterns.json, made by golden/make_periodic_golden.py)
and against a brute force; the depth-first and level orders built from
shuffled pattern trees by the C ABI; the temporal input rules.
GPU part: the drop-in miners and cpm_periodic_counts against the same
fixtures and the oracle -- supports and periodicities exact, order included.
"""
import json
import struct
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).parent / "golden" / "periodic_patterns.json"


@pytest.fixture(scope="module")
def fixtures():
    return json.loads(GOLDEN.read_text())


def _runs(fixtures):
    for case in fixtures["cases"]:
        for run in case["results"]:
            yield case, run


# ---- CPU: the oracle against the reference's own outputs ---------------------

def test_oracle_reproduces_reference_miners(fixtures):
    from oracle import periodic

    checked = 0
    for case, run in _runs(fixtures):
        for name, algo in (("cuPFEclat", "eclat"), ("cuPFApriori", "apriori")):
            got = periodic.mine(case["rows"], run["minSup"], run["maxPer"], algo, run["endTime"])
            assert [[k, s, p] for k, (s, p) in got.items()] == run[name], (case["name"], name)
            checked += 1
    assert checked == 2 * sum(len(c["results"]) for c in fixtures["cases"])


def test_paper_example_known_answer(fixtures):
    run = fixtures["cases"][0]["results"][0]
    assert len(run["cuPFApriori"]) == 9
    assert ["a\tb", 4, 3] in run["cuPFApriori"]


def test_oracle_matches_brute_force(fixtures):
    from oracle import periodic

    for case, run in _runs(fixtures):
        labels = {str(x).strip() for r in case["rows"] for x in r[1:]}
        if len(labels) > 12:
            continue
        want = periodic.brute_force(case["rows"], run["minSup"], run["maxPer"], run["endTime"])
        got = periodic.mine(case["rows"], run["minSup"], run["maxPer"], "apriori", run["endTime"])
        assert got == want, case["name"]


def _tree(patterns, rng, prefix_tree):
    """Pattern tree of (sorted column tuple, support, period) in a random emission order."""
    order = sorted(range(len(patterns)), key=lambda i: (len(patterns[i][0]), rng.random()))
    by_set, parent, item, support, period = {}, [], [], [], []
    for new_id, i in enumerate(order):
        items, sup, per = patterns[i]
        if len(items) == 1:
            parent.append(-1)
            item.append(items[0])
        else:
            drop = len(items) - 1 if prefix_tree else int(rng.integers(len(items)))
            parent.append(by_set[frozenset(items[:drop] + items[drop + 1:])])
            item.append(items[drop])
        support.append(sup)
        period.append(per)
        by_set[frozenset(items)] = new_id
    return parent, item, support, period


@pytest.mark.parametrize("prefix_tree", [False, True])
@pytest.mark.parametrize("name,order", [("cuPFEclat", 3), ("cuPFApriori", 1)])
def test_insertion_order_from_shuffled_trees(fixtures, name, order, prefix_tree):
    from cupami_b200._native import Result

    rng = np.random.default_rng(1)
    checked = 0
    for case, run in _runs(fixtures):
        pats = [(k.split("\t"), s, p) for k, s, p in run[name]]
        if not pats:
            continue
        labels = sorted({x for p, _, _ in pats for x in p})
        col = {x: i for i, x in enumerate(labels)}
        patterns = [(tuple(sorted(col[x] for x in p)), s, per) for p, s, per in pats]
        parent, item, support, period = _tree(patterns, rng, prefix_tree)
        res = Result.from_tree(parent, item, support, order, period=period)
        o = res.offsets.tolist()
        got = [["\t".join(labels[c] for c in res.items[o[k]:o[k + 1]].tolist()), int(res.supports[k]),
                int(res.periods[k])] for k in range(len(res))]
        assert got == run[name], (case["name"], name)
        checked += 1
    assert checked >= 12


# ---- CPU: temporal input rules -------------------------------------------------

@pytest.mark.parametrize("cls_name", ["cuPFEclat", "cuPFApriori"])
def test_input_files_read_as_the_reference_reads_them(tmp_path, fixtures, cls_name):
    """Temporal CSV/TSV/whitespace text (BOM, blank lines and values, explicit
    separator), CUPAMIT1 BIN and Parquet files: timestamps, baskets, row count
    and resolved thresholds equal the reference constructor's."""
    import base64

    import cupami_b200

    inputs = fixtures["inputs"]
    for name, content in inputs["files"].items():
        path = tmp_path / name
        if "text" in content:
            path.write_bytes(content["text"].encode("utf-8"))
        else:
            path.write_bytes(base64.b64decode(content["base64"]))
    cls = getattr(cupami_b200, cls_name)
    for run in inputs["runs"]:
        m = cls(tmp_path / run["file"], run["minSup"], run["maxPer"], run["sep"], endTime=run["endTime"])
        got = {"timestamps": m._timestamps, "baskets": [list(b) for b in m._Database],
               "transactions": m._transactionCount, "resolvedMinSup": m._minSup,
               "resolvedMaxPer": m._maxPer, "end": m._endTimestamp}
        assert got == {k: run[k] for k in got}, run["file"]
    assert len(inputs["runs"]) >= 8


@pytest.mark.parametrize("index", [0, 1])
def test_save_and_dataframe_match_the_reference(tmp_path, fixtures, inject, index):
    """save() lines "{pattern} : {support} : {periodicity}" and the DataFrame
    (Patterns, Support, Periodicity), the reference's own, from its patterns
    (_temporal.py:173-181); the result is given to the miner on the host."""
    import cupami_b200
    from cupami_b200 import _native

    case = fixtures["outputs"][index]
    cls = getattr(cupami_b200, case["algorithm"])
    order = _native.CPM_ORDER_DEPTH_FIRST if case["algorithm"] == "cuPFEclat" else _native.CPM_ORDER_APRIORI
    m = inject(cls(case["rows"], case["minSup"], case["maxPer"]), case["patterns"], order)
    assert [[k, s, p] for k, (s, p) in m.getPatterns().items()] == case["patterns"]
    m.save(tmp_path / "out.txt")
    assert (tmp_path / "out.txt").read_text(encoding="utf-8") == case["save"]
    df = m.getPatternsAsDataFrame()
    assert list(df.columns) == case["columns"]
    assert [[str(a), int(b), int(c)] for a, b, c in df.values.tolist()] == case["frame"]


# tests/test_miner_examples.py:52-72 of the reference: a manual known answer.
MANUAL_ROWS = [[1, 1, 2], [1, 2, 3], [3, 1, 3], [5, 1, 2, 3], [8]]
MANUAL_EXPECTED = {"1": (3, 3), "2": (3, 4), "3": (3, 3), "1\t2": (2, 4), "1\t3": (2, 3), "2\t3": (2, 4)}


def _manual_files(directory):
    csv_path = directory / "manual.csv"
    csv_path.write_text("".join(",".join(map(str, r)) + "\n" for r in MANUAL_ROWS), encoding="utf-8")
    offsets, flat = [0], []
    for r in MANUAL_ROWS:
        flat.extend(r[1:])
        offsets.append(len(flat))
    bin_path = directory / "manual.bin"
    bin_path.write_bytes(struct.pack("<8sQQQ", b"CUPAMIT1", len(MANUAL_ROWS), len(flat), 3)
                         + struct.pack(f"<{len(MANUAL_ROWS)}q", *[r[0] for r in MANUAL_ROWS])
                         + struct.pack(f"<{len(offsets)}Q", *offsets) + struct.pack(f"<{len(flat)}I", *flat))
    import pyarrow as pa
    import pyarrow.parquet as pq

    pq_path = directory / "manual.parquet"
    pq.write_table(pa.table({"timestamp": pa.array([r[0] for r in MANUAL_ROWS], pa.int64()),
                             "items": pa.array([r[1:] for r in MANUAL_ROWS], pa.list_(pa.uint32()))}), pq_path)
    return [MANUAL_ROWS, csv_path, bin_path, pq_path]


@pytest.mark.parametrize("support", [2, 0.4])
def test_manual_known_answer_on_the_oracle(tmp_path, support):
    import cupami_b200
    from oracle import periodic

    for algo in ("eclat", "apriori"):
        assert periodic.mine(MANUAL_ROWS, support, 4, algo) == MANUAL_EXPECTED
    ref = cupami_b200.cuPFEclat(MANUAL_ROWS, support, 4)
    for source in _manual_files(tmp_path)[1:]:  # every format reads as the rows do
        m = cupami_b200.cuPFEclat(source, support, 4)
        assert (m._timestamps, m._Database, m._minSup, m._endTimestamp) == \
            (ref._timestamps, ref._Database, ref._minSup, ref._endTimestamp), source


def test_temporal_rows_sorting_empties_and_thresholds():
    import cupami_b200

    m = cupami_b200.cuPFEclat([[9, "a"], [0, " a", "a ", "0"], [4], ["", " "], [9, "a", "b"], [15]], 0.5, 0.5)
    assert m._timestamps == [0, 4, 9, 9, 15]
    assert m._Database == [("a", "0"), (), ("a",), ("a", "b"), ()]
    assert m._transactionCount == 5 and m._minSup == 3
    assert m._endTimestamp == 15 and m._maxPer == 7.5 and m._periodLimit() == 7
    m = cupami_b200.cuPFApriori([[2, "x"], [3, "x"]], 1, 5, endTime=20)
    assert m._endTimestamp == 20 and m._maxPer == 5
    big = cupami_b200.cuPFApriori([[1, "x"]], 1, 1e30)
    assert big._periodLimit() == np.iinfo(np.int64).max


@pytest.mark.parametrize("cls_name", ["cuPFEclat", "cuPFApriori"])
def test_invalid_temporal_inputs(tmp_path, cls_name):
    import cupami_b200

    cls = getattr(cupami_b200, cls_name)
    for rows in ([[-1, "a"]], [[1.2, "a"]], [["bad", "a"]], [[2**63, "a"]]):
        with pytest.raises(ValueError):
            cls(rows, 1, 2)
    for support, period in [(0, 1), (1, -1), (1, float("nan")), (float("inf"), 1), (True, 1), (1, True)]:
        with pytest.raises((ValueError, OverflowError)):
            cls([[1, "a"]], support, period)
    with pytest.raises(ValueError):
        cls([[5, "a"]], 1, 2, endTime=3)
    path = tmp_path / "transactional.bin"
    path.write_bytes(b"CUPAMI01" + bytes(24))
    with pytest.raises(ValueError, match="temporal BIN"):
        cls(path, 1, 2)


def test_temporal_text_bin_and_parquet_inputs(tmp_path):
    import pyarrow as pa
    import pyarrow.parquet as pq

    import cupami_b200

    tab = tmp_path / "tab.txt"
    tab.write_text("1\ta\tb\n3\ta\n5\tb\n")
    assert cupami_b200.cuPFApriori(tab, 1, 5)._timestamps == [1, 3, 5]
    space = tmp_path / "space.txt"
    space.write_text("4 x y\n\n2 y\n")
    m = cupami_b200.cuPFApriori(space, 1, 5)
    assert m._timestamps == [2, 4] and m._Database == [("y",), ("x", "y")]
    rows = [[3, 7, 7, 1], [1], [2, 4294967295]]
    offsets, flat = [0], []
    for r in rows:
        flat.extend(r[1:])
        offsets.append(len(flat))
    path = tmp_path / "t.bin"
    path.write_bytes(struct.pack("<8sQQQ", b"CUPAMIT1", len(rows), len(flat), 4294967295)
                     + struct.pack(f"<{len(rows)}q", *[r[0] for r in rows])
                     + struct.pack(f"<{len(offsets)}Q", *offsets) + struct.pack(f"<{len(flat)}I", *flat))
    m = cupami_b200.cuPFEclat(path, 1, 3)
    assert m._timestamps == [1, 2, 3]
    assert m._Database == [(), ("4294967295",), ("7", "1")]
    path.write_bytes(path.read_bytes()[:-4])
    with pytest.raises(ValueError, match="size"):
        cupami_b200.cuPFEclat(path, 1, 3)
    table = pa.table({"timestamp": pa.array([r[0] for r in rows], pa.int64()),
                      "items": pa.array([r[1:] for r in rows], pa.list_(pa.uint32()))})
    pq.write_table(table, tmp_path / "t.parquet")
    m = cupami_b200.cuPFEclat(tmp_path / "t.parquet", 1, 3)
    assert m._timestamps == [1, 2, 3] and m._Database == [(), ("4294967295",), ("7", "1")]


def _row_pairs(offsets, cols):
    o = np.asarray(offsets, dtype=np.int64)
    return [sorted(set(cols[o[r]:o[r + 1]].tolist())) for r in range(o.size - 1)]


@pytest.mark.parametrize("seed,large_ids", [(0, True), (1, True), (2, False), (3, False)])
def test_temporal_csr_input_builds_the_string_paths_tidsets(seed, large_ids):
    """A TemporalCSR (integer ids, unsorted timestamps, repeated ids in a row,
    empty rows) gives the same labels, rows, timestamps and thresholds as the
    same data given as rows -- the arrays handed to cpm_tdb_from_csr agree."""
    import cupami_b200
    from cupami_b200.datasets import TemporalCSR

    rng = np.random.default_rng(seed)
    n = 500
    lengths = rng.integers(0, 6, n)
    offsets = np.zeros(n + 1, dtype=np.uint64)
    np.cumsum(lengths, out=offsets[1:])
    pool = [1, 2, 3, 10, 11, 20, 100, 4294967295] if large_ids else [0, 1, 2, 3, 10, 11, 20, 100, 1000, 99]
    ids = rng.choice(np.array(pool, dtype=np.uint32), int(offsets[-1]))
    ts = rng.integers(0, 300, n).astype(np.int64)
    tcsr = TemporalCSR(offsets, ids, ts)
    for cls in (cupami_b200.cuPFEclat, cupami_b200.cuPFApriori):
        a = cls(tcsr, 0.05, 0.2)
        b = cls(tcsr.rows(), 0.05, 0.2)
        assert a._Database is None and a.getInputBackend()["backend"] == "numpy-cuda"
        assert (a._transactionCount, a._minSup, a._endTimestamp, a._maxPer) == \
            (b._transactionCount, b._minSup, b._endTimestamp, b._maxPer)
        assert a._timestamps == b._timestamps
        oa, ca, na, tsa, la = a._temporalColumns()
        ob, cb, nb, tsb, lb = b._temporalColumns()
        assert la == lb and na == nb and np.array_equal(tsa, tsb)
        assert _row_pairs(oa, ca) == _row_pairs(ob, cb)


def test_temporal_csr_input_checks():
    import cupami_b200
    from cupami_b200.datasets import TemporalCSR

    off = np.array([0, 1, 2], dtype=np.uint64)
    ids = np.array([1, 2], dtype=np.uint32)
    with pytest.raises(ValueError):
        cupami_b200.cuPFEclat(TemporalCSR(off, ids, np.array([1, -1])), 1, 2)
    with pytest.raises(ValueError):
        cupami_b200.cuPFEclat(TemporalCSR(off, ids, np.array([1])), 1, 2)
    with pytest.raises(ValueError):
        cupami_b200.cuPFEclat(TemporalCSR(np.array([0, 2, 1], dtype=np.uint64), ids, np.array([1, 2])), 1, 2)
    with pytest.raises(ValueError):
        cupami_b200.cuPFEclat(TemporalCSR(off, ids, np.array([1.5, 2.0])), 1, 2)
    with pytest.raises(ValueError):
        cupami_b200.cuPFEclat(TemporalCSR(off, ids, np.array([5, 1])), 1, 2, endTime=3)
    m = cupami_b200.cuPFApriori(TemporalCSR(np.zeros(1, np.uint64), np.zeros(0, np.uint32),
                                            np.zeros(0, np.int64)), 1, 0)
    assert m._transactionCount == 0 and m._temporalColumns()[2] == 0


def test_temporal_workload_generator():
    """The benchmark's temporal database: seeded, one row per transaction, empty
    baskets kept, timestamps sorted with repeats, planted patterns periodic."""
    from cupami_b200 import datasets

    csr, ts = datasets.temporal_planted(n=20_000, seed=5)
    again, ts2 = datasets.temporal_planted(n=20_000, seed=5)
    assert np.array_equal(csr.offsets, again.offsets) and np.array_equal(csr.items, again.items)
    assert np.array_equal(ts, ts2) and ts.dtype == np.int64
    lengths = np.diff(csr.offsets.astype(np.int64))
    assert csr.n_transactions == 20_000 == ts.size
    assert 0.01 < np.mean(lengths == 0) < 0.03  # empty baskets kept
    assert np.all(np.diff(ts) >= 0) and np.any(np.diff(ts) == 0) and ts[0] >= 0
    for r in range(0, 20_000, 997):  # baskets are sets of ids in [1, 200]
        basket = csr.items[csr.offsets[r]:csr.offsets[r + 1]]
        assert np.unique(basket).size == basket.size and (basket.size == 0 or basket.min() >= 1)
    assert csr.items.max() <= 200


def test_temporal_workload_mines_deep_patterns_on_the_oracle():
    """At the benchmark's thresholds a quarter-size database still yields periodic
    patterns several items long (the workload exercises the level loop)."""
    from cupami_b200 import datasets
    from oracle import periodic

    csr, ts = datasets.temporal_planted(n=25_000, seed=23)
    o, it = csr.offsets.tolist(), csr.items.tolist()
    rows = [[int(t), *it[o[i]:o[i + 1]]] for i, t in enumerate(ts.tolist())]
    got = periodic.mine(rows, 0.005, 2500 // 4, "apriori")
    lengths = [len(k.split("\t")) for k in got]
    assert len(got) > 100 and max(lengths) >= 4


# ---- GPU: the drop-in miners against the reference's outputs ------------------

@pytest.mark.gpu
@pytest.mark.parametrize("name", ["cuPFEclat", "cuPFApriori"])
def test_gpu_miners_match_reference(fixtures, name):
    import cupami_b200

    cls = getattr(cupami_b200, name)
    for case, run in _runs(fixtures):
        miner = cls(case["rows"], run["minSup"], run["maxPer"], endTime=run["endTime"])
        miner.mine()
        got = [[k, s, p] for k, (s, p) in miner.getPatterns().items()]
        assert got == run[name], (case["name"], run["minSup"], run["maxPer"])
        miner.mine()  # mining again gives the same answer
        assert [[k, s, p] for k, (s, p) in miner.getPatterns().items()] == run[name]


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["cuPFEclat", "cuPFApriori"])
def test_gpu_manual_known_answer_all_formats(tmp_path, name):
    import cupami_b200

    cls = getattr(cupami_b200, name)
    for source in _manual_files(tmp_path):
        for support in (2, 0.4):
            m = cls(source, support, maxPer=4)
            m.mine()
            assert m.getPatterns() == MANUAL_EXPECTED, (source, support)


@pytest.mark.gpu
def test_gpu_temporal_csr_input_matches_rows():
    import cupami_b200
    from cupami_b200 import datasets

    csr, ts = datasets.temporal_planted(n=30_000, seed=9)
    tcsr = datasets.TemporalCSR(csr.offsets, csr.items, ts[::-1].copy())  # unsorted rows
    rows = tcsr.rows()
    for cls in (cupami_b200.cuPFEclat, cupami_b200.cuPFApriori):
        a = cls(tcsr, 0.005, 900)
        a.mine()
        b = cls(rows, 0.005, 900)
        b.mine()
        assert list(a.getPatterns().items()) == list(b.getPatterns().items())
        assert len(a.getPatterns()) > 50


@pytest.mark.gpu
def test_gpu_output_apis(tmp_path, fixtures):
    import cupami_b200

    case = fixtures["cases"][0]
    miner = cupami_b200.cuPFApriori(case["rows"], 3, 3)
    miner.mine()
    df = miner.getPatternsAsDataFrame()
    assert list(df.columns) == ["Patterns", "Support", "Periodicity"] and len(df) == 9
    out = tmp_path / "patterns.txt"
    miner.save(out)
    lines = out.read_text().splitlines()
    assert "a\tb : 4 : 3" in lines and lines == sorted(lines, key=lambda x: tuple(x.split(" : ")[0].split("\t")))
    assert miner.getRuntime() >= 0 and miner.getInputBackend()["backend"] == "cpu"
    assert miner.getKernelStats()["n_patterns"] == 9


def _random_temporal(seed, n_rows, n_items, density=(0.2, 0.9), max_step=5):
    rng = np.random.default_rng(seed)
    p = rng.uniform(*density, n_items)
    ts = np.cumsum(rng.integers(0, max_step, n_rows))
    return [[int(t), *[f"v{j}" for j in np.nonzero(rng.random(n_items) < p)[0]]] for t in ts]


@pytest.mark.gpu
@pytest.mark.parametrize("seed,n_rows,n_items", [(5, 20000, 14), (6, 70001, 10), (7, 3000, 40)])
def test_gpu_miners_match_oracle_on_larger_inputs(seed, n_rows, n_items):
    """Many 64-row words, ragged last word, deep levels; both miners, order included."""
    import cupami_b200
    from oracle import periodic

    rows = _random_temporal(seed, n_rows, n_items, density=(0.3, 0.95) if n_items <= 20 else (0.05, 0.6))
    end = rows[-1][0]
    for min_sup, max_per in ((0.25, max(6, end // 400)), (0.1, end // 50)):
        labels, bits, timestamps, end_ts = periodic.prepare(rows)
        count, limit = periodic.thresholds(min_sup, max_per, len(timestamps), end_ts)
        want_a = periodic.pf_apriori(labels, bits, timestamps, end_ts, count, limit)
        for name, want in (("cuPFApriori", want_a), ("cuPFEclat", None)):
            miner = getattr(cupami_b200, name)(rows, min_sup, max_per)
            miner.mine()
            got = [(k, s, p) for k, (s, p) in miner.getPatterns().items()]
            if want is None:
                want = periodic.pf_eclat(labels, bits, timestamps, end_ts, count, limit)
            assert got == [("\t".join(p), s, per) for p, s, per in want], (name, min_sup, max_per)


@pytest.mark.gpu
def test_gpu_periodic_counts_kernel_exact():
    """cpm_periodic_counts (the reference kernel's drop-in) on random candidates:
    supports and periodicities equal the oracle's for every candidate, passing or not."""
    import torch

    from cupami_b200.frequentPattern import _bitsets
    from cupami_b200.periodicFrequentPattern import _temporal
    from oracle import periodic

    rng = np.random.default_rng(11)
    for n_rows, n_items, base in ((1, 3, 0), (31, 5, 7), (32, 5, 0), (33, 6, 2**40), (1000, 12, 0), (4097, 9, 2**53),
                                  (100000, 6, 0)):
        rows = _random_temporal(int(rng.integers(1 << 30)), n_rows, n_items, density=(0.05, 0.95))
        for r in rows:
            r[0] += base
        labels, bits, timestamps, end = periodic.prepare(rows, end_time=rows[-1][0] + 3)
        if not labels:
            continue
        d_bits = torch.from_numpy(bits.view(np.int32).copy()).cuda()
        d_ts = torch.from_numpy(timestamps.copy()).cuda()
        for width in (1, 2, 3, len(labels)):
            cands = [sorted(rng.choice(len(labels), size=min(width, len(labels)), replace=False).tolist())
                     for _ in range(50)]
            got = _temporal.periodic_counts(d_bits, cands, d_ts, len(timestamps), end)
            assert got == periodic.periodic_counts(bits, cands, timestamps, len(timestamps), end), (n_rows, width)
        # fewer transactions than bitset rows: rows past n are skipped
        cut = max(0, len(timestamps) - 5)
        cands = [[c] for c in range(len(labels))]
        assert (_temporal.periodic_counts(d_bits, cands, d_ts, cut, end)
                == periodic.periodic_counts(bits, cands, timestamps, cut, end))
    assert _bitsets is not None


@pytest.mark.gpu
def test_gpu_periodic_counts_kernel_any_timestamps():
    """The drop-in kernel is exact on any timestamps, as the reference kernel's
    scan is: unsorted and negative timestamps, negative, zero and positive ends
    (the periodicity then starts from 0, _temporal.py:38-53)."""
    import torch

    from cupami_b200.periodicFrequentPattern import _temporal
    from oracle import periodic

    rng = np.random.default_rng(21)
    for n_rows, n_items in ((700, 3), (3000, 5), (40000, 4)):
        rows = [[0, *[f"v{j}" for j in range(n_items) if rng.random() < 0.4]] for _ in range(n_rows)]
        labels, bits, _, _ = periodic.prepare(rows)
        ts = rng.integers(-100, 100, n_rows).astype(np.int64)
        d_bits = torch.from_numpy(bits.view(np.int32).copy()).cuda()
        d_ts = torch.from_numpy(ts.copy()).cuda()
        singles = [[c] for c in range(len(labels))]
        pairs = [sorted(rng.choice(len(labels), 2, replace=False).tolist()) for _ in range(20)]
        for end in (-7, 0, 150):
            for cands in (singles, pairs):  # one candidate width per call, as the reference launches
                assert (_temporal.periodic_counts(d_bits, cands, d_ts, n_rows, end)
                        == periodic.periodic_counts(bits, cands, ts, n_rows, end)), (n_rows, end, len(cands[0]))


@pytest.mark.gpu
def test_gpu_empty_and_degenerate_inputs():
    import cupami_b200

    for cls in (cupami_b200.cuPFEclat, cupami_b200.cuPFApriori):
        m = cls([], 1, 0)
        m.mine()
        assert m.getPatterns() == {}
        m = cls([[3], [5]], 1, 10)  # only empty baskets: no items
        m.mine()
        assert m.getPatterns() == {}
        m = cls([[0, "x"], [0, "y"]], 1, 0)
        m.mine()
        assert m.getPatterns() == {"x": (1, 0), "y": (1, 0)}


@pytest.mark.gpu
def test_gpu_reference_kernel_agrees_with_fixtures(fixtures):
    """The reference's own periodic_counts (compiled from its source into
    oracle/_ref) under the restated drivers gives the fixtures' answers: the
    kernel statement used to make the fixtures is the reference kernel's."""
    from oracle import periodic, ref_gpu

    if not ref_gpu.available():
        pytest.skip("oracle/_ref/libref_bitsets.so is not built")
    kernels = ref_gpu.RefKernels(0)
    for case, run in _runs(fixtures):
        rows = case["rows"]
        labels, bits, timestamps, end = periodic.prepare(rows, run["endTime"])
        count, limit = periodic.thresholds(run["minSup"], run["maxPer"], len(timestamps), end)
        limit = min(int(np.floor(limit)), np.iinfo(np.int64).max)
        records = sorted(((int(str(r[0]).strip()), r) for r in rows if any(str(v).strip() for v in r)),
                         key=lambda x: x[0])
        baskets = []
        for _, r in records:
            items = []
            for v in r[1:]:
                label = str(v).strip()
                if label and label not in items:
                    items.append(label)
            baskets.append(tuple(items))
        for name, algo in (("cuPFEclat", "eclat"), ("cuPFApriori", "apriori")):
            found = ref_gpu.periodic_mine(baskets, timestamps.tolist(), end, count, limit, algo, kernels)
            assert [["\t".join(p), s, per] for p, s, per in found] == run[name], (case["name"], name)


@pytest.mark.parametrize("seed", range(6))
def test_depth_first_and_level_orders_on_random_families(seed):
    """For random downward-closed families of itemsets, the C ABI's
    CPM_ORDER_DEPTH_FIRST / CPM_ORDER_APRIORI rebuild, from trees in a random
    emission order, the insertion orders of the restated cuPFEclat /
    cuPFApriori drivers run with 'is in the family' as their acceptance test."""
    from itertools import combinations

    from cupami_b200._native import Result
    from oracle import periodic

    rng = np.random.default_rng(seed)
    n_items = int(rng.integers(4, 9))
    labels = [f"L{i}" for i in range(n_items)]
    # a random family closed under subsets: keep each itemset whose subsets are all kept, with probability p
    family = set()
    for width in range(1, n_items + 1):
        for combo in combinations(range(n_items), width):
            if all(sub in family for sub in combinations(combo, width - 1) if sub) and rng.random() < 0.7:
                family.add(combo)
    index = {label: i for i, label in enumerate(labels)}

    def counts(cands):  # support 1 and periodicity 0 inside the family, support 0 outside
        return [(1, 0) if tuple(sorted(c)) in family else (0, 0) for c in cands]

    for order, driver in ((3, periodic.pf_eclat), (1, periodic.pf_apriori)):
        want = [p for p, _, _ in driver(labels, None, None, 0, 1, 0, counts=counts)]
        assert {tuple(index[x] for x in p) for p in want} == family
        pats = [(tuple(index[x] for x in p), 1, 0) for p in want]
        for prefix_tree in (False, True):
            parent, item, support, period = _tree(pats, rng, prefix_tree)
            res = Result.from_tree(parent, item, support, order, period=period)
            o = res.offsets.tolist()
            got = [tuple(labels[c] for c in res.items[o[k]:o[k + 1]].tolist()) for k in range(len(res))]
            assert got == want, (seed, order, prefix_tree)
