"""C-ABI library: exports, host-side ordering logic, loader semantics (no GPU)."""
import re
import struct
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]


def test_library_exports_every_declared_symbol():
    import ctypes

    from cupami_b200 import _native

    header = (ROOT / "include" / "cupami_b200.h").read_text()
    declared = set(re.findall(r"\b(cpm_[a-z_]+)\s*\(", header))
    assert len(declared) >= 20
    lib = ctypes.CDLL(str(_native.LIB_PATH))
    missing = [name for name in sorted(declared) if not hasattr(lib, name)]
    assert not missing
    # the Python binding declares exactly the header's functions
    assert set(_native.declared_symbols()) == declared


def test_no_device_raises_loudly():
    import cupami_b200

    miner = cupami_b200.cuEclat([[1, 2]], 1)
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except ImportError:
        has_gpu = False
    if has_gpu:
        pytest.skip("a GPU is present")
    with pytest.raises(RuntimeError, match="CUDA device"):
        miner.mine()


def _random_tree(patterns, rng, prefix_tree=False):
    """A valid pattern tree for ``patterns`` built in a random emission order.

    With ``prefix_tree`` every parent is the pattern minus its largest item
    (the device's trees); otherwise a random item is dropped."""
    by_set = {}
    order = list(range(len(patterns)))
    # parents must precede children: shuffle within lengths, shortest first
    order.sort(key=lambda i: (len(patterns[i][0]), rng.random()))
    parent, item, support = [], [], []
    for new_id, i in enumerate(order):
        items, sup = patterns[i]
        if len(items) == 1:
            parent.append(-1)
            item.append(items[0])
        else:
            drop = len(items) - 1 if prefix_tree else int(rng.integers(len(items)))
            rest = frozenset(items[:drop] + items[drop + 1:])
            parent.append(by_set[rest])
            item.append(items[drop])
        support.append(sup)
        by_set[frozenset(items)] = new_id
    return parent, item, support


@pytest.mark.parametrize("prefix_tree", [False, True])
@pytest.mark.parametrize("algo,order", [("cuEclat", 0), ("cuApriori", 1)])
def test_reference_insertion_order_from_shuffled_trees(golden, algo, order, prefix_tree):
    from cupami_b200._native import Result

    rng = np.random.default_rng(0)
    checked = 0
    for case in golden["cases"]:
        for run in case["results"][algo]:
            pats = [k.split("\t") for k, _ in run["patterns"]]
            if not pats:
                continue
            labels = sorted({x for p in pats for x in p})
            col = {x: i for i, x in enumerate(labels)}
            patterns = [(tuple(sorted(col[x] for x in p)), s) for p, (_, s) in zip(pats, run["patterns"])]
            parent, item, support = _random_tree(patterns, rng, prefix_tree)
            res = Result.from_tree(parent, item, support, order)
            o = res.offsets.tolist()
            got = [("\t".join(labels[c] for c in res.items[o[k]:o[k + 1]].tolist()), int(res.supports[k]))
                   for k in range(len(res))]
            assert got == [tuple(p) for p in run["patterns"]], (case["name"], algo)
            checked += 1
    assert checked > 40


def test_invalid_tree_is_rejected():
    from cupami_b200._native import NativeError, Result

    with pytest.raises(NativeError):
        Result.from_tree([0], [1], [1], 0)  # a pattern cannot be its own parent


# ---- loader semantics (constructor runs on the host only) -------------------

def test_constructor_support_rule_and_cleaning():
    import cupami_b200

    rows = [[" a", "a ", "b"], [], ["b", 10]]
    m = cupami_b200.cuApriori(rows, 0.5)
    assert m._Database == [("a", "b"), ("b", "10")]
    assert m._transactionCount == 2 and m._minSup == 1
    assert cupami_b200.cuEclat(rows, 2.5)._minSup == 2
    assert cupami_b200.cuEclat(rows, 1.0)._minSup == 2
    with pytest.raises(ValueError):
        cupami_b200.cuEclat(rows, 1, use_gds="maybe")
    with pytest.raises(ValueError):
        cupami_b200.cuEclat(rows, 1, use_gds=True)


def test_bin_and_parquet_readers(tmp_path):
    import pyarrow as pa
    import pyarrow.parquet as pq

    import cupami_b200

    rows = [[1, 1, 2], [], [0, 2], [4294967295, 2]]
    offsets = [0]
    flat = []
    for r in rows:
        flat.extend(r)
        offsets.append(len(flat))
    path = tmp_path / "t.bin"
    path.write_bytes(struct.pack("<8sQQQ", b"CUPAMI01", len(rows), len(flat), 4294967295)
                     + struct.pack(f"<{len(offsets)}Q", *offsets) + struct.pack(f"<{len(flat)}I", *flat))
    m = cupami_b200.cuEclat(path, 1, use_gds=False)
    assert m._Database is None and m._transactionCount == 3
    assert m.getInputBackend()["backend"] == "numpy-cuda"
    m = cupami_b200.cuEclat(path, 1, use_gds=False, use_gpu_io=False)
    assert m._Database == [("1", "2"), ("0", "2"), ("4294967295", "2")]
    with pytest.raises(RuntimeError, match="GDS input requested"):
        cupami_b200.cuEclat(path, 1, use_gds=True)
    for bad in (b"short", struct.pack("<8sQQQ", b"INVALID!", 0, 0, 8),
                struct.pack("<8sQQQ", b"CUPAMI01", 1, 1, 8),
                struct.pack("<8sQQQ2QI", b"CUPAMI01", 1, 1, 8, 1, 1, 2),
                struct.pack("<8sQQQ3Q2I", b"CUPAMI01", 2, 2, 8, 0, 3, 2, 1, 2),
                struct.pack("<8sQQQ2QI", b"CUPAMI01", 1, 1, 8, 0, 1, 9)):
        path.write_bytes(bad)
        with pytest.raises(ValueError):
            cupami_b200.cuApriori(path, 1)
    pq_path = tmp_path / "t.parquet"
    pq.write_table(pa.table({"items": pa.array(rows, type=pa.list_(pa.uint32()))}), pq_path)
    m = cupami_b200.cuEclat(pq_path, 1)
    assert m._transactionCount == 3 and m._csr is not None
    m = cupami_b200.cuEclat(pq_path, 1, use_gpu_io=False)
    assert m._Database == [("1", "2"), ("0", "2"), ("4294967295", "2")]
    for table in (pa.table({"other": [1]}), pa.table({"items": ["1,2"]}),
                  pa.table({"items": pa.array([None], type=pa.list_(pa.uint32()))}),
                  pa.table({"items": pa.array([[None]], type=pa.list_(pa.uint32()))})):
        pq.write_table(table, pq_path)
        with pytest.raises(ValueError):
            cupami_b200.cuApriori(pq_path, 1)


def test_text_url_and_timing(tmp_path):
    import io
    from unittest.mock import patch

    import importlib

    import cupami_b200

    mod = importlib.import_module("cupami_b200.frequentPattern.cuApriori")

    data = b'"apple,pear"\tbanana\r\nbanana\tcherry\r\n'
    with patch.object(mod, "urlopen", return_value=io.BytesIO(data)):
        m = cupami_b200.cuEclat("https://example.test/t.csv", 1, sep="\t")
    assert m._Database == [("apple,pear", "banana"), ("banana", "cherry")]
    assert m.getMiningTime() == 0 and m.getLoadingTime() >= 0
    assert m.getTotalRuntime() == m.getLoadingTime()
    m._startTime, m._endTime = 100, 104
    assert m.getRuntime() == m.getMiningTime() == 4
    csv_path = tmp_path / "q.csv"
    csv_path.write_text('"apple,pear",banana\nbanana\n', encoding="utf-8")
    m = cupami_b200.cuApriori(csv_path, 1)
    assert m.getInputBackend()["backend"] == "cpu"
    assert m._Database == [("apple,pear", "banana"), ("banana",)]


@pytest.mark.parametrize("cls_name", ["cuEclat", "cuApriori"])
def test_input_files_read_as_the_reference_reads_them(tmp_path, golden, cls_name):
    """CSV/TSV text (detected or explicit separator, blank lines and values, a
    byte-order mark kept as the reference keeps it), CUPAMI01 BIN and Parquet:
    baskets, transaction count and resolved threshold equal the reference
    constructor's; the numeric BIN/Parquet path agrees on the counts."""
    import base64

    import cupami_b200

    inputs = golden["inputs"]
    for name, content in inputs["files"].items():
        data = content["text"].encode("utf-8") if "text" in content else base64.b64decode(content["base64"])
        (tmp_path / name).write_bytes(data)
    cls = getattr(cupami_b200, cls_name)
    for run in inputs["runs"]:
        path = tmp_path / run["file"]
        m = cls(path, run["minSup"], run["sep"], use_gds=False, use_gpu_io=False)
        got = {"baskets": [list(b) for b in m._Database], "transactions": m._transactionCount,
               "resolvedMinSup": m._minSup}
        assert got == {k: run[k] for k in got}, run["file"]
        if path.suffix in (".bin", ".parquet"):
            fast = cls(path, run["minSup"], run["sep"])
            assert (fast._transactionCount, fast._minSup) == (run["transactions"], run["resolvedMinSup"])
    assert len(inputs["runs"]) >= 8


@pytest.mark.parametrize("index", range(4))
def test_save_and_dataframe_match_the_reference(tmp_path, golden, inject, index):
    """save() text and getPatternsAsDataFrame() rows, byte for byte the
    reference's, from the reference's patterns (cuApriori.py:537-560)."""
    import cupami_b200
    from cupami_b200 import _native

    case = golden["outputs"][index]
    cls = getattr(cupami_b200, case["algorithm"])
    order = _native.CPM_ORDER_ECLAT if case["algorithm"] == "cuEclat" else _native.CPM_ORDER_APRIORI
    m = inject(cls(case["rows"], case["minSup"]), case["patterns"], order)
    assert [[k, v] for k, v in m.getPatterns().items()] == case["patterns"]
    m.save(tmp_path / "out.txt")
    assert (tmp_path / "out.txt").read_text(encoding="utf-8") == case["save"]
    df = m.getPatternsAsDataFrame()
    assert list(df.columns) == case["columns"]
    assert [[str(a), int(b)] for a, b in df.values.tolist()] == case["frame"]


@pytest.mark.parametrize("cls_name", ["cuEclat", "cuApriori"])
def test_timing_labels_exclude_idle_time(cls_name):
    """Loading time covers the constructor only, mining time mine() only
    (the reference's tests/test_miner_examples.py:18-28)."""
    from unittest.mock import patch

    import importlib

    import cupami_b200

    mod = importlib.import_module("cupami_b200.frequentPattern.cuApriori")
    cls = getattr(cupami_b200, cls_name)
    with patch.object(cls, "_readTransactions", return_value=[("a",)]), \
            patch.object(mod.time, "perf_counter", side_effect=[10, 12.5]):
        miner = cls([], 1, use_gpu_io=False, use_gds=False)
    assert miner.getLoadingTime() == 2.5
    assert miner.getMiningTime() == 0
    assert miner.getTotalRuntime() == 2.5
    miner._startTime, miner._endTime = 100, 104
    assert miner.getMiningTime() == 4 and miner.getRuntime() == 4
    assert miner.getTotalRuntime() == 6.5


def test_id_labels_are_decimal_strings_on_first_use():
    """Labels of integer-id databases: a sequence of the ids' decimal strings,
    built only when read (a batch of miners does not build them while mining)."""
    import numpy as np

    from cupami_b200.frequentPattern.cuApriori import IdLabels

    lab = IdLabels(np.array([7, 10, 300], dtype=np.uint32))
    assert lab._str is None and len(lab) == 3
    assert lab[1] == "10" and list(lab) == ["7", "10", "300"] and lab[-1] == "300"
    assert list(lab[0:2]) == ["7", "10"]
