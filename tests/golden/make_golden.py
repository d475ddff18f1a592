"""Regenerate the golden fixtures from the reference miners themselves.

Run where the cuPAMI sources can be read: ``$CUPAMI_REFERENCE``, else a
directory named ``reference`` beside this repository's own directory.  The reference drivers ``cuEclat.mine``
and ``cuApriori.mine`` run unchanged; only their CUDA plumbing is replaced:

* ``cuApriori._getCudaModule`` returns a NumPy namespace with the CuPy calls
  the drivers make (``asarray``, ``concatenate``, ``unique``, ...);
* the three kernel wrappers of ``cupami/frequentPattern/_bitsets.py:91-125``
  are replaced by NumPy statements of the kernels at ``_bitsets.py:20-77``.

The fixtures record each case's input and the reference's ``getPatterns()``
as an ordered list, so the checks can compare insertion order as well as
content.  Nothing at test time reads the reference checkout.
"""

from __future__ import annotations

import json
import os
import random
import sys
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF = Path(os.environ.get("CUPAMI_REFERENCE", HERE.parents[2] / "reference"))


def numpy_cuda_namespace():
    ns = types.SimpleNamespace(**{name: getattr(np, name) for name in (
        "asarray", "concatenate", "uint32", "uint64", "int64", "zeros", "unique",
        "searchsorted", "cumsum", "arange", "empty_like", "count_nonzero", "any")})
    ns.asnumpy = np.asarray
    stream = types.SimpleNamespace(synchronize=lambda: None)
    ns.cuda = types.SimpleNamespace(get_current_stream=lambda: stream,
                                    runtime=types.SimpleNamespace(getDevice=lambda: 0))
    return ns


def np_build_bitsets(cp, rows, columns, transactions, items):
    words = (transactions + 31) // 32
    bits = np.zeros((items, words), dtype=np.uint32)
    rows = np.asarray(rows, dtype=np.uint64)
    cols = np.asarray(columns, dtype=np.uint64)
    if rows.size:
        np.bitwise_or.at(bits, (cols, rows // 32),
                         (np.uint32(1) << (rows % 32).astype(np.uint32)))
    return bits


def np_count_supports(cp, bitsets, candidates):
    if not len(candidates):
        return []
    idx = np.asarray(candidates, dtype=np.int64)
    inter = np.bitwise_and.reduce(bitsets[idx], axis=1)
    return np.bitwise_count(inter).sum(axis=1, dtype=np.uint64).tolist()


def np_intersect_extensions(cp, prefix, extensions):
    out = extensions & prefix
    return out, np.bitwise_count(out).sum(axis=1, dtype=np.uint64).tolist()


def load_reference():
    sys.path.insert(0, str(REF))
    import importlib

    import cupami
    _bitsets = importlib.import_module("cupami.frequentPattern._bitsets")
    apriori_mod = importlib.import_module("cupami.frequentPattern.cuApriori")

    _bitsets.build_bitsets = np_build_bitsets
    _bitsets.count_supports = np_count_supports
    _bitsets.intersect_extensions = np_intersect_extensions
    ns = numpy_cuda_namespace()
    apriori_mod.cuApriori._getCudaModule = staticmethod(lambda: ns)
    return cupami


def run(cupami, cls_name, rows, minsup, **attrs):
    cls = getattr(cupami, cls_name)
    miner = cls(rows, minsup, use_gpu_io=False, use_gds=False)
    for k, v in attrs.items():
        setattr(miner, k, v)
    miner.mine()
    return {"minSup": minsup, "resolved": int(miner._minSup),
            "patterns": [[k, int(v)] for k, v in miner.getPatterns().items()]}


def cases(cupami):
    out = []

    def add(name, rows, supports, store_rows=True, **attrs):
        entry = {"name": name, "rows": [list(map(str, r)) if store_rows else None for r in rows]
                 if store_rows else None, "results": {}}
        for s in supports:
            for algo in ("cuEclat", "cuApriori"):
                entry["results"].setdefault(algo, []).append(run(cupami, algo, rows, s, **attrs))
        out.append(entry)

    # tests/test_cu_eclat.py:37-48 -- randomized brute force, Eclat == Apriori.
    for seed in range(5):
        rng = random.Random(seed)
        rows = [rng.sample(range(8), rng.randrange(9)) for _ in range(33 + seed)]
        add(f"randomized-seed{seed}", rows, (1, 7, 0.25, 1.0, 100))
    # :50-58 -- 65 identical rows of 8 items, tiny batches -> 255 patterns.
    add("dense-8x65-small-batches", [list(range(8))] * 65, (1,),
        _PAIR_BATCH_SIZE=3, _INTERSECTION_BATCH_BYTES=12)
    # :60-65 -- empty, duplicate baskets, large ids.
    for k, rows in enumerate(([], [[], []], [[0, 0, 1], [], [1, 4294967295], [0, 1, 4294967295]])):
        add(f"empty-duplicates-large-ids-{k}", rows, (1,))
    # :89-106 -- repeated mining data.
    add("output-apis", [[1, 2], [2, 3], [1, 2, 3]], (1,))
    # tests/test_miner_examples.py:30-50 -- manual counts.
    add("manual-counts", [[1, 2, 2, 3], [], [1, 2], [1, 3], [2, 3]], (2, 0.5))
    # tests/test_cl_apriori.py:128-134 -- 63 deep patterns.
    add("deep-6x8", [["a", "b", "c", "d", "e", "f"]] * 8, (2,))
    # Labels with spaces, commas and mixed types; thresholds 2.5 / 0 / -1.
    add("labels-and-thresholds", [[" a", "a ", "b,c"], ["b,c", 10, "10"], ["a", 9, "b,c"], [2, 10]],
        (1, 2.5, 0, -1, 1.0))
    # tests/test_transaction_formats.py:147-167 -- word boundaries (reference sampler).
    from cupami import TransactionalDatabase
    for count in (0, 1, 31, 32, 33, 63, 64, 65, 127, 128, 129):
        g = TransactionalDatabase(count, 8, avg_length=3, seed=42)
        g.create()
        add(f"word-boundary-{count}", g.getTransactions(), (max(1, count // 8),))
    # notebooks/frequentPattern/cuEclat.ipynb -- 100 x 8, avg 3, seed 42, 0.1 -> 35 patterns.
    g = TransactionalDatabase(100, 8, avg_length=3, seed=42)
    g.create()
    add("notebook-100x8", g.getTransactions(), (0.1,))
    # Denser random cases that reach depth >= 5.
    for seed in range(3):
        rng = np.random.default_rng(100 + seed)
        p = rng.uniform(0.3, 0.9, 14)
        rows = [[int(i) for i in np.nonzero(rng.random(14) < p)[0]] for _ in range(300)]
        add(f"dense-random-{seed}", rows, (0.3, 60))
    return out


def quickstart(cupami):
    """quickstart.ipynb: 10,000 x 50, avg 6, seed 42, minSup 0.01 -> 1275 patterns."""
    from cupami import BinaryTransactionalDatabase
    g = BinaryTransactionalDatabase(10000, 50, avg_length=6, seed=42)
    rows = g.create()
    lengths = np.array([len(r) for r in rows], dtype=np.uint64)
    offsets = np.zeros(len(rows) + 1, dtype=np.uint64)
    np.cumsum(lengths, out=offsets[1:])
    items = np.array([v for r in rows for v in r], dtype=np.uint32)
    np.savez_compressed(HERE / "quickstart_10000x50.npz", offsets=offsets, items=items)
    res = {algo: run(cupami, algo, rows, 0.01) for algo in ("cuEclat", "cuApriori")}
    return {"name": "quickstart-10000x50-seed42", "data": "quickstart_10000x50.npz", "results": res}


def input_cases(cupami):
    """The reference constructor's view of input files (cuApriori.__init__ and its
    readers, cupami/frequentPattern/cuApriori.py:173-456, with use_gpu_io=False
    and use_gds=False): baskets, transaction count and resolved threshold."""
    import base64
    import struct
    import tempfile

    texts = {
        "comma.csv": "a,b\n b ,a,a\n\n10,2\n",
        "tab.tsv": "x\ty\n\ny\n",
        "semicolon.txt": "1;2\n2;3;;\n",
        "bom.csv": "\ufeffa,b\nb\n",
        "spaces.csv": " , ,\nq, r \n",
    }
    out = []
    with tempfile.TemporaryDirectory() as d:
        d = Path(d)
        files = {}
        for name, text in texts.items():
            (d / name).write_bytes(text.encode("utf-8"))
            files[name] = {"text": text}
        rows = [[1, 1, 2], [], [0, 2], [4294967295, 2]]
        flat, offsets = [], [0]
        for r in rows:
            flat.extend(r)
            offsets.append(len(flat))
        blob = (struct.pack("<8sQQQ", b"CUPAMI01", len(rows), len(flat), 4294967295)
                + struct.pack(f"<{len(offsets)}Q", *offsets) + struct.pack(f"<{len(flat)}I", *flat))
        (d / "t.bin").write_bytes(blob)
        files["t.bin"] = {"base64": base64.b64encode(blob).decode()}
        import pyarrow as pa
        import pyarrow.parquet as pq
        pq.write_table(pa.table({"items": pa.array(rows, pa.list_(pa.uint32()))}), d / "t.parquet")
        files["t.parquet"] = {"base64": base64.b64encode((d / "t.parquet").read_bytes()).decode()}
        settings = {"comma.csv": [(1, None), (0.5, None)], "tab.tsv": [(1, None)], "semicolon.txt": [(1, ";")],
                    "bom.csv": [(1, None)], "spaces.csv": [(1, None)], "t.bin": [(0.5, None)],
                    "t.parquet": [(2, None)]}
        for name, runs in settings.items():
            for min_sup, sep in runs:
                miner = cupami.cuApriori(d / name, min_sup, sep, use_gds=False, use_gpu_io=False)
                out.append({"file": name, "minSup": min_sup, "sep": sep,
                            "baskets": [list(b) for b in miner._Database],
                            "transactions": int(miner._transactionCount), "resolvedMinSup": int(miner._minSup)})
    return {"files": files, "runs": out}


def output_cases(cupami):
    """The reference's save() text and getPatternsAsDataFrame() rows
    (cuApriori.py:537-560) for a few cases, both miners."""
    import tempfile

    out = []
    for name, rows, min_sup in (("labels", [[" a", "a ", "b,c"], ["b,c", 10, "10"], ["a", 9, "b,c"], [2, 10]], 1),
                                ("deep", [["a", "b", "c", "d"]] * 3 + [["a", "c"], ["b", "d"]], 2)):
        for algo in ("cuEclat", "cuApriori"):
            miner = getattr(cupami, algo)(rows, min_sup, use_gpu_io=False, use_gds=False)
            miner.mine()
            with tempfile.TemporaryDirectory() as d:
                path = Path(d) / "out.txt"
                miner.save(path)
                text = path.read_text(encoding="utf-8")
            df = miner.getPatternsAsDataFrame()
            out.append({"name": name, "algorithm": algo, "minSup": min_sup, "rows": [list(map(str, r)) for r in rows],
                        "patterns": [[k, int(v)] for k, v in miner.getPatterns().items()],
                        "save": text, "columns": list(df.columns),
                        "frame": [[str(a), int(b)] for a, b in df.values.tolist()]})
    return out


def main():
    cupami = load_reference()
    fixtures = {"generator": "tests/golden/make_golden.py", "reference": "cuPAMI 2026.11.02",
                "cases": cases(cupami), "quickstart": quickstart(cupami), "inputs": input_cases(cupami),
                "outputs": output_cases(cupami)}
    (HERE / "reference_patterns.json").write_text(json.dumps(fixtures, separators=(",", ":")))
    n = sum(len(r["patterns"]) for c in fixtures["cases"] for rs in c["results"].values() for r in rs)
    print(f"wrote {len(fixtures['cases'])} cases, {n} patterns, quickstart "
          f"{len(fixtures['quickstart']['results']['cuEclat']['patterns'])} patterns")


if __name__ == "__main__":
    main()
