"""Regenerate ``periodic_patterns.json`` from the reference periodic miners.

Run where the cuPAMI sources can be read: ``$CUPAMI_REFERENCE``, else a
directory named ``reference`` beside this repository's own directory.  ``cuPFEclat.mine`` and
``cuPFApriori.mine`` (cupami/periodicFrequentPattern/cuPFEclat.py:146-175,
cuPFApriori.py:141-157) and everything they call in ``TemporalInput`` run
unchanged; only the CUDA plumbing is replaced:

* ``cuApriori._getCudaModule`` returns the NumPy namespace of
  ``make_golden.py`` (plus ``empty``);
* ``_bitsets.build_bitsets`` is the NumPy statement of ``make_golden.py``;
* ``_temporal._kernel`` returns a launcher that computes the
  ``periodic_counts`` kernel (_temporal.py:26-53) with ``oracle.periodic``.

Each case records its rows, thresholds and both miners' ``getPatterns()`` as
ordered lists, so the checks compare insertion order as well as content.
Nothing at test time reads the reference checkout.
"""

from __future__ import annotations

import json
import random
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
sys.path.insert(0, str(HERE.parents[1]))

from make_golden import REF, load_reference, numpy_cuda_namespace  # noqa: E402

from oracle import periodic  # noqa: E402


def numpy_launcher(device):
    def launch(grid, block, args):
        bits, words, idx, width, count, ts, n, end, supports, periods = args
        assert bits.shape[1] == int(words) and idx.shape == (int(count), int(width))
        out = periodic.periodic_counts(bits, idx.astype(np.int64).tolist(), np.asarray(ts), int(n), int(end))
        supports[:] = [s for s, _ in out]
        periods[:] = [p for _, p in out]
    return launch


def load():
    cupami = load_reference()
    import importlib

    temporal = importlib.import_module("cupami.periodicFrequentPattern._temporal")
    apriori_mod = importlib.import_module("cupami.frequentPattern.cuApriori")
    ns = numpy_cuda_namespace()
    ns.empty = np.empty
    apriori_mod.cuApriori._getCudaModule = staticmethod(lambda: ns)
    temporal._kernel = numpy_launcher
    return cupami


def run(cupami, rows, min_sup, max_per, end=None):
    out = {"minSup": min_sup, "maxPer": max_per, "endTime": end}
    for name in ("cuPFEclat", "cuPFApriori"):
        miner = getattr(cupami, name)(rows, min_sup, max_per, endTime=end)
        miner.mine()
        out[name] = [[k, int(s), int(p)] for k, (s, p) in miner.getPatterns().items()]
    return out


def cases(cupami):
    out = []

    def add(name, rows, settings):
        out.append({"name": name, "rows": rows,
                    "results": [run(cupami, rows, *s) for s in settings]})

    # tests/test_periodic_miners.py: the paper example (9 patterns, a-b = (4, 3)).
    baskets = ["ab", "acdi", "cefj", "abfgh", "bcd", "def", "abi", "cde", "abef", "acg"]
    add("paper-example", [[i + 1, *b] for i, b in enumerate(baskets)], [(3, 3)])
    # Randomized rows with empty baskets, shuffled (rows are re-sorted by timestamp).
    for seed in range(4):
        rng = random.Random(seed)
        rows = [[i * 3, *rng.sample(range(6), rng.randint(0, 6))] for i in range(1, 19)]
        rng.shuffle(rows)
        add(f"random-seed{seed}", rows, [(1, 54), (3, 15), (5, 9)])
    # Boundaries: duplicates, empty baskets, explicit end, empty input, equal
    # timestamps, timestamps past 2**53.
    add("boundaries-0", [[9, "a"], [0, "a", "a", "0"], [4], [9, "a", "b"], [15]], [(1, 10)])
    add("boundaries-1", [[2, "x"], [3, "x"]], [(1, 5, 20)])
    add("boundaries-2", [], [(1, 0)])
    add("boundaries-3", [[0, "x"], [0, "y"]], [(1, 0)])
    add("boundaries-4", [[2**53 + 1, "x"], [2**53 + 3, "x"]], [(1, 2**53 + 1)])
    # One path across a 64-row word boundary.
    add("word-boundaries", [[i, "a", "b", *(["c"] if i % 2 else [])] for i in range(1, 66)], [(1, 4)])
    # Fractional thresholds: minSup 0.4 of 5 rows, maxPer 0.4 of the timeline.
    add("fractional", [[2, "a"], [4, "a"], [6, "b"], [8, "a"], [10, "a"]], [(0.4, 0.4)])
    # The reference's temporal generator (50 rows, 5 items, repeats and gaps).
    from cupami import TemporalDatabase
    g = TemporalDatabase(50, 5, avg_length=2.5, seed=42, repeatAllowed=True, missingAllowed=True)
    g.create()
    add("generator-50x5", [list(r) for r in g.getTransactions()], [(3, 20)])
    # Deeper seeded cases: dense baskets over 14-16 items, increasing timestamps
    # with repeats, several 64-row words.
    for seed, n_rows, n_items in ((0, 600, 14), (1, 1500, 16), (2, 4000, 12)):
        rng = np.random.default_rng(200 + seed)
        p = rng.uniform(0.35, 0.95, n_items)
        ts = np.cumsum(rng.integers(0, 4, n_rows))
        rows = [[int(t), *[f"i{j}" for j in np.nonzero(rng.random(n_items) < p)[0]]] for t in ts]
        end = int(ts[-1])
        add(f"dense-seed{seed}", rows, [(0.3, max(8, end // 40)), (0.5, end // 10)])
    return out


def input_cases(cupami):
    """The reference constructor's view of input files: timestamps, baskets,
    counts and resolved thresholds (TemporalInput.__init__ and readers,
    _temporal.py:56-147; formats of cupami/extras/_temporal_io.py)."""
    import base64
    import tempfile

    from cupami.extras import _temporal_io

    texts = {
        "comma.csv": "3,a,b\n1,b\n2,a,a, c \n",
        "tab.txt": "1\ta\tb\n3\ta\n5\tb\n",
        "space.txt": "4 x y\n\n2 y\n 6 x\n",
        "bom-blank.csv": "\ufeff5,p\n\n,\n7,q,p\n7\n",
        "semicolon.txt": "2;a;b\n1;b\n",
    }
    out = []
    with tempfile.TemporaryDirectory() as d:
        d = Path(d)
        files = {}
        for name, text in texts.items():
            (d / name).write_text(text, encoding="utf-8")
            files[name] = {"text": text}
        rows = [[3, 7, 7, 1], [1], [2, 4294967295], [2, 5]]
        _temporal_io.write_binary(d / "t.bin", rows, 4294967295)
        files["t.bin"] = {"base64": base64.b64encode((d / "t.bin").read_bytes()).decode()}
        _temporal_io.write_parquet(d / "t.parquet", rows, 4294967295)
        files["t.parquet"] = {"base64": base64.b64encode((d / "t.parquet").read_bytes()).decode()}
        settings = {"comma.csv": [(1, 2, None, None), (0.5, 0.5, None, None)],
                    "tab.txt": [(1, 5, None, None)], "space.txt": [(2, 3, None, 10)],
                    "bom-blank.csv": [(1, 4, None, None)], "semicolon.txt": [(1, 2, ";", None)],
                    "t.bin": [(0.25, 1.0, None, None)], "t.parquet": [(2, 2, None, 5)]}
        for name, runs in settings.items():
            for min_sup, max_per, sep, end in runs:
                miner = cupami.cuPFApriori(d / name, min_sup, max_per, sep, endTime=end)
                out.append({"file": name, "minSup": min_sup, "maxPer": max_per, "sep": sep, "endTime": end,
                            "timestamps": list(miner._timestamps),
                            "baskets": [list(b) for b in miner._Database],
                            "transactions": int(miner._transactionCount), "resolvedMinSup": int(miner._minSup),
                            "resolvedMaxPer": miner._maxPer, "end": int(miner._endTimestamp)})
    return {"files": files, "runs": out}


def output_cases(cupami):
    """The reference's save() text and getPatternsAsDataFrame() rows
    (_temporal.py:173-181) for the paper example, both miners."""
    import tempfile

    baskets = ["ab", "acdi", "cefj", "abfgh", "bcd", "def", "abi", "cde", "abef", "acg"]
    rows = [[i + 1, *b] for i, b in enumerate(baskets)]
    out = []
    for name in ("cuPFEclat", "cuPFApriori"):
        miner = getattr(cupami, name)(rows, 3, 3)
        miner.mine()
        with tempfile.TemporaryDirectory() as d:
            path = Path(d) / "out.txt"
            miner.save(path)
            text = path.read_text(encoding="utf-8")
        df = miner.getPatternsAsDataFrame()
        out.append({"algorithm": name, "rows": rows, "minSup": 3, "maxPer": 3,
                    "patterns": [[k, int(s), int(p)] for k, (s, p) in miner.getPatterns().items()],
                    "save": text, "columns": list(df.columns),
                    "frame": [[str(a), int(b), int(c)] for a, b, c in df.values.tolist()]})
    return out


def main():
    cupami = load()
    fixtures = {"generator": "tests/golden/make_periodic_golden.py", "reference": str(REF.name),
                "cases": cases(cupami), "inputs": input_cases(cupami),
                "outputs": output_cases(cupami)}
    (HERE / "periodic_patterns.json").write_text(json.dumps(fixtures, separators=(",", ":")))
    n = sum(len(r[m]) for c in fixtures["cases"] for r in c["results"] for m in ("cuPFEclat", "cuPFApriori"))
    print(f"wrote {len(fixtures['cases'])} cases, {n} patterns")


if __name__ == "__main__":
    main()
