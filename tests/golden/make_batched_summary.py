"""Order-independent summaries of the exact answers for the 512 batched databases.

Runs the C oracle (oracle/eclat_oracle.c) on every database of
``cupami_b200.datasets.batched_zipf()`` (512 databases, 1,000-200,000
transactions each, 200 items, Poisson(8) lengths, Zipf(1.1), seed 19) at
minSup 0.01, each with its own threshold, and writes
``batched_zipf_512_summary.json``: per database the transaction count, the
pattern count per length, the two 64-bit hash sums over (sorted item ids,
support) of ``make_sparse_summary.summarize`` and the support sum.  The GPU test
mines the whole batch in one ``cuEclat.mineBatch`` and compares every database.
"""

import json
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))
sys.path.insert(0, str(HERE))


def one(i):
    """Summary of database i (regenerated from its own seed), mined on one thread."""
    import oracle
    from cupami_b200 import datasets
    from make_sparse_summary import summarize

    csr = datasets.batched_zipf_database(i)
    labels, (po, pi, ps) = oracle.mine_csr(csr.offsets, csr.items, 0.01, threads=1)
    s = summarize(labels, po, pi, ps)
    s["transactions"] = int(np.count_nonzero(np.diff(csr.offsets.astype(np.int64)) > 0))
    return s


def main():
    import multiprocessing as mp
    import os

    t = time.time()
    with mp.get_context("spawn").Pool(os.cpu_count()) as pool:
        out = pool.map(one, range(512), chunksize=4)
    doc = {"workload": "batched_zipf(n_db=512, low=1_000, high=200_000, n_items=200, mean=8, s=1.1, seed=19)",
           "minSup": 0.01, "patterns": sum(d["patterns"] for d in out),
           "oracle_seconds": round(time.time() - t, 1), "generator": "tests/golden/make_batched_summary.py",
           "databases": out}
    (HERE / "batched_zipf_512_summary.json").write_text(json.dumps(doc, separators=(",", ":")))
    print(doc["patterns"], doc["oracle_seconds"])


if __name__ == "__main__":
    main()
