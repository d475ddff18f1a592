"""Order-independent summary of the exact answer for the 1M x 20k sparse workload.

Runs the C oracle (oracle/eclat_oracle.c, OpenMP) on
``cupami_b200.datasets.sparse_zipf()`` (1,000,000 transactions, 20,000 items,
Poisson(40) lengths, Zipf(1.0), seed 3) at minSup 0.001 and writes
``sparse_zipf_1m_summary.json``: the pattern count per length and two 64-bit
sums over all patterns of a hash of (sorted item ids, support).  The GPU test
compares the CUDA path against it; the full answer (6.3 million patterns)
is too large to commit and takes about 30 minutes on 8 cores.
"""

import json
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))


def pattern_hashes(labels, offsets, items, supports):
    """Two independent 64-bit hashes per pattern of (sorted ids, support)."""
    ids = np.asarray([int(x) for x in labels], dtype=np.uint64)[items.astype(np.int64)]
    lens = np.diff(offsets.astype(np.int64))
    row = np.repeat(np.arange(lens.size), lens)
    # items within a pattern are in column order; hash the sorted original ids
    order = np.lexsort((ids, row))
    ids = ids[order]
    m1 = np.uint64(0x9E3779B97F4A7C15)
    m2 = np.uint64(0xC2B2AE3D27D4EB4F)
    with np.errstate(over="ignore"):
        pos = (np.arange(ids.size, dtype=np.int64) - np.repeat(offsets[:-1].astype(np.int64), lens)).astype(np.uint64)
        t1 = (ids + np.uint64(1)) * m1 ^ (pos * m2)
        t2 = (ids * m2 + pos + np.uint64(7)) * m1
        h1 = np.add.reduceat(t1, offsets[:-1].astype(np.int64)) if ids.size else np.zeros(0, np.uint64)
        h2 = np.bitwise_xor.reduceat(t2, offsets[:-1].astype(np.int64)) if ids.size else np.zeros(0, np.uint64)
        s = supports.astype(np.uint64)
        h1 = (h1 ^ (s * m2)) * m1
        h2 = (h2 + s * m1) * m2
    return h1, h2, lens


def summarize(labels, offsets, items, supports):
    h1, h2, lens = pattern_hashes(labels, offsets, items, supports)
    with np.errstate(over="ignore"):
        return {"patterns": int(supports.size),
                "per_length": np.bincount(lens).tolist()[1:],
                "hash_sum": int(h1.sum(dtype=np.uint64)), "hash_xor_sum": int(h2.sum(dtype=np.uint64)),
                "support_sum": int(supports.astype(np.uint64).sum())}


def main():
    import oracle
    from cupami_b200 import datasets

    csr = datasets.sparse_zipf()
    t = time.time()
    labels, (po, pi, ps) = oracle.mine_csr(csr.offsets, csr.items, 0.001)
    out = summarize(labels, po, pi, ps)
    out.update({"workload": "sparse_zipf(n=1_000_000, n_items=20_000, mean=40, s=1.0, seed=3)", "minSup": 0.001,
                "oracle_seconds": round(time.time() - t, 1), "generator": "tests/golden/make_sparse_summary.py"})
    (HERE / "sparse_zipf_1m_summary.json").write_text(json.dumps(out, indent=1))
    print(json.dumps(out))


if __name__ == "__main__":
    main()
