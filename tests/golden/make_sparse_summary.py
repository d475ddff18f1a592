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


def search_counts(offsets, items):
    """How much work the reference's Eclat driver does on this answer.

    ``items`` lists every pattern in emission order, each as its parent's items
    plus one column (the reference builds ``head + (name,)``, cuEclat.py:230-236).
    A pattern with c >= 2 children is a search frame of c members
    (cuEclat.py:195-201 for single items, :237-239 deeper): c - 1 positions and
    c(c - 1)/2 intersections (one ``intersect_extensions`` row per later
    member, cuEclat.py:221-229).  Every pattern of length >= 3 is one child row
    the driver copies out (``take``, cuEclat.py:231-236); every member of a
    top-level class is one row of its vertical gather (cuEclat.py:199).
    """
    off = offsets.astype(np.int64)
    lens = np.diff(off)
    n = lens.size
    m1 = np.uint64(0x9E3779B97F4A7C15)
    # rolling hash of every prefix of every pattern
    with np.errstate(over="ignore"):
        full = np.zeros(n, dtype=np.uint64)
        prefix = np.zeros(n, dtype=np.uint64)
        for k in range(int(lens.max()) if n else 0):
            has = lens > k
            v = items[off[:-1][has] + k].astype(np.uint64) + np.uint64(1)
            h = full[has] * m1 + v
            last = lens[has] == k + 1
            idx = np.nonzero(has)[0]
            prefix[idx[last]] = full[idx[last]]
            full[has] = h
    parents = lens >= 2
    order = np.argsort(full, kind="stable")
    pos = np.searchsorted(full[order], prefix[parents])
    parent_idx = order[np.minimum(pos, n - 1)]
    assert np.array_equal(full[parent_idx], prefix[parents]), "parent not found"
    children = np.bincount(parent_idx, minlength=n).astype(np.int64)
    frame = children >= 2
    top = frame & (lens == 1)
    deep = frame & (lens >= 2)
    f = int(np.count_nonzero(lens == 1))
    return {"frequent_items": f, "pair_candidates": f * (f - 1) // 2,
            "top_frames": int(top.sum()), "top_members": int(children[top].sum()),
            "top_positions": int((children[top] - 1).sum()),
            "top_intersections": int((children[top] * (children[top] - 1) // 2).sum()),
            "deep_frames": int(deep.sum()), "deep_positions": int((children[deep] - 1).sum()),
            "deep_intersections": int((children[deep] * (children[deep] - 1) // 2).sum()),
            "copied_children": int(np.count_nonzero(lens >= 3))}


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
    out["reference_search"] = search_counts(po, pi)
    out.update({"workload": "sparse_zipf(n=1_000_000, n_items=20_000, mean=40, s=1.0, seed=3)", "minSup": 0.001,
                "oracle_seconds": round(time.time() - t, 1), "generator": "tests/golden/make_sparse_summary.py"})
    (HERE / "sparse_zipf_1m_summary.json").write_text(json.dumps(out, indent=1))
    print(json.dumps(out))


if __name__ == "__main__":
    main()
