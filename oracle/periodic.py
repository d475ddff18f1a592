"""Periodic-frequent mining on the CPU -- TEST INFRASTRUCTURE ONLY.

Restates, with NumPy, what cuPAMI's periodic-frequent miners compute, so that
the tests can check the CUDA path (``cpm_periodic_counts``,
``cpm_mine_periodic``) against it.  Nothing in the product imports it.

Followed step by step:
  temporal rows, labels, timeline    cupami/periodicFrequentPattern/_temporal.py:89-147
  occurrence bitsets (_prepare)      _temporal.py:150-157 with _bitsets.build_bitsets
  periodic_counts kernel             _temporal.py:26-53 (launch :156-165)
  acceptance                         _temporal.py:166-171
  cuPFEclat.mine (insertion order)   cupami/periodicFrequentPattern/cuPFEclat.py:146-175
  cuPFApriori.mine (level order)     cupami/periodicFrequentPattern/cuPFApriori.py:141-157
                                     with cuApriori._generateCandidates (cupami/frequentPattern/cuApriori.py:473-492)

Parity pin: ``tests/golden/periodic_patterns.json`` holds the reference
miners' own outputs (``tests/golden/make_periodic_golden.py`` runs them with
this module's kernel in place of the CUDA one); ``tests/test_periodic.py``
checks these drivers against every case and against a brute force.
"""

from __future__ import annotations

import math
from itertools import combinations

import numpy as np

from .numpy_port import pack


def prepare(rows, end_time=None):
    """Temporal rows ``[timestamp, item, ...]`` -> (labels, bits, timestamps, end).

    Rows are sorted by timestamp (stable), blank rows skipped, items cleaned as
    ``str(v).strip()`` with repeats dropped; every remaining row is a
    transaction, empty baskets included (_temporal.py:125-136)."""
    records = []
    for row in rows:
        row = list(row)
        if not row or not any(str(v).strip() for v in row):
            continue
        items = []
        for v in row[1:]:
            label = str(v).strip()
            if label and label not in items:
                items.append(label)
        records.append((int(str(row[0]).strip()), tuple(items)))
    records.sort(key=lambda r: r[0])
    timestamps = np.array([r[0] for r in records], dtype=np.int64)
    last = int(timestamps[-1]) if len(records) else 0
    end = last if end_time is None else int(end_time)
    labels = sorted({item for _, basket in records for item in basket})
    index = {label: i for i, label in enumerate(labels)}
    r_idx = [r for r, (_, basket) in enumerate(records) for _ in basket]
    c_idx = [index[item] for _, basket in records for item in basket]
    bits = pack(np.asarray(r_idx, dtype=np.uint64), np.asarray(c_idx, dtype=np.uint64), len(records), len(labels))
    return labels, bits, timestamps, end


def periodic_counts(bits, candidates, timestamps, n, end):
    """``[(support, periodicity)]`` per candidate (column lists): the kernel
    of _temporal.py:26-53 -- AND the rows, then scan the set rows < n in order,
    the periodicity being the largest of 0, ts[first] - 0, the gaps between
    consecutive set rows and end - ts[last] (max(0, end) when no row is set)."""
    out = []
    if not len(candidates):
        return out
    words = bits.shape[1]
    for cand in candidates:
        acc = np.full(words, 0xFFFFFFFF, dtype=np.uint32)
        for c in cand:
            acc &= bits[c]
        rows = np.flatnonzero(np.unpackbits(acc.view(np.uint8), bitorder="little"))
        rows = rows[rows < n]
        # the scan starts from a periodicity of 0 (_temporal.py:38)
        if rows.size == 0:
            out.append((0, max(0, int(end))))
            continue
        ts = timestamps[rows]
        if abs(int(end)) < 2**62 and np.all(np.abs(ts) < 2**62):  # no int64 overflow in the differences
            gaps = np.diff(np.concatenate(([0], ts, [end])).astype(np.int64))
            out.append((int(rows.size), max(0, int(gaps.max()))))
        else:  # exact Python integers
            points = [0, *ts.tolist(), int(end)]
            out.append((int(rows.size), max(0, *(b - a for a, b in zip(points, points[1:])))))
    return out


def _accept(support, period, min_sup, max_per):
    return support >= min_sup and support > 0 and period <= max_per


def _counter(bits, timestamps, end, counts):
    """Candidate column lists -> [(support, periodicity)]: the NumPy kernel, or
    ``counts`` (another implementation of the same kernel, e.g. the reference's
    CUDA kernel) when given."""
    if counts is not None:
        return counts
    n = len(timestamps)
    return lambda cands: periodic_counts(bits, cands, timestamps, n, end)


def pf_eclat(labels, bits, timestamps, end, min_sup, max_per, batch=4096, counts=None):
    """cuPFEclat.mine: ``[(pattern tuple, support, periodicity)]`` in insertion order."""
    index = {label: i for i, label in enumerate(labels)}
    found = []
    count = _counter(bits, timestamps, end, counts)

    def evaluate(patterns):
        return count([[index[x] for x in p] for p in patterns])

    singles = [(label,) for label in labels]
    frequent = []
    for start in range(0, len(singles), batch):
        chunk = singles[start:start + batch]
        for pattern, (s, p) in zip(chunk, evaluate(chunk)):
            if _accept(s, p, min_sup, max_per):
                found.append((pattern, s, p))
                frequent.append(pattern[0])
    stack = [[(), frequent, 0]]
    while stack:
        prefix, extensions, position = stack[-1]
        if position >= len(extensions) - 1:
            stack.pop()
            continue
        stack[-1][2] += 1
        child = prefix + (extensions[position],)
        tails = extensions[position + 1:]
        kept = []
        for start in range(0, len(tails), batch):
            chunk = [child + (item,) for item in tails[start:start + batch]]
            for pattern, (s, p) in zip(chunk, evaluate(chunk)):
                if _accept(s, p, min_sup, max_per):
                    found.append((pattern, s, p))
                    kept.append(pattern[-1])
        if len(kept) > 1:
            stack.append([child, kept, 0])
    return found


def _generate(level):
    """cuApriori._generateCandidates: prefix join of a level plus subset pruning, sorted."""
    if not level:
        return []
    size = len(level[0]) + 1
    previous = set(level)
    ordered = sorted(level)
    out = set()
    for i, left in enumerate(ordered):
        for right in ordered[i + 1:]:
            if left[:-1] != right[:-1]:
                continue
            cand = left + (right[-1],)
            if all(sub in previous for sub in combinations(cand, size - 1)):
                out.add(cand)
    return sorted(out)


def pf_apriori(labels, bits, timestamps, end, min_sup, max_per, batch=4096, counts=None):
    """cuPFApriori.mine: ``[(pattern tuple, support, periodicity)]`` level by level."""
    index = {label: i for i, label in enumerate(labels)}
    found = []
    count = _counter(bits, timestamps, end, counts)
    candidates = [(label,) for label in labels]
    while candidates:
        level = []
        for start in range(0, len(candidates), batch):
            chunk = candidates[start:start + batch]
            for pattern, (s, p) in zip(chunk, count([[index[x] for x in p] for p in chunk])):
                if _accept(s, p, min_sup, max_per):
                    found.append((pattern, s, p))
                    level.append(pattern)
        candidates = _generate(level)
    return found


def thresholds(min_sup, max_per, n_rows, end):
    """(support count, periodicity limit) as the reference resolves them
    (cuApriori.py:452-456 for minSup; _temporal.py:85 for maxPer)."""
    count = math.ceil(min_sup * n_rows) if isinstance(min_sup, float) and 0 < min_sup <= 1 else int(min_sup)
    limit = max_per * end if isinstance(max_per, float) and 0 < max_per <= 1 else max_per
    return count, limit


def mine(rows, min_sup, max_per, algorithm="eclat", end_time=None):
    """``{tab-joined labels: (support, periodicity)}`` in the miner's insertion order."""
    labels, bits, timestamps, end = prepare(rows, end_time)
    count, limit = thresholds(min_sup, max_per, len(timestamps), end)
    fn = pf_eclat if algorithm == "eclat" else pf_apriori
    return {"\t".join(p): (s, per) for p, s, per in fn(labels, bits, timestamps, end, count, limit)}


def brute_force(rows, min_sup, max_per, end_time=None):
    """Every itemset of the labels checked directly (small inputs only), as a dict
    without order: the definition the miners implement."""
    labels, bits, timestamps, end = prepare(rows, end_time)
    count, limit = thresholds(min_sup, max_per, len(timestamps), end)
    out = {}
    n = len(timestamps)
    for width in range(1, len(labels) + 1):
        for combo in combinations(range(len(labels)), width):
            (s, p), = periodic_counts(bits, [list(combo)], timestamps, n, end)
            if _accept(s, p, count, limit):
                out["\t".join(labels[c] for c in combo)] = (s, p)
    return out
