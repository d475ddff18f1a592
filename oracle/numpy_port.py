"""The reference miners' host path with NumPy kernels -- TEST INFRASTRUCTURE ONLY.

This restates how cuPAMI's ``cuEclat`` and ``cuApriori`` run when NumPy stands
in for CuPy: the same driver loop (pair batches of ``PAIR_BATCH`` candidates,
one intersect call per class position in batches of ``INTERSECTION_BYTES``,
level-wise Apriori joins with subset pruning) over 32-bit word bitsets, with
each kernel written as NumPy array arithmetic.  It is the CPU baseline the
benchmark reports beside the CUDA path, never part of the product.

The drivers take the kernels as an object (``NUMPY`` here); ``oracle.ref_gpu``
passes the reference's own CUDA kernels instead, which makes the same drivers
the reference's GPU path.

Followed step by step:
  singletons + pairs + classes    cupami/frequentPattern/cuEclat.py:168-203
  class search                    cupami/frequentPattern/cuEclat.py:211-245
  Apriori levels                  cupami/frequentPattern/cuApriori.py:473-535
  label order / row numbering     cupami/frequentPattern/cuApriori.py:378-404
  kernels                         cupami/frequentPattern/_bitsets.py:20-77
"""

from __future__ import annotations

from itertools import combinations, islice

import numpy as np

PAIR_BATCH = 65536
INTERSECTION_BYTES = 64 * 1024 * 1024


def pack(rows, cols, n_tx, n_items):
    words = (n_tx + 31) // 32
    bits = np.zeros((n_items, words), dtype=np.uint32)
    if rows.size:
        np.bitwise_or.at(bits, (cols.astype(np.int64), (rows // 32).astype(np.int64)),
                         np.left_shift(np.uint32(1), (rows % 32).astype(np.uint32)))
    return bits


def supports_of(bits, candidates):
    if not len(candidates):
        return []
    idx = np.asarray(candidates, dtype=np.int64)
    acc = bits[idx[:, 0]].copy()
    for j in range(1, idx.shape[1]):
        acc &= bits[idx[:, j]]
    return np.bitwise_count(acc).sum(axis=1, dtype=np.uint64).tolist()


def intersect(prefix, ext):
    child = ext & prefix
    return child, np.bitwise_count(child).sum(axis=1, dtype=np.uint64).tolist()


class NumpyKernels:
    """The three reference kernels plus the array steps the drivers use, on host arrays."""

    pack = staticmethod(pack)
    supports = staticmethod(supports_of)
    intersect = staticmethod(intersect)

    @staticmethod
    def vertical(bits, members, left):
        return bits[np.asarray(members, dtype=np.int64)] & bits[left]

    @staticmethod
    def take(child, keep):
        return child[np.asarray(keep, dtype=np.int64)]

    @staticmethod
    def concat(chunks):
        return np.concatenate(chunks)

    @staticmethod
    def sync():
        pass


NUMPY = NumpyKernels()


def device_pairs_from_csr(offsets, ids):
    """(labels, rows, cols) the way the reference's BIN bulk path builds them."""
    offsets = np.asarray(offsets, dtype=np.uint64)
    ids = np.asarray(ids, dtype=np.uint32)
    uniq = np.unique(ids)
    labels = sorted(map(str, uniq.tolist()))
    index = {label: i for i, label in enumerate(labels)}
    colmap = np.array([index[str(v)] for v in uniq.tolist()], dtype=np.uint32)
    lengths = np.diff(offsets.astype(np.int64))
    active = np.cumsum(lengths > 0) - 1
    rows = np.repeat(active, lengths).astype(np.uint64)
    cols = colmap[np.searchsorted(uniq, ids)] if ids.size else np.zeros(0, np.uint32)
    n_tx = int(np.count_nonzero(lengths > 0))
    return labels, rows, cols, n_tx


def eclat(labels, rows, cols, n_tx, minsup, k=NUMPY, out=None):
    """``{tuple(labels): support}`` in the reference's insertion order (filled into ``out`` if given)."""
    out = {} if out is None else out
    bits = k.pack(rows, cols, n_tx, len(labels))
    sup1 = k.supports(bits, [[i] for i in range(len(labels))])
    frequent = []
    for i, s in enumerate(sup1):
        if s >= minsup:
            frequent.append(i)
            out[(labels[i],)] = int(s)
    classes = {}
    pairs = combinations(frequent, 2)
    while True:
        batch = list(islice(pairs, PAIR_BATCH))
        if not batch:
            break
        for (a, b), s in zip(batch, k.supports(bits, batch)):
            if s >= minsup:
                out[(labels[a], labels[b])] = int(s)
                classes.setdefault(a, []).append(b)
    for a, members in classes.items():
        if len(members) < 2:
            continue
        vertical = k.vertical(bits, members, a)
        _search(out, (labels[a],), [labels[m] for m in members], vertical, minsup, k)
    k.sync()
    return out


def _search(out, prefix, names, vertical, minsup, k=NUMPY):
    stack = [[prefix, names, vertical, 0]]
    while stack:
        top = stack[-1]
        pre, nm, vert, pos = top
        if pos >= len(nm) - 1:
            stack.pop()
            continue
        top[3] += 1
        head = pre + (nm[pos],)
        step = max(1, INTERSECTION_BYTES // max(1, 4 * vert.shape[1]))
        kept_names, kept_bits = [], []
        for start in range(pos + 1, len(nm), step):
            stop = min(len(nm), start + step)
            child, sups = k.intersect(vert[pos], vert[start:stop])
            keep = [j for j, s in enumerate(sups) if s >= minsup]
            for j in keep:
                out[head + (nm[start + j],)] = int(sups[j])
                kept_names.append(nm[start + j])
            if keep:
                kept_bits.append(k.take(child, keep))
        if len(kept_names) > 1:
            stack.append([head, kept_names, kept_bits[0] if len(kept_bits) == 1 else k.concat(kept_bits), 0])


def apriori(labels, rows, cols, n_tx, minsup, k=NUMPY, out=None):
    out = {} if out is None else out
    bits = k.pack(rows, cols, n_tx, len(labels))
    index = {label: i for i, label in enumerate(labels)}
    level = []
    for i, s in enumerate(k.supports(bits, [[i] for i in range(len(labels))])):
        if s >= minsup:
            level.append((labels[i],))
            out[(labels[i],)] = int(s)
    while level:
        known = set(level)
        ordered = sorted(level)
        cands = set()
        for i, left in enumerate(ordered):
            for right in ordered[i + 1:]:
                if left[:-1] != right[:-1]:
                    continue
                cand = left + (right[-1],)
                if all(sub in known for sub in combinations(cand, len(cand) - 1)):
                    cands.add(cand)
        cands = sorted(cands)
        if not cands:
            break
        sups = k.supports(bits, [[index[x] for x in c] for c in cands])
        level = []
        for c, s in zip(cands, sups):
            if s >= minsup:
                level.append(c)
                out[c] = int(s)
    k.sync()
    return out


def mine_csr(offsets, ids, minsup_count, algorithm="eclat"):
    labels, rows, cols, n_tx = device_pairs_from_csr(offsets, ids)
    fn = eclat if algorithm == "eclat" else apriori
    return fn(labels, rows, cols, n_tx, minsup_count)
