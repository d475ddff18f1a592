"""Seeded synthetic transaction databases for the five benchmark workloads.

Every generator returns a :class:`TransactionCSR`: ``offsets`` (uint64[N+1]) and
``items`` (uint32[nnz]) with each basket sorted and free of duplicates, item
identifiers starting at 1 as in the reference's own basket sampler
(``cupami/extras/syntheticDataGenerator/TransactionalDatabase.py:104``).  The
generators are this project's own; none of them is the reference's sampler
except :func:`reference_uniform_baskets`, which restates it (same
``random.Random`` call sequence) so that the reference's published quickstart
output can be pinned.

Sampling "without replacement with weights" uses the sequential definition:
each next item is drawn from the weights restricted to the items not yet in the
basket.  That process is the same as drawing an i.i.d. stream from the full
weights and keeping the first ``L`` distinct values, which is what
:func:`_first_distinct` does for a whole chunk of baskets at once.
"""

from __future__ import annotations

import math
import random
from dataclasses import dataclass

import numpy as np

__all__ = [
    "TransactionCSR", "TemporalCSR", "uniform_poisson", "planted_zipf", "dense_fixed_length",
    "dense_bernoulli", "sparse_zipf", "batched_zipf", "reference_uniform_baskets",
    "temporal_planted", "workload",
]


@dataclass
class TransactionCSR:
    """A transaction database in compressed-row form (offsets + item ids)."""

    offsets: np.ndarray  # uint64[N + 1]
    items: np.ndarray    # uint32[nnz]
    universe: int        # largest item id that may appear

    @property
    def n_transactions(self) -> int:
        return int(self.offsets.size - 1)

    @property
    def nnz(self) -> int:
        return int(self.items.size)

    def rows(self):
        """Baskets as Python lists (small databases only)."""
        o = self.offsets.tolist()
        it = self.items.tolist()
        return [it[o[i]:o[i + 1]] for i in range(len(o) - 1)]

    @classmethod
    def from_rows(cls, rows, universe=None):
        lengths = np.fromiter((len(r) for r in rows), dtype=np.uint64, count=len(rows))
        offsets = np.zeros(len(rows) + 1, dtype=np.uint64)
        np.cumsum(lengths, out=offsets[1:])
        flat = np.fromiter((int(v) for r in rows for v in r), dtype=np.uint32,
                           count=int(offsets[-1]))
        if universe is None:
            universe = int(flat.max()) if flat.size else 1
        return cls(offsets, flat, max(1, int(universe)))


@dataclass
class TemporalCSR:
    """A temporal database in compressed-row form: row r holds the item ids
    ``items[offsets[r]:offsets[r + 1]]`` (empty rows allowed) at ``timestamps[r]``."""

    offsets: np.ndarray     # uint64[N + 1]
    items: np.ndarray       # uint32[nnz]
    timestamps: np.ndarray  # int64[N], nonnegative

    @property
    def n_transactions(self) -> int:
        return int(self.offsets.size - 1)

    @property
    def nnz(self) -> int:
        return int(self.items.size)

    def rows(self):
        """Rows ``[timestamp, *item ids]`` as Python lists (small databases only)."""
        o, it = self.offsets.tolist(), self.items.tolist()
        return [[t, *it[o[i]:o[i + 1]]] for i, t in enumerate(self.timestamps.tolist())]


def _zipf_cdf(n_items: int, s: float) -> np.ndarray:
    w = 1.0 / np.arange(1, n_items + 1, dtype=np.float64) ** s
    cdf = np.cumsum(w)
    return cdf / cdf[-1]


def _first_distinct(draws: np.ndarray, want: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """Keep, per row of ``draws``, the first ``want[row]`` distinct values.

    Returns ``(keep_mask, short_rows)``; ``short_rows`` flags rows whose stream
    held fewer than ``want`` distinct values (the caller redraws those).
    """
    order = np.argsort(draws, axis=1, kind="stable")
    sv = np.take_along_axis(draws, order, axis=1)
    first_sorted = np.ones_like(sv, dtype=bool)
    first_sorted[:, 1:] = sv[:, 1:] != sv[:, :-1]
    first = np.zeros_like(first_sorted)
    np.put_along_axis(first, order, first_sorted, axis=1)
    cum = np.cumsum(first, axis=1)
    keep = first & (cum <= want[:, None])
    short = cum[:, -1] < want
    return keep, short


def _sample_distinct(rng, sampler, lengths: np.ndarray, prefix=None,
                     chunk: int = 1 << 16) -> tuple[np.ndarray, np.ndarray]:
    """Baskets of ``lengths[i]`` distinct items drawn sequentially from ``sampler``.

    ``sampler(rng, shape)`` returns i.i.d. item ids.  ``prefix`` optionally
    gives, per row, items placed first (a planted pattern, already distinct).
    Returns CSR (offsets uint64, items uint32) with each basket sorted.
    """
    n = lengths.size
    out_len = np.zeros(n, dtype=np.int64)
    pieces = []
    for start in range(0, n, chunk):
        stop = min(n, start + chunk)
        want = lengths[start:stop].astype(np.int64)
        pre = None
        if prefix is not None:
            pre = prefix[start:stop]
            want = np.maximum(want, (pre >= 0).sum(axis=1))
        rows = np.arange(stop - start)
        result = np.zeros((stop - start, int(want.max()) if want.size else 0), dtype=np.int64)
        filled = np.zeros(stop - start, dtype=bool)
        factor = 2
        pending = rows
        while pending.size:
            k = int(factor * want[pending].max() + 32)
            draws = sampler(rng, (pending.size, k)).astype(np.int64)
            if pre is not None:
                p = pre[pending]
                # Negative entries pad the planted prefix; replace them by a
                # draw repeated from the stream so they never add a new value.
                p = np.where(p >= 0, p, draws[:, :1])
                draws = np.concatenate([p, draws], axis=1)
            keep, short = _first_distinct(draws, want[pending])
            ok = ~short
            idx = pending[ok]
            kept = keep[ok]
            vals = np.where(kept, draws[ok], np.iinfo(np.int64).max)
            vals.sort(axis=1)
            width = result.shape[1]
            result[idx] = vals[:, :width]
            filled[idx] = True
            pending = pending[short]
            factor *= 2
        lens = want
        out_len[start:stop] = lens
        mask = np.arange(result.shape[1])[None, :] < lens[:, None]
        pieces.append(result[mask].astype(np.uint32))
    offsets = np.zeros(n + 1, dtype=np.uint64)
    np.cumsum(out_len, out=offsets[1:])
    items = np.concatenate(pieces) if pieces else np.zeros(0, dtype=np.uint32)
    return offsets, items


def _zipf_sampler(n_items: int, s: float):
    cdf = _zipf_cdf(n_items, s)

    def sample(rng, shape):
        return np.searchsorted(cdf, rng.random(shape), side="right") + 1

    return sample


def _weighted_sampler(weights: np.ndarray):
    cdf = np.cumsum(weights / weights.sum())
    cdf[-1] = 1.0

    def sample(rng, shape):
        return np.searchsorted(cdf, rng.random(shape), side="right") + 1

    return sample


def uniform_poisson(n=10_000, n_items=50, mean=6, seed=42) -> TransactionCSR:
    """Lengths ~ Poisson(mean) clipped to [1, n_items]; items uniform, distinct."""
    rng = np.random.default_rng(seed)
    lengths = np.clip(rng.poisson(mean, n), 1, n_items)

    def sample(r, shape):
        return r.integers(1, n_items + 1, size=shape)

    offsets, items = _sample_distinct(rng, sample, lengths)
    return TransactionCSR(offsets, items, n_items)


def planted_zipf(n=100_000, n_items=1_000, mean=10, n_patterns=2_000,
                 pattern_mean=4, s=1.1, seed=7) -> TransactionCSR:
    """Planted patterns plus Zipf noise.

    A pool of ``n_patterns`` patterns is drawn first: each has length
    max(1, Poisson(pattern_mean)) and Zipf(s) items without replacement.  Each
    transaction takes one pattern chosen uniformly from the pool, draws a target
    length Poisson(mean) clipped to [1, n_items], and is filled with Zipf(s)
    noise items (without replacement) until it reaches that length; a pattern
    longer than the target is kept whole.
    """
    rng = np.random.default_rng(seed)
    zipf = _zipf_sampler(n_items, s)
    plen = np.clip(rng.poisson(pattern_mean, n_patterns), 1, n_items)
    p_off, p_items = _sample_distinct(rng, zipf, plen)
    width = int(plen.max())
    pool = np.full((n_patterns, width), -1, dtype=np.int64)
    for i in range(n_patterns):
        seg = p_items[p_off[i]:p_off[i + 1]]
        pool[i, :seg.size] = seg
    choice = rng.integers(0, n_patterns, n)
    lengths = np.clip(rng.poisson(mean, n), 1, n_items)
    offsets, items = _sample_distinct(rng, zipf, lengths, prefix=pool[choice])
    return TransactionCSR(offsets, items, n_items)


def dense_fixed_length(n=65_536, n_items=128, length=43, seed=11) -> TransactionCSR:
    """Exactly ``length`` distinct items per basket, weights ~ Beta(5,2) normalised."""
    rng = np.random.default_rng(seed)
    weights = rng.beta(5.0, 2.0, n_items)
    lengths = np.full(n, length, dtype=np.int64)
    offsets, items = _sample_distinct(rng, _weighted_sampler(weights), lengths)
    return TransactionCSR(offsets, items, n_items)


def dense_bernoulli(n=65_536, n_items=128, seed=11) -> TransactionCSR:
    """Item i present independently with probability p_i ~ Beta(5,2).

    The dense deep-lattice stand-in for the fixed-length workload, whose item
    frequencies all stay below 0.44 and so leave nothing frequent at 0.6.
    """
    rng = np.random.default_rng(seed)
    p = rng.beta(5.0, 2.0, n_items)
    rows = []
    counts = np.zeros(n, dtype=np.int64)
    for start in range(0, n, 1 << 15):
        stop = min(n, start + (1 << 15))
        m = rng.random((stop - start, n_items)) < p[None, :]
        r, c = np.nonzero(m)
        counts[start:stop] = m.sum(axis=1)
        rows.append((c + 1).astype(np.uint32))
    offsets = np.zeros(n + 1, dtype=np.uint64)
    np.cumsum(counts, out=offsets[1:])
    return TransactionCSR(offsets, np.concatenate(rows), n_items)


def sparse_zipf(n=1_000_000, n_items=20_000, mean=40, s=1.0, seed=3) -> TransactionCSR:
    """Lengths ~ Poisson(mean) clipped to [1, n_items]; Zipf(s) items, distinct."""
    rng = np.random.default_rng(seed)
    lengths = np.clip(rng.poisson(mean, n), 1, n_items)
    offsets, items = _sample_distinct(rng, _zipf_sampler(n_items, s), lengths)
    return TransactionCSR(offsets, items, n_items)


def sparse_zipf_250k(seed=3) -> TransactionCSR:
    """``sparse_zipf`` at 250,000 transactions (a profiling-sized case of the same shape)."""
    return sparse_zipf(n=250_000, seed=seed)


def batched_zipf(n_db=512, low=1_000, high=200_000, n_items=200, mean=8, s=1.1,
                 seed=19, limit=None) -> list[TransactionCSR]:
    """``n_db`` independent databases with log-uniform transaction counts.

    Database sizes come from the parent seed; database ``i`` is then drawn from
    its own child seed, so any subset can be regenerated on its own.
    ``limit`` keeps only the first ``limit`` databases.
    """
    return [batched_zipf_database(i, n_db, low, high, n_items, mean, s, seed)
            for i in range(n_db if limit is None else min(limit, n_db))]


def batched_zipf_database(i, n_db=512, low=1_000, high=200_000, n_items=200, mean=8, s=1.1,
                          seed=19) -> TransactionCSR:
    """Database ``i`` of ``batched_zipf`` with the same arguments, on its own."""
    root = np.random.SeedSequence(seed)
    rng = np.random.default_rng(root)
    sizes = np.round(np.exp(rng.uniform(math.log(low), math.log(high), n_db))).astype(np.int64)
    r = np.random.default_rng(root.spawn(n_db)[i])
    lengths = np.clip(r.poisson(mean, int(sizes[i])), 1, n_items)
    offsets, items = _sample_distinct(r, _zipf_sampler(n_items, s), lengths)
    return TransactionCSR(offsets, items, n_items)


def reference_uniform_baskets(transactions, items, avg_length=None, seed=None):
    """The reference's uniform basket sampler, restated call for call.

    Follows ``TransactionalDatabase._generateTransactions``
    (``cupami/extras/syntheticDataGenerator/TransactionalDatabase.py:103-114``):
    a symmetric uniform length around ``avg_length`` with stochastic rounding,
    then ``random.sample`` of item ids 1..items, sorted.  Used to rebuild the
    dataset behind the reference's published quickstart output.
    """
    if avg_length is None:
        avg_length = (items + 1) / 2
    avg_length = float(avg_length)
    rnd = random.Random(seed)
    ids = range(1, items + 1)
    radius = min(avg_length - 1, items - avg_length)
    rows = []
    for _ in range(transactions):
        target = rnd.uniform(avg_length - radius, avg_length + radius)
        length = math.floor(target)
        if rnd.random() < target - length:
            length += 1
        rows.append(sorted(rnd.sample(ids, length)))
    return rows


def quickstart(seed=42) -> TransactionCSR:
    """The reference's quickstart dataset (10,000 baskets over items 1..50, mean
    length 6, seed 42), rebuilt with the reference's own sampler."""
    return TransactionCSR.from_rows(reference_uniform_baskets(10_000, 50, avg_length=6, seed=seed), universe=51)


_WORKLOADS = {
    "uniform-10k": (uniform_poisson, 0.01),
    "planted-100k": (planted_zipf, 0.005),
    "dense-fixed-64k": (dense_fixed_length, 0.6),
    "dense-bernoulli-64k": (dense_bernoulli, 0.6),
    "sparse-zipf-1m": (sparse_zipf, 0.001),
}


def temporal_planted(n=100_000, n_items=200, mean=6, n_patterns=40, pattern_mean=3, planted=0.35,
                     empty=0.02, s=1.1, seed=23):
    """A temporal database: ``(csr, timestamps)`` with one row per transaction.

    Timestamps are a running sum of gaps drawn uniformly from {0, 1, 2, 3}
    (equal timestamps occur).  A pool of ``n_patterns`` patterns (lengths
    max(1, Poisson(pattern_mean)), Zipf(s) items) is drawn first; each row
    holds one pattern from the pool with probability ``planted`` and is filled
    with Zipf(s) noise to a Poisson(mean) length; a fraction ``empty`` of the
    rows are empty baskets, which temporal databases keep.
    """
    rng = np.random.default_rng(seed)
    zipf = _zipf_sampler(n_items, s)
    plen = np.clip(rng.poisson(pattern_mean, n_patterns), 1, n_items)
    p_off, p_items = _sample_distinct(rng, zipf, plen)
    width = int(plen.max())
    pool = np.full((n_patterns + 1, width), -1, dtype=np.int64)  # last row: no pattern
    for i in range(n_patterns):
        seg = p_items[p_off[i]:p_off[i + 1]]
        pool[i, :seg.size] = seg
    choice = np.where(rng.random(n) < planted, rng.integers(0, n_patterns, n), n_patterns)
    lengths = np.clip(rng.poisson(mean, n), 1, n_items)
    offsets, items = _sample_distinct(rng, zipf, lengths, prefix=pool[choice])
    lengths = np.diff(offsets.astype(np.int64))
    keep = rng.random(n) >= empty
    starts = offsets[:-1].astype(np.int64)
    mask = np.repeat(keep, lengths)
    new_len = np.where(keep, lengths, 0).astype(np.uint64)
    new_off = np.zeros(n + 1, dtype=np.uint64)
    np.cumsum(new_len, out=new_off[1:])
    del starts
    timestamps = np.cumsum(rng.integers(0, 4, n)).astype(np.int64)
    return TransactionCSR(new_off, items[mask], n_items), timestamps


def workload(name: str):
    """``(csr, minSup)`` for a named single-database workload."""
    gen, minsup = _WORKLOADS[name]
    return gen(), minsup
