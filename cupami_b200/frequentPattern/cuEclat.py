"""Drop-in ``cuEclat`` on the B200 vertical-bitset engine.

Same API as cuPAMI's ``cupami.frequentPattern.cuEclat``
(``cupami/frequentPattern/cuEclat.py:81-248``).  ``mine()`` runs the whole
search on the device: singleton supports, the pair level as a Gram matrix of
the frequent items' tidsets, and every deeper equivalence class in one
persistent work-queue kernel (``libcupami_b200.so``).  Patterns and supports
equal the reference's, and ``getPatterns()`` lists them in the reference's
insertion order (singletons, pairs, then each class in search order).

Subclasses that override the ``_candidatePairs`` / ``_extensionBatch`` hooks
(``cupami/georeferencedFrequentPattern/cuSpatialEclat.py:197-211`` does) get a
host-scheduled class search that calls the hooks exactly where the reference
does and counts with the device kernels of :mod:`._bitsets`.
"""

from __future__ import annotations

import sys
import time
from itertools import combinations, islice

from .. import _native
from . import _bitsets
from .cuApriori import IdLabels, _cli, cuApriori


class cuEclat(cuApriori):
    """Depth-first prefix-class search over device tidsets."""

    _ALGORITHM = _native.CPM_ECLAT
    _ORDER = _native.CPM_ORDER_ECLAT

    # Batch limits of the reference (cuEclat.py:165-166).  They bound host-side
    # batches of the hook-driven search; the fused device search does not need
    # them and gives the same patterns either way.
    _PAIR_BATCH_SIZE = 65536
    _INTERSECTION_BATCH_BYTES = 64 * 1024 * 1024

    def _hooksOverridden(self):
        cls = type(self)
        return (cls._candidatePairs is not cuEclat._candidatePairs
                or cls._extensionBatch is not cuEclat._extensionBatch)

    def mine(self):
        if not self._hooksOverridden():
            return super().mine()
        self._mineWithHooks()

    @classmethod
    def mineBatch(cls, sources, minSup, **kwargs):
        """Mine many independent databases in one device pass.

        ``sources`` are anything the constructor accepts; ``minSup`` is one
        threshold for all or a list.  Returns one miner per source with its
        patterns in place, as if ``mine()`` had run on each.  Every miner's
        mining time is the time of the whole batch.  (The reference mines one
        database per call.)
        """
        sups = list(minSup) if isinstance(minSup, (list, tuple)) else [minSup] * len(sources)
        miners = [cls(src, sup, **kwargs) for src, sup in zip(sources, sups)]
        if not miners:
            return miners
        ctx = cls._getCudaModule()
        mine_start = time.perf_counter()
        if miners[0].scheduler == "learned":
            from .. import costmodel

            costmodel.ensure_default(ctx)
        if all(m._csr is not None for m in miners):
            # Integer-id sources: one upload and one packing pass for the whole batch.
            dbs = _native.Database.from_ids_batch(ctx, [m._csr for m in miners])
            labels = [IdLabels(db.labels) for db in dbs]  # strings on first use
        else:
            dbs, labels = zip(*(m._deviceDatabase(ctx) for m in miners))
        try:
            results = _native.mine_batch(ctx, list(dbs), [m._minSup for m in miners], miners[0]._options(),
                                         cls._ORDER)
        finally:
            for db in dbs:
                db.close()
        end = time.perf_counter()
        for m, res, lab in zip(miners, results, labels):
            m._result, m._labels, m._patterns = res, lab, None
            m._startTime, m._endTime = mine_start, end
        return miners

    def _candidatePairs(self, frequent, items):
        return combinations(frequent, 2)

    def _extensionBatch(self, cp, prefix, labels, bitsets, start, stop):
        return labels[start:stop], bitsets[start:stop]

    # ---- host-scheduled search for subclasses with hooks -------------------

    def _mineWithHooks(self):
        """The reference's driver order (cuEclat.py:168-245) over device kernels."""
        self._startTime = time.perf_counter()
        self._getCudaModule()
        xp = _bitsets.array_module()
        patterns = {}
        items, rows, columns = self._getDevicePairs(xp)
        bitsets = _bitsets.build_bitsets(xp, rows, columns, self._transactionCount, len(items))
        supports = _bitsets.count_supports(xp, bitsets, [[i] for i in range(len(items))])
        frequent = [i for i, s in enumerate(supports) if s >= self._minSup]
        for i in frequent:
            patterns[(items[i],)] = int(supports[i])
        classes = {}
        pairs = self._candidatePairs(frequent, items)
        while True:
            batch = list(islice(pairs, max(1, int(self._PAIR_BATCH_SIZE))))
            if not batch:
                break
            for (left, right), support in zip(batch, _bitsets.count_supports(xp, bitsets, batch)):
                if support >= self._minSup:
                    patterns[(items[left], items[right])] = int(support)
                    classes.setdefault(left, []).append(right)
        for left, members in classes.items():
            if len(members) < 2:
                continue
            vertical = bitsets[xp.asarray(members, dtype=xp.int64)] & bitsets[left]
            self._searchClassWithHooks(xp, (items[left],), [items[m] for m in members], vertical, patterns)
        _bitsets.synchronize()
        self._labels = []
        self._result = None
        self._patterns = patterns
        self._endTime = time.perf_counter()

    def _searchClassWithHooks(self, xp, prefix, labels, vertical, patterns):
        stack = [(prefix, labels, vertical, 0)]
        while stack:
            prefix, labels, vertical, position = stack.pop()
            if position >= len(labels) - 1:
                continue
            stack.append((prefix, labels, vertical, position + 1))
            head = prefix + (labels[position],)
            words = int(vertical.shape[1])
            batch = max(1, int(self._INTERSECTION_BATCH_BYTES) // max(1, 4 * words))
            names, kept = [], []
            for start in range(position + 1, len(labels), batch):
                stop = min(len(labels), start + batch)
                batchLabels, batchBits = self._extensionBatch(xp, head, labels, vertical, start, stop)
                if not batchLabels:
                    continue
                children, sups = _bitsets.intersect_extensions(xp, vertical[position], batchBits)
                keep = [k for k, s in enumerate(sups) if s >= self._minSup]
                for k in keep:
                    patterns[head + (batchLabels[k],)] = int(sups[k])
                    names.append(batchLabels[k])
                if keep:
                    kept.append(children[xp.asarray(keep, dtype=xp.int64)])
            if len(names) > 1:
                stack.append((head, names, kept[0] if len(kept) == 1 else xp.concatenate(kept), 0))

    def _getDevicePairs(self, xp):
        """(sorted labels, row per occurrence, column per occurrence) on the device."""
        import numpy as np

        if self._csr is not None:
            offsets, ids = self._csr
            uniq = np.unique(ids)
            items = sorted(map(str, uniq.tolist()))
            index = {label: i for i, label in enumerate(items)}
            colmap = np.array([index[str(v)] for v in uniq.tolist()], dtype=np.uint32)
            lengths = np.diff(offsets.astype(np.int64))
            active = np.cumsum(lengths > 0) - 1
            rows = np.repeat(active, lengths).astype(np.uint64)
            cols = colmap[np.searchsorted(uniq, ids)] if ids.size else np.zeros(0, np.uint32)
            return items, xp.asarray(rows, dtype=xp.uint64), xp.asarray(cols, dtype=xp.uint32)
        items = sorted({item for row in self._Database for item in row})
        index = {item: i for i, item in enumerate(items)}
        rows, cols = [], []
        for r, row in enumerate(self._Database):
            rows.extend([r] * len(row))
            cols.extend(index[item] for item in row)
        return (items, xp.asarray(np.array(rows, dtype=np.uint64), dtype=xp.uint64),
                xp.asarray(np.array(cols, dtype=np.uint32), dtype=xp.uint32))


Eclat = cuEclat


if __name__ == "__main__":
    _cli(cuEclat, sys.argv)
