"""Temporal input and the periodicity measure of cuPAMI's periodic-frequent miners.

Drop-in for ``cupami/periodicFrequentPattern/_temporal.py``: the same
constructor, input rules and output API as ``TemporalInput`` (``:56-181``),
with the mining done by ``libcupami_b200.so`` (``cpm_tdb_from_csr`` and
``cpm_mine_periodic``) instead of a Python search that launches the
``periodic_counts`` kernel per batch of candidates (``:26-53``, ``:156-165``).

Input rules (reference ``:67-147``):

* a row is ``timestamp, item, item, ...``; timestamps are nonnegative int64
  integers given as integers or digit strings (``:89-99``);
* rows that are empty or blank are skipped; a row with a timestamp and no items
  is an empty basket: it keeps its timestamp and counts in the support
  denominator (``:125-136``);
* rows are sorted by timestamp, equal timestamps stay separate transactions in
  input order (``:133``);
* the timeline runs from 0 to the largest timestamp or ``endTime`` (``:134-137``);
* ``minSup`` as in ``cuApriori``; ``maxPer`` floats in (0, 1] are fractions of
  the timeline end, anything else is in timestamp units (``:85``).

Integer inputs given as a :class:`~cupami_b200.datasets.TemporalCSR` take a
numeric path: the arrays are checked and sorted by timestamp as they are, and
the ids are mapped to columns in the order of their decimal strings -- the
labels and columns the string path builds, without Python rows.

An itemset is kept when its support is positive and reaches ``minSup`` and its
periodicity -- the largest gap between consecutive timestamps of the rows
holding it, counting the gap from 0 to the first and from the last to the end
-- is at most ``maxPer`` (``:166-171``).
"""

from __future__ import annotations

import csv
import io
import math
import numbers
import struct
import time
from itertools import chain
from pathlib import Path
from urllib.parse import urlparse
from urllib.request import urlopen

import numpy as np

from .. import _native
from ..datasets import TemporalCSR
from ..frequentPattern.cuApriori import _PatternDict, cuApriori

__all__ = ["TemporalInput", "periodic_counts", "read_binary", "read_parquet"]

_MAGIC = b"CUPAMIT1"
_HEADER = struct.Struct("<8sQQQ")
_INT64_MAX = np.iinfo(np.int64).max


def read_binary(path):
    """Rows ``[timestamp, *items]`` of a temporal BIN file.

    Layout (cupami/extras/_temporal_io.py:28-71): header ``<8sQQQ>`` = magic
    ``CUPAMIT1``, row count, item count, item universe; then int64 timestamps
    (one per row), uint64 offsets (rows + 1) and uint32 item ids.
    """
    with Path(path).open("rb") as source:
        header = source.read(_HEADER.size)
        if len(header) != _HEADER.size:
            raise ValueError("Invalid temporal BIN header")
        magic, count, total, universe = _HEADER.unpack(header)
        if magic != _MAGIC:
            raise ValueError("Expected a temporal BIN file with timestamp data")
        if not 1 <= universe <= 0xFFFFFFFF:
            raise ValueError("Invalid temporal BIN item range")
        if Path(path).stat().st_size != _HEADER.size + 8 * count + 8 * (count + 1) + 4 * total:
            raise ValueError("Invalid temporal BIN file size")
        timestamps = np.fromfile(source, dtype="<i8", count=count)
        offsets = np.fromfile(source, dtype="<u8", count=count + 1)
        items = np.fromfile(source, dtype="<u4", count=total)
    if timestamps.size != count or offsets.size != count + 1 or items.size != total:
        raise ValueError("Truncated temporal BIN arrays")
    if np.any(timestamps < 0):
        raise ValueError("Temporal timestamps must be nonnegative")
    if offsets[0] != 0 or offsets[-1] != total or np.any(offsets[1:] < offsets[:-1]):
        raise ValueError("Invalid temporal BIN offsets")
    if np.any(items > universe):
        raise ValueError("Temporal BIN item ID exceeds header range")
    ids = items.tolist()
    bounds = offsets.tolist()
    return [[int(t), *ids[bounds[i]:bounds[i + 1]]] for i, t in enumerate(timestamps.tolist())]


def read_parquet(path):
    """Rows ``[timestamp, *items]`` of a temporal Parquet file (columns
    ``timestamp: int64`` and ``items: list<uint32>``, cupami/extras/_temporal_io.py:105-118)."""
    try:
        import pyarrow as pa
        import pyarrow.parquet as pq
    except ImportError as error:
        raise ImportError("Temporal Parquet requires pyarrow: pip install pyarrow") from error
    table = pq.read_table(path)
    if "timestamp" not in table.column_names or "items" not in table.column_names:
        raise ValueError("Temporal Parquet requires timestamp and items columns")
    timestamp, items = table["timestamp"].combine_chunks(), table["items"].combine_chunks()
    if timestamp.type != pa.int64() or not pa.types.is_list(items.type) or items.type.value_type != pa.uint32():
        raise ValueError("Temporal Parquet requires timestamp: int64 and items: list<uint32>")
    if timestamp.null_count or items.null_count or items.flatten().null_count:
        raise ValueError("Temporal Parquet cannot contain null timestamps, baskets, or items")
    stamps = timestamp.to_pylist()
    if any(value < 0 for value in stamps):
        raise ValueError("Temporal timestamps must be nonnegative")
    return [[t, *basket] for t, basket in zip(stamps, items.to_pylist())]


def periodic_counts(bitsets, candidates, timestamps, transactions, end):
    """``[(support, periodicity)]`` of each candidate: the reference kernel
    ``periodic_counts`` (_temporal.py:26-53) as ``_evaluate`` launches it
    (:156-165).  ``bitsets`` is the uint32[items][words] tensor of
    ``frequentPattern._bitsets.build_bitsets``, ``timestamps`` an int64 CUDA
    tensor with one entry per transaction row."""
    import torch

    from ..frequentPattern import _bitsets

    if not len(candidates):
        return []
    cand = np.ascontiguousarray(np.asarray(candidates, dtype=np.uint32)).view(np.int32)
    d_cand = torch.from_numpy(cand.copy()).cuda()
    supports = torch.zeros(cand.shape[0], dtype=torch.int64, device="cuda")
    periods = torch.zeros(cand.shape[0], dtype=torch.int64, device="cuda")
    bitsets = bitsets.contiguous()
    timestamps = timestamps.contiguous()
    ctx = _bitsets._ctx(bitsets)
    with ctx.lock:
        ctx.check(_native.library().cpm_periodic_counts(
            ctx.handle, bitsets.data_ptr() if bitsets.numel() else None, int(bitsets.shape[1]),
            d_cand.data_ptr(), cand.shape[0], cand.shape[1],
            timestamps.data_ptr() if timestamps.numel() else None, int(transactions), int(end),
            supports.data_ptr(), periods.data_ptr()))
        ctx.check(_native.library().cpm_synchronize(ctx.handle))
    return list(zip(supports.cpu().tolist(), periods.cpu().tolist()))


class TemporalInput(cuApriori):
    """Timestamp-first CSV, temporal BIN/Parquet, or iterable input.

    Equal timestamps remain separate transactions; duplicate items within a
    basket count once.  Empty baskets retain their timestamp and count in the
    support denominator.  Rows are sorted by timestamp.  The timeline starts
    at 0 and ends at the largest input timestamp (or explicit ``endTime``).
    """

    _ALGORITHM = _native.CPM_ECLAT
    _ORDER = _native.CPM_ORDER_DEPTH_FIRST

    def __init__(self, iFile, minSup, maxPer, sep=None, *, endTime=None):
        loading_start = time.perf_counter()
        self._timestamps = []
        self._tcsr = None  # (offsets, ids, timestamps) of a TemporalCSR input, rows sorted by timestamp
        self.endTime = endTime
        self.maxPer = maxPer
        super().__init__(iFile, minSup, sep, use_gds=False, use_gpu_io=False)
        if isinstance(minSup, bool) or not isinstance(minSup, numbers.Real) or not math.isfinite(minSup) or minSup <= 0:
            raise ValueError("minSup must be a positive finite number")
        if isinstance(maxPer, bool) or not isinstance(maxPer, numbers.Real) or not math.isfinite(maxPer) or maxPer < 0:
            raise ValueError("maxPer must be a nonnegative finite number")
        # Fractions refer to elapsed timestamp units, not to the number of records.
        self._maxPer = maxPer * self._endTimestamp if isinstance(maxPer, float) and 0 < maxPer <= 1 else maxPer
        self._loadingTime = time.perf_counter() - loading_start

    @staticmethod
    def _timestamp(value):
        if isinstance(value, (bool, float)):
            raise ValueError("timestamps must be nonnegative int64 integers")
        text = str(value).strip()
        if not text or any(c not in "0123456789" for c in text):
            raise ValueError("timestamps must be nonnegative int64 integers")
        timestamp = int(text)
        if timestamp > _INT64_MAX:
            raise ValueError("timestamp exceeds int64")
        return timestamp

    def _readTransactions(self, source):
        if isinstance(source, TemporalCSR):
            return self._useTemporalCsr(source)
        if isinstance(source, (str, Path)):
            suffix = Path(str(source)).suffix.lower()
            is_url = urlparse(str(source)).scheme in ("http", "https")
            if suffix in (".bin", ".parquet"):
                if is_url:
                    raise ValueError("Temporal BIN and Parquet input requires a local file")
                rows = read_binary(source) if suffix == ".bin" else read_parquet(source)
                return self._cleanTemporalRows(rows)
            if is_url:
                with urlopen(str(source), timeout=30) as response:
                    text = response.read().decode("utf-8-sig")
            else:
                text = Path(source).read_text(encoding="utf-8-sig")
            separator = self.sep
            if separator is None:
                first = next((line for line in text.splitlines() if line.strip()), "")
                separator = "\t" if "\t" in first else "," if "," in first else None
            rows = (csv.reader(io.StringIO(text), delimiter=separator) if separator
                    else (line.split() for line in text.splitlines()))
        else:
            rows = source
        return self._cleanTemporalRows(rows)

    def _setTimeline(self, last):
        self._endTimestamp = last if self.endTime is None else self._timestamp(self.endTime)
        if self._endTimestamp < last:
            raise ValueError("endTime must be at least the last timestamp")

    def _useTemporalCsr(self, source):
        """Integer arrays: every row a transaction (empty ones too), sorted by timestamp (stable)."""
        offsets = np.ascontiguousarray(source.offsets, dtype=np.uint64)
        ids = np.ascontiguousarray(source.items, dtype=np.uint32)
        ts = np.asarray(source.timestamps)
        n = offsets.size - 1
        if n < 0 or ts.shape != (n,):
            raise ValueError("TemporalCSR needs one timestamp per row")
        if not np.issubdtype(ts.dtype, np.integer) or (ts.size and (ts.min() < 0 or ts.max() > _INT64_MAX)):
            raise ValueError("timestamps must be nonnegative int64 integers")
        ts = ts.astype(np.int64)
        if offsets[0] != 0 or offsets[-1] != ids.size or np.any(offsets[1:] < offsets[:-1]):
            raise ValueError("Invalid TemporalCSR offsets")
        if np.any(ts[1:] < ts[:-1]):
            order = np.argsort(ts, kind="stable")
            lengths = np.diff(offsets.astype(np.int64))[order]
            starts = offsets[:-1].astype(np.int64)[order]
            new_offsets = np.zeros(n + 1, dtype=np.int64)
            np.cumsum(lengths, out=new_offsets[1:])
            gather = np.repeat(starts - new_offsets[:-1], lengths) + np.arange(int(new_offsets[-1]), dtype=np.int64)
            ids = ids[gather]
            offsets = new_offsets.astype(np.uint64)
            ts = ts[order]
        self._tcsr = (offsets, ids, ts)
        self._transactionCount = n
        self._timestamps = ts.tolist()
        self._setTimeline(int(ts[-1]) if n else 0)
        self._inputBackend = {"backend": "numpy-cuda",
                              "reason": "Integer temporal arrays sent to the GPU; no Python transactions"}
        return None

    def _cleanTemporalRows(self, rows):
        records = []
        for row in rows:
            row = list(row)
            if not row or not any(str(value).strip() for value in row):
                continue
            records.append((self._timestamp(row[0]), self._cleanTransaction(row[1:])))
        records.sort(key=lambda record: record[0])
        self._timestamps = [record[0] for record in records]
        self._setTimeline(self._timestamps[-1] if records else 0)
        self._inputBackend = {"backend": "cpu", "reason": "Temporal reader; mining uses CUDA"}
        return [record[1] for record in records]

    def _periodLimit(self):
        """The largest periodicity that passes, as an int64 (periods are integers)."""
        return min(math.floor(self._maxPer), int(_INT64_MAX))

    def _temporalColumns(self):
        """(offsets, columns, n_items, timestamps, labels) of the tidsets to build."""
        if self._tcsr is not None:
            offsets, ids, ts = self._tcsr
            top = int(ids.max()) if ids.size else 0
            small = top < (1 << 24)  # a dense table over the id range
            if small:
                present = np.zeros(top + 1, dtype=bool)
                present[ids] = True
                uniq = np.flatnonzero(present)
            else:
                uniq = np.unique(ids)
            names = [str(v) for v in uniq.tolist()]
            order = sorted(range(len(names)), key=names.__getitem__)  # decimal-string order of the ids
            rank = np.empty(len(names), dtype=np.uint32)
            rank[order] = np.arange(len(names), dtype=np.uint32)
            if not ids.size:
                cols = np.zeros(0, dtype=np.uint32)
            elif small:
                table = np.zeros(top + 1, dtype=np.uint32)
                table[uniq] = rank
                cols = table[ids]
            else:
                cols = rank[np.searchsorted(uniq, ids)]
            return offsets, cols, len(names), ts, [names[i] for i in order]
        flat = list(chain.from_iterable(self._Database))
        labels = sorted(set(flat))
        index = dict(zip(labels, range(len(labels))))
        n = len(self._Database)
        offsets = np.zeros(n + 1, dtype=np.uint64)
        np.cumsum(np.fromiter(map(len, self._Database), dtype=np.uint64, count=n), out=offsets[1:])
        cols = np.fromiter(map(index.__getitem__, flat), dtype=np.uint32, count=len(flat))
        return offsets, cols, len(labels), np.asarray(self._timestamps, dtype=np.int64), labels

    def _deviceDatabase(self, ctx):
        """Temporal tidsets (every row, empty ones too) and the sorted labels."""
        offsets, cols, n_items, timestamps, labels = self._temporalColumns()
        return _native.Database.from_temporal(ctx, offsets, cols, n_items, timestamps, self._endTimestamp), labels

    def autotune(self):
        raise NotImplementedError("the periodic miners have no launch shapes to tune")

    def mine(self):
        self._startTime = time.perf_counter()
        ctx = self._getCudaModule()
        db, labels = self._deviceDatabase(ctx)
        try:
            result = db.mine_periodic(self._minSup, self._periodLimit(), self._ALGORITHM, self._ORDER)
        finally:
            db.close()
        self._labels = labels
        self._result = result
        self._patterns = None
        self._endTime = time.perf_counter()

    @property
    def _periods(self):
        res = self._result
        if res is None:
            return {}
        return _PatternDict(zip(self._finalPatterns.keys(), res.periods.tolist()))

    def getPatterns(self):
        periods = self._result.periods.tolist() if self._result is not None else []
        return {"\t".join(pattern): (support, period)
                for (pattern, support), period in zip(self._finalPatterns.items(), periods)}

    def getPatternsAsDataFrame(self):
        import pandas as pd

        periods = self._periods
        return pd.DataFrame([("\t".join(p), s, periods[p]) for p, s in self._finalPatterns.items()],
                            columns=["Patterns", "Support", "Periodicity"])

    def save(self, outputFile):
        periods = self._periods
        with Path(outputFile).open("w", encoding="utf-8") as output:
            for pattern, support in sorted(self._finalPatterns.items()):
                output.write("{} : {} : {}\n".format("\t".join(pattern), support, periods[pattern]))
