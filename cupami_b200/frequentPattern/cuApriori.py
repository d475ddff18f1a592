"""Drop-in ``cuApriori`` on the B200 vertical-bitset engine.

Same constructor, threshold rule, output and timing API as cuPAMI's
``cupami.frequentPattern.cuApriori`` (``cupami/frequentPattern/cuApriori.py:173-593``);
the mining runs in ``libcupami_b200.so`` (sm_100a kernels behind a C ABI), not
in CuPy.  There is no CPU fallback: without the library or a CUDA device,
``mine()`` raises.

Input handling follows the reference's semantics:

* labels are ``str(value).strip()``; repeated labels in a basket count once;
  empty baskets are dropped and do not count towards the transaction total
  (``cuApriori.py:435-450``);
* item order is the sorted order of the label strings (``cuApriori.py:397``);
* ``minSup`` floats in (0, 1] are fractions rounded up, anything else is
  ``int(minSup)`` (``cuApriori.py:452-456``).

Integer inputs (BIN files, Parquet ``list<uint32>`` columns and
:class:`~cupami_b200.datasets.TransactionCSR` objects) take a numeric path:
the CSR arrays go to the device as they are and the library orders the ids as
their decimal strings sort, which yields the same labels and columns as the
string path without building Python baskets.
"""

from __future__ import annotations

import csv
import io
import math
import struct
import sys
import time
from collections.abc import Sequence
from itertools import chain
from pathlib import Path
from urllib.parse import urlparse
from urllib.request import urlopen

import numpy as np

from .. import _native
from ..datasets import TransactionCSR

_BIN_MAGIC = b"CUPAMI01"


class IdLabels(Sequence):
    """Column labels of a database loaded from integer ids: the decimal string
    of each column's id, made on first use (a batch of databases need not
    build them while it mines)."""

    def __init__(self, ids):
        self._ids = ids
        self._str = None

    def _strings(self):
        if self._str is None:
            self._str = [str(v) for v in self._ids.tolist()]
        return self._str

    def __len__(self):
        return len(self._ids)

    def __getitem__(self, i):
        return self._strings()[i]

    def __iter__(self):
        return iter(self._strings())


class _PatternDict(dict):
    """``_finalPatterns`` built on first use from the mined arrays."""


class cuApriori:
    """Level-wise frequent itemset mining with device-side support counting.

    Parameters mirror the reference: ``iFile`` (rows, CSV/TSV/text path, BIN,
    Parquet, HTTP(S) text URL or a ``TransactionCSR``), ``minSup``, ``sep``,
    ``use_gds`` and ``use_gpu_io`` ("auto", True or False).
    """

    _ALGORITHM = _native.CPM_APRIORI
    _ORDER = _native.CPM_ORDER_APRIORI

    #: Deep-level scheduler: "plain" (size ordered) or "learned" (cost model).
    scheduler = "plain"
    #: Bound on every device wait (0: the library default).  A small value
    #: makes a wait run out and mine() raise instead of waiting on.
    _SPIN_LIMIT = 0
    #: Pair-level engine: 0 automatic, 1 tensor-core Gram, 2 CUDA-core Gram.
    _PAIR_ENGINE = 0
    #: Device arena for child tidsets in bytes (0: as much as the GPU holds).
    #: A small arena makes the deep levels run in memory-bounded rounds.
    _ARENA_BYTES = 0
    #: Deep-level launch shape: threads per CTA (128/256/512/1024) and CTAs per SM
    #: (1-4); 0 leaves each to the library (or to the autotuner's table).
    _DEEP_BLOCK = 0
    _DEEP_CTAS_PER_SM = 0
    #: Tidset forms of the deep levels: 0 automatic (bitsets, plus transaction-id
    #: lists for sparse tidsets of databases too big for the L2); 1 bitsets
    #: only; 2 lists wherever possible.
    _TIDSETS = 0
    #: Deep-level siblings of a unit: 0 automatic, 1 one warp per sibling,
    #: 2 split over the warps by size.
    _DEEP_BALANCE = 0
    #: Deep levels below small prefixes: 0 automatic (children of a prefix of
    #: at most 65,408 transactions become bitsets numbered by rank within it,
    #: mined one unit per warp, when the search is large enough); 1 off;
    #: 128-65408 the largest projected prefix, always.
    _DEEP_PROJECT = 0
    #: Deep levels of one database with projection: 0 automatic (units whose
    #: prefix rows are cheaper than their siblings' tidsets count row by
    #: row); 1 off.
    _DEEP_ROWS = 0

    def __init__(self, iFile, minSup, sep=None, use_gds="auto", use_gpu_io="auto"):
        t0 = time.perf_counter()
        # The two switches accept the same three values as the reference, with its messages.
        for flag, value in (("use_gds", use_gds), ("use_gpu_io", use_gpu_io)):
            if value not in ("auto", True, False):
                raise ValueError(f'{flag} must be "auto", True, or False')
        self.iFile, self.minSup, self.sep = iFile, minSup, sep
        self.use_gds, self.use_gpu_io = use_gds, use_gpu_io
        self._csr = None               # (offsets, ids) when the input is numeric
        self._inputBackend = {"backend": "cpu", "reason": "Text or Parquet input"}
        if use_gds is True and not self._isLocalBin(iFile):
            raise ValueError("Required GDS input currently supports local BIN files only")
        # Numeric inputs set _csr and the transaction count and return None.
        self._Database = self._readTransactions(iFile)
        if self._Database is not None:
            self._transactionCount = len(self._Database)
        self._minSup = self._getSupportCount(minSup, self._transactionCount)
        self._patterns = None          # cached dict built from the arrays
        self._result = None            # _native.Result of the latest mine()
        self._labels = []
        self._startTime = self._endTime = 0.0
        self._loadingTime = time.perf_counter() - t0

    @staticmethod
    def _isLocalBin(source):
        return (isinstance(source, (str, Path)) and Path(source).suffix.lower() == ".bin"
                and urlparse(str(source)).scheme not in ("http", "https"))

    # ---- input -----------------------------------------------------------

    def _readTransactions(self, source):
        if isinstance(source, TransactionCSR):
            return self._useCsr(source.offsets, source.items, "numpy-cuda",
                                "Integer CSR arrays; no Python transactions")
        if isinstance(source, str) and urlparse(source).scheme in ("http", "https"):
            with urlopen(source, timeout=30) as response:
                stream = io.TextIOWrapper(response, encoding="utf-8", newline="")
                return self._readDelimitedFile(stream)
        if isinstance(source, (str, Path)):
            suffix = Path(source).suffix.lower()
            if suffix == ".bin":
                return self._readBinaryFile(Path(source))
            if suffix == ".parquet":
                return self._readParquetFile(source)
            if self._tryDeviceText(Path(source)):
                return None
            with Path(source).open("r", newline="", encoding="utf-8") as stream:
                return self._readDelimitedFile(stream)
        return self._cleanTransactions(source)

    def _useCsr(self, offsets, ids, backend, reason):
        offsets = np.ascontiguousarray(offsets, dtype=np.uint64)
        ids = np.ascontiguousarray(ids, dtype=np.uint32)
        self._csr = (offsets, ids)
        self._transactionCount = int(np.count_nonzero(offsets[1:] > offsets[:-1]))
        previous = self._inputBackend.get("reason")
        self._inputBackend = {"backend": backend, "reason": reason}
        if previous and backend == "numpy-cuda":
            self._inputBackend["gds_fallback_reason"] = previous
        self._inputBackend["direct_gds_verified"] = False
        return None

    def _tryDeviceText(self, path):
        """Integer baskets in delimited text, parsed on the GPU (the role of the
        reference's cuDF reader, _gpu_io.py:34-54); False leaves the file to the
        CPU reader: use_gpu_io=False, no usable device, or another layout."""
        if self.use_gpu_io is False:
            return False
        try:
            data = path.read_bytes()
            head = data.split(b"\n", 1)[0].decode("utf-8", "replace")
            sep = self.sep if self.sep is not None else ("\t" if "\t" in head else ",")
            if len(sep) != 1 or not sep.isascii():
                raise _native.NativeError(_native.CPM_EINVAL, "the GPU text reader takes a one-byte separator")
            offsets, ids = _native.parse_int_text(self._getCudaModule(), data, sep)
        except (ImportError, RuntimeError) as error:
            if self.use_gpu_io is True:
                raise RuntimeError(f"GPU input unavailable: {error}") from error
            self._inputBackend = {"backend": "cpu", "reason": str(error)}
            return False
        self._useCsr(offsets, ids, "cuda-text", "Integer baskets parsed on the GPU; no Python transactions")
        return True

    def _gdsUnavailable(self):
        reason = "GDS (cuFile/KvikIO) is not part of this engine"
        self._inputBackend = {"backend": "cpu", "reason": reason}
        if self.use_gds is True:
            raise RuntimeError(f"GDS input requested but unavailable: {reason}")

    def _readBinaryFile(self, path):
        """The CUPAMI01 BIN layout (docs/transaction-formats.md, 'Transactional BIN')."""
        with path.open("rb") as source:
            header = source.read(32)
            if len(header) != 32:
                raise ValueError("Invalid BIN file: truncated header")
            magic, count, total, universe = struct.unpack("<8sQQQ", header)
            if magic != _BIN_MAGIC:
                raise ValueError("Invalid BIN file: expected CUPAMI01 format")
            if not 1 <= universe <= 0xFFFFFFFF:
                raise ValueError("Invalid BIN file: item universe must fit in uint32")
            if path.stat().st_size != 32 + 8 * (count + 1) + 4 * total:
                raise ValueError("Invalid BIN file: size does not match header")
            if self.use_gds is False:
                self._inputBackend = {"backend": "cpu", "reason": "GDS disabled"}
            else:
                self._gdsUnavailable()
            offsets = np.fromfile(source, dtype="<u8", count=count + 1)
            ids = np.fromfile(source, dtype="<u4", count=total)
        if offsets.size != count + 1 or ids.size != total:
            raise ValueError("Invalid BIN file: truncated arrays")
        if offsets[0] != 0 or offsets[-1] != total or np.any(offsets[1:] < offsets[:-1]):
            raise ValueError("Invalid BIN file: invalid transaction offsets")
        if np.any(ids > universe):
            raise ValueError("Invalid BIN file: item ID outside configured universe")
        if self.use_gpu_io is False:
            rows = (ids[offsets[i]:offsets[i + 1]].tolist() for i in range(count))
            return self._cleanTransactions(rows)
        return self._useCsr(offsets, ids, "numpy-cuda",
                            "Bulk numeric BIN reads and GPU transfers; no Python transactions")

    def _readParquetFile(self, path):
        try:
            import pyarrow as pa
            import pyarrow.parquet as pq
        except ImportError as error:
            raise ImportError("Parquet input requires pyarrow: pip install pyarrow") from error
        parquet = pq.ParquetFile(path)
        schema = parquet.schema_arrow
        if "items" not in schema.names:
            raise ValueError("Invalid Parquet file: missing items column")
        itemType = schema.field("items").type
        if not pa.types.is_list(itemType) or not pa.types.is_uint32(itemType.value_type):
            raise ValueError("Invalid Parquet file: items must be a list of uint32 IDs")
        column = parquet.read(columns=["items"]).column("items").combine_chunks()
        if column.null_count or (len(column) and column.values.null_count):
            raise ValueError("Invalid Parquet file: null transactions or item IDs")
        if self.use_gpu_io is False:
            return self._cleanTransactions(column.to_pylist())
        offsets = np.asarray(column.offsets, dtype=np.int64)
        values = np.asarray(column.values, dtype=np.uint32)
        base = offsets[0] if offsets.size else 0
        return self._useCsr((offsets - base).astype(np.uint64), values[base:offsets[-1]] if offsets.size else values,
                            "arrow-cuda", "Parquet list arrays sent to the GPU; no Python transactions")

    def _readDelimitedFile(self, inputStream):
        """Rows of delimited text; with no ``sep`` the first line decides between
        a tab (when it holds one) and a comma, as the reference does."""
        head = inputStream.readline()
        sep = self.sep if self.sep is not None else ("\t" if "\t" in head else ",")
        return self._cleanTransactions(csv.reader(chain((head,), inputStream), delimiter=sep))

    def _cleanTransactions(self, rows):
        """Cleaned baskets, empty ones left out."""
        return [basket for basket in map(self._cleanTransaction, rows) if basket]

    @staticmethod
    def _cleanTransaction(transaction):
        """Stripped, non-empty labels in first-seen order, each once."""
        labels = (str(value).strip() for value in transaction)
        return tuple(dict.fromkeys(label for label in labels if label))

    @staticmethod
    def _getSupportCount(minSup, transactionCount):
        if isinstance(minSup, float) and 0 < minSup <= 1:
            return math.ceil(minSup * transactionCount)
        return int(minSup)

    @staticmethod
    def _getCudaModule():
        """The native device context; raises like the reference when CUDA is missing."""
        return _native.context(0)

    def getInputBackend(self):
        return dict(self._inputBackend)

    # ---- mining ------------------------------------------------------------

    def _deviceDatabase(self, ctx):
        """Tidsets on the device plus the label of every column (sorted strings)."""
        if self._csr is not None:
            offsets, ids = self._csr
            db = _native.Database.from_ids(ctx, offsets, ids)
            return db, IdLabels(db.labels)
        flat = list(chain.from_iterable(self._Database))
        labels = sorted(set(flat))
        index = dict(zip(labels, range(len(labels))))
        offsets = np.zeros(len(self._Database) + 1, dtype=np.uint64)
        np.cumsum(np.fromiter(map(len, self._Database), dtype=np.uint64, count=len(self._Database)),
                  out=offsets[1:])
        cols = np.fromiter(map(index.__getitem__, flat), dtype=np.uint32, count=len(flat))
        return _native.Database.from_columns(ctx, offsets, cols, len(labels)), labels

    def _options(self):
        opts = _native.Opts()
        _native.library().cpm_default_opts(opts)
        opts.scheduler = (_native.CPM_SCHED_LEARNED if self.scheduler == "learned"
                          else _native.CPM_SCHED_PLAIN)
        if self._SPIN_LIMIT:
            opts.spin_limit = int(self._SPIN_LIMIT)
        opts.pair_engine = int(self._PAIR_ENGINE)
        opts.arena_bytes = int(self._ARENA_BYTES)
        opts.deep_block = int(self._DEEP_BLOCK)
        opts.deep_ctas_per_sm = int(self._DEEP_CTAS_PER_SM)
        opts.autotune = 1
        opts.tidsets = int(self._TIDSETS)
        opts.deep_balance = int(self._DEEP_BALANCE)
        opts.deep_project = int(self._DEEP_PROJECT)
        opts.deep_rows = int(self._DEEP_ROWS)
        return opts

    def autotune(self):
        """Time the deep-level launch shapes on this database and keep the fastest
        for databases with tidsets of this length (later mine() calls in this
        process use it), and the tidset form at that shape (``list_div`` 0:
        bitsets only).  Returns {"block", "ctas_per_sm", "list_div", "ms_deep"}."""
        ctx = self._getCudaModule()
        db, _ = self._deviceDatabase(ctx)
        try:
            return _native.autotune(ctx, db, self._minSup, self._options())
        finally:
            db.close()

    def mine(self):
        self._startTime = time.perf_counter()
        ctx = self._getCudaModule()
        if self.scheduler == "learned":
            from .. import costmodel

            costmodel.ensure_default(ctx)
        db, labels = self._deviceDatabase(ctx)
        try:
            result = db.mine(self._minSup, self._ALGORITHM, self._options(), self._ORDER)
        finally:
            db.close()
        self._labels = labels
        self._result = result
        self._patterns = None
        self._endTime = time.perf_counter()

    # ---- output --------------------------------------------------------------

    def _patternTuples(self):
        res = self._result
        if res is None:
            return []
        labels = self._labels
        o = res.offsets.tolist()
        items = [labels[c] for c in res.items.tolist()]
        return [tuple(items[o[k]:o[k + 1]]) for k in range(len(o) - 1)]

    @property
    def _finalPatterns(self):
        if self._patterns is None:
            res = self._result
            tuples = self._patternTuples()
            supports = res.supports.tolist() if res is not None else []
            self._patterns = _PatternDict(zip(tuples, supports))
        return self._patterns

    @_finalPatterns.setter
    def _finalPatterns(self, value):
        self._patterns = value

    def getPatternArrays(self):
        """``(offsets, columns, supports, labels)`` without building a dict."""
        res = self._result
        if res is None:
            return (np.zeros(1, np.uint64), np.zeros(0, np.uint32), np.zeros(0, np.uint64), [])
        return res.offsets, res.items, res.supports, self._labels

    def getKernelStats(self):
        """Device-side counters of the latest mine() (launches, bytes, times)."""
        return dict(self._result.stats) if self._result is not None else {}

    def getPatterns(self):
        """{tab-joined pattern: support} in the reference's insertion order."""
        res = self._result
        if self._patterns is None and res is not None and (
                isinstance(self._labels, IdLabels) or not any("\n" in label for label in self._labels)):
            # Keys joined in C straight from the result arrays: no tuple per pattern.
            keys = _native.join_labels(res.offsets, res.items, self._labels)
            return dict(zip(keys, res.supports.tolist()))
        return dict(zip(map("\t".join, self._finalPatterns), self._finalPatterns.values()))

    def getPatternsAsDataFrame(self):
        """The patterns of getPatterns() as a DataFrame with columns Patterns and Support."""
        import pandas as pd

        found = self.getPatterns()
        return pd.DataFrame({"Patterns": list(found), "Support": list(found.values())},
                            columns=["Patterns", "Support"])

    def save(self, outputFile):
        """One ``"<tab-joined pattern> : <support>"`` line per pattern, in sorted tuple order."""
        lines = ("\t".join(p) + f" : {v}\n" for p, v in sorted(self._finalPatterns.items()))
        with Path(outputFile).open("w", encoding="utf-8") as file:
            file.writelines(lines)

    def getRuntime(self):
        """Seconds the latest mine() took: upload, packing, mining and copy-back;
        the constructor's reading of the input is not in it."""
        return self._endTime - self._startTime

    def getLoadingTime(self):
        """Seconds the constructor spent reading and cleaning the input."""
        return self._loadingTime

    def getMiningTime(self):
        """Same as getRuntime()."""
        return self.getRuntime()

    def getTotalRuntime(self):
        """Reading plus the latest mine()."""
        return self.getLoadingTime() + self.getMiningTime()

    @staticmethod
    def _memory(kind):
        """Resident ("rss") or unique ("uss") bytes of this process; 0 without psutil."""
        try:
            import psutil
        except ImportError:
            return 0
        proc = psutil.Process()
        info = proc.memory_info() if kind == "rss" else proc.memory_full_info()
        return int(getattr(info, kind))

    def getMemoryRSS(self):
        return self._memory("rss")

    def getMemoryUSS(self):
        return self._memory("uss")

    def printResults(self):
        report = (("Total number of Frequent Patterns:", len(self._finalPatterns)),
                  ("Total Memory in USS:", self.getMemoryUSS()),
                  ("Total Memory in RSS:", self.getMemoryRSS()),
                  ("Loading time (seconds):", self.getLoadingTime()),
                  ("Mining time (seconds):", self.getMiningTime()),
                  ("Total time (seconds):", self.getTotalRuntime()))
        for caption, value in report:
            print(caption, value)


Apriori = cuApriori


def _cli(cls, argv):
    if len(argv) not in (4, 5):
        sys.exit(f"Usage: python -m {cls.__module__} <inputFile> <outputFile> <minSup> [sep]")
    try:
        minSup = int(argv[3])
    except ValueError:
        minSup = float(argv[3])
    miner = cls(argv[1], minSup, argv[4] if len(argv) == 5 else None)
    miner.mine()
    miner.save(argv[2])
    miner.printResults()


if __name__ == "__main__":
    _cli(cuApriori, sys.argv)
