"""CPU oracle for the vertical-bitset mining path -- TEST INFRASTRUCTURE ONLY.

Nothing in the product imports this package.  The test suite, the smoke check
and the benchmark's CPU-baseline leg use it as the checker:

* ``eclat`` / ``apriori`` call the C restatement in ``eclat_oracle.c``
  (built into ``oracle/_build/liboracle.so`` by :func:`build`);
* ``numpy_port`` restates the reference drivers with NumPy kernels, the way the
  reference runs when NumPy stands in for CuPy;
* ``labels_and_columns`` restates the reference's label handling
  (``cupami/frequentPattern/cuApriori.py:397-404`` and ``:443-456``).

Parity pin: ``tests/golden`` holds outputs of the reference drivers themselves,
produced by ``tests/golden/make_golden.py``; ``tests/test_oracle.py`` checks this
package against every one of them.
"""

from __future__ import annotations

import ctypes
import math
import os
import subprocess
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
_SO = _HERE / "_build" / "liboracle.so"
_lib = None


def build(force: bool = False) -> Path:
    """Compile the C restatement with gcc (OpenMP); returns the library path."""
    src = _HERE / "eclat_oracle.c"
    if force or not _SO.exists() or _SO.stat().st_mtime < src.stat().st_mtime:
        _SO.parent.mkdir(exist_ok=True)
        tmp = _SO.with_suffix(".so.tmp%d" % os.getpid())
        subprocess.check_call(["gcc", "-O3", "-fopenmp", "-fPIC", "-shared", "-mpopcnt",
                               "-o", str(tmp), str(src)])
        os.replace(tmp, _SO)
    return _SO


def _load():
    global _lib
    if _lib is None:
        if not _SO.exists():
            build()
        lib = ctypes.CDLL(str(_SO))
        for name in ("oracle_eclat", "oracle_apriori"):
            fn = getattr(lib, name)
            fn.restype = ctypes.c_void_p
            fn.argtypes = [ctypes.c_uint64, ctypes.c_uint32, ctypes.c_void_p,
                           ctypes.c_void_p, ctypes.c_int64, ctypes.c_int]
        lib.oracle_count.restype = ctypes.c_uint64
        lib.oracle_count.argtypes = [ctypes.c_void_p]
        lib.oracle_item_slots.restype = ctypes.c_uint64
        lib.oracle_item_slots.argtypes = [ctypes.c_void_p]
        lib.oracle_copy.argtypes = [ctypes.c_void_p] * 4
        lib.oracle_free.argtypes = [ctypes.c_void_p]
        _lib = lib
    return _lib


def support_count(minSup, transactionCount):
    """The reference's threshold rule (``cuApriori.py:452-456``)."""
    if isinstance(minSup, float) and 0 < minSup <= 1:
        return math.ceil(minSup * transactionCount)
    return int(minSup)


def clean_rows(rows):
    """Strip labels, drop in-basket repeats and empty baskets (``cuApriori.py:435-450``)."""
    out = []
    for row in rows:
        items = []
        for value in row:
            item = str(value).strip()
            if item and item not in items:
                items.append(item)
        if items:
            out.append(tuple(items))
    return out


def labels_and_columns(database):
    """Sorted string labels plus a CSR of column indices (``cuApriori.py:397-404``)."""
    labels = sorted({item for row in database for item in row})
    index = {label: i for i, label in enumerate(labels)}
    offsets = np.zeros(len(database) + 1, dtype=np.uint64)
    np.cumsum([len(r) for r in database], out=offsets[1:])
    cols = np.fromiter((index[i] for r in database for i in r), dtype=np.uint32,
                       count=int(offsets[-1]))
    return labels, offsets, cols


def numeric_columns(offsets, ids):
    """Label order for integer item ids: ``sorted(map(str, unique_ids))``.

    Returns ``(labels, cols)`` with ``cols`` the column of every occurrence.
    """
    uniq = np.unique(ids)
    strs = uniq.astype(str)
    order = np.argsort(strs, kind="stable")
    rank = np.empty(uniq.size, dtype=np.uint32)
    rank[order] = np.arange(uniq.size, dtype=np.uint32)
    cols = rank[np.searchsorted(uniq, ids)] if ids.size else np.zeros(0, np.uint32)
    return [str(s) for s in strs[order]], cols.astype(np.uint32)


def _run(fn_name, offsets, cols, n_items, minsup, threads):
    lib = _load()
    offsets = np.ascontiguousarray(offsets, dtype=np.uint64)
    cols = np.ascontiguousarray(cols, dtype=np.uint32)
    n_rows = offsets.size - 1
    ms = max(-(1 << 62), min(int(minsup), 1 << 62))
    handle = getattr(lib, fn_name)(n_rows, n_items, offsets.ctypes.data, cols.ctypes.data,
                                   ms, threads)
    if not handle:
        raise MemoryError("oracle allocation failed")
    try:
        n = lib.oracle_count(handle)
        slots = lib.oracle_item_slots(handle)
        po = np.zeros(n + 1, dtype=np.uint64)
        pi = np.zeros(max(1, slots), dtype=np.uint32)
        ps = np.zeros(max(1, n), dtype=np.uint64)
        lib.oracle_copy(handle, po.ctypes.data, pi.ctypes.data, ps.ctypes.data)
    finally:
        lib.oracle_free(handle)
    return po, pi[:slots], ps[:n]


def eclat_arrays(offsets, cols, n_items, minsup, threads=0):
    """Patterns as CSR arrays (offsets, column items, supports) in emission order."""
    return _run("oracle_eclat", offsets, cols, n_items, minsup, threads)


def apriori_arrays(offsets, cols, n_items, minsup, threads=0):
    return _run("oracle_apriori", offsets, cols, n_items, minsup, threads)


def to_dict(labels, arrays):
    po, pi, ps = arrays
    po = po.tolist()
    pi = pi.tolist()
    out = {}
    for k, s in enumerate(ps.tolist()):
        out["\t".join(labels[c] for c in pi[po[k]:po[k + 1]])] = int(s)
    return out


def mine_rows(rows, minSup, algorithm="eclat", threads=0):
    """``getPatterns()`` of the reference miner for an iterable of rows."""
    database = clean_rows(rows)
    labels, offsets, cols = labels_and_columns(database)
    minsup = support_count(minSup, len(database))
    fn = eclat_arrays if algorithm == "eclat" else apriori_arrays
    return to_dict(labels, fn(offsets, cols, len(labels), minsup, threads))


def mine_csr(offsets, ids, minSup, algorithm="eclat", threads=0):
    """Same for an integer CSR (offsets uint64[N+1], ids uint32[nnz])."""
    offsets = np.asarray(offsets, dtype=np.uint64)
    ids = np.asarray(ids, dtype=np.uint32)
    n = int(np.count_nonzero(offsets[1:] > offsets[:-1]))
    labels, cols = numeric_columns(offsets, ids)
    minsup = support_count(minSup, n)
    fn = eclat_arrays if algorithm == "eclat" else apriori_arrays
    return labels, fn(offsets, cols, len(labels), minsup, threads)
