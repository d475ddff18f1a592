"""ctypes binding of ``libcupami_b200.so`` (the C ABI in include/cupami_b200.h).

The library is built in-tree next to this file by ``cupami_b200.build``.  There
is no fallback: if the library or a CUDA device is missing, the miners raise,
exactly as the reference raises when CuPy or a device is missing
(``cupami/frequentPattern/cuApriori.py:458-471``).
"""

from __future__ import annotations

import atexit
import ctypes
import threading
import weakref
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libcupami_b200.so"

CPM_OK = 0
CPM_EINVAL = -1
CPM_ENOMEM = -2
CPM_ECUDA = -3
CPM_EOVERFLOW = -4
CPM_ETIMEOUT = -5
CPM_ENODEV = -6
CPM_EINTERNAL = -7

CPM_ECLAT = 0
CPM_APRIORI = 1
CPM_ORDER_ECLAT = 0
CPM_ORDER_APRIORI = 1
CPM_ORDER_NONE = 2
CPM_ORDER_DEPTH_FIRST = 3
CPM_SCHED_PLAIN = 0
CPM_SCHED_LEARNED = 1

_ERRORS = {
    CPM_EINVAL: "invalid argument", CPM_ENOMEM: "out of memory", CPM_ECUDA: "CUDA error",
    CPM_EOVERFLOW: "buffer overflow", CPM_ETIMEOUT: "device wait ran out", CPM_ENODEV: "no CUDA device",
    CPM_EINTERNAL: "internal error",
}


class NativeError(RuntimeError):
    """A C-ABI call returned a negative status."""

    def __init__(self, code, message):
        super().__init__(f"{_ERRORS.get(code, 'error')} ({code}): {message}")
        self.code = code


class Opts(ctypes.Structure):
    _fields_ = [
        ("scheduler", ctypes.c_int32), ("pair_engine", ctypes.c_int32),
        ("pair_batch", ctypes.c_uint64), ("intersection_bytes", ctypes.c_uint64),
        ("arena_bytes", ctypes.c_uint64), ("spin_limit", ctypes.c_uint64),
        ("collect_trace", ctypes.c_int32), ("deep_block", ctypes.c_int32),
        ("deep_ctas_per_sm", ctypes.c_int32), ("autotune", ctypes.c_int32), ("tidsets", ctypes.c_int32),
        ("list_div", ctypes.c_int32), ("deep_balance", ctypes.c_int32), ("deep_project", ctypes.c_int32),
        ("deep_rows", ctypes.c_int32),
    ]


class Stats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint64) for n in (
        "n_patterns", "n_frequent_items", "n_frequent_pairs", "frames", "work_items",
        "intersections", "bytes_alg", "pair_ops", "kernel_launches", "retries", "deep_rounds")] + [
        (n, ctypes.c_double) for n in (
            "ms_pack", "ms_pairs", "ms_deep", "ms_total", "deep_gbs", "pair_tops")] + [
        ("projected_units", ctypes.c_uint64), ("ms_local", ctypes.c_double), ("row_units", ctypes.c_uint64)]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


_P = ctypes.c_void_p
_U64 = ctypes.c_uint64
_SIGNATURES = {
    "cpm_init": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(_P)]),
    "cpm_shutdown": (None, [_P]),
    "cpm_last_error": (ctypes.c_char_p, [_P]),
    "cpm_version": (ctypes.c_char_p, []),
    "cpm_default_opts": (ctypes.c_int, [ctypes.POINTER(Opts)]),
    "cpm_db_from_csr": (ctypes.c_int, [_P, _P, _U64, _P, _U64, ctypes.c_uint32, ctypes.POINTER(_P)]),
    "cpm_db_from_ids": (ctypes.c_int, [_P, _P, _U64, _P, _U64, ctypes.POINTER(_P)]),
    "cpm_db_from_ids_batch": (ctypes.c_int, [_P, ctypes.c_uint32, ctypes.POINTER(_P), ctypes.POINTER(_U64),
                                             ctypes.POINTER(_P), ctypes.POINTER(_U64), ctypes.POINTER(_P)]),
    "cpm_autotune": (ctypes.c_int, [_P, _P, ctypes.c_int64, ctypes.POINTER(Opts), ctypes.POINTER(ctypes.c_int32),
                                    ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_int32),
                                    ctypes.POINTER(ctypes.c_double)]),
    "cpm_db_info": (ctypes.c_int, [_P, ctypes.POINTER(_U64), ctypes.POINTER(ctypes.c_uint32),
                                   ctypes.POINTER(_U64)]),
    "cpm_db_labels": (ctypes.c_int, [_P, _P]),
    "cpm_db_free": (None, [_P]),
    "cpm_mine": (ctypes.c_int, [_P, _P, ctypes.c_int64, ctypes.c_int, ctypes.POINTER(Opts),
                                ctypes.POINTER(_P)]),
    "cpm_mine_batch": (ctypes.c_int, [_P, ctypes.POINTER(_P), ctypes.c_uint32, ctypes.POINTER(ctypes.c_int64),
                                      ctypes.POINTER(Opts), ctypes.POINTER(_P)]),
    "cpm_result_size": (ctypes.c_int, [_P, ctypes.POINTER(_U64), ctypes.POINTER(_U64)]),
    "cpm_result_copy": (ctypes.c_int, [_P, ctypes.c_int, _P, _P, _P]),
    "cpm_result_tree": (ctypes.c_int, [_P, _P, _P, _P]),
    "cpm_results_copy": (ctypes.c_int, [ctypes.POINTER(_P), ctypes.c_uint32, ctypes.c_int, _P, _P, _P, _P]),
    "cpm_result_stats": (ctypes.c_int, [_P, ctypes.POINTER(Stats)]),
    "cpm_result_from_tree": (ctypes.c_int, [_P, _P, _P, _U64, ctypes.POINTER(_P)]),
    "cpm_result_free": (None, [_P]),
    "cpm_build_bitsets": (ctypes.c_int, [_P, _P, _P, _U64, _U64, ctypes.c_uint32, _P]),
    "cpm_count_supports": (ctypes.c_int, [_P, _P, _U64, _P, _U64, ctypes.c_uint32, _P]),
    "cpm_intersect_extensions": (ctypes.c_int, [_P, _P, _P, _U64, _U64, _P, _P]),
    "cpm_synchronize": (ctypes.c_int, [_P]),
    "cpm_stream": (ctypes.c_void_p, [_P]),
    "cpm_costmodel_params": (ctypes.c_int, [ctypes.POINTER(ctypes.c_uint32), ctypes.POINTER(ctypes.c_uint32)]),
    "cpm_costmodel_train": (ctypes.c_int, [_P, _P, _P, _U64, ctypes.c_uint32, ctypes.c_float, _U64, _P, _P]),
    "cpm_costmodel_predict": (ctypes.c_int, [_P, _P, _P, _U64, _P]),
    "cpm_costmodel_gradient": (ctypes.c_int, [_P, _P, _P, _P, _U64, _P, _P]),
    "cpm_costmodel_set": (ctypes.c_int, [_P, _P]),
    "cpm_result_trace": (ctypes.c_int, [_P, _P, _P, ctypes.POINTER(_U64)]),
    "cpm_tdb_from_csr": (ctypes.c_int, [_P, _P, _U64, _P, _U64, ctypes.c_uint32, _P, ctypes.c_int64,
                                        ctypes.POINTER(_P)]),
    "cpm_mine_periodic": (ctypes.c_int, [_P, _P, ctypes.c_int64, ctypes.c_int64, ctypes.c_int, ctypes.POINTER(_P)]),
    "cpm_result_copy_periodic": (ctypes.c_int, [_P, ctypes.c_int, _P, _P, _P, _P]),
    "cpm_result_from_tree_periodic": (ctypes.c_int, [_P, _P, _P, _P, _U64, ctypes.POINTER(_P)]),
    "cpm_periodic_counts": (ctypes.c_int, [_P, _P, _U64, _P, _U64, ctypes.c_uint32, _P, _U64, ctypes.c_int64,
                                           _P, _P]),
    "cpm_join_labels": (ctypes.c_int, [_P, _P, _U64, _P, _P, ctypes.c_uint32, ctypes.c_char, ctypes.c_char, _P,
                                       _U64, ctypes.POINTER(_U64)]),
    "cpm_parse_int_text": (ctypes.c_int, [_P, _P, _U64, ctypes.c_int32, ctypes.POINTER(_P)]),
    "cpm_csr_size": (ctypes.c_int, [_P, ctypes.POINTER(_U64), ctypes.POINTER(_U64)]),
    "cpm_csr_copy": (ctypes.c_int, [_P, _P, _P]),
    "cpm_csr_free": (None, [_P]),
    "cpm_mine_eclat_noalloc": (ctypes.c_int, [_P, _P, _U64, ctypes.c_uint32, _U64, ctypes.c_int64,
                                              ctypes.POINTER(Opts), _P, _P, _P, _U64, ctypes.POINTER(_U64)]),
}

_lib = None
_lock = threading.RLock()
_contexts: dict[int, "Context"] = {}


def library():
    """Load the shared library (raises ImportError when it has not been built)."""
    global _lib
    if _lib is None:
        with _lock:
            if _lib is None:
                if not LIB_PATH.exists():
                    raise ImportError(
                        f"{LIB_PATH.name} is not built; run cupami_b200.build.build() "
                        "(nvcc for sm_100a) before mining")
                lib = ctypes.CDLL(str(LIB_PATH))
                for name, (res, args) in _SIGNATURES.items():
                    fn = getattr(lib, name)
                    fn.restype = res
                    fn.argtypes = args
                _lib = lib
    return _lib


def declared_symbols():
    return list(_SIGNATURES)


class Context:
    """One cpm_ctx (device + stream).  Calls on a context must not overlap."""

    def __init__(self, device=0):
        lib = library()
        handle = _P()
        code = lib.cpm_init(int(device), ctypes.byref(handle))
        if code == CPM_ENODEV:
            raise RuntimeError("GPU mining requires a CUDA device; no CUDA device was found.")
        if code != CPM_OK:
            raise RuntimeError(f"could not initialise CUDA device {device} (status {code})")
        self.handle = handle
        self.device = device
        self.lock = threading.Lock()
        self.databases = weakref.WeakSet()  # freed before the context (they point to it)

    def check(self, code):
        if code != CPM_OK:
            msg = library().cpm_last_error(self.handle)
            raise NativeError(code, msg.decode() if msg else "")

    def stream(self):
        """The library's CUDA stream on this context, as an integer handle."""
        return int(library().cpm_stream(self.handle) or 0)

    def close(self):
        if self.handle:
            for db in list(self.databases):
                db.close()
            library().cpm_shutdown(self.handle)
            self.handle = None


def context(device=0) -> Context:
    library()
    ctx = _contexts.get(device)
    if ctx is None:
        with _lock:
            ctx = _contexts.get(device)
            if ctx is None:
                ctx = Context(device)
                _contexts[device] = ctx
    return ctx


@atexit.register
def _shutdown():
    for ctx in list(_contexts.values()):
        try:
            ctx.close()
        except Exception:  # interpreter teardown
            pass
    _contexts.clear()


def _ptr(a):
    return a.ctypes.data if a.size else None


class Database:
    """Device tidsets of one transaction database (owned by the library)."""

    def __init__(self, ctx: Context, handle, labels=None):
        self.ctx = ctx
        self.handle = handle
        ctx.databases.add(self)
        n_tx, n_items, words = _U64(), ctypes.c_uint32(), _U64()
        ctx.check(library().cpm_db_info(handle, ctypes.byref(n_tx), ctypes.byref(n_items),
                                        ctypes.byref(words)))
        self.n_transactions = n_tx.value
        self.n_items = n_items.value
        self.words = words.value
        self.labels = labels

    @classmethod
    def from_columns(cls, ctx, offsets, cols, n_items):
        offsets = np.ascontiguousarray(offsets, dtype=np.uint64)
        cols = np.ascontiguousarray(cols, dtype=np.uint32)
        handle = _P()
        with ctx.lock:
            ctx.check(library().cpm_db_from_csr(ctx.handle, _ptr(offsets), offsets.size - 1,
                                                _ptr(cols), cols.size, int(n_items),
                                                ctypes.byref(handle)))
        return cls(ctx, handle)

    @classmethod
    def from_ids(cls, ctx, offsets, ids):
        offsets = np.ascontiguousarray(offsets, dtype=np.uint64)
        ids = np.ascontiguousarray(ids, dtype=np.uint32)
        handle = _P()
        with ctx.lock:
            ctx.check(library().cpm_db_from_ids(ctx.handle, _ptr(offsets), offsets.size - 1,
                                                _ptr(ids), ids.size, ctypes.byref(handle)))
        db = cls(ctx, handle)
        labels = np.zeros(db.n_items, dtype=np.uint32)
        if db.n_items:
            ctx.check(library().cpm_db_labels(handle, labels.ctypes.data))
        db.labels = labels
        return db

    @classmethod
    def from_ids_batch(cls, ctx, sources):
        """One Database per (offsets, ids) pair, loaded with one upload and one packing pass."""
        n = len(sources)
        offs = [np.ascontiguousarray(o, dtype=np.uint64) for o, _ in sources]
        idss = [np.ascontiguousarray(i, dtype=np.uint32) for _, i in sources]
        n_rows = (_U64 * max(1, n))(*[o.size - 1 for o in offs])
        nnz = (_U64 * max(1, n))(*[i.size for i in idss])
        p_off = (_P * max(1, n))(*[o.ctypes.data for o in offs])
        p_ids = (_P * max(1, n))(*[i.ctypes.data for i in idss])
        outs = (_P * max(1, n))()
        with ctx.lock:
            ctx.check(library().cpm_db_from_ids_batch(ctx.handle, n, p_off, n_rows, p_ids, nnz, outs))
        dbs = []
        for k in range(n):
            db = cls(ctx, _P(outs[k]))
            labels = np.zeros(db.n_items, dtype=np.uint32)
            if db.n_items:
                ctx.check(library().cpm_db_labels(db.handle, labels.ctypes.data))
            db.labels = labels
            dbs.append(db)
        return dbs

    @classmethod
    def from_temporal(cls, ctx, offsets, cols, n_items, timestamps, end):
        """Temporal tidsets: every row kept (empty ones too), rows sorted by timestamp."""
        offsets = np.ascontiguousarray(offsets, dtype=np.uint64)
        cols = np.ascontiguousarray(cols, dtype=np.uint32)
        timestamps = np.ascontiguousarray(timestamps, dtype=np.int64)
        handle = _P()
        with ctx.lock:
            ctx.check(library().cpm_tdb_from_csr(ctx.handle, _ptr(offsets), offsets.size - 1, _ptr(cols),
                                                 cols.size, int(n_items), _ptr(timestamps), int(end),
                                                 ctypes.byref(handle)))
        return cls(ctx, handle)

    def mine_periodic(self, min_sup, max_per, algorithm, order):
        """Periodic-frequent itemsets of a temporal database (Result with ``periods``)."""
        res = _P()
        with self.ctx.lock:
            self.ctx.check(library().cpm_mine_periodic(self.ctx.handle, self.handle, int(min_sup), int(max_per),
                                                       int(algorithm), ctypes.byref(res)))
        try:
            return Result.collect(res, order, periodic=True)
        finally:
            library().cpm_result_free(res)

    def mine(self, min_sup, algorithm, opts=None, order=None):
        if opts is None:
            opts = Opts()
            library().cpm_default_opts(ctypes.byref(opts))
        res = _P()
        with self.ctx.lock:
            self.ctx.check(library().cpm_mine(self.ctx.handle, self.handle, int(min_sup),
                                              int(algorithm), ctypes.byref(opts), ctypes.byref(res)))
        try:
            return Result.collect(res, CPM_ORDER_ECLAT if order is None else order)
        finally:
            library().cpm_result_free(res)

    def close(self):
        # A database outliving its context (interpreter teardown) was freed with it.
        if self.handle and self.ctx.handle:
            library().cpm_db_free(self.handle)
        self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def join_labels(offsets, items, labels, sep="\t"):
    """Keys of a pattern CSR: every pattern's labels joined by ``sep`` (a list
    of str), built in one C pass over the arrays."""
    lib = library()
    offsets = np.ascontiguousarray(offsets, dtype=np.uint64)
    items = np.ascontiguousarray(items, dtype=np.uint32)
    n = offsets.size - 1
    if n <= 0:
        return []
    enc = [str(x).encode("utf-8") for x in labels]
    blob = b"".join(enc)
    loff = np.zeros(len(enc) + 1, dtype=np.uint64)
    np.cumsum([len(e) for e in enc], out=loff[1:])
    src = np.frombuffer(blob, dtype=np.uint8) if blob else np.zeros(1, np.uint8)
    need = _U64()
    args = (offsets.ctypes.data, items.ctypes.data if items.size else None, n, src.ctypes.data, loff.ctypes.data,
            len(enc), sep.encode(), b"\n")
    if lib.cpm_join_labels(*args, None, 0, ctypes.byref(need)) != CPM_OK:
        raise NativeError(CPM_EINVAL, "pattern items outside the labels")
    out = bytearray(need.value)
    buf = (ctypes.c_char * len(out)).from_buffer(out)
    if lib.cpm_join_labels(*args, buf, len(out), ctypes.byref(need)) != CPM_OK:
        raise NativeError(CPM_EINVAL, "pattern items outside the labels")
    keys = out.decode("utf-8").split("\n")
    keys.pop()  # after the last end mark
    return keys


def parse_int_text(ctx, data: bytes, sep: str):
    """(offsets uint64[n+1], ids uint32[nnz]) of delimited integer baskets,
    parsed on the device; raises NativeError (CPM_EINVAL) for any other layout."""
    lib = library()
    buf = np.frombuffer(data, dtype=np.uint8)
    handle = _P()
    with ctx.lock:
        ctx.check(lib.cpm_parse_int_text(ctx.handle, buf.ctypes.data if buf.size else None, buf.size,
                                         ord(sep), ctypes.byref(handle)))
    try:
        n, nnz = _U64(), _U64()
        lib.cpm_csr_size(handle, ctypes.byref(n), ctypes.byref(nnz))
        offsets = np.zeros(n.value + 1, dtype=np.uint64)
        ids = np.zeros(max(1, nnz.value), dtype=np.uint32)
        ctx.check(lib.cpm_csr_copy(handle, offsets.ctypes.data, ids.ctypes.data))
        return offsets, ids[:nnz.value]
    finally:
        lib.cpm_csr_free(handle)


def autotune(ctx, db, min_sup, opts=None):
    """cpm_autotune: fastest deep-level launch shape for this database, recorded in ctx."""
    if opts is None:
        opts = Opts()
        library().cpm_default_opts(ctypes.byref(opts))
    block, ctas, div, ms = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32(), ctypes.c_double()
    with ctx.lock:
        ctx.check(library().cpm_autotune(ctx.handle, db.handle, int(min_sup), ctypes.byref(opts),
                                         ctypes.byref(block), ctypes.byref(ctas), ctypes.byref(div),
                                         ctypes.byref(ms)))
    return {"block": block.value, "ctas_per_sm": ctas.value, "list_div": div.value, "ms_deep": ms.value}


def mine_batch(ctx, databases, min_sups, opts=None, order=CPM_ORDER_ECLAT):
    """Eclat over a list of Database objects in one pass; one Result each."""
    n = len(databases)
    if opts is None:
        opts = Opts()
        library().cpm_default_opts(ctypes.byref(opts))
    handles = (_P * max(1, n))(*[db.handle for db in databases])
    sups = (ctypes.c_int64 * max(1, n))(*[int(s) for s in min_sups])
    outs = (_P * max(1, n))()
    with ctx.lock:
        ctx.check(library().cpm_mine_batch(ctx.handle, handles, n, sups, ctypes.byref(opts), outs))
    try:
        lib = library()
        sizes = np.zeros(2 * max(1, n), dtype=np.uint64)
        if lib.cpm_results_copy(outs, n, int(order), sizes.ctypes.data, None, None, None) != CPM_OK:
            raise NativeError(CPM_EINTERNAL, "result sizes")
        npat = sizes[0::2][:n].astype(np.int64)
        nslot = sizes[1::2][:n].astype(np.int64)
        offsets = np.zeros(max(1, int(npat.sum() + n)), dtype=np.uint64)
        items = np.zeros(max(1, int(nslot.sum())), dtype=np.uint32)
        supports = np.zeros(max(1, int(npat.sum())), dtype=np.uint64)
        code = lib.cpm_results_copy(outs, n, int(order), sizes.ctypes.data, offsets.ctypes.data,
                                    items.ctypes.data, supports.ctypes.data)
        if code != CPM_OK:
            raise NativeError(code, "result copy")
        st = Stats()
        lib.cpm_result_stats(outs[0], ctypes.byref(st))
        stats = st.as_dict()
        results, o, it, sp = [], 0, 0, 0
        for k in range(n):
            results.append(Result(offsets[o:o + npat[k] + 1], items[it:it + nslot[k]], supports[sp:sp + npat[k]],
                                  stats))
            o += npat[k] + 1
            it += nslot[k]
            sp += npat[k]
    finally:
        for k in range(n):
            if outs[k]:
                library().cpm_result_free(outs[k])
    return results


class Result:
    """Mined patterns as arrays: pattern k = items[offsets[k]:offsets[k+1]]."""

    def __init__(self, offsets, items, supports, stats):
        self.offsets = offsets
        self.items = items
        self.supports = supports
        self.stats = stats
        self.trace = None  # (features, log1p(subtree intersections)) per root unit, when traced
        self.periods = None  # int64 periodicity per pattern (periodic results)

    @classmethod
    def collect(cls, handle, order, periodic=False):
        lib = library()
        n, slots = _U64(), _U64()
        if lib.cpm_result_size(handle, ctypes.byref(n), ctypes.byref(slots)) != CPM_OK:
            raise NativeError(CPM_EINTERNAL, "result size")
        offsets = np.zeros(n.value + 1, dtype=np.uint64)
        items = np.zeros(max(1, slots.value), dtype=np.uint32)
        supports = np.zeros(max(1, n.value), dtype=np.uint64)
        periods = np.zeros(max(1, n.value), dtype=np.int64) if periodic else None
        if periodic:
            code = lib.cpm_result_copy_periodic(handle, int(order), offsets.ctypes.data, items.ctypes.data,
                                                supports.ctypes.data, periods.ctypes.data)
        else:
            code = lib.cpm_result_copy(handle, int(order), offsets.ctypes.data, items.ctypes.data,
                                       supports.ctypes.data)
        if code != CPM_OK:
            raise NativeError(code, "result copy")
        st = Stats()
        lib.cpm_result_stats(handle, ctypes.byref(st))
        out = cls(offsets, items[:slots.value], supports[:n.value], st.as_dict())
        if periodic:
            out.periods = periods[:n.value]
        nt = _U64()
        lib.cpm_result_trace(handle, None, None, ctypes.byref(nt))
        if nt.value:
            nf = ctypes.c_uint32()
            lib.cpm_costmodel_params(ctypes.byref(nf), None)
            X = np.zeros((nt.value, nf.value), dtype=np.float32)
            y = np.zeros(nt.value, dtype=np.float32)
            lib.cpm_result_trace(handle, X.ctypes.data, y.ctypes.data, ctypes.byref(nt))
            out.trace = (X, y)
        return out

    def __len__(self):
        return int(self.supports.size)

    def patterns(self, labels):
        """{tab-joined labels: support}, in result order."""
        names = [str(v) for v in (labels.tolist() if hasattr(labels, "tolist") else labels)]
        off, items = self.offsets.tolist(), self.items.tolist()
        return {"\t".join(names[c] for c in items[off[k]:off[k + 1]]): int(s)
                for k, s in enumerate(self.supports.tolist())}

    @classmethod
    def from_tree(cls, parent, item, support, order, period=None):
        """Order a host pattern tree (no device work); with ``period`` a periodic result."""
        parent = np.ascontiguousarray(parent, dtype=np.int64)
        item = np.ascontiguousarray(item, dtype=np.uint32)
        support = np.ascontiguousarray(support, dtype=np.uint64)
        handle = _P()
        if period is None:
            code = library().cpm_result_from_tree(_ptr(parent), _ptr(item), _ptr(support), parent.size,
                                                  ctypes.byref(handle))
        else:
            period = np.ascontiguousarray(period, dtype=np.int64)
            code = library().cpm_result_from_tree_periodic(_ptr(parent), _ptr(item), _ptr(support), _ptr(period),
                                                           parent.size, ctypes.byref(handle))
        if code != CPM_OK:
            raise NativeError(code, "invalid pattern tree")
        try:
            return cls.collect(handle, order, periodic=period is not None)
        finally:
            library().cpm_result_free(handle)
