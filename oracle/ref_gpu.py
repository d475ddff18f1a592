"""The reference's GPU path on this GPU -- TEST INFRASTRUCTURE ONLY.

cuPAMI runs its miners as Python drivers over CuPy arrays and three CUDA
kernels compiled from its own source (cupami/frequentPattern/_bitsets.py:19-125).
CuPy is not available here, so this module stands torch CUDA tensors in for
the CuPy arrays and calls the reference's kernels, compiled ahead of time from
that source by ``oracle/build_ref.py`` (``oracle/_ref/libref_bitsets.so``),
with the reference wrappers' launch shapes.  The drivers are the ones in
``oracle.numpy_port`` (the reference's driver loops restated), so the kernel
launches, their batching and every host/device synchronisation happen where
the reference has them:

  device pairs (BIN bulk path)   cupami/frequentPattern/cuApriori.py:381-394
  singletons, pair batches       cupami/frequentPattern/cuEclat.py:168-203
  class search                   cupami/frequentPattern/cuEclat.py:211-245
  Apriori levels                 cupami/frequentPattern/cuApriori.py:473-535
  periodic miners                cupami/periodicFrequentPattern/_temporal.py:150-171,
                                 cuPFEclat.py:146-175, cuPFApriori.py:141-157
                                 (drivers restated in ``oracle.periodic``)

Used by the benchmark's reference-GPU leg and by a parity test; the product
never imports it.
"""

from __future__ import annotations

import ctypes
import time
from pathlib import Path

from . import numpy_port

LIB = Path(__file__).resolve().parent / "_ref" / "libref_bitsets.so"
_lib = None


def available() -> bool:
    return LIB.exists()


def _load():
    global _lib
    if _lib is None:
        if not LIB.exists():
            raise FileNotFoundError(f"{LIB} is not built (python oracle/build_ref.py)")
        lib = ctypes.CDLL(str(LIB))
        u64, u32, p = ctypes.c_uint64, ctypes.c_uint32, ctypes.c_void_p
        lib.ref_build_bitsets.argtypes = [u64, p, p, u64, p, p]
        lib.ref_count_supports.argtypes = [p, u64, p, u32, u64, p, p]
        lib.ref_intersect_extensions.argtypes = [p, p, u64, u64, p, p, p]
        lib.ref_periodic_counts.argtypes = [p, u64, p, u32, u32, p, u64, ctypes.c_int64, p, p, p]
        for f in (lib.ref_build_bitsets, lib.ref_count_supports, lib.ref_intersect_extensions,
                  lib.ref_periodic_counts):
            f.restype = ctypes.c_int
        _lib = lib
    return _lib


class RefKernels:
    """The reference kernels and CuPy's array steps, on torch CUDA tensors (32-bit words as int32)."""

    def __init__(self, device=0, deadline=None):
        import torch

        self.torch = torch
        self.device = torch.device("cuda", device)
        self.lib = _load()
        self.deadline = deadline  # time.perf_counter() value after which kernel calls raise TimeoutError

    def _time_left(self):
        if self.deadline is not None and time.perf_counter() > self.deadline:
            raise TimeoutError("reference GPU path ran past its time budget")

    def _stream(self):
        return ctypes.c_void_p(self.torch.cuda.current_stream(self.device).cuda_stream)

    def _check(self, code, what):
        if code:
            raise RuntimeError(f"reference kernel {what} failed to launch (cudaError {code})")

    def pack(self, rows, cols, n_tx, n_items):
        t = self.torch
        words = (n_tx + 31) // 32
        bits = t.zeros((n_items, words), dtype=t.int32, device=self.device)
        if rows.numel():
            self._check(self.lib.ref_build_bitsets(rows.numel(), rows.data_ptr(), cols.data_ptr(), words,
                                                   bits.data_ptr(), self._stream()), "build_bitsets")
        return bits

    def supports(self, bits, candidates):
        t = self.torch
        self._time_left()
        if not len(candidates):
            return []
        idx = t.tensor(candidates, dtype=t.int32).to(self.device)
        sup = t.zeros(idx.shape[0], dtype=t.int64, device=self.device)
        self._check(self.lib.ref_count_supports(bits.data_ptr(), bits.shape[1], idx.data_ptr(), idx.shape[1],
                                                idx.shape[0], sup.data_ptr(), self._stream()), "count_supports")
        return sup.cpu().tolist()

    def intersect(self, prefix, ext):
        t = self.torch
        self._time_left()
        ext = ext.contiguous()
        prefix = prefix.contiguous()
        out = t.empty_like(ext)
        sup = t.zeros(ext.shape[0], dtype=t.int64, device=self.device)
        if ext.shape[0]:
            self._check(self.lib.ref_intersect_extensions(prefix.data_ptr(), ext.data_ptr(), ext.shape[1],
                                                          ext.shape[0], out.data_ptr(), sup.data_ptr(),
                                                          self._stream()), "intersect_extensions")
        return out, sup.cpu().tolist()

    def vertical(self, bits, members, left):
        t = self.torch
        return bits[t.tensor(members, dtype=t.int64).to(self.device)] & bits[left]

    def take(self, child, keep):
        t = self.torch
        return child[t.tensor(keep, dtype=t.int64).to(self.device)]

    def concat(self, chunks):
        return self.torch.cat(chunks)

    def sync(self):
        self.torch.cuda.synchronize(self.device)


def upload(offsets, ids, device=0):
    """The BIN loader's device copies (done at load time, outside mine())."""
    import torch

    dev = torch.device("cuda", device)
    off = torch.from_numpy(offsets.astype("int64", copy=False)).to(dev)
    it = torch.from_numpy(ids.astype("int64", copy=False)).to(dev)
    return off, it


def device_pairs(off, ids):
    """(labels, rows, columns, non-empty transactions) as the BIN bulk path builds them on the device."""
    import torch

    unique = torch.unique(ids)
    numeric = unique.cpu().tolist()
    labels = sorted(map(str, numeric))
    index = {label: i for i, label in enumerate(labels)}
    original = torch.searchsorted(off[1:], torch.arange(ids.numel(), dtype=torch.int64, device=ids.device),
                                  right=True)
    active = torch.cumsum((off[1:] > off[:-1]).to(torch.int64), 0) - 1
    rows = active[original]
    colmap = torch.tensor([index[str(v)] for v in numeric], dtype=torch.int32, device=ids.device)
    cols = colmap[torch.searchsorted(unique, ids)]
    n_tx = int((off[1:] > off[:-1]).sum().item())
    return labels, rows, cols, n_tx


def mine(off, ids, minsup_count, algorithm="eclat", kernels=None, out=None):
    """``{tuple(labels): support}`` from device CSR arrays, in the reference's insertion order.

    A float ``minsup_count`` in (0, 1] is a fraction of the non-empty
    transactions (the reference's threshold rule)."""
    k = kernels or RefKernels(ids.device.index or 0)
    labels, rows, cols, n_tx = device_pairs(off, ids)
    if isinstance(minsup_count, float):
        from . import support_count

        minsup_count = support_count(minsup_count, n_tx)
    fn = numpy_port.eclat if algorithm == "eclat" else numpy_port.apriori
    return fn(labels, rows, cols, n_tx, minsup_count, k, out)


def periodic_mine(transactions, timestamps, end, min_sup, max_per, algorithm="eclat", kernels=None):
    """The reference's periodic miners on this GPU: ``[(pattern, support, periodicity)]``.

    ``transactions`` are the cleaned baskets in timestamp order (empty ones
    included) and ``timestamps`` their timestamps; ``min_sup`` and ``max_per``
    are resolved thresholds.  As ``TemporalInput._prepare`` does
    (_temporal.py:150-157): (row, column) pairs built on the host
    (cuApriori.py:396-404), tidsets by the reference's build_bitsets, the
    timestamps uploaded; then the restated driver loop launches the reference's
    periodic_counts on every candidate batch with one upload of the candidates
    and one download of the results per batch, as ``_evaluate`` does (:159-165)."""
    import torch

    from . import periodic

    k = kernels or RefKernels()
    labels = sorted({item for row in transactions for item in row})
    index = {label: i for i, label in enumerate(labels)}
    rows, cols = [], []
    for r, basket in enumerate(transactions):
        rows.extend([r] * len(basket))
        cols.extend(index[item] for item in basket)
    d_rows = torch.tensor(rows, dtype=torch.int64).to(k.device)
    d_cols = torch.tensor(cols, dtype=torch.int32).to(k.device)
    n = len(transactions)
    bits = k.pack(d_rows, d_cols, n, len(labels))
    d_ts = torch.tensor(list(timestamps), dtype=torch.int64).to(k.device)

    def counts(cands):
        k._time_left()
        idx = torch.tensor(cands, dtype=torch.int64).to(torch.int32).to(k.device)
        m = idx.shape[0]
        sup = torch.empty(m, dtype=torch.int64, device=k.device)
        per = torch.empty(m, dtype=torch.int64, device=k.device)
        k._check(k.lib.ref_periodic_counts(bits.data_ptr(), bits.shape[1], idx.data_ptr(), idx.shape[1], m,
                                           d_ts.data_ptr() if n else None, n, int(end), sup.data_ptr(),
                                           per.data_ptr(), k._stream()), "periodic_counts")
        return list(zip(sup.cpu().tolist(), per.cpu().tolist()))

    fn = periodic.pf_eclat if algorithm == "eclat" else periodic.pf_apriori
    return fn(labels, None, None, end, min_sup, max_per, counts=counts)
