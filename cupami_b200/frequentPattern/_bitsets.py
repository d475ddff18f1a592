"""Drop-in for cuPAMI's kernel module ``cupami/frequentPattern/_bitsets.py``.

The three functions keep the reference's signatures and 32-bit word layout
(``_bitsets.py:91-125``): ``bitsets[item][word]``, bit ``row % 32`` of word
``row // 32``.  Device arrays are torch CUDA tensors (32-bit words stored as
``torch.int32``, 64-bit counts as ``torch.int64``); the arithmetic runs in
``libcupami_b200.so`` through ``cpm_build_bitsets``, ``cpm_count_supports``
and ``cpm_intersect_extensions``.  The first argument (the reference's CuPy
module) is accepted for compatibility and may be the namespace returned by
:func:`array_module`.
"""

from __future__ import annotations

import numpy as np

from .. import _native

__all__ = ["array_module", "build_bitsets", "count_supports", "intersect_extensions", "synchronize"]


def _torch():
    import torch

    if not torch.cuda.is_available():
        raise RuntimeError("GPU mining requires a CUDA device; no CUDA device was found.")
    return torch


class _ArrayModule:
    """The small part of an array module that the search hooks use."""

    def __init__(self):
        torch = _torch()
        self._torch = torch
        self.int64 = torch.int64
        self.uint64 = "uint64"
        self.uint32 = "uint32"
        self.int32 = torch.int32

    def asarray(self, values, dtype=None):
        torch = self._torch
        if dtype == "uint64":
            a = np.ascontiguousarray(np.asarray(values, dtype=np.uint64)).view(np.int64)
            return torch.from_numpy(a.copy()).cuda()
        if dtype == "uint32":
            a = np.ascontiguousarray(np.asarray(values, dtype=np.uint32)).view(np.int32)
            return torch.from_numpy(a.copy()).cuda()
        if isinstance(values, torch.Tensor):
            return values.to(device="cuda", dtype=dtype) if dtype is not None else values.cuda()
        return torch.as_tensor(np.asarray(values), dtype=dtype, device="cuda")

    def concatenate(self, arrays):
        return self._torch.cat(list(arrays))


_xp = None


def array_module():
    global _xp
    if _xp is None:
        _xp = _ArrayModule()
    return _xp


def _ctx(tensor):
    torch = _torch()
    torch.cuda.current_stream(tensor.device).synchronize()
    return _native.context(tensor.device.index or 0)


def synchronize():
    torch = _torch()
    torch.cuda.synchronize()


def build_bitsets(cp, rows, columns, transactions, items):
    """uint32[items][ceil(transactions / 32)] tidsets (reference _bitsets.py:91-100)."""
    torch = _torch()
    words = (int(transactions) + 31) // 32
    bitsets = torch.zeros((int(items), words), dtype=torch.int32, device="cuda")
    ctx = _ctx(bitsets)
    rows = rows.contiguous()
    columns = columns.contiguous()
    with ctx.lock:
        ctx.check(_native.library().cpm_build_bitsets(
            ctx.handle, rows.data_ptr() if rows.numel() else None,
            columns.data_ptr() if columns.numel() else None, rows.numel(), int(transactions),
            int(items), bitsets.data_ptr() if bitsets.numel() else None))
        ctx.check(_native.library().cpm_synchronize(ctx.handle))
    return bitsets


def count_supports(cp, bitsets, candidates):
    """Support of each candidate row list (reference _bitsets.py:103-113)."""
    torch = _torch()
    if not len(candidates):
        return []
    cand = np.ascontiguousarray(np.asarray(candidates, dtype=np.uint32)).view(np.int32)
    width = cand.shape[1]
    d_cand = torch.from_numpy(cand.copy()).cuda()
    supports = torch.zeros(cand.shape[0], dtype=torch.int64, device="cuda")
    bitsets = bitsets.contiguous()
    ctx = _ctx(bitsets)
    with ctx.lock:
        ctx.check(_native.library().cpm_count_supports(
            ctx.handle, bitsets.data_ptr() if bitsets.numel() else None, int(bitsets.shape[1]),
            d_cand.data_ptr(), cand.shape[0], width, supports.data_ptr()))
        ctx.check(_native.library().cpm_synchronize(ctx.handle))
    return supports.cpu().tolist()


def intersect_extensions(cp, prefix, extensions):
    """Children ``prefix & extensions[e]`` and their supports (reference _bitsets.py:116-125)."""
    torch = _torch()
    extensions = extensions.contiguous()
    prefix = prefix.contiguous()
    out = torch.empty_like(extensions)
    supports = torch.zeros(len(extensions), dtype=torch.int64, device="cuda")
    if len(extensions):
        ctx = _ctx(extensions)
        with ctx.lock:
            ctx.check(_native.library().cpm_intersect_extensions(
                ctx.handle, prefix.data_ptr(), extensions.data_ptr(), int(extensions.shape[1]),
                len(extensions), out.data_ptr(), supports.data_ptr()))
            ctx.check(_native.library().cpm_synchronize(ctx.handle))
    return out, supports.cpu().tolist()
