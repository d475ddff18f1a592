"""cpm_mine_eclat_noalloc against cpm_mine, through the C ABI.

Callers whose device memory belongs to another runtime's pool, or whose
process may not allocate once it has started, cannot let the library call
cudaMalloc.  cpm_mine_eclat_noalloc takes the tidsets and the output arrays
from the caller and keeps all of its scratch in a fixed static device array.
This test builds the tidsets and outputs itself, calls the entry point twice
in a row, and requires both results to equal cpm_mine's pattern for pattern
(bit-exact, like every other parity test here).  The file is named so that
pytest collects it last.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _database(seed=11, n=4000, n_items=22):
    rng = np.random.default_rng(seed)
    p = rng.uniform(0.15, 0.6, n_items)
    rows = []
    while len(rows) < n:
        row = np.nonzero(rng.random(n_items) < p)[0]
        if row.size:  # the entry point takes tidsets of non-empty rows only
            rows.append(row.astype(np.uint32))
    offsets = np.zeros(n + 1, dtype=np.uint64)
    np.cumsum([r.size for r in rows], out=offsets[1:])
    return offsets, np.concatenate(rows), n_items


def _pack(offsets, cols, n_items):
    n = offsets.size - 1
    stride = max(2, ((n + 63) // 64 + 1) & ~1)
    bits = np.zeros((n_items, stride), dtype=np.uint64)
    row = np.repeat(np.arange(n, dtype=np.uint64), np.diff(offsets.astype(np.int64)))
    np.bitwise_or.at(bits, (cols.astype(np.int64), (row // 64).astype(np.int64)),
                     np.left_shift(np.uint64(1), row % np.uint64(64)))
    return bits, stride


def test_noalloc_matches_cpm_mine_on_two_calls():
    import torch

    from cupami_b200 import _native

    offsets, cols, n_items = _database()
    n_tx = offsets.size - 1
    min_sup = int(0.04 * n_tx)
    ctx = _native.context(0)
    lib = _native.library()
    want = _native.Database.from_columns(ctx, offsets, cols, n_items).mine(
        min_sup, _native.CPM_ECLAT, order=_native.CPM_ORDER_ECLAT)
    assert len(want) > 1000

    bits, stride = _pack(offsets, cols, n_items)
    d_bits = torch.from_numpy(bits.view(np.int64)).cuda()
    capacity = len(want) + 16
    outs = [torch.empty(capacity, dtype=torch.int32, device="cuda") for _ in range(3)]
    for call in range(2):
        for t in outs:
            t.fill_(-7 - call)  # stale contents must not leak into the result
        torch.cuda.synchronize()
        count = ctypes.c_uint64()
        ctx.check(lib.cpm_mine_eclat_noalloc(
            ctx.handle, d_bits.data_ptr(), stride, n_items, n_tx, min_sup,
            outs[0].data_ptr(), outs[1].data_ptr(), outs[2].data_ptr(), capacity, ctypes.byref(count)))
        ctx.check(lib.cpm_synchronize(ctx.handle))
        n = count.value
        assert n == len(want)
        parent = outs[0][:n].cpu().numpy().view(np.uint32).astype(np.int64)
        parent[parent == 0xFFFFFFFF] = -1
        item = outs[1][:n].cpu().numpy().view(np.uint32)
        support = outs[2][:n].cpu().numpy().view(np.uint32).astype(np.uint64)
        got = _native.Result.from_tree(parent, item, support, _native.CPM_ORDER_ECLAT)
        assert np.array_equal(got.offsets, want.offsets), call
        assert np.array_equal(got.items, want.items), call
        assert np.array_equal(got.supports, want.supports), call


def test_noalloc_rejects_inputs_beyond_its_scratch():
    import torch

    from cupami_b200 import _native

    ctx = _native.context(0)
    lib = _native.library()
    # 5,000 items that all pass need a 100 MB pair matrix: more than the scratch.
    n_items, stride = 5000, 2
    d_bits = torch.full((n_items, stride), -1, dtype=torch.int64, device="cuda")
    outs = [torch.empty(n_items + 8, dtype=torch.int32, device="cuda") for _ in range(3)]
    count = ctypes.c_uint64()
    code = lib.cpm_mine_eclat_noalloc(ctx.handle, d_bits.data_ptr(), stride, n_items, 128, 1,
                                      outs[0].data_ptr(), outs[1].data_ptr(), outs[2].data_ptr(),
                                      n_items + 8, ctypes.byref(count))
    assert code == _native.CPM_EINVAL
    assert b"static scratch" in lib.cpm_last_error(ctx.handle)
    # The context stays usable after the rejection.
    ctx.check(lib.cpm_synchronize(ctx.handle))
