"""cpm_mine_eclat_noalloc against cpm_mine, through the C ABI.

Callers whose device memory belongs to another runtime's pool, or whose
process may not allocate once it has started, cannot let the library call
cudaMalloc.  cpm_mine_eclat_noalloc takes the tidsets and the output arrays
from the caller and keeps all of its scratch in a fixed static device array.
This test builds the tidsets and outputs itself, calls the entry point twice
in a row, and requires both results to equal cpm_mine's pattern for pattern
(bit-exact, like every other parity test here).  Around the second call it
reads the device's stream-ordered pool watermarks and free memory: the one
promise of the entry point is that it allocates nothing.  The file is named so
that pytest collects it last.
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


def _pool_usage(device=0):
    """(used high, reserved high, used now, free bytes) of the device's default
    stream-ordered pool, with both watermarks first reset to the current use."""
    from cuda.bindings import driver as dr
    from cuda.bindings import runtime as rt

    err, pool = rt.cudaDeviceGetDefaultMemPool(device)
    assert err == rt.cudaError_t.cudaSuccess
    A = rt.cudaMemPoolAttr

    def get(attr):
        e, v = rt.cudaMemPoolGetAttribute(pool, attr)
        assert e == rt.cudaError_t.cudaSuccess
        return int(v)

    def reset():
        for attr in (A.cudaMemPoolAttrUsedMemHigh, A.cudaMemPoolAttrReservedMemHigh):
            (e,) = rt.cudaMemPoolSetAttribute(pool, attr, dr.cuuint64_t(0))
            assert e == rt.cudaError_t.cudaSuccess

    def read():
        e, free, _ = rt.cudaMemGetInfo()
        assert e == rt.cudaError_t.cudaSuccess
        return (get(A.cudaMemPoolAttrUsedMemHigh), get(A.cudaMemPoolAttrReservedMemHigh),
                get(A.cudaMemPoolAttrUsedMemCurrent), int(free))

    return reset, read


def _call(lib, ctx, d_bits, stride, n_items, n_tx, min_sup, outs, capacity, opts=None):
    import ctypes as ct

    count = ct.c_uint64()
    code = lib.cpm_mine_eclat_noalloc(ctx.handle, d_bits.data_ptr(), stride, n_items, n_tx, min_sup,
                                      ct.byref(opts) if opts is not None else None,
                                      outs[0].data_ptr(), outs[1].data_ptr(), outs[2].data_ptr(), capacity,
                                      ct.byref(count))
    return code, count.value


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
    reset, read = _pool_usage()
    for call in range(2):
        for t in outs:
            t.fill_(-7 - call)  # stale contents must not leak into the result
        torch.cuda.synchronize()
        reset()
        before = read()
        code, n = _call(lib, ctx, d_bits, stride, n_items, n_tx, min_sup, outs, capacity)
        ctx.check(code)
        ctx.check(lib.cpm_synchronize(ctx.handle))
        if call == 1:
            # Nothing was taken from the pool (watermarks unchanged) and no
            # device memory is held afterwards (free bytes unchanged).
            assert read() == before
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
    code, _ = _call(lib, ctx, d_bits, stride, n_items, 128, 1, outs, n_items + 8)
    assert code == _native.CPM_EINVAL
    assert b"static scratch" in lib.cpm_last_error(ctx.handle)
    # The context stays usable after the rejection.
    ctx.check(lib.cpm_synchronize(ctx.handle))


def test_noalloc_empty_database_and_spin_limit():
    import torch

    from cupami_b200 import _native

    ctx = _native.context(0)
    lib = _native.library()
    outs = [torch.empty(8, dtype=torch.int32, device="cuda") for _ in range(3)]
    empty = torch.empty(0, dtype=torch.int64, device="cuda")
    # No items: no patterns and no error, whatever the stride.
    code, n = _call(lib, ctx, empty, 0, 0, 0, 1, outs, 8)
    assert (code, n) == (_native.CPM_OK, 0)
    # The caller's spin limit bounds the deep-level queue wait: one spin runs out.
    offsets, cols, n_items = _database(seed=5, n=3000, n_items=18)
    bits, stride = _pack(offsets, cols, n_items)
    d_bits = torch.from_numpy(bits.view(np.int64)).cuda()
    big = [torch.empty(1 << 16, dtype=torch.int32, device="cuda") for _ in range(3)]
    opts = _native.Opts()
    lib.cpm_default_opts(ctypes.byref(opts))
    opts.spin_limit = 1
    code, _ = _call(lib, ctx, d_bits, stride, n_items, offsets.size - 1, 150, big, 1 << 16, opts)
    assert code == _native.CPM_ETIMEOUT
    assert b"limit 1" in lib.cpm_last_error(ctx.handle)
    opts.spin_limit = 0  # the default limit: the same call completes
    code, n = _call(lib, ctx, d_bits, stride, n_items, offsets.size - 1, 150, big, 1 << 16, opts)
    ctx.check(code)
    assert n > 100


def test_cpm_mine_after_noalloc_keeps_large_prefixes():
    """A no-alloc call on short tidsets leaves the deep kernel able to stage
    prefixes above 48 KB of shared memory in a later cpm_mine."""
    import torch

    import oracle
    from cupami_b200 import _native

    ctx = _native.context(0)
    lib = _native.library()
    offsets, cols, n_items = _database(seed=3, n=600, n_items=14)
    bits, stride = _pack(offsets, cols, n_items)
    d_bits = torch.from_numpy(bits.view(np.int64)).cuda()
    outs = [torch.empty(1 << 16, dtype=torch.int32, device="cuda") for _ in range(3)]
    code, n = _call(lib, ctx, d_bits, stride, n_items, offsets.size - 1, 30, outs, 1 << 16)
    ctx.check(code)
    assert n > 100
    # 420,000 transactions: 6,564-word (51 KB) tidsets, so the deep kernel's
    # prefix needs more than the default 48 KB of dynamic shared memory.
    rng = np.random.default_rng(8)
    n_tx, k = 420_000, 10
    take = rng.random((n_tx, k)) < np.linspace(0.85, 0.4, k)
    take[:, 0] |= ~take.any(axis=1)  # no empty rows
    lengths = take.sum(axis=1)
    big_off = np.zeros(n_tx + 1, dtype=np.uint64)
    np.cumsum(lengths, out=big_off[1:])
    big_cols = np.nonzero(take)[1].astype(np.uint32)
    res = _native.Database.from_columns(ctx, big_off, big_cols, k).mine(
        int(0.05 * n_tx), _native.CPM_ECLAT, order=_native.CPM_ORDER_ECLAT)
    assert res.stats["work_items"] > 0  # the deep kernel ran
    labels, arrays = oracle.mine_csr(big_off, big_cols, int(0.05 * n_tx), "eclat")
    want = oracle.to_dict(labels, arrays)
    assert len(res) == len(want)
    assert sorted(res.supports.tolist()) == sorted(want.values())
