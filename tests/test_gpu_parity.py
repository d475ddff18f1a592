"""CUDA path vs the reference's outputs and the CPU oracle (bit-exact)."""
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).parent / "golden"


def _miner(algo):
    import cupami_b200

    return cupami_b200.cuEclat if algo == "cuEclat" else cupami_b200.cuApriori


def test_native_library_is_loaded():
    import cupami_b200._native as n

    ctx = n.context(0)
    assert ctx.handle
    assert n.LIB_PATH.exists()


def test_every_golden_case_in_reference_order(golden):
    for case in golden["cases"]:
        for algo, runs in case["results"].items():
            for run in runs:
                miner = _miner(algo)(case["rows"], run["minSup"])
                assert miner._minSup == run["resolved"]
                miner.mine()
                got = list(miner.getPatterns().items())
                assert got == [tuple(p) for p in run["patterns"]], (case["name"], algo, run["minSup"])


def test_quickstart_known_answer(golden):
    from cupami_b200 import TransactionCSR

    q = golden["quickstart"]
    data = np.load(GOLDEN / q["data"])
    csr = TransactionCSR(data["offsets"], data["items"], 50)
    for algo in ("cuEclat", "cuApriori"):
        miner = _miner(algo)(csr, 0.01)
        miner.mine()
        got = miner.getPatterns()
        assert len(got) == 1275
        assert list(got.items()) == [tuple(p) for p in q["results"][algo]["patterns"]]


def test_small_batches_and_dense_known_answer():
    import cupami_b200

    rows = [list(range(8))] * 65
    miner = cupami_b200.cuEclat(rows, 1)
    miner._PAIR_BATCH_SIZE = 3
    miner._INTERSECTION_BATCH_BYTES = 12
    miner.mine()
    assert len(miner.getPatterns()) == 255
    assert "0\t1\t2\t3\t4\t5\t6\t7" in miner.getPatterns()


def test_repeated_mining_is_identical():
    import cupami_b200

    miner = cupami_b200.cuEclat([[1, 2], [2, 3], [1, 2, 3]], 1)
    miner.mine()
    first = miner.getPatterns()
    miner.mine()
    assert miner.getPatterns() == first
    assert miner.getRuntime() >= 0


def _oracle_check(oracle_lib, csr, minsup, algo="eclat"):
    import cupami_b200

    labels, arrays = oracle_lib.mine_csr(csr.offsets, csr.items, minsup, algo)
    want = oracle_lib.to_dict(labels, arrays)
    cls = cupami_b200.cuEclat if algo == "eclat" else cupami_b200.cuApriori
    miner = cls(csr, minsup)
    miner.mine()
    got = miner.getPatterns()
    assert list(got.items()) == list(want.items())
    return miner


@pytest.mark.parametrize("name", ["uniform-10k", "planted-100k", "dense-fixed-64k", "dense-bernoulli-64k"])
def test_workloads_match_oracle(oracle_lib, name):
    from cupami_b200 import datasets

    csr, minsup = datasets.workload(name)
    miner = _oracle_check(oracle_lib, csr, minsup, "eclat")
    if name == "dense-fixed-64k":
        assert miner.getPatterns() == {}
    if name in ("uniform-10k", "planted-100k"):
        _oracle_check(oracle_lib, csr, minsup, "apriori")


def test_batched_databases_match_oracle(oracle_lib):
    from cupami_b200 import datasets

    for csr in datasets.batched_zipf(limit=6):
        _oracle_check(oracle_lib, csr, 0.01, "eclat")


@pytest.mark.parametrize("count", [0, 1, 31, 32, 33, 63, 64, 65, 127, 128, 129, 1000])
def test_word_boundaries_dense(oracle_lib, count):
    from cupami_b200 import TransactionCSR

    rng = np.random.default_rng(count)
    rows = [[int(i) for i in np.nonzero(rng.random(10) < 0.6)[0]] for _ in range(count)]
    csr = TransactionCSR.from_rows(rows, universe=10)
    _oracle_check(oracle_lib, csr, max(1, count // 6), "eclat")
    _oracle_check(oracle_lib, csr, max(1, count // 6), "apriori")


def test_batch_of_databases_matches_single_mines(oracle_lib):
    from cupami_b200 import _native, cuEclat, datasets

    csrs = datasets.batched_zipf(limit=10)
    miners = cuEclat.mineBatch(csrs, 0.01)
    for csr, m in zip(csrs, miners):
        single = cuEclat(csr, 0.01)
        single.mine()
        assert list(m.getPatterns().items()) == list(single.getPatterns().items())
        labels, arrays = oracle_lib.mine_csr(csr.offsets, csr.items, 0.01)
        assert m.getPatterns() == oracle_lib.to_dict(labels, arrays)
    # mixed sizes and thresholds, including an empty database
    rows_a = [[1, 2, 3]] * 40 + [[2, 3]] * 10
    rows_b = []
    ms = cuEclat.mineBatch([rows_a, rows_b, csrs[0]], [5, 1, 0.02])
    assert ms[1].getPatterns() == {}
    assert ms[0].getPatterns() == oracle_lib.mine_rows(rows_a, 5)
    assert ms[2].getPatterns() == oracle_lib.to_dict(*oracle_lib.mine_csr(csrs[0].offsets, csrs[0].items, 0.02))


def test_batched_loader_matches_single_loads(oracle_lib):
    """cpm_db_from_ids_batch: same shapes, labels and patterns as one cpm_db_from_ids per database,
    with databases whose rows share a warp, empty databases and empty rows."""
    from cupami_b200 import TransactionCSR, _native

    rng = np.random.default_rng(11)
    csrs = []
    for n in [17, 0, 45, 3, 1, 64, 33, 500, 2, 129]:
        rows = [[int(v) for v in rng.choice(40, size=rng.integers(0, 8), replace=False)] for _ in range(n)]
        csrs.append(TransactionCSR.from_rows(rows))
    csrs.append(TransactionCSR.from_rows([[], [], []]))
    csrs.append(TransactionCSR.from_rows([[1 << 20, 5], [5], [1 << 20, 7, 5]]))
    ctx = _native.context(0)
    batch = _native.Database.from_ids_batch(ctx, [(c.offsets, c.items) for c in csrs])
    try:
        assert len(batch) == len(csrs)
        for csr, db in zip(csrs, batch):
            single = _native.Database.from_ids(ctx, csr.offsets, csr.items)
            try:
                assert (db.n_transactions, db.n_items) == (single.n_transactions, single.n_items)
                assert db.labels.tolist() == single.labels.tolist()
                a = db.mine(1, _native.CPM_ECLAT)
                b = single.mine(1, _native.CPM_ECLAT)
                assert a.patterns(db.labels) == b.patterns(single.labels)
            finally:
                single.close()
            labels, arrays = oracle_lib.mine_csr(csr.offsets, csr.items, 1)
            assert a.patterns(db.labels) == oracle_lib.to_dict(labels, arrays)
    finally:
        for db in batch:
            db.close()
    # ids past the batched presence table fall back to the one-database loader
    big = TransactionCSR.from_rows([[1 << 27, 3], [3]])
    (db,) = _native.Database.from_ids_batch(ctx, [(big.offsets, big.items)])
    try:
        assert db.labels.tolist() == sorted([1 << 27, 3], key=str)
    finally:
        db.close()
