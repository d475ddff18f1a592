"""GPU: the tensor-core (tcgen05 INT8) pair Gram against the CUDA-core Gram and the oracle."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _csr(n, n_items, lo, hi, seed):
    from cupami_b200 import TransactionCSR

    rng = np.random.default_rng(seed)
    p = rng.uniform(lo, hi, n_items)
    rows = [[int(i) for i in np.nonzero(rng.random(n_items) < p)[0]] for _ in range(n)]
    return TransactionCSR.from_rows(rows, universe=n_items)


def _mine(csr, minsup, engine, cls_name="cuEclat"):
    import cupami_b200

    cls = getattr(cupami_b200, cls_name)
    m = cls(csr, minsup)
    m._PAIR_ENGINE = engine
    m.mine()
    return m


@pytest.mark.parametrize("n,n_items,seed", [(200, 40, 1), (2049, 130, 2), (5000, 300, 3), (777, 513, 4)])
def test_tensor_core_gram_matches_cuda_core_gram(oracle_lib, n, n_items, seed):
    csr = _csr(n, n_items, 0.02, 0.12, seed)
    minsup = 0.01
    tc = _mine(csr, minsup, 1)
    simt = _mine(csr, minsup, 2)
    assert tc.getKernelStats()["n_frequent_pairs"] > 0
    assert list(tc.getPatterns().items()) == list(simt.getPatterns().items())
    labels, arrays = oracle_lib.mine_csr(csr.offsets, csr.items, minsup)
    assert tc.getPatterns() == oracle_lib.to_dict(labels, arrays)


def test_tensor_core_gram_on_the_planted_workload(oracle_lib):
    from cupami_b200 import datasets

    csr, minsup = datasets.workload("planted-100k")
    for cls in ("cuEclat", "cuApriori"):
        tc = _mine(csr, minsup, 1, cls)
        simt = _mine(csr, minsup, 2, cls)
        assert list(tc.getPatterns().items()) == list(simt.getPatterns().items())
    labels, arrays = oracle_lib.mine_csr(csr.offsets, csr.items, minsup)
    assert tc.getPatterns() == oracle_lib.to_dict(labels, arrays)
