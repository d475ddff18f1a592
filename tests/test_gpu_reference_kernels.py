"""The CUDA path against the reference's own GPU path on the same GPU.

``oracle.ref_gpu`` runs the reference's three kernels (compiled from its own
CUDA source by ``oracle/build_ref.py``) under the reference's driver loops,
with torch tensors in place of CuPy arrays.  Both paths must give the same
patterns, supports and order.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ref():
    from oracle import ref_gpu

    if not ref_gpu.available():
        pytest.skip("oracle/_ref/libref_bitsets.so not built (needs the reference sources)")
    return ref_gpu


def _ours(csr, minsup, algo):
    from cupami_b200 import cuApriori, cuEclat

    m = (cuEclat if algo == "eclat" else cuApriori)(csr, minsup)
    m.mine()
    return list(m.getPatterns().items())


def _theirs(ref, csr, minsup, algo):
    off, ids = ref.upload(csr.offsets, csr.items)
    return [("\t".join(k), v) for k, v in ref.mine(off, ids, minsup, algo).items()]


@pytest.mark.parametrize("name,minsup,algos", [
    ("uniform_poisson", 0.01, ("eclat", "apriori")),
    ("planted_zipf", 0.005, ("eclat", "apriori")),
    ("dense_bernoulli", 0.6, ("eclat",)),
])
def test_workloads_match_reference_gpu_path(ref, name, minsup, algos):
    from cupami_b200 import datasets

    kwargs = {"dense_bernoulli": {"n": 8192}}.get(name, {})
    csr = getattr(datasets, name)(**kwargs)
    for algo in algos:
        assert _ours(csr, minsup, algo) == _theirs(ref, csr, minsup, algo), algo


@pytest.mark.parametrize("count", [1, 31, 32, 33, 64, 65, 1000])
def test_word_boundaries_match_reference_gpu_path(ref, count):
    from cupami_b200 import TransactionCSR

    rng = np.random.default_rng(100 + count)
    rows = [[int(i) for i in np.nonzero(rng.random(12) < 0.5)[0]] for _ in range(count)]
    rows[0] = rows[0] or [3]
    csr = TransactionCSR.from_rows(rows, universe=12)
    for algo in ("eclat", "apriori"):
        assert _ours(csr, 2, algo) == _theirs(ref, csr, 2, algo)


def test_batched_databases_match_reference_gpu_path(ref):
    from cupami_b200 import cuEclat, datasets

    csrs = datasets.batched_zipf(limit=4)
    miners = cuEclat.mineBatch(csrs, 0.01)
    for csr, m in zip(csrs, miners):
        assert list(m.getPatterns().items()) == _theirs(ref, csr, 0.01, "eclat")
