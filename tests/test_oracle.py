"""The CPU oracle against the reference's own outputs (tests/golden)."""
import numpy as np
import pytest


def _cases(golden):
    for case in golden["cases"]:
        for algo, runs in case["results"].items():
            for run in runs:
                yield case, algo, run


def test_oracle_matches_every_golden_case(golden, oracle_lib):
    checked = 0
    for case, algo, run in _cases(golden):
        got = oracle_lib.mine_rows(case["rows"], run["minSup"],
                                   "eclat" if algo == "cuEclat" else "apriori")
        want = [(k, v) for k, v in run["patterns"]]
        assert list(got.items()) == want, (case["name"], algo, run["minSup"])
        checked += 1
    assert checked >= 50


def test_oracle_quickstart_known_answer(golden, oracle_lib):
    from pathlib import Path

    q = golden["quickstart"]
    data = np.load(Path(__file__).parent / "golden" / q["data"])
    for algo in ("cuEclat", "cuApriori"):
        labels, arrays = oracle_lib.mine_csr(data["offsets"], data["items"], 0.01,
                                             "eclat" if algo == "cuEclat" else "apriori")
        got = oracle_lib.to_dict(labels, arrays)
        want = q["results"][algo]["patterns"]
        assert len(got) == 1275
        assert list(got.items()) == [(k, v) for k, v in want]
    assert got["1"] == 1208 and got["10"] == 1151 and got["11"] == 1201


def test_reference_sampler_restatement_matches_fixture(golden):
    """datasets.reference_uniform_baskets rebuilds the quickstart data exactly."""
    from pathlib import Path

    from cupami_b200.datasets import TransactionCSR, reference_uniform_baskets

    data = np.load(Path(__file__).parent / "golden" / golden["quickstart"]["data"])
    rows = reference_uniform_baskets(10000, 50, avg_length=6, seed=42)
    csr = TransactionCSR.from_rows(rows)
    assert np.array_equal(csr.offsets, data["offsets"])
    assert np.array_equal(csr.items, data["items"])


@pytest.mark.parametrize("threshold", [0, -3])
def test_oracle_nonpositive_threshold_emits_zero_supports(oracle_lib, threshold):
    rows = [["a", "b"], ["c"]]
    got = oracle_lib.mine_rows(rows, threshold)
    assert got["a\tc"] == 0 and got["a\tb\tc"] == 0 and len(got) == 7


def test_support_rule():
    from oracle import support_count

    assert support_count(0.25, 10) == 3
    assert support_count(1.0, 7) == 7
    assert support_count(2.5, 10) == 2
    assert support_count(100, 10) == 100
    assert support_count(True, 10) == 1
