import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")


@pytest.fixture(scope="session")
def golden():
    import json

    return json.loads((ROOT / "tests" / "golden" / "reference_patterns.json").read_text())


@pytest.fixture(scope="session")
def oracle_lib():
    import oracle

    oracle.build()
    return oracle


def _inject_result(miner, patterns, order):
    """Give a miner the result `patterns` ([[tab-joined labels, support], ...] or
    [[labels, support, periodicity], ...] in insertion order, prefixes first)
    without a GPU: a host pattern tree ordered by the C ABI, as mine() would
    leave it."""
    from cupami_b200._native import Result

    labels = sorted({x for key, *_ in patterns for x in key.split("\t")})
    col = {x: i for i, x in enumerate(labels)}
    ids = {}
    parent, item, support, period = [], [], [], []
    for k, (key, sup, *rest) in enumerate(patterns):
        items = [col[x] for x in key.split("\t")]
        parent.append(ids[tuple(items[:-1])] if len(items) > 1 else -1)
        item.append(items[-1])
        support.append(sup)
        period.extend(rest)
        ids[tuple(items)] = k
    miner._result = Result.from_tree(parent, item, support, order, period=period if period else None)
    miner._labels = labels
    miner._patterns = None
    return miner


@pytest.fixture(scope="session")
def inject():
    return _inject_result
