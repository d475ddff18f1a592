"""Drop-in ``cuPFEclat``: periodic-frequent itemsets, reported in the
reference's depth-first insertion order.

Reference: ``cupami/periodicFrequentPattern/cuPFEclat.py:142-175``.  The
reference walks the prefix classes depth first on the host and evaluates every
class's extensions with the ``periodic_counts`` kernel; here the whole search
runs on the device (``cpm_mine_periodic``) and the patterns come back in the
reference's order (``CPM_ORDER_DEPTH_FIRST``): singletons, then for each
pattern, depth first, the extensions it keeps.
"""

from __future__ import annotations

import sys

from .. import _native
from ._temporal import TemporalInput


class cuPFEclat(TemporalInput):
    """Depth-first periodic-frequent itemset mining over timestamp occurrence bitsets.

    Parameters: ``iFile`` (rows ``timestamp, item, ...``, a temporal CSV/TSV/BIN/
    Parquet path or an HTTP(S) CSV URL), ``minSup``, ``maxPer``, ``sep`` and
    the keyword ``endTime``.
    """

    #: Kept for compatibility: the reference evaluates candidates in batches of
    #: this size; the device search has no batches.
    _BATCH_SIZE = 4096
    _ALGORITHM = _native.CPM_ECLAT
    _ORDER = _native.CPM_ORDER_DEPTH_FIRST


def _cli(cls, argv):
    if len(argv) not in (5, 6):
        sys.exit(f"Usage: python -m {cls.__module__} <inputFile> <outputFile> <minSup> <maxPer> [sep]")

    def number(text):
        try:
            return int(text)
        except ValueError:
            return float(text)

    miner = cls(argv[1], number(argv[3]), number(argv[4]), argv[5] if len(argv) == 6 else None)
    miner.mine()
    miner.save(argv[2])
    miner.printResults()


if __name__ == "__main__":
    _cli(cuPFEclat, sys.argv)
