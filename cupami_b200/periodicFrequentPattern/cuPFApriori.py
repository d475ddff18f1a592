"""Drop-in ``cuPFApriori``: periodic-frequent itemsets, reported level by level.

Reference: ``cupami/periodicFrequentPattern/cuPFApriori.py:136-157`` -- every
level's candidates from ``cuApriori._generateCandidates`` (prefix join and
subset pruning, ``cupami/frequentPattern/cuApriori.py:473-492``) evaluated by
the ``periodic_counts`` kernel.  Here the levels run on the device
(``cpm_mine_periodic``) and the patterns come back by length, then tuple.
"""

from __future__ import annotations

import sys

from .. import _native
from ._temporal import TemporalInput
from .cuPFEclat import _cli


class cuPFApriori(TemporalInput):
    """Level-wise periodic-frequent itemset mining over timestamp occurrence bitsets."""

    #: Kept for compatibility (the reference's candidate batch size).
    _BATCH_SIZE = 4096
    _ALGORITHM = _native.CPM_APRIORI
    _ORDER = _native.CPM_ORDER_APRIORI


if __name__ == "__main__":
    _cli(cuPFApriori, sys.argv)
