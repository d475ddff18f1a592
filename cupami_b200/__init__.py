"""cupami_b200: B200-native vertical-bitset frequent-itemset mining.

Drop-in replacements for cuPAMI's ``cuEclat`` and ``cuApriori`` (and the
periodic-frequent ``cuPFEclat`` / ``cuPFApriori`` over the same tidsets) whose
mining runs in hand-written sm_100a CUDA behind a C ABI (``libcupami_b200.so``,
declared in ``include/cupami_b200.h``).  Importing the package needs neither a
GPU nor the built library; ``mine()`` needs both and raises without them.
"""

from .datasets import TransactionCSR
from .frequentPattern import Apriori, Eclat, cuApriori, cuEclat
from .periodicFrequentPattern import cuPFApriori, cuPFEclat

__all__ = ["TransactionCSR", "cuApriori", "cuEclat", "Apriori", "Eclat", "cuPFApriori", "cuPFEclat"]
__version__ = "0.1.0"
