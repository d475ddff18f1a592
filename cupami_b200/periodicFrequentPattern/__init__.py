"""Drop-in periodic-frequent miners (cuPAMI ``cupami.periodicFrequentPattern`` names)."""

from ._temporal import TemporalInput
from .cuPFApriori import cuPFApriori
from .cuPFEclat import cuPFEclat

__all__ = ["TemporalInput", "cuPFApriori", "cuPFEclat"]
