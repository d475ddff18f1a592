"""Drop-in frequent-itemset miners (cuPAMI ``cupami.frequentPattern`` names)."""

from .cuApriori import Apriori, cuApriori
from .cuEclat import Eclat, cuEclat

__all__ = ["Apriori", "cuApriori", "Eclat", "cuEclat"]
