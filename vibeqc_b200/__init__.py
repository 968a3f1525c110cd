"""B200-native density-fitted RHF/UHF energy and analytic forces.

Public surface mirrors the reference's Calculator / prepare_batch API for the
DF path: :class:`Calculator`, :class:`PreparedBatch`, :class:`Result`,
:class:`BatchResult`, :class:`BatchItemResult`; and its fixed-density J/K
source for other methods (hybrid DFT): :class:`FockPlan`,
:class:`FockBuildSpec`, :class:`FockTerm`, :class:`FockEvaluation`.
"""

from . import geometry  # noqa: F401
from .calculator import (  # noqa: F401
    BatchItemResult,
    BatchResult,
    Calculator,
    PreparedBatch,
    Result,
)
from .fock import FockBuildSpec, FockEvaluation, FockPlan, FockTerm  # noqa: F401

__all__ = ["Calculator", "PreparedBatch", "Result", "BatchResult", "BatchItemResult", "geometry",
           "FockPlan", "FockBuildSpec", "FockTerm", "FockEvaluation"]
