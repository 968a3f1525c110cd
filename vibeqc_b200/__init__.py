"""B200-native density-fitted RHF energy and analytic forces.

Public surface mirrors the reference's Calculator / prepare_batch API for the
DF-RHF path: :class:`Calculator`, :class:`PreparedBatch`, :class:`Result`,
:class:`BatchResult`, :class:`BatchItemResult`.
"""

from . import geometry  # noqa: F401
from .calculator import (  # noqa: F401
    BatchItemResult,
    BatchResult,
    Calculator,
    PreparedBatch,
    Result,
)

__all__ = ["Calculator", "PreparedBatch", "Result", "BatchResult", "BatchItemResult", "geometry"]
