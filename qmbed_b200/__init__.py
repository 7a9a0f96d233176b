"""B200-native engine for QMBED's symmetry-reduced spin-chain H.v and Krylov solvers.

``qmbed_b200.model`` mirrors the reference Python API (JSON boundary);
``qmbed_b200.engine`` exposes typed GPU handles (bases, operators, eigsh,
exponential action). Both call ``libqmbed_b200.so``; there is no CPU path.
"""

from ._lib import QmbedError
from .engine import GpuBasis, GpuOperator, deterministic_start, device_count, heisenberg_terms, tfim_terms
from .model import (Coupling, Eigensystem, EigshOptions, LocalOperator, NativeExpmAction, NativeModel, OperatorSpec,
                    OpProduct, SpinBasis, eigsh, heisenberg_specs)

__all__ = [
    "QmbedError", "GpuBasis", "GpuOperator", "deterministic_start", "device_count", "heisenberg_terms",
    "tfim_terms", "Coupling", "Eigensystem", "EigshOptions", "LocalOperator", "NativeExpmAction", "NativeModel",
    "OperatorSpec", "OpProduct", "SpinBasis", "eigsh", "heisenberg_specs",
]
