"""propaq_b200 -- a B200-native engine for Heisenberg-picture Pauli and Majorana
propagation, exposing the propagation surface of hkbelagali/propaq.

The hot path (branching, merging, truncation, noise damping and the expectation
reduction) runs as hand-written sm_100a CUDA kernels in lib/libpropaq_cuda.so,
behind the C ABI of include/propaq_cuda.h.  This package is the host-side mirror
of the reference's Python/pyo3 API over that library.
"""

from .circuits import MajoranaCircuit, MajoranaRotation, PauliCircuit, PauliRotation
from .datatypes import MajoranaMonomial, MajoranaTermSum, PauliString, PauliTermSum
from .noise import GateNoiseModel, NativeNoiseModel, UniformNoiseModel
from .propagators import Logger, MajoranaPropagator, PauliPropagator, PropagationResult
from .truncation import (
    CoefficientTruncator,
    FrequencyTruncator,
    NativeTruncator,
    Simplify,
    TermBudget,
    TruncationPolicy,
    WeightTruncator,
)

__all__ = [
    "PauliString", "PauliTermSum", "MajoranaMonomial", "MajoranaTermSum",
    "PauliRotation", "PauliCircuit", "MajoranaRotation", "MajoranaCircuit",
    "PauliPropagator", "MajoranaPropagator", "PropagationResult", "Logger",
    "UniformNoiseModel", "GateNoiseModel", "NativeNoiseModel",
    "TruncationPolicy", "WeightTruncator", "CoefficientTruncator", "TermBudget",
    "FrequencyTruncator", "Simplify", "NativeTruncator",
]
