"""propaq._rust_core on the B200 engine.

The reference's Python package re-exports every propagation class from its
compiled pyo3 module `propaq._rust_core` (propaq/__init__.py:18-81,
propaq/propagators/pauli.py:13, propaq/noise/uniform.py:3,7; the module's
surface is propaq/_rust_core/__init__.pyi).  This module offers the same names,
constructors and methods over this package, so the reference's own
pure-Python modules (its extrapolators, propagator base classes, log parser,
circuits) run on the GPU engine unchanged once it stands in for the compiled
module:

    import propaq_b200.rust_core
    propaq_b200.rust_core.install()   # before `import propaq`
    import propaq                     # propaq._rust_core is now this module

The numerical path is the engine's: PauliPropagator / MajoranaPropagator,
term sums, truncators, noise models, plugins, term files and the verbose
Logger.  The surrogate propagators and models and the hybrid MPS expectation
are outside this engine; their names exist so that imports succeed, and
constructing or calling them raises NotImplementedError.
"""

from __future__ import annotations

import gzip
import struct
import sys
import types

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
    "CoefficientTruncator", "FrequencyTruncationPolicy", "FrequencyTruncator", "GateNoiseModel", "Logger",
    "MajoranaMonomial", "MajoranaPropagator", "MajoranaSurrogateModel", "MajoranaSurrogatePropagator",
    "MajoranaTermStreamer", "MajoranaTermSum", "NativeNoiseModel", "NativeTruncator", "PauliPropagator",
    "PauliString", "PauliSurrogateModel", "PauliSurrogatePropagator", "PauliTermStreamer", "PauliTermSum",
    "PropagationResult", "Simplify", "TermBudget", "TruncationPolicy", "UniformNoiseModel", "WeightTruncator",
    "hybrid_expectation", "rust_available", "install",
]

_OUTSIDE = ("is not part of the B200 propagation engine (it runs the numerical propagators only); "
            "use the reference's own build for it")


class FrequencyTruncationPolicy:
    """The surrogate build's legacy policy (crates/core/src/policy/truncators.rs:
    225-285); like FrequencyTruncator it only applies to surrogate propagation,
    and the numerical propagators refuse it."""

    def __init__(self, max_frequency: int | None = None, weight_cutoff: int | None = None,
                 min_terms: int | None = None):
        self.max_frequency = max_frequency
        self.weight_cutoff = weight_cutoff
        self.min_terms = min_terms

    def __repr__(self):
        return (f"FrequencyTruncationPolicy(max_frequency={self.max_frequency}, "
                f"weight_cutoff={self.weight_cutoff}, min_terms={self.min_terms})")


class _TermStreamer:
    """Streams (term, coeff) pairs out of a term file one record at a time
    (crates/core/src/interface/streamer.rs; the file layout of term_io.rs:24-56)."""

    _pauli = True

    def __init__(self, path: str):
        self._f = gzip.open(path, "rb")
        n, stride, size = struct.unpack("<QQQ", self._f.read(24))
        self._left, self._stride, self._size = n, stride, size

    @classmethod
    def from_file(cls, path: str):
        return cls(path)

    def __iter__(self):
        return self

    def _term(self, kb: bytes):
        if self._pauli:
            nb = (self._size + 7) // 8
            return PauliString(int.from_bytes(kb[:nb], "little"), int.from_bytes(kb[nb:2 * nb], "little"), self._size)
        modes = int.from_bytes(kb, "little")
        single = any((modes >> (2 * k) & 1) != (modes >> (2 * k + 1) & 1) for k in range(self._size // 2))
        return MajoranaMonomial(modes, self._size, is_number_preserving=not single)

    def __next__(self):
        if self._left == 0:
            self._f.close()
            raise StopIteration
        self._left -= 1
        kb = self._f.read(self._stride)
        (c,) = struct.unpack("<d", self._f.read(8))
        return self._term(kb), c


class PauliTermStreamer(_TermStreamer):
    """PauliTermStreamer.from_file(path) yields (PauliString, coeff) pairs."""

    _pauli = True


class MajoranaTermStreamer(_TermStreamer):
    """MajoranaTermStreamer.from_file(path) yields (MajoranaMonomial, coeff) pairs."""

    _pauli = False


def _merge_from_file(self, streamer) -> None:
    """Adds every streamed term to this sum (duplicates add up)."""
    for term, coeff in streamer:
        self.add(term, coeff)


PauliTermSum.merge_from_file = _merge_from_file
MajoranaTermSum.merge_from_file = _merge_from_file


class _Outside:
    """A class of the reference's surface that this engine does not provide."""

    def __init__(self, *args, **kwargs):
        raise NotImplementedError(f"{type(self).__name__} {_OUTSIDE}")

    @classmethod
    def load(cls, path: str):
        raise NotImplementedError(f"{cls.__name__} {_OUTSIDE}")


class PauliSurrogatePropagator(_Outside):
    pass


class MajoranaSurrogatePropagator(_Outside):
    pass


class PauliSurrogateModel(_Outside):
    pass


class MajoranaSurrogateModel(_Outside):
    pass


def hybrid_expectation(observable, mps_arrays) -> float:
    raise NotImplementedError(f"hybrid_expectation {_OUTSIDE}")


def rust_available() -> bool:
    """True: the compiled propagation core is present (here, the CUDA engine)."""
    return True


def install() -> types.ModuleType:
    """Registers this module as propaq._rust_core, so that the reference's
    Python package imports the engine instead of its compiled module."""
    mod = sys.modules[__name__]
    sys.modules["propaq._rust_core"] = mod
    pkg = sys.modules.get("propaq")
    if pkg is not None:
        pkg._rust_core = mod
    return mod
