"""Truncation policy API (crates/core/src/policy/truncators.rs).

The truncators, the legacy TruncationPolicy that decomposes into them, and
the flattening into one ResolvedConfig the engine receives.
"""

from __future__ import annotations

from dataclasses import dataclass

from . import _native


class FrequencyTruncator:
    """Surrogate-only: bound on a symbolic coefficient's trigonometric frequency."""

    def __init__(self, frequency: int | None = None):
        self.frequency = frequency

    def __repr__(self):
        return f"FrequencyTruncator(frequency={self.frequency})"


class CoefficientTruncator:
    """Drops a branch or term whose |coefficient| is strictly below `coefficient`."""

    def __init__(self, coefficient: float | None = None):
        self.coefficient = coefficient

    def __repr__(self):
        return f"CoefficientTruncator(coefficient={self.coefficient})"


class WeightTruncator:
    """Drops terms whose Pauli (or Jordan-Wigner) weight exceeds `weight`."""

    def __init__(self, weight: int | None = None):
        self.weight = weight

    def __repr__(self):
        return f"WeightTruncator(weight={self.weight})"


class TermBudget:
    """Live-term floor below which lossy truncation is suppressed."""

    def __init__(self, min_terms: int | None = None):
        self.min_terms = min_terms

    def __repr__(self):
        return f"TermBudget(min_terms={self.min_terms})"


class Simplify:
    """Surrogate-only: symbolic simplification switch."""

    def __init__(self, enabled: bool = True):
        self.enabled = enabled

    def __repr__(self):
        return f"Simplify(enabled={self.enabled})"


class NativeTruncator:
    """Truncation policy from a native plugin (propaq_truncator_* C ABI,
    crates/core/src/policy/native_truncator.rs:13-33)."""

    def __init__(self, path: str, config: str | None = None):
        self._plugin = _native.Plugin(path, config, noise=False)

    @property
    def abi_version(self) -> int:
        return 1

    @property
    def depends(self) -> int:
        return self._plugin.depends

    @property
    def handle(self) -> int:
        return self._plugin.handle

    def keep_term(self, basis_kind, words, n_units, weight, coeff_magnitude, layer_index=0, n_layers=0) -> bool:
        if basis_kind not in (0, 1):
            raise ValueError(f"basis_kind must be 0 (Pauli) or 1 (Majorana), got {basis_kind}")
        return self._plugin.keep(basis_kind, words, n_units, weight, coeff_magnitude, layer_index, n_layers)

    def __repr__(self):
        return f"NativeTruncator(<native plugin, depends={self.depends}>)"


class TruncationPolicy:
    """Legacy single-object policy (truncators.rs:225-285)."""

    def __init__(self, weight_cutoff: int | None = None, coeff_cutoff: float = 0.0, min_terms: int | None = None):
        self.weight_cutoff = weight_cutoff
        self.coeff_cutoff = coeff_cutoff
        self.min_terms = min_terms

    def should_truncate(self, weight: int, abs_coeff: float) -> bool:
        return (self.weight_cutoff is not None and weight > self.weight_cutoff) or abs_coeff < self.coeff_cutoff

    def decompose(self) -> list:
        ops: list = []
        if self.weight_cutoff is not None:
            ops.append(WeightTruncator(self.weight_cutoff))
        if self.coeff_cutoff > 0.0:
            ops.append(CoefficientTruncator(self.coeff_cutoff))
        if self.min_terms is not None:
            ops.append(TermBudget(self.min_terms))
        return ops

    def __repr__(self):
        return (f"TruncationPolicy(weight_cutoff={self.weight_cutoff}, coeff_cutoff={self.coeff_cutoff}, "
                f"min_terms={self.min_terms})")


_TRUNCATORS = (FrequencyTruncator, CoefficientTruncator, WeightTruncator, TermBudget, Simplify, NativeTruncator)


def resolve_truncation(truncation) -> list:
    """A truncator list from the constructor's `truncation` (truncators.rs:293-311)."""
    if truncation is None:
        return []
    if isinstance(truncation, TruncationPolicy):
        return truncation.decompose()
    if isinstance(truncation, (list, tuple)):
        if all(isinstance(t, _TRUNCATORS) for t in truncation):
            return list(truncation)
    elif isinstance(truncation, _TRUNCATORS):
        return [truncation]
    raise TypeError(
        "truncation must be a truncator (FrequencyTruncator/CoefficientTruncator/WeightTruncator/TermBudget/"
        "Simplify/NativeTruncator), a list of truncators, a TruncationPolicy, or None"
    )


def reject_surrogate_only(truncators: list) -> None:
    if any(isinstance(t, (FrequencyTruncator, Simplify)) for t in truncators):
        raise ValueError(
            "FrequencyTruncator/Simplify only apply to surrogate propagation, use WeightTruncator / "
            "CoefficientTruncator / TermBudget with the numerical propagator"
        )


@dataclass
class ResolvedConfig:
    """The flat form of a truncator pipeline (truncators.rs:187-213); later entries win."""

    frequency: int | None = None
    coefficient: float | None = None
    weight: int | None = None
    min_terms: int | None = None
    simplify: bool = False
    native: NativeTruncator | None = None


def resolve_config(truncators: list) -> ResolvedConfig:
    r = ResolvedConfig()
    for t in truncators:
        if isinstance(t, FrequencyTruncator):
            r.frequency = t.frequency
        elif isinstance(t, CoefficientTruncator):
            r.coefficient = t.coefficient
        elif isinstance(t, WeightTruncator):
            r.weight = t.weight
        elif isinstance(t, TermBudget):
            r.min_terms = t.min_terms
        elif isinstance(t, Simplify):
            r.simplify = t.enabled
        elif isinstance(t, NativeTruncator):
            r.native = t
    return r
