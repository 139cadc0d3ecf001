"""Zero-noise and zero-cutoff extrapolation over batched propagation.

The reference's drivers (propaq/extrapolators/zne.py:38-108,
propaq/extrapolators/zce.py:46-160) sweep a noise value or a truncation
cutoff, call `expectation_value` once per value, fit the curve with
scipy.optimize.curve_fit and read it at zero.  These classes keep their
names, arguments, results and the propagator's restored state, but run the
whole sweep as one pq_run_batch (propagators.expectation_values): every sweep
point is an instance of the same persistent launches.  A sweep the batch does
not run (a plugin the host must consult per term, or a TermBudget floor that
decides Clifford deferral mid-run) falls back to one call per value.
"""

from __future__ import annotations

from abc import ABC, abstractmethod
from collections.abc import Callable
from dataclasses import dataclass

import numpy as np
from scipy.optimize import curve_fit

from .noise import UniformNoiseModel
from .propagators import expectation_values
from .truncation import CoefficientTruncator, WeightTruncator


def _sweep(propagators, observable, circuit, initial_state, device):
    """Expectation values of the same problem under each propagator."""
    jobs = [(p, observable, circuit, initial_state) for p in propagators]
    try:
        return [r.expectation_value for r in expectation_values(jobs, device=device)]
    except NotImplementedError:
        return [p.expectation_value(observable, circuit, initial_state=initial_state).expectation_value
                for p in propagators]


def _like(propagator, noise, truncators):
    """A propagator of the same class and device with the given noise and truncation."""
    return type(propagator)(noise=noise, truncation=list(truncators), device=propagator.device)


@dataclass
class ZNEResult:
    """Zero-noise extrapolation: the value at zero noise and the fit behind it."""

    zero_noise_value: float
    noise_values: list[float]
    expectation_values: list[float]
    fit_params: np.ndarray
    fit_covariance: np.ndarray


class ZeroNoiseExtrapolator:
    """Fits `fitting_fn(noise, *params)` to the expectation values at
    `noise_values` and evaluates it at zero."""

    def __init__(self, fitting_fn: Callable, noise_values: list[float]) -> None:
        self.fitting_fn = fitting_fn
        self.noise_values = list(noise_values)

    def build_noise(self, value: float):
        """The noise model of one sweep point; `UniformNoiseModel(value)` unless
        overridden (e.g. to sweep one parameter of a custom model)."""
        return UniformNoiseModel(value)

    def run(self, propagator, observable, circuit, initial_state=0, **curve_fit_kwargs) -> ZNEResult:
        """Sweeps the noise values (one batch), fits, and extrapolates to zero.
        `propagator` is left with its own noise model."""
        truncators = propagator.truncators
        props = [_like(propagator, self.build_noise(v), truncators) for v in self.noise_values]
        values = _sweep(props, observable, circuit, initial_state, propagator.device)
        popt, pcov = curve_fit(self.fitting_fn, self.noise_values, values, **curve_fit_kwargs)
        return ZNEResult(zero_noise_value=float(self.fitting_fn(0.0, *popt)), noise_values=self.noise_values,
                         expectation_values=values, fit_params=popt, fit_covariance=pcov)


@dataclass
class ZCEResult:
    """Zero-cutoff extrapolation: the value at zero cutoff and the fit behind it."""

    zero_cutoff_value: float
    cutoff_values: list[float]
    expectation_values: list[float]
    fit_params: np.ndarray
    fit_covariance: np.ndarray


class ZeroCutoffExtrapolator(ABC):
    """Fits `fitting_fn(cutoff, *params)` to the expectation values with one
    truncator of the propagator's pipeline set to each of `cutoff_values`."""

    def __init__(self, fitting_fn: Callable, cutoff_values: list[float]) -> None:
        self.fitting_fn = fitting_fn
        self.cutoff_values = list(cutoff_values)

    @abstractmethod
    def truncator_cls(self) -> type:
        """The truncator class whose slot in the pipeline is swept."""

    @abstractmethod
    def build_truncator(self, cutoff):
        """A truncator carrying `cutoff` (None = no cutoff)."""

    def _set_cutoff(self, propagator, cutoff) -> None:
        """Replaces the matching truncator of the propagator's pipeline
        (propaq/extrapolators/zce.py:74-88); ValueError if it has none."""
        propagator.set_truncation(self._pipeline(propagator.truncators, cutoff))

    def _pipeline(self, truncators, cutoff):
        truncators = list(truncators)
        idx = next((i for i, t in enumerate(truncators) if isinstance(t, self.truncator_cls())), None)
        if idx is None:
            raise ValueError("Propagator has no truncation policy for this cutoff.")
        truncators[idx] = self.build_truncator(cutoff)
        return truncators

    def run(self, propagator, observable, circuit, initial_state=0, **curve_fit_kwargs) -> ZCEResult:
        """Sweeps the cutoff values (one batch), fits, and extrapolates to zero.
        `propagator` keeps its own truncation pipeline."""
        base = propagator.truncators
        props = [_like(propagator, propagator.noise, self._pipeline(base, c)) for c in self.cutoff_values]
        values = _sweep(props, observable, circuit, initial_state, propagator.device)
        popt, pcov = curve_fit(self.fitting_fn, self.cutoff_values, values, **curve_fit_kwargs)
        return ZCEResult(zero_cutoff_value=float(self.fitting_fn(0.0, *popt)), cutoff_values=self.cutoff_values,
                         expectation_values=values, fit_params=popt, fit_covariance=pcov)


class WeightCutoffExtrapolator(ZeroCutoffExtrapolator):
    """Sweeps the `WeightTruncator` of the pipeline."""

    def truncator_cls(self) -> type:
        return WeightTruncator

    def build_truncator(self, cutoff):
        return WeightTruncator(int(cutoff) if cutoff is not None else None)


class CoefficientCutoffExtrapolator(ZeroCutoffExtrapolator):
    """Sweeps the `CoefficientTruncator` of the pipeline."""

    def truncator_cls(self) -> type:
        return CoefficientTruncator

    def build_truncator(self, cutoff):
        return CoefficientTruncator(float(cutoff) if cutoff is not None else None)


__all__ = ["ZeroNoiseExtrapolator", "ZNEResult", "ZeroCutoffExtrapolator", "ZCEResult", "WeightCutoffExtrapolator",
           "CoefficientCutoffExtrapolator"]
