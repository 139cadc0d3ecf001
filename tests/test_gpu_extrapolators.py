"""Zero-noise / zero-cutoff extrapolation over batched propagation: the sweep
values equal one expectation_value call per value, the fit is scipy's, and
the propagator keeps its own noise and truncation."""

import math

import numpy as np
import pytest

import propaq_b200 as pq
from propaq_b200 import workloads
from propaq_b200.extrapolators import (
    CoefficientCutoffExtrapolator,
    WeightCutoffExtrapolator,
    ZeroNoiseExtrapolator,
)

pytestmark = pytest.mark.gpu


def linear(x, a, b):
    return a + b * x


def close(x, y):
    return abs(x - y) <= 1e-12 * max(1.0, abs(y))


def test_zero_noise_extrapolation_matches_sequential_calls(gpu_engine):
    wl = workloads.kicked_ising(4, 5, 3)
    prop = pq.PauliPropagator(noise=pq.UniformNoiseModel(0.5), truncation=wl.truncation())
    zne = ZeroNoiseExtrapolator(linear, [1e-3, 2e-3, 4e-3])
    res = zne.run(prop, wl.observable, wl.circuit, 0)
    for v, e in zip(res.noise_values, res.expectation_values):
        want = pq.PauliPropagator(noise=pq.UniformNoiseModel(v), truncation=wl.truncation()).expectation_value(
            wl.observable, wl.circuit, 0).expectation_value
        assert close(e, want)
    assert close(res.zero_noise_value, linear(0.0, *res.fit_params))
    assert prop.noise.damping == 0.5  # restored / untouched


def test_zero_cutoff_extrapolation(gpu_engine):
    wl = workloads.tfim_chain(14, 4)
    prop = pq.PauliPropagator(truncation=[pq.WeightTruncator(8), pq.CoefficientTruncator(1e-4)])
    zce = CoefficientCutoffExtrapolator(linear, [1e-2, 3e-3, 1e-3])
    res = zce.run(prop, wl.observable, wl.circuit, 0)
    for c, e in zip(res.cutoff_values, res.expectation_values):
        p = pq.PauliPropagator(truncation=[pq.WeightTruncator(8), pq.CoefficientTruncator(c)])
        assert close(e, p.expectation_value(wl.observable, wl.circuit, 0).expectation_value)
    wce = WeightCutoffExtrapolator(linear, [3, 4, 6])
    res_w = wce.run(prop, wl.observable, wl.circuit, 0)
    assert len(res_w.expectation_values) == 3
    assert [type(t).__name__ for t in prop.truncators] == ["WeightTruncator", "CoefficientTruncator"]
    assert prop.truncators[1].coefficient == 1e-4


def test_sweep_falls_back_to_one_call_per_value(gpu_engine):
    # A TermBudget floor with a weight cut over weight-changing Clifford
    # rotations is refused by the batch; the sweep runs call by call instead.
    wl = workloads.kicked_ising(4, 4, 2)
    prop = pq.PauliPropagator(truncation=[pq.WeightTruncator(6), pq.TermBudget(50)])
    res = ZeroNoiseExtrapolator(linear, [1e-3, 3e-3]).run(prop, wl.observable, wl.circuit, 0)
    want = [pq.PauliPropagator(noise=pq.UniformNoiseModel(v), truncation=[pq.WeightTruncator(6), pq.TermBudget(50)])
            .expectation_value(wl.observable, wl.circuit, 0).expectation_value for v in (1e-3, 3e-3)]
    assert res.expectation_values == want
    assert math.isfinite(res.zero_noise_value)
