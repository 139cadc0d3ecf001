"""The reference's extrapolator behaviour tests, restated against this package
(tests/extrapolators/test_zne.py:24-160 and tests/extrapolators/test_zce.py:
25-185 of hkbelagali/propaq): the same 8-mode one-gate Majorana problem, the
same sweeps and fits, result shapes, the propagator's noise and truncation
restored (None included), the exponential fit with p0, a custom noise model
swept through build_noise, and _set_cutoff refusing a propagator with no
matching truncator."""

from __future__ import annotations

import math

import numpy as np
import pytest

from propaq_b200 import MajoranaMonomial, MajoranaPropagator, MajoranaTermSum, TruncationPolicy
from propaq_b200.circuits import MajoranaCircuit, MajoranaRotation
from propaq_b200.extrapolators import (
    CoefficientCutoffExtrapolator,
    WeightCutoffExtrapolator,
    ZCEResult,
    ZeroNoiseExtrapolator,
    ZNEResult,
)
from propaq_b200.noise import GateNoiseModel, UniformNoiseModel

N = 8


def mon(modes_int):
    return MajoranaMonomial(modes_int, N)


def one_gate_circuit():
    return MajoranaCircuit([MajoranaRotation(mon(0b11), 0.0)], N)


def trunc(weight_cutoff=None, coeff_cutoff=0.0):
    return TruncationPolicy(weight_cutoff=weight_cutoff, coeff_cutoff=coeff_cutoff)


# ------------------------------------------------------------ host side only
def test_noise_getter_setter_roundtrip():
    prop = MajoranaPropagator()
    assert prop.noise is None
    prop.set_noise(UniformNoiseModel(0.05))
    assert prop.noise is not None
    prop = MajoranaPropagator(noise=UniformNoiseModel(0.1))
    prop.set_noise(None)
    assert prop.noise is None


def test_truncation_getter_setter_roundtrip():
    prop = MajoranaPropagator()
    assert prop.truncators == []
    prop.set_truncation(trunc(weight_cutoff=4))
    assert prop.truncators[0].weight == 4
    prop = MajoranaPropagator(truncation=trunc(coeff_cutoff=0.01))
    prop.set_truncation(None)
    assert prop.truncators == []


def test_build_noise_default_returns_uniform_noise_model():
    built = ZeroNoiseExtrapolator(lambda x, a, b: a + b * x, [0.01, 0.02]).build_noise(0.05)
    assert isinstance(built, UniformNoiseModel) and built.damping == 0.05


def test_set_cutoff_raises_when_no_truncation():
    prop = MajoranaPropagator()
    with pytest.raises(ValueError, match="no truncation policy"):
        CoefficientCutoffExtrapolator(lambda e, a, b: a + b * e, [0.01, 0.02])._set_cutoff(prop, 0.01)
    with pytest.raises(ValueError, match="no truncation policy"):
        WeightCutoffExtrapolator(lambda w, a, b: a + b / (w + 1), [3, 4, 5])._set_cutoff(prop, 3)


# ------------------------------------------------------------------- on GPU
@pytest.mark.gpu
def test_zne_result_fields(gpu_engine):
    obs = MajoranaTermSum({mon(0b11): 1.0})
    res = ZeroNoiseExtrapolator(lambda x, a, b: a + b * x, [0.01, 0.02, 0.03]).run(
        MajoranaPropagator(), obs, one_gate_circuit(), initial_state=0)
    assert isinstance(res, ZNEResult)
    assert len(res.noise_values) == 3 and len(res.expectation_values) == 3
    assert res.fit_params.shape == (2,) and res.fit_covariance.shape == (2, 2)


@pytest.mark.gpu
def test_zne_linear_and_exponential_fits_close_to_noiseless(gpu_engine):
    obs = MajoranaTermSum({mon(0b11): 1.0})
    prop = MajoranaPropagator()
    noiseless = prop.expectation_value(obs, one_gate_circuit(), initial_state=0).expectation_value
    lin = ZeroNoiseExtrapolator(lambda x, a, b: a + b * x, [0.01, 0.02, 0.03, 0.04]).run(
        prop, obs, one_gate_circuit(), initial_state=0)
    assert lin.zero_noise_value == pytest.approx(noiseless, abs=0.05)
    exp = ZeroNoiseExtrapolator(lambda x, a, b: a * np.exp(-b * x), [0.01, 0.02, 0.03, 0.04]).run(
        prop, obs, one_gate_circuit(), initial_state=0, p0=[-1.0, 2.0])
    assert exp.zero_noise_value == pytest.approx(noiseless, abs=1e-4)


@pytest.mark.gpu
def test_zne_restores_original_noise(gpu_engine):
    obs = MajoranaTermSum({mon(0b11): 1.0})
    prop = MajoranaPropagator()
    ZeroNoiseExtrapolator(lambda x, a, b: a + b * x, [0.01, 0.02]).run(prop, obs, one_gate_circuit())
    assert prop.noise is None
    prop = MajoranaPropagator(noise=UniformNoiseModel(0.005))
    ZeroNoiseExtrapolator(lambda x, a, b: a + b * x, [0.01, 0.02]).run(prop, obs, one_gate_circuit())
    assert prop.noise is not None and prop.noise.damping == 0.005


class StretchedExponentialNoise(GateNoiseModel):
    """A custom Python noise model with a fixed beta, swept on gamma."""

    def __init__(self, gamma: float, beta: float) -> None:
        self.gamma = gamma
        self.beta = beta

    def damping_factor(self, term_weight, active_modes):
        return math.exp(-((self.gamma * term_weight) ** self.beta))


@pytest.mark.gpu
def test_custom_noise_subclass_sweeps_a_custom_model(gpu_engine):
    seen = []

    class StretchedExponentialExtrapolator(ZeroNoiseExtrapolator):
        def build_noise(self, value):
            seen.append(value)
            return StretchedExponentialNoise(gamma=value, beta=0.8)

    obs = MajoranaTermSum({mon(0b11): 1.0})
    prop = MajoranaPropagator()
    noiseless = prop.expectation_value(obs, one_gate_circuit(), initial_state=0).expectation_value
    res = StretchedExponentialExtrapolator(lambda x, a, b: a + b * x, [0.01, 0.02, 0.03, 0.04]).run(
        prop, obs, one_gate_circuit(), initial_state=0)
    assert seen == [0.01, 0.02, 0.03, 0.04]
    assert res.zero_noise_value == pytest.approx(noiseless, abs=0.05)
    assert prop.noise is None


@pytest.mark.gpu
def test_zce_result_fields(gpu_engine):
    obs = MajoranaTermSum({mon(0b11): 1.0})
    res = CoefficientCutoffExtrapolator(lambda e, a, b: a + b * e, [0.001, 0.002, 0.003]).run(
        MajoranaPropagator(truncation=trunc(coeff_cutoff=0.001)), obs, one_gate_circuit(), initial_state=0)
    assert isinstance(res, ZCEResult)
    assert len(res.cutoff_values) == 3 and len(res.expectation_values) == 3
    assert res.fit_params.shape == (2,) and res.fit_covariance.shape == (2, 2)
    res = WeightCutoffExtrapolator(lambda w, a, b: a + b / (w + 1), [2, 3, 4]).run(
        MajoranaPropagator(truncation=trunc(weight_cutoff=4)), obs, one_gate_circuit(), initial_state=0)
    assert res.fit_params.shape == (2,) and res.fit_covariance.shape == (2, 2)


@pytest.mark.gpu
def test_zce_coeff_linear_extrapolation_close_to_reference(gpu_engine):
    obs = MajoranaTermSum({mon(0b11): 1.0})
    exact = MajoranaPropagator(truncation=trunc(coeff_cutoff=0.0)).expectation_value(
        obs, one_gate_circuit(), initial_state=0).expectation_value
    res = CoefficientCutoffExtrapolator(lambda e, a, b: a + b * e, [0.001, 0.002, 0.003, 0.004]).run(
        MajoranaPropagator(truncation=trunc(coeff_cutoff=0.001)), obs, one_gate_circuit(), initial_state=0)
    assert res.zero_cutoff_value == pytest.approx(exact, abs=1e-4)


@pytest.mark.gpu
def test_zce_truncation_changes_and_converges(gpu_engine):
    obs = MajoranaTermSum({mon(0b11): 1.0, mon(0b1111): 0.05})
    ev = lambda t: MajoranaPropagator(truncation=t).expectation_value(  # noqa: E731
        obs, one_gate_circuit(), initial_state=0).expectation_value
    assert ev(trunc(coeff_cutoff=0.0)) != pytest.approx(ev(trunc(coeff_cutoff=0.06)), abs=1e-10)
    obs = MajoranaTermSum({mon(0b11): 1.0, mon(0b1111): 0.5})
    ev = lambda t: MajoranaPropagator(truncation=t).expectation_value(  # noqa: E731
        obs, one_gate_circuit(), initial_state=0).expectation_value
    ref = ev(trunc(weight_cutoff=None))
    errors = [abs(ev(trunc(weight_cutoff=w)) - ref) for w in (2, 3, 4, 5)]
    assert all(errors[i] >= errors[i + 1] for i in range(len(errors) - 1))


@pytest.mark.gpu
def test_zce_restores_original_truncation(gpu_engine):
    obs = MajoranaTermSum({mon(0b11): 1.0})
    prop = MajoranaPropagator(truncation=trunc(coeff_cutoff=0.001))
    CoefficientCutoffExtrapolator(lambda e, a, b: a + b * e, [0.002, 0.004]).run(prop, obs, one_gate_circuit())
    assert prop.truncators[0].coefficient == pytest.approx(0.001)
    prop = MajoranaPropagator(truncation=trunc(weight_cutoff=6))
    WeightCutoffExtrapolator(lambda w, a, b: a + b / (w + 1), [3, 4, 5]).run(prop, obs, one_gate_circuit())
    assert prop.truncators[0].weight == 6
    prop = MajoranaPropagator(truncation=trunc(coeff_cutoff=0.001))
    ext = CoefficientCutoffExtrapolator(lambda e, a, b: a + b * e, [0.002, 0.004])
    ext.run(prop, obs, one_gate_circuit())
    prop.set_truncation(None)
    with pytest.raises(ValueError):
        ext.run(prop, obs, one_gate_circuit())
    assert prop.truncators == []
