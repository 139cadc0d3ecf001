"""Host-side behaviour of the extrapolators (no GPU needed)."""

import pytest

import propaq_b200 as pq
from propaq_b200 import workloads
from propaq_b200.extrapolators import CoefficientCutoffExtrapolator, WeightCutoffExtrapolator


def test_cutoff_sweep_needs_the_truncator_in_the_pipeline():
    wl = workloads.tfim_chain(6, 2)
    prop = pq.PauliPropagator(truncation=[pq.CoefficientTruncator(1e-3)])
    with pytest.raises(ValueError, match="no truncation policy"):
        WeightCutoffExtrapolator(lambda x, a: a, [1, 2]).run(prop, wl.observable, wl.circuit)


def test_build_truncator_values():
    assert WeightCutoffExtrapolator(None, []).build_truncator(4.0).weight == 4
    assert WeightCutoffExtrapolator(None, []).build_truncator(None).weight is None
    assert CoefficientCutoffExtrapolator(None, []).build_truncator(1e-3).coefficient == 1e-3
