"""Batched propagation (pq_run_batch): many independent instances sharing one
persistent grid.  Every instance must give what pq_run gives on the same
arguments -- the same live counts per gate, the same terms with bit-identical
coefficients, the expectation value to its last bit or so -- whatever the grid
split, the rebalancing, the key-width padding or the number of launches, and
agree with the oracle."""

import math

import numpy as np
import pytest
from harness import (
    assert_terms_equal,
    expectation_close,
    from_workload,
    run_gpu,
    run_gpu_batch,
    run_oracle,
)

import propaq_b200 as pq
from propaq_b200 import workloads
from propaq_b200.propagators import expectation_values

pytestmark = pytest.mark.gpu


def close(x, y):
    # An instance's slice of the grid decides how rows are tiled, which
    # decides the order new rows are appended in; the double-double
    # expectation sum then agrees to its last bit or so.
    return abs(x - y) <= 1e-13 * max(1.0, abs(y))


def assert_same(batch_res, single_res):
    assert np.array_equal(batch_res.n_terms, single_res.n_terms), "live counts per gate differ"
    assert_terms_equal(batch_res.keys, batch_res.coeffs, single_res.keys, single_res.coeffs)
    assert batch_res.terms_below_cutoff == single_res.terms_below_cutoff
    assert close(batch_res.expectation, single_res.expectation)


def mixed_problems():
    """Instances of 1-, 2- and 4-word keys, with and without noise and cuts."""
    wls = [
        workloads.kicked_ising(4, 4, 3),                       # 16 qubits, W=1
        workloads.kicked_ising(5, 8, 4, theta=0.8),            # 40 qubits, W=2
        workloads.kicked_ising(6, 10, 3, p=2e-3, min_coeff=1e-4),  # 60 qubits, W=2
        workloads.kicked_ising(7, 10, 3, theta=0.3),           # 70 qubits, W=4
        workloads.tfim_chain(20, 4),                           # W=1, no noise
        workloads.kicked_ising(10, 10, 2, p=0.0),              # 100 qubits, W=4, no noise
    ]
    return [from_workload(w) for w in wls]


def test_batch_matches_single_runs_and_oracle(gpu_engine, oracle):
    probs = mixed_problems()
    batch = run_gpu_batch(gpu_engine, probs)
    for p, b in zip(probs, batch):
        s = run_gpu(gpu_engine, p)
        assert_same(b, s)
        o = run_oracle(oracle, p)
        assert np.array_equal(b.n_terms, o.n_terms)
        assert_terms_equal(b.keys, b.coeffs, o.keys, o.coeffs)
        ok, err, tol = expectation_close(b.expectation, o)
        assert ok, f"{p.name}: {b.expectation!r} vs oracle {o.expectation_accurate!r}"


@pytest.mark.parametrize("tuning", [
    dict(split=0, rebalance_pct=0),
    dict(split=1, rebalance_pct=0),
    dict(split=1, rebalance_pct=1),
    dict(split=0, rebalance_pct=100),
    dict(blocks_per_sm=1, split=1, rebalance_pct=25),
], ids=lambda t: ",".join(f"{k}={v}" for k, v in t.items()))
def test_batch_results_do_not_depend_on_grid_sharing(gpu_engine, tuning):
    probs = mixed_problems()
    ref = [run_gpu(gpu_engine, p) for p in probs]
    for b, s in zip(run_gpu_batch(gpu_engine, probs, **tuning), ref):
        assert_same(b, s)


def test_batch_capacity_growth_inside_a_batch(gpu_engine):
    # The 8x8 instance outgrows the initial 64 Ki rows while the small ones run
    # beside it; it is grown and resumed in a later launch.
    probs = [from_workload(workloads.kicked_ising(8, 8, 10))] + mixed_problems()[:3]
    batch = run_gpu_batch(gpu_engine, probs, rebalance_pct=0)
    assert batch[0].res.peak_terms > 32768
    assert batch[0].res.sweep_launches >= 2
    for p, b in zip(probs, batch):
        assert_same(b, run_gpu(gpu_engine, p))


def test_batch_more_instances_than_blocks(gpu_engine):
    # 1 block per SM gives a grid smaller than the batch: instances wait for a
    # later launch.
    probs = [from_workload(workloads.tfim_chain(12, 2 + i % 3, seed=i)) for i in range(200)]
    batch = run_gpu_batch(gpu_engine, probs, blocks_per_sm=1)
    for i in (0, 1, 2, 147, 148, 149, 199):
        assert_same(batch[i], run_gpu(gpu_engine, probs[i]))


def test_batch_majorana(gpu_engine, oracle):
    probs = [from_workload(workloads.majorana_givens(n_sites=n, reps=2, seed=s))
             for n, s in ((8, 0), (12, 1), (16, 2), (40, 3))]  # W = 1, 1, 1, 2
    batch = run_gpu_batch(gpu_engine, probs)
    for p, b in zip(probs, batch):
        assert_same(b, run_gpu(gpu_engine, p))
        ok, _, _ = expectation_close(b.expectation, run_oracle(oracle, p))
        assert ok


def test_config_batch_reduced(gpu_engine, oracle):
    # The extrapolation sweep's instance grid (4 noise scales x 4 cutoffs x 4
    # sites) on smaller lattices and fewer steps, so the oracle keeps up.
    wls = workloads.kicked_ising_batch(64, seed=1, n_range=(16, 72), steps_range=(2, 4))
    probs = [from_workload(w) for w in wls]
    batch = run_gpu_batch(gpu_engine, probs, want_terms=False)
    for p, b in zip(probs, batch):
        o = run_oracle(oracle, p, want_terms=False)
        assert np.array_equal(b.n_terms, o.n_terms), p.name
        ok, err, tol = expectation_close(b.expectation, o)
        assert ok, f"{p.name}: {b.expectation!r} vs oracle {o.expectation_accurate!r}"


def test_expectation_values_api(gpu_engine):
    wl = workloads.kicked_ising(5, 6, 4)
    jobs, singles = [], []
    for p in (0.5e-3, 1e-3, 2e-3):
        for cut in (1e-3, 1e-5):
            prop = pq.PauliPropagator(noise=pq.UniformNoiseModel(-math.log1p(-p)),
                                      truncation=[pq.WeightTruncator(10), pq.CoefficientTruncator(cut)])
            jobs.append((prop, wl.observable, wl.circuit, 0))
            singles.append(prop.expectation_value(wl.observable, wl.circuit, 0))
    for r, s in zip(expectation_values(jobs), singles):
        assert close(r.expectation_value, s.expectation_value)
        assert r.n_terms == s.n_terms
        assert r.terms_below_cutoff == s.terms_below_cutoff


def test_autotuned_batch(gpu_engine):
    # The autotuner runs the batch once per candidate setting and keeps the
    # fastest; any setting gives every instance its pq_run result, and the
    # propagator-level call with autotune=True reuses the remembered choice.
    from harness import make_cfg

    from propaq_b200.tuning import CANDIDATES, KERNEL_DEFAULTS, KERNEL_DIMENSIONS, BatchTuner, batch_signature

    probs = mixed_problems()[:4]
    items, keep = [], []
    for p in probs:
        cfg, k = make_cfg(p, want_terms=False)
        keep.append(k)
        items.append((cfg, p.obs_keys, p.obs_coeffs, p.gate_keys, p.angles, p.offsets, p.diag))
    tuner = BatchTuner()
    t = tuner.tune(items)
    assert (t.blocks_per_sm, t.split, t.rebalance_pct) in CANDIDATES
    n_kernel = sum(len([v for v in vals if v != KERNEL_DEFAULTS[d]]) for d, vals in KERNEL_DIMENSIONS.items())
    assert len(tuner.trials[batch_signature(items)]) == len(CANDIDATES) + n_kernel
    for b, p in zip(run_gpu_batch(gpu_engine, probs, **t.as_dict()), probs):
        assert_same(b, run_gpu(gpu_engine, p))
    wl = workloads.kicked_ising(5, 6, 4)
    jobs = [(pq.PauliPropagator(noise=pq.UniformNoiseModel(d), truncation=wl.truncation()), wl.observable, wl.circuit, 0)
            for d in (1e-3, 2e-3)]
    for r, (prop, o, c, s) in zip(expectation_values(jobs, autotune=True), jobs):
        single = prop.expectation_value(o, c, s)
        assert close(r.expectation_value, single.expectation_value)
        assert r.n_terms == single.n_terms


def test_batch_refusals(gpu_engine):
    wl = workloads.kicked_ising(4, 4, 2)
    maj = workloads.majorana_givens(n_sites=8, reps=1)
    with pytest.raises(ValueError, match="mixes Pauli and Majorana"):
        expectation_values([(pq.PauliPropagator(), wl.observable, wl.circuit, 0),
                            (pq.MajoranaPropagator(), maj.observable, maj.circuit, 0)])
    # RZZ(-pi/2) changes weight: with a TermBudget floor and a weight cut the
    # deferral decision needs the live count mid-run.
    budget = pq.PauliPropagator(truncation=[pq.WeightTruncator(4), pq.TermBudget(10)])
    with pytest.raises(NotImplementedError, match="run that instance with pq_run"):
        expectation_values([(budget, wl.observable, wl.circuit, 0)])
    assert expectation_values([]) == []
