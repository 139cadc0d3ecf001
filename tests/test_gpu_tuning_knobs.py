"""The tuning knobs (pq_run_config::fuse_max, tile_items, bucket_slots) change
how the engine runs, never what it computes: every setting gives the oracle's
per-gate live counts, term set, coefficients (bit for bit),
terms_below_cutoff and expectation value.

Cases: layers of pairwise commuting rotations (X0X1, Z0Z1, X2X3, Z2Z3) that
fused pairs take whole families of four members from (rows such as Y0Y2
anticommute with all of them); random circuits; a kicked Ising run whose live
set outgrows one tile per block on a one-block-per-SM grid (the many-row gate
tiles); and a Majorana run.  Bad values are refused."""

from __future__ import annotations

import itertools

import numpy as np
import pytest
from harness import (assert_terms_equal, expectation_close, from_circuit, from_workload, make_cfg,
                     random_pauli_problem, run_oracle)

from propaq_b200 import workloads
from propaq_b200.circuits import PauliCircuit, PauliRotation
from propaq_b200.datatypes import PauliString, PauliTermSum

pytestmark = pytest.mark.gpu

SETTINGS = [dict(fuse_max=f, tile_items=t, bucket_slots=b)
            for f, t, b in [(1, 0, 0), (2, 0, 0), (0, 1, 2), (0, 2, 8), (1, 3, 4), (2, 4, 8), (2, 1, 8)]]


def run_with(engine, p, blocks_per_sm=0, **knobs):
    cfg, keep = make_cfg(p)
    cfg.blocks_per_sm = blocks_per_sm
    for k, v in knobs.items():
        setattr(cfg, k, v)
    res, nt = engine.run(cfg, p.obs_keys, p.obs_coeffs, p.gate_keys, p.angles, p.offsets, p.diag)
    keys, coeffs = engine.terms(p.n_words)
    return res, nt, keys, coeffs


def check_all(engine, oracle, p, settings=SETTINGS, blocks_per_sm=0):
    o = run_oracle(oracle, p)
    for knobs in settings:
        res, nt, keys, coeffs = run_with(engine, p, blocks_per_sm, **knobs)
        assert np.array_equal(nt, o.n_terms), f"per-gate live counts differ with {knobs}"
        assert int(res.terms_below_cutoff) == o.terms_below_cutoff, knobs
        assert_terms_equal(keys, coeffs, o.keys, o.coeffs)
        assert expectation_close(res.expectation_value, o)[0], knobs


def pauli(n, **ops):
    x = z = 0
    for q, t in ops.items():
        q = int(q[1:])
        if t in "XY":
            x |= 1 << q
        if t in "ZY":
            z |= 1 << q
    return PauliString(x, z, n)


def test_commuting_layers(gpu_engine, oracle):
    n = 8
    rng = np.random.default_rng(5)
    layers = []
    for rep in range(6):
        base = 2 * (rep % 3)
        gens = [pauli(n, **{f"q{base}": "X", f"q{base + 1}": "X"}), pauli(n, **{f"q{base}": "Z", f"q{base + 1}": "Z"}),
                pauli(n, **{f"q{base + 2}": "X", f"q{base + 3}": "X"}),
                pauli(n, **{f"q{base + 2}": "Z", f"q{base + 3}": "Z"})]
        layers.append([PauliRotation(g, float(rng.uniform(-1.2, 1.2))) for g in gens])
        layers.append([PauliRotation(pauli(n, **{f"q{q}": "Y"}), float(rng.uniform(-1.0, 1.0))) for q in range(0, n, 3)])
    obs = PauliTermSum()
    for q0, q1 in itertools.combinations(range(0, 6, 2), 2):
        obs.add(pauli(n, **{f"q{q0}": "Y", f"q{q1}": "Y"}), float(rng.normal()))
    obs.add(pauli(n, q0="Z", q2="X"), 0.7)
    for wcut, ccut in [(None, None), (6, 1e-6), (4, 1e-3)]:
        p = from_circuit(0, n, obs, PauliCircuit(layers), 0b10110010, max_weight=wcut, min_coeff=ccut)
        check_all(gpu_engine, oracle, p)


@pytest.mark.parametrize("seed", range(4))
def test_random_circuits(gpu_engine, oracle, seed):
    n = [20, 48, 90, 130][seed]
    p = random_pauli_problem(seed + 40, n, n_gates=80, layer_size=6, clifford_frac=0.1, max_weight=6,
                             min_coeff=1e-5 if seed % 2 else None)
    check_all(gpu_engine, oracle, p)


def test_many_row_tiles(gpu_engine, oracle):
    # one block per SM: 148 x 256 rows fit one tile per block, the run grows
    # well past that, so the gate ops switch to the ticketed many-row tiles
    p = from_workload(workloads.kicked_ising(8, 8, 10))
    res = run_with(gpu_engine, p, blocks_per_sm=1)[0]
    assert int(res.peak_terms) > 148 * 256 * 2
    check_all(gpu_engine, oracle, p, settings=[dict(tile_items=t, bucket_slots=b) for t, b in
                                                [(1, 4), (2, 2), (3, 8), (4, 4)]], blocks_per_sm=1)


def test_majorana(gpu_engine, oracle):
    p = from_workload(workloads.majorana_givens(10, 2))
    check_all(gpu_engine, oracle, p, settings=SETTINGS[:2] + [dict(tile_items=1, bucket_slots=8)])


def test_bad_values_are_refused(gpu_engine):
    p = from_workload(workloads.tfim_chain(8, 2))
    for knobs in (dict(fuse_max=3), dict(tile_items=9), dict(bucket_slots=3), dict(bucket_slots=1)):
        with pytest.raises(ValueError):
            run_with(gpu_engine, p, **knobs)
    run_with(gpu_engine, p)  # the engine answers afterwards
