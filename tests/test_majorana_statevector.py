"""Majorana propagation against an independent physics check: the Jordan-Wigner
dense statevector (the Majorana counterpart of the Pauli statevector check in
test_oracle_unit.py; the reference checks its propagators against qiskit's
Statevector, tests/propagator/test_cross_propagator.py).

A rotation exp(-i theta M / 2) of the monomial M = i^herm(l) gamma_m1...gamma_ml
is applied to the state as a dense unitary of the JW matrix of M; the
expectation <psi|O|psi> of the observable's JW matrix is compared with the
oracle's Heisenberg propagation (CPU) and with the engine's (GPU), without
truncation.  Circuits mix the gate tables of config 3 (Givens xx_plus_yy,
number-number cp), odd single-mode generators and random monomials.  The gate
tables themselves are checked against the qubit gates they stand for."""

from __future__ import annotations

import numpy as np
import pytest
import scipy.linalg as sl
from harness import from_circuit, run_gpu, run_oracle
from test_algebra_known_answers import I2, PX, PY, jw_matrix

from propaq_b200.circuits import MajoranaCircuit, MajoranaRotation, majorana_cp, majorana_xx_plus_yy
from propaq_b200.datatypes import MajoranaMonomial, MajoranaTermSum


def two_site(a, b, i, j, n):
    mats = [I2] * n
    mats[i], mats[j] = a, b
    m = np.array([[1.0 + 0j]])
    for q in reversed(range(n)):
        m = np.kron(m, mats[q])
    return m


def unitary(rots, n_sites):
    dim = 1 << n_sites
    u = np.eye(dim, dtype=complex)
    for r in rots:
        m = jw_matrix(r.generator.modes, n_sites)
        u = (np.cos(r.angle / 2) * np.eye(dim) - 1j * np.sin(r.angle / 2) * m) @ u
    return u


@pytest.mark.parametrize("i,j", [(0, 1), (1, 0), (1, 2), (0, 2)])
def test_givens_table_is_xx_plus_yy(i, j):
    # xx_plus_yy(theta, 0) = exp(-i theta/4 (XX + YY)) on the two qubits
    # (propaq/datatypes/majorana/termsum.py:19-44 under Jordan-Wigner)
    n, theta = 3, 0.7
    u = unitary(majorana_xx_plus_yy(i, j, theta, 2 * n), n)
    want = sl.expm(-0.25j * theta * (two_site(PX, PX, i, j, n) + two_site(PY, PY, i, j, n)))
    assert np.allclose(u, want)


def test_cp_table_is_controlled_phase():
    # cp(phi) = diag(1, 1, 1, e^{i phi}) on the two sites' occupations, up to
    # the global phase e^{-i phi/4} that the three rotations carry
    # (propaq/datatypes/majorana/termsum.py:57-67)
    n, phi = 3, 0.9
    u = unitary(majorana_cp(0, 2, phi, 2 * n), n)
    want = np.diag([np.exp(1j * phi) if (k & 1) and (k >> 2 & 1) else 1.0 for k in range(1 << n)])
    assert np.allclose(u, np.exp(-0.25j * phi) * want)


def random_problem(seed, n_sites=4, n_rot=30):
    """Givens, cp, odd single-mode and random-monomial rotations; an observable of
    quadratic and random monomials; a random determinant."""
    rng = np.random.default_rng(seed)
    n_modes = 2 * n_sites
    rots = []
    while len(rots) < n_rot:
        kind = rng.integers(0, 4)
        if kind == 0:
            p = int(rng.integers(0, n_sites - 1))
            q = p + 1 if rng.random() < 0.7 else int(rng.integers(p + 1, n_sites))
            rots += majorana_xx_plus_yy(p, q, float(rng.uniform(-np.pi, np.pi)), n_modes)
        elif kind == 1:
            p, q = sorted(rng.choice(n_sites, size=2, replace=False))
            rots += majorana_cp(int(p), int(q), float(rng.normal(0, 0.5)), n_modes)
        elif kind == 2:  # an odd generator: one mode
            rots.append(MajoranaRotation(MajoranaMonomial(1 << int(rng.integers(0, n_modes)), n_modes,
                                                          is_number_preserving=False),
                                         float(rng.uniform(-1.5, 1.5))))
        else:
            m = int(rng.integers(1, 1 << n_modes))
            rots.append(MajoranaRotation(MajoranaMonomial(m, n_modes, is_number_preserving=False),
                                         float(rng.uniform(-1.5, 1.5))))
    obs = MajoranaTermSum()
    for p in range(n_sites):
        obs.add(MajoranaMonomial(0b11 << (2 * p), n_modes), float(rng.normal()))
    for _ in range(3):
        obs.add(MajoranaMonomial(int(rng.integers(1, 1 << n_modes)), n_modes, is_number_preserving=False),
                float(rng.normal()))
    state = int(rng.integers(0, 1 << n_sites))
    layers = [rots[k:k + 3] for k in range(0, len(rots), 3)]
    return obs, layers, state


def dense_expectation(obs, layers, state, n_sites):
    psi = np.zeros(1 << n_sites, complex)
    psi[state] = 1.0
    psi = unitary([r for layer in layers for r in layer], n_sites) @ psi
    o = sum(c * jw_matrix(m.modes, n_sites) for m, c in obs.items())
    return float(np.real(np.conj(psi) @ o @ psi))


@pytest.mark.parametrize("seed", range(8))
def test_oracle_matches_jordan_wigner_statevector(oracle, seed):
    n = 4
    obs, layers, state = random_problem(seed, n)
    p = from_circuit(1, n, obs, MajoranaCircuit(layers), state)
    r = run_oracle(oracle, p)
    assert abs(r.expectation - dense_expectation(obs, layers, state, n)) < 1e-10


@pytest.mark.gpu
@pytest.mark.parametrize("seed", range(8))
def test_engine_matches_jordan_wigner_statevector(gpu_engine, seed):
    n = 4 if seed < 6 else 5
    obs, layers, state = random_problem(seed, n, n_rot=40)
    p = from_circuit(1, n, obs, MajoranaCircuit(layers), state)
    g = run_gpu(gpu_engine, p)
    assert abs(g.expectation - dense_expectation(obs, layers, state, n)) < 1e-10
