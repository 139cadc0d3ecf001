"""Known-answer cases of crates/core/tests/unit/engine/termsum.rs restated on
Pauli keys, plus an independent dense-statevector check of the oracle."""

import math

import numpy as np
import pytest
from harness import from_circuit, run_oracle

from propaq_b200.circuits import PauliCircuit, PauliRotation
from propaq_b200.datatypes import PauliString, PauliTermSum

N = 4


def ps(x, z):
    return PauliString(x, z, N)


def run(oracle, terms, rots, layered=False, initial_state=0, **kw):
    obs = PauliTermSum()
    for t, c in terms:
        obs.add(t, c)
    circ = PauliCircuit([[r] for r in rots] if layered else [PauliRotation(g, a) for g, a in rots])
    p = from_circuit(0, N, obs, circ, initial_state, **kw)
    r = run_oracle(oracle, p)
    vals = {PauliString.from_key(int(k[0]), N): c for k, c in zip(r.keys, r.coeffs)}
    return r, vals


X0, Y0, Z0, Z1 = ps(1, 0), ps(1, 1), ps(0, 1), ps(0, 2)


def test_cos_sin_split(oracle):
    # termsum.rs:78-93: an anticommuting term splits into cos and sin branches.
    r, v = run(oracle, [(X0, 2.0)], [(Z0, 0.3)])
    assert len(v) == 2
    assert v[X0] == 2.0 * math.cos(0.3)
    assert v[Y0] == (2.0 * math.sin(0.3)) * -1.0  # Z.X = iY -> -(Im i) = -1


def test_commuting_term_untouched(oracle):
    r, v = run(oracle, [(Z1, 5.0)], [(Z0, 0.7)])
    assert v == {Z1: 5.0}


def test_sin_taken_from_pre_rotation_coefficient(oracle):
    # termsum.rs:117-140
    a, c0, c1 = 0.4, 2.0, 5.0
    r, v = run(oracle, [(X0, c0), (Y0, c1)], [(Z0, a)])
    s, c = math.sin(a), math.cos(a)
    assert v[X0] == c0 * c + (c1 * s) * 1.0
    assert v[Y0] == c1 * c + (c0 * s) * -1.0


def test_phase_only_rotation(oracle):
    # termsum.rs:143-158
    r, v = run(oracle, [(X0, 2.0), (Z1, 3.0)], [(Z0, math.pi)])
    assert len(v) == 2 and abs(v[X0] + 2.0) < 1e-12 and v[Z1] == 3.0


def test_weight_cutoff_at_emit(oracle):
    # termsum.rs:161-173: the over-weight child is never created.
    xx = ps(0b011, 0)
    r, v = run(oracle, [(xx, 1.0)], [(PauliString(0b100, 0b001, N), 0.3)], max_weight=2)
    assert len(v) == 1


# The driver admits observable terms only with |c| >= min_coeff
# (crates/pauli/src/engine.rs:104-111), so the tiny branches below come from a
# small angle rather than a tiny coefficient.
TINY = 1e-3


def test_coefficient_cutoff_at_emit(oracle):
    # termsum.rs:176-188: the tiny child is never created.
    r, v = run(oracle, [(X0, 1e-5)], [(Z0, TINY)], min_coeff=1e-6)
    assert len(v) == 1


def test_pair_rescue(oracle):
    # termsum.rs:191-216: the partner pays for the held-back branch.
    big, small = 1.0, 1e-5
    r, v = run(oracle, [(X0, big), (Y0, small)], [(Z0, TINY)], min_coeff=1e-6)
    s, c = math.sin(TINY), math.cos(TINY)
    assert len(v) == 2
    assert v[X0] == big * c + small * s
    assert v[Y0] == small * c - big * s


def test_pair_rescue_needs_one_earning_half(oracle):
    # termsum.rs:285-302
    r, v = run(oracle, [(X0, 1e-5), (Y0, 2e-5)], [(Z0, TINY)], min_coeff=1e-6)
    assert v[X0] == 1e-5 * math.cos(TINY) and v[Y0] == 2e-5 * math.cos(TINY)


def test_lone_tiny_term_makes_no_child(oracle):
    # termsum.rs:305-317
    r, v = run(oracle, [(X0, 1e-5)], [(Z0, TINY)], min_coeff=1e-6)
    assert len(v) == 1


def test_term_budget_floor(oracle):
    # termsum.rs:219-269: below the floor the tiny branch survives.
    r, v = run(oracle, [(X0, 1e-5)], [(Z0, TINY)], min_coeff=1e-6, min_terms=1000)
    assert len(v) == 2
    r, v = run(oracle, [(X0, 1e-5)], [(Z0, TINY)], min_coeff=1e-6, min_terms=1)
    assert len(v) == 1


def test_repeated_rotations_stay_deduplicated(oracle):
    # termsum.rs:320-329
    r, v = run(oracle, [(X0, 1.0)], [(Z0, 0.3)] * 12)
    assert len(v) == 2


def test_expectation_sums_coeff_times_trace(oracle):
    r, _ = run(oracle, [(Z0, 2.0), (Z1, 3.0)], [], initial_state=0b01)
    assert r.expectation == -2.0 + 3.0


def test_clifford_rotation_is_deferred(oracle):
    # A |cos| < 1e-9 rotation goes into the frame: no branching, the image is
    # applied at readout.  exp(-i pi/4 Z) maps X -> -Y under conjugation.
    r, v = run(oracle, [(X0, 1.0)], [(Z0, math.pi / 2)])
    assert list(r.n_terms) == [1]
    assert v == {Y0: -1.0}


def test_clifford_changing_weight_not_deferred_with_weight_cut(oracle):
    # Z0 X1 (-pi/2) changes weight: with a weight cutoff it runs the normal
    # branch path and leaves the cos remnant.
    g = PauliString(0b10, 0b01, N)
    r, v = run(oracle, [(X0, 1.0)], [(g, -math.pi / 2)], max_weight=4)
    assert list(r.n_terms) == [2]
    r, v = run(oracle, [(X0, 1.0)], [(g, -math.pi / 2)])
    assert list(r.n_terms) == [1]


# ---------------------------------------------------------- statevector check
def _pauli_matrix(p: PauliString):
    I = np.eye(2)
    X = np.array([[0, 1], [1, 0]], complex)
    Z = np.array([[1, 0], [0, -1]], complex)
    Y = np.array([[0, -1j], [1j, 0]])
    m = np.array([[1.0]], complex)
    for q in reversed(range(p.n_qubits)):
        x, z = p.x >> q & 1, p.z >> q & 1
        m = np.kron(m, [I, X, Z, Y][x | (z << 1)])
    return m


@pytest.mark.parametrize("seed", range(6))
def test_oracle_matches_dense_statevector(oracle, seed):
    rng = np.random.default_rng(seed)
    n = 4
    rots = []
    for _ in range(25):
        x, z = int(rng.integers(0, 16)), int(rng.integers(0, 16))
        if x == 0 and z == 0:
            z = 1
        rots.append((PauliString(x, z, n), float(rng.uniform(-1.5, 1.5))))
    obs_terms = [(PauliString(0, 1, n), 1.0), (PauliString(0, 0b0110, n), -0.5)]
    state = int(rng.integers(0, 16))
    r, _ = run(oracle, obs_terms, rots, initial_state=state)
    psi = np.zeros(2**n, complex)
    psi[state] = 1.0
    for g, a in rots:
        m = _pauli_matrix(g)
        u = np.cos(a / 2) * np.eye(2**n) - 1j * np.sin(a / 2) * m
        psi = u @ psi
    o = sum(c * _pauli_matrix(t) for t, c in obs_terms)
    want = float(np.real(np.conj(psi) @ o @ psi))
    assert abs(r.expectation - want) < 1e-10
