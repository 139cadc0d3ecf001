"""CPU checks behind the adjoint tests: the forward-mode reference against the
oracle (same expectation value) and against an exact dense-statevector
derivative (no truncation), and the angle bookkeeping of
propaq_b200.adjoint."""

import math

import numpy as np
import pytest
from adjoint_ref import propagate_with_tangents
from harness import from_circuit, run_oracle

import propaq_b200 as pq
from propaq_b200 import workloads
from propaq_b200.adjoint import ParametrizedExpectation, _heisenberg_order
from propaq_b200.circuits import PauliCircuit, PauliRotation
from propaq_b200.datatypes import PauliString, PauliTermSum
from propaq_b200.propagators import heisenberg_gates


def random_circuit(seed, n, n_gates, layer_size=4, clifford=False):
    rng = np.random.default_rng(seed)
    rots = []
    for _ in range(n_gates):
        x = z = 0
        for q in rng.choice(n, size=int(rng.integers(1, 4)), replace=False):
            t = int(rng.integers(1, 4))
            x |= (t & 1) << int(q)
            z |= (t >> 1) << int(q)
        a = float(rng.choice([math.pi / 2, -math.pi / 2])) if clifford and rng.random() < 0.2 else \
            float(rng.uniform(-1.2, 1.2))
        rots.append(PauliRotation(PauliString(x, z, n), a))
    obs = PauliTermSum()
    for _ in range(3):
        obs.add(PauliString(0, 1 << int(rng.integers(0, n)), n), float(rng.normal()))
    obs.add(PauliString(0, (1 << int(rng.integers(0, n))) | 1, n), 0.5)
    layers = [rots[k:k + layer_size] for k in range(0, len(rots), layer_size)]
    return obs, PauliCircuit(layers), int(rng.integers(0, 1 << n))


def pauli_matrix(p: PauliString):
    mats = [np.eye(2), np.array([[0, 1], [1, 0]], complex), np.diag([1.0, -1.0]).astype(complex),
            np.array([[0, -1j], [1j, 0]])]
    m = np.array([[1.0]], complex)
    for q in reversed(range(p.n_qubits)):
        m = np.kron(m, mats[(p.x >> q & 1) | ((p.z >> q & 1) << 1)])
    return m


def dense_expectation(obs, circuit, state, n, angles=None):
    """<s|U^dag O U|s> with U the circuit in order; `angles` overrides the
    circuit's angles (circuit order)."""
    psi = np.zeros(2**n, complex)
    psi[state] = 1.0
    k = 0
    for layer in circuit.layers:
        for rot in layer:
            a = rot.angle if angles is None else angles[k]
            m = pauli_matrix(rot.generator)
            psi = (math.cos(a / 2) * np.eye(2**n) - 1j * math.sin(a / 2) * m) @ psi
            k += 1
    o = sum(c * pauli_matrix(t) for t, c in obs.items())
    return float(np.real(np.conj(psi) @ o @ psi))


def dense_gradient(obs, circuit, state, n):
    """Exact dE/d angle per rotation (circuit order) by the shift rule."""
    base = np.array([r.angle for layer in circuit.layers for r in layer])
    g = np.zeros(len(base))
    for k in range(len(base)):
        a = base.copy()
        a[k] += math.pi / 2
        ep = dense_expectation(obs, circuit, state, n, a)
        a[k] -= math.pi
        g[k] = 0.5 * (ep - dense_expectation(obs, circuit, state, n, a))
    return g


@pytest.mark.parametrize("seed", range(4))
def test_reference_value_matches_oracle(oracle, seed):
    obs, circ, state = random_circuit(seed, 6, 40)
    for kw in (dict(), dict(max_weight=3, min_coeff=1e-3), dict(min_coeff=1e-2, min_terms=6)):
        p = from_circuit(0, 6, obs, circ, state, **kw)
        if seed % 2:
            p.noise_table = np.array([math.exp(-0.01 * w) for w in range(7)])
        e, _ = propagate_with_tangents(oracle, p)
        o = run_oracle(oracle, p)
        assert abs(e - o.expectation_accurate) <= 1e-12 * max(1.0, o.expectation_abs)


@pytest.mark.parametrize("seed", range(3))
def test_reference_gradient_is_exact_without_truncation(oracle, seed):
    n = 4
    obs, circ, state = random_circuit(seed, n, 16)
    p = from_circuit(0, n, obs, circ, state)
    _, g_engine_order = propagate_with_tangents(oracle, p)
    order = _heisenberg_order(circ)
    g = np.zeros(len(order))
    g[order] = g_engine_order
    np.testing.assert_allclose(g, dense_gradient(obs, circ, state, n), atol=1e-11)


def test_heisenberg_order_matches_gate_arrays():
    obs, circ, state = random_circuit(7, 5, 23, layer_size=5)
    flat = [r for layer in circ.layers for r in layer]
    gw, ga, _ = heisenberg_gates(circ, 1, lambda g: g.key())
    order = _heisenberg_order(circ)
    assert [flat[k].angle for k in order] == list(ga)
    assert [flat[k].generator.key() for k in order] == [int(w[0]) for w in gw]


def test_parametrized_angles_follow_the_index():
    wl = workloads.hardware_efficient(5, 2, seed=3)
    spec = ParametrizedExpectation(pq.PauliPropagator(truncation=wl.truncation()), wl.observable, wl.circuit,
                                   wl.meta["param_index"])
    assert spec.n_params == 2 * 5 * 2
    np.testing.assert_array_equal(spec.angles(wl.meta["theta"]), spec._fixed)
    th = np.arange(spec.n_params, dtype=float)
    a = spec.angles(th)
    flat_idx = np.asarray(wl.meta["param_index"])[_heisenberg_order(wl.circuit)]
    assert np.all(a[flat_idx >= 0] == th[flat_idx[flat_idx >= 0]])
    with pytest.raises(ValueError):
        spec.angles(th[:-1])
