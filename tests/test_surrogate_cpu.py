"""The surrogate restatement (oracle/pq_surrogate.py) pinned before it is used
as a checker: the reference's own known answers for the coefficient DAG
(crates/surrogate/tests/unit/symcoeff.rs) and for the build
(tests/surrogate/test_surrogate_pauli.py: agreement with numerical
propagation, frequency truncation), restated; agreement with the C oracle's
numerical propagation on random circuits with Clifford rotations; and its
reverse-mode derivative against central differences of itself."""

import math
import time

import numpy as np
import pytest
from harness import from_circuit, run_oracle
from surrogate_ref import build_surrogate, sur, to_int, to_words
from test_adjoint_cpu import random_circuit

from propaq_b200.circuits import PauliCircuit, PauliRotation
from propaq_b200.datatypes import PauliString, PauliTermSum

PH = -1j  # the phase the reference's unit tests rotate with


def lut_of(n):
    return sur.make_lut([0.37 * (i + 1) for i in range(n)])


def ev(c, lut):
    t = sur.Tape([c])
    return 0.0 if t.roots[0] < 0 else t.evaluate_all(lut)[t.roots[0]]


def rot(c, p, phase=PH):
    return sur.apply_rotation(c, ("sym", p), phase)


# ------------------------------------------------------------ DAG known answers
def test_scalar_and_count_saturation():
    c = sur.scalar(2.5)
    assert sur.monomial_count(c) == 1 and ev(c, []) == 2.5
    for _ in range(135):
        c = sur.add_assign(c, c)
    assert sur.monomial_count(c) == sur.U128_MAX
    assert sur.monomial_count(None) == 0 and ev(None, []) == 0.0


def test_rotation_trig_identities():
    lut = lut_of(8)
    c = sur.scalar(0.75)
    for p in (0, 1, 2, 5, 7):
        before = ev(c, lut)
        c, s = rot(c, p)
        assert abs(ev(c, lut) - lut[2 * p] * before) < 1e-12
        assert abs(ev(s, lut) - lut[2 * p + 1] * before) < 1e-12
    c, s = sur.apply_rotation(sur.scalar(0.75), ("num", 0.4), PH)
    assert abs(ev(c, []) - 0.75 * math.cos(0.4)) < 1e-12 and abs(ev(s, []) - 0.75 * math.sin(0.4)) < 1e-12


def test_paths_powers_and_simplify():
    lut = lut_of(1)
    c, _ = rot(sur.scalar(1.0), 0)
    c, _ = rot(c, 0)
    assert sur.monomial_count(c) == 1 and abs(ev(c, lut) - lut[0] ** 2) < 1e-12
    _, p1 = rot(sur.scalar(1.0), 0)
    p1, _ = rot(p1, 0)
    b, _ = rot(sur.scalar(1.0), 0)
    _, p2 = rot(b, 0)
    total = sur.add_assign(sur.add_assign(None, p1), p2)
    assert sur.monomial_count(total) == 2 and abs(ev(total, lut) - 2 * lut[0] * lut[1]) < 1e-12
    (s1,) = sur.simplify_batch([total])
    assert sur.monomial_count(s1) == 1 and abs(ev(s1, lut) - 2 * lut[0] * lut[1]) < 1e-12
    (s2,) = sur.simplify_batch([s1])
    assert sur.monomial_count(s2) == 1 and abs(ev(s2, lut) - ev(s1, lut)) < 1e-15
    a, _ = rot(sur.scalar(3.0), 0)
    b, _ = rot(sur.scalar(-3.0), 0)
    (z,) = sur.simplify_batch([sur.add(a, b)])
    assert z is None, "an exact cancellation simplifies to the empty coefficient"


def test_simplify_bounds_heavy_parameter_reuse():
    base = sur.scalar(1.0)
    for r in range(14):
        a, b = rot(base, r % 3)
        base = sur.add(a, b)
    pre = sur.monomial_count(base)
    lut = lut_of(3)
    v = ev(base, lut)
    (post,) = sur.simplify_batch([base])
    assert pre >= 1 << 14
    assert sur.monomial_count(post) <= (14 // 3 + 2) ** 3 and sur.monomial_count(post) * 10 < pre
    assert abs(ev(post, lut) - v) < 1e-6 * max(abs(v), 1.0)


def test_prune_known_answers():
    lut = lut_of(2)
    total = sur.add_assign(sur.scalar(5.0), rot(sur.scalar(3.0), 0)[0])
    assert abs(ev(sur.prune(total, 0, None), lut) - 5.0) < 1e-12
    c, _ = rot(sur.scalar(2.0), 0)
    c, _ = rot(c, 1)
    assert sur.prune(c, 2, None) is c, "the provably safe path keeps the node itself"
    assert sur.prune(c, None, None) is c
    m = sur.add(sur.cos_node(0, sur.scale(2.0, sur.scalar(3.0))), sur.sin_node(1, sur.scalar(0.5)))
    want = 6.0 * math.cos(0.37) + 0.5 * math.sin(0.74)
    assert abs(ev(m, lut) - want) < 1e-12
    assert sur.prune(m, 0, None) is None
    assert abs(ev(sur.prune(m, 1, None), lut) - want) < 1e-12
    assert abs(ev(sur.prune(m, None, 1.0), lut) - 6.0 * math.cos(0.37)) < 1e-12
    assert sur.prune(m, None, 10.0) is None


def test_prune_memoises_shared_subtrees():
    base, nxt = sur.scalar(1.0), 0
    for _ in range(12):
        merged = None
        for _ in range(3):
            b, _ = rot(base, nxt)
            nxt += 1
            merged = sur.add_assign(merged, b)
        base = merged
    lut = sur.make_lut([0.37 * (i + 1) for i in range(nxt)])
    before = ev(base, lut)
    t0 = time.perf_counter()
    after = ev(sur.prune(base, None, 1e-9), lut)
    assert time.perf_counter() - t0 < 10.0
    assert abs(after - before) < 1e-6 * max(abs(before), 1.0)


def test_compile_shares_roots_and_marks_empty():
    c, _ = rot(sur.scalar(1.5), 0)
    t = sur.Tape([c, c, None])
    assert t.roots[0] == t.roots[1] >= 0 and t.roots[2] == -1


# ----------------------------------------------------------- build known answers
N = 4


def ps(x, z):
    return PauliString(x, z, N)


def numeric(oracle, obs, circ, state=0):
    p = from_circuit(0, N, obs, circ, state)
    return run_oracle(oracle, p, want_terms=False).expectation


def surrogate(obs, circ, param_indices, state=0, **trunc):
    p = from_circuit(0, N, obs, circ, state)
    flat = [r for layer in circ.layers for r in layer]
    heis = [r for layer in reversed(circ.layers) for r in reversed(layer)]
    index = {id(r): i for i, r in enumerate(flat)}
    params = [("sym", param_indices[index[id(r)]]) if param_indices[index[id(r)]] is not None
              else ("num", r.angle) for r in heis]
    alg = sur.PauliAlgebra(N)
    o = [(to_int(k), float(c)) for k, c in zip(p.obs_keys.reshape(-1, 1), p.obs_coeffs)]
    g = [(to_int(k), prm) for k, prm in zip(p.gate_keys.reshape(-1, 1), params)]
    n_params = 1 + max([i for i in param_indices if i is not None], default=-1)
    return sur.build(alg, N, 64, o, g, initial_state=state, n_params=n_params, **trunc)


CASES = [
    ([(1, 0)], [0.3], [0]),                        # X_0 on Z_0
    ([(1, 0), (2, 0)], [0.7, 1.2], [0, 1]),        # independent parameters
    ([(1, 0), (3, 0), (0, 2)], [0.3, 0.7, 1.1], [0, 1, 2]),
    ([(1, 0), (2, 0)], [0.5, 0.5], [0, 0]),        # a shared parameter
    ([(1, 0), (2, 0), (4, 0)], [0.4, 0.4, 0.4], [0, 0, 0]),
]


@pytest.mark.parametrize("gens,angles,idx", CASES)
def test_surrogate_agrees_with_numerical_propagation(oracle, gens, angles, idx):
    obs = PauliTermSum({ps(0, 1): 1.0})
    circ = PauliCircuit([PauliRotation(ps(*g), a) for g, a in zip(gens, angles)])
    vals = [0.0] * (max(idx) + 1)
    for i, a in zip(idx, angles):
        vals[i] = a
    model = surrogate(obs, circ, idx)
    assert model.evaluate(vals) == pytest.approx(numeric(oracle, obs, circ), rel=1e-9)


def test_empty_circuit_excited_state_and_multi_term_observable(oracle):
    obs = PauliTermSum({ps(0, 1): 1.0})
    assert surrogate(obs, PauliCircuit([]), []).evaluate([]) == pytest.approx(1.0)
    circ = PauliCircuit([PauliRotation(ps(1, 0), 0.4)])
    for state in (0, 1):
        assert surrogate(obs, circ, [0], state).evaluate([0.4]) == pytest.approx(numeric(oracle, obs, circ, state),
                                                                                rel=1e-9)
    obs2 = PauliTermSum({ps(0, 1): 1.0, ps(0, 2): 0.5})
    circ2 = PauliCircuit([PauliRotation(ps(1, 0), 0.6)])
    assert surrogate(obs2, circ2, [0]).evaluate([0.6]) == pytest.approx(numeric(oracle, obs2, circ2), rel=1e-9)


def test_frequency_truncation_converges(oracle):
    obs = PauliTermSum({ps(0, 1): 1.0})
    gens, angles = [(1, 0), (3, 0), (0, 2)], [0.3, 0.7, 1.1]
    circ = PauliCircuit([PauliRotation(ps(*g), a) for g, a in zip(gens, angles)])
    exact = numeric(oracle, obs, circ)
    prev = math.inf
    for f in range(4):
        err = abs(surrogate(obs, circ, [0, 1, 2], frequency=f).evaluate(angles) - exact)
        assert err <= prev + 1e-12
        prev = err
    assert prev <= 1e-9 * max(1.0, abs(exact)), "exact once max_frequency reaches the rotation count"
    assert surrogate(obs, circ, [0, 1, 2], frequency=0).n_terms >= 0


# -------------------------------------------------------------------- algebra
def test_pauli_algebra_matches_the_c_oracle(oracle):
    rng = np.random.default_rng(3)
    for w in (1, 2):
        n = 32 * w
        alg = sur.PauliAlgebra(n)
        for _ in range(300):
            g = to_int(rng.integers(0, 2**63, size=w, dtype=np.uint64) * 2 + rng.integers(0, 2, size=w, dtype=np.uint64))
            k = to_int(rng.integers(0, 2**63, size=w, dtype=np.uint64) * 2 + rng.integers(0, 2, size=w, dtype=np.uint64))
            s = int(rng.integers(0, 2**62))
            gw, kw = to_words(g, w), to_words(k, w)
            assert alg.anticommutes(g, k) == oracle.anticommutes(0, gw, kw)
            child, p = oracle.product(0, gw, kw)
            assert alg.product(g, k) == (to_int(child), p)
            assert alg.weight(k) == oracle.weight(0, n, kw)
            zk = k & ~int("01" * (32 * w), 2)
            assert alg.trace(zk, s) == oracle.trace(0, n, to_words(zk, w), to_words(s, w))


# ---------------------------------------------- random circuits, frame, gradient
@pytest.mark.parametrize("seed", range(4))
def test_random_circuits_with_cliffords_match_the_oracle(oracle, seed):
    n = 5
    obs, circ, state = random_circuit(300 + seed, n, 24, clifford=True)
    p = from_circuit(0, n, obs, circ, state)
    model = build_surrogate(p)
    o = run_oracle(oracle, p, want_terms=False)
    assert model.evaluate(list(p.angles)) == pytest.approx(o.expectation, rel=1e-10, abs=1e-12)


@pytest.mark.parametrize("seed", range(2))
def test_weight_truncated_build_matches_the_weight_truncated_oracle(oracle, seed):
    # Without Clifford rotations a post-gate weight cut (surrogate) and an
    # emit-time one (numerical) keep the same terms.
    n = 7
    obs, circ, state = random_circuit(400 + seed, n, 30)
    p = from_circuit(0, n, obs, circ, state, max_weight=3)
    model = build_surrogate(p, weight=3)
    o = run_oracle(oracle, p, want_terms=False)
    assert model.evaluate(list(p.angles)) == pytest.approx(o.expectation, rel=1e-10, abs=1e-12)


def test_reverse_mode_derivative_matches_central_differences():
    n = 5
    obs, circ, state = random_circuit(500, n, 20)
    p = from_circuit(0, n, obs, circ, state)
    model = build_surrogate(p)
    th = list(p.angles)
    g = model.gradient(th)
    h = 1e-5
    for k in range(0, len(th), 3):
        tp, tm = list(th), list(th)
        tp[k] += h
        tm[k] -= h
        fd = (model.evaluate(tp) - model.evaluate(tm)) / (2 * h)
        assert g[k] == pytest.approx(fd, rel=1e-6, abs=1e-8)


def test_majorana_build_matches_the_oracle(oracle):
    from harness import from_workload

    from propaq_b200 import workloads

    p = from_workload(workloads.majorana_givens(n_sites=5, reps=1, seed=2, max_weight=None, min_coeff=None))
    model = build_surrogate(p, oracle)
    o = run_oracle(oracle, p, want_terms=False)
    assert model.evaluate(list(p.angles)) == pytest.approx(o.expectation, rel=1e-10, abs=1e-12)


def test_config5_shape_surrogate_matches_the_oracle(oracle):
    # The gradient's ansatz (RY, RZ, CNOT ladder of Z_c(pi/2), X_t(pi/2),
    # Z_c X_t(-pi/2); sum Z_i Z_i+1; |0..0>) at 6 qubits, untruncated: the
    # CNOT pieces go to the surrogate's frame as numeric Clifford rotations.
    from harness import from_workload

    from propaq_b200 import workloads

    p = from_workload(workloads.hardware_efficient(6, 3, seed=7, sigma=0.6, max_weight=None, min_coeff=None))
    model = build_surrogate(p)
    o = run_oracle(oracle, p, want_terms=False)
    assert model.evaluate(list(p.angles)) == pytest.approx(o.expectation, rel=1e-10, abs=1e-12)
