"""The adjoint gradient (pq_run_adjoint / propaq_b200.adjoint) on the GPU.

  - exact: without truncation the gradient is the exact derivative, checked
    against a dense-statevector shift rule (Clifford rotations included: they
    are deferred into the frame and conjugate every later generator);
  - frozen decisions: with truncation, noise, phase-only rotations and a
    TermBudget floor it matches the forward-mode reference, which carries
    derivatives through the same decisions;
  - checkpointing changes memory, not results: every segment length gives
    bit-identical gradients;
  - the full config: central finite differences on 20 seeded angles;
  - the surrogate derivative: the reference's surrogate model of the same
    circuit (restated in oracle/pq_surrogate.py), differentiated over its
    tape, on the ansatz untruncated and on a weight-cut circuit.
"""

import math

import numpy as np
import pytest
from adjoint_ref import propagate_with_tangents
from harness import from_circuit, from_workload, make_cfg, random_pauli_problem, spread_units
from test_adjoint_cpu import dense_gradient, random_circuit

import propaq_b200 as pq
from propaq_b200 import workloads
from propaq_b200.adjoint import ParametrizedExpectation, _heisenberg_order

pytestmark = pytest.mark.gpu


def gpu_grad(engine, p, checkpoint_layers=0, record_bytes=0):
    cfg, keep = make_cfg(p, want_terms=False)
    res, nt, g = engine.run_adjoint(cfg, p.obs_keys, p.obs_coeffs, p.gate_keys, p.angles, p.offsets, p.diag,
                                    checkpoint_layers=checkpoint_layers, record_bytes=record_bytes)
    return res, nt, g


def replay_pool(p, res):
    """A record pool 2% short of what the whole run records, so the gradient
    re-runs segments to record them (one at a time, each well inside the
    pool).  The forward run records one 12-byte element per row entering each
    rotation or reclaim, and one key per row entering each reclaim; the pool
    gives 85% of its bytes to the elements and 15% to the keys."""
    reclaim = p.max_weight is not None or p.min_coeff is not None or p.min_terms is not None
    keys = res.sum_rows_noise if reclaim else 0
    rows = res.sum_rows_gate + res.sum_rows_phase + keys
    return int(max(0.98 * rows * 12 / 0.85, 0.98 * keys * 8 * p.n_words / 0.15))


@pytest.mark.parametrize("seed", range(4))
def test_gradient_is_exact_without_truncation(gpu_engine, seed):
    n = 5
    obs, circ, state = random_circuit(seed, n, 30, clifford=True)
    p = from_circuit(0, n, obs, circ, state)
    res, _, g = gpu_grad(gpu_engine, p, checkpoint_layers=2)
    order = _heisenberg_order(circ)
    want = dense_gradient(obs, circ, state, n)[order]
    cliff = np.abs(np.cos(p.angles)) < 1e-9
    assert np.all(np.isnan(g[cliff])), "deferred Clifford rotations have no gradient entry"
    np.testing.assert_allclose(g[~cliff], want[~cliff], atol=1e-10)


CASES = [
    dict(max_weight=3, min_coeff=1e-3),
    dict(max_weight=4, min_coeff=1e-2, noise=0.02),
    dict(min_coeff=3e-3, min_terms=8),
    dict(max_weight=3, noise_layered=True),
    dict(min_coeff=1e-3, phase=True),
]


@pytest.mark.parametrize("seed", range(3))
@pytest.mark.parametrize("case", CASES, ids=lambda c: "-".join(f"{k}{v}" for k, v in c.items()))
def test_gradient_matches_forward_mode_reference(gpu_engine, oracle, case, seed):
    case = dict(case)
    noise = case.pop("noise", None)
    layered = case.pop("noise_layered", False)
    phase = case.pop("phase", False)
    n = 7
    obs, circ, state = random_circuit(100 + seed, n, 48)
    if phase:  # two rotations with |sin| < 1e-9: phase-only ops
        circ.layers[1][0].angle = 1e-11
        circ.layers[3][2].angle = -2e-10
    p = from_circuit(0, n, obs, circ, state, **case)
    if noise:
        p.noise_table = np.array([math.exp(-noise * w) for w in range(n + 1)])
    if layered:
        L = len(p.offsets) - 1
        p.noise_tables_layered = np.array([[math.exp(-0.01 * (l + 1) * w) for w in range(n + 1)] for l in range(L)])
    e_ref, g_ref = propagate_with_tangents(oracle, p)
    res, nt, g = gpu_grad(gpu_engine, p, checkpoint_layers=3)
    assert abs(res.expectation_value - e_ref) <= 1e-12 * max(1.0, abs(e_ref))
    scale = max(1.0, float(np.abs(g_ref).max()))
    np.testing.assert_allclose(g, g_ref, rtol=1e-9, atol=1e-12 * scale)
    _, _, g2 = gpu_grad(gpu_engine, p, checkpoint_layers=1, record_bytes=replay_pool(p, res))
    np.testing.assert_allclose(g2, g_ref, rtol=1e-9, atol=1e-12 * scale)


def test_gradient_on_a_wide_register(gpu_engine, oracle):
    # 64-word keys (2048 qubits), 10 active qubits spread over the register.
    p = random_pauli_problem(4, 2048, n_gates=50, clifford_frac=0.0, units=spread_units(4, 2048, 10), max_weight=4,
                             min_coeff=1e-3)
    e_ref, g_ref = propagate_with_tangents(oracle, p)
    res, nt, g = gpu_grad(gpu_engine, p, checkpoint_layers=2)
    assert abs(res.expectation_value - e_ref) <= 1e-12 * max(1.0, abs(e_ref))
    scale = max(1.0, float(np.abs(g_ref).max()))
    np.testing.assert_allclose(g, g_ref, rtol=1e-9, atol=1e-12 * scale)


@pytest.mark.parametrize("wl", [workloads.hardware_efficient(12, 5, seed=2), workloads.kicked_ising(4, 5, 4)],
                         ids=["hea", "kicked_noisy"])
def test_recording_in_the_forward_pass_equals_replayed_segments(gpu_engine, wl):
    # One reverse sweep over records made in the forward pass, and segment
    # replays into a small pool, give the same gradient bit for bit.
    p = from_workload(wl)
    gpu_grad(gpu_engine, p, 1)  # the engine's buffers grow to size here
    full = gpu_grad(gpu_engine, p, 1)
    replayed = gpu_grad(gpu_engine, p, 1, record_bytes=replay_pool(p, full[0]))
    assert replayed[0].gpu_launches > full[0].gpu_launches, "the small pool must force replays"
    ok = ~np.isnan(full[2])
    assert np.array_equal(np.isnan(replayed[2]), ~ok)
    assert np.array_equal(replayed[2][ok], full[2][ok])
    with pytest.raises(MemoryError, match="fewer checkpoint layers"):
        gpu_grad(gpu_engine, p, 0, record_bytes=1 << 12)


SURROGATE_CASES = [
    # the gradient's ansatz (RY, RZ, CNOT ladder; sum Z_i Z_i+1; |0..0>), untruncated
    (lambda: workloads.hardware_efficient(6, 3, seed=7, sigma=0.6, max_weight=None, min_coeff=None)),
    (lambda: workloads.hardware_efficient(8, 4, seed=7, sigma=0.6, max_weight=None, min_coeff=None)),
    # a weight cut with no Clifford rotation: the surrogate's post-gate cut and
    # the engine's emit-time cut keep the same terms
    (lambda: workloads.tfim_chain(16, 6, seed=3, max_weight=4, min_coeff=None)),
]


@pytest.mark.parametrize("make", SURROGATE_CASES, ids=["hea6x3", "hea8x4", "tfim16-w4"])
def test_gradient_matches_the_surrogate_derivative(gpu_engine, make):
    # The surrogate model's derivative (reverse mode over its tape, one
    # parameter per rotation) against the adjoint gradient: the same function
    # of the angles wherever the truncation is structural.
    from surrogate_ref import build_surrogate

    wl = make()
    p = from_workload(wl)
    res, _, g = gpu_grad(gpu_engine, p, 1)
    model = build_surrogate(p, weight=wl.max_weight)
    th = list(p.angles)
    e_s, g_s = model.evaluate(th), np.array(model.gradient(th))
    assert abs(res.expectation_value - e_s) <= 1e-10 * max(1.0, abs(e_s))
    param = np.abs(np.cos(p.angles)) >= 1e-9  # the CNOT pieces are fixed rotations
    assert np.array_equal(~np.isnan(g), param)
    scale = max(1.0, float(np.abs(g_s).max()))
    np.testing.assert_allclose(g[param], g_s[param], rtol=1e-9, atol=1e-12 * scale)


def test_default_pool_follows_the_problem(gpu_engine):
    # The engine keeps the default-sized pool at what the last gradient
    # needed; a larger problem after a small one outgrows it, grows it and
    # re-runs segments; the gradient is the same as with an explicit pool.
    small = from_workload(workloads.hardware_efficient(6, 2, seed=1))
    big = from_workload(workloads.hardware_efficient(12, 5, seed=2))
    ref = gpu_grad(gpu_engine, big, 1, record_bytes=1 << 30)
    gpu_grad(gpu_engine, small, 1)
    after_small = gpu_grad(gpu_engine, big, 1)
    again = gpu_grad(gpu_engine, big, 1)
    assert after_small[0].gpu_launches > again[0].gpu_launches, "the first big gradient must re-run segments"
    ok = ~np.isnan(ref[2])
    for r in (after_small, again):
        assert r[0].expectation_value == ref[0].expectation_value
        assert np.array_equal(np.isnan(r[2]), ~ok)
        assert np.array_equal(r[2][ok], ref[2][ok])


def test_checkpoint_segments_do_not_change_the_gradient(gpu_engine):
    wl = workloads.hardware_efficient(12, 5, seed=2)
    p = from_workload(wl)
    ref = gpu_grad(gpu_engine, p, 0)
    for c in (1, 2, 3, 4, 7):
        res, nt, g = gpu_grad(gpu_engine, p, c)
        assert res.expectation_value == ref[0].expectation_value
        assert np.array_equal(nt, ref[1])
        assert np.array_equal(np.isnan(g), np.isnan(ref[2]))
        ok = ~np.isnan(g)
        assert np.array_equal(g[ok], ref[2][ok]), f"checkpoint_layers={c}"


def test_forward_part_equals_plain_run(gpu_engine):
    # The gradient's forward pass runs every rotation on its own while a plain
    # run fuses commuting pairs; the terms are the same, appended in another
    # order, so only the expectation sum's last bits may differ.
    wl = workloads.kicked_ising(5, 6, 4)
    p = from_workload(wl)
    cfg, keep = make_cfg(p, want_terms=False)
    plain, nt_plain = gpu_engine.run(cfg, p.obs_keys, p.obs_coeffs, p.gate_keys, p.angles, p.offsets, p.diag)
    res, nt, g = gpu_grad(gpu_engine, p, 2)
    assert abs(res.expectation_value - plain.expectation_value) <= 1e-12 * max(1.0, abs(plain.expectation_value))
    assert np.array_equal(nt, nt_plain)
    assert np.isfinite(g[np.abs(np.cos(p.angles)) >= 1e-9]).all()


def test_torch_autograd_function(gpu_engine):
    import torch

    wl = workloads.hardware_efficient(10, 3, seed=4)
    spec = ParametrizedExpectation(pq.PauliPropagator(truncation=wl.truncation()), wl.observable, wl.circuit,
                                   wl.meta["param_index"], checkpoint_layers=1)
    theta = torch.tensor(wl.meta["theta"], dtype=torch.float64, device="cuda", requires_grad=True)
    loss = 3.0 * spec(theta)
    loss.backward()
    e, g = spec.value_and_grad(wl.meta["theta"])
    assert float(loss.detach()) == pytest.approx(3.0 * e, rel=1e-15)
    np.testing.assert_array_equal(theta.grad.cpu().numpy(), 3.0 * g)
    with torch.no_grad():
        assert float(spec(theta)) == e


def test_parameter_shift_agrees_without_truncation(gpu_engine):
    wl = workloads.hardware_efficient(8, 2, seed=5, max_weight=None, min_coeff=None)
    spec = ParametrizedExpectation(pq.PauliPropagator(), wl.observable, wl.circuit, wl.meta["param_index"])
    _, g = spec.value_and_grad(wl.meta["theta"])
    np.testing.assert_allclose(spec.parameter_shift(wl.meta["theta"], batch=8), g, atol=1e-11)


def test_config_hardware_efficient_finite_differences(gpu_engine):
    # 50 qubits, 12 layers, 1200 angles, w <= 8, |c| >= 1e-5: central
    # differences on 20 seeded angles.  A difference quotient that straddles a
    # truncation decision (a term crossing the cutoff within +-h) jumps by
    # about cutoff / h, so h starts at 1e-5 and shrinks (1e-6, 1e-7) while any
    # per-gate live count at theta +- h differs from theta's.
    from propaq_b200 import _native

    wl = workloads.hardware_efficient()
    spec = ParametrizedExpectation(pq.PauliPropagator(truncation=wl.truncation()), wl.observable, wl.circuit,
                                   wl.meta["param_index"], checkpoint_layers=3)
    th = wl.meta["theta"]
    e, g = spec.value_and_grad(th)

    def run(t):
        res, nt = _native.engine(0).run(*spec._call_args(t))
        return res.expectation_value, nt

    e0, nt0 = run(th)
    assert e0 == e
    picks = np.random.default_rng(0).choice(len(th), size=20, replace=False)
    bad = []
    for k in picks:
        for h in (1e-5, 1e-6, 1e-7):
            tp, tm = th.copy(), th.copy()
            tp[k] += h
            tm[k] -= h
            (ep, ntp), (em, ntm) = run(tp), run(tm)
            if np.array_equal(ntp, nt0) and np.array_equal(ntm, nt0):
                break
        fd = (ep - em) / (2 * h)
        tol = 1e-5 * abs(g[k]) + 64 * np.finfo(float).eps * abs(e) / h
        if not abs(fd - g[k]) <= tol:
            bad.append((int(k), h, float(g[k]), fd))
    assert not bad, f"adjoint vs central differences (angle, h, adjoint, fd): {bad}"


def test_gradient_refusals(gpu_engine):
    wl = workloads.kicked_ising(4, 4, 2)  # RZZ(-pi/2) changes weight
    p = from_workload(wl)
    p.min_terms = 10
    with pytest.raises(NotImplementedError, match="TermBudget"):
        gpu_grad(gpu_engine, p)
