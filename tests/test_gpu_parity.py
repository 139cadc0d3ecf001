"""Parity of the CUDA engine (through the C ABI) with the CPU oracle.

Term sets must match bit for bit and every coefficient must be identical:
each merge in the reference is one two-operand FP64 add whose operands do not
depend on processing order (K -> G.K is an involution), so the engine
reproduces every coefficient exactly.  Only the expectation value is a sum
whose rounding depends on order; it is compared against the oracle's
compensated sum at 1e-12 relative (harness.expectation_close).
"""

import math

import numpy as np
import pytest
from harness import (
    Problem,
    assert_terms_equal,
    expectation_close,
    from_circuit,
    from_workload,
    golden_fixture,
    golden_problem,
    make_cfg,
    random_pauli_problem,
    run_gpu,
    run_oracle,
    spread_units,
)
from oracle_client import REF_PLUGINS
from plugin_build import build_all

import propaq_b200 as pq
from propaq_b200 import workloads
from propaq_b200.circuits import MajoranaCircuit, MajoranaRotation, PauliCircuit, PauliRotation
from propaq_b200.datatypes import MajoranaMonomial, MajoranaTermSum, PauliString, PauliTermSum

pytestmark = pytest.mark.gpu


def check(engine, oracle, p: Problem, parts=1):
    g = run_gpu(engine, p)
    o = run_oracle(oracle, p, n_partitions=parts)
    assert np.array_equal(g.n_terms, o.n_terms), "live counts per gate differ"
    assert_terms_equal(g.keys, g.coeffs, o.keys, o.coeffs)
    assert g.terms_below_cutoff == o.terms_below_cutoff
    if p.diag is not None:
        ok, err, tol = expectation_close(g.expectation, o)
        assert ok, f"expectation {g.expectation!r} vs oracle {o.expectation_accurate!r} (err {err:.3g} > {tol:.3g})"
    return g, o


# ------------------------------------------------------------ golden circuit
GOLD = [c for c in golden_fixture()["cases"] if "plugin" not in c]


@pytest.mark.parametrize("case", GOLD, ids=[c["name"] for c in GOLD])
def test_golden_builtin(gpu_engine, oracle, case):
    p = golden_problem(max_weight=case.get("max_weight"), min_coeff=case.get("min_coeff"))
    if "noise" in case:
        d = case["noise"]["uniform"]
        p.noise_table = np.array([math.exp(-d * float(w)) for w in range(p.n_units + 1)])
    g, o = check(gpu_engine, oracle, p)
    assert abs(g.expectation - case["expected"]) <= 1e-12 * abs(case["expected"])


def test_golden_through_propagator_api(gpu_engine):
    fx = golden_fixture()
    n = fx["n_qubits"]
    circ = pq.PauliCircuit([pq.PauliRotation(PauliString(r["x"], r["z"], n), r["angle"]) for r in fx["rotations"]])
    obs = pq.PauliTermSum()
    obs.add(PauliString(0, 1, n), 1.0)
    for case in GOLD:
        trunc = []
        if case.get("max_weight") is not None:
            trunc.append(pq.WeightTruncator(case["max_weight"]))
        if case.get("min_coeff") is not None:
            trunc.append(pq.CoefficientTruncator(case["min_coeff"]))
        noise = pq.UniformNoiseModel(case["noise"]["uniform"]) if "noise" in case else None
        prop = pq.PauliPropagator(noise=noise, truncation=trunc, n_threads=4)
        res = prop.expectation_value(obs, circ, initial_state=0)
        assert abs(res.expectation_value - case["expected"]) <= 1e-12 * abs(case["expected"])
        assert len(res.n_terms) == 40


@pytest.fixture(scope="module")
def test_plugins(tmp_path_factory):
    return build_all(tmp_path_factory.mktemp("gpu_plugins"))


@pytest.mark.parametrize("name", ["uniform", "layered"])
def test_weight_only_plugins_match_oracle(gpu_engine, oracle, test_plugins, name):
    # A plugin that does not read keys is tabulated by weight (per layer when
    # it reads the layer), noise_resolver.rs:78-131.
    p = golden_problem(max_weight=3, min_coeff=1e-4)
    cfg = '{"damping": 0.03}'
    g_plugin = pq.NativeNoiseModel(str(test_plugins[name]), cfg)
    o_plugin = oracle.load_plugin(test_plugins[name], cfg, noise=True)
    try:
        g = run_gpu(gpu_engine, p, noise_plugin=g_plugin.handle)
        o = oracle.run(p.basis, p.n_units, p.n_words, p.obs_keys, p.obs_coeffs, p.gate_keys, p.angles, p.offsets,
                       max_weight=3, min_coeff=1e-4, noise_plugin=o_plugin, diag_state=p.diag)
    finally:
        oracle.lib.pqo_plugin_free(o_plugin)
    assert np.array_equal(g.n_terms, o.n_terms)
    assert_terms_equal(g.keys, g.coeffs, o.keys, o.coeffs)


PLUGIN_CASES = [c for c in golden_fixture()["cases"] if "plugin" in c]


@pytest.mark.parametrize("case", PLUGIN_CASES, ids=lambda c: c["name"])
def test_reference_plugins_golden_and_oracle(gpu_engine, oracle, case):
    # The reference's nine example plugins on its notebooks' circuit.  The
    # key-reading noise model and the truncators are asked on the host for
    # every row / branch (the conformance path); the rest is tabulated.
    so = REF_PLUGINS / f"{case['plugin']}.so"
    if not so.exists():
        pytest.skip("reference example plugins not built")
    noise = case["plugin_kind"] == "noise"
    p = golden_problem()
    m = (pq.NativeNoiseModel if noise else pq.NativeTruncator)(str(so), case["plugin_config"])
    g = run_gpu(gpu_engine, p, **({"noise_plugin": m.handle} if noise else {"truncator": m.handle}))
    assert abs(g.expectation - case["expected"]) <= 1e-12 * abs(case["expected"])
    h = oracle.load_plugin(so, case["plugin_config"], noise=noise)
    try:
        o = oracle.run(p.basis, p.n_units, p.n_words, p.obs_keys, p.obs_coeffs, p.gate_keys, p.angles, p.offsets,
                       diag_state=p.diag, **({"noise_plugin": h} if noise else {"truncator": h}))
    finally:
        oracle.lib.pqo_plugin_free(h)
    assert np.array_equal(g.n_terms, o.n_terms)
    assert_terms_equal(g.keys, g.coeffs, o.keys, o.coeffs)


@pytest.mark.parametrize("seed", [0, 1])
@pytest.mark.parametrize("kw", [dict(max_weight=4, min_coeff=1e-3), dict(min_coeff=1e-3, min_terms=40), dict()],
                         ids=["cuts", "floor", "plain"])
def test_key_reading_noise_and_truncator_match_oracle(gpu_engine, oracle, test_plugins, seed, kw):
    # Key-reading noise (damps terms on unit 0) and a truncator plugin, with and
    # without the built-in cuts and a TermBudget floor, on random circuits with
    # Clifford rotations (no deferral: the noise reads keys).
    for which in ("noise", "truncator", "both"):
        p = random_pauli_problem(seed, 8, n_gates=60, **kw)
        nm = pq.NativeNoiseModel(str(test_plugins["keyed"]), '{"damping": 0.05}')
        tm = pq.NativeTruncator(str(test_plugins["truncator"]), '{"max_weight": 4}')
        gk = {}
        if which in ("noise", "both"):
            gk["noise_plugin"] = nm.handle
        if which in ("truncator", "both"):
            gk["truncator"] = tm.handle
        g = run_gpu(gpu_engine, p, **gk)
        hn = oracle.load_plugin(test_plugins["keyed"], '{"damping": 0.05}', noise=True)
        ht = oracle.load_plugin(test_plugins["truncator"], '{"max_weight": 4}', noise=False)
        try:
            ok = {}
            if which in ("noise", "both"):
                ok["noise_plugin"] = hn
            if which in ("truncator", "both"):
                ok["truncator"] = ht
            o = run_oracle(oracle, p, **ok)
        finally:
            oracle.lib.pqo_plugin_free(hn)
            oracle.lib.pqo_plugin_free(ht)
        assert np.array_equal(g.n_terms, o.n_terms), which
        assert_terms_equal(g.keys, g.coeffs, o.keys, o.coeffs)
        ok_e, err, tol = expectation_close(g.expectation, o)
        assert ok_e, which


class QubitLocalNoise:
    """A key-aware Python noise model (damping_factor_term), the same formula as
    the reference's qubit_local_noise example plugin."""

    def __init__(self, damping, mask):
        self.damping, self.mask = damping, mask
        self.calls = 0

    def damping_factor(self, term_weight, active_modes):  # pragma: no cover
        raise AssertionError("a key-aware model must not fall back to the weight path")

    def damping_factor_term(self, basis_kind, words, n_units, weight):
        self.calls += 1
        count = 0
        for q in range(min(n_units, 64)):
            if not (self.mask >> q) & 1:
                continue
            bit = 2 * q
            if bit // 64 >= len(words):
                break
            if (words[bit // 64] >> (bit % 64)) & 3:
                count += 1
        return math.exp(-self.damping * float(count))


def test_python_term_hook_matches_the_native_plugin(gpu_engine, oracle):
    so = REF_PLUGINS / "qubit_local_noise.so"
    if not so.exists():
        pytest.skip("reference example plugins not built")
    wl = workloads.tfim_chain(n=8, steps=3)
    model = QubitLocalNoise(0.05, 0b10110101)
    got = pq.PauliPropagator(noise=model, truncation=wl.truncation()).propagate(wl.observable, wl.circuit)
    assert model.calls > 0
    p = from_workload(wl)
    h = oracle.load_plugin(so, '{"damping": 0.05, "mask": 181}', noise=True)
    try:
        o = run_oracle(oracle, p, noise_plugin=h)
    finally:
        oracle.lib.pqo_plugin_free(h)
    want = {PauliString.from_key(int(k[0]), 8): c for k, c in zip(o.keys, o.coeffs)}
    assert dict(got.items()) == want


def test_python_term_hook_errors_propagate(gpu_engine):
    class Broken(QubitLocalNoise):
        def damping_factor_term(self, basis_kind, words, n_units, weight):
            raise KeyError("boom")

    wl = workloads.tfim_chain(n=6, steps=2)
    with pytest.raises(KeyError, match="boom"):
        pq.PauliPropagator(noise=Broken(0.1, 1)).expectation_value(wl.observable, wl.circuit, 0)


# ------------------------------------------------------------ random circuits
PAULI_CASES = [
    dict(n=6),
    dict(n=6, min_coeff=1e-3),
    dict(n=12, max_weight=4, min_coeff=1e-4),
    dict(n=20, max_weight=5, min_coeff=1e-5, min_terms=200),
    dict(n=40, max_weight=6, min_coeff=1e-4),       # W = 2
    dict(n=70, max_weight=6, min_coeff=1e-4),       # W = 4
    dict(n=130, max_weight=5, min_coeff=1e-3),      # W = 8
    dict(n=33, clifford_frac=0.5, max_weight=5),    # deferral-heavy, W = 2
]


@pytest.mark.parametrize("seed", [0, 1, 2])
@pytest.mark.parametrize("case", PAULI_CASES, ids=lambda c: "-".join(f"{k}{v}" for k, v in c.items()))
def test_random_pauli(gpu_engine, oracle, case, seed):
    case = dict(case)
    n = case.pop("n")
    cf = case.pop("clifford_frac", 0.15)
    p = random_pauli_problem(seed, n, clifford_frac=cf, **case)
    check(gpu_engine, oracle, p)


@pytest.mark.parametrize("seed", [0, 1])
def test_random_pauli_with_noise(gpu_engine, oracle, seed):
    p = random_pauli_problem(seed + 10, 24, n_gates=90, max_weight=5, min_coeff=1e-4)
    p.noise_table = np.array([math.exp(-0.02 * w) for w in range(p.n_units + 1)])
    check(gpu_engine, oracle, p)
    # noise without any truncation only scales (no reclaim); 10 qubits bound the growth
    q = random_pauli_problem(seed + 20, 10, n_gates=40)
    q.noise_table = np.array([math.exp(-0.02 * w) for w in range(q.n_units + 1)])
    check(gpu_engine, oracle, q)


@pytest.mark.parametrize("seed", [0, 1])
@pytest.mark.parametrize("n", [300, 700, 2048], ids=["W16", "W32", "W64"])
def test_wide_registers(gpu_engine, oracle, n, seed):
    # 16-, 32- and 64-word keys (257-2048 qubits): 12 active qubits spread
    # over the whole register, so keys and generators span every word.
    p = random_pauli_problem(seed, n, n_gates=80, units=spread_units(seed, n, 12), max_weight=6, min_coeff=1e-4)
    g, o = check(gpu_engine, oracle, p)
    assert max(g.n_terms) > 100


def random_majorana_problem(seed, n_sites, n_gates=50, sites=None, **kw):
    """Random Givens, number-number and single-mode rotations; with `sites`,
    gates and observable act on those sites only."""
    rng = np.random.default_rng(seed)
    n_modes = 2 * n_sites
    rots = []
    for _ in range(n_gates):
        kind = rng.random()
        pool = n_sites if sites is None else sites
        i, j = sorted(int(v) for v in rng.choice(pool, size=2, replace=False))
        if kind < 0.4:
            rots += pq.circuits.majorana_xx_plus_yy(i, j, float(rng.uniform(-math.pi, math.pi)), n_modes)
        elif kind < 0.8:
            rots += pq.circuits.majorana_cp(i, j, float(rng.normal(0, 0.5)), n_modes)
        else:  # an odd-length generator (exercises the odd anticommutation fold)
            m = 1 << (int(rng.integers(0, n_modes)) if sites is None else 2 * int(rng.choice(sites)) + int(rng.integers(0, 2)))
            rots.append(MajoranaRotation(MajoranaMonomial(m, n_modes, False), float(rng.uniform(-1, 1))))
    layers = [rots[k:k + 5] for k in range(0, len(rots), 5)]
    obs = MajoranaTermSum()
    for _ in range(4):
        s = int(rng.integers(0, n_sites)) if sites is None else int(rng.choice(sites))
        obs.add(MajoranaMonomial(3 << (2 * s), n_modes), float(rng.normal()))
    state = int(rng.integers(0, 1 << min(n_sites, 62)))
    if sites is not None:
        state |= sum(int(rng.integers(0, 2)) << int(q) for q in sites)
    return from_circuit(1, n_sites, obs, MajoranaCircuit(layers), state, **kw)


@pytest.mark.parametrize("seed", [0, 1, 2])
@pytest.mark.parametrize("case", [dict(n=6), dict(n=16, max_weight=6, min_coeff=1e-4),
                                  dict(n=32, max_weight=6, min_coeff=1e-4), dict(n=40, max_weight=5, min_coeff=1e-3)],
                         ids=lambda c: "-".join(f"{k}{v}" for k, v in c.items()))
def test_random_majorana(gpu_engine, oracle, case, seed):
    case = dict(case)
    n = case.pop("n")
    check(gpu_engine, oracle, random_majorana_problem(seed, n, **case))


@pytest.mark.parametrize("n", [400, 2048], ids=["W16", "W64"])
def test_wide_majorana(gpu_engine, oracle, n):
    check(gpu_engine, oracle, random_majorana_problem(3, n, n_gates=60, sites=spread_units(3, n, 9), max_weight=6,
                                                      min_coeff=1e-4))


def test_wide_registers_in_a_batch(gpu_engine, oracle):
    # A 64-word instance with 8-, 4- and 1-word ones: the narrow keys are
    # widened to the batch's width (results unchanged).
    probs = [random_pauli_problem(s, n, n_gates=60, units=spread_units(s, n, 10), max_weight=5, min_coeff=1e-4)
             for s, n in ((5, 2048), (6, 200), (7, 100), (8, 20))]
    from harness import run_gpu_batch

    for p, b in zip(probs, run_gpu_batch(gpu_engine, probs)):
        o = run_oracle(oracle, p)
        assert np.array_equal(b.n_terms, o.n_terms)
        assert_terms_equal(b.keys, b.coeffs, o.keys, o.coeffs)


# ------------------------------------------------------------ configurations
def test_config_tfim_chain(gpu_engine, oracle):
    check(gpu_engine, oracle, from_workload(workloads.tfim_chain()))


@pytest.mark.parametrize("shape", [(4, 4, 6), (6, 6, 8), (8, 8, 10)])
def test_config_kicked_ising_reduced(gpu_engine, oracle, shape):
    check(gpu_engine, oracle, from_workload(workloads.kicked_ising(*shape)), parts=4)


def test_config_majorana_givens_reduced(gpu_engine, oracle):
    check(gpu_engine, oracle, from_workload(workloads.majorana_givens(n_sites=16, reps=3)), parts=4)


# ------------------------------------------------------------ edge cases
def test_empty_observable_and_empty_circuit(gpu_engine, oracle):
    p = from_circuit(0, 5, PauliTermSum(), PauliCircuit([PauliRotation(PauliString(1, 0, 5), 0.3)]), 0)
    p.n_units = 5
    check(gpu_engine, oracle, p)
    obs = PauliTermSum({PauliString(0, 3, 5): 2.0, PauliString(1, 1, 5): -1.0})
    check(gpu_engine, oracle, from_circuit(0, 5, obs, PauliCircuit([]), 3))


def test_observable_truncated_at_admission_and_duplicates(gpu_engine, oracle):
    n = 8
    obs = PauliTermSum({PauliString(0xff, 0, n): 1.0, PauliString(1, 0, n): 1e-9, PauliString(0, 2, n): 0.5})
    circ = PauliCircuit([PauliRotation(PauliString(2, 0, n), 0.4)])
    check(gpu_engine, oracle, from_circuit(0, n, obs, circ, 0, max_weight=4, min_coeff=1e-6))
    # duplicate rows in the raw arrays fold by addition in order
    p = from_circuit(0, n, PauliTermSum({PauliString(0, 1, n): 0.1}), circ, 0)
    p.obs_keys = np.concatenate([p.obs_keys, p.obs_keys, p.obs_keys])
    p.obs_coeffs = np.array([0.1, 0.2, 0.3])
    check(gpu_engine, oracle, p)


def test_capacity_growth_and_engine_reuse(gpu_engine, oracle):
    # 8x8 kicked Ising grows past the initial 64 Ki-row capacity; a second run on
    # the same engine starts from a clean state and gives the same answer.
    p = from_workload(workloads.kicked_ising(8, 8, 10))
    a = run_gpu(gpu_engine, p)
    b = run_gpu(gpu_engine, p)
    assert a.res.peak_terms > 32768
    assert np.array_equal(a.n_terms, b.n_terms)
    assert_terms_equal(a.keys, a.coeffs, b.keys, b.coeffs)
    assert a.expectation == b.expectation


def test_capacity_stops_inside_fused_rotations(oracle):
    # A fresh engine starts at 64 Ki rows, so this run stops for capacity many
    # times, some of them between the two rotations of a fused pair (the second
    # then runs alone when the sweep resumes).
    from propaq_b200 import _native

    eng = _native.Engine(0)
    p = from_workload(workloads.kicked_ising(4, 4, 6))
    g = run_gpu(eng, p)
    o = run_oracle(oracle, p)
    assert g.res.sweep_launches > 3
    assert np.array_equal(g.n_terms, o.n_terms)
    assert_terms_equal(g.keys, g.coeffs, o.keys, o.coeffs)


@pytest.mark.parametrize("make", [lambda: workloads.kicked_ising(6, 6, 6),
                                  lambda: workloads.majorana_givens(n_sites=12, reps=2, seed=4)],
                         ids=["kicked6x6", "majorana12"])
def test_grid_follows_the_live_count(gpu_engine, oracle, make):
    # The default grid starts at one block per SM and the sweep stops and is
    # relaunched on a larger grid as the live count grows past 148 x 256 rows
    # (and past 2^20); a fixed grid runs without those stops.  Both give the
    # oracle's terms and counts.
    p = from_workload(make())
    run_gpu(gpu_engine, p)  # the engine's buffers grow to size here
    cfg, keep = make_cfg(p)
    auto = run_gpu(gpu_engine, p)
    cfg.blocks_per_sm = 3
    res, nt = gpu_engine.run(cfg, p.obs_keys, p.obs_coeffs, p.gate_keys, p.angles, p.offsets, p.diag)
    keys, coeffs = gpu_engine.terms(p.n_words)
    assert auto.res.peak_terms > 148 * 256
    assert auto.res.sweep_launches > res.sweep_launches, "the default grid must have grown during the run"
    o = run_oracle(oracle, p)
    for n_terms, k, c in ((auto.n_terms, auto.keys, auto.coeffs), (nt, keys, coeffs)):
        assert np.array_equal(n_terms, o.n_terms)
        assert_terms_equal(k, c, o.keys, o.coeffs)
    ok, _, _ = expectation_close(auto.expectation, o)
    assert ok


def test_six_block_build_on_a_large_live_set(gpu_engine):
    # Config 3 (32 sites, 99M live rows): past 2^24 rows the default grid
    # switches to the sweep built for six resident blocks per SM.  A fixed
    # grid (four blocks per SM, never that build) must give the same live
    # count after every gate and the same expectation value.
    p = from_workload(workloads.majorana_givens())
    cfg, keep = make_cfg(p, want_terms=False)
    auto, nt_auto = gpu_engine.run(cfg, p.obs_keys, p.obs_coeffs, p.gate_keys, p.angles, p.offsets, p.diag)
    cfg.blocks_per_sm = 4
    fixed, nt_fixed = gpu_engine.run(cfg, p.obs_keys, p.obs_coeffs, p.gate_keys, p.angles, p.offsets, p.diag)
    assert auto.peak_terms > 1 << 24
    assert auto.sweep_launches > fixed.sweep_launches
    assert np.array_equal(nt_auto, nt_fixed)
    assert auto.terms_below_cutoff == fixed.terms_below_cutoff
    assert abs(auto.expectation_value - fixed.expectation_value) <= 1e-13 * max(1.0, abs(fixed.expectation_value))


def test_width_errors(gpu_engine):
    big = PauliTermSum({PauliString(0, 1, 2049): 1.0})
    with pytest.raises(ValueError, match="exceeds the engine's maximum of 2048"):
        pq.PauliPropagator().expectation_value(big, PauliCircuit([]), 0)
    odd = MajoranaTermSum({MajoranaMonomial(3, 7): 1.0})
    with pytest.raises(ValueError):
        pq.MajoranaPropagator().expectation_value(odd, MajoranaCircuit([]), 0)


def test_propagate_returns_oracle_terms(gpu_engine, oracle):
    wl = workloads.tfim_chain(n=10, steps=3)
    out = pq.PauliPropagator(truncation=wl.truncation()).propagate(wl.observable, wl.circuit)
    o = run_oracle(oracle, from_workload(wl))
    want = {PauliString.from_key(int(k[0]), 10): c for k, c in zip(o.keys, o.coeffs)}
    assert dict(out.items()) == want


def test_op_times_on_a_fresh_engine():
    # A fresh engine grows its buffers inside fused pairs (a capacity stop
    # between the two rotations): every op still has its device time, so the
    # per-kind sums stay finite and no gate record is negative or huge.
    from propaq_b200 import _native as nat

    p = from_workload(workloads.kicked_ising(8, 8, 6))
    eng = nat.Engine(0)
    for _ in range(2):
        cfg, keep = make_cfg(p, want_terms=False)
        res, nt = eng.run(cfg, p.obs_keys, p.obs_coeffs, p.gate_keys, p.angles, p.offsets, p.diag)
        assert int(res.sweep_launches) >= 1
        total = res.gate_ms + res.noise_ms + res.phase_ms
        assert 0.0 < total < 1e4, (res.gate_ms, res.noise_ms, res.phase_ms)
        assert res.gate_ms <= 10.0 * res.device_ms + 10.0
