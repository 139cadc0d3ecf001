"""Shared problem builders and comparisons for the parity tests."""

from __future__ import annotations

import json
import math
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

from propaq_b200 import _native
from propaq_b200.circuits import PauliCircuit, PauliRotation
from propaq_b200.datatypes import PauliString, PauliTermSum
from propaq_b200.propagators import heisenberg_gates, state_words

GOLDEN = Path(__file__).resolve().parent / "golden"


def words_for(n_units: int) -> int:
    w = 1
    while 32 * w < n_units:
        w *= 2
    return w


@dataclass
class Problem:
    basis: int
    n_units: int
    n_words: int
    obs_keys: np.ndarray
    obs_coeffs: np.ndarray
    gate_keys: np.ndarray
    angles: np.ndarray
    offsets: np.ndarray
    diag: np.ndarray | None
    max_weight: int | None = None
    min_coeff: float | None = None
    min_terms: int | None = None
    noise_table: np.ndarray | None = None
    noise_tables_layered: np.ndarray | None = None
    name: str = ""
    meta: dict = field(default_factory=dict)

    @property
    def n_gates(self):
        return len(self.angles)


def from_workload(wl, min_terms=None) -> Problem:
    n_words = words_for(wl.n_units)
    ok, oc = wl.observable.to_arrays(n_words)
    gk, ga, off = heisenberg_gates(wl.circuit, n_words, lambda g: g.key())
    table = None
    if wl.noise_damping is not None:
        table = np.array([math.exp(-wl.noise_damping * float(w)) for w in range(wl.n_units + 1)])
    return Problem(wl.basis, wl.n_units, n_words, ok, oc, gk, ga, off, state_words(wl.initial_state, wl.n_units),
                   wl.max_weight, wl.min_coeff, min_terms, table, name=wl.name)


def from_circuit(basis, n_units, observable, circuit, initial_state=0, **kw) -> Problem:
    n_words = words_for(n_units)
    ok, oc = observable.to_arrays(n_words)
    gk, ga, off = heisenberg_gates(circuit, n_words, lambda g: g.key())
    diag = None if initial_state is None else state_words(initial_state, n_units)
    return Problem(basis, n_units, n_words, ok, oc, gk, ga, off, diag, **kw)


def golden_fixture():
    return json.loads((GOLDEN / "plugin_notebooks.json").read_text())


def golden_problem(**kw) -> Problem:
    """The plugin notebooks' 4-qubit, 40-rotation circuit, one rotation per layer."""
    fx = golden_fixture()
    n = fx["n_qubits"]
    circ = PauliCircuit([PauliRotation(PauliString(r["x"], r["z"], n), r["angle"]) for r in fx["rotations"]])
    obs = PauliTermSum()
    obs.add(PauliString(fx["observable"]["x"], fx["observable"]["z"], n), fx["observable"]["coeff"])
    return from_circuit(0, n, obs, circ, fx["initial_state"], **kw)


def run_oracle(oracle, p: Problem, n_partitions=1, **kw):
    return oracle.run(p.basis, p.n_units, p.n_words, p.obs_keys, p.obs_coeffs, p.gate_keys, p.angles, p.offsets,
                      max_weight=p.max_weight, min_coeff=p.min_coeff, min_terms=p.min_terms,
                      noise_table=p.noise_table, noise_tables_layered=p.noise_tables_layered, diag_state=p.diag,
                      n_partitions=n_partitions, **kw)


class GpuResult:
    def __init__(self, res, nt, keys, coeffs):
        self.expectation = res.expectation_value
        self.terms_below_cutoff = int(res.terms_below_cutoff)
        self.n_final = int(res.n_final)
        self.n_terms = nt
        self.keys = keys
        self.coeffs = coeffs
        self.res = res


def make_cfg(p: Problem, want_terms=True, noise_plugin=None, truncator=None, sort_terms=False):
    """The RunConfig of a problem and the arrays it points into."""
    cfg = _native.RunConfig()
    cfg.basis_kind = p.basis
    cfg.n_units = p.n_units
    cfg.max_weight = -1 if p.max_weight is None else p.max_weight
    cfg.has_min_coeff = 0 if p.min_coeff is None else 1
    cfg.min_coeff = 0.0 if p.min_coeff is None else p.min_coeff
    cfg.min_terms = -1 if p.min_terms is None else p.min_terms
    keep = []
    if p.noise_table is not None:
        t = np.ascontiguousarray(p.noise_table, dtype=np.float64)
        keep.append(t)
        cfg.noise_kind, cfg.noise_tables, cfg.noise_table_len = _native.PQ_NOISE_TABLE, t.ctypes.data, len(t)
    elif p.noise_tables_layered is not None:
        t = np.ascontiguousarray(p.noise_tables_layered, dtype=np.float64)
        keep.append(t)
        cfg.noise_kind, cfg.noise_tables, cfg.noise_table_len = _native.PQ_NOISE_LAYERED, t.ctypes.data, t.shape[1]
    elif noise_plugin is not None:
        cfg.noise_kind, cfg.noise_plugin = _native.PQ_NOISE_PLUGIN, noise_plugin
    cfg.truncator = truncator
    cfg.want_terms = (2 if sort_terms else 1) if want_terms else 0
    return cfg, keep


def run_gpu(engine, p: Problem, want_terms=True, noise_plugin=None, truncator=None, sort_terms=False) -> GpuResult:
    """pq_run; sort_terms asks the engine for its final terms in key order."""
    cfg, keep = make_cfg(p, want_terms, noise_plugin, truncator, sort_terms)
    res, nt = engine.run(cfg, p.obs_keys, p.obs_coeffs, p.gate_keys, p.angles, p.offsets, p.diag)
    keys = coeffs = None
    if want_terms:
        keys, coeffs = engine.terms(p.n_words)
    return GpuResult(res, nt, keys, coeffs)


def run_gpu_batch(engine, problems, want_terms=True, **tuning) -> list[GpuResult]:
    """All problems in one pq_run_batch call."""
    items, keep = [], []
    for p in problems:
        cfg, k = make_cfg(p, want_terms)
        keep.append(k)
        items.append((cfg, p.obs_keys, p.obs_coeffs, p.gate_keys, p.angles, p.offsets, p.diag))
    out = engine.run_batch(items, **tuning)
    results = []
    for i, (p, (res, nt)) in enumerate(zip(problems, out)):
        keys = coeffs = None
        if want_terms:
            keys, coeffs = engine.terms(p.n_words, index=i)
        results.append(GpuResult(res, nt, keys, coeffs))
    return results


def sorted_terms(keys: np.ndarray, coeffs: np.ndarray):
    order = np.lexsort(keys.T[::-1]) if len(keys) else np.arange(0)
    return keys[order], coeffs[order]


def assert_terms_equal(gk, gc, ok, oc, exact=True, rtol=1e-12):
    gk, gc = sorted_terms(gk, gc)
    ok, oc = sorted_terms(ok, oc)
    assert gk.shape == ok.shape, f"term count differs: gpu {len(gk)} vs oracle {len(ok)}"
    assert np.array_equal(gk, ok), "term sets differ"
    if exact:
        bad = np.nonzero(gc != oc)[0]
        assert len(bad) == 0, (f"{len(bad)} coefficients differ bit-wise; first: key {gk[bad[0]]} "
                               f"gpu {gc[bad[0]]!r} oracle {oc[bad[0]]!r}")
    else:
        np.testing.assert_allclose(gc, oc, rtol=rtol, atol=0)


def expectation_close(gpu_value, oracle_result, rel=1e-12):
    """|gpu - oracle| <= rel * |oracle| + 4 eps * sum|c * trace| : both sums are
    compensated, so only their last-bit rounding may differ."""
    ref = oracle_result.expectation_accurate
    tol = rel * abs(ref) + 4 * np.finfo(float).eps * oracle_result.expectation_abs
    return abs(gpu_value - ref) <= tol, abs(gpu_value - ref), tol


def spread_units(seed, n, k):
    """k units spread over a register of n: one in each of k equal stretches."""
    rng = np.random.default_rng(1000 + seed)
    edges = np.linspace(0, n, k + 1).astype(int)
    return [int(rng.integers(edges[i], edges[i + 1])) for i in range(k)]


def random_pauli_problem(seed, n, n_gates=60, layer_size=4, clifford_frac=0.15, units=None, **kw):
    """Random rotations on 1-3 qubits; with `units`, gates and observable act
    on those qubits only (a few qubits spread over a wide register)."""
    rng = np.random.default_rng(seed)
    layers, layer = [], []
    for _ in range(n_gates):
        k = int(rng.integers(1, 4))
        qs = rng.choice(n, size=k, replace=False) if units is None else rng.choice(units, size=k, replace=False)
        x = z = 0
        for q in qs:
            t = int(rng.integers(1, 4))
            x |= (t & 1) << int(q)
            z |= (t >> 1) << int(q)
        r = rng.random()
        if r < clifford_frac:
            a = float(rng.choice([math.pi / 2, -math.pi / 2, 3 * math.pi / 2]))
        elif r < clifford_frac + 0.05:
            a = math.pi
        else:
            a = float(rng.uniform(-1.2, 1.2))
        layer.append(PauliRotation(PauliString(x, z, n), a))
        if len(layer) == layer_size:
            layers.append(layer)
            layer = []
    if layer:
        layers.append(layer)
    obs = PauliTermSum()
    pick = (lambda: int(rng.integers(0, n))) if units is None else (lambda: int(rng.choice(units)))
    for _ in range(3):
        q = pick()
        obs.add(PauliString(0, 1 << q, n), float(rng.normal()))
    obs.add(PauliString(0, (1 << pick()) | (1 if units is None else 1 << int(units[0])), n), 0.5)
    state = int(rng.integers(0, 1 << min(n, 62)))
    if units is not None:
        state |= sum(int(rng.integers(0, 2)) << int(q) for q in units)
    return from_circuit(0, n, obs, PauliCircuit(layers), state, **kw)
