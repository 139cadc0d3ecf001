"""The verbose run log in the reference's schema (crates/pauli/src/propagator.rs:
23-101: `gate`, `truncation` and `engine_phases` events), read back by the
reference's own parser (propaq/log_parser.py) and checked against the oracle's
emit statistics.

The CPU test writes a log from synthetic gate records and parses it with the
reference's LogParser, loaded as a plain module from the reference tree
(PROPAQ_REFERENCE, skipped when the tree is absent).  The GPU test logs a real
run: per-gate live counts equal PropagationResult.n_terms, and the totals of
declined, emitted and claimed-onto-existing branches, the rows visited and the
discarded coefficient mass equal the oracle's counters."""

from __future__ import annotations

import importlib.util
import json
import sys
from pathlib import Path
from types import SimpleNamespace

import numpy as np
import pytest
from harness import from_circuit, run_oracle

from propaq_b200 import Logger, PauliPropagator, PauliString, PauliTermSum, WeightTruncator
from propaq_b200.circuits import PauliCircuit, PauliRotation
from propaq_b200.propagators import write_gate_log
from propaq_b200.truncation import CoefficientTruncator, resolve_config, resolve_truncation

from conftest import REFERENCE_TREE as REF


def reference_log_parser():
    path = REF / "propaq" / "log_parser.py"
    if not path.exists():
        pytest.skip("the reference tree is not present")
    spec = importlib.util.spec_from_file_location("ref_log_parser", path)
    mod = importlib.util.module_from_spec(spec)
    sys.modules[spec.name] = mod  # its dataclasses look their module up
    spec.loader.exec_module(mod)
    return mod


def fake_record(i):
    return SimpleNamespace(terms_before=10 + i, terms_after=12 + i, terms_gained=2, declined=i % 3, emitted=4,
                           exchange_hits=1, discarded_coeff_l1=1.5e-6 * i, discarded_coeff_max=1e-6,
                           elapsed_ms=0.0125 * (i + 1), layer_idx=i // 2, op=i)


def test_reference_parser_reads_the_log(tmp_path):
    mod = reference_log_parser()
    log = Logger(str(tmp_path / "run.jsonl"), log_every=2)
    recs = [fake_record(i) for i in range(7)]
    qidx = [None, 3, 5, None, 8, 9, 11]
    cfg = resolve_config(resolve_truncation([WeightTruncator(4), CoefficientTruncator(1e-4)]))
    res = SimpleNamespace(gate_ms=2.5, n_final=19, sum_anti=40)
    write_gate_log(log, recs, qidx, cfg, res)
    p = mod.LogParser(log.filename)
    gates = p.gate_events
    assert [g.gate_idx for g in gates] == [0, 2, 4, 6]
    assert [g.terms for g in gates] == [12, 14, 16, 18]
    assert [g.layer_idx for g in gates] == [0, 1, 2, 3]
    assert [g.qiskit_gate_idx for g in gates] == [None, 5, 8, 11]
    assert gates[1].ms_per_gate == pytest.approx(0.0375, rel=1e-3)
    tr = p.truncation_events
    assert [t.terms_discarded for t in tr] == [0, 2, 1, 0]
    assert tr[1].weight_cutoff == 4 and tr[1].coeff_cutoff == pytest.approx(1e-4)
    assert tr[2].discarded_coeff_l1 == pytest.approx(6e-6)
    (ph,) = p.engine_phases_events
    assert ph.partitions == 1 and ph.terms == 19 and ph.visited == 40
    assert ph.emitted == 28 and ph.exchange_hits == 7 and ph.declined == sum(i % 3 for i in range(7))


def test_log_without_weight_cut_writes_null(tmp_path):
    log = Logger(str(tmp_path / "run.jsonl"))
    cfg = resolve_config(resolve_truncation(None))
    write_gate_log(log, [fake_record(0)], [None], cfg, SimpleNamespace(gate_ms=0.0, n_final=1, sum_anti=0))
    lines = [json.loads(x) for x in Path(log.filename).read_text().splitlines()]
    assert lines[1]["weight_cutoff"] is None and lines[1]["coeff_cutoff"] == 0.0
    assert lines[0]["ms_per_gate"] == pytest.approx(0.0125, rel=1e-3)


@pytest.mark.gpu
def test_logged_run_matches_oracle_counters(oracle, tmp_path):
    rng = np.random.default_rng(3)
    n = 8
    rots = []
    for _ in range(60):
        x, z = int(rng.integers(0, 1 << n)), int(rng.integers(0, 1 << n))
        if x == 0 and z == 0:
            z = 1
        a = float(rng.uniform(-1.2, 1.2)) if rng.random() > 0.1 else np.pi / 2
        rots.append(PauliRotation(PauliString(x, z, n), a, qiskit_gate_idx=len(rots)))
    layers = [rots[k:k + 4] for k in range(0, len(rots), 4)]
    obs = PauliTermSum()
    obs.add(PauliString(0, 0b101, n), 1.0)
    obs.add(PauliString(0b10, 0b10, n), -0.5)
    log = Logger(str(tmp_path / "gpu.jsonl"))
    prop = PauliPropagator(truncation=[WeightTruncator(5), CoefficientTruncator(1e-3)], logger=log)
    res = prop.expectation_value(obs, PauliCircuit(layers), initial_state=0b1011)
    events = [json.loads(x) for x in Path(log.filename).read_text().splitlines()]
    gates = [e for e in events if e["event"] == "gate"]
    trunc = [e for e in events if e["event"] == "truncation"]
    (ph,) = [e for e in events if e["event"] == "engine_phases"]
    assert [g["terms"] for g in gates] == res.n_terms
    assert all(t["terms_after"] - t["terms_before"] == t["terms_gained"] for t in trunc)
    # Heisenberg order: the last circuit rotation comes first
    assert [g["qiskit_gate_idx"] for g in gates] == list(range(len(rots)))[::-1]
    p = from_circuit(0, n, obs, PauliCircuit(layers), 0b1011, max_weight=5, min_coeff=1e-3)
    o = run_oracle(oracle, p)
    assert ph["declined"] == o.stats["declined"] == sum(t["terms_discarded"] for t in trunc)
    assert ph["emitted"] == o.stats["emitted"]
    assert ph["exchange_hits"] == o.stats["hits"]
    assert ph["visited"] == o.stats["visited"]
    l1 = sum(t["discarded_coeff_l1"] for t in trunc)
    assert l1 == pytest.approx(o.stats["discarded_l1"], rel=1e-5)  # the log prints 7 digits
