"""The engine's radix sort by key and the folding of duplicate keys on the
device (propaq_b200/csrc/pq_sort.cu).

* Final terms requested in key order (want_terms = 2) come back sorted as
  64W-bit integers and are the same terms and coefficient bits as the
  engine's row order gives, for 1- to 8-word keys.
* An observable of at least 2^15 admitted terms folds its duplicate keys on
  the device: a stable sort by key, then each run of equal keys summed in
  input order.  The sums must round exactly as the host loop over the input
  (the reference's admission, crates/pauli/src/engine.rs:104-111) and the
  oracle do, so the whole propagation stays bit-identical to the oracle."""

from __future__ import annotations

import numpy as np
import pytest
from harness import (Problem, assert_terms_equal, expectation_close, random_pauli_problem, run_gpu, run_oracle,
                     spread_units, words_for)

from propaq_b200.propagators import heisenberg_gates, state_words

pytestmark = pytest.mark.gpu


def as_ints(keys):
    return [sum(int(w) << (64 * i) for i, w in enumerate(row)) for row in keys]


@pytest.mark.parametrize("n", [20, 50, 100, 200])
def test_sorted_terms(gpu_engine, n):
    p = random_pauli_problem(300 + n, n, n_gates=70, layer_size=6, max_weight=5, min_coeff=1e-5,
                             units=spread_units(n, n, 12))
    plain = run_gpu(gpu_engine, p)
    srt = run_gpu(gpu_engine, p, sort_terms=True)
    ints = as_ints(srt.keys)
    assert ints == sorted(ints) and len(set(ints)) == len(ints)
    assert_terms_equal(srt.keys, srt.coeffs, plain.keys, plain.coeffs)
    assert srt.expectation == plain.expectation


def big_observable(seed, n, n_terms, n_distinct):
    """n_terms raw terms over n_distinct keys (weight <= 4), random coefficients:
    most keys occur several times, in scattered input order."""
    rng = np.random.default_rng(seed)
    W = words_for(n)
    distinct = set()
    while len(distinct) < n_distinct:
        x = z = 0
        for q in rng.choice(n, size=int(rng.integers(1, 5)), replace=False):
            t = int(rng.integers(1, 4))
            x |= (t & 1) << int(q)
            z |= (t >> 1) << int(q)
        key = 0
        for q in range(n):
            key |= (x >> q & 1) << (2 * q) | (z >> q & 1) << (2 * q + 1)
        distinct.add(key)
    distinct = sorted(distinct)
    pick = rng.integers(0, n_distinct, size=n_terms)
    keys = np.array([[(distinct[i] >> (64 * w)) & ((1 << 64) - 1) for w in range(W)] for i in pick], dtype=np.uint64)
    coeffs = rng.normal(size=n_terms) * 10.0 ** rng.integers(-3, 2, size=n_terms)
    return keys, coeffs


@pytest.mark.parametrize("n,max_weight", [(24, 6), (100, 5)])
def test_device_fold_matches_oracle(gpu_engine, oracle, n, max_weight):
    base = random_pauli_problem(11 + n, n, n_gates=40, layer_size=4, max_weight=max_weight, min_coeff=1e-4)
    keys, coeffs = big_observable(n, n, 60000, 9000)
    p = Problem(0, n, base.n_words, keys, coeffs, base.gate_keys, base.angles, base.offsets,
                state_words(5, n), max_weight, 1e-4, name="fold")
    g = run_gpu(gpu_engine, p, sort_terms=True)
    o = run_oracle(oracle, p)
    assert np.array_equal(g.n_terms, o.n_terms)
    assert_terms_equal(g.keys, g.coeffs, o.keys, o.coeffs)
    assert expectation_close(g.expectation, o)[0]
