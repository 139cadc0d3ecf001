"""Glue between the parity tests and the surrogate restatement in
oracle/pq_surrogate.py: problems in the tests' layout (interleaved u64 key
words, gates in Heisenberg order) become surrogate builds, and the C oracle's
algebra probes back the Majorana keys."""

from __future__ import annotations

import importlib.util
import math
from pathlib import Path

import numpy as np

_spec = importlib.util.spec_from_file_location(
    "pq_surrogate", Path(__file__).resolve().parent.parent / "oracle" / "pq_surrogate.py")
sur = importlib.util.module_from_spec(_spec)
_spec.loader.exec_module(sur)


def to_int(words) -> int:
    return sum(int(w) << (64 * i) for i, w in enumerate(np.asarray(words, dtype=np.uint64).ravel()))


def to_words(k: int, n_words: int) -> np.ndarray:
    return np.array([(k >> (64 * i)) & 0xFFFFFFFFFFFFFFFF for i in range(n_words)], dtype=np.uint64)


class OracleAlgebra:
    """The C oracle's key algebra (Pauli or Majorana) behind the surrogate's
    four-method interface."""

    def __init__(self, oracle, basis, n_units, n_words):
        self.o, self.basis, self.n_units, self.n_words = oracle, basis, n_units, n_words

    def anticommutes(self, g, k):
        return self.o.anticommutes(self.basis, to_words(g, self.n_words), to_words(k, self.n_words))

    def product(self, g, k):
        child, p = self.o.product(self.basis, to_words(g, self.n_words), to_words(k, self.n_words))
        return to_int(child), p

    def weight(self, k):
        return self.o.weight(self.basis, self.n_units, to_words(k, self.n_words))

    def trace(self, k, state):
        return self.o.trace(self.basis, self.n_units, to_words(k, self.n_words), to_words(state, self.n_words))


def algebra_for(p, oracle=None):
    if p.basis == 0 and oracle is None:
        return sur.PauliAlgebra(p.n_units)
    return OracleAlgebra(oracle, p.basis, p.n_units, p.n_words)


def surrogate_params(p):
    """One parameter per gate (its Heisenberg index); gates at a Clifford
    angle stay numeric, as the engine defers them into its frame."""
    params = []
    for g, a in enumerate(p.angles):
        params.append(("num", float(a)) if abs(math.cos(a)) < sur.EPS else ("sym", g))
    return params


def build_surrogate(p, oracle=None, params=None, **trunc):
    """The surrogate model of problem `p`; its parameter g is gate g's angle."""
    alg = algebra_for(p, oracle)
    obs = [(to_int(k), float(c)) for k, c in zip(p.obs_keys.reshape(-1, p.n_words), p.obs_coeffs)]
    params = surrogate_params(p) if params is None else params
    gates = [(to_int(k), prm) for k, prm in zip(p.gate_keys.reshape(-1, p.n_words), params)]
    state = 0 if p.diag is None else to_int(p.diag)
    return sur.build(alg, p.n_units, 64 * p.n_words, obs, gates, initial_state=state, n_params=len(p.angles), **trunc)
