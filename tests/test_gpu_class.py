"""Class ops: runs of rotations whose generators act on disjoint qubits, each
family of keys run through all of its rotations in one pass (class_op).

Every result is compared with the oracle, which applies the reference's steps
one rotation at a time: the live count after every rotation, the term set,
every coefficient bit for bit, terms_below_cutoff and the expectation value.
Cases: layers of two-qubit Clifford rotations on disjoint pairs (classes)
between layers of generic rotations, with coefficient and weight cuts, with
and without noise (lone and multi-member families, pair rescue, held and
dropped branches); the kicked Ising workload; a fresh engine whose buffers
grow inside class ops; the TFIM chain (generic angles: no class is formed);
and a weight cut above the class limit (no class)."""

from __future__ import annotations

import math

import numpy as np
import pytest
from harness import assert_terms_equal, expectation_close, from_circuit, from_workload, run_gpu, run_oracle

from propaq_b200 import _native, workloads
from propaq_b200.circuits import PauliCircuit, PauliRotation
from propaq_b200.datatypes import PauliString, PauliTermSum

pytestmark = pytest.mark.gpu


def check(engine, oracle, p, want_classes=True):
    g = run_gpu(engine, p)
    o = run_oracle(oracle, p)
    assert np.array_equal(g.n_terms, o.n_terms), "per-gate live counts differ"
    assert g.terms_below_cutoff == o.terms_below_cutoff
    assert_terms_equal(g.keys, g.coeffs, o.keys, o.coeffs)
    assert expectation_close(g.expectation, o)[0]
    if want_classes is not None:
        assert (int(g.res.class_ops) > 0) == want_classes, int(g.res.class_ops)
    return g


def pair_layers(seed, n, n_layers):
    """Even layers: two-qubit Clifford rotations (angle +-pi/2, random Pauli
    types) on disjoint qubit pairs -- they change weight, so with a weight cut
    they stay out of the Clifford frame and form classes.  Odd layers: generic
    one- and two-qubit rotations on disjoint supports (pair-fused ops), which
    make the families of the next class hold several members."""
    rng = np.random.default_rng(seed)
    layers = []
    for li in range(n_layers):
        perm = rng.permutation(n)
        layer, i = [], 0
        while i < n:
            size = 2 if (li % 2 == 0 and i + 1 < n) else (1 if (i == n - 1 or rng.random() < 0.5) else 2)
            x = z = 0
            for q in perm[i:i + size]:
                t = int(rng.integers(1, 4))
                x |= (t & 1) << int(q)
                z |= (t >> 1) << int(q)
            if li % 2 == 0:
                a = float(rng.choice([math.pi / 2, -math.pi / 2]))
            else:
                a = float(rng.uniform(-1.5, 1.5)) if rng.random() > 0.1 else float(rng.uniform(-1e-3, 1e-3))
            layer.append(PauliRotation(PauliString(x, z, n), a))
            i += size
        layers.append(layer)
    return layers


def random_obs(seed, n, k=4, max_w=3):
    rng = np.random.default_rng(seed + 99)
    obs = PauliTermSum()
    for _ in range(k):
        x = z = 0
        for q in rng.choice(n, size=int(rng.integers(1, max_w + 1)), replace=False):
            t = int(rng.integers(1, 4))
            x |= (t & 1) << int(q)
            z |= (t >> 1) << int(q)
        obs.add(PauliString(x, z, n), float(rng.normal()))
    return obs


@pytest.mark.parametrize("seed", range(12))
def test_random_disjoint_layers(gpu_engine, oracle, seed):
    n = [12, 20, 40, 64][seed % 4]
    wcut = [4, 6, 8, 10][(seed // 4) % 4]
    ccut = [1e-3, 1e-4, 1e-5][seed % 3]
    p = from_circuit(0, n, random_obs(seed, n), PauliCircuit(pair_layers(seed, n, 7)),
                     int(np.random.default_rng(seed).integers(0, 1 << min(n, 60))), max_weight=wcut, min_coeff=ccut)
    if seed % 2:
        p.noise_table = np.array([math.exp(-0.02 * w) for w in range(n + 1)])
    check(gpu_engine, oracle, p)


def test_kicked_ising_and_tfim(gpu_engine, oracle):
    check(gpu_engine, oracle, from_workload(workloads.kicked_ising(6, 6, 8)))
    check(gpu_engine, oracle, from_workload(workloads.tfim_chain(20, 10)), want_classes=False)


def test_growth_inside_class_ops():
    """A fresh engine starts with 2^16 rows; the kicked-Ising 10x10 run grows
    to ~476k live terms, so class ops stop for capacity and run again."""
    from oracle_client import Oracle

    engine = _native.Engine(0)
    check(engine, Oracle.load(), from_workload(workloads.kicked_ising(10, 10, 6)))


def test_no_class_above_the_weight_limit(gpu_engine, oracle):
    wl = workloads.kicked_ising(5, 5, 6, max_weight=12)
    check(gpu_engine, oracle, from_workload(wl), want_classes=False)
