"""Parity at the benchmarked sizes: the full kicked-Ising 10x10 run (20 steps,
p = 1e-3, w <= 10, |c| >= 1e-5; 100 qubits, 4-word keys, ~476k peak live terms)
and the full 32-site Majorana Givens run (4 repetitions, w <= 8, |c| >= 1e-6;
~99M peak live terms), each against the oracle run on every host core.

Required, bit for bit: the live count after every gate, terms_below_cutoff,
the final term set and every final coefficient.  The expectation value is an
order-dependent sum (double-double on the device, compensated on the host);
its plain relative error against the oracle is printed and must be below
1e-12, the tolerance the engine is built to."""

from __future__ import annotations

import os

import numpy as np
import pytest
from harness import from_workload, run_gpu, run_oracle

from propaq_b200 import workloads

pytestmark = pytest.mark.gpu


def sorted_w1(keys, coeffs):
    order = np.argsort(keys[:, 0], kind="stable")
    return keys[order, 0], coeffs[order]


def check_full(gpu_engine, oracle, wl, label):
    p = from_workload(wl)
    g = run_gpu(gpu_engine, p)
    o = run_oracle(oracle, p, n_partitions=os.cpu_count() or 1)
    assert np.array_equal(g.n_terms, o.n_terms), "per-gate live counts differ"
    assert g.terms_below_cutoff == o.terms_below_cutoff
    assert g.n_final == o.n_final == len(o.coeffs)
    if p.n_words == 1:
        gk, gc = sorted_w1(g.keys, g.coeffs)
        ok, oc = sorted_w1(o.keys, o.coeffs)
    else:
        og = np.lexsort(g.keys.T[::-1])
        oo = np.lexsort(o.keys.T[::-1])
        gk, gc, ok, oc = g.keys[og], g.coeffs[og], o.keys[oo], o.coeffs[oo]
    assert np.array_equal(gk, ok), "term sets differ"
    bad = np.count_nonzero(gc.view(np.uint64) != oc.view(np.uint64))
    assert bad == 0, f"{bad} of {len(gc)} coefficients differ bit-wise"
    ref = o.expectation_accurate
    rel = abs(g.expectation - ref) / abs(ref)
    print(f"{label}: {g.n_final} final terms identical; peak {int(g.res.peak_terms)}; E = {g.expectation!r}, "
          f"oracle {ref!r}, relative error {rel:.3e}")
    assert rel <= 1e-12


def test_kicked_ising_10x10_full_size(gpu_engine, oracle):
    check_full(gpu_engine, oracle, workloads.kicked_ising(10, 10, 20), "kicked Ising 10x10 s20")


def test_majorana_givens_32_sites_full_size(gpu_engine, oracle):
    check_full(gpu_engine, oracle, workloads.majorana_givens(32, 4), "Majorana Givens 32 sites x4")
