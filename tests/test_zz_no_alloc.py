"""pq_expectation_noalloc: the expectation value for callers that may not
allocate device memory (programs that own the whole GPU's memory, such as
frameworks that preallocate it for their own allocators).

The entry point stages the caller's host terms into a static device array and
reduces them there.  Its value must match the expectation pq_run computes for
the same final terms, on two calls in a row (the array keeps the previous
call's contents).  This file is collected last so that a failure here leaves
every other test already run; it passes alone in a fresh process as well."""

import ctypes
import math

import numpy as np
import pytest
from harness import expectation_close, golden_problem, run_gpu, run_oracle

from propaq_b200 import _native

pytestmark = pytest.mark.gpu

SCRATCH_BYTES = 16 << 20


def noalloc(basis, n_units, keys, coeffs, diag):
    lib = _native.lib()
    fn = lib.pq_expectation_noalloc
    fn.restype = ctypes.c_int
    V, Z = ctypes.c_void_p, ctypes.c_size_t
    fn.argtypes = [ctypes.c_uint32, ctypes.c_uint32, V, V, Z, V, Z, ctypes.POINTER(ctypes.c_double),
                   ctypes.c_char_p, Z]
    keys = np.ascontiguousarray(keys, dtype=np.uint64)
    coeffs = np.ascontiguousarray(coeffs, dtype=np.float64)
    diag = np.ascontiguousarray(diag, dtype=np.uint64)
    out = ctypes.c_double(float("nan"))
    err = ctypes.create_string_buffer(512)
    rc = fn(basis, n_units, keys.ctypes.data if len(coeffs) else None, coeffs.ctypes.data if len(coeffs) else None,
            len(coeffs), diag.ctypes.data, len(diag), ctypes.byref(out), err, 512)
    return rc, out.value, err.value.decode()


def test_noalloc_expectation_matches_pq_run_twice(gpu_engine, oracle):
    p = golden_problem(max_weight=3, min_coeff=1e-5)
    p.noise_table = np.array([math.exp(-0.01 * w) for w in range(p.n_units + 1)])
    g = run_gpu(gpu_engine, p)  # the existing entry point: pq_run with its terms
    o = run_oracle(oracle, p)
    for _ in range(2):
        rc, value, msg = noalloc(p.basis, p.n_units, g.keys, g.coeffs, p.diag)
        assert rc == 0, msg
        ok, err, tol = expectation_close(value, o)
        assert ok, f"no-alloc {value!r} vs oracle {o.expectation_accurate!r}"
        assert abs(value - g.expectation) <= 1e-12 * abs(g.expectation) + 4 * np.finfo(float).eps * o.expectation_abs


def test_noalloc_expectation_majorana_and_refusal(gpu_engine, oracle):
    from harness import from_workload

    from propaq_b200 import workloads

    p = from_workload(workloads.majorana_givens(n_sites=10, reps=2))
    g = run_gpu(gpu_engine, p)
    o = run_oracle(oracle, p)
    for _ in range(2):
        rc, value, msg = noalloc(p.basis, p.n_units, g.keys, g.coeffs, p.diag)
        assert rc == 0, msg
        assert expectation_close(value, o)[0]
    # more terms than the static scratch holds are refused before any device work
    n = SCRATCH_BYTES // 16
    rc, _, msg = noalloc(0, 20, np.zeros((n, 1), np.uint64), np.zeros(n), np.zeros(1, np.uint64))
    assert rc == _native.PQ_ERR_INVALID and "static scratch" in msg


@pytest.mark.parametrize("n_units,basis", [(50, 0), (100, 0), (200, 0), (48, 1), (100, 1)])
def test_noalloc_every_key_width(gpu_engine, oracle, n_units, basis):
    """2-, 4- and 8-word keys (Pauli 50 / 100 / 200 qubits, Majorana 48 / 100
    sites) against pq_run's expectation of the same final terms and the
    oracle's, on two calls in a row."""
    from harness import from_workload, random_pauli_problem, spread_units

    from propaq_b200 import workloads

    if basis == 0:
        # a dozen active qubits spread over the register, so keys use every word
        p = random_pauli_problem(40 + n_units, n_units, n_gates=70, layer_size=6, max_weight=5, min_coeff=1e-5,
                                 units=spread_units(n_units, n_units, 12))
    else:
        p = from_workload(workloads.majorana_givens(n_sites=n_units, reps=1, max_weight=5, min_coeff=1e-5))
    assert p.n_words == {50: 2, 100: 4, 200: 8, 48: 2}[n_units]
    g = run_gpu(gpu_engine, p)
    o = run_oracle(oracle, p)
    assert len(g.coeffs) > 1
    for _ in range(2):
        rc, value, msg = noalloc(p.basis, p.n_units, g.keys, g.coeffs, p.diag)
        assert rc == 0, msg
        assert expectation_close(value, o)[0], (value, o.expectation_accurate)
        assert abs(value - g.expectation) <= 1e-12 * abs(g.expectation) + 4 * np.finfo(float).eps * o.expectation_abs


def test_noalloc_zero_terms_and_unit_limit(gpu_engine):
    """No terms give 0.0; more than 256 units are refused before any device work."""
    rc, value, msg = noalloc(0, 20, np.zeros((0, 1), np.uint64), np.zeros(0), np.zeros(1, np.uint64))
    assert rc == 0 and value == 0.0, msg
    rc, _, msg = noalloc(1, 257, np.zeros((1, 16), np.uint64), np.ones(1), np.zeros(5, np.uint64))
    assert rc == _native.PQ_ERR_INVALID and "256-unit" in msg
