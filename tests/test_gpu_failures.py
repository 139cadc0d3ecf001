"""Failure paths of the engine, exercised without faulting, trapping or hanging
the GPU (the reference's counterparts: the term index ceiling of
crates/core/src/storage/operator_index.rs:116-127 raising RuntimeError, and
allocation failure).

Each test uses an engine of its own, provokes one failure through
pq_engine_set_limits, checks the error the Python layer raises, then restores
the defaults and checks that the same engine gives the oracle's answer:
  * a row ceiling below the run's live count -> PQ_ERR_CEILING -> RuntimeError;
  * a device-memory budget below what the run's growth needs -> PQ_ERR_OOM ->
    MemoryError;
  * a grid-barrier wait limit of a few polls while one block holds back before
    its first op -> the other blocks' waits run out -> PQ_ERR_DEVICE_TIMEOUT;
  * the same for the look-back wait of the first gate's tiles.
Every device wait is bounded (the hold itself is a bounded wait of 20 ms); the
kernels return and the host reads the error bits."""

from __future__ import annotations

import numpy as np
import pytest
from harness import assert_terms_equal, from_circuit, from_workload, run_gpu, run_oracle

from propaq_b200 import _native, workloads
from propaq_b200.circuits import PauliCircuit
from propaq_b200.datatypes import PauliString, PauliTermSum

pytestmark = pytest.mark.gpu


@pytest.fixture
def engine():
    e = _native.Engine(0)
    yield e
    del e


def tfim():
    return from_workload(workloads.tfim_chain(20, 10))


def check_recovers(engine, oracle, p):
    engine.set_limits()
    g = run_gpu(engine, p)
    o = run_oracle(oracle, p)
    assert np.array_equal(g.n_terms, o.n_terms)
    assert_terms_equal(g.keys, g.coeffs, o.keys, o.coeffs)


def test_row_ceiling_raises_runtime_error(engine, oracle):
    p = tfim()  # peaks near 31k live terms
    engine.set_limits(max_rows=4096)
    with pytest.raises(RuntimeError, match="ceiling"):
        run_gpu(engine, p)
    check_recovers(engine, oracle, p)


def test_device_memory_budget_raises_memory_error(engine, oracle):
    p = from_workload(workloads.kicked_ising(10, 10, 8))  # grows to ~476k rows of 4-word keys
    engine.set_limits(max_device_bytes=8 << 20)
    with pytest.raises(MemoryError):
        run_gpu(engine, p, want_terms=False)
    assert engine.device_bytes() <= 8 << 20
    check_recovers(engine, oracle, tfim())


def test_barrier_wait_limit_raises_device_timeout(engine, oracle):
    p = tfim()
    engine.set_limits(barrier_spins=32, hold_block=1, hold_us=20000)
    with pytest.raises(RuntimeError, match="grid barrier wait expired"):
        run_gpu(engine, p)
    check_recovers(engine, oracle, p)


def test_lookback_wait_limit_raises_device_timeout(engine, oracle):
    # 300 observable terms: the first gate has two tiles, and tile 1's look-back
    # waits on tile 0, whose block holds back.
    n = 20
    obs = PauliTermSum()
    rng = np.random.default_rng(5)
    for z in rng.choice(1 << n, size=300, replace=False):
        obs.add(PauliString(0, int(z) | 1, n), float(rng.normal()))
    circ = workloads.tfim_chain(n, 3).circuit
    p = from_circuit(0, n, obs, PauliCircuit(circ.layers), 0, max_weight=8, min_coeff=1e-4)
    engine.set_limits(lookback_spins=32, hold_block=0, hold_us=20000)
    with pytest.raises(RuntimeError, match="look-back wait expired"):
        run_gpu(engine, p)
    check_recovers(engine, oracle, p)
