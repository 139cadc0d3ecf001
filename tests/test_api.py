"""Host-side logic of the product that needs no GPU: the C ABI library loads
and exports every declared symbol, plugin loading and its errors, the term
types' algebra against the oracle, truncation/noise resolution, term files."""

import ctypes
import gzip
import math
import re
import struct
from pathlib import Path

import numpy as np
import pytest
from plugin_build import build_all

import propaq_b200 as pq
from propaq_b200 import _native
from propaq_b200.datatypes import MajoranaMonomial, PauliString, jw_weight
from propaq_b200.propagators import heisenberg_gates, state_words
from propaq_b200.truncation import resolve_config, resolve_truncation

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "propaq_cuda.h"


@pytest.fixture(scope="module")
def plugins(tmp_path_factory):
    return build_all(tmp_path_factory.mktemp("plugins"))


def declared_functions():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:[\w\*]+\s+)+\**(pq_\w+)\s*\(", text, re.M)))


def test_library_exports_every_declared_symbol():
    lib = _native.lib()
    names = declared_functions()
    assert len(names) >= 12
    for n in names:
        assert hasattr(lib, n), f"libpropaq_cuda.so does not export {n}"


def test_words_for_units_dispatch_ladder():
    # crates/pauli/src/engine.rs:289-301
    want = {1: 1, 32: 1, 33: 2, 64: 2, 65: 4, 128: 4, 129: 8, 256: 8, 512: 16, 1024: 32, 2048: 64, 2049: 0}
    for n, w in want.items():
        assert _native.words_for_units(n) == w


def test_engine_without_gpu_fails_loudly():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(_native.EngineUnavailable):
        _native.Engine(0)
    with pytest.raises(_native.EngineUnavailable):
        pq.PauliPropagator().expectation_value(
            pq.PauliTermSum({PauliString(0, 1, 2): 1.0}), pq.PauliCircuit([]), 0)


def test_plugin_loads_and_reports(plugins):
    m = pq.NativeNoiseModel(str(plugins["uniform"]), '{"damping": 0.5}')
    assert m.depends == 0 and m.abi_version == 1
    assert m.factor_term(0, [], 4, 2) == math.exp(-0.5 * 2)
    lay = pq.NativeNoiseModel(str(plugins["layered"]), '{"damping": 0.5}')
    assert lay.depends == 2
    t = pq.NativeTruncator(str(plugins["truncator"]), '{"max_weight": 3}')
    assert t.keep_term(0, [], 4, 3, 1.0) and not t.keep_term(0, [], 4, 4, 1.0)


def test_plugin_errors(plugins, tmp_path):
    # crates/core/src/policy/native_noise.rs:217-260 error kinds and messages
    with pytest.raises(OSError, match="failed to load noise plugin"):
        pq.NativeNoiseModel(str(tmp_path / "missing.so"))
    with pytest.raises(ValueError, match="targets ABI version 2, expected 1"):
        pq.NativeNoiseModel(str(plugins["bad_abi"]))
    with pytest.raises(ValueError, match="unknown dependency bits 0x4"):
        pq.NativeNoiseModel(str(plugins["unknown_depends"]))
    with pytest.raises(ValueError, match="does not export propaq_noise_factor"):
        pq.NativeNoiseModel(str(plugins["no_factor"]))
    with pytest.raises(ValueError, match="must export both propaq_noise_create and propaq_noise_destroy"):
        pq.NativeNoiseModel(str(plugins["no_destroy"]))
    with pytest.raises(ValueError, match="basis_kind must be 0"):
        pq.NativeNoiseModel(str(plugins["uniform"])).factor_term(2, [], 4, 1)


def test_truncation_resolution():
    assert resolve_truncation(None) == []
    pol = pq.TruncationPolicy(weight_cutoff=3, coeff_cutoff=1e-4, min_terms=10)
    cfg = resolve_config(resolve_truncation(pol))
    assert (cfg.weight, cfg.coefficient, cfg.min_terms) == (3, 1e-4, 10)
    cfg = resolve_config(resolve_truncation(pq.TruncationPolicy(weight_cutoff=None, coeff_cutoff=0.0)))
    assert cfg.weight is None and cfg.coefficient is None
    cfg = resolve_config(resolve_truncation([pq.WeightTruncator(2), pq.WeightTruncator(5)]))
    assert cfg.weight == 5  # later entries win (truncators.rs:200-213)
    with pytest.raises(TypeError):
        resolve_truncation(3.0)
    with pytest.raises(ValueError, match="surrogate"):
        pq.PauliPropagator(truncation=pq.FrequencyTruncator(3))
    assert pol.should_truncate(4, 1.0) and pol.should_truncate(1, 1e-5) and not pol.should_truncate(3, 1e-4)


def test_heisenberg_order():
    # extract_layers reverses layers and the gates within each layer.
    n = 3
    a, b, c = (pq.PauliRotation(PauliString(1 << i, 0, n), 0.1 * (i + 1)) for i in range(3))
    gw, ga, off = heisenberg_gates(pq.PauliCircuit([[a, b], [c]]), 1, lambda g: g.key())
    assert list(ga) == [c.angle, b.angle, a.angle]
    assert list(off) == [0, 1, 3]


def test_gate_words_from_cached_key_bytes():
    # the propagators' path (keys kept as bytes on the generators) gives the
    # same words as converting every key, at every width, and again after the
    # generators were used at another width
    from propaq_b200.propagators import _plain_key

    rng = np.random.default_rng(3)
    for n, n_words in [(100, 4), (200, 8), (60, 2), (100, 4)]:
        layers = [[pq.PauliRotation(PauliString(int(rng.integers(0, 1 << 60)) << (n - 60),
                                                int(rng.integers(0, 1 << 60)), n), float(rng.normal()))
                   for _ in range(5)] for _ in range(4)]
        circ = pq.PauliCircuit(layers)
        fast = heisenberg_gates(circ, n_words, _plain_key)
        slow = heisenberg_gates(circ, n_words, lambda g: g.key())
        for f, s in zip(fast, slow):
            assert f.dtype == s.dtype and np.array_equal(f, s)
        wider = heisenberg_gates(circ, 2 * n_words, _plain_key)[0]
        assert np.array_equal(wider[:, :n_words], slow[0]) and not wider[:, n_words:].any()


def _keys_of(p):
    return np.array([p.key()], dtype=np.uint64)


def test_pauli_algebra_matches_oracle(oracle):
    rng = np.random.default_rng(1)
    n = 20
    for _ in range(300):
        a = PauliString(int(rng.integers(0, 1 << n)), int(rng.integers(0, 1 << n)), n)
        b = PauliString(int(rng.integers(0, 1 << n)), int(rng.integers(0, 1 << n)), n)
        phase, prod = a @ b
        out, p = oracle.product(0, _keys_of(a), _keys_of(b))
        assert int(out[0]) == prod.key()
        assert phase == (1, 1j, -1, -1j)[p]
        assert oracle.anticommutes(0, _keys_of(a), _keys_of(b)) == (not a.commutes_with(b))
        assert oracle.weight(0, n, _keys_of(a)) == a.weight
        s = int(rng.integers(0, 1 << n))
        assert oracle.trace(0, n, _keys_of(a), [s]) == a.trace_with_diag_state(s)


def _device_jw_weight(key: int, n_sites: int, n_words: int) -> int:
    """Python transcription of the bit-parallel JW weight in csrc/pq_device.cuh."""
    EVEN = 0x5555555555555555
    M = (1 << 64) - 1
    words = [(key >> (64 * i)) & M for i in range(n_words)]
    total = sum(bin((w ^ (w >> 1)) & EVEN).count("1") for w in words)
    odd = total & 1
    wsum, carry = 0, 0
    for i, k in enumerate(words):
        s = (k ^ (k >> 1)) & EVEN
        occ = (k | (k >> 1)) & EVEN
        p = s
        for sh in (2, 4, 8, 16, 32):
            p = (p ^ (p << sh)) & M
        p ^= carry
        carry = EVEN if (p >> 62) & 1 else 0
        live_sites = n_sites - 32 * i
        live = 0 if live_sites <= 0 else (EVEN if live_sites >= 32 else EVEN & ((1 << (2 * live_sites)) - 1))
        st = ((p ^ EVEN) if odd else p) & live
        wsum += bin((s | (occ ^ st)) & live).count("1")
    return wsum


@pytest.mark.parametrize("n_sites", [5, 32, 40, 64, 100])
def test_majorana_algebra_matches_oracle(oracle, n_sites):
    rng = np.random.default_rng(n_sites)
    n_modes = 2 * n_sites
    W = 1
    while 32 * W < n_sites:
        W *= 2
    for _ in range(200):
        a_int = int(rng.integers(0, 1 << 62)) | (int(rng.integers(0, 1 << 62)) << 62)
        b_int = int(rng.integers(0, 1 << 62)) | (int(rng.integers(0, 1 << 62)) << 62)
        a_int &= (1 << n_modes) - 1
        b_int &= (1 << n_modes) - 1
        if rng.random() < 0.3:  # paired monomials
            a_int = (a_int & int("55" * 32, 16)) * 3 & ((1 << n_modes) - 1)
        a, b = MajoranaMonomial(a_int, n_modes), MajoranaMonomial(b_int, n_modes)
        ka = np.array([(a_int >> (64 * i)) & ((1 << 64) - 1) for i in range(W)], dtype=np.uint64)
        kb = np.array([(b_int >> (64 * i)) & ((1 << 64) - 1) for i in range(W)], dtype=np.uint64)
        w = oracle.weight(1, n_sites, ka)
        assert w == a.weight == jw_weight(a_int, n_sites) == _device_jw_weight(a_int, n_sites, W)
        phase, prod = a @ b
        out, p = oracle.product(1, ka, kb)
        assert sum(int(x) << (64 * i) for i, x in enumerate(out)) == prod.modes
        assert phase == (1, 1j, -1, -1j)[p]
        assert oracle.anticommutes(1, ka, kb) == (not a.commutes_with(b))
        s = int(rng.integers(0, 1 << min(n_sites, 62)))
        assert oracle.trace(1, n_sites, ka, [s, 0]) == a.trace_with_diag_state(s)


def test_term_file_round_trip(tmp_path):
    ts = pq.PauliTermSum()
    ts.add(PauliString(0b101, 0b011, 12), 0.25)
    ts.add(PauliString(0, 0b1, 12), -1.5)
    f = tmp_path / "t.gz"
    ts.save(str(f))
    back = pq.PauliTermSum.from_file(str(f))
    assert dict(back.items()) == dict(ts.items())
    with gzip.open(f, "rb") as fh:
        n, stride, size = struct.unpack("<QQQ", fh.read(24))
    assert (n, stride, size) == (2, 4, 12)  # x then z bytes, ceil(12/8) each
    ms = pq.MajoranaTermSum({MajoranaMonomial(0b1111, 8): 2.0})
    ms.save(str(tmp_path / "m.gz"))
    assert dict(pq.MajoranaTermSum.from_file(str(tmp_path / "m.gz")).items()) == dict(ms.items())


def test_engine_output_file_layout(tmp_path):
    from propaq_b200.term_io import save_terms

    ps = PauliString(0b1010_0011, 0b0110_0001, 70)
    keys = np.array([[ps.key() & ((1 << 64) - 1), ps.key() >> 64]], dtype=np.uint64)
    save_terms(str(tmp_path / "e.gz"), keys, np.array([0.5]), 0, 70)
    back = pq.PauliTermSum.from_file(str(tmp_path / "e.gz"))
    assert dict(back.items()) == {ps: 0.5}


def test_state_words():
    assert list(state_words(0b101, 4)) == [5]
    assert list(state_words(1 << 70, 100)) == [0, 1 << 6]
    with pytest.raises(ValueError):
        state_words(-1, 4)


def test_term_sum_api():
    ts = pq.PauliTermSum()
    a = PauliString(1, 0, 2)
    ts.add(a, 1.0)
    ts.add(a, 2.0)
    assert ts[a] == 3.0 and len(ts) == 1
    ts[a] = 0.5
    ts.scale(2.0)
    assert ts[a] == 1.0 and ts.norm_squared() == 1.0
    ts.apply_damping(pq.UniformNoiseModel(0.5), 0)
    assert ts[a] == math.exp(-0.5)
    ts.add(PauliString(3, 3, 2), 1e-9)
    ts.truncate(pq.TruncationPolicy(coeff_cutoff=1e-6))
    assert len(ts) == 1
