"""ctypes client of the CPU oracle (oracle/pq_oracle.h).  Test infrastructure:
the oracle is the checker, never part of the product path."""

from __future__ import annotations

import ctypes
import subprocess
import threading
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent
ORACLE_DIR = ROOT / "oracle"
ORACLE_LIB = ORACLE_DIR / "_build" / "libpq_oracle.so"
REF_PLUGINS = ORACLE_DIR / "_ref"

_V, _Z = ctypes.c_void_p, ctypes.c_size_t


class Cfg(ctypes.Structure):
    _fields_ = [("basis_kind", ctypes.c_uint32), ("n_units", ctypes.c_uint32), ("n_words", ctypes.c_uint32),
                ("n_partitions", ctypes.c_uint32), ("max_weight", ctypes.c_int64),
                ("has_min_coeff", ctypes.c_uint32), ("min_coeff", ctypes.c_double), ("min_terms", ctypes.c_int64),
                ("truncator", _V), ("noise_kind", ctypes.c_uint32), ("noise_tables", _V),
                ("noise_table_len", _Z), ("noise_plugin", _V)]


class Res(ctypes.Structure):
    _fields_ = [("expectation", ctypes.c_double), ("expectation_accurate", ctypes.c_double),
                ("expectation_abs", ctypes.c_double), ("terms_below_cutoff", ctypes.c_uint64),
                ("n_final", ctypes.c_uint64), ("emitted", ctypes.c_uint64), ("hits", ctypes.c_uint64),
                ("visited", ctypes.c_uint64), ("declined", ctypes.c_uint64), ("discarded_l1", ctypes.c_double)]


_lock = threading.Lock()


def build_oracle() -> Path:
    """Builds the oracle with its Makefile if the library is missing or stale."""
    with _lock:
        src = ORACLE_DIR / "pq_oracle.cpp"
        if not ORACLE_LIB.exists() or ORACLE_LIB.stat().st_mtime < src.stat().st_mtime:
            subprocess.run(["make", "-s", "-C", str(ORACLE_DIR)], check=True)
    return ORACLE_LIB


class OracleResult:
    def __init__(self, res: Res, n_terms, keys, coeffs):
        self.expectation = res.expectation
        self.expectation_accurate = res.expectation_accurate
        self.expectation_abs = res.expectation_abs
        self.terms_below_cutoff = int(res.terms_below_cutoff)
        self.n_final = int(res.n_final)
        self.n_terms = n_terms
        self.keys = keys
        self.coeffs = coeffs
        self.stats = dict(emitted=res.emitted, hits=res.hits, visited=res.visited, declined=res.declined,
                          discarded_l1=res.discarded_l1)


class Oracle:
    _inst = None

    @classmethod
    def load(cls) -> "Oracle":
        if cls._inst is None:
            cls._inst = cls(build_oracle())
        return cls._inst

    def __init__(self, path: Path):
        lib = ctypes.CDLL(str(path))
        lib.pqo_run.restype = _V
        lib.pqo_run.argtypes = [ctypes.POINTER(Cfg), _V, _V, _Z, _V, _V, _Z, _V, _Z, _V, _Z, _V, ctypes.POINTER(Res)]
        lib.pqo_run_free.argtypes = [_V]
        lib.pqo_terms_count.restype = _Z
        lib.pqo_terms_count.argtypes = [_V]
        lib.pqo_terms_copy.argtypes = [_V, _V, _V]
        lib.pqo_last_error.restype = ctypes.c_char_p
        for n in ("pqo_load_noise", "pqo_load_truncator"):
            f = getattr(lib, n)
            f.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.POINTER(_V), ctypes.c_char_p, _Z]
        lib.pqo_plugin_free.argtypes = [_V]
        lib.pqo_plugin_depends.restype = ctypes.c_uint32
        lib.pqo_plugin_depends.argtypes = [_V]
        lib.pqo_weight.restype = ctypes.c_uint32
        lib.pqo_weight.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, _V]
        lib.pqo_anticommutes.argtypes = [ctypes.c_uint32, ctypes.c_uint32, _V, _V]
        lib.pqo_product.argtypes = [ctypes.c_uint32, ctypes.c_uint32, _V, _V, _V]
        lib.pqo_trace.restype = ctypes.c_double
        lib.pqo_trace.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, _V, _V, _Z]
        self.lib = lib

    def load_plugin(self, path, config=None, noise=True):
        h = _V()
        err = ctypes.create_string_buffer(1024)
        fn = self.lib.pqo_load_noise if noise else self.lib.pqo_load_truncator
        rc = fn(str(path).encode(), None if config is None else config.encode(), ctypes.byref(h), err, 1024)
        if rc:
            raise (OSError if rc == 1 else ValueError)(err.value.decode())
        return h

    def run(self, basis, n_units, n_words, obs_keys, obs_coeffs, gate_keys, angles, layer_offsets, *,
            max_weight=None, min_coeff=None, min_terms=None, noise_table=None, noise_tables_layered=None,
            noise_plugin=None, truncator=None, diag_state=None, n_partitions=1, want_terms=True):
        c = Cfg()
        c.basis_kind, c.n_units, c.n_words, c.n_partitions = basis, n_units, n_words, n_partitions
        c.max_weight = -1 if max_weight is None else int(max_weight)
        c.has_min_coeff = 0 if min_coeff is None else 1
        c.min_coeff = 0.0 if min_coeff is None else float(min_coeff)
        c.min_terms = -1 if min_terms is None else int(min_terms)
        c.truncator = truncator
        keep = []
        if noise_table is not None:
            t = np.ascontiguousarray(noise_table, dtype=np.float64)
            keep.append(t)
            c.noise_kind, c.noise_tables, c.noise_table_len = 1, t.ctypes.data, len(t)
        elif noise_tables_layered is not None:
            t = np.ascontiguousarray(noise_tables_layered, dtype=np.float64)
            keep.append(t)
            c.noise_kind, c.noise_tables, c.noise_table_len = 2, t.ctypes.data, t.shape[1]
        elif noise_plugin is not None:
            c.noise_kind, c.noise_plugin = 3, noise_plugin
        ok = np.ascontiguousarray(obs_keys, dtype=np.uint64).reshape(-1, n_words)
        oc = np.ascontiguousarray(obs_coeffs, dtype=np.float64)
        gk = np.ascontiguousarray(gate_keys, dtype=np.uint64).reshape(-1, n_words)
        ga = np.ascontiguousarray(angles, dtype=np.float64)
        lo = np.ascontiguousarray(layer_offsets, dtype=np.uint32)
        ds = None if diag_state is None else np.ascontiguousarray(diag_state, dtype=np.uint64)
        nt = np.zeros(len(ga), dtype=np.uint64)
        r = Res()
        h = self.lib.pqo_run(ctypes.byref(c), ok.ctypes.data, oc.ctypes.data, len(oc), gk.ctypes.data,
                             ga.ctypes.data, len(ga), lo.ctypes.data, len(lo) - 1,
                             None if ds is None else ds.ctypes.data, 0 if ds is None else len(ds),
                             nt.ctypes.data, ctypes.byref(r))
        if not h:
            raise RuntimeError(self.lib.pqo_last_error().decode())
        try:
            keys = coeffs = None
            if want_terms:
                n = self.lib.pqo_terms_count(h)
                keys = np.zeros((n, n_words), dtype=np.uint64)
                coeffs = np.zeros(n, dtype=np.float64)
                if n:
                    self.lib.pqo_terms_copy(h, keys.ctypes.data, coeffs.ctypes.data)
        finally:
            self.lib.pqo_run_free(h)
        return OracleResult(r, nt, keys, coeffs)

    # single-key algebra probes
    def weight(self, basis, n_units, words):
        w = np.ascontiguousarray(words, dtype=np.uint64)
        return int(self.lib.pqo_weight(basis, n_units, len(w), w.ctypes.data))

    def product(self, basis, gen, key):
        g = np.ascontiguousarray(gen, dtype=np.uint64)
        k = np.ascontiguousarray(key, dtype=np.uint64)
        out = np.zeros_like(k)
        p = self.lib.pqo_product(basis, len(k), g.ctypes.data, k.ctypes.data, out.ctypes.data)
        return out, p

    def anticommutes(self, basis, gen, key):
        g = np.ascontiguousarray(gen, dtype=np.uint64)
        k = np.ascontiguousarray(key, dtype=np.uint64)
        return bool(self.lib.pqo_anticommutes(basis, len(k), g.ctypes.data, k.ctypes.data))

    def trace(self, basis, n_units, key, state):
        k = np.ascontiguousarray(key, dtype=np.uint64)
        s = np.ascontiguousarray(state, dtype=np.uint64)
        return float(self.lib.pqo_trace(basis, n_units, len(k), k.ctypes.data, s.ctypes.data, len(s)))
