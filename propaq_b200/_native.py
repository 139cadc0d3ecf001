"""ctypes binding of libpropaq_cuda.so (declared in include/propaq_cuda.h).

This is the only module that touches the CUDA engine.  There is no CPU
fallback: if the library is missing or no CUDA device is present, every
propagation call raises.
"""

from __future__ import annotations

import ctypes
import threading
from pathlib import Path

import numpy as np

_LIB_PATH = Path(__file__).resolve().parent / "lib" / "libpropaq_cuda.so"

PQ_OK = 0
PQ_ERR_INVALID = 1
PQ_ERR_CUDA = 2
PQ_ERR_OOM = 3
PQ_ERR_CEILING = 4
PQ_ERR_PLUGIN_LOAD = 5
PQ_ERR_PLUGIN = 6
PQ_ERR_DEVICE_TIMEOUT = 7
PQ_ERR_UNSUPPORTED = 8

PQ_NOISE_NONE = 0
PQ_NOISE_TABLE = 1
PQ_NOISE_LAYERED = 2
PQ_NOISE_PLUGIN = 3


class EngineUnavailable(RuntimeError):
    """The CUDA engine library or a CUDA device is missing."""


class RunConfig(ctypes.Structure):
    _fields_ = [
        ("basis_kind", ctypes.c_uint32),
        ("n_units", ctypes.c_uint32),
        ("max_weight", ctypes.c_int64),
        ("has_min_coeff", ctypes.c_uint32),
        ("min_coeff", ctypes.c_double),
        ("min_terms", ctypes.c_int64),
        ("truncator", ctypes.c_void_p),
        ("noise_kind", ctypes.c_uint32),
        ("noise_tables", ctypes.c_void_p),
        ("noise_table_len", ctypes.c_size_t),
        ("noise_plugin", ctypes.c_void_p),
        ("want_terms", ctypes.c_uint32),
        ("blocks_per_sm", ctypes.c_uint32),
        ("log_gates", ctypes.c_uint32),
        ("fuse_max", ctypes.c_uint32),
        ("tile_items", ctypes.c_uint32),
        ("bucket_slots", ctypes.c_uint32),
    ]


class GateRecord(ctypes.Structure):
    """pq_gate_record: one gate of a logged run (the reference's GateRecord)."""

    _fields_ = [
        ("terms_before", ctypes.c_uint64),
        ("terms_after", ctypes.c_uint64),
        ("terms_gained", ctypes.c_uint64),
        ("declined", ctypes.c_uint64),
        ("emitted", ctypes.c_uint64),
        ("exchange_hits", ctypes.c_uint64),
        ("discarded_coeff_l1", ctypes.c_double),
        ("discarded_coeff_max", ctypes.c_double),
        ("elapsed_ms", ctypes.c_double),
        ("layer_idx", ctypes.c_uint32),
        ("op", ctypes.c_int32),
    ]


class RunResult(ctypes.Structure):
    _fields_ = [
        ("expectation_value", ctypes.c_double),
        ("terms_below_cutoff", ctypes.c_uint64),
        ("sparse_key_bytes", ctypes.c_uint64),
        ("n_final", ctypes.c_uint64),
        ("n_layers_run", ctypes.c_uint64),
        ("n_gates_run", ctypes.c_uint64),
        ("gpu_launches", ctypes.c_uint64),
        ("peak_terms", ctypes.c_uint64),
        ("device_ms", ctypes.c_double),
        ("sweep_ms", ctypes.c_double),
        ("sweep_launches", ctypes.c_uint64),
        ("gate_ms", ctypes.c_double),
        ("noise_ms", ctypes.c_double),
        ("phase_ms", ctypes.c_double),
        ("gate_ops", ctypes.c_uint64),
        ("noise_ops", ctypes.c_uint64),
        ("phase_ops", ctypes.c_uint64),
        ("sum_rows_gate", ctypes.c_uint64),
        ("sum_anti", ctypes.c_uint64),
        ("sum_children", ctypes.c_uint64),
        ("sum_rows_phase", ctypes.c_uint64),
        ("sum_rows_noise", ctypes.c_uint64),
        ("sum_kept", ctypes.c_uint64),
        ("class_ops", ctypes.c_uint64),
    ]


_V = ctypes.c_void_p
_Z = ctypes.c_size_t
_U32 = ctypes.c_uint32

class Instance(ctypes.Structure):
    """pq_instance: one propagation of a pq_run_batch call."""

    _fields_ = [
        ("cfg", RunConfig),
        ("obs_words", _V),
        ("obs_coeffs", _V),
        ("n_obs", _Z),
        ("gate_words", _V),
        ("gate_angles", _V),
        ("n_gates", _Z),
        ("layer_offsets", _V),
        ("n_layers", _Z),
        ("diag_state", _V),
        ("diag_words", _Z),
        ("n_terms_out", _V),
        ("result", ctypes.POINTER(RunResult)),
    ]


class EngineLimits(ctypes.Structure):
    """pq_engine_limits."""

    _fields_ = [("max_rows", ctypes.c_uint64), ("max_device_bytes", ctypes.c_uint64),
                ("barrier_spins", ctypes.c_uint32), ("lookback_spins", ctypes.c_uint32),
                ("hold_block", ctypes.c_uint32), ("hold_us", ctypes.c_uint32)]


class BatchTuning(ctypes.Structure):
    """pq_batch_tuning."""

    _fields_ = [("blocks_per_sm", ctypes.c_uint32), ("split", ctypes.c_uint32), ("rebalance_pct", ctypes.c_uint32),
                ("fuse_max", ctypes.c_uint32), ("tile_items", ctypes.c_uint32), ("bucket_slots", ctypes.c_uint32)]


NOISE_FACTOR_FN = ctypes.CFUNCTYPE(ctypes.c_double, ctypes.c_void_p, ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint64),
                                   ctypes.c_size_t, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                   ctypes.c_uint32)

_SIGNATURES = {
    "pq_words_for_units": (_U32, [_U32]),
    "pq_engine_create": (ctypes.c_int, [ctypes.POINTER(_V), ctypes.c_int]),
    "pq_engine_destroy": (None, [_V]),
    "pq_engine_last_error": (ctypes.c_char_p, [_V]),
    "pq_engine_set_limits": (ctypes.c_int, [_V, ctypes.POINTER(EngineLimits)]),
    "pq_engine_device_bytes": (ctypes.c_uint64, [_V]),
    "pq_run": (ctypes.c_int, [_V, ctypes.POINTER(RunConfig), _V, _V, _Z, _V, _V, _Z, _V, _Z, _V, _Z, _V,
                              ctypes.POINTER(RunResult)]),
    "pq_result_terms": (_Z, [_V, _V, _V, _Z]),
    "pq_result_gates": (_Z, [_V, _V, _Z]),
    "pq_run_batch": (ctypes.c_int, [_V, ctypes.POINTER(Instance), _Z, ctypes.POINTER(BatchTuning)]),
    "pq_result_terms_at": (_Z, [_V, _Z, _V, _V, _Z]),
    "pq_run_adjoint": (ctypes.c_int, [_V, ctypes.POINTER(RunConfig), _V, _V, _Z, _V, _V, _Z, _V, _Z, _V, _Z, _U32,
                                      ctypes.c_uint64, _V, _V, ctypes.POINTER(RunResult)]),
    "pq_plugin_load_noise": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_char_p, ctypes.POINTER(_V),
                                            ctypes.c_char_p, _Z]),
    "pq_plugin_load_truncator": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_char_p, ctypes.POINTER(_V),
                                                ctypes.c_char_p, _Z]),
    "pq_plugin_free": (None, [_V]),
    "pq_plugin_from_callback": (ctypes.c_int, [NOISE_FACTOR_FN, _V, _U32, ctypes.POINTER(_V)]),
    "pq_plugin_depends": (_U32, [_V]),
    "pq_plugin_noise_factor": (ctypes.c_double, [_V, _U32, _V, _Z, _U32, _U32, _U32, _U32]),
    "pq_plugin_truncator_keep": (ctypes.c_int, [_V, _U32, _V, _Z, _U32, _U32, ctypes.c_double, _U32, _U32]),
}

_lib = None
_lib_lock = threading.Lock()


def library_path() -> Path:
    return _LIB_PATH


def lib() -> ctypes.CDLL:
    """Loads libpropaq_cuda.so (built in-tree by propaq_b200.build)."""
    global _lib
    with _lib_lock:
        if _lib is None:
            if not _LIB_PATH.exists():
                raise EngineUnavailable(
                    f"{_LIB_PATH} is missing: build it with `python -m propaq_b200.build` "
                    "(there is no CPU fallback)"
                )
            handle = ctypes.CDLL(str(_LIB_PATH))
            for name, (res, args) in _SIGNATURES.items():
                fn = getattr(handle, name)
                fn.restype = res
                fn.argtypes = args
            _lib = handle
        return _lib


def words_for_units(n_units: int) -> int:
    return int(lib().pq_words_for_units(n_units))


def _ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


class Engine:
    """One CUDA engine (device memory + stream) on one device."""

    def __init__(self, device: int = 0):
        handle = ctypes.c_void_p()
        rc = lib().pq_engine_create(ctypes.byref(handle), device)
        if rc != PQ_OK:
            raise EngineUnavailable(f"no usable CUDA device {device} for the propagation engine (code {rc})")
        self._h = handle
        self.device = device
        self.lock = threading.Lock()

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None:
            _lib.pq_engine_destroy(h)
            self._h = None

    def set_limits(self, max_rows: int = 0, max_device_bytes: int = 0, barrier_spins: int = 0,
                   lookback_spins: int = 0, hold_block: int = 0, hold_us: int = 0):
        """pq_engine_set_limits; no arguments restore every default."""
        lim = EngineLimits(max_rows, max_device_bytes, barrier_spins, lookback_spins, hold_block, hold_us)
        with self.lock:
            rc = lib().pq_engine_set_limits(self._h, ctypes.byref(lim))
        if rc != PQ_OK:
            raise_for(rc, "pq_engine_set_limits failed")

    def device_bytes(self) -> int:
        """Device bytes held in buffers allocated since the limits were last set."""
        with self.lock:
            return int(lib().pq_engine_device_bytes(self._h))

    def run(self, cfg: RunConfig, obs_words, obs_coeffs, gate_words, gate_angles, layer_offsets,
            diag_state=None, want_n_terms=True):
        """Runs pq_run; returns (RunResult, n_terms array or None)."""
        obs_words = np.ascontiguousarray(obs_words, dtype=np.uint64)
        obs_coeffs = np.ascontiguousarray(obs_coeffs, dtype=np.float64)
        gate_words = np.ascontiguousarray(gate_words, dtype=np.uint64)
        gate_angles = np.ascontiguousarray(gate_angles, dtype=np.float64)
        layer_offsets = np.ascontiguousarray(layer_offsets, dtype=np.uint32)
        n_gates = len(gate_angles)
        nt = np.zeros(n_gates, dtype=np.uint64) if want_n_terms else None
        diag = None if diag_state is None else np.ascontiguousarray(diag_state, dtype=np.uint64)
        res = RunResult()
        with self.lock:
            rc = lib().pq_run(self._h, ctypes.byref(cfg), _ptr(obs_words), _ptr(obs_coeffs), len(obs_coeffs),
                              _ptr(gate_words), _ptr(gate_angles), n_gates, _ptr(layer_offsets),
                              len(layer_offsets) - 1, _ptr(diag), 0 if diag is None else len(diag), _ptr(nt),
                              ctypes.byref(res))
            if rc != PQ_OK:
                raise_for(rc, lib().pq_engine_last_error(self._h).decode(errors="replace"))
        return res, nt

    def run_adjoint(self, cfg: RunConfig, obs_words, obs_coeffs, gate_words, gate_angles, layer_offsets,
                    diag_state, checkpoint_layers: int = 0, record_bytes: int = 0):
        """Runs pq_run_adjoint; returns (RunResult, n_terms array, dE/d gate_angles)."""
        obs_words = np.ascontiguousarray(obs_words, dtype=np.uint64)
        obs_coeffs = np.ascontiguousarray(obs_coeffs, dtype=np.float64)
        gate_words = np.ascontiguousarray(gate_words, dtype=np.uint64)
        gate_angles = np.ascontiguousarray(gate_angles, dtype=np.float64)
        layer_offsets = np.ascontiguousarray(layer_offsets, dtype=np.uint32)
        diag = np.ascontiguousarray(diag_state, dtype=np.uint64)
        n_gates = len(gate_angles)
        nt = np.zeros(n_gates, dtype=np.uint64)
        grad = np.zeros(n_gates, dtype=np.float64)
        res = RunResult()
        with self.lock:
            rc = lib().pq_run_adjoint(self._h, ctypes.byref(cfg), _ptr(obs_words), _ptr(obs_coeffs), len(obs_coeffs),
                                      _ptr(gate_words), _ptr(gate_angles), n_gates, _ptr(layer_offsets),
                                      len(layer_offsets) - 1, _ptr(diag), len(diag), checkpoint_layers,
                                      record_bytes, _ptr(grad),
                                      _ptr(nt), ctypes.byref(res))
            if rc != PQ_OK:
                raise_for(rc, lib().pq_engine_last_error(self._h).decode(errors="replace"))
        return res, nt, grad

    def run_batch(self, items, blocks_per_sm: int = 0, split: int = 1, rebalance_pct: int = 25,
                  want_n_terms: bool = True, fuse_max: int = 0, tile_items: int = 0, bucket_slots: int = 0):
        """Runs pq_run_batch on a list of (cfg, obs_words, obs_coeffs, gate_words,
        gate_angles, layer_offsets, diag_state) tuples; returns one
        (RunResult, n_terms array or None) per instance.  fuse_max, tile_items
        and bucket_slots (0 = each instance's own) tune every instance."""
        keep = []
        insts = (Instance * len(items))()
        out = []
        for inst, (cfg, ow, oc, gw, ga, lo, diag) in zip(insts, items):
            ow = np.ascontiguousarray(ow, dtype=np.uint64)
            oc = np.ascontiguousarray(oc, dtype=np.float64)
            gw = np.ascontiguousarray(gw, dtype=np.uint64)
            ga = np.ascontiguousarray(ga, dtype=np.float64)
            lo = np.ascontiguousarray(lo, dtype=np.uint32)
            diag = None if diag is None else np.ascontiguousarray(diag, dtype=np.uint64)
            nt = np.zeros(len(ga), dtype=np.uint64) if want_n_terms else None
            res = RunResult()
            keep += [ow, oc, gw, ga, lo, diag, nt, res]
            inst.cfg = cfg
            inst.obs_words, inst.obs_coeffs, inst.n_obs = _ptr(ow), _ptr(oc), len(oc)
            inst.gate_words, inst.gate_angles, inst.n_gates = _ptr(gw), _ptr(ga), len(ga)
            inst.layer_offsets, inst.n_layers = _ptr(lo), len(lo) - 1
            inst.diag_state, inst.diag_words = _ptr(diag), 0 if diag is None else len(diag)
            inst.n_terms_out = _ptr(nt)
            inst.result = ctypes.pointer(res)
            out.append((res, nt))
        with self.lock:
            tune = BatchTuning(blocks_per_sm, split, rebalance_pct, fuse_max, tile_items, bucket_slots)
            rc = lib().pq_run_batch(self._h, insts, len(items), ctypes.byref(tune))
            if rc != PQ_OK:
                raise_for(rc, lib().pq_engine_last_error(self._h).decode(errors="replace"))
        return out

    def gates(self):
        """Per-gate records (GateRecord array) of the last run made with log_gates."""
        with self.lock:
            n = lib().pq_result_gates(self._h, None, 0)
            out = (GateRecord * n)()
            if n:
                lib().pq_result_gates(self._h, out, n)
        return out

    def terms(self, n_words: int, index: int = 0):
        """Final (keys, coeffs) of the last run made with want_terms (instance
        `index` of the last batch)."""
        with self.lock:
            n = lib().pq_result_terms_at(self._h, index, None, None, 0)
            keys = np.zeros((n, n_words), dtype=np.uint64)
            coeffs = np.zeros(n, dtype=np.float64)
            if n:
                lib().pq_result_terms_at(self._h, index, _ptr(keys), _ptr(coeffs), n)
        return keys, coeffs


def raise_for(code: int, message: str):
    if code in (PQ_ERR_INVALID, PQ_ERR_PLUGIN):
        raise ValueError(message)
    if code == PQ_ERR_PLUGIN_LOAD:
        raise OSError(message)
    if code == PQ_ERR_OOM:
        raise MemoryError(message)
    if code == PQ_ERR_UNSUPPORTED:
        raise NotImplementedError(message)
    raise RuntimeError(message)


_engines: dict[int, Engine] = {}
_engines_lock = threading.Lock()


def engine(device: int = 0) -> Engine:
    """The process-wide engine for a device (created on first use)."""
    with _engines_lock:
        e = _engines.get(device)
        if e is None:
            e = Engine(device)
            _engines[device] = e
        return e


class Plugin:
    """A loaded native noise / truncation plugin (owned; freed on collection)."""

    def __init__(self, path: str, config: str | None, noise: bool):
        handle = ctypes.c_void_p()
        err = ctypes.create_string_buffer(1024)
        fn = lib().pq_plugin_load_noise if noise else lib().pq_plugin_load_truncator
        rc = fn(str(path).encode(), None if config is None else config.encode(), ctypes.byref(handle), err, 1024)
        if rc != PQ_OK:
            raise_for(rc, err.value.decode(errors="replace"))
        self._h = handle
        self.noise = noise

    @property
    def handle(self) -> int:
        return self._h.value

    @property
    def depends(self) -> int:
        return int(lib().pq_plugin_depends(self._h))

    def factor(self, basis_kind, words, n_units, weight, layer_index=0, n_layers=0) -> float:
        w = np.ascontiguousarray(list(words), dtype=np.uint64)
        return float(lib().pq_plugin_noise_factor(self._h, basis_kind, _ptr(w) if len(w) else None, len(w),
                                                  n_units, weight, layer_index, n_layers))

    def keep(self, basis_kind, words, n_units, weight, coeff_magnitude, layer_index=0, n_layers=0) -> bool:
        w = np.ascontiguousarray(list(words), dtype=np.uint64)
        return bool(lib().pq_plugin_truncator_keep(self._h, basis_kind, _ptr(w) if len(w) else None, len(w),
                                                   n_units, weight, coeff_magnitude, layer_index, n_layers))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None:
            _lib.pq_plugin_free(h)
            self._h = None


class CallbackNoise:
    """A Python function of (basis_kind, words, n_units, weight, layer_index,
    n_layers) as a noise plugin handle (pq_plugin_from_callback).  An
    exception inside the function is kept, the factor of that call is NaN, and
    `raise_pending()` re-raises it after the run."""

    def __init__(self, fn, depends: int):
        self._fn = fn
        self.error = None

        def trampoline(ctx, basis_kind, words, n_words, n_units, weight, layer, n_layers):
            if self.error is not None:
                return float("nan")
            try:
                w = [int(words[i]) for i in range(n_words)] if words else []
                return float(fn(basis_kind, w, n_units, weight, layer, n_layers))
            except BaseException as exc:  # noqa: BLE001 -- re-raised by raise_pending
                self.error = exc
                return float("nan")

        self._cb = NOISE_FACTOR_FN(trampoline)
        handle = ctypes.c_void_p()
        rc = lib().pq_plugin_from_callback(self._cb, None, depends, ctypes.byref(handle))
        if rc != PQ_OK:
            raise_for(rc, "could not wrap the noise callback")
        self._h = handle
        self.depends = depends

    @property
    def handle(self) -> int:
        return self._h.value

    def raise_pending(self):
        if self.error is not None:
            err, self.error = self.error, None
            raise err

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and _lib is not None:
            _lib.pq_plugin_free(h)
            self._h = None
