"""PauliPropagator / MajoranaPropagator: the reference's propagator surface
(crates/pauli/src/propagator.rs:117-426, crates/majorana/src/propagator.rs,
propaq/_rust_core/__init__.pyi:225-277, :502-560) over the CUDA engine.

`n_threads` and `pin_threads` are accepted for API compatibility; the engine
runs on one GPU and has no host worker pool.
"""

from __future__ import annotations

import json

import numpy as np

from . import _native
from .datatypes import MajoranaMonomial, MajoranaTermSum, PauliString, PauliTermSum, words_to_int
from .noise import NativeNoiseModel, resolve_noise
from .truncation import reject_surrogate_only, resolve_config, resolve_truncation

MAX_UNITS = 2048


class PropagationResult:
    """crates/core/src/interface/results.rs:8-51."""

    def __init__(self, expectation_value: float, n_terms, sparse_key_bytes: int = 0, terms_below_cutoff: int = 0):
        self.expectation_value = float(expectation_value)
        self.n_terms = list(n_terms)
        self.sparse_key_bytes = int(sparse_key_bytes)
        self.terms_below_cutoff = int(terms_below_cutoff)

    def __repr__(self):
        return (f"PropagationResult(expectation_value={self.expectation_value}, n_terms=[{len(self.n_terms)} gates], "
                f"sparse_key_bytes={self.sparse_key_bytes}, terms_below_cutoff={self.terms_below_cutoff})")


class Logger:
    """JSON-lines verbose run log (crates/core/src/interface/logger.rs:13-57).

    A propagator given a Logger rewrites `filename` after each run with the
    reference's events (crates/pauli/src/propagator.rs:23-101): per gate (every
    `log_every`-th, Heisenberg order) a `gate` and a `truncation` record, then
    one `engine_phases` record; propaq's LogParser reads it.  The engine runs
    such a run with every rotation as an op of its own, so ms_per_gate is that
    op's device time.  The engine has no scan / absorb / claims phases: its
    gate ops do all three, and their device time is reported as scan_s.
    """

    def __init__(self, filename: str, log_every: int = 1):
        self.filename = filename
        self.log_every = max(1, int(log_every))


def _rust_exp(x: float, digits: int) -> str:
    """Rust's `{:.Ne}` formatting of a float (e.g. 1.234e-2, 0.000e0)."""
    m, e = f"{x:.{digits}e}".split("e")
    return f"{m}e{int(e)}"


def write_gate_log(logger: Logger, records, qiskit_idx, cfg, res) -> None:
    """The reference's write_gate_log (crates/pauli/src/propagator.rs:23-101)
    from the engine's per-gate records."""
    every = logger.log_every
    wc = "null" if cfg.weight is None else str(int(cfg.weight))
    cc = _rust_exp(0.0 if cfg.coefficient is None else float(cfg.coefficient), 6)
    lines = []
    tot_decl = tot_emit = tot_hits = 0
    for g, r in enumerate(records):
        tot_decl += r.declined
        tot_emit += r.emitted
        tot_hits += r.exchange_hits
        if g % every:
            continue
        q = qiskit_idx[g]
        qk = "null" if q is None else str(int(q))
        lines.append(f'{{"event":"gate","gate_idx":{g},"layer_idx":{r.layer_idx},"qiskit_gate_idx":{qk},'
                     f'"terms":{r.terms_after},"ms_per_gate":{_rust_exp(r.elapsed_ms, 3)}}}')
        lines.append(f'{{"event":"truncation","gate_idx":{g},"layer_idx":{r.layer_idx},"qiskit_gate_idx":{qk},'
                     f'"trigger":"emit","truncation_model":"emit_gate","terms_before":{r.terms_before},'
                     f'"terms_after":{r.terms_after},"terms_gained":{r.terms_gained},"terms_discarded":{r.declined},'
                     f'"discarded_coeff_l1":{_rust_exp(r.discarded_coeff_l1, 6)},'
                     f'"discarded_coeff_max":{_rust_exp(r.discarded_coeff_max, 6)},"weight_cutoff":{wc},'
                     f'"coeff_cutoff":{cc},"elapsed_ms":{_rust_exp(r.elapsed_ms, 3)}}}')
    visited = int(res.sum_anti)
    share = lambda part, whole: part / max(whole, 1)  # noqa: E731
    lines.append(json.dumps({
        "event": "engine_phases", "partitions": 1, "scan_s": res.gate_ms * 1e-3, "absorb_s": 0.0, "claims_s": 0.0,
        "scan_occupancy": 1.0, "absorb_occupancy": 0.0, "claims_occupancy": 0.0, "terms": int(res.n_final),
        "inline_positions": 0, "overflow_rows": 0, "overflow_share": 0.0, "visited": visited,
        "emitted": int(tot_emit), "declined": int(tot_decl), "emitted_share": share(tot_emit, visited),
        "declined_share": share(tot_decl, visited), "exchange_hits": int(tot_hits),
        "exchange_hit_share": share(tot_hits, tot_emit)}, separators=(",", ":")))
    with open(logger.filename, "w") as f:
        f.write("\n".join(lines) + "\n")


def heisenberg_gates(circuit, n_words: int, key_of):
    """Flattens circuit.layers into arrays in Heisenberg order: layers reversed and
    the gates within each layer reversed (crates/pauli/src/engine.rs:44-70).
    Returns (gate_words [G, n_words], angles [G], layer_offsets [L+1])."""
    rots, offsets = [], [0]
    for layer in reversed(list(circuit.layers)):
        rots.extend(layer[::-1] if isinstance(layer, (list, tuple)) else list(layer)[::-1])
        offsets.append(len(rots))
    angles = np.fromiter((r.angle for r in rots), dtype=np.float64, count=len(rots))
    gens = [r.generator for r in rots]
    if key_of is _plain_key and n_words > 1 and all(type(g) is PauliString for g in gens):
        # keys the generators keep as bytes: one join instead of a conversion per gate
        buf = b"".join([g.key_bytes(n_words) for g in gens])
        words = np.frombuffer(buf, dtype="<u8").reshape(len(gens), n_words).astype(np.uint64)
    else:
        words = keys_to_words([key_of(g) for g in gens], n_words)
    return words, angles, np.array(offsets, dtype=np.uint32)


def _plain_key(term) -> int:
    return term.key()


def keys_to_words(keys, n_words: int) -> np.ndarray:
    """Python-int keys -> [len, n_words] little-endian u64 words."""
    if n_words == 1:
        return np.fromiter(keys, dtype=np.uint64, count=len(keys)).reshape(len(keys), 1)
    nb = 8 * n_words
    buf = b"".join(k.to_bytes(nb, "little") for k in keys)
    return np.frombuffer(buf, dtype="<u8").reshape(len(keys), n_words).astype(np.uint64)


def state_words(initial_state, n_units: int) -> np.ndarray:
    """A computational-basis state (Python int, bit u = unit u) as u64 words."""
    s = int(initial_state or 0)
    if s < 0:
        raise ValueError("initial_state must be a non-negative integer bitstring")
    n_words = max(1, (n_units + 63) // 64)
    mask = (1 << 64) - 1
    return np.array([(s >> (64 * i)) & mask for i in range(n_words)], dtype=np.uint64)


class _Propagator:
    _basis = 0

    def __init__(self, noise=None, truncation=None, n_threads=None, logger=None, pin_threads=True,
                 progress_bar=False, progress_every=1, device: int = 0):
        self._truncators = resolve_truncation(truncation)
        reject_surrogate_only(self._truncators)
        self._noise = noise
        self.n_threads = n_threads
        self.logger = logger
        self.pin_threads = pin_threads
        self.progress_bar = progress_bar
        self.progress_every = progress_every
        self.device = device
        self.last_run = None  # the engine's RunResult of the latest call

    @property
    def noise(self):
        return self._noise

    def set_noise(self, noise=None):
        self._noise = noise

    @property
    def truncators(self):
        return list(self._truncators)

    def set_truncation(self, truncation=None):
        t = resolve_truncation(truncation)
        reject_surrogate_only(t)
        self._truncators = t

    # --- basis hooks
    def _n_units(self, observable) -> int:
        raise NotImplementedError

    def _width_error(self, observable):
        raise NotImplementedError

    def _key(self, term) -> int:
        return term.key()

    def _make_sum(self, keys, coeffs, observable):
        raise NotImplementedError

    def _inputs(self, observable, circuit, initial_state, want_terms):
        """The engine arguments of one propagation: (RunConfig, obs_words,
        obs_coeffs, gate_words, angles, layer_offsets, diag_state), the key
        width and unit count, and the objects the RunConfig points into (they
        must stay alive until the run returns)."""
        n_units = self._n_units(observable)
        if n_units > MAX_UNITS:
            self._width_error(observable)
        n_words = _native.words_for_units(n_units)
        if n_words == 0:
            self._width_error(observable)
        cfg = resolve_config(self._truncators)
        kind, tables, plugin = resolve_noise(self._noise, n_units)
        rc = _native.RunConfig()
        rc.basis_kind = self._basis
        rc.n_units = n_units
        rc.max_weight = -1 if cfg.weight is None else int(cfg.weight)
        rc.has_min_coeff = 0 if cfg.coefficient is None else 1
        rc.min_coeff = 0.0 if cfg.coefficient is None else float(cfg.coefficient)
        rc.min_terms = -1 if cfg.min_terms is None else int(cfg.min_terms)
        rc.truncator = None if cfg.native is None else cfg.native.handle
        rc.noise_kind = kind
        if tables is not None:
            rc.noise_tables = tables.ctypes.data
            rc.noise_table_len = len(tables)
        if plugin is not None:
            rc.noise_plugin = plugin.handle
        rc.want_terms = 1 if want_terms else 0
        rc.log_gates = 1 if self.logger is not None else 0
        obs_keys, obs_coeffs = observable.to_arrays(n_words)
        gw, ga, off = heisenberg_gates(circuit, n_words,
                                       _plain_key if type(self)._key is _Propagator._key else self._key)
        diag = None if initial_state is None else state_words(initial_state, n_units)
        args = (rc, obs_keys, obs_coeffs, gw, ga, off, diag)
        return args, n_words, n_units, (tables, plugin, cfg)

    def _run(self, observable, circuit, initial_state, want_terms):
        args, n_words, n_units, keep = self._inputs(observable, circuit, initial_state, want_terms)
        eng = _native.engine(self.device)
        plugin = keep[1]
        try:
            res, nt = eng.run(*args)
        except Exception:
            if isinstance(plugin, _native.CallbackNoise):
                plugin.raise_pending()
            raise
        if isinstance(plugin, _native.CallbackNoise):
            plugin.raise_pending()
        self.last_run = res
        terms = eng.terms(n_words) if want_terms else None
        if self.logger is not None:
            rots = [r for layer in reversed(list(circuit.layers)) for r in list(layer)[::-1]]
            write_gate_log(self.logger, eng.gates(), [getattr(r, "qiskit_gate_idx", None) for r in rots],
                           keep[2], res)
        return res, nt, terms, n_words

    def propagate(self, observable, circuit, filename=None):
        """Back-propagates `observable` through `circuit`; returns the evolved term sum."""
        res, nt, terms, n_words = self._run(observable, circuit, None, True)
        keys, coeffs = terms
        out = self._make_sum(keys, coeffs, observable)
        if filename is not None:
            from .term_io import save_terms

            save_terms(filename, keys, coeffs, self._basis, self._n_units_io(observable))
        return out

    def expectation_value(self, observable, circuit, initial_state=None, filename=None) -> PropagationResult:
        """<initial_state| U^dag O U |initial_state> via Heisenberg propagation."""
        res, nt, terms, n_words = self._run(observable, circuit, 0 if initial_state is None else initial_state,
                                            filename is not None)
        if filename is not None:
            from .term_io import save_terms

            save_terms(filename, terms[0], terms[1], self._basis, self._n_units_io(observable))
        return PropagationResult(res.expectation_value, nt.tolist(), res.sparse_key_bytes,
                                 res.terms_below_cutoff)

    def _n_units_io(self, observable) -> int:
        return observable.n_units()


def expectation_values(jobs, blocks_per_sm: int = 0, split: int = 1, rebalance_pct: int = 25, device: int = 0,
                       autotune: bool = False, fuse_max: int = 0, tile_items: int = 0, bucket_slots: int = 0):
    """Expectation values of many independent propagations in shared
    persistent launches on one GPU (pq_run_batch).

    `jobs` is a list of (propagator, observable, circuit, initial_state); all
    propagators are Pauli or all Majorana, each with its own noise and
    truncation.  Returns one PropagationResult per job, identical to
    `propagator.expectation_value(observable, circuit, initial_state)`.  The
    reference runs such sweeps as one call after another
    (propaq/extrapolators/zne.py:63-108, zce.py:88-137).

    blocks_per_sm: grid size per SM (0 = as many as fit); split: 0 shares the
    grid equally among the jobs, 1 in proportion to their remaining work;
    rebalance_pct: re-split the grid among the running jobs once this share of
    it is idle (0 = never).  fuse_max, tile_items, bucket_slots: the kernel
    knobs of pq_batch_tuning (0 = the engine's defaults).  autotune: choose all
    six by measurement instead (propaq_b200.tuning; the first batch of a shape
    runs once per setting tried, later ones reuse the choice).
    """
    jobs = list(jobs)
    if not jobs:
        return []
    items, keep = [], []
    for prop, observable, circuit, initial_state in jobs:
        args, _, _, k = prop._inputs(observable, circuit, 0 if initial_state is None else initial_state, False)
        items.append(args)
        keep.append(k)
    eng = _native.engine(device)
    if autotune:
        from .tuning import default_tuner

        t = default_tuner().tune(items, device)
        blocks_per_sm, split, rebalance_pct = t.blocks_per_sm, t.split, t.rebalance_pct
        fuse_max, tile_items, bucket_slots = t.fuse_max, t.tile_items, t.bucket_slots
    out = eng.run_batch(items, blocks_per_sm=blocks_per_sm, split=split, rebalance_pct=rebalance_pct,
                        fuse_max=fuse_max, tile_items=tile_items, bucket_slots=bucket_slots)
    results = []
    for (prop, *_), (res, nt) in zip(jobs, out):
        prop.last_run = res
        results.append(PropagationResult(res.expectation_value, nt.tolist(), res.sparse_key_bytes,
                                         res.terms_below_cutoff))
    return results


class PauliPropagator(_Propagator):
    """Back-propagates Pauli observables through circuits of Pauli rotations on the GPU."""

    _basis = 0

    def _n_units(self, observable) -> int:
        if not isinstance(observable, PauliTermSum):
            raise TypeError("observable must be a PauliTermSum")
        return observable.n_units()

    def _width_error(self, observable):
        raise ValueError(f"propaq: {observable.n_units()} qubits exceeds the engine's maximum of {MAX_UNITS}")

    def _make_sum(self, keys, coeffs, observable):
        return PauliTermSum.from_arrays(keys, coeffs, observable.n_units())


class MajoranaPropagator(_Propagator):
    """Back-propagates Majorana observables through circuits of Majorana rotations on the GPU."""

    _basis = 1

    def _n_units(self, observable) -> int:
        if not isinstance(observable, MajoranaTermSum):
            raise TypeError("observable must be a MajoranaTermSum")
        n_modes = observable.n_units()
        if n_modes % 2:
            self._width_error(observable)
        return n_modes // 2

    def _width_error(self, observable):
        raise ValueError(f"propaq: {observable.n_units()} qubits exceeds the engine's maximum of {MAX_UNITS}")

    def _make_sum(self, keys, coeffs, observable):
        return MajoranaTermSum.from_arrays(keys, coeffs, observable.n_units())


__all__ = ["PauliPropagator", "MajoranaPropagator", "PropagationResult", "Logger", "heisenberg_gates", "expectation_values",
           "state_words", "PauliString", "MajoranaMonomial", "words_to_int", "NativeNoiseModel"]
