"""Noise models (crates/core/src/policy/noise.rs, native_noise.rs) and their
resolution into what the engine applies (crates/core/src/engine/noise_resolver.rs).
"""

from __future__ import annotations

import math

import numpy as np

from . import _native


class UniformNoiseModel:
    """Each term of weight w is scaled by exp(-damping * w) at every layer."""

    def __init__(self, damping: float):
        self.damping = float(damping)

    def damping_factor(self, term_weight: int, active_modes: int = 0) -> float:
        return math.exp(-self.damping * float(term_weight))

    def apply_noise(self, term_sum) -> None:
        term_sum.apply_damping(self, 0)

    def __repr__(self):
        return f"UniformNoiseModel(damping={self.damping})"


class GateNoiseModel:
    """Base class of a custom Python noise model; subclasses define
    `damping_factor(weight, active_modes)` or the key-aware
    `damping_factor_term(basis_kind, words, n_units, weight)`."""

    def __init__(self, *args, **kwargs):
        pass

    def damping_factor(self, term_weight: int, active_modes: int) -> float:
        raise NotImplementedError("GateNoiseModel.damping_factor must be overridden by a subclass")


class NativeNoiseModel:
    """Noise model from a native plugin (propaq_noise_* C ABI, native_noise.rs:12-28)."""

    def __init__(self, path: str, config: str | None = None):
        self._plugin = _native.Plugin(path, config, noise=True)

    @property
    def abi_version(self) -> int:
        return 1

    @property
    def depends(self) -> int:
        return self._plugin.depends

    @property
    def handle(self) -> int:
        return self._plugin.handle

    def factor_term(self, basis_kind, words, n_units, weight, layer_index=0, n_layers=0) -> float:
        if basis_kind not in (0, 1):
            raise ValueError(f"basis_kind must be 0 (Pauli) or 1 (Majorana), got {basis_kind}")
        return self._plugin.factor(basis_kind, words, n_units, weight, layer_index, n_layers)

    def __repr__(self):
        return f"NativeNoiseModel(<native plugin, depends={self.depends}>)"


PYTHON_TERM_HOOK = "damping_factor_term"


def resolve_noise(model, n_units: int):
    """(kind, tables, plugin) for the engine, by what the model depends on
    (noise_resolver.rs:78-131)."""
    if model is None:
        return _native.PQ_NOISE_NONE, None, None
    if isinstance(model, UniformNoiseModel):
        d = model.damping
        table = np.array([math.exp(-d * float(w)) for w in range(n_units + 1)], dtype=np.float64)
        return _native.PQ_NOISE_TABLE, table, None
    if isinstance(model, NativeNoiseModel):
        return _native.PQ_NOISE_PLUGIN, None, model
    if hasattr(model, PYTHON_TERM_HOOK):
        # ResolvedNoise::PythonTerm: called per live term at every noise op, with
        # the reference's arguments (basis_kind, words, n_units, weight).
        hook = getattr(model, PYTHON_TERM_HOOK)
        return _native.PQ_NOISE_PLUGIN, None, _native.CallbackNoise(
            lambda kind, words, n_units, weight, layer, n_layers: hook(kind, words, n_units, weight), 1)
    table = np.array([float(model.damping_factor(w, 0)) for w in range(n_units + 1)], dtype=np.float64)
    return _native.PQ_NOISE_TABLE, table, None
