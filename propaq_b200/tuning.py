"""Autotuning of the batched path's launch parameters.

`pq_run_batch` takes three knobs (`blocks_per_sm`, `split`, `rebalance_pct`)
whose best values depend on the batch: how uneven the instances are, how
large they grow and how many there are.  `BatchTuner.tune` runs the batch
once per candidate setting on the GPU, keeps the one with the least device
time, and remembers it per batch shape (basis, and per instance: units, gates,
layers and truncation settings), so a sweep that is run again -- an
extrapolation inside an optimisation loop, say -- pays for the tuning once.
Results do not depend on the setting (every instance is bit-identical to its
own `pq_run`), only the time does.
"""

from __future__ import annotations

from dataclasses import dataclass

from . import _native

# (blocks_per_sm, split, rebalance_pct): the default first, then the grid
# sizes, splits and rebalancing thresholds that moved the time of the
# 64-instance extrapolation sweep in measurement (993-1250 ms per batch).
# Never rebalancing is left out: it took that sweep 7.3 s, the largest
# instances running on their first small share of the grid.
CANDIDATES = [
    (0, 1, 25),
    (0, 1, 10),
    (0, 1, 50),
    (0, 0, 25),
    (0, 0, 10),
    (2, 1, 25),
]


@dataclass
class Tuning:
    blocks_per_sm: int
    split: int
    rebalance_pct: int

    def as_dict(self) -> dict:
        return {"blocks_per_sm": self.blocks_per_sm, "split": self.split, "rebalance_pct": self.rebalance_pct}


def batch_signature(items) -> tuple:
    """The shape of a batch: what the tuning depends on (not the angles,
    coefficients or states)."""
    sig = []
    for cfg, obs_keys, obs_coeffs, gate_keys, angles, offsets, diag in items:
        sig.append((cfg.basis_kind, cfg.n_units, len(angles), len(offsets), len(obs_coeffs), cfg.max_weight,
                    cfg.has_min_coeff, cfg.min_coeff, cfg.min_terms, cfg.noise_kind))
    return tuple(sig)


class BatchTuner:
    """Chooses pq_run_batch's launch parameters by measurement, per batch shape."""

    def __init__(self, candidates=None):
        self.candidates = list(candidates or CANDIDATES)
        self._best: dict[tuple, Tuning] = {}
        self.trials: dict[tuple, list] = {}  # shape -> [(Tuning, device ms)] of its tuning run

    def choice(self, items) -> Tuning | None:
        return self._best.get(batch_signature(items))

    def tune(self, items, device: int = 0, run=None) -> Tuning:
        """The fastest candidate for this batch (measured now, or remembered).
        `run(items, tuning) -> device ms` replaces the GPU run (tests)."""
        sig = batch_signature(items)
        if sig in self._best:
            return self._best[sig]
        if run is None:
            eng = _native.engine(device)

            def run(its, t):
                out = eng.run_batch(its, want_n_terms=False, **t.as_dict())
                return out[0][0].device_ms

        trials = []
        for c in self.candidates:
            t = Tuning(*c)
            trials.append((t, float(run(items, t))))
        best = min(trials, key=lambda x: x[1])[0]
        self._best[sig] = best
        self.trials[sig] = trials
        return best


_TUNER = BatchTuner()


def default_tuner() -> BatchTuner:
    """The process-wide tuner that `expectation_values(..., autotune=True)` uses."""
    return _TUNER


__all__ = ["BatchTuner", "Tuning", "CANDIDATES", "batch_signature", "default_tuner"]
