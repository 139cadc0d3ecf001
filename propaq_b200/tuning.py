"""Autotuning of the batched path's launch and kernel parameters.

`pq_run_batch` takes three launch knobs (`blocks_per_sm`, `split`,
`rebalance_pct`) and three kernel knobs (`fuse_max`: commuting rotations run
in one pass over the rows; `tile_items`: rows per thread of a many-row gate
tile; `bucket_slots`: the hash table's bucket width) whose best values depend
on the batch: how uneven the instances are, how large they grow and how many
there are.  `BatchTuner.tune` measures the batch on the GPU: first each launch
candidate with the kernel defaults, then, from the fastest, one kernel knob at
a time over its values (keeping a value only when it is faster), and it
remembers the winner per batch shape (basis, and per instance: units, gates,
layers and truncation settings), so a sweep that is run again -- an
extrapolation inside an optimisation loop, say -- pays for the tuning once.
Results do not depend on the setting (every instance is bit-identical to its
own `pq_run`), only the time does.
"""

from __future__ import annotations

from dataclasses import dataclass, replace

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

# Kernel knobs tried one at a time after the launch knobs, and the engine's
# default of each (0 in the tuning means that default).
KERNEL_DIMENSIONS = {
    "fuse_max": (1, 2),
    "tile_items": (1, 2, 4),
    "bucket_slots": (2, 4, 8),
}
KERNEL_DEFAULTS = {"fuse_max": 2, "tile_items": 4, "bucket_slots": 2}


@dataclass(frozen=True)
class Tuning:
    blocks_per_sm: int
    split: int
    rebalance_pct: int
    fuse_max: int = 0
    tile_items: int = 0
    bucket_slots: int = 0

    def as_dict(self) -> dict:
        return {"blocks_per_sm": self.blocks_per_sm, "split": self.split, "rebalance_pct": self.rebalance_pct,
                "fuse_max": self.fuse_max, "tile_items": self.tile_items, "bucket_slots": self.bucket_slots}

    def resolved(self) -> tuple:
        """The setting with kernel defaults spelled out (0 and the default run alike)."""
        k = {d: getattr(self, d) or KERNEL_DEFAULTS[d] for d in KERNEL_DIMENSIONS}
        return (self.blocks_per_sm, self.split, self.rebalance_pct, k["fuse_max"], k["tile_items"],
                k["bucket_slots"])


def batch_signature(items) -> tuple:
    """The shape of a batch: what the tuning depends on (not the angles,
    coefficients or states)."""
    sig = []
    for cfg, obs_keys, obs_coeffs, gate_keys, angles, offsets, diag in items:
        sig.append((cfg.basis_kind, cfg.n_units, len(angles), len(offsets), len(obs_coeffs), cfg.max_weight,
                    cfg.has_min_coeff, cfg.min_coeff, cfg.min_terms, cfg.noise_kind))
    return tuple(sig)


class BatchTuner:
    """Chooses pq_run_batch's launch and kernel parameters by measurement, per
    batch shape."""

    def __init__(self, candidates=None, dimensions=None):
        self.candidates = list(candidates or CANDIDATES)
        self.dimensions = dict(KERNEL_DIMENSIONS if dimensions is None else dimensions)
        self._best: dict[tuple, Tuning] = {}
        self.trials: dict[tuple, list] = {}  # shape -> [(Tuning, device ms)] of its tuning run

    def choice(self, items) -> Tuning | None:
        return self._best.get(batch_signature(items))

    def tune(self, items, device: int = 0, run=None) -> Tuning:
        """The fastest setting for this batch (measured now, or remembered).
        `run(items, tuning) -> device ms` replaces the GPU run (tests)."""
        sig = batch_signature(items)
        if sig in self._best:
            return self._best[sig]
        if run is None:
            eng = _native.engine(device)

            def run(its, t):
                out = eng.run_batch(its, want_n_terms=False, **t.as_dict())
                return out[0][0].device_ms

        trials, seen = [], {}

        def measure(t: Tuning) -> float:
            key = t.resolved()
            if key not in seen:
                seen[key] = float(run(items, t))
                trials.append((t, seen[key]))
            return seen[key]

        best = min((Tuning(*c) for c in self.candidates), key=measure)
        best_ms = measure(best)
        for dim, values in self.dimensions.items():
            for v in values:
                t = replace(best, **{dim: v})
                ms = measure(t)
                if ms < best_ms:
                    best, best_ms = t, ms
        self._best[sig] = best
        self.trials[sig] = trials
        return best


_TUNER = BatchTuner()


def default_tuner() -> BatchTuner:
    """The process-wide tuner that `expectation_values(..., autotune=True)` uses."""
    return _TUNER


__all__ = ["BatchTuner", "Tuning", "CANDIDATES", "KERNEL_DIMENSIONS", "KERNEL_DEFAULTS", "batch_signature",
           "default_tuner"]
