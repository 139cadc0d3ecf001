"""The batch autotuner's choice and memory (propaq_b200.tuning), with a fake
run in place of the GPU."""

from types import SimpleNamespace

import numpy as np

from propaq_b200.tuning import CANDIDATES, KERNEL_DEFAULTS, KERNEL_DIMENSIONS, BatchTuner, Tuning, batch_signature

# kernel settings tried after the launch candidates: every value but the default
N_KERNEL = sum(len([v for v in vals if v != KERNEL_DEFAULTS[d]]) for d, vals in KERNEL_DIMENSIONS.items())


def item(n_units, n_gates, max_weight=10, angle=0.3):
    cfg = SimpleNamespace(basis_kind=0, n_units=n_units, max_weight=max_weight, has_min_coeff=1, min_coeff=1e-5,
                          min_terms=-1, noise_kind=1)
    return (cfg, np.zeros((1, 1), np.uint64), np.ones(1), np.zeros((n_gates, 1), np.uint64),
            np.full(n_gates, angle), np.array([0, n_gates], np.uint32), None)


def test_picks_the_fastest_candidate_and_remembers_it_per_shape():
    times = {c: 10.0 + i for i, c in enumerate(CANDIDATES)}
    times[(0, 1, 50)] = 3.0
    calls = []

    def run(items, t):
        calls.append(t)
        return times[(t.blocks_per_sm, t.split, t.rebalance_pct)]

    tuner = BatchTuner()
    batch = [item(40, 100), item(90, 300)]
    assert tuner.tune(batch, run=run) == Tuning(0, 1, 50)
    assert len(calls) == len(CANDIDATES) + N_KERNEL
    # the same shape with other angles: remembered, no new runs
    again = [item(40, 100, angle=0.9), item(90, 300, angle=0.1)]
    assert tuner.tune(again, run=run) == Tuning(0, 1, 50)
    assert len(calls) == len(CANDIDATES) + N_KERNEL
    assert tuner.choice(again) == Tuning(0, 1, 50)
    # another shape is tuned on its own
    other = [item(40, 100, max_weight=8)]
    assert batch_signature(other) != batch_signature(batch)
    tuner.tune(other, run=run)
    assert len(calls) == 2 * (len(CANDIDATES) + N_KERNEL)


def test_kernel_knobs_one_at_a_time_from_the_best_launch_setting():
    # fuse_max 1 and bucket_slots 8 each help on their own; tile_items never
    # does: the tuner keeps the first two, each found from the best so far
    def run(items, t):
        ms = 20.0 if (t.blocks_per_sm, t.split, t.rebalance_pct) == (2, 1, 25) else 30.0
        if t.fuse_max == 1:
            ms -= 4.0
        if t.bucket_slots == 8:
            ms -= 1.0
        if t.tile_items in (1, 2):
            ms += 2.0
        return ms

    tuner = BatchTuner()
    batch = [item(60, 200)]
    best = tuner.tune(batch, run=run)
    assert best == Tuning(2, 1, 25, fuse_max=1, tile_items=0, bucket_slots=8)
    trials = tuner.trials[batch_signature(batch)]
    assert len(trials) == len(CANDIDATES) + N_KERNEL
    assert min(ms for _, ms in trials) == 15.0
    # a default value spelled out is the same setting, not measured again
    assert len({t.resolved() for t, _ in trials}) == len(trials)


def test_kernel_defaults_match_the_engine():
    # The tuner treats a knob at KERNEL_DEFAULTS as the engine's own default
    # (0) and does not measure it twice, so the two must agree: the host's
    # FUSE_DEFAULT and BUCKET_DEFAULT, and the kernel's MAX_ITEMS (what a
    # tile_items of 0 runs).
    import re
    from pathlib import Path

    csrc = Path(__file__).resolve().parent.parent / "propaq_b200" / "csrc"
    host = (csrc / "pq_host.cu").read_text()
    kern = (csrc / "pq_kernels.cu").read_text()

    def const(text, name):
        m = re.search(rf"constexpr\s+\w+\s+{name}\s*=\s*(\d+)\s*;", text)
        assert m, name
        return int(m.group(1))

    assert KERNEL_DEFAULTS["fuse_max"] == const(host, "FUSE_DEFAULT")
    assert KERNEL_DEFAULTS["bucket_slots"] == const(host, "BUCKET_DEFAULT")
    assert KERNEL_DEFAULTS["tile_items"] == const(kern, "MAX_ITEMS")
    for d, vals in KERNEL_DIMENSIONS.items():
        assert KERNEL_DEFAULTS[d] in vals, d
