"""Benchmark of the propagation hot path (one JSON line on rank 0).

A step is one full Heisenberg propagation of the workload plus its expectation
value.  The default workload is the large noisy Pauli configuration: a 10x10
open-lattice kicked Ising circuit (20 steps of RZZ(-pi/2) on the 4 edge colour
classes + RX(0.6) on all qubits), observable Z at the centre, depolarising
p = 1e-3 per qubit per layer as (1-p)^weight damping, weight cutoff 10,
coefficient cutoff 1e-5, FP64 coefficients.

    value  = sum over gates of the live terms after the gate, per second of
             device time (CUDA events on the engine's stream, inputs resident)
    e2e    = the same metric through PauliPropagator.expectation_value with
             host inputs, host<->device copies inside the timed region
    roofline: the sweep kernel's algorithmic bytes over its event-timed
             duration, against the measured HBM copy bandwidth.  Per gate:
             8W N + 16 A + (8+8W) A + (8W+16) E (N live rows, A anticommuting
             rows, E children); per noisy layer (8W+16)(N + kept); per
             phase-only gate 8W N.

`--workload batch` runs the extrapolation-sweep batch instead: 64 independent
kicked-Ising instances of 40..100 qubits (4 noise scales x 4 coefficient
cutoffs x 4 observable sites) in shared persistent launches (pq_run_batch),
beside the same 64 instances as sequential pq_run calls on the same GPU.

`--workload adjoint` times the full gradient of a 50-qubit, 12-layer
hardware-efficient ansatz (1200 angles, sum of Z_i Z_i+1, w <= 8,
|c| >= 1e-5) through the adjoint pass, beside a timed sample of the
2400-evaluation parameter-shift gradient (batched propagations) on the same GPU.

`--impl reference` times the CPU restatement of the reference engine (the
oracle) on the host cores instead.  With torchrun (N > 1) every rank runs an
independent replica of the workload (the path does not shard).
"""

from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--workload", default="kicked_ising", choices=["kicked_ising", "kicked_ising_small", "majorana", "majorana_small", "tfim", "batch",
                             "batch_small", "adjoint", "adjoint_small"])
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="CPU baseline sample length")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--blocks-per-sm", type=int, default=0, help="sweep blocks per SM (0 = by live count; batch: as many as fit)")
    ap.add_argument("--fuse-max", type=int, default=0, help="rotations fused into one pass, 1-2 (0 = the engine's 2)")
    ap.add_argument("--tile-items", type=int, default=0, help="rows per thread of a many-row gate tile, 1-4 (0 = 4)")
    ap.add_argument("--no-scattered-reference", action="store_true",
                    help="Majorana lines: skip the scattered-read reference rate (5 GB of device memory)")
    ap.add_argument("--bucket-slots", type=int, default=0, help="hash-table bucket width: 2, 4 or 8 (0 = 2)")
    ap.add_argument("--split", type=int, default=1, help="batch: 0 equal grid shares, 1 by remaining work")
    ap.add_argument("--rebalance-pct", type=int, default=25, help="batch: re-split when this %% of the grid idles")
    ap.add_argument("--no-sequential", action="store_true", help="batch: skip the sequential pq_run comparison")
    ap.add_argument("--no-autotune", action="store_true",
                    help="batch: time the given --blocks-per-sm/--split/--rebalance-pct instead of the autotuner's")
    ap.add_argument("--checkpoint-layers", type=int, default=3, help="adjoint: layers per checkpoint segment")
    ap.add_argument("--shift-sample", type=int, default=480,
                    help="adjoint: parameter-shift evaluations timed in batches of 8")
    ap.add_argument("--shift-sequential", type=int, default=96,
                    help="adjoint: parameter-shift evaluations timed as plain pq_run calls")
    return ap.parse_args()


def make_workload(name):
    from propaq_b200 import workloads

    if name == "kicked_ising":
        wl = workloads.kicked_ising()
        desc = ("kicked Ising 10x10 open lattice, 20 steps, RZZ(-pi/2) x 180 edges + RX(0.6) x 100 per step, "
                "Z(centre), p=1e-3 depolarising as (1-p)^w, w<=10, |c|>=1e-5")
    elif name == "kicked_ising_small":
        wl = workloads.kicked_ising(steps=8)
        desc = ("kicked Ising 10x10 open lattice, 8 steps, RZZ(-pi/2) + RX(0.6), Z(centre), p=1e-3, w<=10, "
                "|c|>=1e-5 (profiling case)")
    elif name == "majorana_small":
        wl = workloads.majorana_givens(n_sites=24, reps=3)
        desc = ("Majorana 24 sites / 48 modes, 3 reps of brick-wall Givens + number-number phases |p-q|<=3, "
                "half filling, JW w<=8, |c|>=1e-6 (profiling case)")
    elif name == "majorana":
        wl = workloads.majorana_givens()
        desc = ("Majorana 32 sites / 64 modes, 4 reps of brick-wall Givens + number-number phases |p-q|<=3, "
                "sum_p c_p g2p g2p+1, half filling, JW w<=8, |c|>=1e-6")
    else:
        wl = workloads.tfim_chain()
        desc = "TFIM chain 20 qubits, 10 Trotter layers, Z10, w<=8, |c|>=1e-4"
    return wl, desc


def measured_peaks():
    f = ROOT / "MEASURED_PEAKS.json"
    if f.exists():
        d = json.loads(f.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def random_sector_rate(device, gib: int = 4, n: int = 1 << 26, reps: int = 5) -> dict:
    """The rate at which this GPU serves scattered reads from memory far larger
    than L2: n 8-byte elements gathered from random positions of a `gib` GiB
    buffer (torch.index_select), each landing in a 32-byte sector of its own.
    A reference point for the HBM-bound sweep, whose partner lookups are such
    reads: `sector_gbs` counts 32 bytes per gathered element, `dram_gbs` adds
    the index and result streams (8 + 8 bytes per element)."""
    import torch

    x = torch.ones(gib * (1 << 30) // 8, dtype=torch.float64, device=device)
    gen = torch.Generator(device=device)
    gen.manual_seed(7)
    idx = torch.randint(0, x.numel(), (n,), device=device, dtype=torch.int64, generator=gen)
    out = torch.empty(n, dtype=torch.float64, device=device)
    for _ in range(2):
        torch.index_select(x, 0, idx, out=out)
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    s.record()
    for _ in range(reps):
        torch.index_select(x, 0, idx, out=out)
    e.record()
    torch.cuda.synchronize()
    sec = s.elapsed_time(e) / 1e3 / reps
    rate = {"elements_per_s": n / sec, "sector_gbs": n * 32 / sec / 1e9, "dram_gbs": n * 48 / sec / 1e9,
            "how": f"{n} random 8-byte reads from a {gib} GiB buffer, torch.index_select, {reps} reps"}
    del x, idx, out
    torch.cuda.empty_cache()
    return rate


class ClockSampler:
    """nvidia-smi clock / throttle samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-i", str(self.dev), "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def dist_backend() -> str:
    """NCCL on GPUs; gloo where there is no GPU (the CPU tests of the replica
    plumbing), or as PQ_DIST_BACKEND says."""
    b = os.environ.get("PQ_DIST_BACKEND")
    if b:
        return b
    import torch

    return "nccl" if torch.cuda.is_available() else "gloo"


def dist_setup():
    """One process per GPU: the replicas share nothing but the barrier and the
    max-over-ranks of the timed region (the path does not shard)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta

        if dist_backend() == "nccl":
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
        else:
            dist.init_process_group("gloo", timeout=timedelta(seconds=120))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def max_over_ranks(world, value: float) -> float:
    if world == 1:
        return value
    import torch
    import torch.distributed as dist

    t = torch.tensor([value], dtype=torch.float64, device="cuda" if dist_backend() == "nccl" else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(world: int, units_per_rank: float, seconds_max: float) -> float:
    """Whole-job throughput of N replicas: all ranks' units over the slowest rank's time."""
    return world * units_per_rank / seconds_max


def gate_bytes(W, rows, anti, children):
    return 8 * W * rows + 16 * anti + (8 + 8 * W) * anti + (8 * W + 16) * children


def run_cpu_baseline(problem_builder, seconds, cores):
    """The oracle (CPU restatement of the reference engine) over whole runs of
    the workload, as many as fit in `seconds` (at least one)."""
    sys.path.insert(0, str(ROOT / "tests"))
    from harness import run_oracle
    from oracle_client import Oracle

    o = Oracle.load()
    p = problem_builder()
    runs, terms, t0 = 0, 0, time.perf_counter()
    while True:
        r = run_oracle(o, p, n_partitions=cores, want_terms=False)
        runs += 1
        terms += int(r.n_terms.sum())
        el = time.perf_counter() - t0
        if el >= seconds:
            break
    return terms / el, runs, el, r


def main_batch(args, world, rank, local):
    """The extrapolation-sweep batch: value = term-gate visits of all 64
    instances per second of the batched launches' device time."""
    sys.path.insert(0, str(ROOT / "tests"))
    from harness import from_workload, make_cfg, run_oracle

    from propaq_b200 import workloads

    if args.workload == "batch_small":  # profiling case: 16 instances, 40..60 qubits, 4..6 steps
        wls = workloads.kicked_ising_batch(16, seed=0, n_range=(40, 60), steps_range=(4, 6))
    else:
        wls = workloads.kicked_ising_batch(64, seed=0)
    probs = [from_workload(w) for w in wls]
    cores = os.cpu_count() or 1
    desc = ("64 kicked-Ising instances, n ~ U{40..100} on the most-square open grid, steps ~ U{8..20}, "
            "RX theta ~ U[0.2,1.0], grid p in {0.5,1,1.5,2}e-3 x |c| cut in {1e-3..1e-6} x 4 Z sites, w<=10")
    base_line = {"metric": "terms/s", "unit": "terms/s", "n_gpus": args.gpus, "steps": args.steps,
                 "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                 "dtype": "f64", "data": "synthetic (seeded; no dataset)",
                 "config": {"workload": desc if args.workload == "batch" else "profiling case: " + args.workload,
                            "name": f"kicked_ising_batch{len(probs)}_seed0", "instances": len(probs),
                            "gates": int(sum(len(p.angles) for p in probs)),
                            "parallelism": f"replicas x{world}", "l2": "flushed between steps"}}
    if args.impl == "reference":
        if rank != 0:
            return
        o = oracle_load()
        # A bounded sample: the instances in order until cpu_seconds pass, per step.
        steps_t, terms_total, inst = [], 0, 0
        for i in range(args.warmup + args.steps):
            t0, terms, k = time.perf_counter(), 0, 0
            while k == 0 or time.perf_counter() - t0 < args.cpu_seconds / max(1, args.warmup + args.steps):
                r = run_oracle(o, probs[(i + k) % len(probs)], n_partitions=cores, want_terms=False)
                terms += int(r.n_terms.sum())
                k += 1
            if i >= args.warmup:
                steps_t.append(time.perf_counter() - t0)
                terms_total += terms
                inst += k
        total = sum(steps_t)
        v = terms_total / total
        line = dict(base_line, impl="reference", value=v, ms_per_step=1e3 * total / len(steps_t),
                    cpu_baseline={"value": v, "unit": "terms/s", "cores": cores, "kind": "port",
                                  "sample": f"{inst} instance runs over {args.steps} steps, oracle with {cores} "
                                            "partitions/threads, instances one after another"},
                    e2e={"value": v, "unit": "terms/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0})
        print(json.dumps(line), flush=True)
        return

    import torch

    from propaq_b200 import PauliPropagator, _native
    from propaq_b200.propagators import expectation_values

    torch.cuda.set_device(local)
    engine = _native.engine(local)
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")
    keep, items = [], []
    for p in probs:
        cfg, k = make_cfg(p, want_terms=False)
        cfg.blocks_per_sm = args.blocks_per_sm
        cfg.fuse_max, cfg.tile_items, cfg.bucket_slots = args.fuse_max, args.tile_items, args.bucket_slots
        keep.append(k)
        items.append((cfg, p.obs_keys, p.obs_coeffs, p.gate_keys, p.angles, p.offsets, p.diag))
    tune = dict(blocks_per_sm=args.blocks_per_sm, split=args.split, rebalance_pct=args.rebalance_pct,
                fuse_max=args.fuse_max, tile_items=args.tile_items, bucket_slots=args.bucket_slots)
    jobs = [(PauliPropagator(noise=w.noise(), truncation=w.truncation(), device=local), w.observable, w.circuit,
             w.initial_state) for w in wls]
    WM = max(p.n_words for p in probs)

    def settle():
        flush.zero_()
        torch.cuda.synchronize()
        barrier(world)

    for _ in range(args.warmup):
        settle()
        engine.run_batch(items, **tune)
    tuned = None
    if not args.no_autotune:
        # The project's autotuner picks the launch and kernel parameters by measurement
        # (propaq_b200.tuning), once per batch shape, before the timed region.
        from propaq_b200.tuning import batch_signature, default_tuner

        tuner = default_tuner()
        t = tuner.tune(items, local)
        tune = t.as_dict()
        tuned = [dict(c.as_dict(), device_ms=ms) for c, ms in tuner.trials[batch_signature(items)]]
    for _ in range(min(1, args.warmup)):
        settle()
        expectation_values(jobs, **tune)
    dev_ms = sweep_ms = 0.0
    terms = launches = sweep_launches = 0
    alg_bytes = 0
    seq_ms, seq_terms, seq_launches = 0.0, 0, 0
    e2e_s, e2e_terms = 0.0, 0
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            settle()
            out = engine.run_batch(items, **tune)
            torch.cuda.synchronize()
            dev_ms += out[0][0].device_ms
            sweep_ms += out[0][0].sweep_ms
            launches += int(out[0][0].gpu_launches)
            sweep_launches += max(int(r.sweep_launches) for r, _ in out)
            for p, (r, nt) in zip(probs, out):
                terms += int(nt.sum())
                W = max(p.n_words, WM // 2)
                alg_bytes += (gate_bytes(W, r.sum_rows_gate, r.sum_anti, r.sum_children) + 8 * W * r.sum_rows_phase
                              + (8 * W + 16) * (r.sum_rows_noise + r.sum_kept))
        for _ in range(args.steps):
            settle()
            t0 = time.perf_counter()
            rs = expectation_values(jobs, **tune)
            torch.cuda.synchronize()
            e2e_s += time.perf_counter() - t0
            e2e_terms += sum(sum(r.n_terms) for r in rs)
        if not args.no_sequential:
            for _ in range(args.steps):
                for p, it in zip(probs, items):
                    settle()
                    r, nt = engine.run(*it)
                    seq_ms += r.device_ms
                    seq_terms += int(nt.sum())
                    seq_launches += int(r.gpu_launches)
    clocks = clk.summary()
    dev_s = max_over_ranks(world, dev_ms / 1e3)
    e2e_s = max_over_ranks(world, e2e_s)
    value = replica_value(world, terms, dev_s)
    h2d = sum(p.obs_keys.nbytes + p.obs_coeffs.nbytes + p.gate_keys.nbytes + p.angles.nbytes + p.offsets.nbytes
              + (0 if p.diag is None else p.diag.nbytes) + (0 if p.noise_table is None else p.noise_table.nbytes)
              for p in probs)
    d2h = sum(8 * len(p.angles) + 16 * (len(p.angles) + len(p.offsets) - 1) + 32 * 4 * 148 for p in probs)
    peak_gbs, peak_kind = measured_peaks()
    achieved = alg_bytes / (sweep_ms / 1e3) / 1e9 if sweep_ms > 0 else None
    line = dict(base_line, value=value, ms_per_step=1e3 * dev_s / args.steps,
                instances_per_s=world * len(probs) * args.steps / dev_s,
                e2e={"value": world * e2e_terms / e2e_s, "unit": "terms/s", "h2d_bytes_per_step": int(h2d),
                     "d2h_bytes_per_step": int(d2h), "ms_per_step": 1e3 * e2e_s / args.steps},
                gpu_launches=launches // max(1, args.steps),
                roofline={"bound": "hbm", "achieved": achieved, "peak": peak_gbs, "unit": "GB/s",
                          "frac": None if achieved is None else achieved / peak_gbs, "traffic": None,
                          "kernel": "batch_sweep_kernel", "peak_source": f"{peak_kind} hbm_gbs",
                          "launches_per_step": sweep_launches / max(1, args.steps),
                          "share_of_device_time": sweep_ms / dev_ms if dev_ms else None},
                tuning=dict(tune, autotuned=tuned is not None, trials=tuned), clocks=clocks)
    if seq_ms:
        line["sequential"] = {"what": "the same 64 instances as pq_run calls one after another, same GPU",
                              "value": seq_terms / (seq_ms / 1e3), "ms_per_step": seq_ms / args.steps,
                              "instances_per_s": len(probs) * args.steps / (seq_ms / 1e3),
                              "gpu_launches_per_step": seq_launches // args.steps}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        o = oracle_load()
        t0, terms_c, k = time.perf_counter(), 0, 0
        while k == 0 or time.perf_counter() - t0 < args.cpu_seconds:
            r = run_oracle(o, probs[k % len(probs)], n_partitions=cores, want_terms=False)
            terms_c += int(r.n_terms.sum())
            k += 1
        el = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": terms_c / el, "unit": "terms/s", "cores": cores, "kind": "port",
                                "sample": f"the first {k} instance(s) one after another in {el:.1f} s, oracle "
                                          f"with {cores} partitions/threads"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()


def main_adjoint(args, world, rank, local):
    """The ansatz gradient.  value = full gradients per second of device time
    (forward + reverse pass)."""
    sys.path.insert(0, str(ROOT / "tests"))
    from harness import from_workload, run_oracle

    from propaq_b200 import PauliPropagator, workloads
    from propaq_b200.adjoint import ParametrizedExpectation

    # adjoint_small is the profiling case: 20 qubits, 4 layers
    wl = workloads.hardware_efficient(20, 4) if args.workload == "adjoint_small" else workloads.hardware_efficient()
    th = wl.meta["theta"]
    desc = ("hardware-efficient ansatz 50 qubits, 12 layers of RY+RZ on all + CNOT ladder (Z_c(pi/2), X_t(pi/2), "
            "Z_cX_t(-pi/2)), 1200 angles ~ N(0,0.1), sum Z_i Z_i+1, |0..0>, w<=8, |c|>=1e-5, no noise")
    cores = os.cpu_count() or 1
    base_line = {"metric": "gradients/s", "unit": "gradients/s", "n_gpus": args.gpus, "steps": args.steps,
                 "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                 "dtype": "f64", "data": "synthetic (seeded; no dataset)",
                 "config": {"workload": desc if args.workload == "adjoint" else "profiling case: " + wl.name,
                            "name": wl.name, "n_units": wl.n_units, "angles": len(th),
                            "gates": len(wl.circuit.rotations), "checkpoint_layers": args.checkpoint_layers,
                            "parallelism": f"replicas x{world}", "l2": "flushed between steps"}}
    spec_cpu = ParametrizedExpectation(PauliPropagator(truncation=wl.truncation()), wl.observable, wl.circuit,
                                       wl.meta["param_index"])
    n_shift = 2 * len(spec_cpu._param_gates)
    if args.impl == "reference":
        if rank != 0:
            return
        # The reference has no gradient: its CPU arm is the parameter-shift rule
        # on the oracle, timed on a bounded sample of evaluations.
        o = oracle_load()
        p = from_workload(wl)
        base = spec_cpu._call_args(th)
        n_eval, t0 = 0, time.perf_counter()
        while n_eval < 2 or time.perf_counter() - t0 < args.cpu_seconds:
            g = spec_cpu._param_gates[(n_eval // 2) % len(spec_cpu._param_gates)]
            p.angles = base[4].copy()
            p.angles[g] += (1 if n_eval % 2 == 0 else -1) * math.pi / 2
            run_oracle(o, p, n_partitions=cores, want_terms=False)
            n_eval += 1
        el = time.perf_counter() - t0
        per_grad = el / n_eval * n_shift
        v = 1.0 / per_grad
        line = dict(base_line, impl="reference", value=v, ms_per_step=1e3 * per_grad,
                    cpu_baseline={"value": v, "unit": "gradients/s", "cores": cores, "kind": "port",
                                  "sample": f"{n_eval} parameter-shift evaluations in {el:.1f} s on the oracle "
                                            f"({cores} threads), scaled to {n_shift}"},
                    e2e={"value": v, "unit": "gradients/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0})
        print(json.dumps(line), flush=True)
        return

    import torch

    from propaq_b200 import _native

    torch.cuda.set_device(local)
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{local}")
    prop = PauliPropagator(truncation=wl.truncation(), device=local)
    spec = ParametrizedExpectation(prop, wl.observable, wl.circuit, wl.meta["param_index"],
                                   checkpoint_layers=args.checkpoint_layers)
    theta = torch.tensor(th, dtype=torch.float64)

    def settle():
        flush.zero_()
        torch.cuda.synchronize()
        barrier(world)

    for _ in range(args.warmup):
        settle()
        spec.value_and_grad(th)
    dev_ms = fwd_ms = 0.0
    launches = 0
    e2e_s = 0.0
    alg = 0.0
    W = _native.words_for_units(wl.n_units)
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            settle()
            spec.value(th)
            fwd_ms += prop.last_run.device_ms
            settle()
            e, g = spec.value_and_grad(th)
            r = prop.last_run
            dev_ms += r.device_ms
            launches += int(r.gpu_launches)
            # algorithmic bytes: the forward sweep (as the plain bench) and the
            # reverse sweep: per gate op keys, lambda in and out of every row,
            # the record (coefficient + partner index) and the partner's lambda
            # of every anticommuting row; per noise op keys, both lambdas and
            # the reclaim map
            fwd = (gate_bytes(W, r.sum_rows_gate, r.sum_anti, r.sum_children) + 8 * W * r.sum_rows_phase
                   + (8 * W + 16) * (r.sum_rows_noise + r.sum_kept))
            rev = (8 * W + 16) * (r.sum_rows_gate + r.sum_rows_phase) + 20 * r.sum_anti + (8 * W + 20) * r.sum_rows_noise
            alg += fwd + rev
        for _ in range(args.steps):
            settle()
            t0 = time.perf_counter()
            th_req = theta.clone().requires_grad_(True)
            spec(th_req).backward()
            _ = th_req.grad.numpy().sum()
            e2e_s += time.perf_counter() - t0
        # Parameter shift: timed samples of its 2 x 1200 propagations, spread
        # over the angles, scaled to the full count: one plain pq_run call per
        # evaluation, and 8 evaluations per pq_run_batch call.
        base = spec._call_args(th)
        eng = _native.engine(local)
        items = []
        step = max(1, n_shift // args.shift_sample)
        for k in range(0, n_shift, step):
            gi = spec._param_gates[(k // 2) % len(spec._param_gates)]
            a = base[4].copy()
            a[gi] += (1 if k % 2 == 0 else -1) * math.pi / 2
            items.append(tuple(base[:4]) + (a,) + tuple(base[5:]))
        items = items[:args.shift_sample]
        settle()
        ps_ms = 0.0
        for i in range(0, len(items), 8):
            out = eng.run_batch(items[i:i + 8], want_n_terms=False)
            ps_ms += out[0][0].device_ms
        settle()
        seq_ms = 0.0
        n_seq = min(len(items), args.shift_sequential)
        for it in items[:n_seq]:
            res, _ = eng.run(*it, want_n_terms=False)
            seq_ms += res.device_ms
    clocks = clk.summary()
    dev_s = max_over_ranks(world, dev_ms / 1e3)
    e2e_s = max_over_ranks(world, e2e_s)
    shift_ms = ps_ms / len(items) * n_shift
    seq_shift_ms = seq_ms / max(1, n_seq) * n_shift
    h2d = sum(int(np.asarray(x).nbytes) for x in base[1:] if x is not None) + 8 * len(th)
    peak_gbs, peak_kind = measured_peaks()
    achieved = alg / (dev_ms / 1e3) / 1e9 if dev_ms > 0 else None
    line = dict(base_line, value=world * args.steps / dev_s, ms_per_step=1e3 * dev_s / args.steps,
                forward_ms=fwd_ms / args.steps, expectation_value=e,
                e2e={"value": world * args.steps / e2e_s, "unit": "gradients/s", "h2d_bytes_per_step": int(h2d),
                     "d2h_bytes_per_step": 8 * len(spec._fixed) * 2, "ms_per_step": 1e3 * e2e_s / args.steps,
                     "path": "torch.autograd: ParametrizedExpectation(theta).backward()"},
                gpu_launches=launches // max(1, args.steps),
                parameter_shift={"evaluations": n_shift, "timed_sample": len(items),
                                 "sample": f"every {step}th of the {n_shift} shifted circuits",
                                 "ms_per_evaluation": ps_ms / len(items), "ms_per_gradient": shift_ms,
                                 "how": "pq_run_batch, 8 shifted circuits per call, device time",
                                 "adjoint_speedup": shift_ms / (1e3 * dev_s / args.steps),
                                 "sequential": {"timed_sample": n_seq, "ms_per_evaluation": seq_ms / max(1, n_seq),
                                                "ms_per_gradient": seq_shift_ms,
                                                "how": "one pq_run call per shifted circuit, device time",
                                                "adjoint_speedup": seq_shift_ms / (1e3 * dev_s / args.steps)}},
                roofline={"bound": "hbm", "achieved": achieved, "peak": peak_gbs, "unit": "GB/s",
                          "frac": None if achieved is None else achieved / peak_gbs, "traffic": None,
                          "kernel": "sweep_kernel + adjoint_kernel", "peak_source": f"{peak_kind} hbm_gbs",
                          "algorithmic_bytes_per_gradient": alg / args.steps,
                          "note": "forward sweep and reverse sweep bytes over the gradient's device time"},
                clocks=clocks)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # the reference has no gradient: its CPU path is parameter shift on the
        # oracle, timed on a bounded sample of evaluations
        o = oracle_load()
        p = from_workload(wl)
        n_eval, t0 = 0, time.perf_counter()
        while n_eval < 2 or time.perf_counter() - t0 < args.cpu_seconds:
            gi = spec_cpu._param_gates[(n_eval // 2) % len(spec_cpu._param_gates)]
            p.angles = base[4].copy()
            p.angles[gi] += (1 if n_eval % 2 == 0 else -1) * math.pi / 2
            run_oracle(o, p, n_partitions=cores, want_terms=False)
            n_eval += 1
        el = time.perf_counter() - t0
        v = 1.0 / (el / n_eval * n_shift)
        line["cpu_baseline"] = {"value": v, "unit": "gradients/s", "cores": cores, "kind": "port",
                                "sample": f"{n_eval} parameter-shift evaluations in {el:.1f} s on the oracle "
                                          f"({cores} threads), scaled to {n_shift}"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()


def oracle_load():
    sys.path.insert(0, str(ROOT / "tests"))
    from oracle_client import Oracle

    return Oracle.load()


def main():
    args = parse()
    world, rank, local = dist_setup()
    if args.workload in ("batch", "batch_small"):
        return main_batch(args, world, rank, local)
    if args.workload in ("adjoint", "adjoint_small"):
        return main_adjoint(args, world, rank, local)
    wl, desc = make_workload(args.workload)
    cores = os.cpu_count() or 1
    W = 1
    while 32 * W < wl.n_units:
        W *= 2

    def builder():
        sys.path.insert(0, str(ROOT / "tests"))
        from harness import from_workload

        return from_workload(wl)

    base_line = {"metric": "terms/s", "unit": "terms/s", "n_gpus": args.gpus, "steps": args.steps,
                 "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                 "dtype": "f64", "data": "synthetic (seeded; no dataset)",
                 "config": {"workload": desc, "name": wl.name, "n_units": wl.n_units, "key_words": W,
                            "gates": len(wl.circuit.rotations), "layers": len(wl.circuit.layers),
                            "parallelism": f"replicas x{world}", "l2": "flushed between steps"}}

    if args.impl == "reference":
        if rank != 0:
            return
        steps_t, terms_total = [], 0
        sys.path.insert(0, str(ROOT / "tests"))
        from harness import run_oracle
        from oracle_client import Oracle

        o = Oracle.load()
        p = builder()
        for i in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            r = run_oracle(o, p, n_partitions=cores, want_terms=False)
            dt = time.perf_counter() - t0
            if i >= args.warmup:
                steps_t.append(dt)
                terms_total += int(r.n_terms.sum())
        total = sum(steps_t)
        v = terms_total / total
        line = dict(base_line, impl="reference", value=v, ms_per_step=1e3 * total / len(steps_t),
                    cpu_baseline={"value": v, "unit": "terms/s", "cores": cores, "kind": "port",
                                  "sample": f"whole workload per step, oracle with {cores} partitions/threads"},
                    e2e={"value": v, "unit": "terms/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
                    expectation_value=r.expectation)
        print(json.dumps(line), flush=True)
        return

    import torch

    from propaq_b200 import MajoranaPropagator, PauliPropagator, _native

    torch.cuda.set_device(local)
    dev = f"cuda:{local}"
    engine = _native.engine(local)
    prob = builder()
    # A 512 MB write between steps evicts the 126 MB L2.
    flush = torch.empty(512 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    cfg = _native.RunConfig()
    cfg.basis_kind = prob.basis
    cfg.n_units = prob.n_units
    cfg.max_weight = -1 if prob.max_weight is None else prob.max_weight
    cfg.has_min_coeff = 0 if prob.min_coeff is None else 1
    cfg.min_coeff = 0.0 if prob.min_coeff is None else prob.min_coeff
    cfg.min_terms = -1
    table = None
    if prob.noise_table is not None:
        table = np.ascontiguousarray(prob.noise_table, dtype=np.float64)
        cfg.noise_kind, cfg.noise_tables, cfg.noise_table_len = _native.PQ_NOISE_TABLE, table.ctypes.data, len(table)
    cfg.want_terms = 0
    cfg.blocks_per_sm = args.blocks_per_sm
    cfg.fuse_max, cfg.tile_items, cfg.bucket_slots = args.fuse_max, args.tile_items, args.bucket_slots

    def device_step():
        return engine.run(cfg, prob.obs_keys, prob.obs_coeffs, prob.gate_keys, prob.angles, prob.offsets, prob.diag)

    prop_cls = PauliPropagator if wl.basis == 0 else MajoranaPropagator
    prop = prop_cls(noise=wl.noise(), truncation=wl.truncation(), device=local)

    def api_step():
        return prop.expectation_value(wl.observable, wl.circuit, initial_state=wl.initial_state)

    def settle():
        flush.zero_()
        torch.cuda.synchronize()
        barrier(world)

    for _ in range(args.warmup):
        settle()
        device_step()
        settle()
        api_step()

    dev_ms = sweep_ms = gate_ms = 0.0
    terms = launches = sweep_launches = gate_ops = 0
    alg_bytes = galg = 0
    e2e_s = 0.0
    e2e_terms = 0
    peak = 0
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            settle()
            res, nt = device_step()
            torch.cuda.synchronize()
            dev_ms += res.device_ms
            sweep_ms += res.sweep_ms
            gate_ms += res.gate_ms
            terms += int(nt.sum())
            launches += int(res.gpu_launches)
            sweep_launches += int(res.sweep_launches)
            gate_ops += int(res.gate_ops)
            peak = max(peak, int(res.peak_terms))
            g = gate_bytes(W, res.sum_rows_gate, res.sum_anti, res.sum_children)
            galg += g
            alg_bytes += (g + 8 * W * res.sum_rows_phase
                          + (8 * W + 16) * (res.sum_rows_noise + res.sum_kept))
        for _ in range(args.steps):
            settle()
            t0 = time.perf_counter()
            r = api_step()
            torch.cuda.synchronize()
            e2e_s += time.perf_counter() - t0
            e2e_terms += sum(r.n_terms)
    clocks = clk.summary()
    dev_s = max_over_ranks(world, dev_ms / 1e3)
    e2e_s = max_over_ranks(world, e2e_s)
    value = replica_value(world, terms, dev_s)
    e2e_value = world * e2e_terms / e2e_s
    # host <-> device bytes per step of pq_run: observable, gates, offsets,
    # state and noise table in; per-gate counts, per-op counters and the
    # expectation partials out.
    n_ops = len(prob.angles) + len(prob.offsets) - 1
    h2d = (prob.obs_keys.nbytes + prob.obs_coeffs.nbytes + prob.gate_keys.nbytes + prob.angles.nbytes
           + prob.offsets.nbytes + (0 if prob.diag is None else prob.diag.nbytes)
           + (0 if table is None else table.nbytes))
    d2h = 8 * len(prob.angles) + 16 * n_ops + 32 * 4 * 148
    peak_gbs, peak_kind = measured_peaks()
    # The dominant kernel is the sweep: one cooperative launch per step (plus
    # one per capacity growth) runs every gate and noise op.
    achieved = alg_bytes / (sweep_ms / 1e3) / 1e9 if sweep_ms > 0 else None
    # DRAM bytes of the sweep launches of one step, from an ncu capture
    # (profiles/sweep_traffic_*.json), as bytes per launch like `achieved`:
    # the step's bytes over the launches a step took here (the grid follows
    # the live count, so a step can be several launches).
    traffic = None
    tf = ROOT / "profiles" / f"sweep_traffic_{wl.name}.json"
    if tf.exists() and sweep_launches:
        per_step = json.loads(tf.read_text()).get("dram_bytes_per_step")
        if per_step is not None:
            traffic = per_step / (sweep_launches / args.steps)
    # For the HBM-bound Majorana runs: the sweep's DRAM rate (traffic over the
    # launch time) beside the rate random 32-byte reads reach on this GPU.
    scattered = None
    if wl.basis == 1 and traffic is not None and sweep_ms > 0 and not args.no_scattered_reference:
        rate = random_sector_rate(f"cuda:{local}")
        dram_gbs = traffic / (sweep_ms / max(1, sweep_launches) / 1e3) / 1e9
        scattered = dict(rate, sweep_dram_gbs=dram_gbs, sweep_frac_of_scattered=dram_gbs / rate["dram_gbs"])
    line = dict(base_line, value=value, ms_per_step=1e3 * dev_s / args.steps,
                e2e={"value": e2e_value, "unit": "terms/s", "h2d_bytes_per_step": int(h2d),
                     "d2h_bytes_per_step": int(d2h), "ms_per_step": 1e3 * e2e_s / args.steps},
                gpu_launches=launches,
                roofline={"bound": "hbm", "achieved": achieved, "peak": peak_gbs, "unit": "GB/s",
                          "frac": None if achieved is None else achieved / peak_gbs, "traffic": traffic,
                          "kernel": "sweep_kernel", "peak_source": f"{peak_kind} hbm_gbs",
                          "launches": sweep_launches,
                          "algorithmic_bytes_per_launch": alg_bytes / max(1, sweep_launches),
                          "ms_per_launch": sweep_ms / max(1, sweep_launches),
                          "share_of_device_time": sweep_ms / dev_ms if dev_ms else None,
                          "gate_ops_gbs": galg / (gate_ms / 1e3) / 1e9 if gate_ms > 0 else None,
                          "us_per_gate_op": 1e3 * gate_ms / max(1, gate_ops),
                          "scattered_reads": scattered},
                clocks=clocks, peak_terms=peak, expectation_value=r.expectation_value)
    line["config"]["parallelism"] = f"replicas x{world}"
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, runs, el, ores = run_cpu_baseline(builder, args.cpu_seconds, cores)
        line["cpu_baseline"] = {"value": v, "unit": "terms/s", "cores": cores, "kind": "port",
                                "sample": f"{runs} whole run(s) of the workload in {el:.1f} s, oracle with "
                                          f"{cores} partitions/threads"}
        # the same run's answer from the oracle, with the plain relative error
        # of the engine's expectation value against it
        ref = ores.expectation_accurate
        line["oracle_expectation_value"] = ref
        line["rel_err_vs_oracle"] = abs(r.expectation_value - ref) / abs(ref) if ref else abs(r.expectation_value)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
