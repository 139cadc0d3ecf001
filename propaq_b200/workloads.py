"""Seeded synthetic workloads with the shapes of the reference's headline
propagation configurations (the circuits, observables, cutoffs and noise the
benchmarks and parity tests run).  Angles and coefficients are drawn with
numpy.random.default_rng(seed); no dataset is involved.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from .circuits import (
    MajoranaCircuit,
    PauliCircuit,
    majorana_cp,
    majorana_xx_plus_yy,
    pauli_cx,
    pauli_rx,
    pauli_ry,
    pauli_rz,
    pauli_rzz,
)
from .datatypes import MajoranaMonomial, MajoranaTermSum, PauliString, PauliTermSum
from .noise import UniformNoiseModel
from .truncation import CoefficientTruncator, WeightTruncator


@dataclass
class Workload:
    name: str
    basis: int                  # 0 Pauli, 1 Majorana
    n_units: int                # qubits, or sites for Majorana
    observable: object
    circuit: object
    max_weight: int | None
    min_coeff: float | None
    noise_damping: float | None = None
    initial_state: int = 0
    meta: dict = field(default_factory=dict)

    def truncation(self):
        t = []
        if self.max_weight is not None:
            t.append(WeightTruncator(self.max_weight))
        if self.min_coeff is not None:
            t.append(CoefficientTruncator(self.min_coeff))
        return t

    def noise(self):
        return None if self.noise_damping is None else UniformNoiseModel(self.noise_damping)


def tfim_chain(n: int = 20, steps: int = 10, seed: int = 0, max_weight=8, min_coeff=1e-4, site: int | None = None):
    """Open chain: per Trotter step RZZ(theta) on even bonds, then odd bonds, then
    RX(theta) on every qubit; theta ~ U[0, pi/2) per gate; observable Z on the
    middle qubit; state |0...0>."""
    rng = np.random.default_rng(seed)
    layers = []
    for _ in range(steps):
        for parity in (0, 1):
            layers.append([r for i in range(parity, n - 1, 2)
                           for r in pauli_rzz(i, i + 1, float(rng.uniform(0, math.pi / 2)), n)])
        layers.append([r for q in range(n) for r in pauli_rx(q, float(rng.uniform(0, math.pi / 2)), n)])
    obs = PauliTermSum()
    obs.add(PauliString(0, 1 << (n // 2 if site is None else site), n), 1.0)
    return Workload(f"tfim_chain_n{n}_d{steps}", 0, n, obs, PauliCircuit(layers), max_weight, min_coeff,
                    meta={"seed": seed, "steps": steps})


def grid_edges(rows: int, cols: int):
    """The four colour classes of an open rows x cols lattice: horizontal bonds
    starting at even / odd columns, vertical bonds starting at even / odd rows."""
    q = lambda r, c: r * cols + c  # noqa: E731
    h_even = [(q(r, c), q(r, c + 1)) for r in range(rows) for c in range(0, cols - 1, 2)]
    h_odd = [(q(r, c), q(r, c + 1)) for r in range(rows) for c in range(1, cols - 1, 2)]
    v_even = [(q(r, c), q(r + 1, c)) for r in range(0, rows - 1, 2) for c in range(cols)]
    v_odd = [(q(r, c), q(r + 1, c)) for r in range(1, rows - 1, 2) for c in range(cols)]
    return [h_even, h_odd, v_even, v_odd]


def kicked_ising(rows: int = 10, cols: int = 10, steps: int = 20, theta: float = 0.6, p: float = 1e-3,
                 max_weight=10, min_coeff=1e-5, site: int | None = None):
    """Kicked Ising on an open lattice: per step RZZ(-pi/2) on every edge, one
    circuit layer per colour class, then RX(theta) on every qubit as one layer;
    depolarising p per qubit per layer as (1-p)^weight damping; observable Z at
    the centre."""
    n = rows * cols
    classes = grid_edges(rows, cols)
    layers = []
    for _ in range(steps):
        for cls in classes:
            layers.append([r for (i, j) in cls for r in pauli_rzz(i, j, -math.pi / 2, n)])
        layers.append([r for qb in range(n) for r in pauli_rx(qb, theta, n)])
    centre = (rows // 2) * cols + cols // 2 if site is None else site
    obs = PauliTermSum()
    obs.add(PauliString(0, 1 << centre, n), 1.0)
    damping = None if not p else -math.log1p(-p)
    return Workload(f"kicked_ising_{rows}x{cols}_s{steps}", 0, n, obs, PauliCircuit(layers), max_weight,
                    min_coeff, damping, meta={"steps": steps, "theta": theta, "p": p})


def majorana_givens(n_sites: int = 32, reps: int = 4, seed: int = 0, max_weight=8, min_coeff=1e-6,
                    cp_range: int = 3, n_occupied: int | None = None):
    """Per repetition: brick-wall nearest-neighbour Givens rotations
    xx_plus_yy(theta, 0) on (p, p+1), even then odd pairs, theta ~ U[-pi, pi);
    then number-number phases cp(theta) on every pair with |p-q| <= cp_range,
    theta ~ N(0, 0.5).  Observable sum_p c_p gamma_2p gamma_2p+1, c_p ~ N(0,1);
    state: a determinant with n_sites/2 seeded occupied sites."""
    rng = np.random.default_rng(seed)
    n_modes = 2 * n_sites
    layers = []
    for _ in range(reps):
        for parity in (0, 1):
            layers.append([r for pp in range(parity, n_sites - 1, 2)
                           for r in majorana_xx_plus_yy(pp, pp + 1, float(rng.uniform(-math.pi, math.pi)), n_modes)])
        layers.append([r for pp in range(n_sites) for qq in range(pp + 1, min(n_sites, pp + cp_range + 1))
                       for r in majorana_cp(pp, qq, float(rng.normal(0.0, 0.5)), n_modes)])
    obs = MajoranaTermSum()
    for pp in range(n_sites):
        obs.add(MajoranaMonomial((1 << (2 * pp)) | (1 << (2 * pp + 1)), n_modes), float(rng.normal()))
    occ = rng.choice(n_sites, size=n_sites // 2 if n_occupied is None else n_occupied, replace=False)
    state = 0
    for s in occ:
        state |= 1 << int(s)
    return Workload(f"majorana_givens_{n_sites}s_r{reps}", 1, n_sites, obs, MajoranaCircuit(layers), max_weight,
                    min_coeff, None, state, meta={"seed": seed, "reps": reps})


def most_square_grid(n: int):
    """(rows, cols) with rows * cols = n and rows the largest divisor <= sqrt(n)."""
    rows = max(d for d in range(1, math.isqrt(n) + 1) if n % d == 0)
    return rows, n // rows


def kicked_ising_batch(n_instances: int = 64, seed: int = 0, n_range=(40, 100), steps_range=(8, 20),
                       theta_range=(0.2, 1.0), ps=(0.5e-3, 1e-3, 1.5e-3, 2e-3),
                       min_coeffs=(1e-3, 1e-4, 1e-5, 1e-6), max_weight=10):
    """Independent kicked-Ising instances of uneven size, as a zero-noise /
    zero-cutoff extrapolation sweep runs them: instance i takes noise p and
    coefficient cutoff from the grid ps x min_coeffs x 4 observable sites
    (i mod 64), and its qubit count (on the most-square open grid), step count
    and RX angle from numpy.random.default_rng(seed).  The 4 observables are Z
    on the centre site and its neighbours up, left and up-left."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n_instances):
        n = int(rng.integers(n_range[0], n_range[1] + 1))
        steps = int(rng.integers(steps_range[0], steps_range[1] + 1))
        theta = float(rng.uniform(*theta_range))
        g = i % (len(ps) * len(min_coeffs) * 4)
        p = ps[g // (len(min_coeffs) * 4)]
        cut = min_coeffs[(g // 4) % len(min_coeffs)]
        rows, cols = most_square_grid(n)
        r0, c0 = rows // 2, cols // 2
        dr, dc = [(0, 0), (-1, 0), (0, -1), (-1, -1)][g % 4]
        site = max(r0 + dr, 0) * cols + max(c0 + dc, 0)
        wl = kicked_ising(rows, cols, steps, theta, p, max_weight, cut, site=site)
        wl.name = f"batch{i}_{rows}x{cols}_s{steps}"
        wl.meta.update({"index": i, "site": site, "min_coeff": cut})
        out.append(wl)
    return out


def hardware_efficient(n: int = 50, layers: int = 12, seed: int = 0, sigma: float = 0.1, max_weight=8,
                       min_coeff=1e-5):
    """Hardware-efficient ansatz: per layer RY(theta) on every qubit, RZ(theta)
    on every qubit, then a CNOT ladder (q, q+1) for q = 0..n-2 (each CNOT as
    Z_c(pi/2), X_t(pi/2), Z_c X_t(-pi/2)); one circuit layer per ansatz layer.
    2 n layers angles ~ N(0, sigma) from numpy.random.default_rng(seed).
    Observable sum_i Z_i Z_i+1; state |0...0>; no noise.

    meta["param_index"][k] is the angle index of rotation k (circuit order), or
    -1 for the fixed CNOT pieces; meta["theta"] holds the angles."""
    rng = np.random.default_rng(seed)
    theta = rng.normal(0.0, sigma, size=2 * n * layers)
    circ_layers, pidx = [], []
    k = 0
    for _ in range(layers):
        rots = []
        for gate in (pauli_ry, pauli_rz):
            for q in range(n):
                rots += gate(q, float(theta[k]), n)
                pidx.append(k)
                k += 1
        for q in range(n - 1):
            cx = pauli_cx(q, q + 1, n)
            rots += cx
            pidx += [-1] * len(cx)
        circ_layers.append(rots)
    obs = PauliTermSum()
    for i in range(n - 1):
        obs.add(PauliString(0, (1 << i) | (1 << (i + 1)), n), 1.0)
    return Workload(f"hea_{n}q_{layers}l", 0, n, obs, PauliCircuit(circ_layers), max_weight, min_coeff,
                    meta={"seed": seed, "layers": layers, "theta": theta, "param_index": np.array(pidx)})
