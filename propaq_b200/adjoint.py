"""Gradients of expectation values with respect to circuit angles.

E(theta) = <s| U(theta)^dag O U(theta) |s> for a circuit whose rotation k
(circuit order) has angle  scale[k] * theta[index[k]]  (index[k] = -1 keeps
the circuit's own angle, e.g. the fixed pieces of a CNOT).

The gradient comes from pq_run_adjoint: one forward propagation that records
every op (and keeps the live terms every `checkpoint_layers` circuit layers),
then a reverse sweep on the GPU that carries dE/dc back through every op with
the forward run's truncation decisions held fixed.  `record_bytes` bounds the
device memory of the records (0: 40% of the free memory); past it, segments
are re-run to record them.  It is the exact derivative of
the function the engine evaluates wherever those decisions do not change
under a small change of theta (and the exact derivative of the untruncated
expectation when nothing is truncated).

`ParametrizedExpectation(...)(theta)` is a torch.autograd.Function: the
forward pass returns E as a 0-d tensor, the backward pass returns
grad_output * dE/dtheta.  parameter_shift() gives the 2-evaluations-per-angle
alternative through batched propagation, for comparison.

The reference has no derivative of a truncated propagation; its surrogate
models (crates/surrogate) evaluate symbolic coefficients for new angles but
expose no gradient.
"""

from __future__ import annotations

import math

import numpy as np

from . import _native
from .propagators import heisenberg_gates


def _heisenberg_order(circuit) -> np.ndarray:
    """order[g] = circuit-order index of the rotation the engine applies g-th
    (layers reversed, gates of each layer reversed, as heisenberg_gates)."""
    starts, k = [], 0
    layers = [list(layer) for layer in circuit.layers]
    for layer in layers:
        starts.append(k)
        k += len(layer)
    order = []
    for li in reversed(range(len(layers))):
        order.extend(starts[li] + j for j in reversed(range(len(layers[li]))))
    return np.array(order, dtype=np.int64)


class ParametrizedExpectation:
    """E(theta) and dE/dtheta of one observable, circuit and state under one
    propagator's noise and truncation, with the circuit's angles tied to a
    parameter vector."""

    def __init__(self, propagator, observable, circuit, param_index, param_scale=None, initial_state=0,
                 checkpoint_layers: int = 3, record_bytes: int = 0):
        args, n_words, n_units, keep = propagator._inputs(observable, circuit, initial_state, False)
        self._args = list(args)
        self._keep = keep
        self.propagator = propagator
        self.device = propagator.device
        self.checkpoint_layers = int(checkpoint_layers)
        self.record_bytes = int(record_bytes)
        self.n_words = n_words
        order = _heisenberg_order(circuit)
        idx = np.asarray(param_index, dtype=np.int64)
        if len(idx) != len(order):
            raise ValueError(f"param_index has {len(idx)} entries for {len(order)} rotations")
        scale = np.ones(len(idx)) if param_scale is None else np.asarray(param_scale, dtype=np.float64)
        self.n_params = int(idx.max()) + 1 if len(idx) and idx.max() >= 0 else 0
        self._gate_param = idx[order]            # parameter of engine gate g, or -1
        self._gate_scale = scale[order]
        self._fixed = np.array(args[4], dtype=np.float64)  # the circuit's own angles, engine order
        self._param_gates = np.nonzero(self._gate_param >= 0)[0]

    def angles(self, theta) -> np.ndarray:
        theta = np.asarray(theta, dtype=np.float64).reshape(-1)
        if len(theta) != self.n_params:
            raise ValueError(f"expected {self.n_params} angles, got {len(theta)}")
        a = self._fixed.copy()
        g = self._param_gates
        a[g] = self._gate_scale[g] * theta[self._gate_param[g]]
        return a

    def _call_args(self, theta):
        args = list(self._args)
        args[4] = self.angles(theta)
        return args

    def value(self, theta) -> float:
        res, _ = _native.engine(self.device).run(*self._call_args(theta))
        self.propagator.last_run = res
        return float(res.expectation_value)

    def value_and_grad(self, theta):
        """(E, dE/dtheta) from one forward and one reverse pass."""
        res, _, g_gate = _native.engine(self.device).run_adjoint(*self._call_args(theta),
                                                                 checkpoint_layers=self.checkpoint_layers,
                                                                 record_bytes=self.record_bytes)
        self.propagator.last_run = res
        return float(res.expectation_value), self._chain(g_gate)

    def _chain(self, g_gate) -> np.ndarray:
        grad = np.zeros(self.n_params)
        g = self._param_gates
        np.add.at(grad, self._gate_param[g], self._gate_scale[g] * g_gate[g])
        return grad

    def parameter_shift(self, theta, batch: int = 16, **tuning) -> np.ndarray:
        """dE/dtheta by the two-term shift rule, E(angle + pi/2) - E(angle - pi/2)
        over 2, for every parametrised rotation: 2 propagations per rotation,
        run `batch` at a time through pq_run_batch."""
        base = self._call_args(theta)
        eng = _native.engine(self.device)
        g_gate = np.zeros(len(self._fixed))
        jobs = [(g, sgn) for g in self._param_gates for sgn in (1.0, -1.0)]
        vals = {}
        for i in range(0, len(jobs), batch):
            items = []
            for g, sgn in jobs[i:i + batch]:
                a = base[4].copy()
                a[g] += sgn * math.pi / 2
                items.append(tuple(base[:4]) + (a,) + tuple(base[5:]))
            out = eng.run_batch(items, want_n_terms=False, **tuning)
            for (g, sgn), (res, _) in zip(jobs[i:i + batch], out):
                vals[(g, sgn)] = res.expectation_value
        for g in self._param_gates:
            g_gate[g] = 0.5 * (vals[(g, 1.0)] - vals[(g, -1.0)])
        return self._chain(g_gate)

    def __call__(self, theta):
        return ExpectationFunction.apply(theta, self)


def _torch_function():
    import torch

    class _Expectation(torch.autograd.Function):
        """E(theta) with dE/dtheta from the adjoint pass (computed in the
        forward call when theta requires grad, returned by backward)."""

        @staticmethod
        def forward(ctx, theta, spec):
            th = theta.detach().to("cpu", torch.float64).numpy()
            if theta.requires_grad:
                e, g = spec.value_and_grad(th)
                ctx.save_for_backward(torch.as_tensor(g, dtype=theta.dtype, device=theta.device))
            else:
                e = spec.value(th)
            return torch.tensor(e, dtype=theta.dtype, device=theta.device)

        @staticmethod
        def backward(ctx, grad_out):
            (g,) = ctx.saved_tensors
            return grad_out * g, None

    return _Expectation


class _Lazy:
    """torch is imported on first use, not when propaq_b200 is imported."""

    _fn = None

    def apply(self, *a):
        if _Lazy._fn is None:
            _Lazy._fn = _torch_function()
        return _Lazy._fn.apply(*a)


ExpectationFunction = _Lazy()

__all__ = ["ParametrizedExpectation", "ExpectationFunction", "heisenberg_gates"]
