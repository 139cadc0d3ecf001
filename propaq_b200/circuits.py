"""Circuits as layers of rotations (propaq/circuits/abstract.py,
propaq/circuits/pauli/circuit.py, propaq/circuits/majorana/circuit.py) and the
native gate tables the reference's front-ends dispatch to
(propaq/datatypes/pauli/termsum.py:17-44, propaq/datatypes/majorana/termsum.py:19-67,
propaq/circuits/_gates.py:133-153), without a Qiskit dependency.

A rotation about generator G with angle theta is U = exp(-i theta G / 2).
"""

from __future__ import annotations

import math

from .datatypes import MajoranaMonomial, PauliString


class _Rotation:
    def __init__(self, generator, angle: float, is_intermediate: bool = False, qiskit_gate_idx: int | None = None):
        self.generator = generator
        self.angle = angle
        self.is_intermediate = is_intermediate
        self.qiskit_gate_idx = qiskit_gate_idx

    def __repr__(self):
        return f"{type(self).__name__}({self.generator!r}, {self.angle!r})"


class PauliRotation(_Rotation):
    """exp(-i angle P / 2) for a Pauli string P."""


class MajoranaRotation(_Rotation):
    """exp(-i angle M / 2) for a Majorana monomial M."""


class _Circuit:
    _rotation_cls = _Rotation

    def __init__(self, rotations_or_layers):
        if rotations_or_layers and isinstance(rotations_or_layers[0], list):
            self._layers = rotations_or_layers
        else:
            self._layers = [[r] for r in rotations_or_layers]

    @property
    def layers(self):
        return self._layers

    @property
    def rotations(self):
        return [r for layer in self._layers for r in layer]

    @classmethod
    def from_generators_and_angles(cls, generators, angles):
        return cls([cls._rotation_cls(g, a) for g, a in zip(generators, angles)])

    def inverse(self):
        """Reversed order and negated angles (U dagger), compound gates kept in order
        (propaq/circuits/_utils.py: compound_gate_reversed)."""
        out = type(self).__new__(type(self))
        out.__dict__.update(self.__dict__)
        out._layers = [_compound_reversed(layer) for layer in reversed(self._layers)]
        return out


def _compound_reversed(rotations):
    groups, current = [], []
    for rot in rotations:
        current.append(rot)
        if not rot.is_intermediate:
            groups.append(current)
            current = []
    if current:
        groups.append(current)
    result = []
    for group in reversed(groups):
        rev = list(reversed(group))
        for i, rot in enumerate(rev):
            result.append(type(rot)(rot.generator, -rot.angle, i < len(rev) - 1))
    return result


class PauliCircuit(_Circuit):
    _rotation_cls = PauliRotation


class MajoranaCircuit(_Circuit):
    """Layers of Majorana rotations; `n_modes` as the reference's constructor
    takes it (propaq/circuits/majorana/circuit.py:35-47), optional here."""

    _rotation_cls = MajoranaRotation

    def __init__(self, rotations_or_layers, n_modes: int | None = None):
        super().__init__(rotations_or_layers)
        self.n_modes = n_modes


# ---------------------------------------------------------------- Pauli gates
def pauli_rz(q: int, angle: float, n: int):
    return [PauliRotation(PauliString(0, 1 << q, n), angle)]


def pauli_rx(q: int, angle: float, n: int):
    return [PauliRotation(PauliString(1 << q, 0, n), angle)]


def pauli_ry(q: int, angle: float, n: int):
    return [PauliRotation(PauliString(1 << q, 1 << q, n), angle)]


def pauli_rzz(i: int, j: int, angle: float, n: int):
    return [PauliRotation(PauliString(0, (1 << i) | (1 << j), n), angle)]


def pauli_rxx(i: int, j: int, angle: float, n: int):
    return [PauliRotation(PauliString((1 << i) | (1 << j), 0, n), angle)]


def pauli_cp(i: int, j: int, phi: float, n: int):
    zi, zj = 1 << i, 1 << j
    return [PauliRotation(PauliString(0, zi, n), phi / 2), PauliRotation(PauliString(0, zj, n), phi / 2),
            PauliRotation(PauliString(0, zi | zj, n), -phi / 2)]


def pauli_xx_plus_yy(i: int, j: int, theta: float, n: int):
    b = (1 << i) | (1 << j)
    return [PauliRotation(PauliString(b, 0, n), theta / 2), PauliRotation(PauliString(b, b, n), theta / 2)]


def pauli_cx(c: int, t: int, n: int):
    """CNOT as Z_c(pi/2), X_t(pi/2), Z_c X_t(-pi/2), the decomposition a
    registered custom gate uses (examples/usage/09_custom_gate_registration.ipynb)."""
    return [PauliRotation(PauliString(0, 1 << c, n), math.pi / 2),
            PauliRotation(PauliString(1 << t, 0, n), math.pi / 2),
            PauliRotation(PauliString(1 << t, 1 << c, n), -math.pi / 2)]


# ------------------------------------------------------------- Majorana gates
def majorana_rz(q: int, raw_angle: float, n_modes: int):
    m = MajoranaMonomial((1 << (2 * q)) | (1 << (2 * q + 1)), n_modes, is_number_preserving=True)
    return [MajoranaRotation(m, -raw_angle)]


def majorana_cp(i: int, j: int, phi: float, n_modes: int):
    mi = (1 << (2 * i)) | (1 << (2 * i + 1))
    mj = (1 << (2 * j)) | (1 << (2 * j + 1))
    return [MajoranaRotation(MajoranaMonomial(mi, n_modes), -phi / 2),
            MajoranaRotation(MajoranaMonomial(mj, n_modes), -phi / 2),
            MajoranaRotation(MajoranaMonomial(mi | mj, n_modes), phi / 2)]


def majorana_xx_plus_yy(i: int, j: int, theta: float, n_modes: int):
    lo, hi = min(i, j), max(i, j)
    d = hi - lo
    factor = theta / 2.0
    jw = 0
    for k in range(lo + 1, hi):
        jw |= (1 << (2 * k)) | (1 << (2 * k + 1))
    sign = 1 if ((d - 1) // 2) % 2 == 0 else -1
    if i > j:
        m1 = (1 << (2 * hi)) | jw | (1 << (2 * lo + 1))
        m2 = (1 << (2 * hi + 1)) | jw | (1 << (2 * lo))
        s1, s2 = -sign * factor, sign * factor
    else:
        m1 = (1 << (2 * lo)) | jw | (1 << (2 * hi + 1))
        m2 = (1 << (2 * lo + 1)) | jw | (1 << (2 * hi))
        s1, s2 = sign * factor, -sign * factor
    return [MajoranaRotation(MajoranaMonomial(m1, n_modes, is_number_preserving=False), s1),
            MajoranaRotation(MajoranaMonomial(m2, n_modes, is_number_preserving=False), s2)]
