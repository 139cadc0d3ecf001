"""The reference's gzip term file (crates/core/src/interface/term_io.rs:15-89).

All integers little-endian:
    u64 n_terms
    u64 key_stride   (bytes per key; 0 when n_terms == 0)
    u64 system_size  (n_qubits for Pauli, n_modes for Majorana)
    per term: key_stride key bytes, then the f64 coefficient.
Pauli keys are the x bytes then the z bytes, ceil(n_qubits / 8) each; Majorana
keys are the mode bytes, ceil(n_modes / 8).
"""

from __future__ import annotations

import gzip
import struct

import numpy as np

_EVEN = np.uint64(0x5555555555555555)
_MASKS = [np.uint64(m) for m in (0x3333333333333333, 0x0F0F0F0F0F0F0F0F, 0x00FF00FF00FF00FF,
                                 0x0000FFFF0000FFFF, 0x00000000FFFFFFFF)]


def _gather_even(w: np.ndarray) -> np.ndarray:
    """Bits 0,2,4,... of each u64 packed into the low 32 bits."""
    x = w & _EVEN
    for sh, m in zip((1, 2, 4, 8, 16), _MASKS):
        x = (x | (x >> np.uint64(sh))) & m
    return x


def pauli_planes(keys: np.ndarray, n_qubits: int):
    """Interleaved keys [n, W] -> (x, z) little-endian byte planes [n, ceil(n/8)]."""
    n, nw = keys.shape
    x = np.zeros((n, nw), dtype=np.uint64)
    z = np.zeros((n, nw), dtype=np.uint64)
    for i in range(nw):
        xi = _gather_even(keys[:, i])
        zi = _gather_even(keys[:, i] >> np.uint64(1))
        x[:, i // 2] |= xi << np.uint64(32 * (i % 2))
        z[:, i // 2] |= zi << np.uint64(32 * (i % 2))
    nb = (n_qubits + 7) // 8
    xb = x.view(np.uint8).reshape(n, -1)[:, :nb]
    zb = z.view(np.uint8).reshape(n, -1)[:, :nb]
    return xb, zb


def save_terms(path: str, keys: np.ndarray, coeffs: np.ndarray, basis: int, system_size: int) -> None:
    """Writes engine output (interleaved keys) in the reference's format."""
    keys = np.ascontiguousarray(keys, dtype=np.uint64)
    n = len(coeffs)
    if basis == 0:
        xb, zb = pauli_planes(keys, system_size)
        kb = np.concatenate([xb, zb], axis=1)
    else:
        nb = (system_size + 7) // 8
        kb = keys.view(np.uint8).reshape(n, -1)[:, :nb] if n else np.zeros((0, nb), np.uint8)
    stride = kb.shape[1] if n else 0
    rec = np.zeros(n, dtype=[("k", np.uint8, (stride,)), ("c", "<f8")]) if n else None
    with gzip.open(path, "wb") as f:
        f.write(struct.pack("<QQQ", n, stride, system_size if n else 0))
        if n:
            rec["k"] = kb
            rec["c"] = coeffs
            f.write(rec.tobytes())


def save_term_sum(path: str, ts) -> None:
    items = ts.items()
    with gzip.open(path, "wb") as f:
        if not items:
            f.write(struct.pack("<QQQ", 0, 0, 0))
            return
        first = items[0][0]
        kb = first.to_bytes()
        size = first.n_qubits if hasattr(first, "n_qubits") else first.n_modes
        f.write(struct.pack("<QQQ", len(items), len(kb), size))
        for t, c in items:
            f.write(t.to_bytes())
            f.write(struct.pack("<d", c))


def load_term_sum(path: str, cls):
    from .datatypes import MajoranaMonomial, PauliString

    out = cls()
    with gzip.open(path, "rb") as f:
        n, stride, size = struct.unpack("<QQQ", f.read(24))
        for _ in range(n):
            kb = f.read(stride)
            (c,) = struct.unpack("<d", f.read(8))
            if cls.__name__.startswith("Pauli"):
                nb = (size + 7) // 8
                t = PauliString(int.from_bytes(kb[:nb], "little"), int.from_bytes(kb[nb:2 * nb], "little"), size)
            else:
                modes = int.from_bytes(kb, "little")
                single = 0
                for k in range(size // 2):
                    single |= (modes >> (2 * k) & 1) ^ (modes >> (2 * k + 1) & 1)
                t = MajoranaMonomial(modes, size, is_number_preserving=single == 0)
            out._terms[t] = c
    return out
