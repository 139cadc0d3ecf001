"""Term types of the propagation API: PauliString / PauliTermSum and
MajoranaMonomial / MajoranaTermSum.

They mirror the reference's pyo3 classes (propaq/_rust_core/__init__.pyi:129-222,
:330-418, :561-641, :723-809).  A term's engine key is W u64 words with two
bits per unit, interleaved: Pauli qubit q uses bit 2q for x and bit 2q+1 for z
(crates/pauli/src/algebra.rs:242-257); a Majorana monomial uses bit m for mode
m (crates/majorana/src/algebra.rs:218-233).
"""

from __future__ import annotations

import numpy as np

_SPREAD8 = [0] * 256
for _b in range(256):
    _v = 0
    for _i in range(8):
        if _b >> _i & 1:
            _v |= 1 << (2 * _i)
    _SPREAD8[_b] = _v


def _spread(x: int) -> int:
    """Moves bit i of x to bit 2i."""
    out, shift = 0, 0
    while x:
        out |= _SPREAD8[x & 0xFF] << shift
        x >>= 8
        shift += 16
    return out


def _compact(k: int) -> int:
    """Inverse of _spread over the even bits of k."""
    out, i = 0, 0
    while k:
        if k & 1:
            out |= 1 << i
        k >>= 2
        i += 1
    return out


def int_to_words(value: int, n_words: int) -> np.ndarray:
    mask = (1 << 64) - 1
    return np.array([(value >> (64 * i)) & mask for i in range(n_words)], dtype=np.uint64)


def words_to_int(words) -> int:
    v = 0
    for i, w in enumerate(words):
        v |= int(w) << (64 * i)
    return v


_EVEN = int("55" * 256, 16)


def _popcount(x: int) -> int:
    return bin(x).count("1")


class PauliString:
    """A Pauli string on n_qubits qubits, as x and z bitmasks (bit q = qubit q)."""

    __slots__ = ("_x", "_z", "_n", "_key", "_kb")

    def __init__(self, x, z, n_qubits: int):
        self._x = int(x)
        self._z = int(z)
        self._n = int(n_qubits)
        if self._x >> self._n or self._z >> self._n:
            raise ValueError("PauliString bitmask has bits beyond n_qubits")
        self._key = None
        self._kb = None

    @property
    def n_qubits(self) -> int:
        return self._n

    @property
    def x(self) -> int:
        return self._x

    @property
    def z(self) -> int:
        return self._z

    @property
    def weight(self) -> int:
        return _popcount(self._x | self._z)

    def key(self) -> int:
        """Interleaved basis-string key (bit 2q = x_q, bit 2q+1 = z_q)."""
        if self._key is None:
            self._key = _spread(self._x) | (_spread(self._z) << 1)
        return self._key

    def key_bytes(self, n_words: int) -> bytes:
        """The key as n_words little-endian u64 words (kept: a circuit's
        generators are converted once, however many propagations use them)."""
        kb = self._kb
        if kb is None or len(kb) != 8 * n_words:
            kb = self._kb = self.key().to_bytes(8 * n_words, "little")
        return kb

    @classmethod
    def from_key(cls, key: int, n_qubits: int) -> "PauliString":
        p = cls(_compact(key & _EVEN_MASK(n_qubits)), _compact((key >> 1) & _EVEN_MASK(n_qubits)), n_qubits)
        return p

    def commutes_with(self, other: "PauliString") -> bool:
        return (_popcount(self._x & other._z) + _popcount(self._z & other._x)) % 2 == 0

    def __matmul__(self, other: "PauliString"):
        """self * other = phase * product (crates/pauli/src/algebra.rs:206-213)."""
        g, k = self.key(), other.key()
        out = g ^ k

        def ys(m):
            return _popcount(m & (m >> 1) & _EVEN)

        p = (ys(g) + ys(k) - ys(out) + 2 * _popcount((g >> 1) & k & _EVEN)) % 4
        phase = (1, 1j, -1, -1j)[p]
        n = max(self._n, other._n)
        return complex(phase), PauliString.from_key(out, n)

    def trace_with_diag_state(self, diag_state) -> float:
        """<s|P|s> for a computational-basis state (crates/pauli/src/algebra.rs:220-239)."""
        if self._x:
            return 0.0
        return -1.0 if _popcount(self._z & int(diag_state)) % 2 else 1.0

    def to_bytes(self) -> bytes:
        """x bytes then z bytes, ceil(n_qubits / 8) each (crates/pauli/src/string.rs:228-236)."""
        nb = (self._n + 7) // 8
        return self._x.to_bytes(nb, "little") + self._z.to_bytes(nb, "little")

    def __hash__(self) -> int:
        return hash((self._x, self._z, self._n))

    def __eq__(self, other) -> bool:
        return isinstance(other, PauliString) and (self._x, self._z, self._n) == (other._x, other._z, other._n)

    def __repr__(self) -> str:
        chars = []
        for q in range(self._n):
            xb, zb = self._x >> q & 1, self._z >> q & 1
            chars.append("IXZY"[xb | (zb << 1)])
        return f"PauliString({''.join(chars)})"


def _EVEN_MASK(n_units: int) -> int:
    return _EVEN & ((1 << (2 * n_units)) - 1)


class MajoranaMonomial:
    """A product of Majorana operators as a mode bitmask (bit 2k = gamma_2k, bit 2k+1 = gamma_2k+1)."""

    __slots__ = ("_modes", "_n", "_np")

    def __init__(self, modes, n_modes: int, is_number_preserving: bool = True):
        self._modes = int(modes)
        self._n = int(n_modes)
        self._np = bool(is_number_preserving)
        if self._modes >> self._n:
            raise ValueError("MajoranaMonomial bitmask has bits beyond n_modes")

    @property
    def n_modes(self) -> int:
        return self._n

    @property
    def modes(self) -> int:
        return self._modes

    @property
    def is_number_preserving(self) -> bool:
        return self._np

    @property
    def length(self) -> int:
        return _popcount(self._modes)

    @property
    def weight(self) -> int:
        """Pauli weight under Jordan-Wigner (crates/majorana/src/algebra.rs:85-123)."""
        return jw_weight(self._modes, self._n // 2)

    def key(self) -> int:
        return self._modes

    @classmethod
    def from_key(cls, key: int, n_modes: int) -> "MajoranaMonomial":
        m = key & ((1 << n_modes) - 1)
        single = (m ^ (m >> 1)) & _EVEN
        return cls(m, n_modes, is_number_preserving=single == 0)

    def overlap(self, other: "MajoranaMonomial") -> int:
        return _popcount(self._modes & other._modes)

    def commutes_with(self, other: "MajoranaMonomial") -> bool:
        return (self.length * other.length + self.overlap(other)) % 2 == 0

    def resulting_weight(self, other: "MajoranaMonomial") -> int:
        """Jordan-Wigner weight of the product self @ other (its modes are the XOR)."""
        return jw_weight(self._modes ^ other._modes, self._n // 2)

    def __matmul__(self, other: "MajoranaMonomial"):
        g, k = self._modes, other._modes
        out = g ^ k

        def herm(n):
            return 0 if n % 4 in (0, 1) else 1

        # parity of the transpositions carrying k's modes past g's
        swaps = 0
        for y in range(k.bit_length()):
            if k >> y & 1:
                swaps += _popcount(g >> (y + 1))
        p = (herm(_popcount(g)) + herm(_popcount(k)) - herm(_popcount(out)) + 2 * (swaps & 1)) % 4
        phase = (1, 1j, -1, -1j)[p]
        return complex(phase), MajoranaMonomial.from_key(out, max(self._n, other._n))

    def trace_with_diag_state(self, diag_state) -> float:
        state = int(diag_state)
        paired, product = 0, 1
        for k in range(self._n // 2):
            lo, hi = self._modes >> (2 * k) & 1, self._modes >> (2 * k + 1) & 1
            if lo != hi:
                return 0.0
            if lo:
                product *= 2 * (state >> k & 1) - 1
                paired += 1
        return float((1 if (paired // 2) % 2 == 0 else -1) * product)

    def to_bytes(self) -> bytes:
        """ceil(n_modes / 8) little-endian bytes (crates/majorana/src/monomial.rs:337-342)."""
        return self._modes.to_bytes((self._n + 7) // 8, "little")

    def __hash__(self) -> int:
        return hash((self._modes, self._n))

    def __eq__(self, other) -> bool:
        return isinstance(other, MajoranaMonomial) and (self._modes, self._n) == (other._modes, other._n)

    def __repr__(self) -> str:
        modes = [m for m in range(self._n) if self._modes >> m & 1]
        return f"MajoranaMonomial({modes}, n_modes={self._n})"


def jw_weight(modes: int, n_sites: int) -> int:
    """Jordan-Wigner weight of a Majorana monomial over n_sites sites."""
    weight, parity = 0, 0
    singles = 0
    for k in range(n_sites):
        if (modes >> (2 * k) & 1) != (modes >> (2 * k + 1) & 1):
            singles += 1
    odd = singles & 1
    for k in range(n_sites):
        lo, hi = modes >> (2 * k) & 1, modes >> (2 * k + 1) & 1
        single = lo ^ hi
        parity ^= single
        string = parity ^ odd
        occupied = lo | hi
        weight += 1 if (single or (occupied ^ string)) else 0
    return weight


class _TermSum:
    """Shared dict-backed term container (host side)."""

    _term_cls: type = object

    def __init__(self, terms: dict | None = None, dtype: str | None = None):
        if dtype not in (None, "f64", "float64", "f32", "float32"):
            raise ValueError(f"unknown dtype {dtype!r}")
        self._dtype = "f32" if dtype in ("f32", "float32") else "f64"
        self._terms: dict = {}
        if terms:
            for t, c in terms.items():
                self.add(t, c)

    @property
    def dtype(self) -> str:
        return self._dtype

    def _check(self, term):
        if not isinstance(term, self._term_cls):
            raise TypeError(f"expected {self._term_cls.__name__}, got {type(term).__name__}")

    def add(self, term, coeff: float) -> None:
        self._check(term)
        self._terms[term] = self._terms.get(term, 0.0) + float(coeff)

    def scale(self, factor: float) -> None:
        for t in self._terms:
            self._terms[t] *= factor

    def merge(self, other) -> None:
        for t, c in other.items():
            self.add(t, c)

    def norm_squared(self) -> float:
        return float(sum(c * c for c in self._terms.values()))

    def items(self):
        return list(self._terms.items())

    def __len__(self) -> int:
        return len(self._terms)

    def __setitem__(self, term, coeff: float) -> None:
        self._check(term)
        self._terms[term] = float(coeff)

    def __getitem__(self, term) -> float:
        return self._terms[term]

    def __contains__(self, term) -> bool:
        return term in self._terms

    def copy(self):
        out = type(self)(dtype=self._dtype)
        out._terms = dict(self._terms)
        return out

    def truncate(self, policy) -> None:
        """Drops terms a truncation policy rejects (weight > cut or |c| < cut)."""
        from .truncation import resolve_config, resolve_truncation

        cfg = resolve_config(resolve_truncation(policy))
        keep = {}
        for t, c in self._terms.items():
            if cfg.weight is not None and t.weight > cfg.weight:
                continue
            if cfg.coefficient is not None and abs(c) < cfg.coefficient:
                continue
            keep[t] = c
        self._terms = keep

    def apply_damping(self, noise, active_modes: int) -> None:
        """Multiplies each coefficient by noise.damping_factor(weight, active_modes)."""
        for t in self._terms:
            self._terms[t] *= float(noise.damping_factor(t.weight, active_modes))

    def save(self, path: str) -> None:
        """Writes the gzip term file of crates/core/src/interface/term_io.rs:24-56."""
        from .term_io import save_term_sum

        save_term_sum(path, self)

    @classmethod
    def from_file(cls, path: str):
        from .term_io import load_term_sum

        return load_term_sum(path, cls)

    @property
    def sparse_key_bytes(self) -> int:
        return sum(len(t.to_bytes()) for t in self._terms)

    def n_units(self) -> int:
        raise NotImplementedError

    def to_arrays(self, n_words: int):
        """(keys [n, n_words] u64, coeffs [n] f64) in insertion order."""
        nb = 8 * n_words
        buf = b"".join(t.key().to_bytes(nb, "little") for t in self._terms)
        keys = np.frombuffer(buf, dtype="<u8").reshape(len(self._terms), n_words).astype(np.uint64)
        coeffs = np.fromiter(self._terms.values(), dtype=np.float64, count=len(self._terms))
        return keys, coeffs


class PauliTermSum(_TermSum):
    """A sum of Pauli strings with FP64 coefficients."""

    _term_cls = PauliString

    def n_units(self) -> int:
        return max((t.n_qubits for t in self._terms), default=0)

    @classmethod
    def from_arrays(cls, keys: np.ndarray, coeffs: np.ndarray, n_qubits: int) -> "PauliTermSum":
        out = cls()
        for row, c in zip(keys, coeffs):
            out._terms[PauliString.from_key(words_to_int(row), n_qubits)] = float(c)
        return out


class MajoranaTermSum(_TermSum):
    """A sum of Majorana monomials with FP64 coefficients."""

    _term_cls = MajoranaMonomial

    def n_units(self) -> int:
        """Mode count (the propagator uses n_modes / 2 sites)."""
        return max((t.n_modes for t in self._terms), default=0)

    @classmethod
    def from_arrays(cls, keys: np.ndarray, coeffs: np.ndarray, n_modes: int) -> "MajoranaTermSum":
        out = cls()
        for row, c in zip(keys, coeffs):
            out._terms[MajoranaMonomial.from_key(words_to_int(row), n_modes)] = float(c)
        return out
