"""The Majorana (and Pauli) algebra of the engine and of the oracle, pinned to
the reference's own known answers and to an independent Jordan-Wigner
construction.

Two implementations are checked side by side on every case:
  * the oracle's algebra probes (oracle/pq_oracle.cpp, through pqo_*), and
  * the engine's device algebra itself -- PauliOps / MajoranaOps / make_gen_info
    of propaq_b200/csrc/pq_device.cuh -- compiled for the host with g++
    (tests/device_algebra_host.cpp).

Known answers restated from crates/majorana/tests/unit/monomial.rs:
hermiticity_exp for every residue (:32-45), resorting_parity (:49-74), the JW
weights including the 33-weight two-word monomial (:77-105), the trace against
every occupation of one and two sites (:108-137), the matmul identities and the
disjoint-product phase (:155-193) and the commutation cases (:195-222).  The
exhaustive checks follow weight_matches_reference_exhaustive_small (:246) with
the weight taken from an explicit Jordan-Wigner product of Pauli matrices
instead of the reference's compute_weight_for."""

from __future__ import annotations

import ctypes
import itertools
import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

HERE = Path(__file__).resolve().parent
U64P = ctypes.POINTER(ctypes.c_uint64)


@pytest.fixture(scope="module")
def dev(tmp_path_factory):
    """The device algebra built for the host."""
    if shutil.which("g++") is None:
        pytest.skip("no g++")
    so = tmp_path_factory.mktemp("devalg") / "libdevalg.so"
    subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-o", str(so),
                    str(HERE / "device_algebra_host.cpp")], check=True)
    lib = ctypes.CDLL(str(so))
    V = ctypes.c_void_p
    lib.da_anticommutes.argtypes = [ctypes.c_uint32, ctypes.c_uint32, V, V]
    lib.da_product.argtypes = [ctypes.c_uint32, ctypes.c_uint32, V, V, V]
    lib.da_weight.restype = ctypes.c_uint32
    lib.da_weight.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, V]
    lib.da_trace.restype = ctypes.c_double
    lib.da_trace.argtypes = [ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, V, V, ctypes.c_uint32]
    return lib


def words(x: int, n_words: int) -> np.ndarray:
    return np.array([(x >> (64 * i)) & ((1 << 64) - 1) for i in range(n_words)], dtype=np.uint64)


def n_words_for_modes(n_modes: int) -> int:
    w = 1
    while 64 * w < n_modes:
        w *= 2
    return w


class Impl:
    """One implementation of the algebra on integer keys."""

    def __init__(self, name, anti, prod, weight, trace):
        self.name, self.anti, self.prod, self.weight, self.trace = name, anti, prod, weight, trace


def oracle_impl(oracle) -> Impl:
    return Impl(
        "oracle",
        lambda alg, nw, g, k: oracle.anticommutes(alg, words(g, nw), words(k, nw)),
        lambda alg, nw, g, k: oracle.product(alg, words(g, nw), words(k, nw))[1],
        lambda alg, nu, nw, k: oracle.weight(alg, nu, words(k, nw)),
        lambda alg, nu, nw, k, s: oracle.trace(alg, nu, words(k, nw), words(s, max(1, (nu + 63) // 64))),
    )


def device_impl(lib) -> Impl:
    def anti(alg, nw, g, k):
        gw, kw = words(g, nw), words(k, nw)
        return bool(lib.da_anticommutes(alg, nw, gw.ctypes.data, kw.ctypes.data))

    def prod(alg, nw, g, k):
        gw, kw, out = words(g, nw), words(k, nw), np.zeros(nw, np.uint64)
        p = lib.da_product(alg, nw, gw.ctypes.data, kw.ctypes.data, out.ctypes.data)
        assert int(sum(int(v) << (64 * i) for i, v in enumerate(out))) == g ^ k
        return p

    def weight(alg, nu, nw, k):
        kw = words(k, nw)
        return int(lib.da_weight(alg, nu, nw, kw.ctypes.data))

    def trace(alg, nu, nw, k, s):
        kw, sw = words(k, nw), words(s, max(1, (nu + 63) // 64))
        return float(lib.da_trace(alg, nu, nw, kw.ctypes.data, sw.ctypes.data, len(sw)))

    return Impl("device", anti, prod, weight, trace)


@pytest.fixture(scope="module", params=["oracle", "device"])
def impl(request, oracle, dev):
    return oracle_impl(oracle) if request.param == "oracle" else device_impl(dev)


# ------------------------------------------------ the reference's definitions
HERMITICITY_EXP = {0: 0, 1: 0, 2: 1, 3: 1, 4: 0, 5: 0, 6: 1, 7: 1, 8: 0}  # monomial.rs:32-45


def hermiticity_exp(length: int) -> int:
    return HERMITICITY_EXP[length % 8]


def resorting_parity(a: int, b: int) -> bool:
    """Parity of the pairs (i in a, j in b) with i > j: the transpositions that
    sort the concatenation a.b (monomial.rs:637-647)."""
    count = 0
    for j in range(b.bit_length()):
        if b >> j & 1:
            count += bin(a >> (j + 1)).count("1")
    return bool(count & 1)


def product_exp(a: int, b: int) -> int:
    """Phase exponent of a @ b (monomial.rs:185-189)."""
    la, lb, lc = bin(a).count("1"), bin(b).count("1"), bin(a ^ b).count("1")
    return (hermiticity_exp(la) + hermiticity_exp(lb) - hermiticity_exp(lc) + 2 * resorting_parity(a, b)) % 4


def commutes(a: int, b: int) -> bool:
    """monomial.rs:40-51."""
    if a == b:
        return True
    return (bin(a).count("1") * bin(b).count("1") + bin(a & b).count("1")) % 2 == 0


I2 = np.eye(2, dtype=complex)
PX = np.array([[0, 1], [1, 0]], complex)
PY = np.array([[0, -1j], [1j, 0]])
PZ = np.array([[1, 0], [0, -1]], complex)


def jw_pauli(modes: int, n_sites: int):
    """The Jordan-Wigner Pauli string of i^herm(l) gamma_m1 ... gamma_ml (modes
    ascending): gamma_2k = Z_0..Z_k-1 X_k, gamma_2k+1 = Z_0..Z_k-1 Y_k.
    Returns (phase, [pauli index per site: 0 I, 1 X, 2 Y, 3 Z])."""
    # single-site Pauli algebra as (phase, label) products
    mul = {}
    mats = {0: I2, 1: PX, 2: PY, 3: PZ}
    for a, b in itertools.product(range(4), repeat=2):
        m = mats[a] @ mats[b]
        for c in range(4):
            for ph in (1, -1, 1j, -1j):
                if np.allclose(m, ph * mats[c]):
                    mul[a, b] = (ph, c)
    phase, string = 1.0 + 0j, [0] * n_sites
    for m in range(2 * n_sites):
        if not modes >> m & 1:
            continue
        k = m // 2
        gam = [3] * k + [1 if m % 2 == 0 else 2] + [0] * (n_sites - k - 1)
        for s in range(n_sites):
            ph, string[s] = mul[string[s], gam[s]]
            phase *= ph
    phase *= 1j ** hermiticity_exp(bin(modes).count("1"))
    return phase, string


def jw_matrix(modes: int, n_sites: int) -> np.ndarray:
    phase, string = jw_pauli(modes, n_sites)
    mats = {0: I2, 1: PX, 2: PY, 3: PZ}
    m = np.array([[1.0 + 0j]])
    for s in reversed(range(n_sites)):
        m = np.kron(m, mats[string[s]])
    return phase * m


# ------------------------------------------------------------ known answers
def test_hermiticity_exp_all_residues(impl):
    # monomial.rs:32-45, through the only place the engine uses it: M @ M = +1
    # for a Hermitian monomial, whose phase is 2 herm(l) + 2 * (l choose 2).
    for length in range(0, 9):
        m = (1 << length) - 1
        assert impl.prod(1, 1, m, m) == 0, f"M @ M for a monomial of length {length}"
        assert (2 * hermiticity_exp(length) + length * (length - 1)) % 4 == 0


@pytest.mark.parametrize("a,b,want", [(0b0011, 0b1100, False), (0b0010, 0b0001, True), (0b1100, 0b0011, False),
                                      (0xFF, 0, False)])
def test_resorting_parity_known_answers(impl, a, b, want):
    # monomial.rs:49-74 through the product phase, which is herm terms plus
    # twice the resorting parity.
    assert resorting_parity(a, b) == want
    la, lb, lc = bin(a).count("1"), bin(b).count("1"), bin(a ^ b).count("1")
    base = (hermiticity_exp(la) + hermiticity_exp(lb) - hermiticity_exp(lc)) % 4
    assert impl.prod(1, 1, a, b) == (base + 2 * want) % 4


@pytest.mark.parametrize("modes,n_modes,want", [
    (0, 8, 0), (0b01, 8, 1), (0b11, 8, 1), (0b0101_0101, 8, 4), (0b01, 128, 1), (1 << 64, 128, 33)])
def test_weight_known_answers(impl, modes, n_modes, want):
    # monomial.rs:77-105; the last is mon_bits(vec![0, 1], 128): mode 64 alone
    assert impl.weight(1, n_modes // 2, n_words_for_modes(n_modes), modes) == want


@pytest.mark.parametrize("modes,state,want", [
    (0, 0, 1.0), (0, 0b1111, 1.0), (0b01, 0, 0.0), (0b01, 1, 0.0), (0b11, 0, -1.0), (0b11, 1, 1.0),
    (0b1111, 0b00, -1.0), (0b1111, 0b01, 1.0), (0b1111, 0b10, 1.0), (0b1111, 0b11, -1.0)])
def test_trace_known_answers(impl, modes, state, want):
    # monomial.rs:108-137 (8 modes = 4 sites)
    assert impl.trace(1, 4, 1, modes, state) == want


def test_matmul_known_answers(impl):
    # monomial.rs:155-193: identity on either side and M @ M have phase 1;
    # (g0 g1) @ (g2 g3) has phase -1.
    assert impl.prod(1, 1, 0, 0b0011) == 0
    assert impl.prod(1, 1, 0b0011, 0) == 0
    assert impl.prod(1, 1, 0b0111, 0b0111) == 0
    assert impl.prod(1, 1, 0b0011, 0b1100) == 2


@pytest.mark.parametrize("a,b,comm", [(0b0011, 0b0011, True), (0b0011, 0b1100, True), (0b0011, 0b0110, False),
                                      (0b0001, 0b0010, False)])
def test_commutation_known_answers(impl, a, b, comm):
    # monomial.rs:195-222
    assert impl.anti(1, 1, a, b) == (not comm)
    assert commutes(a, b) == comm


# ------------------------------------------------------- exhaustive checks
def test_jw_construction_reproduces_the_known_answers():
    """The independent construction agrees with the reference's own table."""
    for modes, n_modes, want in [(0, 8, 0), (0b01, 8, 1), (0b11, 8, 1), (0b0101_0101, 8, 4)]:
        assert sum(1 for s in jw_pauli(modes, n_modes // 2)[1] if s) == want
    # Hermitian: i^herm(l) gamma... squares to the identity
    for modes in range(1, 1 << 6):
        m = jw_matrix(modes, 3)
        assert np.allclose(m @ m, np.eye(8)) and np.allclose(m, m.conj().T)


@pytest.mark.parametrize("n_sites", [1, 2, 3, 4])
def test_majorana_algebra_exhaustive_against_jordan_wigner(impl, n_sites):
    """Every monomial pair on up to 4 sites (a stride of partners on 4): the
    weight against the JW string, anticommutation and the product phase against
    the JW matrices, and the trace of every monomial in every basis state."""
    n_modes = 2 * n_sites
    space = 1 << n_modes
    mats = {m: jw_matrix(m, n_sites) for m in range(space)}
    for a in range(space):
        assert impl.weight(1, n_sites, 1, a) == sum(1 for s in jw_pauli(a, n_sites)[1] if s), a
    stride = 1 if n_sites <= 3 else 7
    for a in range(space):
        for b in range(0, space, stride):
            ma, mb = mats[a], mats[b]
            anti = np.allclose(ma @ mb, -(mb @ ma))
            assert impl.anti(1, 1, a, b) == anti, (a, b)
            p = impl.prod(1, 1, a, b)
            assert p == product_exp(a, b), (a, b)
            assert np.allclose(ma @ mb, (1j ** p) * mats[a ^ b]), (a, b)
    for m in range(space):
        for s in range(1 << n_sites):
            psi = np.zeros(1 << n_sites)
            psi[s] = 1.0
            want = float(np.real(psi @ mats[m] @ psi))
            assert impl.trace(1, n_sites, 1, m, s) == want, (m, s)


def test_majorana_weight_multiword_random(impl, oracle, dev):
    """weight_matches_reference_randomized_multiword (monomial.rs:258-270): random
    monomials on registers across word boundaries, against the JW count."""
    rng = np.random.default_rng(7)
    for n_sites in (30, 31, 32, 33, 63, 64, 65, 100, 127, 128):
        n_modes = 2 * n_sites
        nw = n_words_for_modes(n_modes)
        for _ in range(20):
            m = int(rng.integers(0, 1 << 62)) | (int(rng.integers(0, 1 << 62)) << 62)
            m |= int(rng.integers(0, 1 << 62)) << 124 | int(rng.integers(0, 1 << 62)) << 186
            m &= (1 << n_modes) - 1
            want = sum(1 for s in jw_pauli(m, n_sites)[1] if s)
            assert impl.weight(1, n_sites, nw, m) == want


def test_majorana_product_multiword_random(impl):
    """The product phase across word boundaries against the reference's formula."""
    rng = np.random.default_rng(11)
    for n_modes in (64, 128, 256, 512):
        nw = n_words_for_modes(n_modes)
        for _ in range(150):
            a = int.from_bytes(rng.bytes(n_modes // 8), "little")
            b = int.from_bytes(rng.bytes(n_modes // 8), "little")
            if rng.random() < 0.3:  # sparse cases cross the words with few modes
                a &= int.from_bytes(rng.bytes(n_modes // 8), "little") & int.from_bytes(rng.bytes(n_modes // 8),
                                                                                      "little")
            assert impl.prod(1, nw, a, b) == product_exp(a, b), (n_modes, a, b)
            assert impl.anti(1, nw, a, b) == (not commutes(a, b))


def test_pauli_algebra_exhaustive_against_matrices(impl):
    """Pauli keys on 3 qubits: anticommutation, the product phase, the weight
    and the trace against explicit Pauli matrices (crates/pauli/src/algebra.rs)."""
    n = 3
    mats = {0: I2, 1: PX, 2: PZ, 3: PY}  # (x | z << 1)

    def mat(key):
        m = np.array([[1.0 + 0j]])
        for q in reversed(range(n)):
            m = np.kron(m, mats[(key >> (2 * q)) & 3])
        return m

    space = 1 << (2 * n)
    M = {k: mat(k) for k in range(space)}
    for g in range(space):
        for k in range(space):
            assert impl.anti(0, 1, g, k) == np.allclose(M[g] @ M[k], -(M[k] @ M[g]))
            p = impl.prod(0, 1, g, k)
            assert np.allclose(M[g] @ M[k], (1j ** p) * M[g ^ k]), (g, k)
        assert impl.weight(0, n, 1, g) == sum(1 for q in range(n) if (g >> (2 * q)) & 3)
        for s in range(1 << n):
            psi = np.zeros(1 << n)
            psi[s] = 1.0
            assert impl.trace(0, n, 1, g, s) == float(np.real(psi @ M[g] @ psi))
