"""Forward-mode reference for the adjoint gradient (test infrastructure).

A plain-Python propagation that carries, next to every coefficient, its
derivative with respect to every gate angle, with each truncation decision
(held / dropped / emitted branch, reclaim) taken from the coefficient values
exactly as the engine takes them.  Its derivatives are therefore those of the
function the engine evaluates, with the decisions held fixed -- what
pq_run_adjoint computes in reverse mode.  The single-key algebra (anticommutation,
product phase, weight, trace) comes from the C oracle.

Scope: small cases (tangents are dense vectors over the gates) and circuits
without Clifford rotations (no frame deferral).
"""

from __future__ import annotations

import math

import numpy as np

EPS_CLASSIFY = 1e-9
HELD, DROP, EMIT = 0, 1, 2


def _neg_im(p: int) -> float:
    return -1.0 if p == 1 else (1.0 if p == 3 else 0.0)


def propagate_with_tangents(oracle, p):
    """(E, dE/d angle per gate) for a harness Problem."""
    basis, n_units, W = p.basis, p.n_units, p.n_words
    G = len(p.angles)
    key = lambda a: tuple(int(x) for x in a)  # noqa: E731
    has_w, has_c = p.max_weight is not None, p.min_coeff is not None
    weight = lambda k: oracle.weight(basis, n_units, np.array(k, dtype=np.uint64))  # noqa: E731

    rows_k, rows_c, rows_t, pos = [], [], [], {}
    for k_arr, c in zip(p.obs_keys.reshape(-1, W), p.obs_coeffs):
        k = key(k_arr)
        if has_w and weight(k) > p.max_weight:
            continue
        if has_c and not abs(c) >= p.min_coeff:
            continue
        if k in pos:
            rows_c[pos[k]] += c
        else:
            pos[k] = len(rows_k)
            rows_k.append(k)
            rows_c.append(float(c))
            rows_t.append(np.zeros(G))

    def factors(layer):
        if p.noise_table is not None:
            return p.noise_table
        if p.noise_tables_layered is not None:
            return p.noise_tables_layered[layer]
        return None

    for layer in range(len(p.offsets) - 1):
        f = factors(layer)
        if f is not None:
            last = len(f) - 1
            nk, nc, nt = [], [], []
            for k, c, t in zip(rows_k, rows_c, rows_t):
                w = weight(k)
                fw = float(f[min(w, last)])
                c2, t2 = c * fw, t * fw
                if has_w or has_c:
                    keep = (not has_w or w <= p.max_weight) and (not has_c or abs(c2) >= p.min_coeff)
                    if not keep:
                        continue
                nk.append(k)
                nc.append(c2)
                nt.append(t2)
            rows_k, rows_c, rows_t = nk, nc, nt
        for g in range(int(p.offsets[layer]), int(p.offsets[layer + 1])):
            gen = np.array(p.gate_keys.reshape(-1, W)[g], dtype=np.uint64)
            ang = float(p.angles[g])
            sn, cs = math.sin(ang), math.cos(ang)
            if abs(cs) < EPS_CLASSIFY:
                raise NotImplementedError("the forward-mode reference takes no Clifford rotations")
            e_g = np.zeros(G)
            e_g[g] = 1.0
            N = len(rows_k)
            anti = [oracle.anticommutes(basis, gen, np.array(k, dtype=np.uint64)) for k in rows_k]
            if abs(sn) < EPS_CLASSIFY:
                for r in range(N):
                    if anti[r]:
                        rows_t[r] = rows_t[r] * cs - rows_c[r] * sn * e_g
                        rows_c[r] = rows_c[r] * cs
                continue
            lossless = p.min_terms is not None and N < p.min_terms
            wcut = None if lossless or not has_w else p.max_weight
            ccut = (not lossless) and has_c

            def state(c, child):
                if ccut and abs(c * sn) < p.min_coeff:
                    return HELD
                if wcut is not None and weight(child) > wcut:
                    return DROP
                return EMIT

            index = {k: i for i, k in enumerate(rows_k)}
            new_c, new_t = list(rows_c), list(rows_t)
            children = []
            for r in range(N):
                if not anti[r]:
                    continue
                kr = np.array(rows_k[r], dtype=np.uint64)
                q_arr, ph = oracle.product(basis, gen, kr)
                q = key(kr ^ gen)
                j = index.get(q)
                if j is not None and j < r:
                    continue
                c, t = rows_c[r], rows_t[r]
                s_i = _neg_im(ph)
                bi, bti = c * sn * s_i, (t * sn + c * cs * e_g) * s_i
                si = state(c, q)
                if j is None:
                    new_c[r], new_t[r] = c * cs, t * cs - c * sn * e_g
                    if si == EMIT:
                        children.append((q, bi, bti))
                    continue
                cj, tj = rows_c[j], rows_t[j]
                _, ph_j = oracle.product(basis, gen, np.array(q, dtype=np.uint64))
                s_j = _neg_im(ph_j)
                bj, btj = cj * sn * s_j, (tj * sn + cj * cs * e_g) * s_j
                sj = state(cj, rows_k[r])
                to_j = si == EMIT or (si == HELD and sj == EMIT)
                to_i = sj == EMIT or (sj == HELD and si == EMIT)
                ni, ti = c * cs, t * cs - c * sn * e_g
                if to_i:
                    ni, ti = ni + bj, ti + btj
                nj, tj2 = cj * cs, tj * cs - cj * sn * e_g
                if to_j:
                    nj, tj2 = nj + bi, tj2 + bti
                new_c[r], new_t[r] = ni, ti
                new_c[j], new_t[j] = nj, tj2
            rows_c, rows_t = new_c, new_t
            for q, b, bt in children:
                rows_k.append(q)
                rows_c.append(b)
                rows_t.append(bt)
    e, grad = 0.0, np.zeros(G)
    for k, c, t in zip(rows_k, rows_c, rows_t):
        tr = oracle.trace(basis, n_units, np.array(k, dtype=np.uint64), p.diag)
        e += c * tr
        grad += t * tr
    return e, grad
