"""pq_surrogate.py -- TEST INFRASTRUCTURE, not product code.

A CPU restatement of propaq's surrogate (symbolic) propagation, the
reference's build-once / evaluate-many model of theta -> <s|U(theta)^dag H
U(theta)|s>.  It is the checker behind the gradient's surrogate cross-check:
the derivative of the surrogate model at theta, taken by reverse mode over
its compiled tape, against the adjoint gradient of the numerical engine.

It follows the reference step by step, with its own data structures:

  * the coefficient DAG and its node
    metadata (count, frequencies, scale)   crates/surrogate/src/symcoeff.rs:1-140
  * symbolic / numeric rotation             symcoeff.rs:263-295
  * prune (frequency and coefficient
    bounds, memoised by node, depth and
    scale exponent)                         symcoeff.rs:297-540
  * simplify (FactorRun expansion and
    balanced rebuild)                       symcoeff.rs:542-752
  * compile_batch (post-order, shared
    subtrees once) and tape evaluation      symcoeff.rs:165-257, 876-920
  * the build loop and truncation pass      crates/surrogate/src/engine.rs:22-235
  * the gate dispatch it runs through       crates/core/src/engine/partitioned_termsum.rs:276-350
  * the Clifford frame                      crates/core/src/algebra/tableau.rs:29-228
  * the model's evaluation                  crates/surrogate/src/model.rs:63-107

Keys are Python ints holding the interleaved layout (unit q at bits 2q and
2q+1).  The key algebra comes from an `algebra` object: `PauliAlgebra` below
(pure Python, checked against the C oracle's probes in the tests) or any
object with the same four methods, e.g. one backed by the C oracle for
Majorana keys.

The reference sums the model's terms and groups simplified monomials in
hash-map order; this restatement uses term and insertion order, so values
agree to floating-point rounding, not bit for bit.
"""

from __future__ import annotations

import math

U128_MAX = (1 << 128) - 1
U32_MAX = (1 << 32) - 1
I32_MIN = -(1 << 31)
I32_MAX = (1 << 31) - 1
EPS = 1e-9  # PHASE_ONLY_EPS, partitioned_termsum.rs:41
EVEN = 0x5555555555555555


# ------------------------------------------------------------------ algebra
def _even_mask(nbits):
    return int("01" * (nbits // 2), 2) if nbits else 0


class PauliAlgebra:
    """Pauli keys, unit q = X at bit 2q, Z at bit 2q+1
    (crates/pauli/src/algebra.rs:99-141, 206-213)."""

    basis = 0

    def __init__(self, n_units):
        self.n_units = n_units
        self.even = _even_mask(2 * max(n_units, 1) + 2)

    def _swap(self, g):
        e = self.even
        return ((g & e) << 1) | ((g >> 1) & e)

    def anticommutes(self, g, k):
        return bin(k & self._swap(g)).count("1") & 1 == 1

    def product(self, g, k):
        """(G xor K, p) with G K = i^p (G xor K)."""
        e = self.even
        o = g ^ k
        y = lambda x: bin(x & (x >> 1) & e).count("1")  # noqa: E731
        zx = bin((g >> 1) & k & e).count("1")
        return o, (y(g) + y(k) - y(o) + 2 * zx) & 3

    def weight(self, k):
        return bin((k | (k >> 1)) & self.even).count("1")

    def trace(self, k, state):
        """<state|K|state> for a computational-basis state (bit q = qubit q)."""
        if k & self.even:
            return 0.0
        z = (k >> 1) & self.even
        par = 0
        q = 0
        while z:
            if z & 1 and (state >> q) & 1:
                par ^= 1
            z >>= 2
            q += 1
        return -1.0 if par else 1.0


def _ipow(p):
    return (1 + 0j, 1j, -1 + 0j, -1j)[p & 3]


# ----------------------------------------------------------------- the frame
class Frame:
    """CliffordTableau (tableau.rs:29-228): readout rows P -> C^dag P C and
    generator rows P -> C P C^dag, each (image, sign)."""

    def __init__(self, alg, n_units, n_bits):
        self.alg = alg
        self.n_bits = n_bits
        rows = [((1 << p) if p < n_bits else 0, 1.0) for p in range(2 * n_units)]
        self.readout = list(rows)
        self.generator = list(rows)
        self.identity = True

    def _refresh(self):
        self.identity = all(img == ((1 << p) if p < self.n_bits else 0) and s == 1.0
                            for p, (img, s) in enumerate(self.readout))

    def _apply(self, rows, mono):
        """apply_rows (tableau.rs:109-143)."""
        src, src_ph = 0, 1 + 0j
        img, img_ph = 0, 1 + 0j
        p = 0
        m = mono
        while m:
            if m & 1 and p < len(rows):
                src, ph = self.alg.product(1 << p, src)
                src_ph *= _ipow(ph)
                r_img, r_sign = rows[p]
                img, ph = self.alg.product(r_img, img)
                img_ph *= _ipow(ph) * r_sign
            m >>= 1
            p += 1
        ratio = img_ph / src_ph
        return img, (1.0 if ratio.real >= 0.0 else -1.0)

    def conjugate(self, mono):
        return (mono, 1.0) if self.identity else self._apply(self.readout, mono)

    def conjugate_generator(self, mono):
        return (mono, 1.0) if self.identity else self._apply(self.generator, mono)

    def compose_rotation(self, gen, angle):
        """compose(for_rotation(gen, angle)) (tableau.rs:146-209)."""
        n = len(self.readout)
        step_r = [((1 << p) if p < self.n_bits else 0, 1.0) for p in range(n)]
        step_g = list(step_r)
        changed = False
        sn = math.sin(angle)
        for p in range(min(n, self.n_bits)):
            if not self.alg.anticommutes(gen, 1 << p):
                continue
            image, ph = self.alg.product(gen, 1 << p)
            sign = sn * (-_ipow(ph).imag)
            step_r[p] = (image, sign)
            step_g[p] = (image, -sign)
            changed = True
        step_identity = all(img == ((1 << p) if p < self.n_bits else 0) and s == 1.0
                            for p, (img, s) in enumerate(step_r))
        if not changed or step_identity:
            return
        new_r = []
        for img, s in self.readout:
            i2, s2 = self._apply(step_r, img)
            new_r.append((i2, s2 * s))
        new_g = []
        for img, s in step_g:
            i2, s2 = self._apply(self.generator, img)
            new_g.append((i2, s2 * s))
        self.readout, self.generator = new_r, new_g
        self._refresh()


# ---------------------------------------------------------------- the DAG
S, A, K, C, N = range(5)  # Scalar, Add, Scale, Cos, Sin


class Node:
    """One node of a coefficient's history (symcoeff.rs:21-140)."""

    __slots__ = ("kind", "a", "b", "val", "param", "count", "min_freq", "max_freq", "upper_scale")

    def __init__(self, kind, a=None, b=None, val=0.0, param=0, count=1, min_freq=0, max_freq=0, upper_scale=0.0):
        self.kind, self.a, self.b, self.val, self.param = kind, a, b, val, param
        self.count, self.min_freq, self.max_freq, self.upper_scale = count, min_freq, max_freq, upper_scale


def scalar(c):
    return Node(S, val=c, upper_scale=abs(c))


def add(a, b):
    return Node(A, a, b, count=min(a.count + b.count, U128_MAX), min_freq=min(a.min_freq, b.min_freq),
                max_freq=max(a.max_freq, b.max_freq), upper_scale=max(a.upper_scale, b.upper_scale))


def scale(f, a):
    return Node(K, a, val=f, count=a.count, min_freq=a.min_freq, max_freq=a.max_freq,
                upper_scale=abs(f) * a.upper_scale)


def _trig(kind, p, a):
    return Node(kind, a, param=p, count=a.count, min_freq=min(a.min_freq + 1, U32_MAX),
                max_freq=min(a.max_freq + 1, U32_MAX), upper_scale=a.upper_scale)


def cos_node(p, a):
    return _trig(C, p, a)


def sin_node(p, a):
    return _trig(N, p, a)


def signed(sign, node):
    return node if sign == 1.0 else scale(sign, node)


def add_assign(x, y):
    """CoeffRepr::add_assign (symcoeff.rs:784-791); None is the empty coefficient."""
    if x is None:
        return y
    if y is None:
        return x
    return add(x, y)


def apply_rotation(c, param, phase):
    """(cos branch, sin branch) of coefficient c under a rotation whose
    product phase is `phase` (symcoeff.rs:263-295).  param = ("sym", p) or
    ("num", angle)."""
    if c is None:
        return None, None
    kind, v = param
    if kind == "sym":
        branch = (1j * phase).real
        return cos_node(v, c), signed(branch, sin_node(v, c))
    cos_t, sin_t = math.cos(v), math.sin(v)
    branch = (complex(0.0, sin_t) * phase).real
    return scale(cos_t, c), scale(branch, c)


def monomial_count(c):
    return 0 if c is None else c.count


# ------------------------------------------------------------------ prune
def _ceil_log2_abs_i32(k):
    if k == 0.0:
        return I32_MIN
    if math.isnan(k):
        return 0
    v = math.ceil(math.log2(abs(k)))
    return max(I32_MIN, min(I32_MAX, v))


def _sat_i32(x):
    return max(I32_MIN, min(I32_MAX, x))


def prune(root, max_frequency, coeff_cutoff):
    """SymbolicCoeff::prune / prune_node (symcoeff.rs:255-540)."""
    if root is None or (max_frequency is None and coeff_cutoff is None):
        return root
    has_f, has_c = max_frequency is not None, coeff_cutoff is not None
    cap = max_frequency if has_f else U32_MAX
    cutoff = coeff_cutoff if has_c else 0.0
    log_cut = math.log2(cutoff) if cutoff > 0.0 else 0.0

    def key(node, depth, sexp):
        return (id(node), depth if has_f else 0, sexp if has_c else 0)

    def doomed_by_coeff(sexp, upper):
        if cutoff <= 0.0:
            return False
        lu = math.log2(upper) if upper > 0.0 else -math.inf
        return float(sexp) + lu < log_cut

    memo = {}
    scheduled = {key(root, 0, 0)}
    stack = [(True, root, 0, 0)]
    while stack:
        enter, node, depth, sexp = stack.pop()
        k = key(node, depth, sexp)
        if enter:
            if (has_f and min(depth + node.min_freq, U32_MAX) > cap) or (has_c and doomed_by_coeff(sexp, node.upper_scale)):
                memo[k] = None
                continue
            if (has_f and not has_c and min(depth + node.max_freq, U32_MAX) <= cap) or (not has_f and not has_c):
                memo[k] = node
                continue
            stack.append((False, node, depth, sexp))
            if node.kind == A:
                for ch in (node.b, node.a):
                    kc = key(ch, depth, sexp)
                    if kc not in scheduled:
                        scheduled.add(kc)
                        stack.append((True, ch, depth, sexp))
            elif node.kind == K:
                ns = _sat_i32(sexp + _ceil_log2_abs_i32(node.val)) if has_c else sexp
                kc = key(node.a, depth, ns)
                if kc not in scheduled:
                    scheduled.add(kc)
                    stack.append((True, node.a, depth, ns))
            elif node.kind in (C, N):
                nd = min(depth + 1, U32_MAX)
                kc = key(node.a, nd, sexp)
                if kc not in scheduled:
                    scheduled.add(kc)
                    stack.append((True, node.a, nd, sexp))
            continue
        if node.kind == S:
            res = node
        elif node.kind == A:
            x, y = memo[key(node.a, depth, sexp)], memo[key(node.b, depth, sexp)]
            if x is None and y is None:
                res = None
            elif y is None:
                res = x
            elif x is None:
                res = y
            else:
                res = node if (x is node.a and y is node.b) else add(x, y)
        elif node.kind == K:
            ns = _sat_i32(sexp + _ceil_log2_abs_i32(node.val)) if has_c else sexp
            x = memo[key(node.a, depth, ns)]
            res = None if x is None else (node if x is node.a else scale(node.val, x))
        else:
            x = memo[key(node.a, min(depth + 1, U32_MAX), sexp)]
            res = None if x is None else (node if x is node.a else _trig(node.kind, node.param, x))
        memo[k] = res
    return memo[key(root, 0, 0)]


# --------------------------------------------------------------- simplify
def _post_order(roots):
    """Nodes reachable from `roots`, children before parents, each once."""
    seen = set()
    order = []
    for r in roots:
        if r is None or id(r) in seen:
            continue
        seen.add(id(r))
        stack = [(r, False)]
        while stack:
            node, done = stack.pop()
            if done:
                order.append(node)
                continue
            stack.append((node, True))
            kids = (node.b, node.a) if node.kind == A else ((node.a,) if node.kind != S else ())
            for ch in kids:
                if id(ch) not in seen:
                    seen.add(id(ch))
                    stack.append((ch, False))
    return order


def simplify_batch(coeffs):
    """simplify_batch (symcoeff.rs:564-720): every coefficient expanded into
    monomials keyed by their (param -> (cos power, sin power)) run, equal runs
    summed at each Add, then rebuilt as a balanced sum of leaves."""
    memo = {}
    for node in _post_order(coeffs):
        if node.kind == S:
            terms = {(): node.val}
        elif node.kind == A:
            terms = dict(memo[id(node.a)])
            for run, v in memo[id(node.b)].items():
                terms[run] = terms.get(run, 0.0) + v
        elif node.kind == K:
            terms = {run: v * node.val for run, v in memo[id(node.a)].items()}
        else:
            terms = {}
            for run, v in memo[id(node.a)].items():
                d = dict(run)
                c, s = d.get(node.param, (0, 0))
                d[node.param] = (c + (node.kind == C), s + (node.kind == N))
                terms[tuple(sorted(d.items()))] = v
        memo[id(node)] = terms
    out = []
    rebuilt = {}
    for c in coeffs:
        if c is None:
            out.append(None)
            continue
        if id(c) not in rebuilt:
            rebuilt[id(c)] = _rebuild_balanced(memo[id(c)])
        out.append(rebuilt[id(c)])
    return out


def _rebuild_balanced(terms):
    leaves = []
    for run, v in terms.items():
        if v == 0.0:
            continue
        node = scalar(v)
        for p, (cp, sp) in run:  # ascending parameter order
            for _ in range(cp):
                node = cos_node(p, node)
            for _ in range(sp):
                node = sin_node(p, node)
        leaves.append(node)
    if not leaves:
        return None
    while len(leaves) > 1:
        nxt = [add(leaves[i], leaves[i + 1]) if i + 1 < len(leaves) else leaves[i] for i in range(0, len(leaves), 2)]
        leaves = nxt
    return leaves[0]


# ------------------------------------------------------------ compile / eval
class Tape:
    """compile_batch (symcoeff.rs:165-257): nodes in post-order, each once."""

    def __init__(self, roots):
        self.ops = _post_order(roots)
        index = {id(n): i for i, n in enumerate(self.ops)}
        self.roots = [index[id(r)] if r is not None else -1 for r in roots]
        self.args = [(index[id(n.a)] if n.kind != S else -1, index[id(n.b)] if n.kind == A else -1) for n in self.ops]

    def evaluate_all(self, lut):
        out = [0.0] * len(self.ops)
        for i, (n, (a, b)) in enumerate(zip(self.ops, self.args)):
            if n.kind == S:
                out[i] = n.val
            elif n.kind == A:
                out[i] = out[a] + out[b]
            elif n.kind == K:
                out[i] = n.val * out[a]
            elif n.kind == C:
                out[i] = lut[2 * n.param] * out[a]
            else:
                out[i] = lut[2 * n.param + 1] * out[a]
        return out

    def monomial_counts(self):
        counts = [0] * len(self.ops)
        for i, (n, (a, b)) in enumerate(zip(self.ops, self.args)):
            counts[i] = 1 if n.kind == S else (min(counts[a] + counts[b], U128_MAX) if n.kind == A else counts[a])
        return counts


def make_lut(params):
    """cos/sin per parameter (model.rs:104-107)."""
    lut = []
    for t in params:
        lut += [math.cos(t), math.sin(t)]
    return lut


class Model:
    """SurrogateModel (model.rs:46-125): terms (overlap, root) over one tape."""

    def __init__(self, overlaps, roots, n_params):
        self.tape = Tape(roots)
        self.overlaps = list(overlaps)
        self.n_params = n_params

    @property
    def n_terms(self):
        return len(self.overlaps)

    @property
    def n_monomials(self):
        counts = self.tape.monomial_counts()
        total = 0
        for r in self.tape.roots:
            if r >= 0:
                total = min(total + counts[r], U128_MAX)
        return total

    def evaluate(self, params):
        if len(params) < self.n_params:
            raise ValueError(f"params has {len(params)} elements but model requires {self.n_params}")
        out = self.tape.evaluate_all(make_lut(params))
        return sum(o * out[r] for o, r in zip(self.overlaps, self.tape.roots) if r >= 0)

    def gradient(self, params):
        """dE/dparams by reverse mode over the tape: a Cos(p) node contributes
        -sin(theta_p) * (its input's value) * (its adjoint), a Sin(p) node
        cos(theta_p) * ... ."""
        lut = make_lut(params)
        out = self.tape.evaluate_all(lut)
        adj = [0.0] * len(out)
        for o, r in zip(self.overlaps, self.tape.roots):
            if r >= 0:
                adj[r] += o
        grad = [0.0] * self.n_params
        for i in range(len(out) - 1, -1, -1):
            g = adj[i]
            if g == 0.0:
                continue
            n = self.tape.ops[i]
            a, b = self.tape.args[i]
            if n.kind == A:
                adj[a] += g
                adj[b] += g
            elif n.kind == K:
                adj[a] += n.val * g
            elif n.kind == C:
                adj[a] += lut[2 * n.param] * g
                grad[n.param] -= lut[2 * n.param + 1] * out[a] * g
            elif n.kind == N:
                adj[a] += lut[2 * n.param + 1] * g
                grad[n.param] += lut[2 * n.param] * out[a] * g
        return grad


# ------------------------------------------------------------------ build
def build(alg, n_units, n_bits, observable, gates, *, frequency=None, coefficient=None, weight=None,
          min_terms=None, simplify=False, initial_state=0, n_params=None):
    """The surrogate build (engine.rs:157-235).

    observable: [(key, coeff)]; gates: [(generator key, param)] in Heisenberg
    order (circuit layers reversed, gates in each layer reversed, as
    extract_layers does, engine.rs:237-262); param = ("sym", index) or
    ("num", angle).  Every numeric Clifford rotation is deferred into the
    frame: the build's emit cutoff has no weight (engine.rs:176), so
    partitioned_termsum.rs:288-297 defers whatever the weight cut."""
    terms = {}
    for k, c in observable:
        terms[k] = add_assign(terms.get(k), scalar(c))
    frame = Frame(alg, n_units, n_bits)
    if n_params is None:
        n_params = 1 + max((v for _, (kind, v) in gates if kind == "sym"), default=-1)
    for gen, param in gates:
        _apply_rotation(alg, frame, terms, gen, param)
        # apply_truncation (engine.rs:22-58)
        lossy = len(terms) >= (min_terms or 0)
        if simplify and terms:
            ks = list(terms)
            for k, c in zip(ks, simplify_batch([terms[k] for k in ks])):
                terms[k] = c
        if lossy:
            f = None if frequency is None else min(frequency, U32_MAX)
            for k in list(terms):
                terms[k] = prune(terms[k], f, coefficient)
            for k in [k for k, c in terms.items() if c is None or (weight is not None and alg.weight(k) > weight)]:
                del terms[k]
    # compile (engine.rs:61-107): overlap through the frame, |overlap| > 1e-15
    overlaps, roots = [], []
    for k, c in terms.items():
        image, sign = frame.conjugate(k)
        ov = sign * alg.trace(image, initial_state)
        if abs(ov) > 1e-15:
            overlaps.append(ov)
            roots.append(c)
    return Model(overlaps, roots, n_params)


def _apply_rotation(alg, frame, terms, gen, param):
    """PartitionedTermSum::apply_rotation for symbolic coefficients with no
    emit cutoff (partitioned_termsum.rs:276-350, termsum.rs:551-751)."""
    if not terms:
        return
    kind, v = param
    if kind == "num" and abs(math.cos(v)) < EPS:
        frame.compose_rotation(gen, v)
        return
    g, sign = frame.conjugate_generator(gen)
    if kind == "num" and abs(math.sin(v)) < EPS:
        cos_t = math.cos(v)
        for k in list(terms):
            if alg.anticommutes(g, k):
                terms[k] = scale(cos_t, terms[k])
        return
    routed = []
    for k in list(terms):
        if not alg.anticommutes(g, k):
            continue
        child, p = alg.product(g, k)
        cos_b, sin_b = apply_rotation(terms[k], param, sign * _ipow(p))
        terms[k] = cos_b
        routed.append((child, sin_b))
    for child, b in routed:
        terms[child] = add_assign(terms.get(child), b)
