"""Spin-1/2 operators as sums of canonical masked terms, and their compiled row programs.

Host-side set-up of the sector matvec: the operator algebra and program compilation that feed the device
kernel, restated from the reference's ``MaskedOperator`` (include/ed/ops/algebra.h:19-87,
src/ops/algebra.cpp:20-266) and ``compile_operator`` / ``compile_program`` (src/ops/program.cpp:24-146).

A canonical term acts on a basis state s (a set bit is an up spin) as
``coeff * (-1)^popcount(s & sign) |s ^ flip>`` when ``s & flip == val`` (include/ed/ops/term.h:1-65).
Terms are keyed by (flip, val, sign) and coefficients accumulate in the reference's order, so the compiled
arrays equal the reference's bit for bit (the tests compare them).

A :class:`Program` holds the flip-grouped layout the kernels walk (include/ed/ops/program.h:66-94): groups
by ascending flip mask (the diagonal first), value subgroups ascending, terms in key order.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


def _popc(x: int) -> int:
    return bin(x).count("1")


def _low(x: int) -> int:
    return x & -x


def _rs(x: float, c: complex) -> complex:
    """Real times complex as std::complex does it: componentwise."""
    return complex(x * c.real, x * c.imag)


def _div(c: complex, x: float) -> complex:
    """Complex over real as std::complex does it: componentwise."""
    return complex(c.real / x, c.imag / x)


def _neg(c: complex) -> complex:
    return complex(-c.real, -c.imag)


def permute_mask(m: int, perm, n: int) -> int:
    """Image of a bit mask: new bit i = old bit perm[i] (include/ed/ops/term.h:72-77)."""
    r = 0
    for i in range(n):
        r |= ((m >> int(perm[i])) & 1) << i
    return r


class MaskedOperator:
    """An operator on ``n_sites`` spins as canonical terms (flip, val, sign) -> coeff."""

    def __init__(self, n_sites: int):
        if not 1 <= n_sites <= 64:
            raise ValueError("MaskedOperator: n_sites must be in [1, 64]")
        self.n = n_sites
        self.t: dict[tuple[int, int, int], complex] = {}

    # -- accumulation (algebra.cpp:24-32) --
    def _acc(self, key, c: complex):
        if c == 0:
            return
        v = self.t.get(key, complex(0.0, 0.0)) + c
        if v == 0:
            self.t.pop(key, None)
        else:
            self.t[key] = v

    def add_term(self, cond: int, val: int, flip: int, sign: int, coeff: complex):
        """Bring one term of any form to canonical form (algebra.cpp:34-66)."""
        allm = (1 << self.n) - 1
        if (cond | flip | sign) & ~allm:
            raise ValueError("MaskedOperator.add_term: mask beyond n_sites")
        stack = [(cond, val & cond, flip, sign, complex(coeff))]
        while stack:
            C, V, F, S, c = stack.pop()
            V &= C
            known = S & C
            if known:
                if _popc(known & V) & 1:
                    c = _neg(c)
                S &= ~C
            if c == 0:
                continue
            free = F & ~C
            if free:
                b = _low(free)
                stack.append((C | b, V, F, S, c))
                stack.append((C | b, V | b, F, S, c))
                continue
            proj = C & ~F
            if proj:
                b = _low(proj)
                s = -1.0 if (V & b) else 1.0
                stack.append((C & ~b, V & ~b, F, S, _rs(0.5, c)))
                stack.append((C & ~b, V & ~b, F, S | b, _rs(0.5 * s, c)))
                continue
            self._acc((F, V, S), c)

    @staticmethod
    def product(n_sites: int, ops: str, sites, coeff: complex = 1.0) -> "MaskedOperator":
        """coeff * prod_k ops[k](sites[k]), the last factor acting first (algebra.cpp:68-100).

        ops over '+', '-', 'z', 'x', 'y', 'u', 'd', 'I' (S+, S-, S^z, S^x, S^y, |up><up|, |dn><dn|, 1).
        """
        if len(ops) != len(sites):
            raise ValueError("product: ops and sites differ in length")
        r = MaskedOperator(n_sites)
        r._acc((0, 0, 0), complex(coeff))
        for op, i in zip(ops, sites):
            i = int(i)
            if not 0 <= i < n_sites:
                raise ValueError("product: site out of range")
            b = 1 << i
            f = MaskedOperator(n_sites)
            if op == "+":
                f.add_term(b, 0, b, 0, 1.0)
            elif op == "-":
                f.add_term(b, b, b, 0, 1.0)
            elif op == "z":
                f.add_term(0, 0, 0, b, -0.5)
            elif op == "x":
                f.add_term(b, 0, b, 0, 0.5)
                f.add_term(b, b, b, 0, 0.5)
            elif op == "y":
                f.add_term(b, 0, b, 0, complex(0.0, -0.5))
                f.add_term(b, b, b, 0, complex(0.0, 0.5))
            elif op == "u":
                f.add_term(b, b, 0, 0, 1.0)
            elif op == "d":
                f.add_term(b, 0, 0, 0, 1.0)
            elif op == "I":
                f._acc((0, 0, 0), complex(1.0))
            else:
                raise ValueError(f"product: unknown op {op!r}")
            r = r * f
        return r

    def add(self, o: "MaskedOperator", scale: complex = 1.0) -> "MaskedOperator":
        if o.n != self.n:
            raise ValueError("add: n_sites differ")
        scale = complex(scale)
        for k in sorted(o.t):
            self._acc(k, scale * o.t[k])
        return self

    def __mul__(self, o: "MaskedOperator") -> "MaskedOperator":
        """self * o, o acting first (algebra.cpp:128-145)."""
        r = MaskedOperator(self.n)
        okeys = sorted(o.t)
        for ka in sorted(self.t):
            FA, VA, SA = ka
            ca = self.t[ka]
            for kb in okeys:
                FB, VB, SB = kb
                VA_in = VA ^ (FB & FA)
                if ((VB ^ VA_in) & (FA & FB)) != 0:
                    continue
                c = ca * o.t[kb]
                if _popc(FB & SA) & 1:
                    c = _neg(c)
                r.add_term(FA | FB, VB | VA_in, FA ^ FB, SA ^ SB, c)
        return r

    def dagger(self) -> "MaskedOperator":
        r = MaskedOperator(self.n)
        for (F, V, S) in sorted(self.t):
            r._acc((F, V ^ F, S), self.t[(F, V, S)].conjugate())
        return r

    def image(self, perm, flip_xor: int = 0) -> "MaskedOperator":
        """U_g O U_g^dagger for the element (perm, flip) (algebra.cpp:159-169)."""
        r = MaskedOperator(self.n)
        for (F, V, S) in sorted(self.t):
            c = self.t[(F, V, S)]
            Fp = permute_mask(F, perm, self.n)
            Vp = permute_mask(V, perm, self.n) ^ (flip_xor & Fp)
            Sp = permute_mask(S, perm, self.n)
            r._acc((Fp, Vp, Sp), _neg(c) if (_popc(flip_xor & Sp) & 1) else c)
        return r

    def terms(self, drop: float = 0.0):
        """Canonical terms (flip, val, sign, coeff) in key order, |coeff| above ``drop``."""
        return [(F, V, S, self.t[(F, V, S)]) for (F, V, S) in sorted(self.t) if abs(self.t[(F, V, S)]) > drop]

    def max_abs(self) -> float:
        return max((abs(c) for c in self.t.values()), default=0.0)

    def to_dense(self) -> np.ndarray:
        """M[t, s] = <t|O|s> over the full 2^n space (tests only, n <= 12)."""
        if self.n > 12:
            raise ValueError("to_dense: n_sites > 12")
        dim = 1 << self.n
        M = np.zeros((dim, dim), complex)
        for F, V, S, c in self.terms():
            for s in range(dim):
                if (s & F) != V:
                    continue
                M[s ^ F, s] += (-c if _popc(s & S) & 1 else c)
        return M


def from_products(n_sites: int, products) -> MaskedOperator:
    """The sum over records (ops, sites, coeff) of MaskedOperator.product, in record order."""
    O = MaskedOperator(n_sites)
    for ops, sites, coeff in products:
        O.add(MaskedOperator.product(n_sites, ops, sites, coeff))
    return O


@dataclass
class Program:
    """A row program in the flip-grouped layout (include/ed/ops/program.h:66-94)."""

    group_flip: np.ndarray
    group_setbits: np.ndarray
    group_vbegin: np.ndarray
    vsub_val: np.ndarray
    vsub_tbegin: np.ndarray
    term_sign: np.ndarray
    term_coeff: np.ndarray  # complex128
    n_sites: int = 0
    delta_set_bits: int = 0
    meta: dict = field(default_factory=dict)

    @property
    def n_groups(self) -> int:
        return len(self.group_flip)

    @property
    def n_vsub(self) -> int:
        return len(self.vsub_val)

    @property
    def n_terms(self) -> int:
        return len(self.term_sign)

    def norm_bound(self) -> float:
        """Sum of |coeff|: an upper bound of the operator norm (the solvers' scale)."""
        return float(np.sum(np.abs(self.term_coeff)))

    def coeff_interleaved(self) -> np.ndarray:
        return np.ascontiguousarray(self.term_coeff.astype(np.complex128)).view(np.float64)


def _pack(tree: dict, n_sites: int, delta: int = 0) -> Program:
    """Pack flip -> value -> [(sign, coeff)] into the program arrays (program.cpp:33-53)."""
    gf, gs, gv, vv, vt, ts, tc = [], [], [0], [], [0], [], []
    for F in sorted(tree):
        vmap = tree[F]
        vals = sorted(vmap)
        sb = _popc(vals[0])
        for V in vals:
            if _popc(V) != sb:
                sb = -1
        gf.append(F)
        gs.append(sb)
        for V in vals:
            vv.append(V)
            for S, c in vmap[V]:
                ts.append(S)
                tc.append(c)
            vt.append(len(ts))
        gv.append(len(vv))
    return Program(
        group_flip=np.array(gf, np.uint64),
        group_setbits=np.array(gs, np.int32),
        group_vbegin=np.array(gv, np.uint32),
        vsub_val=np.array(vv, np.uint64),
        vsub_tbegin=np.array(vt, np.uint32),
        term_sign=np.array(ts, np.uint64),
        term_coeff=np.array(tc, np.complex128),
        n_sites=n_sites,
        delta_set_bits=delta,
    )


def compile_operator(O: MaskedOperator) -> Program:
    """O's terms in the flip-grouped layout, no projection (program.cpp:127-136)."""
    tree: dict = {}
    for F, V, S, c in O.terms():
        tree.setdefault(F, {}).setdefault(V, []).append((S, c))
    return _pack(tree, O.n)


def row_program(O: MaskedOperator) -> Program:
    """The program the sector rows walk: compile_operator(O^dagger) (include/ed/ops/operator.h:132-137)."""
    return compile_operator(O.dagger())


def _delta_set_bits(F: int, V: int) -> int:
    return _popc(F & ~V) - _popc(F & V)


def compile_program(O: MaskedOperator, src, tgt, drop: float = 1e-14) -> Program:
    """O lambda-projected for <tgt|O|src> between two sectors of one group (program.cpp:60-124).

    ``src`` / ``tgt`` carry ``perms`` (G x N), ``flips`` (G), ``chars`` (G complex) and ``n_up``.
    """
    G = len(src.chars)
    n = O.n
    perms = np.asarray(src.perms)
    flips = np.zeros(G, np.uint64) if src.flips is None else np.asarray(src.flips, np.uint64)
    if not np.array_equal(perms, np.asarray(tgt.perms)):
        raise ValueError("compile_program: the two sectors come from different groups")
    delta_req = tgt.n_up - src.n_up
    w = [_div((complex(tgt.chars[g]) * complex(src.chars[g]).conjugate()).conjugate(), float(G)) for g in range(G)]
    Ol = MaskedOperator(n)
    for g in range(G):
        if abs(w[g]) < 1e-15:
            continue
        Ol.add(O.image(perms[g], int(flips[g])), w[g])
    scale = O.max_abs()
    tree: dict = {}
    for F, V, S, c in Ol.terms(drop * scale):
        if _delta_set_bits(F, V) != delta_req:
            continue
        tree.setdefault(F, {}).setdefault(V, []).append((S, c))
    p = _pack(tree, n, delta_req)
    return p


def cross_row_program(O: MaskedOperator, row_sector, col_sector) -> Program:
    """Rows in ``row_sector`` of O applied to vectors of ``col_sector``: the program of (O_lambda)^dagger
    compiled with the row sector as the ket and the column sector as the bra (sector_rows.h:16-19,
    src/engine/internal.h:545-551)."""
    return compile_program(O.dagger(), row_sector, col_sector)


# ---------------------------------------------------------------------------------------------
# Model builders (the conventions of python/qed/_builder.py:151-162, 277-286 and the reference
# test zoo's chiral_terms, tests/python/support/models.py:467-476).
# ---------------------------------------------------------------------------------------------
def xxz_products(bonds, Jxy: float, Jz: float):
    """Jxy (Sx Sx + Sy Sy) + Jz Sz Sz per bond as product records."""
    out = []
    for i, j in bonds:
        if i == j:
            continue
        out.append(("+-", (i, j), complex(0.5 * Jxy, 0.0)))
        out.append(("-+", (i, j), complex(0.5 * Jxy, 0.0)))
        if Jz != 0.0:
            out.append(("zz", (i, j), complex(Jz, 0.0)))
    return out


def heisenberg_products(bonds, J: float = 1.0):
    return xxz_products(bonds, J, J)


def zeeman_z_products(n_sites: int, hz: float):
    """-hz S^z on every site."""
    return [("z", (i,), complex(-hz, 0.0)) for i in range(n_sites)] if hz != 0.0 else []


def chiral_products(triangles, K: float):
    """K S_i . (S_j x S_k) per triangle: (i/2) sum_cyclic Sz_a (S+_b S-_c - S-_b S+_c)."""
    out = []
    for i, j, k in triangles:
        for a, b, c in ((i, j, k), (j, k, i), (k, i, j)):
            out.append(("z+-", (a, b, c), complex(0.0, 0.5 * K)))
            out.append(("z-+", (a, b, c), complex(0.0, -0.5 * K)))
    return out


def sz_q_products(n_sites: int, q: float):
    """S^z(q) = N^{-1/2} sum_j e^{-i q j} S^z_j."""
    nrm = 1.0 / np.sqrt(n_sites)
    return [("z", (j,), complex(nrm * np.cos(-q * j), nrm * np.sin(-q * j))) for j in range(n_sites)]
