"""The host operator algebra (a restatement of the reference's MaskedOperator) against dense matrices."""
import numpy as np
import pytest

from qed_spin_b200 import operators as ops

SP = np.array([[0, 0], [1, 0]], complex)   # basis (up=|1>?) -- built below from the set-bit-is-up convention


def site_op(op, i, n):
    """2^n x 2^n matrix of a one-site operator; bit i set = up."""
    up, dn = np.array([0, 1.0]), np.array([1.0, 0])
    Sz = np.diag([-0.5, 0.5])          # index 0 = bit clear = down, index 1 = up
    Sp = np.array([[0, 0], [1.0, 0]])  # |up><dn|
    Sm = Sp.T
    m = {"z": Sz, "+": Sp, "-": Sm, "x": (Sp + Sm) / 2, "y": (Sp - Sm) / 2j,
         "u": np.outer(up, up), "d": np.outer(dn, dn), "I": np.eye(2)}[op]
    out = np.array([[1.0]])
    for k in reversed(range(n)):
        out = np.kron(out, m if k == i else np.eye(2))
    return out


def dense_product(ops_str, sites, c, n):
    M = np.eye(2 ** n, dtype=complex) * c
    for o, s in zip(ops_str, sites):
        M = M @ site_op(o, s, n)
    return M


@pytest.mark.parametrize("seed", range(6))
def test_products_match_dense(seed):
    rng = np.random.default_rng(seed)
    n = 5
    prods = []
    for _ in range(6):
        k = rng.integers(1, 4)
        o = "".join(rng.choice(list("+-zxyudI"), size=k))
        s = tuple(int(x) for x in rng.integers(0, n, size=k))
        prods.append((o, s, complex(rng.normal(), rng.normal())))
    O = ops.from_products(n, prods)
    D = sum(dense_product(o, s, c, n) for o, s, c in prods)
    np.testing.assert_allclose(O.to_dense(), D, atol=1e-12)
    np.testing.assert_allclose(O.dagger().to_dense(), D.conj().T, atol=1e-12)


def test_program_layout_and_walk():
    n = 6
    prods = ops.heisenberg_products([(i, (i + 1) % n) for i in range(n)]) + ops.zeeman_z_products(n, 0.3)
    O = ops.from_products(n, prods)
    p = ops.compile_operator(O)
    assert p.group_flip[0] == 0 and np.all(np.diff(p.group_flip.astype(np.int64)) > 0)
    D = O.to_dense()
    # walk the program on every state: <s^F|O|s> = sum of the subgroup's signed terms
    W = np.zeros_like(D)
    for s in range(2 ** n):
        for g in range(p.n_groups):
            F = int(p.group_flip[g])
            v = s & F
            for vi in range(p.group_vbegin[g], p.group_vbegin[g + 1]):
                if int(p.vsub_val[vi]) != v:
                    continue
                h = 0
                for t in range(p.vsub_tbegin[vi], p.vsub_tbegin[vi + 1]):
                    sg = -1 if bin(s & int(p.term_sign[t])).count("1") & 1 else 1
                    h += sg * p.term_coeff[t]
                W[s ^ F, s] += h
    np.testing.assert_allclose(W, D, atol=1e-12)
