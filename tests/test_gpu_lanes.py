"""The ground-state vector, the k > 1 lane and T = 0 dynamics on the device, through the C-ABI.

Tolerances, written per test:
- ground state: E0 within 1e-12 relative of the reference engine's k = 1 lane (fixtures); the residual
  ||H psi - E psi||, measured with the oracle's host matvec, within the lane's 1e-9 * scale certificate;
- k = 4 levels: within 1e-9 * scale of the reference engine's krylov_schur_kernel (fixtures) and of a dense
  eigensolve of the oracle's matrix;
- S(q, omega): the device's ground state is certified to ||H psi - E psi|| <= 1e-9 * scale, so it differs from the
  dense one by up to residual / gap (~3e-8 here) and S by about twice that: within 1e-6 of max S of the oracle's
  continued fraction from the dense ground state (depth 10, the orthogonal regime of these sectors).
"""
import numpy as np
import pytest

from cases import CASES, NAMES
from oracle import oracle as O
from qed_spin_b200 import lattice as lat
from qed_spin_b200 import operators as ops

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.fail("a GPU test ran without a CUDA device")
    from qed_spin_b200 import build
    build.build()


CASE = {c[0]: c for c in CASES}


def _prog(name):
    _, spec, prods = CASE[name]
    return ops.row_program(ops.from_products(spec.n_sites, prods))


def _scale(prog):
    return float(np.abs(np.asarray(prog.term_coeff)).sum())


def _dense(So, Po, col=None):
    """The sector block of the operator as a dense matrix, column by column through the oracle's matvec."""
    col = So if col is None else col
    n = col.dim
    M = np.zeros((So.dim, n), np.complex128)
    for j in range(n):
        e = np.zeros(n, np.complex128)
        e[j] = 1.0
        M[:, j] = So.gather(Po, e, col=col)
    return M


@pytest.mark.parametrize("name", NAMES)
def test_ground_state(fixtures, name):
    from qed_spin_b200 import device as D
    spec = CASE[name][1]
    prog = _prog(name)
    r = D.ground_state(D.Sector(spec), D.Program(prog))
    re0 = fixtures[f"{name}/e0"][0]
    assert r["certified"]
    assert abs(r["e0"] - re0) <= 1e-12 * abs(re0)
    psi = r["vector"]
    assert abs(np.linalg.norm(psi) - 1.0) < 1e-12
    So, Po = O.Sector(spec), O.Program(prog)
    res = np.linalg.norm(So.gather(Po, psi) - r["e0"] * psi)
    assert res <= 1e-9 * _scale(prog)


@pytest.mark.parametrize("dtype", ["c128", "c64"])
@pytest.mark.parametrize("name", NAMES)
def test_eigs_k4(fixtures, name, dtype):
    """The k > 1 lane in FP64 storage, and in FP32 storage with the FP64 refinement of every pair: the levels
    within 1e-9 * scale of the reference's and of a dense solve, each vector an eigenvector to 1e-8 * scale."""
    from qed_spin_b200 import device as D
    spec = CASE[name][1]
    prog = _prog(name)
    r = D.eigs(D.Sector(spec), D.Program(prog), 4, vectors=True, dtype=dtype, refine=True)
    assert r["converged"] and len(r["values"]) == 4
    sc = _scale(prog)
    np.testing.assert_allclose(r["values"], fixtures[f"{name}/ks4"], rtol=0, atol=1e-9 * sc)
    So, Po = O.Sector(spec), O.Program(prog)
    w = np.linalg.eigvalsh(_dense(So, Po))[:4]
    np.testing.assert_allclose(r["values"], w, rtol=0, atol=1e-9 * sc)
    for e, v in zip(r["values"], r["vectors"]):   # each returned vector is its level's eigenvector
        assert np.linalg.norm(So.gather(Po, v) - e * v) <= 1e-8 * sc


def test_eigs_k6_degenerate_levels():
    """A block without spatial symmetry (the S^z = 0 states of a Heisenberg ring N = 10, the identity group only):
    the momenta k and -k make doubly degenerate levels, which one Krylov space cannot resolve; the lane's deflated
    searches below the k-th level must find both members (against a dense solve, 1e-9 * scale), FP64 and FP32
    storage."""
    from qed_spin_b200 import device as D
    N = 10
    spec = lat.SectorSpec(N, N // 2, np.arange(N, dtype=np.int32)[None, :], np.ones(1, np.complex128))
    prog = ops.row_program(ops.from_products(N, ops.heisenberg_products(lat.chain_bonds(N))))
    So, Po = O.Sector(spec), O.Program(prog)
    w = np.linalg.eigvalsh(_dense(So, Po))
    assert np.min(np.diff(w[:6])) < 1e-9   # the block has degenerate levels among its lowest six
    sc = _scale(prog)
    for dtype in ("c128", "c64"):
        r = D.eigs(D.Sector(spec), D.Program(prog), 6, dtype=dtype, refine=True)
        assert r["converged"], dtype
        np.testing.assert_allclose(r["values"], w[:6], rtol=0, atol=1e-9 * sc, err_msg=dtype)


def test_eigs_k4_chain20():
    """Config 1's block: the periodic Heisenberg chain N = 20, Sz = 0, k = 0 (9,252 representatives)."""
    from qed_spin_b200 import device as D
    spec = lat.chain_sector(20, 10, 0)
    prog = ops.row_program(ops.from_products(20, ops.heisenberg_products(lat.chain_bonds(20))))
    r = D.eigs(D.Sector(spec), D.Program(prog), 4)
    assert r["converged"]
    e_or, _, cv = O.Sector(spec).scan_lowest(O.Program(prog))
    assert cv and abs(r["values"][0] - e_or) <= 1e-10 * abs(e_or)
    assert np.all(np.diff(r["values"]) >= -1e-12)


@pytest.mark.parametrize("N,m", [(12, 3), (12, 6), (10, 1)])
def test_dynamics_szq(N, m):
    """S^z(q) from the k = 0 ground state to the k = q sector, against the oracle's continued fraction."""
    from qed_spin_b200 import device as D
    q = 2 * np.pi * m / N
    src, tgt = lat.chain_sector(N, N // 2, 0), lat.chain_sector(N, N // 2, m)
    prods = ops.heisenberg_products(lat.chain_bonds(N), 1.0) + ops.chiral_products(
        [(i, (i + 1) % N, (i + 2) % N) for i in range(N)], 0.2)
    H = ops.from_products(N, prods)
    h_src = ops.row_program(H)
    Sq = ops.from_products(N, ops.sz_q_products(N, q))
    cross = ops.cross_row_program(Sq, tgt, src)
    omega = np.linspace(-1.0, 6.0, 400)
    eta = 0.05
    r = D.dynamics_t0(D.Sector(src), D.Program(h_src), D.Sector(tgt), D.Program(h_src), D.Program(cross), 10,
                      omega, eta)
    assert r["certified"]
    So, St = O.Sector(src), O.Sector(tgt)
    Ho = O.Program(h_src)
    w, V = np.linalg.eigh(_dense(So, Ho))
    psi = V[:, 0]
    assert abs(r["e0"] - w[0]) <= 1e-11 * abs(w[0])
    phi = St.gather(O.Program(cross), psi, col=So)
    S_or, _ = St.cf(Ho, phi, 10, omega, eta, shift=w[0], tolerance=64 * np.finfo(float).eps * _scale(h_src))
    np.testing.assert_allclose(r["S"], S_or, rtol=0, atol=1e-6 * np.abs(S_or).max())
    assert np.abs(S_or).max() > 1e-3
