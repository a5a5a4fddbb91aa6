"""Parity of the CUDA path with the oracle and the reference engine's fixtures, through the C-ABI.

Bit-exact: representatives, 1/norms, indices, y = H x in FP64 storage (the device sums each row in group
order with the host's complex arithmetic), multi-vector and block applies against the single apply.
Tolerances, written per test: FP32 storage 2e-6 relative; Lanczos scalars 1e-12 over the first steps;
energies 1e-12 relative (FP64) and 1e-10 after FP32-storage + FP64 refinement; FTLM curves 1e-8.
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


def D():
    from qed_spin_b200 import device
    return device


CASE = {c[0]: c for c in CASES}


def _prog(name):
    _, spec, prods = CASE[name]
    return ops.row_program(ops.from_products(spec.n_sites, prods))


def _cx(a):
    return torch.from_numpy(np.ascontiguousarray(a, np.complex128)).cuda()


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint64)


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("lookup", [0, 1, 2, 4])   # auto (the compact hash), rank, buckets, wide hash
def test_sector_and_matvec_bit_exact(fixtures, name, lookup):
    d = D()
    spec = CASE[name][1]
    S = d.Sector(spec, lookup=lookup)
    assert S.info()["lookup"] == {0: "hash8", 1: "rank", 2: "buckets", 4: "hash"}[lookup]
    reps, inv = S.reps()
    assert np.array_equal(reps, fixtures[f"{name}/reps"])
    assert np.array_equal(_bits(inv), _bits(fixtures[f"{name}/inv_norms"]))
    P = d.Program(_prog(name))
    x = _cx(fixtures[f"{name}/x"])
    y = torch.empty_like(x)
    d.matvec(S, S, P, [x], [y])
    torch.cuda.synchronize()
    assert np.array_equal(_bits(y.cpu().numpy()), _bits(fixtures[f"{name}/y"]))
    # the host-pointer twin
    yh = d.matvec_host(S, S, P, fixtures[f"{name}/x"])
    assert np.array_equal(_bits(yh), _bits(fixtures[f"{name}/y"]))


@pytest.mark.parametrize("name", ["heis12_k3", "xxz16_a1f", "chiral13_k2"])
def test_multi_and_block_equal_single(name):
    d = D()
    spec = CASE[name][1]
    S = d.Sector(spec)
    P = d.Program(_prog(name))
    n = S.dim
    rng = np.random.default_rng(7)
    for k in (1, 3, 5, 9, 13, 40):
        X = rng.normal(size=(k, n)) + 1j * rng.normal(size=(k, n))
        singles = []
        for v in range(k):
            x = _cx(X[v])
            y = torch.empty_like(x)
            d.matvec(S, S, P, [x], [y])
            singles.append(y.cpu().numpy())
        xs = [_cx(X[v]) for v in range(k)]
        ys = [torch.empty_like(x) for x in xs]
        d.matvec(S, S, P, xs, ys)
        for v in range(k):
            assert np.array_equal(_bits(ys[v].cpu().numpy()), _bits(singles[v])), (k, v)
        xb = _cx(X.T.reshape(-1))
        yb = torch.empty_like(xb)
        d.matvec_block(S, S, P, xb, yb, k)
        Yb = yb.cpu().numpy().reshape(n, k).T
        for v in range(k):
            assert np.array_equal(_bits(Yb[v]), _bits(singles[v])), ("block", k, v)


def test_fp32_storage_matvec(fixtures):
    d = D()
    name = "j1j2_4x4_k0"
    S = d.Sector(CASE[name][1])
    P = d.Program(_prog(name))
    x = fixtures[f"{name}/x"]
    x32 = torch.from_numpy(x.astype(np.complex64)).cuda()
    y32 = torch.empty_like(x32)
    d.matvec(S, S, P, [x32], [y32], dtype="c64")
    ref = fixtures[f"{name}/y"]
    err = np.abs(y32.cpu().numpy().astype(np.complex128) - ref).max() / np.abs(ref).max()
    assert err < 2e-6


def test_index_and_projection_matches_oracle():
    d = D()
    spec = lat.chain_sector(14, 7, 3)
    S = d.Sector(spec)
    So = O.Sector(spec)
    rng = np.random.default_rng(1)
    states = []
    while len(states) < 400:
        s = int(rng.integers(0, 1 << 14))
        states.append(s)
    idx, proj = S.index_and_projection(states)
    for s, i, p in zip(states, idx, proj):
        k, q = So.index_and_projection(s)
        assert k == i
        if k >= 0:
            assert q == p


@pytest.mark.parametrize("spec", [
    lat.chain_sector(20, 10, 0),                          # config 1's sector: 9,252 representatives
    lat.chain_sector(24, 12, 5),                          # the sublattice key order engaged (L=12, m=2)
    lat.chain_a1_flip_sector(24),                         # reflections + spin flip, key order engaged
    lat.square_k0_sector(6, 4, 12),                       # 2D translations
    lat.chain_sector(10, 0, 0), lat.chain_sector(10, 10, 0), lat.chain_sector(10, 0, 3),   # edge sectors
], ids=["chain20_k0", "chain24_k5", "chain24_a1f", "sq6x4_k0", "n_up0", "n_upN", "empty"])
def test_device_enumeration_matches_oracle(spec):
    d = D()
    S = d.Sector(spec)
    So = O.Sector(spec)
    r1, i1 = S.reps()
    r2, i2 = So.reps()
    assert np.array_equal(r1, r2)
    assert np.array_equal(_bits(i1), _bits(i2))
    info = S.info()
    sl = So.sublattice()
    assert (info["slc_L"], info["slc_m"]) == ((sl["L"], sl["m"]) if sl else (0, 0))


def test_cross_sector_apply():
    """S^z(q) from the k0 = 0 sector to k0 + q: rows of the target, columns of the source."""
    d = D()
    N, m = 12, 3
    q = 2 * np.pi * m / N
    src = lat.chain_sector(N, 6, 0)
    tgt = lat.chain_sector(N, 6, m)
    Sq = ops.from_products(N, ops.sz_q_products(N, q))
    prog = ops.cross_row_program(Sq, tgt, src)
    rs, cs = d.Sector(tgt), d.Sector(src)
    P = d.Program(prog)
    ro, co = O.Sector(tgt), O.Sector(src)
    x = np.random.default_rng(2).normal(size=cs.dim) + 0j
    y_or = ro.gather(O.Program(prog), x, col=co)
    xd = _cx(x)
    yd = torch.zeros(rs.dim, dtype=torch.complex128, device="cuda")
    d.matvec(rs, cs, P, [xd], [yd])
    assert np.array_equal(_bits(yd.cpu().numpy()), _bits(y_or))
    assert np.abs(y_or).max() > 0.01


@pytest.mark.parametrize("name", NAMES)
def test_lanczos_and_lowest_level(fixtures, name):
    d = D()
    S = d.Sector(CASE[name][1])
    P = d.Program(_prog(name))
    a, b = d.lanczos(S, P, fixtures[f"{name}/x"], 40)
    ra, rb = fixtures[f"{name}/lz_alpha"], fixtures[f"{name}/lz_beta"]
    assert len(a) == len(ra)
    np.testing.assert_allclose(a[:10], ra[:10], rtol=0, atol=1e-12)
    np.testing.assert_allclose(b[:11], rb[:11], rtol=0, atol=1e-12)
    r = d.eigs_lowest(S, P)
    re0 = fixtures[f"{name}/e0"][0]
    assert r["converged"] and abs(r["e0"] - re0) <= 1e-12 * abs(re0)
    r32 = d.eigs_lowest(S, P, dtype="c64", refine=True)
    assert r32["converged"] and abs(r32["e0"] - re0) <= 1e-10 * abs(re0)


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("dtype", ["c128", "c64"])
def test_ftlm_and_cf(fixtures, name, dtype):
    d = D()
    S = d.Sector(CASE[name][1])
    P = d.Program(_prog(name))
    betas = 1.0 / np.linspace(0.1, 4.0, 40)
    f = d.ftlm(S, P, 8, 60, 20240601, betas, dtype=dtype)
    tol = 1e-8 if dtype == "c128" else 1e-6   # FP32 storage: the curves move by ~3e-8 relative
    for k in ("lnZ", "E", "V"):
        ref = fixtures[f"{name}/ftlm_{k}"]
        np.testing.assert_allclose(f[k], ref, rtol=tol, atol=tol * np.abs(ref).max())
    omega = np.linspace(-1.0, 6.0, 64)
    # depth 10, inside the orthogonal regime of every case: the device equals the oracle to 1e-8 of max S
    # (deeper, the recurrence without reorthogonalisation loses orthogonality on these 76-822-state
    # sectors and amplifies the summation-order differences of the reductions)
    So = O.Sector(CASE[name][1])
    Sw, sh = d.cf(S, P, fixtures[f"{name}/x"], 10, omega, 0.05)
    Sr, shr = So.cf(O.Program(_prog(name)), fixtures[f"{name}/x"], 10, omega, 0.05)
    assert abs(sh - shr) <= 1e-9
    np.testing.assert_allclose(Sw, Sr, rtol=0, atol=1e-8 * np.abs(Sr).max())
    # depth 80, past the loss of orthogonality: the curve is then chaotic in the reduction order, but the
    # energy shift (the tridiagonal's lowest value, a converged extreme) equals the reference engine's
    Sw, sh = d.cf(S, P, fixtures[f"{name}/x"], 80, omega, 0.05)
    assert abs(sh - fixtures[f"{name}/cf_shift"][0]) <= 1e-9


def test_malformed_program_is_rejected():
    d = D()
    from qed_spin_b200.operators import Program
    p = _prog("heis12_k0")
    bad = Program(p.group_flip[::-1].copy(), p.group_setbits, p.group_vbegin, p.vsub_val, p.vsub_tbegin,
                  p.term_sign, p.term_coeff)
    with pytest.raises(ValueError):
        d.Program(bad)


def test_chain20_lowest_matches_oracle():
    d = D()
    spec = lat.chain_sector(20, 10, 0)
    prog = ops.row_program(ops.from_products(20, ops.heisenberg_products(lat.chain_bonds(20))))
    e_or, it_or, cv = O.Sector(spec).scan_lowest(O.Program(prog))
    S = d.Sector(spec)
    P = d.Program(prog)
    r = d.eigs_lowest(S, P)
    assert cv and r["converged"]
    assert abs(r["e0"] - e_or) <= 1e-12 * abs(e_or)
    assert abs(r["iters"] - it_or) <= 1
