"""The device reduced-CSR lane against the reference engine's CSR and the oracle, through the C-ABI.

Bit-exact: row_ptr, columns and values of the device build against the reference's build_sector_csr
(fixtures) and the oracle's merged rows; y = A x in FP64 storage against the reference's
ReducedSymmetryCsr::spmv (fixtures `csr_y`); k-vector applies against the single apply. Tolerances,
written per test: FP32 storage 2e-6 relative; energies through the attached CSR 1e-12 relative.
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
def test_device_csr_equals_reference_csr(fixtures, name):
    d = D()
    S = d.Sector(CASE[name][1])
    P = d.Program(_prog(name))
    A = d.Csr(S, S, P)
    rp, col, val = A.download()
    assert np.array_equal(rp, fixtures[f"{name}/csr_row_ptr"])
    assert np.array_equal(col, fixtures[f"{name}/csr_col"])
    assert np.array_equal(_bits(val), _bits(fixtures[f"{name}/csr_val"]))
    info = A.info()
    assert info["nnz"] == len(col)
    # y = A x against the reference's ReducedSymmetryCsr::spmv, bit for bit
    x = _cx(fixtures[f"{name}/x"])
    y = torch.empty_like(x)
    A.matvec(x, y)
    torch.cuda.synchronize()
    assert np.array_equal(_bits(y.cpu().numpy()), _bits(fixtures[f"{name}/csr_y"]))
    # the same CSR uploaded from the host arrays applies identically
    B = d.Csr.upload(S, S, fixtures[f"{name}/csr_row_ptr"], fixtures[f"{name}/csr_col"],
                     fixtures[f"{name}/csr_val"])
    y2 = torch.empty_like(x)
    B.matvec(x, y2)
    assert np.array_equal(_bits(y2.cpu().numpy()), _bits(fixtures[f"{name}/csr_y"]))
    assert B.info()["nnz"] == info["nnz"]


@pytest.mark.parametrize("name", ["heis12_k3", "chiral13_k2", "j1j2_4x4_k0"])
def test_csr_multi_equals_single(name):
    d = D()
    S = d.Sector(CASE[name][1])
    P = d.Program(_prog(name))
    A = d.Csr(S, S, P)
    n = S.dim
    rng = np.random.default_rng(11)
    for k in (2, 3, 8, 9, 17, 40, 64):
        X = rng.normal(size=(k, n)) + 1j * rng.normal(size=(k, n))
        singles = []
        for v in range(k):
            x = _cx(X[v])
            y = torch.empty_like(x)
            A.matvec(x, y)
            singles.append(y.cpu().numpy())
        xb = _cx(X.T.reshape(-1))
        yb = torch.empty_like(xb)
        A.matvec(xb, yb, k=k)
        Yb = yb.cpu().numpy().reshape(n, k).T
        for v in range(k):
            assert np.array_equal(_bits(Yb[v]), _bits(singles[v])), (k, v)


def test_csr_fp32_storage(fixtures):
    d = D()
    name = "j1j2_4x4_k0"
    S = d.Sector(CASE[name][1])
    A = d.Csr(S, S, d.Program(_prog(name)))
    x32 = torch.from_numpy(fixtures[f"{name}/x"].astype(np.complex64)).cuda()
    y32 = torch.empty_like(x32)
    A.matvec(x32, y32, dtype="c64")
    ref = fixtures[f"{name}/csr_y"]
    err = np.abs(y32.cpu().numpy().astype(np.complex128) - ref).max() / np.abs(ref).max()
    assert err < 2e-6


@pytest.mark.parametrize("name", ["xxz16_a1f", "j1j2_4x4_k0"])
def test_attached_csr_serves_the_program(fixtures, name):
    """With the CSR attached, qb_matvec, the block apply and the k = 1 lane run on it."""
    d = D()
    S = d.Sector(CASE[name][1])
    P = d.Program(_prog(name))
    A = d.Csr(S, S, P)
    A.attach(P)
    x = _cx(fixtures[f"{name}/x"])
    y = torch.empty_like(x)
    d.matvec(S, S, P, [x], [y])
    assert np.array_equal(_bits(y.cpu().numpy()), _bits(fixtures[f"{name}/csr_y"]))
    yh = d.matvec_host(S, S, P, fixtures[f"{name}/x"])
    assert np.array_equal(_bits(yh), _bits(fixtures[f"{name}/csr_y"]))
    re0 = fixtures[f"{name}/e0"][0]
    r = d.eigs_lowest(S, P)
    assert r["converged"] and abs(r["e0"] - re0) <= 1e-12 * abs(re0)
    r32 = d.eigs_lowest(S, P, dtype="c64", refine=True)
    assert r32["converged"] and abs(r32["e0"] - re0) <= 1e-10 * abs(re0)
    # detached: back to the row walk (the gather's y)
    d.detach_csr(P)
    d.matvec(S, S, P, [x], [y])
    assert np.array_equal(_bits(y.cpu().numpy()), _bits(fixtures[f"{name}/y"]))


def test_cross_sector_csr_matches_oracle():
    d = D()
    N, m = 12, 3
    q = 2 * np.pi * m / N
    src, tgt = lat.chain_sector(N, 6, 0), lat.chain_sector(N, 6, m)
    prog = ops.cross_row_program(ops.from_products(N, ops.sz_q_products(N, q)), tgt, src)
    rs, cs = d.Sector(tgt), d.Sector(src)
    A = d.Csr(rs, cs, d.Program(prog))
    rp, col, val = A.download()
    orp, ocol, oval = O.Sector(tgt).csr(O.Program(prog), col=O.Sector(src))
    assert np.array_equal(rp, orp) and np.array_equal(col, ocol)
    assert np.array_equal(_bits(val), _bits(oval))


def _trivial(n, n_up):
    return lat.SectorSpec(n, n_up, np.arange(n, dtype=np.int32)[None, :], np.ones(1, np.complex128))


@pytest.mark.parametrize("n,expect", [(16, 2), (20, -1)], ids=["u16_ids", "whole_values"])
def test_dictionary_widths(n, expect):
    """Random fields make the diagonal distinct per state: u16 ids up to 65536 values, whole values beyond."""
    d = D()
    rng = np.random.default_rng(n)
    spec = _trivial(n, n // 2)
    prods = ops.heisenberg_products(lat.chain_bonds(n)) + [("z", (i,), complex(rng.uniform(-1, 1), 0.0))
                                                              for i in range(n)]
    prog = ops.row_program(ops.from_products(n, prods))
    S = d.Sector(spec)
    A = d.Csr(S, S, d.Program(prog))
    rp, col, val = A.download()
    orp, ocol, oval = O.Sector(spec).csr(O.Program(prog))
    assert np.array_equal(rp, orp) and np.array_equal(col, ocol)
    assert np.array_equal(_bits(val), _bits(oval))
    nd = A.info()["n_dict"]
    if expect == -1:
        assert nd == -1
    else:
        assert 256 < nd <= 65536


def test_byte_budget_is_enforced():
    d = D()
    name = "j1j2_4x4_k0"
    S = d.Sector(CASE[name][1])
    P = d.Program(_prog(name))
    from qed_spin_b200._lib import ResourceLimit
    with pytest.raises(ResourceLimit):
        d.Csr(S, S, P, max_bytes=1024)


def test_empty_sector_csr():
    d = D()
    spec = lat.chain_sector(10, 0, 3)   # no representative survives
    S = d.Sector(spec)
    assert S.dim == 0
    A = d.Csr(S, S, d.Program(ops.row_program(ops.from_products(10, ops.heisenberg_products(lat.chain_bonds(10))))))
    assert A.info()["nnz"] == 0


@pytest.mark.parametrize("case", ["chain24", "chain20k3", "sq24"])
def test_csr_fp32_storage_apply(case):
    """The FP32-storage CSR apply against the FP64 apply of the same complex64-rounded x: the rows differ only by the
    FP32 rounding of y and the order of the FP64 sums, within 1e-6 of max |y|. The chains (12 to 25 entries a row)
    take the thread-per-row kernel, the 6x4 J1-J2 torus (about 49 a row) the four-lanes-per-row kernel."""
    d = D()
    if case == "sq24":
        nn, nnn = lat.square_j1j2_bonds(6, 4)
        N = 24
        spec = lat.square_k0_sector(6, 4, 12)
        prods = ops.heisenberg_products(nn, 1.0) + ops.heisenberg_products(nnn, 0.5)
    else:
        N, n_up, k = (24, 12, 0) if case == "chain24" else (20, 9, 3)
        spec = lat.chain_sector(N, n_up, k)
        prods = ops.xxz_products(lat.chain_bonds(N), 1.0, 0.7) + ops.zeeman_z_products(N, 0.1)
    S = d.Sector(spec)
    A = d.Csr(S, S, d.Program(ops.row_program(ops.from_products(N, prods))))
    per_row = A.info()["nnz"] / S.dim
    assert (per_row >= 32) == (case == "sq24")
    rng = np.random.default_rng(3)
    x = (rng.normal(size=S.dim) + 1j * rng.normal(size=S.dim)).astype(np.complex64)
    x32 = torch.from_numpy(x).cuda()
    y32 = torch.empty_like(x32)
    A.matvec(x32, y32, dtype="c64")
    x64 = x32.to(torch.complex128)
    y64 = torch.empty_like(x64)
    A.matvec(x64, y64)
    ref = y64.cpu().numpy()
    err = np.abs(y32.cpu().numpy().astype(np.complex128) - ref).max() / np.abs(ref).max()
    assert err < 1e-6
