"""Launch-shape tuning through the C-ABI: every shape of a kernel family gives the same y bit for bit (the row
walk with one thread per state or a warp's states compacted; the block walk with 4, 8, 16 or 32 lanes per state),
and the tuner's choices are kept, saved, loaded and bypassed as its modes say."""
import os
import tempfile

import numpy as np
import pytest

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
    from qed_spin_b200 import device as D
    yield
    D.tune_force("walk", -1)
    D.tune_force("walk_team", -1)
    D.tune_mode(1)


def _cases():
    """(name, row spec, col spec, host program): same-sector walks on 32- and 64-bit states, with and without
    the sublattice key order and with complex characters and three-body terms, and a cross-sector operator."""
    out = []
    n = 20
    h = ops.from_products(n, ops.heisenberg_products(lat.chain_bonds(n), 1.0) + ops.chiral_products(
        [(i, (i + 1) % n, (i + 2) % n) for i in range(n)], 0.3))
    out.append(("chain20_k3_chiral", lat.chain_sector(n, 10, 3), lat.chain_sector(n, 10, 3), ops.row_program(h)))
    n = 24
    h = ops.from_products(n, ops.xxz_products(lat.chain_bonds(n), 1.0, 0.7))
    spec = lat.chain_a1_flip_sector(n)
    out.append(("chain24_a1f", spec, spec, ops.row_program(h)))
    nn, nnn = lat.square_j1j2_bonds(4, 4)
    h = ops.from_products(16, ops.heisenberg_products(nn, 1.0) + ops.heisenberg_products(nnn, 0.5))
    spec = lat.square_k0_sector(4, 4, 8)
    out.append(("sq4x4", spec, spec, ops.row_program(h)))
    n = 36
    h = ops.from_products(n, ops.heisenberg_products(lat.chain_bonds(n), 1.0))
    spec = lat.chain_sector(n, 3, 1)
    out.append(("chain36_u64", spec, spec, ops.row_program(h)))
    n, m = 14, 3
    src, tgt = lat.chain_sector(n, 7, 0), lat.chain_sector(n, 7, m)
    Sq = ops.from_products(n, ops.sz_q_products(n, 2 * np.pi * m / n))
    out.append(("cross_szq", tgt, src, ops.cross_row_program(Sq, tgt, src)))
    return out


CASES = _cases()


def _bits(t):
    a = t.cpu().numpy()
    return a.view(np.uint64 if a.dtype == np.complex128 else np.uint32)


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("dtype", ["c128", "c64"])
def test_walk_shapes_agree_bit_for_bit(case, dtype):
    from qed_spin_b200 import device as D
    _, rspec, cspec, prog = case
    R, Cs = D.Sector(rspec), D.Sector(cspec)
    P = D.Program(prog)
    td = torch.complex128 if dtype == "c128" else torch.complex64
    g = torch.Generator(device="cuda").manual_seed(11)
    for nv in (1, 2, 4, 8):
        xs = [torch.randn(Cs.dim, dtype=td, device="cuda", generator=g) for _ in range(nv)]
        got = []
        for shape in ((0, 1, 2, 3, 4, 5) if nv == 1 else (0, 1)):
            D.tune_force("walk", shape)
            ys = [torch.full((R.dim,), float("nan"), dtype=td, device="cuda") for _ in range(nv)]
            D.matvec(R, Cs, P, xs, ys, dtype=dtype)
            torch.cuda.synchronize()
            got.append([_bits(y) for y in ys])
        for other in got[1:]:
            for v in range(nv):
                assert np.array_equal(got[0][v], other[v]), f"nv={nv} vector {v}"
    D.tune_force("walk", -1)


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("k", [1, 5, 40, 64])
def test_team_shapes_agree_bit_for_bit(case, k):
    from qed_spin_b200 import device as D
    _, rspec, cspec, prog = case
    R, Cs = D.Sector(rspec), D.Sector(cspec)
    P = D.Program(prog)
    g = torch.Generator(device="cuda").manual_seed(5)
    x = torch.randn(Cs.dim * k, dtype=torch.complex128, device="cuda", generator=g)
    got = []
    for shape in ((0, 1, 2, 3) if k <= 32 else (0, 1, 2)):
        D.tune_force("walk_team", shape)
        y = torch.full((R.dim * k,), float("nan"), dtype=torch.complex128, device="cuda")
        D.matvec_block(R, Cs, P, x, y, k)
        torch.cuda.synchronize()
        got.append(_bits(y))
    D.tune_force("walk_team", -1)
    for other in got[1:]:
        assert np.array_equal(got[0], other)


def test_tuner_modes_and_cache():
    from qed_spin_b200 import device as D
    _, spec, _, prog = CASES[1]
    S, P = D.Sector(spec), D.Program(prog)
    x = torch.randn(S.dim, dtype=torch.complex64, device="cuda")
    y = torch.empty_like(x)
    D.tune_clear()
    D.tune_mode(0)   # defaults only: nothing is timed or kept
    D.matvec(S, S, P, [x], [y], dtype="c64")
    assert D.tune_entries() == {}
    D.tune_mode(1)   # measure on first use: one entry with a time per candidate
    D.matvec(S, S, P, [x], [y], dtype="c64")
    ent = D.tune_entries()
    assert len(ent) == 1
    key, (pick, ms) = next(iter(ent.items()))
    assert key.startswith("walk|") and 0 <= pick < 6 and len(ms) == 6 and min(ms) > 0
    D.matvec(S, S, P, [x], [y], dtype="c64")   # a known key is not timed again
    assert D.tune_entries()[key] == (pick, ms)
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "tune.txt")
        D.tune_save(path)
        D.tune_clear()
        assert D.tune_entries() == {}
        D.tune_load(path)
        assert D.tune_entries()[key][0] == pick
        with pytest.raises(ValueError):
            D.tune_load(os.path.join(d, "missing.txt"))
    D.tune_clear()
    D.tune_mode(2)   # known choices only: an unknown key takes the default and is not kept
    D.matvec(S, S, P, [x], [y], dtype="c64")
    assert D.tune_entries() == {}
    D.tune_mode(1)
    with pytest.raises(ValueError):
        D.tune_mode(7)
