"""Batched FTLM over many blocks against the oracle, through the C-ABI.

The blocks are every (S^z, momentum) sector of an XXZ chain in a field: the decomposition the thermal driver
samples (config 3 at N = 12). Each block's curves are checked against the oracle's FTLM of that block with the
call's base seed (tolerances written per test: 1e-8 relative for FP64 storage, 1e-6 for FP32), and the combined
thermodynamics against the oracle's log-space combine.
"""
import numpy as np
import pytest

from oracle import oracle as O
from qed_spin_b200 import lattice as lat
from qed_spin_b200 import operators as ops

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

N = 12
SEED = 20240601
BETAS = 1.0 / np.linspace(0.1, 4.0, 40)


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.fail("a GPU test ran without a CUDA device")
    from qed_spin_b200 import build
    build.build()


def _blocks():
    specs = []
    for n_up in range(N + 1):
        for k in range(N):
            spec = lat.chain_sector(N, n_up, k)
            if O.Sector(spec).dim > 0:
                specs.append(spec)
    prods = ops.xxz_products(lat.chain_bonds(N), 1.0, 0.5) + ops.zeeman_z_products(N, 0.1)
    return specs, ops.row_program(ops.from_products(N, prods))


@pytest.fixture(scope="module")
def oracle_curves():
    specs, prog = _blocks()
    P = O.Program(prog)
    curves = [O.Sector(s).ftlm(P, 8, 30, SEED, BETAS) for s in specs]
    return specs, prog, curves


# pack: the largest block the packed kernel runs whole (QB_FTLM_PACK_DIM; "0" sends every block down the
# per-block path, "40" splits the N = 12 blocks between the two)
@pytest.mark.parametrize("dtype,use_csr,pack", [("c128", True, "4096"), ("c128", True, "40"), ("c128", True, "0"),
                                                ("c128", False, "4096"), ("c64", True, "4096"), ("c64", True, "0")])
def test_blocks_match_oracle(oracle_curves, monkeypatch, dtype, use_csr, pack):
    from qed_spin_b200 import device as D
    monkeypatch.setenv("QB_FTLM_PACK_DIM", pack)
    specs, prog, curves = oracle_curves
    secs = [D.Sector(s) for s in specs]
    P = D.Program(prog)
    r = D.ftlm_blocks(secs, P, 8, 30, SEED, BETAS, dtype=dtype, use_csr=use_csr)
    tol = 1e-8 if dtype == "c128" else 1e-6   # FP32 storage: the curves move by ~3e-8 relative
    assert len(curves) == r["lnZ"].shape[0] > 100
    for b, c in enumerate(curves):
        for key in ("lnZ", "E", "V"):
            ref = np.asarray(c[key])
            np.testing.assert_allclose(r[key][b], ref, rtol=tol, atol=tol * max(np.abs(ref).max(), 1e-3),
                                       err_msg=f"block {b} {key}")
        assert abs(r["e_min"][b] - c["e_min"]) <= tol * max(1.0, abs(c["e_min"]))
    tot = O.combine_blocks(curves, BETAS)
    for key in ("lnZ", "E", "C", "S", "F"):
        np.testing.assert_allclose(r["total"][key], tot[key], rtol=tol, atol=tol * np.abs(tot[key]).max(),
                                   err_msg=key)


def _lcg_seeds(seed, n):
    """The thermal driver's block seeds: one step of its 64-bit LCG before each sampled block
    (src/engine/thermal.cpp:470-471)."""
    out = []
    for _ in range(n):
        seed = (seed * 6364136223846793005 + 1442695040888963407) % (1 << 64)
        out.append(seed)
    return out


@pytest.mark.parametrize("pack", ["4096", "0"])
def test_per_block_seeds_match_the_driver_loop(monkeypatch, pack):
    """QB_SEED_PER_BLOCK: block b draws from the seed the reference's thermal driver gives it (its LCG stepped
    once per sampled block, in the order given); every block's curves equal the oracle's FTLM of that block from
    that seed within 1e-10 relative (FP64 storage), and so do the combined thermodynamics."""
    from qed_spin_b200 import device as D
    monkeypatch.setenv("QB_FTLM_PACK_DIM", pack)
    specs, prog = _blocks()
    seeds = _lcg_seeds(SEED, len(specs))
    P = O.Program(prog)
    curves = [O.Sector(s).ftlm(P, 8, 30, sd, BETAS) for s, sd in zip(specs, seeds)]
    r = D.ftlm_blocks([D.Sector(s) for s in specs], D.Program(prog), 8, 30, SEED, BETAS, per_block_seeds=True)
    tol = 1e-10
    for b, c in enumerate(curves):
        for key in ("lnZ", "E", "V"):
            ref = np.asarray(c[key])
            np.testing.assert_allclose(r[key][b], ref, rtol=tol, atol=tol * max(np.abs(ref).max(), 1e-3),
                                       err_msg=f"block {b} {key}")
    tot = O.combine_blocks(curves, BETAS)
    for key in ("lnZ", "E", "C", "S", "F"):
        np.testing.assert_allclose(r["total"][key], tot[key], rtol=tol, atol=tol * np.abs(tot[key]).max(),
                                   err_msg=key)
    # a block's draws differ from the shared-stream mode's (distinct streams), as the driver's do
    shared = D.ftlm_blocks([D.Sector(s) for s in specs[:3]], D.Program(prog), 8, 30, SEED, BETAS)
    assert not np.array_equal(shared["lnZ"][2], r["lnZ"][2])


def test_combine_matches_oracle(oracle_curves):
    """The C combine equals the oracle's restatement of the thermal driver's (1e-13 relative)."""
    from qed_spin_b200 import device as D
    _, _, curves = oracle_curves
    lnZ = np.stack([c["lnZ"] for c in curves])
    E = np.stack([c["E"] for c in curves])
    V = np.stack([c["V"] for c in curves])
    w = np.linspace(1.0, 2.0, len(curves))
    got = D.thermal_combine(lnZ, E, V, BETAS, weights=w)
    ref = O.combine_blocks(curves, BETAS, weights=w)
    for key in got:
        np.testing.assert_allclose(got[key], ref[key], rtol=1e-13, atol=1e-13 * np.abs(ref[key]).max())


def test_one_block_call_equals_batch(oracle_curves):
    """qb_ftlm on a block equals that block inside the batch (the same start vectors and recurrence)."""
    from qed_spin_b200 import device as D
    specs, prog, _ = oracle_curves
    pick = [len(specs) // 2, len(specs) // 3]
    secs = [D.Sector(specs[i]) for i in pick]
    P = D.Program(prog)
    r = D.ftlm_blocks(secs, P, 8, 30, SEED, BETAS, use_csr=False)
    for j, s in enumerate(secs):
        one = D.ftlm(s, P, 8, 30, SEED, BETAS)
        for key in ("lnZ", "E", "V"):
            np.testing.assert_array_equal(one[key], r[key][j])


@pytest.mark.parametrize("dtype,tol", [("c128", 1e-10), ("c64", 1e-5)])
def test_packed_blocks_equal_per_block_path(monkeypatch, dtype, tol):
    """Blocks of a few hundred states run whole by one CTA each give the curves of the per-block path (the two
    differ only in the order of their inner-product sums): 1e-10 relative in FP64 storage, 1e-5 in FP32."""
    from qed_spin_b200 import device as D
    n = 16
    prods = ops.xxz_products(lat.chain_bonds(n), 1.0, 0.5) + ops.zeeman_z_products(n, 0.1)
    P = D.Program(ops.row_program(ops.from_products(n, prods)))
    secs = [D.Sector(lat.chain_sector(n, n_up, k)) for n_up, k in [(8, 0), (8, 3), (7, 5), (5, 1), (2, 2), (1, 0)]]
    assert max(s.dim for s in secs) > 700
    out = {}
    for pack in ("4096", "0"):
        monkeypatch.setenv("QB_FTLM_PACK_DIM", pack)
        out[pack] = D.ftlm_blocks(secs, P, 12, 40, SEED, BETAS, dtype=dtype)
    for key in ("lnZ", "E", "V"):
        a, b = out["4096"][key], out["0"][key]
        np.testing.assert_allclose(a, b, rtol=tol, atol=tol * np.abs(b).max(), err_msg=key)
