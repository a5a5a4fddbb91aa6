"""Parity at the benchmark sizes: the device path against the reference engine's own CPU code (oracle/_ref,
compiled from the reference sources) on the very sectors bench.py measures, through the C-ABI.

- XXZ chain N = 32 (J = 1, Delta = 0.7), S^z = 0, k = 0, reflection-even, flip-even (4,707,969 states): the
  representatives and 1/norms, the device-built merged CSR (row_ptr, columns, values) and y = H x in FP64
  storage, through the CSR against ReducedSymmetryCsr::spmv and through the walk against sector_gather, all
  bit for bit.
- 6x6 J1-J2 (J2 = 0.5), S^z = 0, momentum (0, 0), translations only (252,091,362 states): the dimension (also
  by Burnside's count), all representatives and 1/norms bit for bit against the reference's own orbit scan,
  and 2^14 strided rows plus the first and last rows of y = H x (the device walk, FP64) bit for bit against
  the reference's row walk (for_each_sector_entry) on the same x.
- The chain-32 sector's two lowest levels (the k > 1 lane, FP64 and FP32 storage + FP64 refinement) against the
  reference engine's krylov_schur_kernel on its host CSR (1e-9 of the coupling scale).
- XXZ chain N = 24 in a field (the batched FTLM workload): three of its blocks, small to largest, 40 samples,
  depth 100, against the reference engine's ftlm_kernel per block (FP64 storage 1e-8 relative).
- The served stream's model (Heisenberg + scalar chirality, random J, K) through the request server: eigs
  levels against a dense solve of the oracle's block (1e-9 of the coupling scale); T = 0 S^z(q) dynamics: E0
  against the dense solve and the spectrum against the oracle's continued fraction from the lane's own certified
  ground state (depth 10, 1e-6 of max S).
"""
import math

import numpy as np
import pytest

from oracle import oracle as O
from oracle import ref as R
from qed_spin_b200 import lattice as lat
from qed_spin_b200 import operators as ops

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.fail("a GPU test ran without a CUDA device")
    if not R.available():
        pytest.fail("the reference engine's CPU library (oracle/_ref) is not built")
    from qed_spin_b200 import build
    build.build()
    import os
    R.set_threads(os.cpu_count() or 1)


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint64)


def _ref_sector(spec):
    return R.Sector(spec.n_sites, spec.n_up, spec.perms, spec.chars, flips=spec.flips, slc_mode=-1)


def _x(n, seed):
    rng = np.random.default_rng(seed)
    return rng.normal(size=n) + 1j * rng.normal(size=n)


def test_chain32_a1_flip_bit_exact():
    from qed_spin_b200 import device as D
    N = 32
    spec = lat.chain_a1_flip_sector(N)
    prods = ops.xxz_products(lat.chain_bonds(N), 1.0, 0.7)
    S = D.Sector(spec)
    rs = _ref_sector(spec)
    assert S.dim == rs.dim == 4707969
    reps, inv = S.reps()
    rreps, rinv = rs.reps()
    assert np.array_equal(reps, rreps)
    assert np.array_equal(_bits(inv), _bits(rinv))
    del rreps, rinv
    rp = R.Operator(N, prods).row_program()
    x = _x(S.dim, 11)
    # the merged CSR, built on the device from the walk, against build_sector_csr
    P = D.Program(ops.row_program(ops.from_products(N, prods)))
    A = D.Csr(S, S, P)
    row_ptr, col, val = A.download()
    r_ptr, r_col, r_val, r_y = rs.csr(rp, x)
    assert np.array_equal(row_ptr, r_ptr)
    assert np.array_equal(col, r_col)
    assert np.array_equal(_bits(val), _bits(r_val))
    del row_ptr, col, val, r_ptr, r_col, r_val
    xd = torch.from_numpy(x).cuda()
    yd = torch.empty_like(xd)
    A.matvec(xd, yd)
    torch.cuda.synchronize()
    assert np.array_equal(_bits(yd.cpu().numpy()), _bits(r_y))      # ReducedSymmetryCsr::spmv
    A.close()
    # the on-the-fly walk against the reference's sector_gather
    D.matvec(S, S, P, [xd], [yd])
    torch.cuda.synchronize()
    assert np.array_equal(_bits(yd.cpu().numpy()), _bits(rs.gather(rp, x)))
    # the host entry point: its 75 MB input goes through the pinned slots in 16 MB chunks (the last one partial)
    assert np.array_equal(_bits(D.matvec_host(S, S, P, x)), _bits(yd.cpu().numpy()))


def test_chain32_k2_levels_against_reference():
    """The two lowest levels of the chain-32 sector: the k > 1 lane on the device CSR in FP64 storage, and in FP32
    storage with the FP64 refinement, against the reference engine's own krylov_schur_kernel on its host CSR
    (1e-9 of the coupling scale)."""
    from qed_spin_b200 import device as D
    N = 32
    spec = lat.chain_a1_flip_sector(N)
    prods = ops.xxz_products(lat.chain_bonds(N), 1.0, 0.7)
    prog = ops.row_program(ops.from_products(N, prods))
    S, P = D.Sector(spec), D.Program(prog)
    A = D.Csr(S, S, P)
    A.attach(P)
    ev, cv, _ = _ref_sector(spec).ks_lowest(R.Operator(N, prods).row_program(), 2, use_csr=True)
    assert cv
    sc = float(np.abs(np.asarray(prog.term_coeff)).sum())
    for dtype in ("c128", "c64"):
        r = D.eigs(S, P, 2, dtype=dtype, refine=True)
        assert r["converged"], dtype
        np.testing.assert_allclose(r["values"], ev, rtol=0, atol=1e-9 * sc, err_msg=dtype)
    A.close()


def _burnside_sq(Lx, Ly, n_up):
    """Orbits of the n_up-up states of an Lx x Ly torus under its translations: (1/|G|) sum_g fix(g); a
    translation (a, b) splits the sites into cycles of one length l, and fixes C(N/l, n_up/l) states."""
    N = Lx * Ly
    tot = 0
    for a in range(Lx):
        for b in range(Ly):
            l = math.lcm(Lx // math.gcd(a, Lx), Ly // math.gcd(b, Ly))
            if n_up % l == 0:
                tot += math.comb(N // l, n_up // l)
    return tot // (Lx * Ly)


def test_square6x6_j1j2_k0_at_size():
    from qed_spin_b200 import device as D
    Lx = Ly = 6
    nn, nnn = lat.square_j1j2_bonds(Lx, Ly)
    prods = ops.heisenberg_products(nn, 1.0) + ops.heisenberg_products(nnn, 0.5)
    spec = lat.square_k0_sector(Lx, Ly, 18)
    S = D.Sector(spec)
    assert S.dim == _burnside_sq(Lx, Ly, 18) == 252091362
    rs = _ref_sector(spec)
    assert rs.dim == S.dim
    reps, inv = S.reps()
    rreps, rinv = rs.reps()
    assert np.array_equal(reps, rreps)
    assert np.array_equal(_bits(inv), _bits(rinv))
    del reps, inv, rreps, rinv
    # y = H x on the device (the walk, FP64 storage) against the reference's row walk on sampled rows
    n = S.dim
    x = _x(n, 5)
    P = D.Program(ops.row_program(ops.from_products(36, prods)))
    xd = torch.from_numpy(x).cuda()
    yd = torch.empty_like(xd)
    D.matvec(S, S, P, [xd], [yd])
    torch.cuda.synchronize()
    rows = np.unique(np.concatenate([np.linspace(0, n - 1, 1 << 14).astype(np.uint64),
                                     np.arange(64, dtype=np.uint64), n - 1 - np.arange(64, dtype=np.uint64)]))
    y_dev = yd[torch.from_numpy(rows.astype(np.int64)).cuda()].cpu().numpy()
    del xd, yd
    rp = R.Operator(36, prods).row_program()
    y_ref = rs.gather_rows(rp, x, rows)
    assert np.array_equal(_bits(y_dev), _bits(y_ref))


def test_ftlm_n24_blocks_against_reference():
    from qed_spin_b200 import device as D
    N, seed = 24, 20240601
    betas = 1.0 / np.linspace(0.1, 4.0, 40)
    prods = ops.xxz_products(lat.chain_bonds(N), 1.0, 0.5) + ops.zeeman_z_products(N, 0.1)
    specs = [lat.chain_sector(N, n_up, k) for n_up, k in [(12, 0), (9, 7), (4, 3)]]
    secs = [D.Sector(s) for s in specs]
    assert secs[0].dim == 112720
    P = D.Program(ops.row_program(ops.from_products(N, prods)))
    r = D.ftlm_blocks(secs, P, 40, 100, seed, betas, dtype="c128")
    rp = R.Operator(N, prods).row_program()
    for b, spec in enumerate(specs):
        c = _ref_sector(spec).ftlm(rp, 40, 100, seed, betas)
        for key in ("lnZ", "E", "V"):
            ref = np.asarray(c[key])
            np.testing.assert_allclose(r[key][b], ref, rtol=1e-8, atol=1e-8 * max(np.abs(ref).max(), 1e-3),
                                       err_msg=f"block {b} {key}")


def _dense(So, Po, col=None):
    col = So if col is None else col
    M = np.zeros((So.dim, col.dim), np.complex128)
    for j in range(col.dim):
        e = np.zeros(col.dim, np.complex128)
        e[j] = 1.0
        M[:, j] = So.gather(Po, e, col=col)
    return M


def test_served_chiral_requests_against_oracle():
    """Requests of the served stream's model (Heisenberg + scalar chirality, random J and K) through the server.
    eigs: the levels against a dense solve of the oracle's block (1e-9 of the coupling scale). T = 0 S^z(q)
    dynamics: E0 against the dense solve (1e-11 relative), and the spectrum against the oracle's continued fraction
    from phi = S^z(q) psi0 with psi0 the lane's own certified ground state (qb_ground_state on the same reduced-CSR
    lane the server attaches; 1e-6 of max S). The spectrum is not compared with the one from the dense ground state:
    on these chains the depth-10 recurrence from phi amplifies a change of psi0 about 1e6 times (a global phase of
    phi alone moves a dense numpy Lanczos by 2e-10), so a ground state certified to 1e-9 of the scale moves S by up
    to a few 1e-3."""
    from qed_spin_b200 import device as D
    rng = np.random.default_rng(29)
    omega = np.linspace(-0.5, 6.0, 400)
    reqs = []
    for N, kind in [(16, "eigs"), (18, "dynamics"), (17, "eigs"), (16, "dynamics")]:
        J, K = float(rng.uniform(0.5, 1.5)), float(rng.uniform(0.0, 0.3))
        prods = ops.heisenberg_products(lat.chain_bonds(N), J) + ops.chiral_products(
            [(a, (a + 1) % N, (a + 2) % N) for a in range(N)], K)
        H = ops.from_products(N, prods)
        h = ops.row_program(H)
        if kind == "eigs":
            reqs.append({"kind": kind, "spec": lat.chain_sector(N, N // 2, int(rng.integers(0, N))), "h": h,
                         "k": int(rng.integers(2, 5))})
        else:
            m = int(rng.integers(1, N))
            src, tgt = lat.chain_sector(N, N // 2, 0), lat.chain_sector(N, N // 2, m)
            op = ops.cross_row_program(ops.from_products(N, ops.sz_q_products(N, 2 * np.pi * m / N)), tgt, src)
            reqs.append({"kind": kind, "src": src, "tgt": tgt, "h": h, "op": op})
    srv = D.Server(max_active=4)
    tickets = []
    for r in reqs:
        if r["kind"] == "eigs":
            tickets.append(srv.submit_eigs(r["spec"], r["h"], r["k"]))
        else:
            tickets.append(srv.submit_dynamics(r["src"], r["tgt"], r["h"], r["op"], 10, omega, 0.05))
    got = [srv.wait(t) for t in tickets]
    srv.close()
    for r, g in zip(reqs, got):
        sc = float(np.abs(np.asarray(r["h"].term_coeff)).sum())
        Ho = O.Program(r["h"])
        if r["kind"] == "eigs":
            So = O.Sector(r["spec"])
            w = np.linalg.eigvalsh(_dense(So, Ho))[: r["k"]]
            assert g["converged"]
            np.testing.assert_allclose(g["values"], w, rtol=0, atol=1e-9 * sc)
        else:
            So, St = O.Sector(r["src"]), O.Sector(r["tgt"])
            w = np.linalg.eigvalsh(_dense(So, Ho))
            assert g["converged"] and abs(g["e0"] - w[0]) <= 1e-11 * abs(w[0])
            Ss, Ph = D.Sector(r["src"]), D.Program(r["h"])
            A = D.Csr(Ss, Ss, Ph)
            A.attach(Ph)
            gs = D.ground_state(Ss, Ph)
            assert gs["certified"] and gs["e0"] == g["e0"]
            phi = St.gather(O.Program(r["op"]), gs["vector"], col=So)
            S_or, _ = St.cf(Ho, phi, 10, omega, 0.05, shift=g["e0"], tolerance=64 * np.finfo(float).eps * sc)
            np.testing.assert_allclose(g["S"], S_or, rtol=0, atol=1e-6 * np.abs(S_or).max())
            A.close()
