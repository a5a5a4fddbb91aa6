"""The restated oracle pinned against the reference: its golden suite's recorded energies, a textbook
ground-state energy, and outputs of the reference engine itself (tests/golden/fixtures.npz)."""
import numpy as np
import pytest

from cases import CASES, NAMES
from conftest import host_program
from oracle import oracle as O
from qed_spin_b200 import lattice as lat
from qed_spin_b200 import operators as ops


def _spec(name):
    return dict((c[0], c[1]) for c in CASES)[name]


def _prods(name):
    return dict((c[0], c[2]) for c in CASES)[name]


@pytest.mark.parametrize("name", NAMES)
def test_program_compile_matches_reference(fixtures, name):
    """The host operator algebra compiles the reference's row program bit for bit."""
    spec = _spec(name)
    p = ops.row_program(ops.from_products(spec.n_sites, _prods(name)))
    for k in ("group_flip", "group_setbits", "group_vbegin", "vsub_val", "vsub_tbegin", "term_sign"):
        ref = fixtures[f"{name}/prog/{k}"]
        assert np.array_equal(np.asarray(getattr(p, k)).astype(ref.dtype), ref), k
    assert np.array_equal(p.term_coeff.view(np.uint64), fixtures[f"{name}/prog/term_coeff"].view(np.uint64))


@pytest.mark.parametrize("name", NAMES)
def test_sector_bit_exact(fixtures, name):
    S = O.Sector(_spec(name))
    reps, inv = S.reps()
    assert np.array_equal(reps, fixtures[f"{name}/reps"])
    assert np.array_equal(inv.view(np.uint64), fixtures[f"{name}/inv_norms"].view(np.uint64))


@pytest.mark.parametrize("name", NAMES)
def test_gather_and_sparsity_bit_exact(fixtures, name):
    S = O.Sector(_spec(name))
    P = O.Program(host_program(fixtures, name))
    y = S.gather(P, fixtures[f"{name}/x"])
    assert np.array_equal(y.view(np.uint64), fixtures[f"{name}/y"].view(np.uint64))
    rp, col, val = S.csr(P)
    assert np.array_equal(rp, fixtures[f"{name}/csr_row_ptr"])
    assert np.array_equal(col, fixtures[f"{name}/csr_col"])
    assert np.array_equal(val.view(np.uint64), fixtures[f"{name}/csr_val"].view(np.uint64))


@pytest.mark.parametrize("name", NAMES)
def test_lanczos_and_lowest(fixtures, name):
    S = O.Sector(_spec(name))
    P = O.Program(host_program(fixtures, name))
    a, b = S.lanczos(P, fixtures[f"{name}/x"], 40)
    ra, rb = fixtures[f"{name}/lz_alpha"], fixtures[f"{name}/lz_beta"]
    assert len(a) == len(ra)
    # the recurrence amplifies roundoff along the run: early steps agree to 1e-13, the tail to 1e-6
    np.testing.assert_allclose(a[:10], ra[:10], rtol=0, atol=1e-12)
    np.testing.assert_allclose(b[:11], rb[:11], rtol=0, atol=1e-12)
    e0, it, cv = S.scan_lowest(P)
    re0, rit, rcv = fixtures[f"{name}/e0"]
    assert cv and rcv
    assert abs(e0 - re0) <= 1e-12 * abs(re0)
    assert abs(it - rit) <= 1


@pytest.mark.parametrize("name", NAMES)
def test_ftlm_and_cf(fixtures, name):
    S = O.Sector(_spec(name))
    P = O.Program(host_program(fixtures, name))
    betas = 1.0 / np.linspace(0.1, 4.0, 40)
    f = S.ftlm(P, 8, 60, 20240601, betas)
    for k in ("lnZ", "E", "V"):
        ref = fixtures[f"{name}/ftlm_{k}"]
        np.testing.assert_allclose(f[k], ref, rtol=1e-9, atol=1e-9 * np.abs(ref).max())
    omega = np.linspace(-1.0, 6.0, 64)
    Sw, sh = S.cf(P, fixtures[f"{name}/x"], 80, omega, 0.05)
    ref = fixtures[f"{name}/cf_S"]
    assert abs(sh - fixtures[f"{name}/cf_shift"][0]) <= 1e-9
    np.testing.assert_allclose(Sw, ref, rtol=0, atol=1e-8 * np.abs(ref).max())


def test_seed_streams(fixtures):
    np.testing.assert_allclose(O.sample_vector(42, 3, 64), fixtures["sample_vector/42/3"], rtol=0, atol=1e-15)
    assert np.array_equal(O.staged_seed(0x51ED0B70, 64), fixtures["staged_seed/0x51ED0B70"])


def test_known_heisenberg_ring(golden):
    spec = lat.chain_sector(12, 6, 0)
    P = O.Program(ops.row_program(ops.from_products(12, ops.heisenberg_products(lat.chain_bonds(12)))))
    e0, _, cv = O.Sector(spec).scan_lowest(P)
    assert cv and abs(e0 - golden["known"]["heis12_k0_e0"]) < 1e-11


def _sector_spectrum(spec, prog):
    S = O.Sector(spec)
    d = S.dim
    if d == 0:
        return np.zeros(0)
    P = O.Program(prog)
    H = np.zeros((d, d), complex)
    for j in range(d):
        e = np.zeros(d, complex)
        e[j] = 1.0
        H[:, j] = S.gather(P, e)
    assert np.allclose(H, H.conj().T, atol=1e-12)
    return np.linalg.eigvalsh(H)


@pytest.mark.parametrize("model", ["chain4", "chain5_odd", "j1j2_chain12", "xy_chain10"])
def test_golden_fixed_sz_spectra(golden, model):
    """The lowest levels of a fixed-S^z space, reassembled from its momentum sectors, equal the energies the
    reference recorded in its golden suite (tier exact, 1e-10)."""
    g = golden["models"][model]
    N = g["n_sites"]
    prods = [(o, tuple(s), complex(c[0], c[1])) for o, s, c in g["products"]]
    prog = ops.row_program(ops.from_products(N, prods))
    for key, ref in g["records"].items():
        n_up = int(key.split("sz=")[1].split("/")[0])
        levels = np.sort(np.concatenate([_sector_spectrum(lat.chain_sector(N, n_up, k), prog) for k in range(N)]))
        np.testing.assert_allclose(levels[: len(ref)], ref, rtol=0, atol=1e-10)


def test_golden_exact_thermodynamics(golden):
    """The whole Hilbert space's thermodynamics of the J1-J2 chain N = 12 -- every S^z x momentum block's dense
    spectrum, its exact trace, and the thermal driver's log-space combine -- equal the reference's golden thermal
    records (its exact method, and its FTLM method, which densifies every block of this size): tier exact,
    1e-10 relative."""
    g = golden["models"]["j1j2_chain12"]
    N = g["n_sites"]
    prods = [(o, tuple(s), complex(c[0], c[1])) for o, s, c in g["products"]]
    prog = ops.row_program(ops.from_products(N, prods))
    recs = golden["thermal"]["j1j2_chain12"]
    T = np.asarray(recs["j1j2_chain12/api/thermal/exact/auto"]["T"])
    betas = 1.0 / T
    curves, n_states = [], 0
    for n_up in range(N + 1):
        for k in range(N):
            lv = _sector_spectrum(lat.chain_sector(N, n_up, k), prog)
            if len(lv) == 0:
                continue
            n_states += len(lv)
            e0 = lv.min()
            w = np.exp(-np.outer(betas, lv - e0))
            z = w.sum(axis=1)
            m1 = (w * (lv - e0)).sum(axis=1) / z
            m2 = (w * (lv - e0) ** 2).sum(axis=1) / z
            curves.append({"lnZ": np.log(z) - betas * e0, "E": e0 + m1, "V": np.maximum(m2 - m1 * m1, 0.0)})
    assert n_states == 2 ** N
    tot = O.combine_blocks(curves, betas)
    for key, rec in recs.items():
        assert np.allclose(rec["T"], T)
        for q in ("E", "C", "S"):
            ref = np.asarray(rec[q])
            np.testing.assert_allclose(tot[q], ref, rtol=1e-10, atol=1e-10 * np.abs(ref).max(), err_msg=f"{key} {q}")


@pytest.mark.parametrize("model", ["square4x3", "tri_chiral4x3"])
def test_golden_exact_thermodynamics_2d(golden, model):
    """The whole spectrum of a 12-site torus model -- the square lattice's Heisenberg model, the triangular
    lattice's with next-nearest exchange and scalar chirality (three-body terms) -- rebuilt block by block (each
    S^z block densely, with the trivial group), traced exactly and combined in log space, equals the
    reference's golden exact thermodynamics (with and without its symmetry sectors): E, C, S within 1e-10."""
    g = golden["models"][model]
    N = g["n_sites"]
    prods = [(o, tuple(s), complex(c[0], c[1])) for o, s, c in g["products"]]
    prog = ops.row_program(ops.from_products(N, prods))
    recs = golden["thermal"][model]
    T = np.asarray(next(iter(recs.values()))["T"])
    betas = 1.0 / T
    curves, n_states = [], 0
    for n_up in range(N + 1):
        spec = lat.SectorSpec(n_sites=N, n_up=n_up, perms=np.arange(N, dtype=np.int32)[None, :],
                              chars=np.array([1.0 + 0.0j]))
        lv = _sector_spectrum(spec, prog)
        n_states += len(lv)
        e0 = lv.min()
        w = np.exp(-np.outer(betas, lv - e0))
        z = w.sum(axis=1)
        m1 = (w * (lv - e0)).sum(axis=1) / z
        m2 = (w * (lv - e0) ** 2).sum(axis=1) / z
        curves.append({"lnZ": np.log(z) - betas * e0, "E": e0 + m1, "V": np.maximum(m2 - m1 * m1, 0.0)})
    assert n_states == 2 ** N
    tot = O.combine_blocks(curves, betas)
    for key, rec in recs.items():
        assert np.allclose(rec["T"], T)
        for q in ("E", "C", "S"):
            ref = np.asarray(rec[q])
            np.testing.assert_allclose(tot[q], ref, rtol=1e-10, atol=1e-10 * np.abs(ref).max(), err_msg=f"{key} {q}")


def test_golden_sampled_ftlm(golden):
    """The reference's golden FTLM record of the J1-J2 chain N = 12 without symmetry sectors -- one block of all
    4096 states, 8 samples, Krylov 40, seed 11 -- reproduced within 1e-10: the block's seed is the call's seed
    advanced once by the thermal driver's 64-bit LCG step (src/engine/thermal.cpp:470-471); sample s is the
    oracle's restatement of sample_engine(seed, s) (include/ed/thermal/sample_seed.h:37-89); the Lanczos run keeps
    the local reorthogonalisation against the previous vector (include/ed/krylov/lanczos.h:189-193); the oracle's
    sample moments, then the samples combined about their least minimum (include/ed/thermal/ftlm.h:199-235)."""
    g = golden["models"]["j1j2_chain12"]
    N = g["n_sites"]
    prods = [(o, tuple(s), complex(c[0], c[1])) for o, s, c in g["products"]]
    H = ops.from_products(N, prods).to_dense()
    rec = golden["thermal_sampled"]["j1j2_chain12"]
    T = np.asarray(rec["T"])
    betas = 1.0 / T
    k, depth, n = rec["samples"], rec["krylov"], H.shape[0]
    seed = (rec["seed"] * 6364136223846793005 + 1442695040888963407) % (1 << 64)
    moms = []
    for s in range(k):
        v = O.sample_vector(seed, s, n)
        v = v / np.linalg.norm(v)
        vp = np.zeros_like(v)
        alpha, beta = [], [0.0]
        for j in range(depth):
            w = H @ v - beta[-1] * vp
            a = np.vdot(v, w).real
            w = w - a * v
            o = np.vdot(v, w)
            if j > 0 and abs(o) > 1.49011611938476562e-08:
                w = w - o * v
            b = np.linalg.norm(w)
            alpha.append(a)
            beta.append(b)
            vp, v = v, w / b
        moms.append(O.sample_moments(alpha, beta, betas))
    e_ref = min(m[0] for m in moms)
    E, C, S = [], [], []
    for t, bt in enumerate(betas):
        zz = e1 = e2 = 0.0
        for em, Z, E1, E2 in moms:
            dd = em - e_ref
            r = np.exp(-bt * dd)
            zz += Z[t] * r
            e1 += (E1[t] + dd * Z[t]) * r
            e2 += (E2[t] + 2.0 * dd * E1[t] + dd * dd * Z[t]) * r
        zz, e1, e2 = zz / k, e1 / k, e2 / k
        m1, m2 = e1 / zz, e2 / zz
        lnZ = np.log(n) + np.log(zz) - bt * e_ref
        E.append(e_ref + m1)
        C.append(bt * bt * (m2 - m1 * m1))
        S.append(lnZ + bt * (e_ref + m1))
    for q, got in (("E", E), ("C", C), ("S", S)):
        ref = np.asarray(rec[q])
        np.testing.assert_allclose(got, ref, rtol=1e-10, atol=1e-10 * np.abs(ref).max(), err_msg=q)


def test_golden_t0_dynamics(golden):
    """The T = 0 S^z(pi) spectrum of the J1-J2 chain N = 12 equals the reference's golden records (tier exact,
    1e-10): for each ground state -- this chain sits at the Majumdar-Ghosh point, so its ground manifold is the
    two dimer states, one at momentum 0 and one at pi -- phi = S^z(pi) psi0 through the oracle's cross-sector
    gather into the block at momentum k + pi, then the oracle's continued fraction shifted by E0 (80 steps span
    every block here, so the fraction is exact); the spectra averaged over the ground manifold, which is what
    the reference's verb returns for a degenerate ground state."""
    g = golden["models"]["j1j2_chain12"]
    N = g["n_sites"]
    prods = [(o, tuple(s), complex(c[0], c[1])) for o, s, c in g["products"]]
    H = ops.from_products(N, prods)
    prog = ops.row_program(H)
    dyn = golden["dynamics"]["j1j2_chain12"]
    lo, hi, n_om = dyn["omega"]
    omega = np.linspace(lo, hi, n_om)
    eta, depth, m = dyn["eta"], dyn["krylov"], N // 2   # q = pi = 2 pi m / N
    Sq = ops.from_products(N, ops.sz_q_products(N, np.pi))
    ground = []   # (energy, n_up, k, vector in the block's basis)
    for n_up in range(N + 1):
        for k in range(N):
            spec = lat.chain_sector(N, n_up, k)
            So = O.Sector(spec)
            d = So.dim
            if d == 0:
                continue
            P = O.Program(prog)
            Hb = np.zeros((d, d), complex)
            for j in range(d):
                e = np.zeros(d, complex)
                e[j] = 1.0
                Hb[:, j] = So.gather(P, e)
            w, V = np.linalg.eigh(Hb)
            ground += [(w[i], n_up, k, V[:, i]) for i in range(d) if w[i] < w[0] + 1e-9]
    e0 = min(x[0] for x in ground)
    ground = [x for x in ground if x[0] < e0 + 1e-9]
    assert len(ground) == 2 and abs(e0 + 4.5) < 1e-12   # the two dimer states, E0 = -3N/8
    total = np.zeros(len(omega))
    for _, n_up, k, psi in ground:
        src, tgt = lat.chain_sector(N, n_up, k), lat.chain_sector(N, n_up, (k + m) % N)
        S_src, S_tgt = O.Sector(src), O.Sector(tgt)
        phi = S_tgt.gather(O.Program(ops.cross_row_program(Sq, tgt, src)), psi, col=S_src)
        S, _ = S_tgt.cf(O.Program(prog), phi, depth, omega, eta, shift=e0)
        total += S
    total /= len(ground)
    for key, ref in dyn["records"].items():
        np.testing.assert_allclose(total, ref, rtol=1e-10, atol=1e-10 * np.abs(ref).max(), err_msg=key)


def _translation_invariant_models(N, seed):
    """Translation-invariant N-site rings: Heisenberg with next-nearest exchange, XXZ in a field, Heisenberg
    with scalar chirality (three-body terms), and random complex exchange (the same couplings on every bond, so
    translations stay a symmetry; no time reversal)."""
    rng = np.random.default_rng(seed)
    ring = lat.chain_bonds(N)
    c = complex(rng.normal(), rng.normal()) * 0.5
    jz = float(rng.normal())
    rand = []
    for i, j in ring:
        rand += [("+-", (i, j), c), ("-+", (i, j), np.conj(c)), ("zz", (i, j), complex(jz))]
    return {
        "j1j2": ops.heisenberg_products(ring) + ops.heisenberg_products(lat.chain_bonds(N, 2), 0.4),
        "xxz_field": ops.xxz_products(ring, 1.0, 0.6) + ops.zeeman_z_products(N, 0.3),
        "chiral": ops.heisenberg_products(ring) + ops.chiral_products([(i, (i + 1) % N, (i + 2) % N)
                                                                       for i in range(N)], 0.7),
        "random_complex": rand,
    }


@pytest.mark.parametrize("N", [8, 9])
def test_momentum_blocks_tile_the_spectrum(N):
    """For a translation-invariant ring, the spectra of the N momentum blocks of a fixed S^z, each built by the
    oracle's sector walk (representatives, characters, 1/norms, phases), together equal the spectrum of the
    whole S^z block built by the same walk with the trivial group (no characters, phases or norms): every level,
    with multiplicity, within 1e-12 of the coupling scale (the reference checks every sector lane against the dense block of H the same way,
    tests/unit/test_row_walk.cpp:386-481)."""
    for name, prods in _translation_invariant_models(N, seed=N).items():
        H = ops.from_products(N, prods)
        prog = ops.row_program(H)
        scale = sum(abs(c) for _, _, c in prods)
        for n_up in range(N + 1):
            levels = np.sort(np.concatenate([_sector_spectrum(lat.chain_sector(N, n_up, k), prog) for k in range(N)]))
            states = [s for s in range(1 << N) if bin(s).count("1") == n_up]
            full = lat.SectorSpec(n_sites=N, n_up=n_up, perms=np.arange(N, dtype=np.int32)[None, :],
                                  chars=np.array([1.0 + 0.0j]))
            direct = _sector_spectrum(full, prog)
            assert len(levels) == len(direct) == len(states), (name, n_up)
            np.testing.assert_allclose(levels, direct, rtol=0, atol=1e-12 * scale, err_msg=f"{name} n_up={n_up}")


def test_flip_and_torus_blocks_tile_the_spectrum():
    """Two more abelian groups whose one-dimensional irreps tile a fixed-S^z space: the ring's translations times
    the spin flip at half filling (momentum x flip parity, on the flip-symmetric J1-J2 and XXZ rings; the flip
    enters as an XOR mask of every element), and the translations of a 4x2 square torus (momentum (kx, ky), on
    the J1-J2 model). The blocks' spectra together equal the whole S^z block's, within 1e-12 of the scale."""
    def check(N, n_up, prog, scale, specs, what):
        levels = np.sort(np.concatenate([_sector_spectrum(sp, prog) for sp in specs]))
        full = lat.SectorSpec(n_sites=N, n_up=n_up, perms=np.arange(N, dtype=np.int32)[None, :],
                              chars=np.array([1.0 + 0.0j]))
        direct = _sector_spectrum(full, prog)
        assert len(levels) == len(direct), what
        np.testing.assert_allclose(levels, direct, rtol=0, atol=1e-12 * scale, err_msg=what)

    N = 8
    flip_symmetric = {"j1j2": _translation_invariant_models(N, seed=3)["j1j2"],
                      "xxz": ops.xxz_products(lat.chain_bonds(N), 1.0, 0.6)}   # no field: the flip stays a symmetry
    for name, prods in flip_symmetric.items():
        prog = ops.row_program(ops.from_products(N, prods))
        perms, flips = lat.with_spin_flip(lat.chain_translations(N), N)
        specs = [lat.SectorSpec(N, N // 2, perms, np.concatenate([lat.momentum_chars(N, k),
                                                                  par * lat.momentum_chars(N, k)]), flips)
                 for k in range(N) for par in (1.0, -1.0)]
        check(N, N // 2, prog, sum(abs(c) for _, _, c in prods), specs, f"{name} with the flip")

    Lx, Ly = 4, 2
    nn, nnn = lat.square_j1j2_bonds(Lx, Ly)
    prods = ops.heisenberg_products(nn) + ops.heisenberg_products(nnn, 0.5)
    prog = ops.row_program(ops.from_products(Lx * Ly, prods))
    perms = lat.square_translations(Lx, Ly)
    a = np.array([e % Lx for e in range(Lx * Ly)])
    b = np.array([e // Lx for e in range(Lx * Ly)])
    for n_up in (2, 3, 4):
        specs = [lat.SectorSpec(Lx * Ly, n_up, perms, np.exp(-2j * np.pi * (kx * a / Lx + ky * b / Ly)))
                 for kx in range(Lx) for ky in range(Ly)]
        check(Lx * Ly, n_up, prog, sum(abs(c) for _, _, c in prods), specs, f"4x2 torus n_up={n_up}")


def test_sublattice_engagement():
    """The key order engages exactly where the reference's relaxed rule does (sublattice_code.h:23-34)."""
    assert O.Sector(lat.chain_sector(20, 1, 0)).sublattice() is None
    s24 = O.Sector(lat.chain_sector(24, 1, 0)).sublattice()
    assert s24 is not None and (s24["L"], s24["m"]) == (12, 2)
    spec = lat.chain_a1_flip_sector(32).with_n_up(1)
    s32 = O.Sector(spec).sublattice()
    assert s32 is not None and (s32["L"], s32["m"]) == (16, 2)
    sq = O.Sector(lat.square_k0_sector(6, 6, 1)).sublattice()
    assert sq is not None and (sq["L"], sq["m"]) == (6, 6)


def test_tridiagonal_solver():
    rng = np.random.default_rng(3)
    for m in (1, 2, 5, 40, 120):
        a = rng.normal(size=m)
        b = np.concatenate([[0.0], np.abs(rng.normal(size=m))])
        T = np.diag(a) + np.diag(b[1:m], 1) + np.diag(b[1:m], -1)
        vals, vecs = O.tridiag_eig(a, b)
        np.testing.assert_allclose(vals, np.linalg.eigvalsh(T), atol=1e-12 * max(1, np.abs(vals).max()))
        np.testing.assert_allclose(T @ vecs, vecs * vals, atol=1e-10)
