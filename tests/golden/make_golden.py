"""Generate the golden fixtures the tests pin the oracle and the CUDA path against.

Run in a tree where the reference sources are present (it reads them and its compiled CPU engine,
oracle/_ref/libqed_ref.so, built by `make -C oracle`):

    python tests/golden/make_golden.py REFERENCE_ROOT [--json-only]

(--json-only rewrites golden.json alone, leaving fixtures.npz as it is.)

Writes
  golden.json   energies the reference recorded in its own golden suite
                (tests/python/golden/refs/api-2026-09/cpu.json.gz, tier "exact" 1e-10), for the chain models
                whose fixed-S^z spectra the sector tests reassemble, plus the N = 12 Heisenberg ring E0; and the
                exact thermodynamics (T, E, C, S) and the T = 0 S^z(pi) spectrum it recorded for the J1-J2 chain
                N = 12.
  fixtures.npz  outputs of the reference engine itself on small seeded cases: representatives and 1/norms,
                row programs, y = H x, the merged CSR pattern and its spmv of x, the k = 4 lane's levels, Lanczos alpha/beta, the k = 1 lane's E0, FTLM
                curves and continued-fraction spectra.
"""
from __future__ import annotations

import gzip
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import ref as R  # noqa: E402
from qed_spin_b200 import lattice as lat  # noqa: E402
from qed_spin_b200 import operators as ops  # noqa: E402

# the models of the reference's test zoo (tests/python/support/models.py:505-540)
ZOO = {
    "chain4": (4, lambda: ops.heisenberg_products(lat.chain_bonds(4))),
    "chain5_odd": (5, lambda: ops.heisenberg_products(lat.chain_bonds(5))),
    "j1j2_chain12": (12, lambda: ops.heisenberg_products(lat.chain_bonds(12))
                     + ops.heisenberg_products(lat.chain_bonds(12, 2), 0.5)),
    "xy_chain10": (10, lambda: ops.xxz_products(lat.chain_bonds(10), 1.0, 0.0)),
}


def triangular_torus(Lx: int, Ly: int):
    """The triangular torus of the golden harness's tri_chiral4x3 (tests/python/support/models.py:439-464): site
    (x, y) is x + Lx y; nearest neighbours at (1, 0), (0, 1), (-1, 1), next-nearest at (1, 1), (-2, 1), (1, -2), each
    unordered pair once; counter-clockwise up triangles (x, y), (x+1, y), (x, y+1) and down triangles (x+1, y),
    (x+1, y+1), (x, y+1)."""
    def idx(x, y):
        return (x % Lx) + Lx * (y % Ly)

    def once(bonds):
        seen, out = set(), []
        for i, j in bonds:
            key = (min(i, j), max(i, j))
            if i != j and key not in seen:
                seen.add(key)
                out.append((i, j))
        return out

    nn, nnn, tri = [], [], []
    for y in range(Ly):
        for x in range(Lx):
            i = idx(x, y)
            nn += [(i, idx(x + 1, y)), (i, idx(x, y + 1)), (i, idx(x - 1, y + 1))]
            nnn += [(i, idx(x + 1, y + 1)), (i, idx(x - 2, y + 1)), (i, idx(x + 1, y - 2))]
            tri += [(i, idx(x + 1, y), idx(x, y + 1)), (idx(x + 1, y), idx(x + 1, y + 1), idx(x, y + 1))]
    return once(nn), once(nnn), tri


def _tri_chiral4x3():
    nn, nnn, tri = triangular_torus(4, 3)
    return ops.heisenberg_products(nn) + ops.heisenberg_products(nnn, 0.2) + ops.chiral_products(tri, 0.5)


# 12-site models whose whole spectrum the thermal test rebuilds block by block (models.py:577-591): the square
# 4x3 torus's nearest-neighbour Heisenberg model, and the triangular 4x3 torus with J2 = 0.2 and chirality 0.5
ZOO2D = {
    "square4x3": (12, lambda: ops.heisenberg_products(lat.square_j1j2_bonds(4, 3)[0])),
    "tri_chiral4x3": (12, _tri_chiral4x3),
}

RECORDS = {
    "chain4": ["chain4/api/eigs/sz=2/k=4"],
    "chain5_odd": ["chain5_odd/api/eigs/sz=2/k=4"],
    "j1j2_chain12": ["j1j2_chain12/api/eigs/sz=6/k=4"],
    "xy_chain10": ["xy_chain10/api/eigs/sz=5/k=4"],
}

# exact thermodynamics of the whole Hilbert space (every block solved densely: the thermal verb's exact method, and
# its FTLM method with the default dense limit of 512 states, which every block of a 12-site chain is under)
THERMAL = {"j1j2_chain12": ["j1j2_chain12/api/thermal/exact/auto", "j1j2_chain12/api/thermal/ftlm/auto"],
           "square4x3": ["square4x3/api/thermal/exact/auto", "square4x3/api/thermal/exact/none"],
           "tri_chiral4x3": ["tri_chiral4x3/api/thermal/exact/auto", "tri_chiral4x3/api/thermal/exact/none"]}

# FTLM without symmetry sectors: one block of all 2^12 states, 8 samples, Krylov 40, seed 11 (the golden
# harness's thermal case, tests/python/golden/cases.py:142-162)
SAMPLED = {"j1j2_chain12": "j1j2_chain12/api/thermal/ftlm/none"}

# T = 0 dynamics of S^z(q = pi) = N^-1/2 sum_i e^{i pi i} S^z_i on 41 frequencies in [-1, 4], eta 0.15, Krylov 80
# (the golden harness's dynamics case, tests/python/golden/cases.py:175-190), with and without symmetry sectors
DYNAMICS = {"j1j2_chain12": ["j1j2_chain12/api/dynamics/T=0/auto/SzQ", "j1j2_chain12/api/dynamics/T=0/none/SzQ"]}

# small seeded cases run through the reference engine: (name, N, n_up, group, products)
def cases():
    out = []
    N = 12
    out.append(("heis12_k0", lat.chain_sector(N, 6, 0), ops.heisenberg_products(lat.chain_bonds(N))))
    out.append(("heis12_k3", lat.chain_sector(N, 6, 3), ops.heisenberg_products(lat.chain_bonds(N))))
    out.append(("xxz14_h_k5", lat.chain_sector(14, 6, 5),
                ops.xxz_products(lat.chain_bonds(14), 1.0, 0.5) + ops.zeeman_z_products(14, 0.1)))
    out.append(("xxz16_a1f", lat.chain_a1_flip_sector(16), ops.xxz_products(lat.chain_bonds(16), 1.0, 0.7)))
    chir = [(i, (i + 1) % 13, (i + 2) % 13) for i in range(13)]
    out.append(("chiral13_k2", lat.chain_sector(13, 6, 2),
                ops.heisenberg_products(lat.chain_bonds(13), 0.8) + ops.chiral_products(chir, 0.3)))
    sq = lat.square_k0_sector(4, 4, 8)
    nn, nnn = lat.square_j1j2_bonds(4, 4)
    out.append(("j1j2_4x4_k0", sq, ops.heisenberg_products(nn, 1.0) + ops.heisenberg_products(nnn, 0.5)))
    return out


def main(ref_root: str, json_only: bool = False):
    golden = {"source": "tests/python/golden/refs/api-2026-09/cpu.json.gz (the reference's golden suite)",
              "tier_exact_tol": 1e-10, "models": {}, "known": {}}
    recs = json.load(gzip.open(os.path.join(ref_root, "tests/python/golden/refs/api-2026-09/cpu.json.gz")))["records"]
    for name, keys in RECORDS.items():
        N, prods = ZOO[name]
        golden["models"][name] = {
            "n_sites": N,
            "products": [[o, list(s), [complex(c).real, complex(c).imag]] for o, s, c in prods()],
            "records": {k: recs[k]["values"]["energies"] for k in keys},
        }
    for name, (N, prods) in ZOO2D.items():
        golden["models"][name] = {
            "n_sites": N,
            "products": [[o, list(s), [complex(c).real, complex(c).imag]] for o, s, c in prods()],
            "records": {},
        }
    # the N = 12 Heisenberg ring, k = 0 (a textbook value; the reference's k = 1 lane reproduces it)
    golden["known"]["heis12_k0_e0"] = -5.387390917445
    golden["thermal"] = {}
    for name, keys in THERMAL.items():
        golden["thermal"][name] = {k: {q: recs[k]["values"][q] for q in ("T", "E", "C", "S")} | {"tier": recs[k]["tier"]}
                                   for k in keys}
    golden["thermal_sampled"] = {}
    for name, key in SAMPLED.items():
        golden["thermal_sampled"][name] = {"record": key, "samples": 8, "krylov": 40, "seed": 11,
                                           "tier": recs[key]["tier"]} | {q: recs[key]["values"][q]
                                                                         for q in ("T", "E", "C", "S")}
    golden["dynamics"] = {}
    for name, keys in DYNAMICS.items():
        golden["dynamics"][name] = {"omega": [-1.0, 4.0, 41], "eta": 0.15, "krylov": 80, "q": "pi",
                                    "records": {k: recs[k]["values"]["S"] for k in keys},
                                    "tiers": {k: recs[k]["tier"] for k in keys}}
    if json_only:
        with open(os.path.join(HERE, "golden.json"), "w") as fh:
            json.dump(golden, fh, indent=1)
        print("wrote", os.path.join(HERE, "golden.json"))
        return

    fx = {}
    for name, spec, prods in cases():
        rs = R.Sector(spec.n_sites, spec.n_up, spec.perms, spec.chars, flips=spec.flips, slc_mode=-1)
        op = R.Operator(spec.n_sites, prods)
        rp = op.row_program()
        arr = rp.arrays()
        for k, v in arr.items():
            fx[f"{name}/prog/{k}"] = v
        reps, inv = rs.reps()
        fx[f"{name}/reps"] = reps
        fx[f"{name}/inv_norms"] = inv
        x = R.staged_seed(1234, rs.dim)
        fx[f"{name}/x"] = x
        fx[f"{name}/y"] = rs.gather(rp, x)
        rowp, col, val, ycsr = rs.csr(rp, x)
        fx[f"{name}/csr_y"] = ycsr
        fx[f"{name}/csr_row_ptr"] = rowp
        fx[f"{name}/csr_col"] = col
        fx[f"{name}/csr_val"] = val
        a, b = rs.lanczos(rp, x, 40, reorth=0)
        fx[f"{name}/lz_alpha"] = a
        fx[f"{name}/lz_beta"] = b
        e0, it, cv = rs.scan_lowest(rp)
        fx[f"{name}/e0"] = np.array([e0, it, cv], np.float64)
        ks, ks_cv, ks_ap = rs.ks_lowest(rp, 4)
        fx[f"{name}/ks4"] = ks   # the k = 4 lane: the reference's krylov_schur_kernel
        betas = 1.0 / np.linspace(0.1, 4.0, 40)
        f = rs.ftlm(rp, 8, 60, 20240601, betas)
        for k in ("lnZ", "E", "V"):
            fx[f"{name}/ftlm_{k}"] = f[k]
        fx[f"{name}/ftlm_emin"] = np.array([f["e_min"]])
        omega = np.linspace(-1.0, 6.0, 64)
        S, sh, cc = rs.cf(rp, x, 80, omega, 0.05)
        fx[f"{name}/cf_S"] = S
        fx[f"{name}/cf_shift"] = np.array([sh])
        fx[f"{name}/dim"] = np.array([rs.dim])
        print(f"{name}: dim {rs.dim}, E0 {e0} ({it} steps)")
    # the sample-vector stream of sample 3 of seed 42 (sample_seed.h)
    fx["sample_vector/42/3"] = R.sample_vector(42, 3, 64)
    fx["staged_seed/0x51ED0B70"] = R.staged_seed(0x51ED0B70, 64)
    with open(os.path.join(HERE, "golden.json"), "w") as fh:
        json.dump(golden, fh, indent=1)
    np.savez_compressed(os.path.join(HERE, "fixtures.npz"), **fx)
    print("wrote", os.path.join(HERE, "golden.json"), os.path.join(HERE, "fixtures.npz"))


if __name__ == "__main__":
    args = [a for a in sys.argv[1:] if not a.startswith("--")]
    if not args:
        sys.exit("usage: make_golden.py REFERENCE_ROOT [--json-only]")
    main(args[0], json_only="--json-only" in sys.argv[1:])
