"""The small seeded cases of tests/golden/fixtures.npz (mirrors tests/golden/make_golden.py)."""
from qed_spin_b200 import lattice as lat
from qed_spin_b200 import operators as ops


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


CASES = cases()
NAMES = [c[0] for c in CASES]
