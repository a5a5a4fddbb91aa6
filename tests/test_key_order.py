"""The sublattice key order (no GPU): the tables the library builds for a group -- the block system, each site's
key bit, the least leading block of every pattern of every block and the elements that reach it -- equal the
reference engine's own SublatticeCode tables (oracle/_ref), bit for bit, for chains (translations, the dihedral
group, the dihedral group times the spin flip) and square tori, under every mode of the size rule. The device
enumeration's representatives depend on exactly these tables."""
import numpy as np
import pytest

from oracle import ref as R
from qed_spin_b200 import lattice as lat

GROUPS = []
for _N in (8, 12, 16, 20, 24, 28, 30, 32):
    GROUPS.append((f"chain{_N}_T", _N, lat.chain_translations(_N), None))
    GROUPS.append((f"chain{_N}_D", _N, lat.chain_dihedral(_N), None))
    _p, _f = lat.with_spin_flip(lat.chain_dihedral(_N), _N)
    GROUPS.append((f"chain{_N}_DxZ2", _N, _p, _f))
for _a, _b in ((4, 3), (4, 4), (5, 5), (6, 4), (6, 5), (6, 6), (8, 4), (8, 8)):
    GROUPS.append((f"square{_a}x{_b}", _a * _b, lat.square_translations(_a, _b), None))


@pytest.mark.parametrize("mode", [1, -1, -2, 0])
@pytest.mark.parametrize("name,N,perms,flips", GROUPS, ids=[g[0] for g in GROUPS])
def test_key_order_tables_equal_the_reference(name, N, perms, flips, mode):
    if not R.available():
        pytest.fail("the reference engine library is not built (oracle/Makefile, run by __graft_entry__.build())")
    from qed_spin_b200 import device as D
    spec = lat.SectorSpec(N, N // 2, np.asarray(perms, np.int32), np.ones(len(perms), np.complex128),
                          None if flips is None else np.asarray(flips, np.uint64))
    mine = D.key_order(spec, sublattice_mode=mode)
    ref = R.key_order(N, perms, flips, mode=mode)
    assert (mine is None) == (ref is None)
    if ref is None:
        return
    assert (mine["L"], mine["m"]) == (ref["L"], ref["m"])
    for key in ("key_bit", "lead", "cand_off", "cand"):
        assert np.array_equal(mine[key], ref[key]), key


def test_the_benchmark_groups_engage_the_key_order():
    """The chain-32 A1 flip-even group and the 6x6 translations use a code under the device size rule."""
    from qed_spin_b200 import device as D
    c32 = D.key_order(lat.chain_a1_flip_sector(32))
    sq = D.key_order(lat.square_k0_sector(6, 6, 18))
    assert (c32["L"], c32["m"]) == (16, 2)
    assert (sq["L"], sq["m"]) == (6, 6)
