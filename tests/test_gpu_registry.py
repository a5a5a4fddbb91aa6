"""Sectors by content and the sector file: one shared sector per descriptor (also across threads), released sectors
cached up to the capacity, and a saved-then-loaded sector equal to the enumerated one bit for bit (basis, 1/norms,
and y = H x through it)."""
import os
import tempfile
import threading

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


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint64)


def test_shared_sectors():
    from qed_spin_b200 import device as D
    D.registry_capacity(0)
    D.registry_capacity(4 << 30)
    spec = lat.chain_sector(16, 8, 3)
    a = D.Sector(spec, shared=True)
    b = D.Sector(spec, shared=True)
    assert a.h.value == b.h.value
    c = D.Sector(lat.chain_sector(16, 8, 4), shared=True)
    assert c.h.value != a.h.value
    st = D.registry_stats()
    assert st["sectors"] == 2 and st["idle_sectors"] == 0
    ptr = a.h.value
    a.close()
    b.close()
    assert D.registry_stats()["idle_sectors"] == 1
    again = D.Sector(spec, shared=True)   # from the cache
    assert again.h.value == ptr
    assert D.registry_stats()["idle_sectors"] == 0
    again.close()
    c.close()
    D.registry_capacity(0)                # empties the cache
    assert D.registry_stats() == {"sectors": 0, "idle_sectors": 0, "idle_bytes": 0}
    D.registry_capacity(4 << 30)


def test_shared_across_threads():
    from qed_spin_b200 import device as D
    spec = lat.chain_a1_flip_sector(20)
    out = [None] * 8

    def grab(i):
        torch.cuda.set_device(0)
        out[i] = D.Sector(spec, shared=True)

    ts = [threading.Thread(target=grab, args=(i,)) for i in range(8)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    assert len({s.h.value for s in out}) == 1
    ref = D.Sector(spec)
    r1, i1 = out[0].reps()
    r2, i2 = ref.reps()
    assert np.array_equal(r1, r2) and np.array_equal(_bits(i1), _bits(i2))
    for s in out:
        s.close()


def test_destroy_of_a_shared_sector_is_refused():
    from qed_spin_b200 import device as D
    from qed_spin_b200._lib import lib
    s = D.Sector(lat.chain_sector(12, 6, 1), shared=True)
    assert lib().qb_sector_destroy(s.h) != 0
    s.close()


@pytest.mark.parametrize("spec", [lat.chain_a1_flip_sector(24), lat.square_k0_sector(4, 4, 8),
                                  lat.chain_sector(14, 7, 5)], ids=["chain24_a1f", "sq4x4", "chain14_k5"])
def test_save_load_roundtrip(spec):
    from qed_spin_b200 import device as D
    S = D.Sector(spec)
    n = spec.n_sites
    prog = ops.row_program(ops.from_products(n, ops.heisenberg_products(
        lat.chain_bonds(n) if spec.perms.shape[0] != 16 else lat.square_j1j2_bonds(4, 4)[0])))
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "sector.qbs")
        S.save(path)
        L = D.Sector.load(path, spec)
        # a damaged file is refused
        raw = bytearray(open(path, "rb").read())
        raw[-20] ^= 0xFF
        bad = os.path.join(d, "bad.qbs")
        open(bad, "wb").write(bytes(raw))
        with pytest.raises(ValueError):
            D.Sector.load(bad, spec)
    r1, i1 = S.reps()
    r2, i2 = L.reps()
    assert np.array_equal(r1, r2) and np.array_equal(_bits(i1), _bits(i2))
    assert S.info()["slc_L"] == L.info()["slc_L"]
    P = D.Program(prog)
    x = torch.randn(S.dim, dtype=torch.complex128, device="cuda")
    y1, y2 = torch.empty_like(x), torch.empty_like(x)
    D.matvec(S, S, P, [x], [y1])
    D.matvec(L, L, P, [x], [y2])
    assert np.array_equal(_bits(y1.cpu().numpy()), _bits(y2.cpu().numpy()))


def test_memory_trim_empties_the_block_cache():
    """Released device blocks stay cached for reuse; qb_memory_trim returns them: after a sector is made and
    destroyed, trimming to 0 leaves no idle bytes, and a sector made afterwards is the same bit for bit."""
    from qed_spin_b200 import device as D
    spec = lat.chain_sector(20, 10, 3)
    S = D.Sector(spec)
    r1, i1 = S.reps()
    S.close()
    torch.cuda.synchronize()
    assert D.memory_trim(0) == 0
    assert D.memory_trim(0) == 0
    T = D.Sector(spec)
    r2, i2 = T.reps()
    assert np.array_equal(r1, r2) and np.array_equal(_bits(i1), _bits(i2))
