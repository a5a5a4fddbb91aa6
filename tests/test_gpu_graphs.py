"""Lanczos steps replayed from captured CUDA graphs give the scalars and vectors of steps launched one by one,
bit for bit (QB_GRAPHS=0 launches every step; sectors of up to 2^20 states otherwise run batches of captured
steps): the ungated recurrence (none and local reorthogonalisation, FP64 and FP32 storage), the certified
ground-state vector (its kept basis filled on the device), and the continued fraction; and the k = 1 lane, which
launches step by step either way, is unchanged by the switch."""
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


def _block(n=18, k=0, K=0.2):
    from qed_spin_b200 import device as D
    prods = (ops.heisenberg_products(lat.chain_bonds(n), 1.0)
             + ops.chiral_products([(i, (i + 1) % n, (i + 2) % n) for i in range(n)], K))
    prog = ops.row_program(ops.from_products(n, prods))
    return D.Sector(lat.chain_sector(n, n // 2, k)), D.Program(prog)


def _both(monkeypatch, fn):
    out = {}
    for flag in ("1", "0"):
        monkeypatch.setenv("QB_GRAPHS", flag)
        out[flag] = fn()
    return out["1"], out["0"]


def _bits(a):
    return np.ascontiguousarray(a).view(np.uint64)


@pytest.mark.parametrize("reorth", [0, 1])
@pytest.mark.parametrize("dtype", ["c128", "c64"])
def test_ungated_recurrence(monkeypatch, reorth, dtype):
    from qed_spin_b200 import device as D
    S, P = _block()
    rng = np.random.default_rng(3)
    v0 = rng.standard_normal(S.dim) + 1j * rng.standard_normal(S.dim)
    g, e = _both(monkeypatch, lambda: D.lanczos(S, P, v0, 61, reorth=reorth, dtype=dtype))
    assert len(g[0]) == len(e[0]) == 61
    assert np.array_equal(_bits(g[0]), _bits(e[0])) and np.array_equal(_bits(g[1]), _bits(e[1]))


@pytest.mark.parametrize("dtype,refine", [("c128", False), ("c64", True)])
def test_k1_lane(monkeypatch, dtype, refine):
    from qed_spin_b200 import device as D
    S, P = _block(k=3)
    g, e = _both(monkeypatch, lambda: D.eigs_lowest(S, P, dtype=dtype, refine=refine))
    assert g["converged"] and e["converged"]
    assert _bits(np.array([g["e0"]]))[0] == _bits(np.array([e["e0"]]))[0]
    assert g["iters"] == e["iters"]
    assert abs(g["matvecs"] - e["matvecs"]) <= 8   # a batch may run past the stopping step


def test_ground_state_vector(monkeypatch):
    from qed_spin_b200 import device as D
    S, P = _block(n=16, k=0)
    g, e = _both(monkeypatch, lambda: D.ground_state(S, P))
    assert g["certified"] and e["certified"]
    assert _bits(np.array([g["e0"]]))[0] == _bits(np.array([e["e0"]]))[0]
    assert np.array_equal(_bits(g["vector"]), _bits(e["vector"]))


def test_continued_fraction(monkeypatch):
    from qed_spin_b200 import device as D
    S, P = _block(n=16, k=2)
    rng = np.random.default_rng(9)
    phi = rng.standard_normal(S.dim) + 1j * rng.standard_normal(S.dim)
    omega = np.linspace(-2.0, 6.0, 200)
    g, e = _both(monkeypatch, lambda: D.cf(S, P, phi, 90, omega, 0.05)[0])
    assert np.array_equal(_bits(g), _bits(e))
