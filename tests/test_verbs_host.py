"""The verbs' request checks and device resolution, on the host without a GPU: malformed requests are refused
before any device work, device="cpu" is refused as the reference engine's lane, and device="gpu" without a
CUDA device is an error, never a fallback."""
import numpy as np
import pytest

from qed_spin_b200 import lattice as lat
from qed_spin_b200 import operators as ops
from qed_spin_b200 import verbs


def _model(N=8):
    return ops.from_products(N, ops.heisenberg_products(lat.chain_bonds(N)))


@pytest.fixture(scope="module", autouse=True)
def _built():
    from qed_spin_b200 import build
    build.build()


def _no_device():
    import torch
    return not torch.cuda.is_available()


def test_malformed_requests_are_refused():
    H = _model()
    blocks = [lat.chain_sector(8, 4, 0)]
    with pytest.raises(verbs.InvalidRequest):
        verbs.eigs(H, 0, sectors=blocks)
    with pytest.raises(verbs.InvalidRequest):
        verbs.eigs(H, 1, sectors=blocks, dense_max_dim=-1)
    with pytest.raises(verbs.InvalidRequest):
        verbs.eigs(H, 1, sectors=blocks, device="tpu")
    with pytest.raises(verbs.InvalidRequest):
        verbs.thermal(H, [0.5, -1.0], sectors=blocks)
    with pytest.raises(verbs.InvalidRequest):
        verbs.thermal(H, [1.0], sectors=blocks, method="qmc")
    with pytest.raises(verbs.InvalidRequest):
        verbs.thermal(H, [1.0], sectors=blocks, samples=0)
    with pytest.raises(verbs.InvalidRequest):
        verbs.thermal(H, [1.0], sectors=blocks, krylov=1)
    Sq = ops.from_products(8, ops.sz_q_products(8, np.pi))
    with pytest.raises(verbs.InvalidRequest):
        verbs.dynamics(H, Sq, source=blocks[0], target=lat.chain_sector(8, 4, 4), omega=[], eta=0.1)
    with pytest.raises(verbs.InvalidRequest):
        verbs.dynamics(H, Sq, source=blocks[0], target=lat.chain_sector(8, 4, 4), omega=[0.0], eta=0.0)


def test_cpu_device_is_the_reference_lane():
    with pytest.raises(verbs.DeviceUnsupported):
        verbs.eigs(_model(), 1, sectors=[lat.chain_sector(8, 4, 0)], device="cpu")


def test_gpu_without_a_device_is_an_error():
    if not _no_device():
        pytest.skip("a CUDA device is visible here")
    for dev in ("gpu", "auto"):
        with pytest.raises(verbs.DeviceUnavailable):
            verbs.eigs(_model(), 1, sectors=[lat.chain_sector(8, 4, 0)], device=dev)
