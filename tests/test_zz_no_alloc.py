"""qb_lanczos_noalloc: the Lanczos kernel for callers that cannot let a library allocate device memory.

Such a caller (a framework whose caching allocator already holds the device, or a service with a memory
plan fixed at start-up) passes every buffer itself; the entry point keeps its own small scratch in a
file-scope device array. This file is collected last so a run that stops at its first failure has run
everything else first. It compares the entry point's alpha / beta with qb_lanczos's, the existing entry
point, to 1e-12 absolute, on two calls in a row (the second must start from a cleared scratch), for both
reorthogonalisation options the entry point accepts and on the default stream as well as a stream the caller
made.
"""
import numpy as np
import pytest

from qed_spin_b200 import lattice as lat
from qed_spin_b200 import operators as ops

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _noalloc(D, S, P, v0_dev, max_iter, dtype, reorth=None, stream=None):
    import ctypes as C
    from qed_spin_b200 import _lib
    reorth = _lib.QB_REORTH_NONE if reorth is None else reorth
    es = 8 if dtype == "c64" else 16
    work = torch.empty(S.dim * (2 * es + 16), dtype=torch.uint8, device="cuda")   # the caller's buffer
    a = np.zeros(max_iter)
    b = np.zeros(max_iter + 1)
    it = C.c_int()
    if stream is not None:   # the caller's buffers were written on the current stream
        stream.wait_stream(torch.cuda.current_stream())
    _lib.check(_lib.lib().qb_lanczos_noalloc(S.h, P.h, v0_dev.data_ptr(), work.data_ptr(), max_iter, reorth,
                                             1e-300, D._dt(dtype), a.ctypes.data, b.ctypes.data, C.byref(it),
                                             None if stream is None else C.c_void_p(stream.cuda_stream)))
    m = it.value
    return a[:m], b[: m + 1]


@pytest.mark.parametrize("on_stream", [False, True])
@pytest.mark.parametrize("reorth", ["none", "local"])
@pytest.mark.parametrize("dtype", ["c128", "c64"])
def test_noalloc_matches_qb_lanczos_twice(dtype, reorth, on_stream):
    if not torch.cuda.is_available():
        pytest.fail("a GPU test ran without a CUDA device")
    from qed_spin_b200 import _lib
    from qed_spin_b200 import build
    from qed_spin_b200 import device as D
    build.build()
    spec = lat.chain_sector(16, 8, 3)
    prog = ops.row_program(ops.from_products(16, ops.xxz_products(lat.chain_bonds(16), 1.0, 0.7)))
    S = D.Sector(spec)
    P = D.Program(prog)
    rng = np.random.default_rng(11)
    for call in range(2):   # two calls in a row: the shared scratch must not leak between them
        v0 = rng.normal(size=S.dim) + 1j * rng.normal(size=S.dim)
        ro = {"none": _lib.QB_REORTH_NONE, "local": _lib.QB_REORTH_LOCAL}[reorth]
        a_ref, b_ref = D.lanczos(S, P, v0, 40, reorth=ro, dtype=dtype)
        stream = torch.cuda.Stream() if on_stream else None
        a, b = _noalloc(D, S, P, torch.from_numpy(v0).cuda(), 40, dtype, reorth=ro, stream=stream)
        assert len(a) == len(a_ref) == 40, call
        np.testing.assert_allclose(a, a_ref, rtol=0, atol=1e-12)
        np.testing.assert_allclose(b, b_ref, rtol=0, atol=1e-12)


def test_noalloc_refuses_past_its_maximum():
    if not torch.cuda.is_available():
        pytest.fail("a GPU test ran without a CUDA device")
    from qed_spin_b200 import _lib
    from qed_spin_b200 import device as D
    spec = lat.chain_sector(12, 6, 0)
    prog = ops.row_program(ops.from_products(12, ops.heisenberg_products(lat.chain_bonds(12))))
    S = D.Sector(spec)
    P = D.Program(prog)
    v0 = torch.ones(S.dim, dtype=torch.complex128, device="cuda")
    with pytest.raises(ValueError, match="QB_NOALLOC_MAX_ITER"):
        _noalloc(D, S, P, v0, _lib.QB_NOALLOC_MAX_ITER + 1, "c128")
