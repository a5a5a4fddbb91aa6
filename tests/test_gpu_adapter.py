"""The reference-side binding run for real: include/qed_b200_linear_operator.hpp (the ed::LinearOperator a
maintainer of the reference binds in place of its device lane) linked with the reference engine's own code
(oracle/_ref/libqed_adapter.so, built by oracle/Makefile) and this library.

For each fixture case: apply() (host buffers) and bind_cuda() (device buffers) give the reference's y = H x bit for
bit; a wrong length is refused by bind_cuda and bind_cuda_multi; norm_bound() is the program's coefficient sum for
the one- and two-sector constructors; and the reference's own lanczos_kernel<CpuBackend>, run over apply(), gives
the reference's alpha / beta (fixtures lz_alpha / lz_beta, the reference's kernel over its own walk) within 1e-12
over 40 steps (its BLAS may sum in another order on another CPU).
"""
import ctypes as C
import os

import numpy as np
import pytest

from cases import CASES, NAMES
from conftest import ROOT
from qed_spin_b200 import operators as ops

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

LIB = os.path.join(ROOT, "oracle", "_ref", "libqed_adapter.so")
CASE = {c[0]: c for c in CASES}


@pytest.fixture(scope="module")
def adapter():
    if not torch.cuda.is_available():
        pytest.fail("a GPU test ran without a CUDA device")
    if not os.path.exists(LIB):
        pytest.fail("oracle/_ref/libqed_adapter.so is not built (oracle/Makefile, run by __graft_entry__.build())")
    from qed_spin_b200 import build
    build.build()
    L = C.CDLL(LIB)
    L.qad_last_error.restype = C.c_char_p
    vp = C.c_void_p
    L.qad_run.argtypes = [C.c_int, C.c_int, C.c_int, vp, vp, vp, vp, vp, C.c_uint64, C.c_int, C.c_int, C.c_char_p, vp,
                          vp, vp, vp, vp, vp, vp, C.c_int, vp, vp, C.POINTER(C.c_int), C.POINTER(C.c_double),
                          C.POINTER(C.c_double)]
    return L


@pytest.mark.parametrize("name", NAMES)
def test_reference_lanczos_through_the_binding(adapter, fixtures, name):
    from qed_spin_b200 import device as D
    _, spec, prods = CASE[name]
    N = spec.n_sites
    perms = np.ascontiguousarray(spec.perms, np.int32)
    G = perms.shape[0]
    flips = None if spec.flips is None else np.ascontiguousarray(spec.flips, np.uint64)
    chars = np.ascontiguousarray(np.asarray(spec.chars, np.complex128)).view(np.float64)
    reps = np.ascontiguousarray(fixtures[f"{name}/reps"], np.uint64)
    inv = np.ascontiguousarray(fixtures[f"{name}/inv_norms"], np.float64)
    slc = 0 if D.key_order(spec, sublattice_mode=-1) is None else 1
    opstr = "".join(p[0] for p in prods).encode()
    nfac = np.array([len(p[0]) for p in prods], np.int32)
    sites = np.ascontiguousarray(np.concatenate([np.asarray(p[1], np.int32) for p in prods]), np.int32)
    coeffs = np.ascontiguousarray(np.array([complex(p[2]) for p in prods], np.complex128)).view(np.float64)
    x = np.ascontiguousarray(fixtures[f"{name}/x"], np.complex128)
    n = len(reps)
    y_apply = np.zeros(n, np.complex128)
    y_bind = np.zeros(n, np.complex128)
    m = 40
    a = np.zeros(m)
    b = np.zeros(m + 1)
    it, nb, xnb = C.c_int(), C.c_double(), C.c_double()
    rc = adapter.qad_run(N, spec.n_up, G, perms.ctypes.data, None if flips is None else flips.ctypes.data,
                         chars.ctypes.data, reps.ctypes.data, inv.ctypes.data, n, slc, len(prods), opstr,
                         nfac.ctypes.data, sites.ctypes.data, coeffs.ctypes.data, x.ctypes.data, y_apply.ctypes.data,
                         y_bind.ctypes.data, x.ctypes.data, m, a.ctypes.data, b.ctypes.data, C.byref(it),
                         C.byref(nb), C.byref(xnb))
    assert rc == 0, adapter.qad_last_error().decode()
    y_ref = fixtures[f"{name}/y"]
    assert np.array_equal(y_apply.view(np.uint64), y_ref.view(np.uint64))
    assert np.array_equal(y_bind.view(np.uint64), y_ref.view(np.uint64))
    scale = float(np.abs(np.asarray(ops.row_program(ops.from_products(N, prods)).term_coeff)).sum())
    assert nb.value == pytest.approx(scale, rel=1e-14) and xnb.value == nb.value
    assert it.value == m
    np.testing.assert_allclose(a, fixtures[f"{name}/lz_alpha"], rtol=0, atol=1e-12)
    np.testing.assert_allclose(b, fixtures[f"{name}/lz_beta"], rtol=0, atol=1e-12)
