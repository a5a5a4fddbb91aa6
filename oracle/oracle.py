"""TEST INFRASTRUCTURE: ctypes access to the restated CPU oracle (oracle/libqed_oracle.so).

The oracle restates the reference engine's CPU algorithm (every function in qed_oracle.cpp cites the
reference file:line it follows) and is pinned against the reference itself (oracle/_ref) and the golden
fixtures under tests/golden. Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU baseline import it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "libqed_oracle.so")
_lib = None

_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")


def build():
    subprocess.run(["make", "-C", _HERE, "libqed_oracle.so"], check=True, stdout=subprocess.DEVNULL)


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        build()
    L = C.CDLL(_LIB_PATH)
    vp = C.c_void_p
    L.qo_last_error.restype = C.c_char_p
    L.qo_sector_new.restype = vp
    L.qo_sector_new.argtypes = [C.c_int, C.c_int, C.c_int, _i32p, vp, _f64p, C.c_int]
    L.qo_sector_free.argtypes = [vp]
    L.qo_sector_dim.restype = C.c_uint64
    L.qo_sector_dim.argtypes = [vp]
    L.qo_sector_get.argtypes = [vp, _u64p, _f64p]
    L.qo_sector_slc.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_int), _i32p]
    L.qo_index_and_projection.restype = C.c_int64
    L.qo_index_and_projection.argtypes = [vp, C.c_uint64, _f64p]
    L.qo_prog_new.restype = vp
    L.qo_prog_new.argtypes = [C.c_uint32, _u64p, _i32p, _u32p, C.c_uint32, _u64p, _u32p, C.c_uint32, _u64p, _f64p]
    L.qo_prog_free.argtypes = [vp]
    L.qo_gather.argtypes = [vp, vp, vp, _f64p, _f64p]
    L.qo_csr.argtypes = [vp, vp, vp, _u64p, vp, vp]
    L.qo_count_emitted.argtypes = [vp, vp, vp, C.POINTER(C.c_uint64)]
    L.qo_lanczos.argtypes = [vp, vp, _f64p, C.c_int, C.c_int, C.c_double, _f64p, _f64p, C.POINTER(C.c_int)]
    L.qo_scan_lowest.argtypes = [vp, vp, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.qo_tridiag_eig.argtypes = [_f64p, _f64p, C.c_int, _f64p, vp]
    L.qo_sample_vector.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64, _f64p]
    L.qo_staged_seed.argtypes = [C.c_uint64, C.c_uint64, _f64p]
    L.qo_ftlm.argtypes = [vp, vp, C.c_int, C.c_int, C.c_uint64, _f64p, C.c_int, _f64p, _f64p, _f64p,
                          C.POINTER(C.c_double)]
    L.qo_sample_moments.argtypes = [_f64p, _f64p, C.c_int, _f64p, C.c_int, C.POINTER(C.c_double), _f64p, _f64p,
                                    _f64p]
    L.qo_continued_fraction.argtypes = [_f64p, _f64p, C.c_int, _f64p, C.c_int, C.c_double, C.c_double, _f64p]
    L.qo_cf.argtypes = [vp, vp, _f64p, C.c_int, _f64p, C.c_int, C.c_double, C.c_double, C.c_double, _f64p,
                        C.POINTER(C.c_double)]
    _lib = L
    return L


def _check(rc):
    if rc != 0:
        raise RuntimeError(lib().qo_last_error().decode())


class Program:
    def __init__(self, prog):
        """prog: a qed_spin_b200.operators.Program (or any object with the same arrays)."""
        self.src = prog
        self._keep = [
            np.ascontiguousarray(prog.group_flip, np.uint64),
            np.ascontiguousarray(prog.group_setbits, np.int32),
            np.ascontiguousarray(prog.group_vbegin, np.uint32),
            np.ascontiguousarray(prog.vsub_val, np.uint64),
            np.ascontiguousarray(prog.vsub_tbegin, np.uint32),
            np.ascontiguousarray(prog.term_sign, np.uint64),
            np.ascontiguousarray(np.asarray(prog.term_coeff, np.complex128)).view(np.float64),
        ]
        k = self._keep
        self.h = lib().qo_prog_new(len(k[0]), k[0], k[1], k[2], len(k[3]), k[3], k[4], len(k[5]), k[5], k[6])

    def __del__(self):
        if getattr(self, "h", None):
            lib().qo_prog_free(self.h)
            self.h = None


class Sector:
    def __init__(self, spec, slc_mode=-1):
        L = lib()
        perms = np.ascontiguousarray(spec.perms, np.int32)
        chars = np.asarray(spec.chars, np.complex128)
        ch = np.ascontiguousarray(np.stack([chars.real, chars.imag], 1).reshape(-1))
        self._flips = None if spec.flips is None else np.ascontiguousarray(spec.flips, np.uint64)
        fp = None if self._flips is None else self._flips.ctypes.data
        self.h = L.qo_sector_new(spec.n_sites, spec.n_up, perms.shape[0], perms.reshape(-1), fp, ch, slc_mode)
        if not self.h:
            raise RuntimeError(L.qo_last_error().decode())
        self.spec = spec

    def __del__(self):
        if getattr(self, "h", None):
            lib().qo_sector_free(self.h)
            self.h = None

    @property
    def dim(self) -> int:
        return int(lib().qo_sector_dim(self.h))

    def reps(self):
        d = self.dim
        reps = np.zeros(d, np.uint64)
        inv = np.zeros(d, np.float64)
        lib().qo_sector_get(self.h, reps, inv)
        return reps, inv

    def sublattice(self):
        L_, m = C.c_int(), C.c_int()
        kb = np.zeros(self.spec.n_sites, np.int32)
        if not lib().qo_sector_slc(self.h, C.byref(L_), C.byref(m), kb):
            return None
        return dict(L=L_.value, m=m.value, key_bit=kb)

    def index_and_projection(self, state: int):
        p = np.zeros(2)
        k = lib().qo_index_and_projection(self.h, int(state), p)
        return int(k), complex(p[0], p[1])

    def gather(self, prog: Program, x, col: "Sector" = None):
        col = self if col is None else col
        x = np.ascontiguousarray(x, np.complex128)
        y = np.zeros(self.dim, np.complex128)
        _check(lib().qo_gather(self.h, col.h, prog.h, x.view(np.float64), y.view(np.float64)))
        return y

    def csr(self, prog: Program, col: "Sector" = None):
        col = self if col is None else col
        rp = np.zeros(self.dim + 1, np.uint64)
        _check(lib().qo_csr(self.h, col.h, prog.h, rp, None, None))
        nnz = int(rp[-1])
        c = np.zeros(max(nnz, 1), np.uint32)
        v = np.zeros(2 * max(nnz, 1), np.float64)
        _check(lib().qo_csr(self.h, col.h, prog.h, rp, c.ctypes.data, v.ctypes.data))
        return rp, c[:nnz], v.view(np.complex128)[:nnz]

    def count_emitted(self, prog: Program, col: "Sector" = None) -> int:
        col = self if col is None else col
        n = C.c_uint64()
        _check(lib().qo_count_emitted(self.h, col.h, prog.h, C.byref(n)))
        return int(n.value)

    def lanczos(self, prog: Program, v0, max_iter, reorth=0, breakdown_tol=1e-300):
        v0 = np.ascontiguousarray(v0, np.complex128)
        a = np.zeros(max_iter)
        b = np.zeros(max_iter + 1)
        it = C.c_int()
        _check(lib().qo_lanczos(self.h, prog.h, v0.view(np.float64), max_iter, reorth, breakdown_tol, a, b,
                                C.byref(it)))
        m = it.value
        return a[:m].copy(), b[: m + 1].copy()

    def scan_lowest(self, prog: Program, max_iter=0):
        e, it, cv = C.c_double(), C.c_int(), C.c_int()
        _check(lib().qo_scan_lowest(self.h, prog.h, max_iter, C.byref(e), C.byref(it), C.byref(cv)))
        return e.value, it.value, bool(cv.value)

    def ftlm(self, prog: Program, samples, depth, seed, betas):
        betas = np.ascontiguousarray(betas, np.float64)
        nb = len(betas)
        lnZ, E, V = np.zeros(nb), np.zeros(nb), np.zeros(nb)
        gs = C.c_double()
        _check(lib().qo_ftlm(self.h, prog.h, samples, depth, seed, betas, nb, lnZ, E, V, C.byref(gs)))
        return dict(lnZ=lnZ, E=E, V=V, e_min=gs.value)

    def cf(self, prog: Program, phi, depth, omega, eta, shift=float("nan"), tolerance=1e-12):
        phi = np.ascontiguousarray(phi, np.complex128)
        omega = np.ascontiguousarray(omega, np.float64)
        S = np.zeros(len(omega))
        sh = C.c_double()
        _check(lib().qo_cf(self.h, prog.h, phi.view(np.float64), depth, omega, len(omega), eta, shift, tolerance, S,
                           C.byref(sh)))
        return S, sh.value


def tridiag_eig(alpha, beta, vectors=True):
    a = np.ascontiguousarray(alpha, np.float64)
    m = len(a)
    b = np.zeros(m + 1)
    b[: min(len(beta), m + 1)] = np.asarray(beta)[: m + 1]
    vals = np.zeros(m)
    vecs = np.zeros(m * m) if vectors else None
    _check(lib().qo_tridiag_eig(a, b, m, vals, None if vecs is None else vecs.ctypes.data))
    return vals, (None if vecs is None else vecs.reshape(m, m).T)


def sample_moments(alpha, beta, betas):
    a = np.ascontiguousarray(alpha, np.float64)
    m = len(a)
    b = np.zeros(m + 1)
    b[: min(len(beta), m + 1)] = np.asarray(beta)[: m + 1]
    betas = np.ascontiguousarray(betas, np.float64)
    nb = len(betas)
    Z, E1, E2 = np.zeros(nb), np.zeros(nb), np.zeros(nb)
    em = C.c_double()
    _check(lib().qo_sample_moments(a, b, m, betas, nb, C.byref(em), Z, E1, E2))
    return em.value, Z, E1, E2


def continued_fraction(alpha, beta, omega, eta, norm_sq):
    a = np.ascontiguousarray(alpha, np.float64)
    m = len(a)
    b = np.zeros(m + 1)
    b[: min(len(beta), m + 1)] = np.asarray(beta)[: m + 1]
    omega = np.ascontiguousarray(omega, np.float64)
    S = np.zeros(len(omega))
    lib().qo_continued_fraction(a, b, m, omega, len(omega), eta, norm_sq, S)
    return S


def sample_vector(seed: int, s: int, n: int):
    out = np.zeros(2 * n)
    lib().qo_sample_vector(seed, s, n, out)
    return out.view(np.complex128)


def staged_seed(seed: int, n: int):
    out = np.zeros(2 * n)
    lib().qo_staged_seed(seed, n, out)
    return out.view(np.complex128)


def combine_blocks(curves, betas, weights=None):
    """Log-space combine of per-block FTLM curves into the whole system's thermodynamics (the thermal
    driver's combine, src/engine/thermal.cpp:608-641): p_b = w_b exp(lnZ_b - max), lnZ = max + ln sum p_b,
    E = sum p_b E_b / Z, C = beta^2 sum p_b (V_b + (E_b - E)^2) / Z (law of total variance), S = lnZ + beta E,
    F = -lnZ / beta. Sums run over the blocks in order, as there."""
    betas = np.asarray(betas, np.float64)
    nb = len(curves)
    w = np.ones(nb) if weights is None else np.asarray(weights, np.float64)
    out = {k: np.zeros(len(betas)) for k in ("lnZ", "E", "C", "S", "F")}
    for i, bt in enumerate(betas):
        mx = max(np.log(w[b]) + curves[b]["lnZ"][i] for b in range(nb))
        p = [np.exp(np.log(w[b]) + curves[b]["lnZ"][i] - mx) for b in range(nb)]
        z = 0.0
        e = 0.0
        for b in range(nb):
            z += p[b]
            e += p[b] * curves[b]["E"][i]
        e /= z
        var = 0.0
        for b in range(nb):
            d = curves[b]["E"][i] - e
            var += p[b] * (curves[b]["V"][i] + d * d)
        var /= z
        out["lnZ"][i] = mx + np.log(z)
        out["E"][i] = e
        out["C"][i] = bt * bt * var
        out["S"][i] = out["lnZ"][i] + bt * e
        out["F"][i] = -out["lnZ"][i] / bt
    return out
