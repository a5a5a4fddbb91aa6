"""TEST INFRASTRUCTURE: ctypes access to the reference engine's own CPU code (oracle/_ref/libqed_ref.so,
built by oracle/Makefile from the reference sources).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline / reference legs import this module;
the product never does. ``available()`` is False when the library was not built (the reference sources
were absent when the tree was assembled).
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_ref", "libqed_ref.so")
_lib = None

_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")


def available() -> bool:
    return os.path.exists(_LIB_PATH)


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not available():
        raise RuntimeError(f"reference library not built: {_LIB_PATH}")
    L = C.CDLL(_LIB_PATH)
    vp = C.c_void_p
    L.qref_last_error.restype = C.c_char_p
    L.qref_op_new.restype = vp
    L.qref_op_new.argtypes = [C.c_int]
    L.qref_op_free.argtypes = [vp]
    L.qref_op_add_product.argtypes = [vp, C.c_char_p, _i32p, C.c_int, C.c_double, C.c_double]
    L.qref_prog_rows.restype = vp
    L.qref_prog_rows.argtypes = [vp]
    L.qref_prog_cross.restype = vp
    L.qref_prog_cross.argtypes = [vp, vp, vp]
    L.qref_prog_free.argtypes = [vp]
    L.qref_prog_sizes.argtypes = [vp, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]
    L.qref_prog_arrays.argtypes = [vp, _u64p, _i32p, _u32p, _u64p, _u32p, _u64p, _f64p]
    L.qref_sector_new.restype = vp
    L.qref_sector_new.argtypes = [C.c_int, C.c_int, C.c_int, _i32p, vp, _f64p, C.c_int, C.c_int]
    L.qref_sector_free.argtypes = [vp]
    L.qref_sector_dim.restype = C.c_uint64
    L.qref_sector_dim.argtypes = [vp]
    L.qref_sector_scanned.restype = C.c_uint64
    L.qref_sector_scanned.argtypes = [vp]
    L.qref_sector_get.argtypes = [vp, _u64p, _f64p]
    L.qref_sector_slc.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_double)]
    L.qref_sector_slc_keybits.argtypes = [vp, _i32p]
    L.qref_index_and_projection.restype = C.c_int64
    L.qref_index_and_projection.argtypes = [vp, C.c_uint64, _f64p]
    L.qref_gather.argtypes = [vp, vp, _f64p, _f64p]
    L.qref_key_order.argtypes = [C.c_int, C.c_int, _i32p, vp, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                 C.POINTER(C.c_uint64), vp, vp, vp, vp]
    L.qref_cross_gather.argtypes = [vp, vp, vp, _f64p, _f64p]
    L.qref_gather_rows.argtypes = [vp, vp, _f64p, _u64p, C.c_uint64, _f64p]
    L.qref_csr_build.restype = vp
    L.qref_csr_build.argtypes = [vp, vp]
    L.qref_csr_free.argtypes = [vp]
    L.qref_csr_nnz.restype = C.c_uint64
    L.qref_csr_nnz.argtypes = [vp]
    L.qref_csr_get.argtypes = [vp, _u64p, _u32p, _f64p]
    L.qref_csr_spmv.argtypes = [vp, _f64p, _f64p]
    L.qref_csr_spmv_real.argtypes = [vp, _f64p, _f64p]
    L.qref_csr_build_rows.restype = vp
    L.qref_csr_build_rows.argtypes = [vp, vp, C.c_uint64, C.c_uint64]
    L.qref_csr_build_rowlist.restype = vp
    L.qref_csr_build_rowlist.argtypes = [vp, vp, _u64p, C.c_uint64]
    L.qref_ftlm_blocks.argtypes = [vp, vp, C.c_int, C.c_int, C.c_int, C.c_uint64, _f64p, C.c_int, _f64p, _f64p,
                                   _f64p, _f64p]
    L.qref_csr_bytes.restype = C.c_uint64
    L.qref_csr_bytes.argtypes = [vp]
    L.qref_sample_vector.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64, _f64p]
    L.qref_staged_seed.argtypes = [C.c_uint64, C.c_uint64, _f64p]
    L.qref_lanczos.argtypes = [vp, vp, _f64p, C.c_int, C.c_int, C.c_double, _f64p, _f64p, C.POINTER(C.c_int)]
    L.qref_scan_lowest.argtypes = [vp, vp, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.qref_ks_lowest.argtypes = [vp, vp, C.c_int, _f64p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int)]
    L.qref_ks_lowest_lane.argtypes = [vp, vp, C.c_int, C.c_int, _f64p, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                      C.POINTER(C.c_int)]
    L.qref_ftlm.argtypes = [vp, vp, C.c_int, C.c_int, C.c_uint64, _f64p, C.c_int, _f64p, _f64p, _f64p,
                            C.POINTER(C.c_double)]
    L.qref_cf.argtypes = [vp, vp, _f64p, C.c_int, _f64p, C.c_int, C.c_double, C.c_double, C.c_double, _f64p,
                          C.POINTER(C.c_double), C.POINTER(C.c_double)]
    L.qref_tridiag_eig.argtypes = [_f64p, _f64p, C.c_int, _f64p, C.c_void_p]
    L.qref_set_threads.argtypes = [C.c_int]
    L.qref_max_threads.restype = C.c_int
    _lib = L
    return L


def _check(rc):
    if rc != 0:
        raise RuntimeError(lib().qref_last_error().decode())


class Operator:
    """The reference's MaskedOperator: a sum of products coeff * prod ops[k](sites[k])."""

    def __init__(self, n_sites: int, products):
        L = lib()
        self.n = n_sites
        self.h = L.qref_op_new(n_sites)
        for ops, sites, coeff in products:
            s = np.ascontiguousarray(sites, dtype=np.int32)
            c = complex(coeff)
            _check(L.qref_op_add_product(self.h, ops.encode(), s, len(ops), c.real, c.imag))

    def __del__(self):
        if getattr(self, "h", None):
            lib().qref_op_free(self.h)
            self.h = None

    def row_program(self) -> "Program":
        return Program(lib().qref_prog_rows(self.h))

    def cross_program(self, row: "Sector", col: "Sector") -> "Program":
        p = lib().qref_prog_cross(self.h, row.h, col.h)
        if not p:
            raise RuntimeError(lib().qref_last_error().decode())
        return Program(p)


class Program:
    def __init__(self, h):
        self.h = h

    def __del__(self):
        if getattr(self, "h", None):
            lib().qref_prog_free(self.h)
            self.h = None

    def arrays(self) -> dict:
        L = lib()
        g, v, t = C.c_uint32(), C.c_uint32(), C.c_uint32()
        L.qref_prog_sizes(self.h, C.byref(g), C.byref(v), C.byref(t))
        G, V, T = g.value, v.value, t.value
        out = dict(
            group_flip=np.zeros(G, np.uint64),
            group_setbits=np.zeros(G, np.int32),
            group_vbegin=np.zeros(G + 1, np.uint32),
            vsub_val=np.zeros(V, np.uint64),
            vsub_tbegin=np.zeros(V + 1, np.uint32),
            term_sign=np.zeros(T, np.uint64),
            term_coeff=np.zeros(2 * T, np.float64),
        )
        L.qref_prog_arrays(self.h, out["group_flip"], out["group_setbits"], out["group_vbegin"], out["vsub_val"],
                           out["vsub_tbegin"], out["term_sign"], out["term_coeff"])
        return out


class Sector:
    """The reference's RepSectorData for a fixed-Sz sector of a group given by its elements."""

    def __init__(self, n_sites, n_up, perms, chars, flips=None, slc_mode=-1, lookup=0):
        L = lib()
        perms = np.ascontiguousarray(perms, dtype=np.int32)
        G = perms.shape[0]
        ch = np.ascontiguousarray(np.stack([np.real(chars), np.imag(chars)], axis=1).reshape(-1), dtype=np.float64)
        self._flips = None if flips is None else np.ascontiguousarray(flips, dtype=np.uint64)
        fp = None if self._flips is None else self._flips.ctypes.data
        self.h = L.qref_sector_new(n_sites, n_up, G, perms.reshape(-1), fp, ch, slc_mode, lookup)
        if not self.h:
            raise RuntimeError(L.qref_last_error().decode())
        self.n_sites, self.n_up, self.G = n_sites, n_up, G

    def __del__(self):
        if getattr(self, "h", None):
            lib().qref_sector_free(self.h)
            self.h = None

    @property
    def dim(self) -> int:
        return int(lib().qref_sector_dim(self.h))

    def reps(self):
        d = self.dim
        reps = np.zeros(d, np.uint64)
        inv = np.zeros(d, np.float64)
        lib().qref_sector_get(self.h, reps, inv)
        return reps, inv

    def sublattice(self):
        L_, m, mc = C.c_int(), C.c_int(), C.c_double()
        if not lib().qref_sector_slc(self.h, C.byref(L_), C.byref(m), C.byref(mc)):
            return None
        kb = np.zeros(self.n_sites, np.int32)
        lib().qref_sector_slc_keybits(self.h, kb)
        return dict(L=L_.value, m=m.value, mean_candidates=mc.value, key_bit=kb)

    def index_and_projection(self, state: int):
        p = np.zeros(2, np.float64)
        k = lib().qref_index_and_projection(self.h, int(state), p)
        return int(k), complex(p[0], p[1])

    def gather(self, prog: Program, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.complex128)
        y = np.zeros(self.dim, np.complex128)
        _check(lib().qref_gather(self.h, prog.h, x.view(np.float64), y.view(np.float64)))
        return y

    def gather_rows(self, prog: Program, x: np.ndarray, rows: np.ndarray) -> np.ndarray:
        """Rows `rows` of O x by the reference's row walk (for_each_sector_entry), OpenMP over the rows."""
        x = np.ascontiguousarray(x, dtype=np.complex128)
        rows = np.ascontiguousarray(rows, dtype=np.uint64)
        y = np.zeros(len(rows), np.complex128)
        _check(lib().qref_gather_rows(self.h, prog.h, x.view(np.float64), rows, len(rows), y.view(np.float64)))
        return y

    def csr(self, prog: Program, x=None):
        """The merged reduced CSR (row_ptr, col, val); with x, also the reference's CSR spmv of x."""
        L = lib()
        c = L.qref_csr_build(self.h, prog.h)
        nnz = int(L.qref_csr_nnz(c))
        rp = np.zeros(self.dim + 1, np.uint64)
        col = np.zeros(nnz, np.uint32)
        val = np.zeros(2 * nnz, np.float64)
        L.qref_csr_get(c, rp, col, val)
        y = None
        if x is not None:
            x = np.ascontiguousarray(x, dtype=np.complex128)
            y = np.zeros(self.dim, np.complex128)
            rc = L.qref_csr_spmv(c, x.view(np.float64), y.view(np.float64))
        L.qref_csr_free(c)
        if x is not None:
            _check(rc)
            return rp, col, val.view(np.complex128), y
        return rp, col, val.view(np.complex128)

    def csr_handle(self, prog: Program) -> "Csr":
        return Csr(self, prog)

    def lanczos(self, prog: Program, v0, max_iter, reorth=0, breakdown_tol=1e-300):
        v0 = np.ascontiguousarray(v0, dtype=np.complex128)
        a = np.zeros(max_iter, np.float64)
        b = np.zeros(max_iter + 1, np.float64)
        it = C.c_int()
        _check(lib().qref_lanczos(self.h, prog.h, v0.view(np.float64), max_iter, reorth, breakdown_tol, a, b,
                                  C.byref(it)))
        m = it.value
        return a[:m].copy(), b[: m + 1].copy()

    def scan_lowest(self, prog: Program, max_iter=0):
        e, it, conv = C.c_double(), C.c_int(), C.c_int()
        _check(lib().qref_scan_lowest(self.h, prog.h, max_iter, C.byref(e), C.byref(it), C.byref(conv)))
        return e.value, it.value, bool(conv.value)

    def ks_lowest(self, prog: Program, k, use_csr=False):
        """The reference's krylov_schur_kernel on the block, applying H through its walk or (use_csr) its
        merged reduced CSR, the host default lane."""
        ev = np.zeros(k, np.float64)
        n, conv, ap = C.c_int(), C.c_int(), C.c_int()
        _check(lib().qref_ks_lowest_lane(self.h, prog.h, k, int(bool(use_csr)), ev, C.byref(n), C.byref(conv),
                                         C.byref(ap)))
        return ev[: n.value].copy(), bool(conv.value), ap.value

    def ftlm(self, prog: Program, samples, depth, seed, betas):
        betas = np.ascontiguousarray(betas, dtype=np.float64)
        nb = len(betas)
        lnZ, E, V = np.zeros(nb), np.zeros(nb), np.zeros(nb)
        gs = C.c_double()
        _check(lib().qref_ftlm(self.h, prog.h, samples, depth, seed, betas, nb, lnZ, E, V, C.byref(gs)))
        return dict(lnZ=lnZ, E=E, V=V, e_min=gs.value)

    def cf(self, prog: Program, phi, depth, omega, eta, shift=float("nan"), tolerance=1e-12):
        phi = np.ascontiguousarray(phi, dtype=np.complex128)
        omega = np.ascontiguousarray(omega, dtype=np.float64)
        S = np.zeros(len(omega))
        sh, cc = C.c_double(), C.c_double()
        _check(lib().qref_cf(self.h, prog.h, phi.view(np.float64), depth, omega, len(omega), eta, shift, tolerance,
                             S, C.byref(sh), C.byref(cc)))
        return S, sh.value, cc.value


def cross_gather(row: Sector, col: Sector, prog: Program, x):
    x = np.ascontiguousarray(x, dtype=np.complex128)
    y = np.zeros(row.dim, np.complex128)
    _check(lib().qref_cross_gather(row.h, col.h, prog.h, x.view(np.float64), y.view(np.float64)))
    return y


def sample_vector(seed: int, s: int, n: int) -> np.ndarray:
    out = np.zeros(2 * n, np.float64)
    lib().qref_sample_vector(seed, s, n, out)
    return out.view(np.complex128)


def staged_seed(seed: int, n: int) -> np.ndarray:
    out = np.zeros(2 * n, np.float64)
    lib().qref_staged_seed(seed, n, out)
    return out.view(np.complex128)


def key_order(n_sites, perms, flips=None, mode=-1):
    """The reference's sublattice code of a group and its tables (SublatticeCode), or None."""
    L = lib()
    perms = np.ascontiguousarray(perms, np.int32)
    fl = None if flips is None else np.ascontiguousarray(flips, np.uint64)
    G = perms.shape[0]
    Lb, mb, nc = C.c_int(), C.c_int(), C.c_uint64()
    fp = None if fl is None else fl.ctypes.data
    _check(L.qref_key_order(n_sites, G, perms.reshape(-1), fp, mode, C.byref(Lb), C.byref(mb), C.byref(nc), None,
                            None, None, None))
    if Lb.value == 0:
        return None
    P = mb.value << Lb.value
    kb = np.zeros(n_sites, np.int32)
    lead = np.zeros(P, np.uint16)
    off = np.zeros(P + 1, np.uint32)
    cand = np.zeros(max(1, nc.value), np.uint16)
    _check(L.qref_key_order(n_sites, G, perms.reshape(-1), fp, mode, C.byref(Lb), C.byref(mb), C.byref(nc),
                            kb.ctypes.data, lead.ctypes.data, off.ctypes.data, cand.ctypes.data))
    return {"L": Lb.value, "m": mb.value, "key_bit": kb, "lead": lead, "cand_off": off, "cand": cand[: nc.value]}


def tridiag_eig(alpha, beta, vectors=True):
    a = np.ascontiguousarray(alpha, dtype=np.float64)
    m = len(a)
    b = np.zeros(m + 1)
    b[: min(len(beta), m + 1)] = beta[: m + 1]
    vals = np.zeros(m)
    vecs = np.zeros(m * m) if vectors else None
    _check(lib().qref_tridiag_eig(a, b, m, vals, None if vecs is None else vecs.ctypes.data))
    return vals, (None if vecs is None else vecs.reshape(m, m).T)


def set_threads(n: int):
    lib().qref_set_threads(n)


def max_threads() -> int:
    return int(lib().qref_max_threads())


class Csr:
    """The reference's ReducedSymmetryCsr of a program on one sector, kept for repeated spmv."""

    def __init__(self, sector: "Sector", prog: Program, rows=None):
        """rows: None for every row, (r0, n) for the merged rows r0 .. r0 + n - 1 alone, or an array of rows
        (columns over the whole sector)."""
        L = lib()
        if rows is None:
            self.dim = sector.dim
            self.h = L.qref_csr_build(sector.h, prog.h)
        elif isinstance(rows, np.ndarray):
            rows = np.ascontiguousarray(rows, np.uint64)
            self.dim = len(rows)
            self.h = L.qref_csr_build_rowlist(sector.h, prog.h, rows, len(rows))
        else:
            self.dim = int(rows[1])
            self.h = L.qref_csr_build_rows(sector.h, prog.h, int(rows[0]), int(rows[1]))
        if not self.h:
            raise RuntimeError(L.qref_last_error().decode())

    @property
    def nnz(self) -> int:
        return int(lib().qref_csr_nnz(self.h))

    @property
    def bytes(self) -> int:
        return int(lib().qref_csr_bytes(self.h))

    def spmv(self, x: np.ndarray, y: np.ndarray) -> None:
        _check(lib().qref_csr_spmv(self.h, x.view(np.float64), y.view(np.float64)))

    def arrays(self):
        """row_ptr (rows + 1), columns and values of the CSR."""
        L = lib()
        nnz = self.nnz
        rp = np.zeros(self.dim + 1, np.uint64)
        col = np.zeros(nnz, np.uint32)
        val = np.zeros(2 * nnz, np.float64)
        L.qref_csr_get(self.h, rp, col, val)
        return rp, col, val.view(np.complex128)

    def spmv_real(self, x: np.ndarray, y: np.ndarray) -> bool:
        """y = Re(A) x on float64 vectors (the host lane of a real sector); False when A is not real."""
        return lib().qref_csr_spmv_real(self.h, x, y) == 0

    def close(self):
        if getattr(self, "h", None):
            try:
                lib().qref_csr_free(self.h)
            except Exception:
                pass
            self.h = None

    __del__ = close


def ftlm_blocks(sectors, prog: "Program", samples: int, depth: int, seed: int, betas) -> dict:
    """The reference's sampled thermal blocks on the host (its CSR lane and block scheduling): per-block
    curves [n_blocks, n_beta] and e_min [n_blocks]."""
    betas = np.ascontiguousarray(betas, np.float64)
    nb, nt = len(sectors), len(betas)
    arr = (C.c_void_p * nb)(*[s.h for s in sectors])
    lnZ, E, V = (np.zeros(nb * nt) for _ in range(3))
    gs = np.zeros(nb)
    _check(lib().qref_ftlm_blocks(arr, prog.h, nb, samples, depth, seed, betas, nt, lnZ, E, V, gs))
    return {"lnZ": lnZ.reshape(nb, nt), "E": E.reshape(nb, nt), "V": V.reshape(nb, nt), "e_min": gs}
