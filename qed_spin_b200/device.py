"""Host handles over the C-ABI: device sectors and programs, the matvec, and the Krylov drivers.

Every call goes to libqed_b200.so (CUDA, sm_100a). Device vectors are torch tensors (complex128 for
QB_C128, complex64 for QB_C64) on the current CUDA device; host vectors are numpy complex128 arrays.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check, lib
from .lattice import SectorSpec
from .operators import Program as HostProgram

DTYPES = {"c128": _lib.QB_C128, "c64": _lib.QB_C64, "fp64": _lib.QB_C128, "fp32": _lib.QB_C64}


def _dt(dtype) -> int:
    if isinstance(dtype, int):
        return dtype
    return DTYPES[dtype]


def device_count() -> int:
    n = C.c_int()
    check(lib().qb_device_count(C.byref(n)))
    return n.value


class Sector:
    """A symmetry sector resident on the device (its representatives enumerated there)."""

    def __init__(self, spec: SectorSpec, sublattice_mode: int = -1, lookup: int = _lib.QB_LOOKUP_AUTO,
                 reps=None, inv_norms=None, shared: bool = False, _handle=None):
        """shared: take the registry's sector for this descriptor (qb_sector_acquire) instead of a private one."""
        self.spec = spec
        self._shared = bool(shared)
        if _handle is not None:
            self.h = _handle
            return
        self._perms = np.ascontiguousarray(spec.perms, np.int32)
        chars = np.asarray(spec.chars, np.complex128)
        self._chars = np.ascontiguousarray(np.stack([chars.real, chars.imag], 1).reshape(-1))
        self._flips = None if spec.flips is None else np.ascontiguousarray(spec.flips, np.uint64)
        d = _lib.SectorDesc(spec.n_sites, spec.n_up, self._perms.shape[0], self._perms.ctypes.data,
                            None if self._flips is None else self._flips.ctypes.data, self._chars.ctypes.data,
                            sublattice_mode, lookup)
        h = C.c_void_p()
        if shared:
            check(lib().qb_sector_acquire(C.byref(d), C.byref(h)))
        elif reps is None:
            check(lib().qb_sector_create(C.byref(d), C.byref(h)))
        else:
            r = np.ascontiguousarray(reps, np.uint64)
            w = np.ascontiguousarray(inv_norms, np.float64)
            check(lib().qb_sector_create_from_reps(C.byref(d), r.ctypes.data, w.ctypes.data, len(r), C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None) and self.h.value:
            try:
                if getattr(self, "_shared", False):
                    lib().qb_sector_release(self.h)
                else:
                    lib().qb_sector_destroy(self.h)
            except Exception:   # interpreter shutdown: the library is already gone
                pass
            self.h = None   # (no module globals here: this also runs at interpreter shutdown)

    __del__ = close

    def save(self, path: str) -> None:
        """Writes the descriptor, representatives and 1/norms (qb_sector_save)."""
        check(lib().qb_sector_save(self.h, str(path).encode()))

    @classmethod
    def load(cls, path: str, spec: SectorSpec = None) -> "Sector":
        """A sector from a file written by save (no enumeration)."""
        h = C.c_void_p()
        check(lib().qb_sector_load(str(path).encode(), C.byref(h)))
        return cls(spec, _handle=h)

    @property
    def dim(self) -> int:
        return int(lib().qb_sector_dim(self.h))

    def reps(self):
        n = self.dim
        reps = np.zeros(n, np.uint64)
        inv = np.zeros(n, np.float64)
        if n:
            check(lib().qb_sector_download(self.h, reps.ctypes.data, inv.ctypes.data))
        return reps, inv

    def info(self) -> dict:
        b, L, m, k = C.c_uint64(), C.c_int(), C.c_int(), C.c_int()
        check(lib().qb_sector_info(self.h, C.byref(b), C.byref(L), C.byref(m), C.byref(k)))
        return dict(device_bytes=b.value, slc_L=L.value, slc_m=m.value,
                    lookup={0: "none", 1: "rank", 2: "buckets", 3: "hash", 4: "hash8"}[k.value])

    def index_and_projection(self, states):
        st = np.ascontiguousarray(states, np.uint64)
        idx = np.zeros(len(st), np.int64)
        proj = np.zeros(2 * len(st), np.float64)
        check(lib().qb_index_and_projection(self.h, st.ctypes.data, len(st), idx.ctypes.data, proj.ctypes.data))
        return idx, proj.view(np.complex128)


def key_order(spec: SectorSpec, sublattice_mode: int = -1) -> dict:
    """The sublattice key order of a sector descriptor and its tables (host work only, no device needed): None
    when the plain order applies, else L, m, key_bit, lead, cand_off, cand (qb_key_order)."""
    keep = []
    d = _sector_desc(spec, keep)
    d.sublattice_mode = sublattice_mode
    L_, m_, nc = C.c_int(), C.c_int(), C.c_uint64()
    check(lib().qb_key_order(C.byref(d), C.byref(L_), C.byref(m_), C.byref(nc), None, None, None, None))
    if L_.value == 0:
        return None
    P = m_.value << L_.value
    kb = np.zeros(spec.n_sites, np.int32)
    lead = np.zeros(P, np.uint16)
    off = np.zeros(P + 1, np.uint32)
    cand = np.zeros(max(1, nc.value), np.uint16)
    check(lib().qb_key_order(C.byref(d), C.byref(L_), C.byref(m_), C.byref(nc), kb.ctypes.data, lead.ctypes.data,
                             off.ctypes.data, cand.ctypes.data))
    return {"L": L_.value, "m": m_.value, "key_bit": kb, "lead": lead, "cand_off": off, "cand": cand[: nc.value]}


class Program:
    """A row program resident on the device."""

    def __init__(self, prog: HostProgram):
        self.host = prog
        self._a = [
            np.ascontiguousarray(prog.group_flip, np.uint64),
            np.ascontiguousarray(prog.group_setbits, np.int32),
            np.ascontiguousarray(prog.group_vbegin, np.uint32),
            np.ascontiguousarray(prog.vsub_val, np.uint64),
            np.ascontiguousarray(prog.vsub_tbegin, np.uint32),
            np.ascontiguousarray(prog.term_sign, np.uint64),
            np.ascontiguousarray(np.asarray(prog.term_coeff, np.complex128)).view(np.float64),
        ]
        a = self._a
        d = _lib.ProgramDesc(len(a[0]), a[0].ctypes.data, a[1].ctypes.data, a[2].ctypes.data, len(a[3]),
                             a[3].ctypes.data, a[4].ctypes.data, len(a[5]), a[5].ctypes.data, a[6].ctypes.data)
        h = C.c_void_p()
        check(lib().qb_program_create(C.byref(d), C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None) and self.h.value:
            try:
                lib().qb_program_destroy(self.h)
            except Exception:   # interpreter shutdown: the library is already gone
                pass
            self.h = None   # (no module globals here: this also runs at interpreter shutdown)

    __del__ = close


class Csr:
    """The merged reduced CSR of a program between two sectors, on the device.

    Built from the row walk on the device (`Csr(row, col, prog)`) or uploaded from host arrays
    (`Csr.upload(row, col, row_ptr, col, val)`). `attach(prog)` routes every apply of `prog` on this
    sector pair through it.
    """

    def __init__(self, row: Sector, col: Sector, prog: Program = None, max_bytes: int = 0, _handle=None):
        self.row, self.col = row, col
        self._attached = []
        if _handle is not None:
            self.h = _handle
            return
        h = C.c_void_p()
        check(lib().qb_csr_build(row.h, col.h, prog.h, int(max_bytes), C.byref(h)))
        self.h = h

    @classmethod
    def upload(cls, row: Sector, col: Sector, row_ptr, col_idx, val, max_bytes: int = 0) -> "Csr":
        rp = np.ascontiguousarray(row_ptr, np.uint64)
        ci = np.ascontiguousarray(col_idx, np.uint32)
        v = np.ascontiguousarray(val, np.complex128)
        h = C.c_void_p()
        check(lib().qb_csr_upload(row.h, col.h, rp.ctypes.data, ci.ctypes.data, v.view(np.float64).ctypes.data,
                                  int(max_bytes), C.byref(h)))
        return cls(row, col, _handle=h)

    def info(self) -> dict:
        nnz, nb, nd = C.c_uint64(), C.c_uint64(), C.c_int()
        check(lib().qb_csr_info(self.h, C.byref(nnz), C.byref(nb), C.byref(nd)))
        return {"nnz": nnz.value, "bytes": nb.value, "n_dict": nd.value}

    def download(self):
        nnz = self.info()["nnz"]
        rp = np.zeros(self.row.dim + 1, np.uint64)
        ci = np.zeros(nnz, np.uint32)
        v = np.zeros(2 * nnz, np.float64)
        check(lib().qb_csr_download(self.h, rp.ctypes.data, ci.ctypes.data, v.ctypes.data))
        return rp, ci, v.view(np.complex128)

    def matvec(self, x, out, k: int = 1, dtype="c128", stream=None):
        """out = A x on device tensors (k > 1: k vectors interleaved by row)."""
        check(lib().qb_csr_matvec(self.h, x.data_ptr(), out.data_ptr(), k, _dt(dtype), _stream_ptr(stream)))

    def attach(self, prog: Program):
        check(lib().qb_program_attach_csr(prog.h, self.h))
        prog._csr = self
        self._attached.append(prog)

    def close(self):
        if getattr(self, "h", None) and self.h.value:
            try:
                for p in self._attached:
                    if getattr(p, "_csr", None) is self and p.h and p.h.value:
                        lib().qb_program_attach_csr(p.h, None)
                        p._csr = None
                lib().qb_csr_destroy(self.h)
            except Exception:   # interpreter shutdown: the library is already gone
                pass
            self.h = None   # (no module globals here: this also runs at interpreter shutdown)
            self._attached = []

    __del__ = close


def detach_csr(prog: Program):
    """Routes prog's applies back to the row walk."""
    check(lib().qb_program_attach_csr(prog.h, None))
    prog._csr = None


def _stream_ptr(stream):
    if stream is None:
        return None
    return getattr(stream, "cuda_stream", stream)


def matvec(row: Sector, col: Sector, prog: Program, xs, outs, dtype="c128", stream=None):
    """outs[i] = O xs[i] for device tensors (lists of equal length)."""
    k = len(xs)
    ins = (C.c_void_p * k)(*[x.data_ptr() for x in xs])
    ous = (C.c_void_p * k)(*[y.data_ptr() for y in outs])
    check(lib().qb_matvec(row.h, col.h, prog.h, ins, ous, k, _dt(dtype), _stream_ptr(stream)))


def matvec_block(row: Sector, col: Sector, prog: Program, x, out, k: int, dtype="c128", stream=None):
    """out = O x on k vectors interleaved by row (device tensors of row.dim * k elements)."""
    check(lib().qb_matvec_block(row.h, col.h, prog.h, x.data_ptr(), out.data_ptr(), k, _dt(dtype),
                                _stream_ptr(stream)))


def matvec_host(row: Sector, col: Sector, prog: Program, x: np.ndarray) -> np.ndarray:
    x = np.ascontiguousarray(x, np.complex128)
    y = np.zeros(row.dim, np.complex128)
    check(lib().qb_matvec_host(row.h, col.h, prog.h, x.ctypes.data, y.ctypes.data))
    return y


def lanczos(sec: Sector, prog: Program, v0: np.ndarray, max_iter: int, reorth: int = _lib.QB_REORTH_NONE,
            breakdown_tol: float = 1e-300, dtype="c128"):
    v0 = np.ascontiguousarray(v0, np.complex128)
    a = np.zeros(max_iter)
    b = np.zeros(max_iter + 1)
    it = C.c_int()
    check(lib().qb_lanczos(sec.h, prog.h, v0.ctypes.data, max_iter, reorth, breakdown_tol, _dt(dtype),
                           a.ctypes.data, b.ctypes.data, C.byref(it)))
    m = it.value
    return a[:m].copy(), b[: m + 1].copy()


def staged_start(seed: int, n: int) -> np.ndarray:
    """The lanes' staged Gaussian start (qb_staged_start): host work, the reference's mt19937_64 stream."""
    out = np.zeros(n, np.complex128)
    check(lib().qb_staged_start(seed, n, out.ctypes.data))
    return out


def eigs_lowest(sec: Sector, prog: Program, max_iter: int = 0, dtype="c128", refine: bool = True) -> dict:
    e, it, cv, mv = C.c_double(), C.c_int(), C.c_int(), C.c_int()
    check(lib().qb_eigs_lowest(sec.h, prog.h, max_iter, _dt(dtype), 1 if refine else 0, C.byref(e), C.byref(it),
                               C.byref(cv), C.byref(mv)))
    return dict(e0=e.value, iters=it.value, converged=bool(cv.value), matvecs=mv.value)


def ground_state(sec: Sector, prog: Program, max_steps: int = 0, vector: bool = True) -> dict:
    """The certified lowest eigenpair: energy, residual, certified, matvecs, and the vector (host complex128)."""
    e0, res, cert, mv = C.c_double(), C.c_double(), C.c_int(), C.c_int()
    vec = np.zeros(sec.dim, np.complex128) if vector else None
    check(lib().qb_ground_state(sec.h, prog.h, max_steps, C.byref(e0), C.byref(res), C.byref(cert), None,
                                None if vec is None else vec.ctypes.data, C.byref(mv)))
    return {"e0": e0.value, "residual": res.value, "certified": bool(cert.value), "matvecs": mv.value, "vector": vec}


def eigs(sec: Sector, prog: Program, k: int, max_iter: int = 0, vectors: bool = False, dtype="c128",
         refine: bool = True) -> dict:
    """The k lowest levels: the k = 1 scan lane for k == 1 (without vectors), thick-restart Lanczos for k > 1.
    dtype "c64" stores the Lanczos vectors in FP32; refine then polishes every pair in FP64."""
    if k == 1 and not vectors:
        r = eigs_lowest(sec, prog, max_iter, dtype=dtype, refine=refine)
        return {"values": np.array([r["e0"]]), "converged": r["converged"], "matvecs": r["matvecs"]}
    vals = np.zeros(k)
    nf, cv, mv = C.c_int(), C.c_int(), C.c_int()
    import torch
    vecs = [torch.empty(sec.dim, dtype=torch.complex128, device="cuda") for _ in range(k)] if vectors else None
    ptrs = (C.c_void_p * k)(*[v.data_ptr() for v in vecs]) if vectors else None
    check(lib().qb_eigs_levels(sec.h, prog.h, k, max_iter, _dt(dtype), 1 if refine else 0, vals.ctypes.data,
                               C.byref(nf), C.byref(cv), C.byref(mv), ptrs))
    out = {"values": vals[: nf.value], "converged": bool(cv.value), "matvecs": mv.value}
    if vectors:
        out["vectors"] = [v.cpu().numpy() for v in vecs[: nf.value]]
    return out


def dense_levels(sec: Sector, prog: Program) -> np.ndarray:
    """The full spectrum of a small block (<= 8192 states), ascending, with multiplicity."""
    vals = np.zeros(sec.dim)
    check(lib().qb_dense_levels(sec.h, prog.h, vals.ctypes.data))
    return vals


def dense_levels_blocks(sectors, prog: Program) -> list:
    """The full spectra of many small blocks at once (host threads), one array per block."""
    nb = len(sectors)
    dims = [s.dim for s in sectors]
    vals = np.zeros(max(1, sum(dims)))
    sh = (C.c_void_p * nb)(*[s.h.value for s in sectors])
    ph = (C.c_void_p * nb)(*[prog.h.value] * nb)
    check(lib().qb_dense_levels_blocks(sh, ph, nb, vals.ctypes.data))
    out, o = [], 0
    for d in dims:
        out.append(vals[o:o + d].copy())
        o += d
    return out


def dynamics_t0(src: Sector, h_src: Program, tgt: Sector, h_tgt: Program, op: Program, depth: int, omega,
                eta: float) -> dict:
    """T = 0 dynamics of the cross-sector operator `op` (rows in tgt, columns in src): S(omega), E0."""
    omega = np.ascontiguousarray(omega, np.float64)
    S = np.zeros(len(omega))
    e0, ch, cert = C.c_double(), C.c_double(), C.c_int()
    check(lib().qb_dynamics_t0(src.h, h_src.h, tgt.h, h_tgt.h, op.h, depth, omega.ctypes.data, len(omega), eta,
                               S.ctypes.data, C.byref(e0), C.byref(ch), C.byref(cert)))
    return {"S": S, "e0": e0.value, "conv_change": ch.value, "certified": bool(cert.value)}


def dynamics_t0_manifold(srcs, h_srcs, tgts, h_tgts, ops, depth: int, omega, eta: float,
                         degeneracy_tol: float = 1e-8) -> dict:
    """T = 0 dynamics averaged over the ground manifold of the source blocks (qb_dynamics_t0_manifold): block b's
    states carried by ops[b] into tgts[b]. Returns S(omega), E0, the manifold's size and whether every solve
    converged."""
    nb = len(srcs)
    omega = np.ascontiguousarray(omega, np.float64)
    S = np.zeros(len(omega))
    arr = lambda xs: (C.c_void_p * nb)(*[x.h.value for x in xs])
    e0, g, cert = C.c_double(), C.c_int(), C.c_int()
    check(lib().qb_dynamics_t0_manifold(nb, arr(srcs), arr(h_srcs), arr(tgts), arr(h_tgts), arr(ops), depth,
                                        omega.ctypes.data, len(omega), eta, degeneracy_tol, S.ctypes.data,
                                        C.byref(e0), C.byref(g), C.byref(cert)))
    return {"S": S, "e0": e0.value, "manifold": g.value, "certified": bool(cert.value)}


def ftlm(sec: Sector, prog: Program, samples: int, depth: int, seed: int, betas, dtype="c128") -> dict:
    betas = np.ascontiguousarray(betas, np.float64)
    nb = len(betas)
    lnZ, E, V = np.zeros(nb), np.zeros(nb), np.zeros(nb)
    em = C.c_double()
    check(lib().qb_ftlm(sec.h, prog.h, samples, depth, seed, betas.ctypes.data, nb, _dt(dtype), lnZ.ctypes.data,
                        E.ctypes.data, V.ctypes.data, C.byref(em)))
    return dict(lnZ=lnZ, E=E, V=V, e_min=em.value)


def ftlm_blocks(sectors, progs, samples: int, depth: int, seed: int, betas, dtype="c128", use_csr=True,
                per_block_seeds: bool = False) -> dict:
    """FTLM over many blocks (each a Sector; progs: one Program for all, or one per block). Returns the
    per-block curves [n_blocks, n_beta] (lnZ, E, V), e_min [n_blocks], and their log-space combination
    (lnZ, E, C, S, F over beta) under "total". per_block_seeds: the reference thermal driver's sample streams (the
    seed advanced by its LCG step before each block, in the order given); else one set of streams for all blocks."""
    nb = len(sectors)
    if isinstance(progs, Program):
        progs = [progs] * nb
    betas = np.ascontiguousarray(betas, np.float64)
    nt = len(betas)
    sh = (C.c_void_p * nb)(*[s.h.value for s in sectors])
    ph = (C.c_void_p * nb)(*[p.h.value for p in progs])
    lnZ, E, V = (np.zeros((nb, nt)) for _ in range(3))
    e_min = np.zeros(nb)
    stats = np.zeros(4)
    mode = _lib.QB_SEED_PER_BLOCK if per_block_seeds else _lib.QB_SEED_SHARED
    check(lib().qb_ftlm_blocks(sh, ph, nb, samples, depth, seed, mode, betas.ctypes.data, nt, _dt(dtype),
                               int(bool(use_csr)), lnZ.ctypes.data, E.ctypes.data, V.ctypes.data, e_min.ctypes.data,
                               stats.ctypes.data))
    return {"lnZ": lnZ, "E": E, "V": V, "e_min": e_min, "total": thermal_combine(lnZ, E, V, betas),
            "stats": dict(zip(("draw_s", "csr_build_s", "recurrence_s", "curves_s"), stats.tolist()))}


def thermal_combine(lnZ, E, V, betas, weights=None) -> dict:
    """Per-block curves [n_blocks, n_beta] combined in log space (the reference thermal driver's combine)."""
    lnZ, E, V = (np.ascontiguousarray(a, np.float64) for a in (lnZ, E, V))
    betas = np.ascontiguousarray(betas, np.float64)
    nb, nt = lnZ.shape
    w = None if weights is None else np.ascontiguousarray(weights, np.float64)
    out = {k: np.zeros(nt) for k in ("lnZ", "E", "C", "S", "F")}
    check(lib().qb_thermal_combine(nb, None if w is None else w.ctypes.data, lnZ.ctypes.data, E.ctypes.data,
                                   V.ctypes.data, betas.ctypes.data, nt, out["lnZ"].ctypes.data, out["E"].ctypes.data,
                                   out["C"].ctypes.data, out["S"].ctypes.data, out["F"].ctypes.data))
    return out


def cf(sec: Sector, prog: Program, phi: np.ndarray, depth: int, omega, eta: float, shift: float = float("nan"),
       tolerance: float = 1e-12):
    phi = np.ascontiguousarray(phi, np.complex128)
    omega = np.ascontiguousarray(omega, np.float64)
    S = np.zeros(len(omega))
    sh = C.c_double()
    check(lib().qb_cf(sec.h, prog.h, phi.ctypes.data, depth, omega.ctypes.data, len(omega), eta, shift, tolerance,
                      S.ctypes.data, C.byref(sh)))
    return S, sh.value


def _sector_desc(spec, keep: list, lookup: int = 0) -> "_lib.SectorDesc":
    perms = np.ascontiguousarray(spec.perms, np.int32)
    chars = np.ascontiguousarray(np.asarray(spec.chars, np.complex128)).view(np.float64)
    flips = None if spec.flips is None else np.ascontiguousarray(spec.flips, np.uint64)
    keep += [perms, chars, flips]
    return _lib.SectorDesc(spec.n_sites, spec.n_up, perms.shape[0], perms.ctypes.data,
                           None if flips is None else flips.ctypes.data, chars.ctypes.data, -1, lookup)


def _program_desc(prog: HostProgram, keep: list) -> "_lib.ProgramDesc":
    a = [
        np.ascontiguousarray(prog.group_flip, np.uint64),
        np.ascontiguousarray(prog.group_setbits, np.int32),
        np.ascontiguousarray(prog.group_vbegin, np.uint32),
        np.ascontiguousarray(prog.vsub_val, np.uint64),
        np.ascontiguousarray(prog.vsub_tbegin, np.uint32),
        np.ascontiguousarray(prog.term_sign, np.uint64),
        np.ascontiguousarray(np.asarray(prog.term_coeff, np.complex128)).view(np.float64),
    ]
    keep += a
    return _lib.ProgramDesc(len(a[0]), a[0].ctypes.data, a[1].ctypes.data, a[2].ctypes.data, len(a[3]),
                            a[3].ctypes.data, a[4].ctypes.data, len(a[5]), a[5].ctypes.data, a[6].ctypes.data)


class Server:
    """The request server (qb_server_*): eigs, thermal (one block's FTLM) and T = 0 dynamics requests served
    concurrently on the device with admission by HBM footprint. submit() returns a ticket at once; wait() returns
    the result."""

    def __init__(self, max_active: int = 8, hbm_budget: int = 0):
        h = C.c_void_p()
        check(lib().qb_server_create(max_active, hbm_budget, C.byref(h)))
        self.h = h
        self.n_omega = {}

    def submit_eigs(self, spec, prog: HostProgram, k: int) -> int:
        keep = []
        r = _lib.Request()
        r.kind = _lib.QB_REQ_EIGS
        r.sector = _sector_desc(spec, keep)
        r.h = _program_desc(prog, keep)
        r.k = k
        t = C.c_uint64()
        check(lib().qb_server_submit(self.h, C.byref(r), C.byref(t)))
        return t.value

    def submit_dynamics(self, src, tgt, h: HostProgram, op: HostProgram, krylov: int, omega, eta: float) -> int:
        keep = []
        omega = np.ascontiguousarray(omega, np.float64)
        keep.append(omega)
        r = _lib.Request()
        r.kind = _lib.QB_REQ_DYNAMICS
        r.sector = _sector_desc(src, keep)
        r.target = _sector_desc(tgt, keep)
        r.h = _program_desc(h, keep)
        r.op = _program_desc(op, keep)
        r.krylov = krylov
        r.omega = omega.ctypes.data
        r.n_omega = len(omega)
        r.eta = eta
        t = C.c_uint64()
        check(lib().qb_server_submit(self.h, C.byref(r), C.byref(t)))
        self.n_omega[t.value] = len(omega)
        return t.value

    def submit_thermal(self, spec, h: HostProgram, samples: int, krylov: int, seed: int, betas) -> int:
        """One block of the thermal driver's sampled path: its FTLM curves (lnZ, E, V per beta)."""
        keep = []
        betas = np.ascontiguousarray(betas, np.float64)
        keep.append(betas)
        r = _lib.Request()
        r.kind = _lib.QB_REQ_THERMAL
        r.sector = _sector_desc(spec, keep)
        r.h = _program_desc(h, keep)
        r.krylov = krylov
        r.samples = samples
        r.seed = seed
        r.betas = betas.ctypes.data
        r.n_beta = len(betas)
        t = C.c_uint64()
        check(lib().qb_server_submit(self.h, C.byref(r), C.byref(t)))
        self.n_omega[t.value] = ("thermal", len(betas))
        return t.value

    def wait(self, ticket: int, timeout_ms: int = -1) -> dict:
        res = _lib.Result()
        no = self.n_omega.pop(ticket, 0)
        thermal = isinstance(no, tuple)
        if thermal:
            no = 3 * no[1]
        S = np.zeros(no) if no else None
        check(lib().qb_server_wait(self.h, ticket, timeout_ms, C.byref(res), None if S is None else S.ctypes.data))
        if res.status != _lib.QB_OK:
            check(res.status)
        out = {"values": np.array(res.values[: res.n_values]), "converged": bool(res.converged),
               "matvecs": res.matvecs, "e0": res.e0, "conv_change": res.conv_change, "S": S,
               "t_submit": res.t_submit, "t_admit": res.t_admit, "t_done": res.t_done, "footprint": res.footprint}
        if thermal:
            nb = no // 3
            out.update(lnZ=S[:nb], E=S[nb:2 * nb], V=S[2 * nb:], e_min=out["values"][0], S=None)
        return out

    def clock(self) -> float:
        t = C.c_double()
        check(lib().qb_server_clock(self.h, C.byref(t)))
        return t.value

    def close(self):
        if getattr(self, "h", None) and self.h.value:
            try:
                lib().qb_server_destroy(self.h)
            except Exception:
                pass
            self.h = None

    __del__ = close


def registry_capacity(nbytes: int) -> None:
    """The byte capacity of the cache of released shared sectors (0 empties it)."""
    check(lib().qb_registry_capacity(int(nbytes)))


def memory_trim(keep_bytes: int = 0) -> int:
    """Frees the library's idle cached device blocks on the current device down to keep_bytes; returns the idle
    bytes left (qb_memory_trim)."""
    left = C.c_uint64()
    check(lib().qb_memory_trim(int(keep_bytes), C.byref(left)))
    return left.value


def registry_stats() -> dict:
    a, b, c = C.c_uint64(), C.c_uint64(), C.c_uint64()
    check(lib().qb_registry_stats(C.byref(a), C.byref(b), C.byref(c)))
    return {"sectors": a.value, "idle_sectors": b.value, "idle_bytes": c.value}


# ---- launch-shape tuning ----

def tune_mode(mode: int = -1) -> int:
    """Sets the tuner's mode (1 measure on first use, 2 known choices only, 0 defaults; -1 leaves it) and
    returns the previous one."""
    prev = C.c_int(0)
    check(lib().qb_tune_mode(int(mode), C.byref(prev)))
    return prev.value


def tune_force(family: str, choice: int) -> None:
    """Forces launch shape `choice` for a kernel family ("walk", "walk_team"); a negative choice removes it."""
    check(lib().qb_tune_force(family.encode(), int(choice)))


def tune_clear() -> None:
    check(lib().qb_tune_clear())


def tune_save(path: str) -> None:
    check(lib().qb_tune_save(str(path).encode()))


def tune_load(path: str) -> None:
    check(lib().qb_tune_load(str(path).encode()))


def tune_entries() -> dict:
    """The known choices: key -> (choice, [ms per candidate])."""
    need = C.c_uint64(0)
    check(lib().qb_tune_entries(None, 0, C.byref(need)))
    buf = C.create_string_buffer(int(need.value) + 1)
    check(lib().qb_tune_entries(buf, len(buf), C.byref(need)))
    out = {}
    for line in buf.value.decode().splitlines():
        parts = line.split("\t")
        if len(parts) >= 2:
            out[parts[0]] = (int(parts[1]), [float(x) for x in parts[2:]])
    return out
