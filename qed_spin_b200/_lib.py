"""ctypes bindings of the C-ABI declared in include/qed_b200.h (libqed_b200.so, built in-tree).

Loading fails loudly: there is no CPU fallback for any entry point.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libqed_b200.so")

QB_OK, QB_EINVAL, QB_ENOMEM, QB_ECUDA, QB_EUNSUPPORTED, QB_ETIMEOUT, QB_ENODEV = range(7)
QB_C128, QB_C64 = 0, 1
QB_REORTH_NONE, QB_REORTH_FULL, QB_REORTH_LOCAL = 0, 1, 2
QB_SEED_SHARED, QB_SEED_PER_BLOCK = 0, 1
QB_LOOKUP_AUTO, QB_LOOKUP_RANK, QB_LOOKUP_BUCKETS, QB_LOOKUP_HASH, QB_LOOKUP_HASH_WIDE = 0, 1, 2, 3, 4
QB_NOALLOC_MAX_ITER = 1024

#: every symbol include/qed_b200.h declares
EXPORTS = [
    "qb_last_error", "qb_device_count",
    "qb_sector_create", "qb_sector_create_from_reps", "qb_sector_destroy", "qb_sector_dim", "qb_sector_download",
    "qb_sector_info", "qb_index_and_projection", "qb_key_order",
    "qb_program_create", "qb_program_destroy",
    "qb_matvec", "qb_matvec_block", "qb_matvec_host",
    "qb_csr_build", "qb_csr_upload", "qb_csr_destroy", "qb_csr_info", "qb_csr_download", "qb_csr_matvec",
    "qb_program_attach_csr",
    "qb_lanczos", "qb_staged_start", "qb_eigs_lowest", "qb_ftlm", "qb_ftlm_blocks", "qb_thermal_combine", "qb_cf",
    "qb_lanczos_noalloc", "qb_ground_state", "qb_eigs_k", "qb_eigs_levels", "qb_dynamics_t0", "qb_dynamics_t0_manifold", "qb_dense_levels",
    "qb_dense_levels_blocks",
    "qb_server_create", "qb_server_submit", "qb_server_wait", "qb_server_clock", "qb_server_destroy",
    "qb_sector_acquire", "qb_sector_release", "qb_registry_capacity", "qb_registry_stats", "qb_memory_trim",
    "qb_sector_save",
    "qb_sector_load",
    "qb_tune_mode", "qb_tune_force", "qb_tune_clear", "qb_tune_save", "qb_tune_load", "qb_tune_entries",
]


class SectorDesc(C.Structure):
    _fields_ = [
        ("n_sites", C.c_int), ("n_up", C.c_int), ("group_size", C.c_int),
        ("perms", C.c_void_p), ("flips", C.c_void_p), ("chars", C.c_void_p),
        ("sublattice_mode", C.c_int), ("lookup", C.c_int),
    ]


class ProgramDesc(C.Structure):
    _fields_ = [
        ("n_groups", C.c_uint32), ("group_flip", C.c_void_p), ("group_setbits", C.c_void_p),
        ("group_vbegin", C.c_void_p), ("n_vsub", C.c_uint32), ("vsub_val", C.c_void_p),
        ("vsub_tbegin", C.c_void_p), ("n_terms", C.c_uint32), ("term_sign", C.c_void_p),
        ("term_coeff", C.c_void_p),
    ]


QB_REQ_EIGS, QB_REQ_DYNAMICS, QB_REQ_THERMAL = 0, 1, 2
QB_SERVER_MAX_LEVELS = 16


class Request(C.Structure):
    _fields_ = [
        ("kind", C.c_int), ("sector", SectorDesc), ("h", ProgramDesc), ("k", C.c_int), ("target", SectorDesc),
        ("op", ProgramDesc), ("krylov", C.c_int), ("omega", C.c_void_p), ("n_omega", C.c_int), ("eta", C.c_double),
        ("samples", C.c_int), ("seed", C.c_uint64), ("betas", C.c_void_p), ("n_beta", C.c_int),
    ]


class Result(C.Structure):
    _fields_ = [
        ("status", C.c_int), ("n_values", C.c_int), ("values", C.c_double * QB_SERVER_MAX_LEVELS),
        ("converged", C.c_int), ("matvecs", C.c_int), ("e0", C.c_double), ("conv_change", C.c_double),
        ("t_submit", C.c_double), ("t_admit", C.c_double), ("t_done", C.c_double), ("footprint", C.c_uint64),
    ]


class QbError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[qb error {code}] {msg}")
        self.code = code


class DeviceUnavailable(QbError):
    pass


class ResourceLimit(QbError):
    pass


class Unsupported(QbError):
    pass


_lib = None


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"the CUDA library is not built ({LIB_PATH}); run `python -m qed_spin_b200.build` "
                           "-- there is no CPU fallback")
    L = C.CDLL(LIB_PATH)
    vp, i, u64, d = C.c_void_p, C.c_int, C.c_uint64, C.c_double
    L.qb_last_error.restype = C.c_char_p
    L.qb_device_count.argtypes = [C.POINTER(i)]
    L.qb_sector_create.argtypes = [C.POINTER(SectorDesc), C.POINTER(vp)]
    L.qb_sector_create_from_reps.argtypes = [C.POINTER(SectorDesc), vp, vp, u64, C.POINTER(vp)]
    L.qb_sector_destroy.argtypes = [vp]
    L.qb_sector_dim.argtypes = [vp]
    L.qb_sector_dim.restype = u64
    L.qb_sector_download.argtypes = [vp, vp, vp]
    L.qb_sector_info.argtypes = [vp, C.POINTER(u64), C.POINTER(i), C.POINTER(i), C.POINTER(i)]
    L.qb_index_and_projection.argtypes = [vp, vp, u64, vp, vp]
    L.qb_key_order.argtypes = [vp, C.POINTER(i), C.POINTER(i), C.POINTER(u64), vp, vp, vp, vp]
    L.qb_program_create.argtypes = [C.POINTER(ProgramDesc), C.POINTER(vp)]
    L.qb_program_destroy.argtypes = [vp]
    L.qb_matvec.argtypes = [vp, vp, vp, vp, vp, i, i, vp]
    L.qb_matvec_block.argtypes = [vp, vp, vp, vp, vp, i, i, vp]
    L.qb_matvec_host.argtypes = [vp, vp, vp, vp, vp]
    L.qb_csr_build.argtypes = [vp, vp, vp, u64, C.POINTER(vp)]
    L.qb_csr_upload.argtypes = [vp, vp, vp, vp, vp, u64, C.POINTER(vp)]
    L.qb_csr_destroy.argtypes = [vp]
    L.qb_csr_info.argtypes = [vp, C.POINTER(u64), C.POINTER(u64), C.POINTER(i)]
    L.qb_csr_download.argtypes = [vp, vp, vp, vp]
    L.qb_csr_matvec.argtypes = [vp, vp, vp, i, i, vp]
    L.qb_program_attach_csr.argtypes = [vp, vp]
    L.qb_lanczos.argtypes = [vp, vp, vp, i, i, d, i, vp, vp, C.POINTER(i)]
    L.qb_eigs_lowest.argtypes = [vp, vp, i, i, i, C.POINTER(d), C.POINTER(i), C.POINTER(i), C.POINTER(i)]
    L.qb_ftlm.argtypes = [vp, vp, i, i, u64, vp, i, i, vp, vp, vp, C.POINTER(d)]
    L.qb_ground_state.argtypes = [vp, vp, i, C.POINTER(d), C.POINTER(d), C.POINTER(i), vp, vp, C.POINTER(i)]
    L.qb_eigs_k.argtypes = [vp, vp, i, u64, vp, C.POINTER(i), C.POINTER(i), C.POINTER(i), vp]
    L.qb_dynamics_t0_manifold.argtypes = [i, vp, vp, vp, vp, vp, i, vp, i, C.c_double, C.c_double, vp, vp,
                                          C.POINTER(i), C.POINTER(i)]
    L.qb_staged_start.argtypes = [u64, u64, vp]
    L.qb_eigs_levels.argtypes = [vp, vp, i, u64, i, i, vp, C.POINTER(i), C.POINTER(i), C.POINTER(i), vp]
    L.qb_dynamics_t0.argtypes = [vp, vp, vp, vp, vp, i, vp, i, d, vp, C.POINTER(d), C.POINTER(d), C.POINTER(i)]
    L.qb_dense_levels.argtypes = [vp, vp, vp]
    L.qb_dense_levels_blocks.argtypes = [vp, vp, i, vp]
    L.qb_sector_acquire.argtypes = [C.POINTER(SectorDesc), C.POINTER(vp)]
    L.qb_sector_release.argtypes = [vp]
    L.qb_registry_capacity.argtypes = [u64]
    L.qb_memory_trim.argtypes = [u64, C.c_void_p]
    L.qb_registry_stats.argtypes = [C.POINTER(u64), C.POINTER(u64), C.POINTER(u64)]
    L.qb_sector_save.argtypes = [vp, C.c_char_p]
    L.qb_sector_load.argtypes = [C.c_char_p, C.POINTER(vp)]
    L.qb_server_create.argtypes = [i, u64, C.POINTER(vp)]
    L.qb_server_submit.argtypes = [vp, C.POINTER(Request), C.POINTER(u64)]
    L.qb_server_wait.argtypes = [vp, u64, i, C.POINTER(Result), vp]
    L.qb_server_clock.argtypes = [vp, C.POINTER(d)]
    L.qb_server_destroy.argtypes = [vp]
    L.qb_ftlm_blocks.argtypes = [vp, vp, i, i, i, u64, i, vp, i, i, i, vp, vp, vp, vp, vp]
    L.qb_thermal_combine.argtypes = [i, vp, vp, vp, vp, vp, i, vp, vp, vp, vp, vp]
    L.qb_cf.argtypes = [vp, vp, vp, i, vp, i, d, d, d, vp, C.POINTER(d)]
    L.qb_lanczos_noalloc.argtypes = [vp, vp, vp, vp, i, i, d, i, vp, vp, C.POINTER(i), vp]
    L.qb_tune_mode.argtypes = [i, C.POINTER(i)]
    L.qb_tune_force.argtypes = [C.c_char_p, i]
    L.qb_tune_clear.argtypes = []
    L.qb_tune_save.argtypes = [C.c_char_p]
    L.qb_tune_load.argtypes = [C.c_char_p]
    L.qb_tune_entries.argtypes = [C.c_char_p, u64, C.POINTER(u64)]
    for name in EXPORTS:
        if name not in ("qb_last_error", "qb_sector_dim"):
            getattr(L, name).restype = i
    _lib = L
    return L


def check(rc: int):
    if rc == QB_OK:
        return
    msg = lib().qb_last_error().decode()
    if rc == QB_ENODEV:
        raise DeviceUnavailable(rc, msg)
    if rc == QB_ENOMEM:
        raise ResourceLimit(rc, msg)
    if rc == QB_EUNSUPPORTED:
        raise Unsupported(rc, msg)
    if rc == QB_EINVAL:
        raise ValueError(f"[qb error {rc}] {msg}")
    raise QbError(rc, msg)
