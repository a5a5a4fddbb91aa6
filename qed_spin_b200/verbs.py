"""The sector-resolved verbs on the B200 lane: eigs, thermal and dynamics with the reference's ``device=``.

They mirror the reference's Python verbs (python/qed/_verbs/eigs.py:119-189, thermal.py:54-121,
dynamics.py:77-124) for a Hamiltonian whose symmetry blocks are given explicitly (``sectors``: the reference
finds them with its symmetry detection, which is not on this path):

- ``eigs``: the ``k`` lowest levels over the blocks, with multiplicity. A block up to ``dense_max_dim`` states is
  solved densely (its full spectrum), a larger one by the k = 1 scan lane, or by thick-restart Krylov-Schur when
  it owes more than one level (or vectors are asked for).
- ``thermal``: per block, FTLM (every sampled block batched into one device call) or, up to ``dense_max_dim``
  states, the exact trace from its full spectrum; then the thermal driver's log-space combine.
- ``dynamics``: T = 0 dynamics of an operator from a source sector to a target sector.

``device``: ``"gpu"`` (strict: :class:`DeviceUnavailable` without a CUDA device) or ``"auto"`` (the device when
one is visible); ``"cpu"`` raises :class:`DeviceUnsupported`: this package is the device lane only, and the
host lane is the reference engine's own.
"""
from __future__ import annotations

import secrets
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

from . import _lib
from . import operators as ops
from ._lib import DeviceUnavailable, Unsupported as DeviceUnsupported
from .lattice import SectorSpec


class InvalidRequest(ValueError):
    """A malformed verb request (the reference's qed.errors.InvalidRequest)."""


class ConvergenceError(RuntimeError):
    """A block could not certify the levels it owes (the reference's qed.errors.ConvergenceError)."""


_DEVICES = ("cpu", "gpu", "auto")
# Blocks of more states than this use a reduced CSR when it fits (the lane choice of RepSectorMatVec); smaller
# ones are cheaper on the walk than the CSR's build.
_CSR_MIN_DIM = 4096


def _resolve(device: str) -> None:
    key = str(device).lower()
    if key not in _DEVICES:
        raise InvalidRequest(f"device must be one of {sorted(_DEVICES)}, got {device!r}")
    if key == "cpu":
        raise DeviceUnsupported(_lib.QB_EUNSUPPORTED, "this package is the device lane; device='cpu' is the "
                                                      "reference engine's host lane")
    from . import device as D
    if D.device_count() == 0:
        raise DeviceUnavailable(_lib.QB_ENODEV, f"device={device!r}, but no CUDA device is visible")


def _program(H) -> ops.Program:
    if isinstance(H, ops.Program):
        return H
    if isinstance(H, ops.MaskedOperator):
        return ops.row_program(H)
    raise InvalidRequest("H must be a MaskedOperator or a compiled row program")


def _blocks(sectors: Sequence[SectorSpec]):
    from . import device as D
    if not sectors:
        raise InvalidRequest("sectors: at least one block")
    out = []
    for i, spec in enumerate(sectors):
        S = D.Sector(spec)
        if S.dim > 0:
            out.append((i, spec, S))
    if not out:
        raise InvalidRequest("sectors: every block is empty")
    return out


def _lane(S, P):
    """Attaches the block's reduced CSR when the block is large enough and the CSR fits; returns it (or None)."""
    from . import device as D
    if S.dim < _CSR_MIN_DIM:
        return None
    try:
        A = D.Csr(S, S, P)
    except (_lib.ResourceLimit, DeviceUnsupported):
        return None
    A.attach(P)
    return A


@dataclass
class Level:
    energy: float
    block: int          # index into ``sectors``
    label: str


@dataclass
class EigResult:
    energies: np.ndarray
    levels: List[Level]
    k: int
    complete: bool
    device_blocks: int
    placement: dict
    vectors: Optional[list] = None   # per returned level (block coordinates), when asked for


def eigs(H, k: int = 1, *, sectors: Sequence[SectorSpec], vectors: bool = False, dense_max_dim: Optional[int] = None,
         allow_partial: bool = False, device: str = "gpu") -> EigResult:
    """The lowest ``k`` eigenvalues of ``H`` over the blocks ``sectors`` (with multiplicity).
    ``dense_max_dim``: blocks up to this dimension are diagonalised densely (default 64; vectors force Krylov)."""
    from . import device as D
    if int(k) < 1:
        raise InvalidRequest(f"k must be >= 1, got {k}")
    if dense_max_dim is not None and int(dense_max_dim) < 0:
        raise InvalidRequest(f"dense_max_dim must be >= 0 or None, got {dense_max_dim}")
    _resolve(device)
    k = int(k)
    dmax = 64 if dense_max_dim is None else int(dense_max_dim)
    prog = _program(H)
    found = []   # (energy, block, label, vector)
    complete = True
    placement = {"device_krylov": 0, "dense": 0}
    for i, spec, S in _blocks(sectors):
        P = D.Program(prog)
        want = min(k, S.dim)
        if S.dim <= dmax and not vectors:
            vals = D.dense_levels(S, P)[:want]
            placement["dense"] += 1
            found += [(float(v), i, spec.label, None) for v in vals]
            continue
        A = _lane(S, P)
        if want == 1 and not vectors:
            r = D.eigs_lowest(S, P)
            ok, vals, vecs = r["converged"], [r["e0"]], [None]
        else:
            r = D.eigs(S, P, want, vectors=vectors)
            ok, vals = r["converged"], list(r["values"])
            vecs = r.get("vectors", [None] * len(vals))
        placement["device_krylov"] += 1
        complete = complete and ok
        found += [(float(v), i, spec.label, x) for v, x in zip(vals, vecs)]
        if A is not None:
            D.detach_csr(P)
            A.close()
    if not complete and not allow_partial:
        raise ConvergenceError("eigs: a block did not converge (allow_partial=True returns what it has)")
    found.sort(key=lambda t: t[0])
    found = found[:k]
    return EigResult(energies=np.array([f[0] for f in found]), levels=[Level(f[0], f[1], f[2]) for f in found], k=k,
                     complete=complete, device_blocks=placement["device_krylov"], placement=placement,
                     vectors=[f[3] for f in found] if vectors else None)


@dataclass
class ThermalResult:
    T: np.ndarray
    lnZ: np.ndarray
    E: np.ndarray
    C: np.ndarray
    S: np.ndarray
    F: np.ndarray
    seed: int
    placement: dict = field(default_factory=dict)
    blocks: dict = field(default_factory=dict)   # per-block curves: lnZ, E, V [n_blocks, n_T]


def _exact_curves(levels: np.ndarray, betas: np.ndarray):
    """A block's exact trace from its full spectrum: lnZ = ln sum e^{-beta E}, E and V of the Boltzmann weights."""
    e0 = levels.min()
    x = levels - e0
    w = np.exp(-np.outer(betas, x))            # [n_T, n]
    z = w.sum(axis=1)
    m1 = (w * x).sum(axis=1) / z
    m2 = (w * x * x).sum(axis=1) / z
    return np.log(z) - betas * e0, e0 + m1, np.maximum(m2 - m1 * m1, 0.0)


def thermal(H, T: Sequence[float], *, sectors: Sequence[SectorSpec], method: str = "ftlm", samples: int = 40,
            krylov: Optional[int] = None, seed: int = 0, device: str = "gpu", dense_max_dim: Optional[int] = None,
            dtype: str = "c128", shared_samples: bool = False) -> ThermalResult:
    """Thermodynamics of ``H`` at the temperatures ``T`` over the blocks ``sectors``.
    ``method``: ``"ftlm"`` (blocks above ``dense_max_dim``, default 512, sampled with ``samples`` vectors at depth
    ``krylov``, default 100) or ``"exact"`` (every block's full spectrum). ``seed`` 0 draws one. The sampled blocks
    draw the reference driver's streams (its seed advanced by one LCG step before each sampled block, in block
    order, src/engine/thermal.cpp:470-471); ``shared_samples`` instead gives every block the prefixes of one set
    of streams from ``seed`` (drawn once: faster, equal in distribution)."""
    from . import device as D
    if method not in ("ftlm", "exact"):
        raise InvalidRequest(f"method must be 'ftlm' or 'exact', got {method!r}")
    T = np.asarray(T, np.float64)
    if T.ndim != 1 or len(T) == 0 or np.any(T <= 0):
        raise InvalidRequest("T: positive temperatures")
    if int(samples) < 1 or int(samples) > 64:
        raise InvalidRequest(f"samples must be in [1, 64], got {samples}")
    depth = 100 if krylov is None else int(krylov)
    if depth < 2:
        raise InvalidRequest(f"krylov must be >= 2, got {krylov}")
    _resolve(device)
    dmax = 512 if dense_max_dim is None else int(dense_max_dim)
    seed = int(seed) if seed else secrets.randbits(64) or 1
    betas = 1.0 / T
    prog = _program(H)
    blocks = _blocks(sectors)
    nb = len(blocks)
    lnZ, E, V = np.zeros((nb, len(T))), np.zeros((nb, len(T))), np.zeros((nb, len(T)))
    sampled = []
    P = D.Program(prog)
    dense = []
    for j, (i, spec, S) in enumerate(blocks):
        if method == "exact" or S.dim <= dmax:
            dense.append(j)
        else:
            sampled.append(j)
    if dense:
        for j, lv in zip(dense, D.dense_levels_blocks([blocks[j][2] for j in dense], P)):
            lnZ[j], E[j], V[j] = _exact_curves(lv, betas)
    if sampled:
        r = D.ftlm_blocks([blocks[j][2] for j in sampled], P, int(samples), depth, seed, betas, dtype=dtype,
                          per_block_seeds=not shared_samples)
        for q, j in enumerate(sampled):
            lnZ[j], E[j], V[j] = r["lnZ"][q], r["E"][q], r["V"][q]
    tot = D.thermal_combine(lnZ, E, V, betas)
    return ThermalResult(T=T, lnZ=tot["lnZ"], E=tot["E"], C=tot["C"], S=tot["S"], F=tot["F"], seed=seed,
                         placement={"dense": nb - len(sampled), "ftlm": len(sampled)},
                         blocks={"lnZ": lnZ, "E": E, "V": V, "index": [b[0] for b in blocks]})


@dataclass
class DynamicsResult:
    omega: np.ndarray
    S: np.ndarray
    e0: float
    conv_change: float
    certified: bool
    manifold: int = 1


def dynamics(H, O, *, source, target, omega: Sequence[float], eta: float = 0.05, krylov: int = 200,
             device: str = "gpu", degeneracy_tol: float = 1e-8) -> DynamicsResult:
    """T = 0 dynamics of the operator ``O`` (a MaskedOperator): S(omega) = -Im <phi| (omega + E0 - H + i eta)^-1
    |phi> / pi, phi = O psi0.

    ``source`` / ``target``: one block each, or equal-length lists, target[b] being the block O carries source[b]
    into (for O = S^z(q) on momentum blocks: momentum k -> k + q). With lists, psi0 runs over the ground manifold of
    the source blocks -- every level within ``degeneracy_tol`` times the scale of H (the sum of |c| over its terms)
    of E0, multiplets inside a block included -- and S is the average over it, as the reference's verb returns for
    a degenerate ground state (src/engine/dynamics.cpp:395-566). With one block, psi0 is that block's ground state."""
    from . import device as D
    omega = np.asarray(omega, np.float64)
    if omega.ndim != 1 or len(omega) == 0:
        raise InvalidRequest("omega: a non-empty frequency grid")
    if eta <= 0:
        raise InvalidRequest(f"eta must be > 0, got {eta}")
    if not isinstance(O, ops.MaskedOperator):
        raise InvalidRequest("O must be a MaskedOperator")
    many = isinstance(source, (list, tuple))
    if many != isinstance(target, (list, tuple)) or (many and len(source) != len(target)):
        raise InvalidRequest("source and target: one block each, or lists of equal length")
    _resolve(device)
    h = _program(H)
    if many:
        srcs = [D.Sector(s) for s in source]
        tgts = [D.Sector(t) for t in target]
        if all(S.dim == 0 for S in srcs):
            raise InvalidRequest("source: the blocks hold no state")
        hs = [D.Program(h) for _ in srcs]
        ht = [D.Program(h) for _ in tgts]
        cross = [D.Program(ops.cross_row_program(O, t, s)) for s, t in zip(source, target)]
        lanes = [(_lane(S, P) if S.dim else None, P) for S, P in zip(srcs + tgts, hs + ht)]
        r = D.dynamics_t0_manifold(srcs, hs, tgts, ht, cross, int(krylov), omega, eta, degeneracy_tol)
        for A, P in lanes:
            if A is not None:
                D.detach_csr(P)
                A.close()
        return DynamicsResult(omega=omega, S=r["S"], e0=r["e0"], conv_change=float("nan"), certified=r["certified"],
                              manifold=r["manifold"])
    Ss, St = D.Sector(source), D.Sector(target)
    if Ss.dim == 0:
        raise InvalidRequest("source: an empty block")
    hs, ht = D.Program(h), D.Program(h)
    lanes = [_lane(Ss, hs), _lane(St, ht) if St.dim else None]
    r = D.dynamics_t0(Ss, hs, St, ht, D.Program(ops.cross_row_program(O, target, source)), int(krylov), omega, eta)
    for A, P in zip(lanes, (hs, ht)):
        if A is not None:
            D.detach_csr(P)
            A.close()
    return DynamicsResult(omega=omega, S=r["S"], e0=r["e0"], conv_change=r["conv_change"], certified=r["certified"])
