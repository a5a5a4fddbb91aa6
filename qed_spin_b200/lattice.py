"""Lattices, their symmetry groups and the sector specifications the matvec runs on.

A group element acts on a basis state as ``permute_bits(s, perm) ^ flip`` with new bit i = old bit perm[i]
(include/ed/basis/compiled_group.h:8-14, include/ed/basis/rep_sector.h:16-20). A sector is a fixed-S^z
subspace (``n_up`` set bits = up spins) reduced by a group in a one-dimensional irrep with characters
``chars`` (include/ed/basis/rep_sector.h:134-160).
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Optional

import numpy as np


@dataclass
class SectorSpec:
    n_sites: int
    n_up: int
    perms: np.ndarray          # G x N int32
    chars: np.ndarray          # G complex128
    flips: Optional[np.ndarray] = None   # G uint64, or None (pure permutations)
    label: str = ""

    @property
    def group_size(self) -> int:
        return int(self.perms.shape[0])

    def with_n_up(self, n_up: int) -> "SectorSpec":
        return SectorSpec(self.n_sites, n_up, self.perms, self.chars, self.flips, self.label)

    def with_chars(self, chars) -> "SectorSpec":
        return SectorSpec(self.n_sites, self.n_up, self.perms, np.asarray(chars, np.complex128), self.flips, self.label)


def chain_bonds(N: int, r: int = 1):
    """Periodic chain bonds (i, i + r mod N)."""
    return [(i, (i + r) % N) for i in range(N)]


def chain_translations(N: int) -> np.ndarray:
    """The N translations p_t[i] = (i + t) mod N."""
    return np.array([[(i + t) % N for i in range(N)] for t in range(N)], np.int32)


def chain_dihedral(N: int) -> np.ndarray:
    """The N translations then the N reflections p[i] = (t - i) mod N."""
    tr = chain_translations(N)
    rf = np.array([[(t - i) % N for i in range(N)] for t in range(N)], np.int32)
    return np.concatenate([tr, rf])


def with_spin_flip(perms: np.ndarray, N: int):
    """The flip-extended group: [g_0..g_{G-1}, g_0 F, .., g_{G-1} F] (orbit_table.h:293-307)."""
    G = perms.shape[0]
    allm = np.uint64((1 << N) - 1) if N < 64 else np.uint64(0xFFFFFFFFFFFFFFFF)
    flips = np.zeros(2 * G, np.uint64)
    flips[G:] = allm
    return np.concatenate([perms, perms]), flips


def momentum_chars(N: int, k: int) -> np.ndarray:
    """chi_k(t) = exp(-2 pi i k t / N) for the translations t = 0..N-1."""
    t = np.arange(N)
    return np.exp(-2j * np.pi * k * t / N).astype(np.complex128)


def square_sites(Lx: int, Ly: int):
    return lambda x, y: (x % Lx) + Lx * (y % Ly)


def square_translations(Lx: int, Ly: int) -> np.ndarray:
    """Translations by (a, b), element a + Lx b: site x + Lx y -> (x + a) + Lx (y + b)."""
    idx = square_sites(Lx, Ly)
    out = []
    for b in range(Ly):
        for a in range(Lx):
            p = [0] * (Lx * Ly)
            for y in range(Ly):
                for x in range(Lx):
                    p[idx(x, y)] = idx(x + a, y + b)
            out.append(p)
    return np.array(out, np.int32)


def square_j1j2_bonds(Lx: int, Ly: int):
    """Nearest (x+1, y), (x, y+1) and next-nearest (x+1, y+1), (x+1, y-1) bonds of a periodic torus."""
    idx = square_sites(Lx, Ly)
    nn, nnn = [], []
    for y in range(Ly):
        for x in range(Lx):
            nn.append((idx(x, y), idx(x + 1, y)))
            nn.append((idx(x, y), idx(x, y + 1)))
            nnn.append((idx(x, y), idx(x + 1, y + 1)))
            nnn.append((idx(x, y), idx(x + 1, y - 1)))
    return nn, nnn


def chain_sector(N: int, n_up: int, k: int = 0) -> SectorSpec:
    """Translations only, momentum k."""
    return SectorSpec(N, n_up, chain_translations(N), momentum_chars(N, k), None, f"chain{N} n_up={n_up} k={k}")


def chain_a1_flip_sector(N: int) -> SectorSpec:
    """k = 0, reflection-even, spin-flip-even at half filling: D_N x Z2, all characters +1."""
    perms, flips = with_spin_flip(chain_dihedral(N), N)
    chars = np.ones(perms.shape[0], np.complex128)
    return SectorSpec(N, N // 2, perms, chars, flips, f"chain{N} k=0 R+ F+")


def square_k0_sector(Lx: int, Ly: int, n_up: int) -> SectorSpec:
    perms = square_translations(Lx, Ly)
    return SectorSpec(Lx * Ly, n_up, perms, np.ones(perms.shape[0], np.complex128), None,
                      f"square{Lx}x{Ly} n_up={n_up} k=(0,0)")
