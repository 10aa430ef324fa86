"""Synthetic silicon cells with the shapes of the benchmark workloads (Angstrom).

Seeds and the random k-points are part of each cell's definition so that every run,
the device engine's and the CPU oracle's, sees the same input.
"""
from __future__ import annotations

import numpy as np

from . import kpoints as kp
from .system import Structure

A_SI = 5.43
_FCC = np.array([[0.0, 0.0, 0.0], [0.0, 0.5, 0.5], [0.5, 0.0, 0.5], [0.5, 0.5, 0.0]])
_DIAMOND = np.vstack([_FCC, _FCC + 0.25])


def si2_primitive(a: float = A_SI) -> Structure:
    """Two-atom fcc primitive diamond cell."""
    cell = 0.5 * a * np.array([[0.0, 1.0, 1.0], [1.0, 0.0, 1.0], [1.0, 1.0, 0.0]])
    frac = np.array([[0.0, 0.0, 0.0], [0.25, 0.25, 0.25]])
    return Structure(["Si", "Si"], frac @ cell, cell)


def si_supercell(n: int, a: float = A_SI, *, vacancy: bool = False, sigma: float = 0.0,
                 seed: int = 0) -> Structure:
    """n x n x n conventional diamond supercell (8 n^3 sites), optional first-site vacancy
    and seeded N(0, sigma) Cartesian displacements (Angstrom)."""
    frac = np.vstack([(_DIAMOND + np.array([i, j, k])) / n
                      for i in range(n) for j in range(n) for k in range(n)])
    cell = np.eye(3) * a * n
    if vacancy:
        frac = frac[1:]
    pos = frac @ cell
    if sigma > 0:
        pos = pos + np.random.default_rng(seed).normal(scale=sigma, size=pos.shape)
    return Structure(["Si"] * len(pos), pos, cell)


def hpsi_bench_kpoints(seed: int = 1) -> kp.KPointSet:
    """Gamma plus three seeded random fractional k-points in [-1/2, 1/2)^3, equal weights."""
    rng = np.random.default_rng(seed)
    points = np.vstack([np.zeros((1, 3)), rng.uniform(-0.5, 0.5, size=(3, 3))])
    return kp.explicit(points)


def workload(name: str):
    """(structure, ecut Ha, k-point set, nbands) of a named workload."""
    if name == "si2_scf":
        return si2_primitive(), 15.0, kp.monkhorst_pack((4, 4, 4), (0.5, 0.5, 0.5)), 8
    if name == "si64_hpsi":
        return si_supercell(2), 20.0, hpsi_bench_kpoints(), 160
    if name == "si8_batched":
        return si_supercell(1, sigma=0.05, seed=8), 20.0, kp.monkhorst_pack((8, 8, 8)), 20
    if name == "si215_gamma":
        return si_supercell(3, vacancy=True, sigma=0.05, seed=215), 15.0, kp.gamma_only(), 440
    raise KeyError(name)
