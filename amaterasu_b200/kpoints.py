"""k-point sets: Gamma, explicit lists and Monkhorst-Pack meshes reduced by time reversal.

The reference reduces meshes with spglib (amaterasu ``system/symmetry.py:135-206``). The
engine runs with symmetry off, so the only reduction applied is time reversal,
k ~ -k: mesh point g (i-major order, shift s = 0/1 per axis meaning a half step) is
represented by the lowest-index member of {g, -g - s mod mesh}. Points are then
``(g + s/2)/mesh`` folded with ``k -= rint(k)``, and each weight is the multiplicity over
the mesh size (``symmetry.py:196-206``).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

__all__ = ["KPointSet", "gamma_only", "explicit", "monkhorst_pack"]


@dataclass
class KPointSet:
    points: np.ndarray   # (nk, 3) fractional
    weights: np.ndarray  # (nk,) summing to 1
    mesh: tuple | None = None
    shift: tuple = (0.0, 0.0, 0.0)

    def __len__(self) -> int:
        return len(self.points)


def gamma_only() -> KPointSet:
    return KPointSet(np.zeros((1, 3)), np.ones(1), (1, 1, 1))


def explicit(points, weights=None) -> KPointSet:
    points = np.atleast_2d(np.asarray(points, dtype=float))
    if weights is None:
        w = np.full(len(points), 1.0 / len(points))
    else:
        w = np.asarray(weights, dtype=float)
        if w.sum() <= 0:
            raise ValueError("explicit k-point weights must sum to a positive number")
        w = w / w.sum()
    return KPointSet(points, w, None)


def monkhorst_pack(mesh, shift=(0.0, 0.0, 0.0), *, time_reversal: bool = True) -> KPointSet:
    mesh = np.asarray(mesh, dtype=int)
    if mesh.shape != (3,) or np.any(mesh < 1):
        raise ValueError(f"mesh must be three positive integers, got {mesh.tolist()}")
    half = np.array([1 if abs(float(s)) > 1e-12 else 0 for s in shift], dtype=int)
    grid = np.stack(np.meshgrid(*[np.arange(n) for n in mesh], indexing="ij"), axis=-1).reshape(-1, 3)
    owner = np.arange(len(grid))
    if time_reversal:
        partner = np.mod(-grid - half, mesh)
        partner_flat = (partner[:, 0] * mesh[1] + partner[:, 1]) * mesh[2] + partner[:, 2]
        for index in range(len(grid)):
            other = partner_flat[index]
            if other < index:
                owner[index] = owner[other]
    unique, counts = np.unique(owner, return_counts=True)
    points = (grid[unique] + 0.5 * half) / mesh
    points -= np.rint(points)
    weights = counts / counts.sum()
    return KPointSet(points, weights, tuple(int(n) for n in mesh), tuple(float(s) for s in shift))
