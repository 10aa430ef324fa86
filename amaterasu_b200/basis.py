"""Plane-wave basis on the host: G-spheres, FFT grid shapes and sphere<->grid index maps.

This is set-up code that runs once per geometry. Its outputs are conventions the device
engine must reproduce exactly, so each one restates the reference's rule:

* sphere membership ``|k+G|^2/2 <= ecut`` (+1e-12) inside the Miller box of
  ``|G| <= gmax + |k|`` (amaterasu ``basis/gvectors.py:118-149``);
* sphere order: ascending ``|k+G|^2`` with ties broken lexicographically on the Miller
  indices (h, k, l) (``gvectors.py:151-155``);
* grid shape: ``next_fast_len(2 h_max + 1)`` per axis from the density sphere
  (``basis/fft.py:151-172``);
* grid index of a plane wave: Miller index modulo the grid shape (``fft.py:174-190``).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import scipy.fft as _sfft

__all__ = ["FFTGrid", "GSphere", "miller_bounds", "reciprocal_cell"]


def reciprocal_cell(cell) -> np.ndarray:
    """Reciprocal vectors as rows in 1/Bohr, ``b_i . a_j = 2 pi delta_ij``."""
    cell = np.asarray(cell, dtype=float)
    if cell.shape != (3, 3):
        raise ValueError(f"cell must be 3x3, got {cell.shape}")
    volume = float(np.linalg.det(cell))
    if abs(volume) < 1e-12:
        raise ValueError(f"cell is singular (volume {volume:.3e} Bohr^3)")
    return 2.0 * np.pi * np.linalg.inv(cell).T


def miller_bounds(cell, gmax: float) -> np.ndarray:
    lengths = np.linalg.norm(np.asarray(cell, dtype=float), axis=1)
    return np.ceil(gmax * lengths / (2.0 * np.pi)).astype(int)


@dataclass
class GSphere:
    """Plane waves inside a cutoff, in the reference's sphere order."""

    miller: np.ndarray      # (npw, 3) int
    cartesian: np.ndarray   # (npw, 3) k+G in 1/Bohr
    g2: np.ndarray          # (npw,) |k+G|^2
    kpoint: np.ndarray      # fractional k
    ecut: float
    cell: np.ndarray

    def __len__(self) -> int:
        return len(self.miller)

    @property
    def kinetic_energy(self) -> np.ndarray:
        return 0.5 * self.g2

    @classmethod
    def build(cls, cell, ecut: float, kpoint=(0.0, 0.0, 0.0), *, sort: bool = True) -> "GSphere":
        if ecut <= 0:
            raise ValueError(f"ecut must be positive, got {ecut}")
        cell = np.asarray(cell, dtype=float)
        reciprocal = reciprocal_cell(cell)
        kpoint = np.asarray(kpoint, dtype=float)
        k_cart = kpoint @ reciprocal
        gmax = np.sqrt(2.0 * ecut)
        bounds = miller_bounds(cell, gmax + float(np.linalg.norm(k_cart)))
        axes = [np.arange(-b, b + 1) for b in bounds]
        miller = np.stack(np.meshgrid(*axes, indexing="ij"), axis=-1).reshape(-1, 3)
        cart = miller @ reciprocal + k_cart
        g2 = np.einsum("ij,ij->i", cart, cart)
        inside = g2 <= 2.0 * ecut + 1e-12
        miller, cart, g2 = miller[inside], cart[inside], g2[inside]
        if sort:
            order = np.lexsort((miller[:, 2], miller[:, 1], miller[:, 0], g2))
            miller, cart, g2 = miller[order], cart[order], g2[order]
        return cls(miller=miller, cartesian=cart, g2=g2, kpoint=kpoint, ecut=float(ecut), cell=cell)


def _fast_length(minimum: int, multiple: int = 1) -> int:
    if multiple <= 1:
        return int(_sfft.next_fast_len(int(minimum)))
    candidate = -(-int(minimum) // multiple) * multiple
    for _ in range(1000):
        if _sfft.next_fast_len(candidate) == candidate:
            return candidate
        candidate += multiple
    return int(_sfft.next_fast_len(int(minimum)))


@dataclass
class FFTGrid:
    """Real-space grid shape and cell; C-order layout, axis 2 fastest."""

    shape: tuple
    cell: np.ndarray

    @property
    def size(self) -> int:
        return int(np.prod(self.shape))

    @property
    def volume(self) -> float:
        return abs(float(np.linalg.det(self.cell)))

    @property
    def cell_volume_per_point(self) -> float:
        return self.volume / self.size

    @classmethod
    def for_cutoff(cls, cell, ecut: float, multiple: int = 1) -> "FFTGrid":
        sphere = GSphere.build(np.asarray(cell, dtype=float), ecut, sort=False)
        h_max = np.abs(sphere.miller).max(axis=0)
        shape = tuple(_fast_length(int(n), multiple) for n in 2 * h_max + 1)
        return cls(shape=shape, cell=np.asarray(cell, dtype=float))

    def indices(self, sphere: GSphere):
        """Per-axis grid indices of each plane wave (Miller index mod shape)."""
        h_max = np.abs(sphere.miller).max(axis=0)
        if np.any(2 * h_max + 1 > np.asarray(self.shape)):
            raise ValueError(
                f"grid {tuple(self.shape)} is too small for Miller indices up to "
                f"{tuple(int(h) for h in h_max)}"
            )
        return tuple(sphere.miller[:, axis] % self.shape[axis] for axis in range(3))

    def flat_indices(self, sphere: GSphere) -> np.ndarray:
        i, j, k = self.indices(sphere)
        n1, n2, n3 = self.shape
        return ((i * n2 + j) * n3 + k).astype(np.int64)

    def gvectors_cartesian(self) -> np.ndarray:
        """Cartesian G of every grid point in FFT frequency order, shape (*shape, 3)."""
        axes = [np.fft.fftfreq(n, d=1.0 / n) for n in self.shape]
        miller = np.stack(np.meshgrid(*axes, indexing="ij"), axis=-1)
        return miller @ reciprocal_cell(self.cell)
