"""H.psi, sphere<->grid maps and the Kleinman-Bylander products (FP64, numpy/scipy).

Follows amaterasu ``hamiltonian/operator.py:60-69`` (T + G[V R[psi]] + V_NL),
``basis/fft.py:192-243`` (scatter/gather, ifftn/fftn with norm="forward") and
``pseudo/kb.py:216-241`` (project, apply, energy).
"""
from __future__ import annotations

import numpy as np
import scipy.fft as sfft


def grid_indices(miller, shape):
    return tuple(np.asarray(miller)[:, a] % shape[a] for a in range(3))


def wave_to_real(coeffs, miller, shape, workers=1):
    i, j, k = grid_indices(miller, shape)
    coeffs = np.asarray(coeffs)
    if coeffs.ndim == 1:
        grid = np.zeros(shape, dtype=complex)
        grid[i, j, k] = coeffs
        return sfft.ifftn(grid, norm="forward", workers=workers)
    grid = np.zeros((coeffs.shape[0], *shape), dtype=complex)
    grid[:, i, j, k] = coeffs
    return sfft.ifftn(grid, axes=(-3, -2, -1), norm="forward", workers=workers)


def real_to_wave(values, miller, shape, workers=1):
    i, j, k = grid_indices(miller, shape)
    axes = (-3, -2, -1) if values.ndim > 3 else (0, 1, 2)
    g = sfft.fftn(values, axes=axes, norm="forward", workers=workers)
    return g[i, j, k] if values.ndim == 3 else g[:, i, j, k]


def kb_project(coeffs, proj):
    return np.asarray(coeffs) @ proj.conj().T


def kb_apply(coeffs, proj, dij):
    if proj.shape[0] == 0:
        return np.zeros_like(coeffs)
    return (kb_project(coeffs, proj) @ dij) @ proj


def kb_energy(coeffs, proj, dij, weights):
    p = kb_project(coeffs, proj)
    return float(np.dot(weights, np.einsum("ni,ij,nj->n", p.conj(), dij, p).real))


def hamiltonian_apply(coeffs, miller, shape, kinetic, veff, proj, dij, workers=1):
    """``H|psi>`` for a block (nbands, npw) or one band, complex128."""
    coeffs = np.asarray(coeffs, dtype=complex)
    result = coeffs * kinetic
    real = wave_to_real(coeffs, miller, shape, workers)
    result = result + real_to_wave(veff * real, miller, shape, workers)
    if proj is not None:
        result = result + kb_apply(coeffs, proj, dij)
    return result
