"""Radial (spherical-Bessel) transforms of pseudopotential tables, evaluated once per
geometry on the host in FP64.

Restates amaterasu ``pseudo/formfactors.py``: ``radial_transform`` (:55-71), the
erf-split local form factor with its finite alpha term at q=0 (:74-103), projector and
density transforms (:106-123) and their q-derivatives for the stress (:133-185). Each
transform depends on |q| alone, so it is evaluated on the distinct |q| values only and
scattered back, which gives the same numbers as evaluating every plane wave.
"""
from __future__ import annotations

import numpy as np
from scipy.special import erf, spherical_jn

from .pseudo import NCPseudopotential, Projector, RadialGrid

_CHUNK = 256


def _unique(q):
    q = np.atleast_1d(np.asarray(q, dtype=float))
    values, inverse = np.unique(q, return_inverse=True)
    return q, values, inverse.reshape(q.shape)


def _integrate_rows(grid: RadialGrid, make_rows, qs: np.ndarray) -> np.ndarray:
    out = np.empty(len(qs))
    for start in range(0, len(qs), _CHUNK):
        block = qs[start:start + _CHUNK]
        out[start:start + len(block)] = grid.integrate(make_rows(block))
    return out


def radial_transform(grid: RadialGrid, values, l: int, q) -> np.ndarray:
    q, uq, inv = _unique(q)
    values = np.asarray(values, dtype=float)
    r = grid.r
    res = _integrate_rows(grid, lambda b: values * spherical_jn(int(l), b[:, None] * r[None, :]), uq)
    return res[inv]


def radial_transform_derivative(grid: RadialGrid, values, l: int, q) -> np.ndarray:
    q, uq, inv = _unique(q)
    values = np.asarray(values, dtype=float)
    r = grid.r
    res = _integrate_rows(
        grid, lambda b: values * r * spherical_jn(int(l), b[:, None] * r[None, :], derivative=True), uq)
    return res[inv]


def local_potential_form_factor(pseudo: NCPseudopotential, q) -> np.ndarray:
    q, uq, inv = _unique(q)
    grid, z = pseudo.grid, float(pseudo.valence_charge)
    r = grid.r
    res = np.empty_like(uq)
    at_zero = uq < 1e-12
    if np.any(at_zero):
        res[at_zero] = 4.0 * np.pi * grid.integrate(r * (r * pseudo.local_potential + z))
    if np.any(~at_zero):
        qq = uq[~at_zero]
        screened = r * pseudo.local_potential + z * erf(r)
        integral = _integrate_rows(grid, lambda b: screened * np.sin(b[:, None] * r[None, :]), qq)
        res[~at_zero] = 4.0 * np.pi / qq * integral - 4.0 * np.pi * z * np.exp(-0.25 * qq**2) / qq**2
    return res[inv]


def local_potential_form_factor_derivative(pseudo: NCPseudopotential, q) -> np.ndarray:
    q, uq, inv = _unique(q)
    grid, z = pseudo.grid, float(pseudo.valence_charge)
    r = grid.r
    res = np.zeros_like(uq)
    nz = uq >= 1e-12
    if np.any(nz):
        qq = uq[nz]
        screened = r * pseudo.local_potential + z * erf(r)
        integral = _integrate_rows(grid, lambda b: screened * np.sin(b[:, None] * r[None, :]), qq)
        deriv = _integrate_rows(grid, lambda b: screened * r * np.cos(b[:, None] * r[None, :]), qq)
        res[nz] = (-4.0 * np.pi / qq**2 * integral + 4.0 * np.pi / qq * deriv
                   + 4.0 * np.pi * z * np.exp(-0.25 * qq**2) * (0.5 / qq + 2.0 / qq**3))
    return res[inv]


def projector_form_factor(grid: RadialGrid, projector: Projector, q) -> np.ndarray:
    return radial_transform(grid, grid.r * projector.values, projector.l, q)


def projector_form_factor_derivative(grid: RadialGrid, projector: Projector, q) -> np.ndarray:
    return radial_transform_derivative(grid, grid.r * projector.values, projector.l, q)


def density_form_factor(grid: RadialGrid, density, q) -> np.ndarray:
    return radial_transform(grid, density, 0, q)


def density_form_factor_derivative(grid: RadialGrid, density, q) -> np.ndarray:
    return radial_transform_derivative(grid, density, 0, q)
