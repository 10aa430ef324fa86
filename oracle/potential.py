"""Hartree and LDA-PZ exchange-correlation in FP64 numpy.

Follows amaterasu ``hamiltonian/hartree.py:28-50``, ``xc/driver.py:108-164`` (LDA
branch) and ``xc/lda.py:122-142`` (exchange), ``:203-262`` (PZ81 correlation and the
chain rule to v_sigma).
"""
from __future__ import annotations

import numpy as np
import scipy.fft as sfft

X_FACTOR_C = 0.9305257363491000250020102180716672510262
RS_FACTOR = 0.6203504908994000166680068120477781673508
THRESHOLD = 1e-24
PZ = dict(gamma=(-0.1423, -0.0843), beta1=(1.0529, 1.3981), beta2=(0.3334, 0.2611),
          a=(0.0311, 0.01555), b=(-0.048, -0.0269), c=(0.0020, 0.0007), d=(-0.0116, -0.0048))


def hartree(density, shape, miller, g2, volume):
    """(E_H, V_H(r)) for a total density, using the density sphere (miller, g2)."""
    coeff_grid = sfft.fftn(np.asarray(density, dtype=complex), norm="forward")
    i, j, k = (np.asarray(miller)[:, a] % shape[a] for a in range(3))
    c = coeff_grid[i, j, k]
    nz = g2 > 1e-12
    vg = np.zeros_like(c)
    vg[nz] = 4.0 * np.pi * c[nz] / g2[nz]
    energy = 0.5 * volume * float(np.sum(4.0 * np.pi * np.abs(c[nz]) ** 2 / g2[nz]))
    grid = np.zeros(shape, dtype=complex)
    grid[i, j, k] = vg
    return energy, np.ascontiguousarray(sfft.ifftn(grid, norm="forward").real)


def lda_pz(rho):
    """(eps, vrho) for a spin density rho of shape (npoints, 2)."""
    rho = np.atleast_2d(np.asarray(rho, dtype=float))
    total = rho[:, 0] + rho[:, 1]
    active = total > THRESHOLD
    spin = np.maximum(rho, 0.0)
    cube = np.cbrt(spin)
    eps_x = np.zeros_like(total)
    np.divide(-X_FACTOR_C * np.sum(cube * spin, axis=1), total, out=eps_x, where=active)
    vx = np.where(active[:, None], -(4.0 / 3.0) * X_FACTOR_C * cube, 0.0)
    safe = np.maximum(total, THRESHOLD)
    rs = RS_FACTOR / np.cbrt(safe)
    zeta = np.clip((rho[:, 0] - rho[:, 1]) / safe, -1.0, 1.0)
    e, de = [], []
    for idx in range(2):
        sq = np.sqrt(rs)
        den = 1.0 + PZ["beta1"][idx] * sq + PZ["beta2"][idx] * rs
        low = PZ["gamma"][idx] / den
        dlow = -PZ["gamma"][idx] * (0.5 * PZ["beta1"][idx] / sq + PZ["beta2"][idx]) / den**2
        lr = np.log(np.maximum(rs, 1e-300))
        high = PZ["a"][idx] * lr + PZ["b"][idx] + PZ["c"][idx] * rs * lr + PZ["d"][idx] * rs
        dhigh = PZ["a"][idx] / rs + PZ["c"][idx] * (lr + 1.0) + PZ["d"][idx]
        dense = rs < 1.0
        e.append(np.where(dense, high, low))
        de.append(np.where(dense, dhigh, dlow))
    den = 2.0 ** (4.0 / 3.0) - 2.0
    opz, omz = np.maximum(1.0 + zeta, 0.0), np.maximum(1.0 - zeta, 0.0)
    fz = (opz ** (4 / 3) + omz ** (4 / 3) - 2.0) / den
    dfz = (4 / 3) * (np.cbrt(opz) - np.cbrt(omz)) / den
    eps_c = e[0] + fz * (e[1] - e[0])
    d_rs = de[0] + fz * (de[1] - de[0])
    d_z = dfz * (e[1] - e[0])
    common = eps_c - (rs / 3.0) * d_rs
    vc = np.stack([common + (1.0 - zeta) * d_z, common - (1.0 + zeta) * d_z], axis=-1)
    eps_c = np.where(active, eps_c, 0.0)
    vc = np.where(active[:, None], vc, 0.0)
    return eps_x + eps_c, vx + vc


def xc_on_grid(density, cell_volume_per_point):
    """(E_xc, v_xc (nspin, ...)) for density (nspin, n1, n2, n3), LDA-PZ."""
    density = np.asarray(density, dtype=float)
    nspin = density.shape[0]
    spin = np.stack([density[0] / 2, density[0] / 2]) if nspin == 1 else density
    rho = spin.reshape(2, -1).T
    eps, vrho = lda_pz(rho)
    energy = float(np.sum(eps * (rho[:, 0] + rho[:, 1])) * cell_volume_per_point)
    pot = vrho.T.reshape(2, *density.shape[1:])
    return energy, pot[:nspin]
