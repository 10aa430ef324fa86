"""Analytic forces and stress for norm-conserving datasets (symmetry off).

Mirrors amaterasu ``properties/forces.py:49-172`` and ``properties/stress.py:64-289``:
forces = Ewald + local (density-sphere sum of i G v_a(|G|) e^{iG.tau_a} n(G)) + nonlocal
(derivative of <beta|psi> through the projector phases) + core; stress = Ewald + kinetic +
Hartree + local + nonlocal (projector q-gradients from the solid harmonics) + xc + core.
n(G) comes from the engine's FP64 grid transform and every band contraction (projections,
derivative projections, |c|^2 sums) runs on the GPU; the per-geometry radial tables and
projector q-gradients are built on the host in FP64 like the projector matrices.
"""
from __future__ import annotations

import ctypes as ct

import numpy as np
import torch

from ._lib import call
from .engine import engine_for, ptr, require_cuda, stream_ptr
from .ewald import ewald
from .formfactors import (density_form_factor, density_form_factor_derivative, local_potential_form_factor,
                          local_potential_form_factor_derivative, projector_form_factor,
                          projector_form_factor_derivative)
from .linalg import gemm_nc
from .local import structure_factors
from .potential import grid_ops
from .projectors import real_spherical_harmonics, solid_harmonics_gradient

__all__ = ["compute_forces", "compute_stress", "density_coefficients"]


def _grid_forward(system, field: torch.Tensor) -> torch.Tensor:
    eng = engine_for(system)
    f = field.reshape(-1).to(eng.device, torch.float64).contiguous()
    out = torch.empty(eng.N, dtype=torch.complex128, device=eng.device)
    call("ama_grid_fft_forward", eng.handle, ptr(f), ptr(out), stream_ptr())
    return out


def density_coefficients(system, field) -> torch.Tensor:
    """Fourier coefficients of a real grid field on the density sphere (device)."""
    f = field if isinstance(field, torch.Tensor) else torch.from_numpy(np.asarray(field, dtype=float))
    full = _grid_forward(system, f)
    idx = torch.from_numpy(system.grid.flat_indices(system.density_sphere)).to(full.device)
    return full[idx]


def _as_dev(x, dev, dtype=None):
    t = x if isinstance(x, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(x))
    return t.to(dev) if dtype is None else t.to(dev, dtype)


class _SphereTables:
    """Density-sphere vectors and per-species radial tables (cached on the system)."""

    def __init__(self, system, dev):
        sph = system.density_sphere
        self.q = np.sqrt(sph.g2)
        self.g = torch.from_numpy(sph.cartesian).to(dev)
        self.g2 = torch.from_numpy(sph.g2).to(dev)
        self.vloc = {s: torch.from_numpy(local_potential_form_factor(p, self.q)).to(dev)
                     for s, p in system.pseudopotentials.items()}
        self._vloc_d = None
        self._core = None
        self.system = system
        self.dev = dev

    def vloc_slope(self):
        if self._vloc_d is None:
            self._vloc_d = {s: torch.from_numpy(local_potential_form_factor_derivative(p, self.q)).to(self.dev)
                            for s, p in self.system.pseudopotentials.items()}
        return self._vloc_d

    def core(self, derivative=False):
        out = {}
        for s, p in self.system.pseudopotentials.items():
            if p.core_density is None:
                out[s] = None
            else:
                fn = density_form_factor_derivative if derivative else density_form_factor
                out[s] = torch.from_numpy(fn(p.grid, p.core_density, self.q)).to(self.dev)
        return out

    def phases(self, atoms):
        pos = torch.from_numpy(self.system.positions[atoms]).to(self.dev)
        return torch.exp(-1j * (pos @ self.g.T))  # (len(atoms), nG)


def _tables(system, dev):
    t = getattr(system, "_sphere_tables", None)
    if t is None:
        t = _SphereTables(system, dev)
        system._sphere_tables = t
    return t


def _atom_chunks(natoms, nG, budget=2**27):
    step = max(1, budget // max(nG, 1))
    for a in range(0, natoms, step):
        yield list(range(a, min(natoms, a + step)))


def _blocks(wavefunctions, spin, ik, dev):
    return _as_dev(wavefunctions[spin][ik], dev)


def _nonlocal_forces(system, wavefunctions, occupations, dev):
    eng = engine_for(system)
    natoms = system.natoms
    forces = torch.zeros((natoms, 3), dtype=torch.float64, device=dev)
    if eng.nproj == 0:
        return forces
    g = 2.0 / system.nspin
    labels = system.projectors[0].labels
    atom_of_row = torch.tensor([lab[0] for lab in labels], device=dev)
    dij = torch.from_numpy(system.projectors[0].dij).to(dev, torch.complex128)
    for spin in range(system.nspin):
        for ik, sphere in enumerate(system.wave_spheres):
            w = g * system.kpoints.weights[ik] * np.asarray(occupations)[spin, ik]
            active = np.nonzero(w > 1e-12)[0]
            if active.size == 0:
                continue
            block = _blocks(wavefunctions, spin, ik, dev)[torch.from_numpy(active).to(dev)].contiguous()
            wt = torch.from_numpy(w[active]).to(dev)
            coupled = eng.project(block, ik).to(torch.complex128) @ dij
            kg = torch.from_numpy(sphere.cartesian).to(dev)
            for axis in range(3):
                deriv_in = (block * (1j * kg[:, axis]).to(block.dtype)).contiguous()
                deriv = eng.project(deriv_in, ik).to(torch.complex128)
                terms = 2.0 * (coupled.conj() * deriv).real
                per_proj = wt @ terms
                forces[:, axis].index_add_(0, atom_of_row, -per_proj)
    return forces


def _xc_potential_mean(system, density):
    ops = grid_ops(system)
    d = density.reshape(system.nspin, -1)
    xc_d = d
    if system.core_density is not None:
        xc_d = d + torch.from_numpy(system.core_density.ravel()).to(d.device)[None] / system.nspin
    e_xc, v_xc, outer = ops.xc(xc_d, system.xc)
    return e_xc, v_xc, xc_d, outer


def compute_forces(system, density, wavefunctions, occupations, *, eigenvalues=None, symmetrize=True,
                   decompose=False):
    """Forces in Ha/Bohr, shape (natoms, 3) (a dict of contributions with decompose)."""
    dev = require_cuda()
    rho = _as_dev(density, dev, torch.float64).reshape(system.nspin, -1)
    tabs = _tables(system, dev)
    n_g = density_coefficients(system, rho.sum(0))
    charges = np.array([system.pseudopotentials[s].valence_charge for s in system.symbols])
    out = {"ewald": ewald(system.cell, system.positions, charges).forces}
    local = torch.zeros((system.natoms, 3), dtype=torch.float64, device=dev)
    for atoms in _atom_chunks(system.natoms, len(tabs.q)):
        ph = tabs.phases(atoms)
        ff = torch.stack([tabs.vloc[system.symbols[a]] for a in atoms])
        weight = 1j * ff * ph.conj() * n_g[None, :]
        local[atoms] = -(weight @ tabs.g.to(torch.complex128)).real
    out["local"] = local.cpu().numpy()
    out["nonlocal"] = _nonlocal_forces(system, wavefunctions, occupations, dev).cpu().numpy()
    if system.core_density is not None:
        _, v_xc, _, _ = _xc_potential_mean(system, rho)
        v_g = density_coefficients(system, v_xc.mean(0))
        core = tabs.core()
        cf = torch.zeros((system.natoms, 3), dtype=torch.float64, device=dev)
        for atoms in _atom_chunks(system.natoms, len(tabs.q)):
            ph = tabs.phases(atoms)
            for j, a in enumerate(atoms):
                c = core[system.symbols[a]]
                if c is None:
                    continue
                w = 1j * v_g.conj() * c * ph[j]
                cf[a] = (w @ tabs.g.to(torch.complex128)).real
        out["core"] = cf.cpu().numpy()
    return out if decompose else sum(out.values())


def _projector_q_gradient(system, sphere):
    """dP_i/dq_alpha for every projector row, shape (3, nproj, npw) (host FP64)."""
    qv = sphere.cartesian
    q = np.sqrt(sphere.g2)
    nz = q > 1e-12
    inv = np.zeros_like(q)
    inv[nz] = 1.0 / q[nz]
    pref = 4.0 * np.pi / np.sqrt(system.grid.volume)
    rows = []
    cache = {}
    for atom, symbol in enumerate(system.symbols):
        pseudo = system.pseudopotentials[symbol]
        phase = np.exp(-1j * (qv @ system.positions[atom]))
        for proj in pseudo.projectors:
            key = (symbol, proj.l, proj.index)
            if key not in cache:
                l = proj.l
                radial = projector_form_factor(pseudo.grid, proj, q)
                slope = projector_form_factor_derivative(pseudo.grid, proj, q)
                harm = real_spherical_harmonics(l, qv)
                grads = solid_harmonics_gradient(l, qv)
                power = inv**l if l else np.ones_like(q)
                ang = []
                for m in range(2 * l + 1):
                    ang.append(grads[m] * (radial * power)[:, None]
                               - l * (harm[m] * radial * inv**2)[:, None] * qv
                               + (harm[m] * slope * inv)[:, None] * qv)
                cache[key] = (l, ang)
            l, ang = cache[key]
            for a in ang:
                rows.append(pref * (-1j) ** l * a * phase[:, None])
    return np.asarray(rows).transpose(2, 0, 1)


def _nonlocal_stress(system, wavefunctions, occupations, dev):
    eng = engine_for(system)
    stress = torch.zeros((3, 3), dtype=torch.float64, device=dev)
    energy = 0.0
    if eng.nproj == 0:
        return np.zeros((3, 3))
    g = 2.0 / system.nspin
    dij = torch.from_numpy(system.projectors[0].dij).to(dev, torch.complex128)
    for ik, sphere in enumerate(system.wave_spheres):
        grad = torch.from_numpy(_projector_q_gradient(system, sphere)).to(dev)  # (3, nproj, npw)
        q = torch.from_numpy(sphere.cartesian).to(dev)
        for spin in range(system.nspin):
            w = g * system.kpoints.weights[ik] * np.asarray(occupations)[spin, ik]
            active = np.nonzero(w > 1e-12)[0]
            if active.size == 0:
                continue
            block = _blocks(wavefunctions, spin, ik, dev)[torch.from_numpy(active).to(dev)]
            block = block.to(torch.complex128).contiguous()
            wt = torch.from_numpy(w[active]).to(dev)
            projected = eng.project(block, ik) if block.dtype == torch.complex128 else None
            if projected is None:
                projected = gemm_nc(block, torch.from_numpy(system.projectors[ik].matrix).to(dev))
            coupled = projected @ dij
            energy += float((wt[:, None] * coupled * projected.conj()).sum().real)
            for mu in range(3):
                for nu in range(3):
                    m = (grad[mu] * q[:, nu][None, :]).contiguous()
                    partial = gemm_nc(block, m)  # sum_G c conj(dP_mu q_nu)
                    stress[mu, nu] -= (wt[:, None] * coupled.conj() * partial).sum().real
    stress = stress + stress.T
    return ((stress - torch.eye(3, device=dev, dtype=torch.float64) * energy) / system.grid.volume).cpu().numpy()


def compute_stress(system, density, wavefunctions, occupations, *, eigenvalues=None, symmetrize=True,
                   decompose=False):
    """Stress tensor in Ha/Bohr^3 (a dict of contributions with decompose)."""
    dev = require_cuda()
    vol = system.grid.volume
    rho = _as_dev(density, dev, torch.float64).reshape(system.nspin, -1)
    total = rho.sum(0)
    tabs = _tables(system, dev)
    n_g = density_coefficients(system, total)
    charges = np.array([system.pseudopotentials[s].valence_charge for s in system.symbols])
    out = {"ewald": ewald(system.cell, system.positions, charges).stress}
    # kinetic
    g = 2.0 / system.nspin
    kin = torch.zeros((3, 3), dtype=torch.float64, device=dev)
    for spin in range(system.nspin):
        for ik, sphere in enumerate(system.wave_spheres):
            w = torch.from_numpy(g * system.kpoints.weights[ik] * np.asarray(occupations)[spin, ik]).to(dev)
            c = _blocks(wavefunctions, spin, ik, dev)
            amp = w @ (c.real.double() ** 2 + c.imag.double() ** 2)
            kg = torch.from_numpy(sphere.cartesian).to(dev)
            kin -= torch.einsum("g,gu,gv->uv", amp, kg, kg)
    out["kinetic"] = (kin / vol).cpu().numpy()
    # Hartree
    ops = grid_ops(system)
    e_h, _ = ops.hartree(total)
    nz = tabs.g2 > 1e-12
    wgt = 4.0 * np.pi * (n_g[nz].abs() ** 2) / tabs.g2[nz] ** 2
    gv = tabs.g[nz]
    out["hartree"] = (-torch.eye(3, device=dev, dtype=torch.float64) * float(e_h) / vol
                      + torch.einsum("g,gu,gv->uv", wgt, gv, gv)).cpu().numpy()
    # local
    q = torch.from_numpy(tabs.q).to(dev)
    ratio = torch.where(q > 1e-12, 1.0 / torch.where(q > 1e-12, q, torch.ones_like(q)), torch.zeros_like(q))
    slope = tabs.vloc_slope()
    energy = 0.0
    tensor = torch.zeros((3, 3), dtype=torch.float64, device=dev)
    for atoms in _atom_chunks(system.natoms, len(tabs.q)):
        ph = tabs.phases(atoms)
        for j, a in enumerate(atoms):
            s = system.symbols[a]
            energy += float((tabs.vloc[s] * ph[j].conj() * n_g).real.sum())
            w = (slope[s] * ratio * ph[j].conj() * n_g).real
            tensor -= torch.einsum("g,gu,gv->uv", w, tabs.g, tabs.g)
    out["local"] = ((-torch.eye(3, device=dev, dtype=torch.float64) * energy + tensor) / vol).cpu().numpy()
    out["nonlocal"] = _nonlocal_stress(system, wavefunctions, occupations, dev)
    # xc: delta_uv (E_xc - sum_s int v_xc^s n_s), minus the GGA gradient outer product
    e_xc, v_xc, xc_d, outer = _xc_potential_mean(system, rho)
    dc = float((v_xc * xc_d).sum()) * system.grid.cell_volume_per_point
    xc_stress = np.eye(3) * (float(e_xc) - dc)
    if outer is not None:
        xc_stress = xc_stress - outer.cpu().numpy()
    out["xc"] = xc_stress / vol
    if system.core_density is not None:
        v_g = density_coefficients(system, v_xc.mean(0))
        core_d = tabs.core(derivative=True)
        ct_ = torch.zeros((3, 3), dtype=torch.float64, device=dev)
        for atoms in _atom_chunks(system.natoms, len(tabs.q)):
            ph = tabs.phases(atoms)
            for j, a in enumerate(atoms):
                c = core_d[system.symbols[a]]
                if c is None:
                    continue
                w = (v_g.conj() * c * ratio * ph[j]).real
                ct_ -= torch.einsum("g,gu,gv->uv", w, tabs.g, tabs.g)
        out["core"] = (ct_ / vol).cpu().numpy()
    return out if decompose else sum(out.values())
