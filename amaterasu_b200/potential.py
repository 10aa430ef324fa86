"""Effective potential on the GPU in FP64: Hartree (reciprocal-space filter kernel),
exchange-correlation (LDA-PZ pointwise kernel; PBE and PBEsol with spectral gradients and
divergence) and the local ionic potential.

Mirrors amaterasu ``scf/driver.py:225-252`` (``effective_potential``),
``hamiltonian/hartree.py:28-50`` and ``xc/driver.py:108-165`` (the unpolarised density is
split n/2, n/2 and the spin-polarised functional evaluated; a GGA adds
-div(2 vsigma_ss grad n_s + vsigma_ud grad n_s') to the potential).
"""
from __future__ import annotations

import ctypes as ct

import numpy as np
import torch

from ._lib import call
from .engine import engine_for, ptr, stream_ptr

HARTREE_SLOT = 0
KERKER_SLOT = 1
BANDLIMIT_SLOT = 2
#: functional name (as the reference spells it, case-insensitive) -> (kind, GGA code)
FUNCTIONALS = {"LDA-PZ": ("lda", None), "PBE": ("gga", 0), "PBESOL": ("gga", 1)}


def functional_key(name) -> str:
    """Canonical key of a functional name or of an object with a ``name`` (the reference's
    XCFunctional)."""
    key = str(getattr(name, "name", name)).strip().upper().replace("_", "-")
    if key not in FUNCTIONALS:
        raise NotImplementedError(f"functional {name!r}: the engine implements "
                                  f"{', '.join(('LDA-PZ', 'PBE', 'PBEsol'))}")
    return key


class GridOps:
    """Grid-space FP64 operations of one FFT grid: the Hartree filter (when the density
    sphere is known), the Kerker filter and LDA-PZ. Cached on the system (and on its grid)
    or, for a bare grid, on the grid object with an engine of its own."""

    def __init__(self, grid, engine, density_sphere=None):
        self.grid = grid
        self.engine = engine
        self.device = self.engine.device
        self.shape = tuple(int(n) for n in grid.shape)
        self.N = int(np.prod(self.shape))
        self.volume = abs(float(np.linalg.det(np.asarray(grid.cell, dtype=float))))
        self.dv = self.volume / self.N
        if density_sphere is not None:
            sphere = density_sphere
            h = np.stack([sphere.miller[:, a] % self.shape[a] for a in range(3)])
            flat = ((h[0] * self.shape[1] + h[1]) * self.shape[2] + h[2]).astype(np.int64)
            f = np.zeros(self.N)
            nz = sphere.g2 > 1e-12
            f[flat[nz]] = 4.0 * np.pi / sphere.g2[nz]
            call("ama_set_grid_filter", self.engine.handle, HARTREE_SLOT, f.ctypes.data_as(ct.c_void_p))
        self._kerker_q0 = None
        self._energy = torch.zeros(1, dtype=torch.float64, device=self.device)

    def hartree(self, total: torch.Tensor):
        """(E_H in Hartree as a 0-d device tensor, V_H(r) flat) for a total density."""
        total = total.reshape(-1).to(self.device, torch.float64).contiguous()
        out = torch.empty_like(total)
        self._energy.zero_()
        call("ama_grid_filter", self.engine.handle, HARTREE_SLOT, HARTREE_SLOT, ptr(total), ptr(out),
             ptr(self._energy), stream_ptr())
        return self._energy[0] * (0.5 * self.volume), out

    def set_kerker(self, q0: float, uniform_factor: float = 0.0):
        if self._kerker_q0 == (q0, uniform_factor):
            return
        g = self.grid.gvectors_cartesian()
        g2 = np.einsum("...i,...i->...", g, g).ravel()
        with np.errstate(invalid="ignore", divide="ignore"):
            f = np.where(g2 > 1e-12, g2 / (g2 + q0**2), float(uniform_factor))
        f = np.ascontiguousarray(f, dtype=np.float64)
        call("ama_set_grid_filter", self.engine.handle, KERKER_SLOT, f.ctypes.data_as(ct.c_void_p))
        self._kerker_q0 = (q0, uniform_factor)

    def kerker(self, field: torch.Tensor) -> torch.Tensor:
        field = field.reshape(-1).to(self.device, torch.float64).contiguous()
        out = torch.empty_like(field)
        call("ama_grid_filter", self.engine.handle, KERKER_SLOT, -1, ptr(field), ptr(out), None,
             stream_ptr())
        return out

    def band_limit(self, field: torch.Tensor) -> torch.Tensor:
        """The field with every Fourier component at or beyond the Nyquist frequency of an
        even axis removed (|m_a| <= (n_a - 1) // 2 kept): the same-shape case of a
        band-limited resampling, as one grid-filter pass on the device."""
        if not getattr(self, "_band_limit_set", False):
            keep = np.ones(self.shape)
            for a, n in enumerate(self.shape):
                if n % 2 == 0:
                    idx = [slice(None)] * 3
                    idx[a] = n // 2
                    keep[tuple(idx)] = 0.0
            call("ama_set_grid_filter", self.engine.handle, BANDLIMIT_SLOT,
                 np.ascontiguousarray(keep.ravel()).ctypes.data_as(ct.c_void_p))
            self._band_limit_set = True
        field = field.reshape(-1).to(self.device, torch.float64).contiguous()
        out = torch.empty_like(field)
        call("ama_grid_filter", self.engine.handle, BANDLIMIT_SLOT, -1, ptr(field), ptr(out), None, stream_ptr())
        return out

    def lda(self, density: torch.Tensor):
        """(E_xc device scalar, v_xc (nspin, N)) for density (nspin, N) in electrons/Bohr^3."""
        d = density.reshape(density.shape[0], -1).to(self.device, torch.float64)
        nspin = d.shape[0]
        spin = torch.stack([0.5 * d[0], 0.5 * d[0]]) if nspin == 1 else d
        spin = spin.contiguous()
        eps = torch.empty(self.N, dtype=torch.float64, device=self.device)
        vrho = torch.empty((2, self.N), dtype=torch.float64, device=self.device)
        call("ama_lda_pz", ptr(spin), self.N, ptr(eps), ptr(vrho), stream_ptr())
        total = d[0].contiguous() if nspin == 1 else (spin[0] + spin[1])
        energy = torch.empty(1, dtype=torch.float64, device=self.device)
        call("ama_vec_reduce", 0, self.N, ptr(eps), ptr(total), float(self.dv), 0, ptr(energy), stream_ptr())
        return energy[0], vrho[:nspin]

    def gga(self, density: torch.Tensor, functional: str = "PBE"):
        """(E_xc device scalar, v_xc (nspin, N), gradient stress term (3, 3) device) for
        density (nspin, N): PBE or PBEsol, gradients and divergence in reciprocal space.
        The stress term is sum_r [2 vsigma_uu g_u g_u + vsigma_ud (g_u g_d + g_d g_u) +
        2 vsigma_dd g_d g_d] dV (the reference subtracts it from the xc stress)."""
        code = FUNCTIONALS[functional_key(functional)][1]
        if code is None:
            raise ValueError(f"{functional} is not a GGA")
        d = density.reshape(density.shape[0], -1).to(self.device, torch.float64).contiguous()
        nspin = d.shape[0]
        v = torch.empty_like(d)
        res = torch.empty(7, dtype=torch.float64, device=self.device)
        cell = np.ascontiguousarray(self.grid.cell, dtype=np.float64)
        call("ama_xc_gga", self.engine.handle, code, nspin, cell.ctypes.data_as(ct.c_void_p), ptr(d), ptr(v),
             ptr(res), stream_ptr())
        xx, yy, zz, yz, xz, xy = (res[i] for i in range(1, 7))
        outer = torch.stack([torch.stack([xx, xy, xz]), torch.stack([xy, yy, yz]), torch.stack([xz, yz, zz])])
        return res[0], v, outer

    def xc(self, density: torch.Tensor, functional: str = "LDA-PZ"):
        """(E_xc, v_xc (nspin, N), gradient stress term or None) for the system's functional."""
        kind = FUNCTIONALS[functional_key(functional)][0]
        if kind == "lda":
            e, v = self.lda(density)
            return e, v, None
        return self.gga(density, functional)


def grid_ops(system) -> GridOps:
    ops = getattr(system, "_grid_ops", None)
    if ops is None:
        ops = GridOps(system.grid, engine_for(system), system.density_sphere)
        system._grid_ops = ops
        try:
            system.grid._grid_ops = ops  # a mixer built from the bare grid reuses it
        except AttributeError:  # pragma: no cover - frozen grid objects
            pass
    return ops


def grid_ops_for_grid(grid) -> GridOps:
    """GridOps of a bare FFT grid (ours or the reference's: anything with ``shape``, ``cell``
    and ``gvectors_cartesian()``): the system's when the grid belongs to one, else one with a
    minimal engine of its own (Kerker filtering only)."""
    ops = getattr(grid, "_grid_ops", None)
    if ops is None:
        from .engine import GridEngine
        ops = GridOps(grid, GridEngine(grid.shape))
        grid._grid_ops = ops
    return ops


def effective_potential(system, density):
    """(v_eff (nspin, n1, n2, n3) device FP64, E_Hartree, E_xc) for a density."""
    ops = grid_ops(system)
    d = density if isinstance(density, torch.Tensor) else torch.from_numpy(np.asarray(density, float))
    d = d.to(ops.device, torch.float64).reshape(system.nspin, -1)
    e_h, v_h = ops.hartree(d.sum(0))
    xc_density = d
    if system.core_density is not None:
        core = torch.from_numpy(system.core_density.ravel()).to(ops.device)
        xc_density = d + core[None, :] / system.nspin
    e_xc, v_xc, _ = ops.xc(xc_density, system.xc)
    vloc = getattr(system, "_v_local_dev", None)
    if vloc is None:
        vloc = torch.from_numpy(system.v_local.ravel()).to(ops.device)
        system._v_local_dev = vloc
    v = vloc[None, :] + v_h[None, :] + v_xc
    return v.reshape(system.nspin, *ops.shape), float(e_h), float(e_xc)
