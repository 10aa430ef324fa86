"""Local ionic potential and superposed atomic densities on the real-space grid (set-up).

Restates amaterasu ``hamiltonian/local.py``: per-species radial transforms on the density
sphere combined with phases ``e^{-iG.tau}``, divided by Omega, scattered to the grid and
transformed with no 1/N (:37-74); the valence density is floored at 1e-12 and rescaled
to the electron count (:77-106). These run once per geometry in FP64: the structure sums on
the GPU (ama_structure_sum) when one is present, else on the host; the transform to the
grid on the host.
"""
from __future__ import annotations

import numpy as np
import scipy.fft as _sfft

from .formfactors import density_form_factor, local_potential_form_factor


def structure_factors(sphere, positions) -> np.ndarray:
    return np.exp(-1j * (np.atleast_2d(positions) @ sphere.cartesian.T))


def _to_real_grid(grid, sphere, coefficients) -> np.ndarray:
    field = np.zeros(tuple(grid.shape), dtype=complex)
    i, j, k = grid.indices(sphere)
    field[i, j, k] = coefficients
    return _sfft.ifftn(field, norm="forward")


def _device_structure_sum(sphere, positions, symbols, radial, scale):
    """sum_a radial[symbol_a](G) exp(-i G.tau_a) * scale through ama_structure_sum when a
    CUDA device is present (the atoms x G phase matrix of the host form is ~2 GB and
    seconds of exp() at 215 atoms and 30 Ry); None without one."""
    try:
        import torch
        if not torch.cuda.is_available():
            return None
        import ctypes as ct

        from ._lib import call, load
        load()
    except Exception:
        return None
    names = sorted(radial)
    dev = torch.device("cuda", torch.cuda.current_device())
    g = torch.from_numpy(np.ascontiguousarray(sphere.cartesian, dtype=np.float64)).to(dev)
    pos = torch.from_numpy(np.ascontiguousarray(np.atleast_2d(positions), dtype=np.float64)).to(dev)
    spc = torch.tensor([names.index(s) for s in symbols], dtype=torch.int32, device=dev)
    rad = torch.from_numpy(np.ascontiguousarray(np.stack([np.asarray(radial[s], float) for s in names]))).to(dev)
    out = torch.empty(len(sphere), dtype=torch.complex128, device=dev)
    stream = torch.cuda.current_stream(dev)
    call("ama_structure_sum", ct.c_void_p(g.data_ptr()), len(sphere), ct.c_void_p(pos.data_ptr()),
         ct.c_void_p(spc.data_ptr()), len(symbols), ct.c_void_p(rad.data_ptr()), float(scale),
         ct.c_void_p(out.data_ptr()), ct.c_void_p(stream.cuda_stream))
    return out.cpu().numpy()


def _superpose(grid, sphere, positions, symbols, radial) -> np.ndarray:
    coefficients = _device_structure_sum(sphere, positions, symbols, radial, 1.0 / grid.volume)
    if coefficients is None:  # host form (CPU-only set-up, tests)
        phases = structure_factors(sphere, positions)
        coefficients = np.zeros(len(sphere), dtype=complex)
        for atom, symbol in enumerate(symbols):
            coefficients += radial[symbol] * phases[atom]
        coefficients /= grid.volume
    return _to_real_grid(grid, sphere, coefficients)


def _real(field, what: str) -> np.ndarray:
    scale = float(np.max(np.abs(field.real)))
    residual = float(np.max(np.abs(field.imag)))
    if scale > 0 and residual > 1e-8 * scale:
        raise ValueError(f"the {what} came out complex ({residual:.3e} against {scale:.3e})")
    return np.ascontiguousarray(field.real)


def local_potential(grid, sphere, positions, symbols, pseudopotentials) -> np.ndarray:
    q = np.sqrt(sphere.g2)
    radial = {s: local_potential_form_factor(p, q) for s, p in pseudopotentials.items()}
    return _real(_superpose(grid, sphere, positions, symbols, radial), "local potential")


def atomic_valence_density(grid, sphere, positions, symbols, pseudopotentials, *,
                           total_electrons=None) -> np.ndarray:
    q = np.sqrt(sphere.g2)
    radial = {}
    for symbol, pseudo in pseudopotentials.items():
        if pseudo.valence_density is None:
            raise ValueError(f"{symbol}: the dataset carries no atomic valence density")
        radial[symbol] = density_form_factor(pseudo.grid, pseudo.valence_density, q)
    density = _real(_superpose(grid, sphere, positions, symbols, radial), "valence density")
    density = np.maximum(density, 1e-12)
    if total_electrons is not None:
        current = float(np.sum(density)) * grid.cell_volume_per_point
        density *= total_electrons / current
    return density


def atomic_core_density(grid, sphere, positions, symbols, pseudopotentials):
    if not any(p.has_core_correction for p in pseudopotentials.values()):
        return None
    q = np.sqrt(sphere.g2)
    radial = {}
    for symbol, pseudo in pseudopotentials.items():
        radial[symbol] = (np.zeros_like(q) if pseudo.core_density is None
                          else density_form_factor(pseudo.grid, pseudo.core_density, q))
    return _real(_superpose(grid, sphere, positions, symbols, radial), "core density")
