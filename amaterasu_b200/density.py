"""Drop-in ``compute_density``: occupation-weighted |psi(r)|^2 on the GPU.

Mirrors amaterasu ``scf/density.py:35-84``: n_s(r) = (1/Omega) sum_k w_k sum_n g f |u|^2
with g = 2/nspin, bands with g w f <= 1e-12 skipped, then (symmetry being off) the floor
at zero with the per-channel rescale that restores the charge. The transform and the
accumulation run in one batched engine call per spin over all k-points (FP64 accumulation
whatever the wavefunction precision).
"""
from __future__ import annotations

import numpy as np
import torch

from .engine import engine_for, require_cuda

__all__ = ["compute_density", "electron_count", "accumulate_packed", "finalize_density"]


def electron_count(system, density) -> float:
    d = density.sum() if isinstance(density, torch.Tensor) else np.sum(density)
    return float(d) * system.grid.cell_volume_per_point


def band_weights(system, occupations, spin: int) -> np.ndarray:
    g = 2.0 / system.nspin
    w = g * np.asarray(system.kpoints.weights)[:, None] * np.asarray(occupations)[spin]
    return np.where(w > 1e-12, w, 0.0)


def accumulate_packed(system, packed: torch.Tensor, nbands: int, weights: np.ndarray, rho: torch.Tensor,
                      k_first: int = 0, k_count: int | None = None) -> None:
    """rho += sum over the packed all-k block of weights * |u|^2 (no 1/Omega)."""
    eng = engine_for(system)
    k_count = eng.nk - k_first if k_count is None else k_count
    wt = torch.from_numpy(np.ascontiguousarray(weights[k_first:k_first + k_count].ravel(), dtype=np.float64))
    eng.density_accumulate(packed, wt.to(rho.device), rho, k_first=k_first, k_count=k_count, nbands=nbands)


def finalize_density(system, rho: torch.Tensor, symmetrize: bool = True) -> torch.Tensor:
    """Divide by Omega; with ``symmetrize`` (symmetry being off, only the floor) also floor at
    zero and rescale each channel to its charge (``ama_density_floor``, in place)."""
    from ._lib import call
    from .engine import ptr, stream_ptr
    rho = rho.contiguous()
    nch, n = rho.shape[0], rho[0].numel()
    if symmetrize:
        call("ama_density_floor", nch, n, float(system.grid.volume), ptr(rho), stream_ptr())
        return rho
    from .mixing import _lincomb
    return _lincomb([rho.reshape(-1)], [1.0 / system.grid.volume]).reshape(rho.shape)


def compute_density(system, wavefunctions, occupations, *, symmetrize: bool = True):
    """Density of shape (nspin, n1, n2, n3) in electrons/Bohr^3."""
    dev = require_cuda()
    eng = engine_for(system)
    first = wavefunctions[0][0]
    as_numpy = not isinstance(first, torch.Tensor)
    occ = occupations.cpu().numpy() if isinstance(occupations, torch.Tensor) else np.asarray(occupations)
    rho = torch.zeros((system.nspin, eng.N), dtype=torch.float64, device=dev)
    for spin in range(system.nspin):
        blocks = wavefunctions[spin]
        nbands = blocks[0].shape[0]
        if any(b.shape[0] != nbands for b in blocks):
            raise ValueError("every k-point must carry the same number of bands")
        tens = [b if isinstance(b, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(b)) for b in blocks]
        dtype = torch.complex64 if tens[0].dtype == torch.complex64 else torch.complex128
        packed = torch.cat([t.to(dev, dtype).reshape(-1) for t in tens])
        accumulate_packed(system, packed, nbands, band_weights(system, occ, spin), rho[spin])
    rho = finalize_density(system, rho, symmetrize).reshape(system.nspin, *system.grid.shape)
    return rho.cpu().numpy() if as_numpy else rho
