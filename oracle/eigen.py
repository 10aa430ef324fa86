"""Block Davidson with the Teter-Payne-Allan preconditioner (FP64 numpy/scipy).

Follows amaterasu ``scf/eigen/davidson.py:48-111``, ``scf/eigen/subspace.py:17-88``
(orthonormalize, orthogonalize_against, rayleigh_ritz, random_bands) and
``scf/eigen/precond.py:27-46``.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
from scipy.linalg import cholesky, eigh, solve_triangular


def orthonormalize(block):
    block = np.asarray(block, dtype=complex)
    overlap = block @ block.conj().T
    try:
        factor = cholesky(overlap, lower=True)
    except np.linalg.LinAlgError:
        return _svd_orthonormalize(block)
    result = solve_triangular(factor, block, lower=True)
    if not np.all(np.isfinite(result)):
        return _svd_orthonormalize(block)
    return result


def _svd_orthonormalize(block, threshold=1e-10):
    _, s, vh = np.linalg.svd(block, full_matrices=False)
    return vh[s > threshold * max(float(s[0]), 1e-300)]


def orthogonalize_against(block, basis, *, threshold=1e-7):
    block = np.asarray(block, dtype=complex)
    for _ in range(2):
        block = block - (block @ basis.conj().T) @ basis
    norms = np.linalg.norm(block, axis=1)
    block = block[norms > threshold]
    if len(block) == 0:
        return block
    _, s, vh = np.linalg.svd(block, full_matrices=False)
    return vh[s > threshold * float(s[0])]


def rayleigh_ritz(basis, h_basis, nbands):
    projected = basis.conj() @ h_basis.T
    projected = 0.5 * (projected + projected.conj().T)
    values, vectors = eigh(projected)
    rotation = vectors[:, :nbands].T
    return values[:nbands], rotation @ basis, rotation @ h_basis


def random_bands(npw, nbands, kinetic, seed=0):
    rng = np.random.default_rng(seed)
    block = rng.normal(size=(nbands, npw)) + 1j * rng.normal(size=(nbands, npw))
    return orthonormalize(block / (1.0 + kinetic))


def teter_payne_allan(residual, kinetic, reference):
    reference = np.maximum(np.atleast_1d(np.asarray(reference, dtype=float)), 1e-8)
    x = kinetic[None, :] / reference[:, None]
    poly = 27.0 + x * (18.0 + x * (12.0 + 8.0 * x))
    return residual * (poly / (poly + 16.0 * x**4))


@dataclass
class DavidsonResult:
    eigenvalues: np.ndarray
    coefficients: np.ndarray
    residual_norms: np.ndarray
    iterations: int
    converged: bool


def davidson(apply_h, guess, kinetic, *, tolerance=1e-8, max_iterations=40, subspace_factor=4):
    basis = orthonormalize(np.asarray(guess, dtype=complex))
    nbands, npw = basis.shape
    max_subspace = min(max(subspace_factor, 2) * nbands, npw)
    h_basis = apply_h(basis)
    eigenvalues, vectors, h_vectors = rayleigh_ritz(basis, h_basis, nbands)
    norms = np.full(nbands, np.inf)
    iteration = 0
    for iteration in range(1, max_iterations + 1):
        residual = h_vectors - eigenvalues[:, None] * vectors
        norms = np.linalg.norm(residual, axis=1)
        active = norms > tolerance
        if not np.any(active):
            break
        band_kinetic = np.einsum("ng,g->n", np.abs(vectors[active]) ** 2, kinetic)
        correction = teter_payne_allan(residual[active], kinetic, band_kinetic)
        correction /= np.maximum(np.linalg.norm(correction, axis=1, keepdims=True), 1e-300)
        new = orthogonalize_against(correction, basis)
        if len(new) == 0:
            break
        basis = np.vstack([basis, new])
        h_basis = np.vstack([h_basis, apply_h(new)])
        eigenvalues, vectors, h_vectors = rayleigh_ritz(basis, h_basis, nbands)
        if len(basis) + nbands > max_subspace:
            basis, h_basis = vectors, h_vectors
    return DavidsonResult(eigenvalues, vectors, norms, iteration, bool(np.all(norms <= tolerance)))
