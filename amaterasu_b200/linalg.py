"""Device linear algebra for the subspace steps, on the engine's own kernels.

GEMMs go to ``ama_zgemm`` (hand-written complex GEMM, FP32 or FP64 by dtype); the small
dense FP64 factorisations (Hermitian eigensolve, inverse Cholesky factor) go to the
hand-written ``ama_heev`` / ``ama_potrf_inv`` (they stand in for the LAPACK routines the
reference reaches through scipy). All tensors are CUDA torch tensors, row-major, contiguous.
"""
from __future__ import annotations

import ctypes as ct

import torch

from ._lib import AMA_C64, AMA_C128, call
from .engine import ptr, stream_ptr

_PREC = {torch.complex64: AMA_C64, torch.complex128: AMA_C128}


def _scal(z: complex):
    return (ct.c_double * 2)(float(z.real), float(z.imag))


def _gemm(form, a, b, m, n, k, lda, ldb, out, alpha, beta):
    prec = _PREC[a.dtype]
    if b.dtype != a.dtype or out.dtype != a.dtype:
        raise TypeError("gemm operands must share one complex dtype")
    al, be = _scal(alpha), _scal(beta)
    call("ama_zgemm", prec, form, m, n, k, al, ptr(a), lda, 0, ptr(b), ldb, 0, be, ptr(out),
         out.stride(0) if out.dim() == 2 else n, 0, 1, stream_ptr())
    return out


def gemm_nn(a: torch.Tensor, b: torch.Tensor, out: torch.Tensor | None = None, alpha=1.0, beta=0.0):
    """out = alpha * a @ b + beta * out; a (m, k), b (k, n)."""
    m, k = a.shape
    k2, n = b.shape
    assert k == k2
    if out is None:
        out = torch.empty((m, n), dtype=a.dtype, device=a.device)
        beta = 0.0
    if m == 0 or n == 0:
        return out
    return _gemm(0, a, b, m, n, k, a.stride(0), b.stride(0), out, complex(alpha), complex(beta))


def gemm_nc(a: torch.Tensor, b: torch.Tensor, out: torch.Tensor | None = None, alpha=1.0, beta=0.0):
    """out = alpha * a @ b^H + beta * out; a (m, k), b (n, k)."""
    m, k = a.shape
    n, k2 = b.shape
    assert k == k2
    if out is None:
        out = torch.empty((m, n), dtype=a.dtype, device=a.device)
        beta = 0.0
    if m == 0 or n == 0:
        return out
    return _gemm(1, a, b, m, n, k, a.stride(0), b.stride(0), out, complex(alpha), complex(beta))


def heev(matrix: torch.Tensor):
    """Eigenvalues (ascending, FP64) and eigenvectors (columns) of a Hermitian matrix."""
    n = matrix.shape[0]
    work = matrix.to(torch.complex128).contiguous().clone()
    w = torch.empty(n, dtype=torch.float64, device=matrix.device)
    call("ama_heev", n, ptr(work), ptr(w), 1, stream_ptr())
    return w, work


def cholesky_inverse_factor(matrix: torch.Tensor) -> torch.Tensor:
    """L^{-1} with matrix = L L^H (FP64); raises ValueError-like AmaError if not SPD."""
    n = matrix.shape[0]
    work = matrix.to(torch.complex128).contiguous().clone()
    call("ama_potrf_inv", n, ptr(work), 1, stream_ptr())
    return work
