"""The hand-written FP64 Hermitian eigensolver and inverse Cholesky factor against LAPACK
(numpy on the host), through the C-ABI.

They stand in for scipy.linalg.eigh / cholesky + solve_triangular in the reference's
Rayleigh-Ritz and orthonormalisation (amaterasu scf/eigen/subspace.py:17-32,63-76).
Tolerances: eigenvalues 1e-12 of ||A||, residual ||A z - lambda z|| 1e-12 of ||A||,
orthonormality 1e-12; inverse Cholesky factor: L^{-1} S L^{-H} = I to 1e-11.
"""
import ctypes as ct

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _random_hermitian(n, seed, spectrum=None):
    rng = np.random.default_rng(seed)
    if spectrum is None:
        a = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))
        return 0.5 * (a + a.conj().T)
    q, _ = np.linalg.qr(rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n)))
    a = (q * spectrum) @ q.conj().T
    return 0.5 * (a + a.conj().T)


def _solve(mats, nvec=None):
    """Eigenpairs through ama_heev (nvec None) or ama_heev_lowest, batch of matrices."""
    from amaterasu_b200._lib import call
    from amaterasu_b200.engine import ptr, stream_ptr
    batch, n, _ = mats.shape
    m = torch.from_numpy(np.ascontiguousarray(mats)).cuda()
    w = torch.empty((batch, n), dtype=torch.float64, device="cuda")
    if nvec is None:
        call("ama_heev", n, ptr(m), ptr(w), batch, stream_ptr())
        nvec = n
    else:
        call("ama_heev_lowest", n, nvec, ptr(m), ptr(w), batch, stream_ptr())
    torch.cuda.synchronize()
    return w.cpu().numpy()[:, :nvec], m.cpu().numpy()[:, :, :nvec]


def _check(a, w, z, tol=1e-12):
    nvec = w.shape[0]
    scale = max(np.abs(np.linalg.eigvalsh(a)).max(), 1.0)
    exact = np.linalg.eigvalsh(a)[:nvec]
    assert np.abs(w - exact).max() <= tol * scale, f"eigenvalues off by {np.abs(w - exact).max():.2e}"
    res = np.linalg.norm(a @ z - z * w, axis=0).max()
    assert res <= tol * scale * 10, f"residual {res:.2e}"
    orth = np.abs(z.conj().T @ z - np.eye(nvec)).max()
    assert orth <= tol * 10, f"orthonormality {orth:.2e}"


def _status():
    from amaterasu_b200._lib import call
    code = ct.c_int32(0)
    call("ama_solver_status", ct.byref(code))
    return code.value


@pytest.mark.parametrize("n", [1, 2, 3, 5, 40, 81, 150, 333])
def test_heev_random_matches_lapack(n):
    a = _random_hermitian(n, n)
    w, z = _solve(a[None])
    _check(a, w[0], z[0])
    assert _status() == 0


@pytest.mark.parametrize("n,nvec", [(200, 50), (881, 440), (1320, 440)])
def test_heev_lowest_matches_lapack(n, nvec):
    a = _random_hermitian(n, 1000 + n)
    w, z = _solve(a[None], nvec)
    _check(a, w[0], z[0])
    assert _status() == 0


def test_heev_degenerate_and_clustered_spectra():
    """Exactly repeated eigenvalues (symmetry-degenerate bands) and a 1e-12-spaced cluster
    get orthonormal eigenvectors of the right eigenspaces."""
    n = 120
    rng = np.random.default_rng(7)
    ev = np.sort(rng.normal(size=n))
    ev[3:6] = ev[3]
    ev[10:14] = ev[10]
    ev[40:44] = ev[40] + 1e-12 * np.arange(4)
    a = _random_hermitian(n, 8, ev)
    for nvec in (None, 60):
        w, z = _solve(a[None], nvec)
        _check(a, w[0], z[0])


def test_heev_batch_diagonal_and_identity():
    """Batched call; a diagonal matrix (every reflector degenerate) and the identity."""
    n = 64
    d = np.diag(np.linspace(-3.0, 5.0, n)[::-1]).astype(complex)
    eye = np.eye(n, dtype=complex)
    mats = np.stack([d, eye, _random_hermitian(n, 3)])
    w, z = _solve(mats)
    for b in range(3):
        _check(mats[b], w[b], z[b])


def test_heev_rejects_oversized_order():
    from amaterasu_b200._lib import call
    from amaterasu_b200.engine import ptr, stream_ptr
    m = torch.zeros(1, dtype=torch.complex128, device="cuda")
    w = torch.zeros(1, dtype=torch.float64, device="cuda")
    with pytest.raises(ValueError):
        call("ama_heev", 5000, ptr(m), ptr(w), 1, stream_ptr())


def test_inverse_cholesky_factor():
    from amaterasu_b200.linalg import cholesky_inverse_factor
    for n, seed in ((1, 0), (7, 1), (120, 2), (440, 3)):
        rng = np.random.default_rng(seed)
        b = rng.normal(size=(n, n + 3)) + 1j * rng.normal(size=(n, n + 3))
        s = b @ b.conj().T
        linv = cholesky_inverse_factor(torch.from_numpy(s).cuda()).cpu().numpy()
        assert np.abs(np.triu(linv, 1)).max() == 0.0
        np.testing.assert_allclose(linv @ s @ linv.conj().T, np.eye(n), rtol=0, atol=1e-11)
        np.testing.assert_allclose(np.linalg.inv(linv), np.linalg.cholesky(s), rtol=0,
                                   atol=1e-11 * np.abs(np.linalg.cholesky(s)).max())


def test_inverse_cholesky_rejects_indefinite():
    from amaterasu_b200._lib import AmaError
    from amaterasu_b200.linalg import cholesky_inverse_factor
    s = np.diag([1.0, -1.0, 2.0]).astype(complex)
    with pytest.raises(AmaError):
        cholesky_inverse_factor(torch.from_numpy(s).cuda())


def test_heev_dense_valence_like_spectrum():
    """A Rayleigh-Ritz-like spectrum: the lowest 440 of 880 eigenvalues packed into 0.5 Ha
    (gaps ~1e-3 Ha, a few exact pairs) under a wide upper part; then a Gram-like matrix whose
    eigenvalues all sit within 1e-7 of 1."""
    rng = np.random.default_rng(11)
    low = np.sort(rng.uniform(-0.3, 0.2, 440))
    low[100] = low[101]
    low[300] = low[301] = low[302]
    ev = np.concatenate([low, np.sort(rng.uniform(1.0, 30.0, 440))])
    a = _random_hermitian(880, 12, ev)
    w, z = _solve(a[None], 440)
    _check(a, w[0], z[0])
    gram = _random_hermitian(300, 13, 1.0 + 1e-7 * rng.normal(size=300))
    w, z = _solve(gram[None])
    _check(gram, w[0], z[0])
    assert _status() == 0
