"""GPU Davidson and subspace steps against dense eigh, the oracle and the reference."""
import numpy as np
import pytest
import torch

from conftest import golden

pytestmark = pytest.mark.gpu


def _hermitian(n, seed):
    rng = np.random.default_rng(seed)
    a = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))
    kinetic = np.linspace(0.0, 20.0, n)
    return 0.05 * (a + a.conj().T) + np.diag(kinetic), kinetic


def test_davidson_matches_dense_eigh():
    """Mirror of the reference's test_eigen.py:28-41 (numpy callable, numpy guess)."""
    from amaterasu_b200.eigen import davidson
    matrix, kinetic = _hermitian(80, 0)
    rng = np.random.default_rng(1)
    guess = rng.normal(size=(6, 80)) + 1j * rng.normal(size=(6, 80))
    res = davidson(lambda b: b @ matrix.T, guess, kinetic, tolerance=1e-10, max_iterations=100)
    exact = np.linalg.eigvalsh(matrix)[:6]
    assert res.converged
    np.testing.assert_allclose(res.eigenvalues, exact, rtol=0, atol=1e-10)
    c = res.coefficients
    np.testing.assert_allclose(c @ c.conj().T, np.eye(6), atol=1e-12)
    # |d eps| <= ||r|| (test_eigen.py:44-55)
    assert np.all(np.abs(res.eigenvalues - exact) <= res.residual_norms + 1e-12)


def test_subspace_pieces_match_reference(mini_system):
    from amaterasu_b200.eigen import orthonormalize, random_bands, rayleigh_ritz, teter_payne_allan
    from amaterasu_b200.hamiltonian import Hamiltonian
    g = golden("mini.npz")
    s = mini_system
    H = Hamiltonian(s, g["veff"])
    for ik, sphere in enumerate(s.wave_spheres):
        guess = random_bands(len(sphere), s.nbands, sphere.kinetic_energy, seed=12345 + ik)
        np.testing.assert_allclose(guess, g[f"guess{ik}"], rtol=0, atol=1e-12)
        basis = orthonormalize(g[f"psi{ik}"][:4])
        np.testing.assert_allclose(basis, g[f"ortho{ik}"], rtol=0, atol=1e-11)
        e, x, hx = rayleigh_ritz(basis, H.apply(basis, ik), 3)
        np.testing.assert_allclose(e, g[f"rr_eig{ik}"], rtol=0, atol=1e-11)
        # the Ritz vectors themselves: H x is the rotated H basis and x^H H x = diag(e)
        np.testing.assert_allclose(hx, H.apply(x, ik), rtol=0, atol=1e-11)
        np.testing.assert_allclose(x.conj() @ hx.T, np.diag(e), rtol=0, atol=1e-11)
        out = teter_payne_allan(g[f"tpa_in{ik}"], sphere.kinetic_energy, g[f"tpa_ref{ik}"])
        np.testing.assert_allclose(out, g[f"tpa_out{ik}"], rtol=0, atol=1e-13)


@pytest.mark.parametrize("device_block", [False, True])
def test_davidson_engine_matches_reference(mini_system, device_block):
    from amaterasu_b200.eigen import davidson
    from amaterasu_b200.hamiltonian import Hamiltonian
    g = golden("mini.npz")
    s = mini_system
    H = Hamiltonian(s, g["veff"])
    for ik, sphere in enumerate(s.wave_spheres):
        guess = g[f"guess{ik}"]
        if device_block:
            guess = torch.from_numpy(guess).cuda()
        res = davidson(lambda b, ik=ik: H.apply(b, ik), guess, sphere.kinetic_energy, tolerance=1e-9,
                       max_iterations=60)
        eig = res.eigenvalues.cpu().numpy() if device_block else res.eigenvalues
        np.testing.assert_allclose(eig, g[f"dav_eig{ik}"], rtol=0, atol=1e-9)


def test_davidson_complex64_working_precision(mini_system):
    from amaterasu_b200.eigen import davidson
    from amaterasu_b200.hamiltonian import Hamiltonian
    g = golden("mini.npz")
    s = mini_system
    H = Hamiltonian(s, g["veff"], precision="complex64")
    guess = torch.from_numpy(g["guess0"]).cuda().to(torch.complex64)
    res = davidson(lambda b: H.apply(b, 0), guess, s.wave_spheres[0].kinetic_energy, tolerance=1e-4,
                   max_iterations=60)
    np.testing.assert_allclose(res.eigenvalues.cpu().numpy()[:5], g["dav_eig0"][:5], rtol=0, atol=2e-5)


def test_solve_dispatch_errors():
    from amaterasu_b200.eigen import solve
    with pytest.raises(NotImplementedError):
        solve("lobpcg", lambda b: b, np.eye(2), np.zeros(2))
    with pytest.raises(NotImplementedError):
        solve("davidson", lambda b: b, np.eye(2), np.zeros(2), apply_overlap=lambda b: b)


@pytest.mark.parametrize("n", [1, 2, 7, 20, 33, 80])
def test_batched_jacobi_matches_eigh(n):
    """ama_heev_small (one CTA per matrix, cyclic Jacobi) against numpy's eigh."""
    from amaterasu_b200._lib import call
    from amaterasu_b200.engine import ptr, stream_ptr
    rng = np.random.default_rng(n)
    batch = 5
    a = rng.normal(size=(batch, n, n)) + 1j * rng.normal(size=(batch, n, n))
    a = a + np.conj(np.transpose(a, (0, 2, 1)))
    a[1] = np.diag(np.repeat(np.arange(1, (n + 1) // 2 + 1), 2)[:n]).astype(complex)  # degenerate, already diagonal
    m = torch.from_numpy(a.copy()).cuda()
    w = torch.empty((batch, n), dtype=torch.float64, device="cuda")
    call("ama_heev_small", n, ptr(m), ptr(w), batch, stream_ptr())
    w = w.cpu().numpy()
    v = m.cpu().numpy()
    for b in range(batch):
        ref = np.linalg.eigvalsh(a[b])
        np.testing.assert_allclose(w[b], ref, rtol=0, atol=1e-11 * max(1.0, np.abs(ref).max()))
        np.testing.assert_allclose(v[b].conj().T @ v[b], np.eye(n), atol=1e-12)
        np.testing.assert_allclose(a[b] @ v[b], v[b] * w[b][None, :], atol=1e-10 * max(1.0, np.abs(ref).max()))


@pytest.mark.parametrize("dtype,tol", [(torch.complex128, 1e-9), (torch.complex64, 1e-5)])
def test_batched_davidson_matches_per_k(mini_system, dtype, tol):
    """All k-points in lockstep (batched launches) against the reference's per-k result."""
    from amaterasu_b200.batched import BatchedDavidson
    from amaterasu_b200.hamiltonian import Hamiltonian
    g = golden("mini.npz")
    s = mini_system
    H = Hamiltonian(s, g["veff"], precision="complex128" if dtype == torch.complex128 else "complex64")
    guess = torch.from_numpy(np.concatenate([g["guess0"].ravel(), g["guess1"].ravel()])).cuda().to(dtype)
    bd = BatchedDavidson(s, s.nbands, dtype)
    eps, X, norms, it = bd.run(H, guess, tolerance=tol, max_iterations=60)
    for ik in range(2):
        np.testing.assert_allclose(eps[ik][:5], g[f"dav_eig{ik}"][:5], rtol=0, atol=max(tol, 1e-9) * 10)
    # orthonormal Ritz vectors per k
    off = 0
    for ik, w in enumerate(s.wave_spheres):
        blk = X[off:off + s.nbands * len(w)].reshape(s.nbands, len(w)).to(torch.complex128).cpu().numpy()
        off += s.nbands * len(w)
        np.testing.assert_allclose(blk @ blk.conj().T, np.eye(s.nbands), atol=1e-5 if dtype == torch.complex64 else 1e-11)


@pytest.mark.parametrize("dtype,tol", [(torch.complex128, 1e-10), (torch.complex64, 2e-6)])
def test_library_davidson_matches_host_loop(mini_system, dtype, tol):
    """ama_davidson (the loop in C++) against the same loop with its host logic in Python
    over the same kernels: eigenvalues (1e-10 Ha complex128, 2e-6 complex64), iteration
    count, and the spans of the Ritz vectors (|<x_python|x_library>| singular values 1)."""
    from amaterasu_b200.batched import BatchedDavidson
    from amaterasu_b200.hamiltonian import Hamiltonian
    g = golden("mini.npz")
    s = mini_system
    H = Hamiltonian(s, g["veff"], precision="complex128" if dtype == torch.complex128 else "complex64")
    guess = torch.from_numpy(np.concatenate([g["guess0"].ravel(), g["guess1"].ravel()])).cuda().to(dtype)
    bd = BatchedDavidson(s, s.nbands, dtype)
    e1, x1, n1, it1 = bd.run(H, guess.clone(), tolerance=1e-7, max_iterations=40)
    e2, x2, n2, it2 = bd.run_python(H, guess.clone(), tolerance=1e-7, max_iterations=40)
    np.testing.assert_allclose(e1, e2, rtol=0, atol=tol)
    assert abs(it1 - it2) <= 1
    off = 0
    for w in s.wave_spheres:
        n = s.nbands * len(w)
        a = x1[off:off + n].reshape(s.nbands, len(w)).to(torch.complex128).cpu().numpy()
        b = x2[off:off + n].reshape(s.nbands, len(w)).to(torch.complex128).cpu().numpy()
        off += n
        sv = np.linalg.svd(a[:4] @ b[:4].conj().T, compute_uv=False)  # well-separated lowest bands
        np.testing.assert_allclose(sv, 1.0, atol=1e-6 if dtype == torch.complex64 else 1e-9)


@pytest.mark.parametrize("dtype", [torch.complex128, torch.complex64])
def test_library_davidson_graph_replay_is_identical(mini_system, dtype):
    """ama_davidson with its recurring iteration segments replayed as CUDA graphs against
    the same call launched kernel by kernel: bit-identical eigenvalues, vectors and residual
    norms, the same iteration count. Of three identical calls with graphs on, the third
    replays every segment (the first two launched or captured those not cached yet)."""
    from amaterasu_b200.batched import BatchedDavidson, graph_stats
    from amaterasu_b200.hamiltonian import Hamiltonian
    g = golden("mini.npz")
    s = mini_system
    H = Hamiltonian(s, g["veff"], precision="complex128" if dtype == torch.complex128 else "complex64")
    guess = torch.from_numpy(np.concatenate([g["guess0"].ravel(), g["guess1"].ravel()])).cuda().to(dtype)
    bd = BatchedDavidson(s, s.nbands, dtype)
    bd.graphs = False
    e0, x0, n0, it0 = bd.run(H, guess.clone(), tolerance=1e-7, max_iterations=40)
    bd.graphs = True
    graph_stats(reset=True)
    runs = []
    for _ in range(3):
        runs.append(bd.run(H, guess.clone(), tolerance=1e-7, max_iterations=40))
        runs[-1] = runs[-1] + (graph_stats(reset=True),)
    # graphs of earlier calls on this engine stay valid, so only the third call's counts are fixed
    assert runs[2][4]["replayed"] > 0 and runs[2][4]["captured"] == 0 and runs[2][4]["launched"] == 0
    for e, x, n, it, _ in runs:
        assert it == it0
        np.testing.assert_array_equal(e, e0)
        np.testing.assert_array_equal(n, n0)
        assert torch.equal(x, x0)


def test_library_davidson_refuses_bad_arguments(mini_system):
    """More bands than plane waves (or no potential yet) is a ValueError, as in Python."""
    from amaterasu_b200._lib import call
    from amaterasu_b200.engine import engine_for, ptr, stream_ptr
    import ctypes as ct
    eng = engine_for(mini_system)
    x = torch.zeros(10, dtype=torch.complex128, device="cuda")
    eps = torch.zeros(10, dtype=torch.float64, device="cuda")
    it = ct.c_int32(0)
    with pytest.raises(ValueError):
        call("ama_davidson", eng.handle, 1, 0, 10 ** 6, ptr(x), 1e-8, 10, 0, ptr(eps), ptr(x), None,
             ct.byref(it), stream_ptr())


@pytest.mark.parametrize("n,nvec", [(120, 24), (300, 60), (97, 97)])
def test_heev_lowest_matches_eigh(n, nvec):
    """ama_heev_lowest (the library's eigensolver, lowest nvec pairs) against numpy's eigh:
    the nvec lowest eigenvalues, orthonormal eigenvectors and their residuals, on a batch
    of two."""
    from amaterasu_b200._lib import call
    from amaterasu_b200.engine import ptr, stream_ptr
    rng = np.random.default_rng(n + nvec)
    batch = 2
    a = rng.normal(size=(batch, n, n)) + 1j * rng.normal(size=(batch, n, n))
    a = a + np.conj(np.transpose(a, (0, 2, 1)))
    m = torch.from_numpy(a.copy()).cuda()
    w = torch.empty((batch, n), dtype=torch.float64, device="cuda")
    call("ama_heev_lowest", n, nvec, ptr(m), ptr(w), batch, stream_ptr())
    w = w.cpu().numpy()[:, :nvec]
    v = m.cpu().numpy()[:, :, :nvec]
    for b in range(batch):
        ref = np.linalg.eigvalsh(a[b])[:nvec]
        scale = max(1.0, np.abs(ref).max())
        np.testing.assert_allclose(w[b], ref, rtol=0, atol=1e-11 * scale)
        np.testing.assert_allclose(v[b].conj().T @ v[b], np.eye(nvec), atol=1e-10)
        np.testing.assert_allclose(a[b] @ v[b], v[b] * w[b][None, :], atol=1e-9 * scale)
