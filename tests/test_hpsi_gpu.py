"""H.psi on the GPU (C-ABI engine) against the CPU oracle and the reference's goldens.

Tolerances: complex128 agrees with the FP64 numpy path to 1e-11 relative to the largest
|H psi| coefficient; complex64 to 2e-5 of it (FP32 FFTs and FP32 projector GEMMs).
"""
import numpy as np
import pytest
import torch

from conftest import golden
from oracle.hamiltonian import hamiltonian_apply

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


@pytest.mark.parametrize("precision,tol", [("complex128", 1e-11), ("complex64", 2e-5)])
def test_hpsi_mini_matches_reference(mini_system, precision, tol):
    from amaterasu_b200.hamiltonian import Hamiltonian
    g = golden("mini.npz")
    H = Hamiltonian(mini_system, g["veff"], precision=precision)
    for ik in range(2):
        out = H.apply(g[f"psi{ik}"], ik)
        assert out.dtype == np.complex128
        assert _rel(out, g[f"hpsi{ik}"]) < tol


def test_hpsi_single_band_and_shape_errors(mini_system):
    from amaterasu_b200.hamiltonian import Hamiltonian
    g = golden("mini.npz")
    H = Hamiltonian(mini_system, g["veff"][0])
    one = H.apply(g["psi0"][3], 0)
    assert one.shape == g["psi0"][3].shape
    assert _rel(one, g["hpsi0"][3]) < 1e-11
    with pytest.raises(ValueError):
        H.apply(g["psi0"][:, :-1], 0)
    with pytest.raises(ValueError):
        Hamiltonian(mini_system, np.zeros((3, 3, 3)))


def test_hpsi_batched_all_k_matches_oracle(mini_system):
    from amaterasu_b200.hamiltonian import Hamiltonian
    s = mini_system
    rng = np.random.default_rng(3)
    veff = rng.normal(size=(1, *s.grid.shape))
    H = Hamiltonian(s, veff)
    nb = 5
    blocks = [(rng.normal(size=(nb, len(w))) + 1j * rng.normal(size=(nb, len(w)))) for w in s.wave_spheres]
    packed = torch.from_numpy(np.concatenate([b.ravel() for b in blocks])).cuda()
    out = H.apply_all(packed, nb).cpu().numpy()
    off = 0
    for ik, (w, b) in enumerate(zip(s.wave_spheres, blocks)):
        ref = hamiltonian_apply(b, w.miller, s.grid.shape, w.kinetic_energy, veff[0],
                                s.projectors[ik].matrix, s.projectors[ik].dij)
        got = out[off:off + b.size].reshape(b.shape)
        off += b.size
        assert _rel(got, ref) < 1e-11


@pytest.mark.parametrize("precision,tol", [("complex128", 1e-11), ("complex64", 2e-5)])
@pytest.mark.parametrize("chunks", [1, 2, 4])
def test_hpsi_host_to_host_matches_oracle(mini_system, precision, tol, chunks):
    """Hamiltonian.apply_host: pinned host blocks in and out, copies pipelined over band
    chunks, same H.psi as the oracle (odd band count: the last chunk is short)."""
    from amaterasu_b200.hamiltonian import Hamiltonian
    s = mini_system
    rng = np.random.default_rng(11)
    veff = rng.normal(size=(1, *s.grid.shape))
    H = Hamiltonian(s, veff, precision=precision)
    nb = 5
    blocks = [(rng.normal(size=(nb, len(w))) + 1j * rng.normal(size=(nb, len(w)))) for w in s.wave_spheres]
    cdt = torch.complex64 if precision == "complex64" else torch.complex128
    host_in = torch.from_numpy(np.concatenate([b.ravel() for b in blocks])).to(cdt).pin_memory()
    host_out = torch.empty_like(host_in).pin_memory()
    H.apply_host(host_in, host_out, nb, chunks_per_k=chunks)
    torch.cuda.synchronize()
    out = host_out.to(torch.complex128).numpy()
    off = 0
    for ik, (w, b) in enumerate(zip(s.wave_spheres, blocks)):
        bq = host_in[off:off + b.size].to(torch.complex128).numpy().reshape(b.shape)
        ref = hamiltonian_apply(bq, w.miller, s.grid.shape, w.kinetic_energy, veff[0],
                                s.projectors[ik].matrix, s.projectors[ik].dij)
        got = out[off:off + b.size].reshape(b.shape)
        off += b.size
        assert _rel(got, ref) < tol


@pytest.fixture(scope="module")
def si64_system(si_pseudo):
    from amaterasu_b200.cells import workload
    from amaterasu_b200.system import build_system
    structure, ecut, ks, nb = workload("si64_hpsi")
    return build_system(structure, {"Si": si_pseudo}, ecut, 4 * ecut, kpoints=ks, nbands=nb)


@pytest.mark.parametrize("precision,tol", [("complex128", 1e-11), ("complex64", 2e-5)])
def test_hpsi_si64_matches_reference(si64_system, precision, tol):
    """Si64, 40 Ry, 84^3 grid: the reference's own H.psi bands (tests/golden/si64.npz)."""
    from amaterasu_b200.hamiltonian import Hamiltonian
    from amaterasu_b200.potential import effective_potential
    g = golden("si64.npz")
    s = si64_system
    assert tuple(s.grid.shape) == tuple(g["grid"])
    veff, e_h, e_xc = effective_potential(s, s.initial_density())
    veff = veff.cpu().numpy()
    np.testing.assert_allclose(veff.ravel()[g["probe"]], g["veff_probe"], rtol=0, atol=1e-10)
    H = Hamiltonian(s, veff, precision=precision)
    for ik, nb in ((0, 2), (1, 1)):
        w = s.wave_spheres[ik]
        rng = np.random.default_rng(300 + ik)
        psi = (rng.normal(size=(nb, len(w))) + 1j * rng.normal(size=(nb, len(w)))) / (1.0 + w.kinetic_energy)
        assert _rel(H.apply(psi, ik), g[f"hpsi{ik}"]) < tol
