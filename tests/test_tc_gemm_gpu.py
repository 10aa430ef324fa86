"""The tcgen05 split-TF32 nonlocal products (complex64 H.psi) against the SIMT GEMM path
and the FP64 oracle. Tolerance: 2e-5 of the largest |H psi| coefficient, as for the
rest of the complex64 engine."""
import numpy as np
import pytest
import torch

from oracle.hamiltonian import hamiltonian_apply

pytestmark = pytest.mark.gpu


def _run(system, veff, blocks, nb, tensor_cores):
    from amaterasu_b200.engine import engine_for
    from amaterasu_b200.hamiltonian import Hamiltonian
    H = Hamiltonian(system, veff, precision="complex64")
    eng = engine_for(system)
    eng.set_tensor_core_nonlocal(tensor_cores)
    packed = torch.from_numpy(np.concatenate([b.ravel() for b in blocks])).cuda().to(torch.complex64)
    out = H.apply_all(packed, nb).cpu().numpy().astype(np.complex128)
    torch.cuda.synchronize()
    eng.set_tensor_core_nonlocal(True)
    assert eng.tc_status() == 0
    return out


def _check(system, nb, seed):
    rng = np.random.default_rng(seed)
    veff = rng.normal(size=(1, *system.grid.shape)) * 0.3
    blocks = [(rng.normal(size=(nb, len(w))) + 1j * rng.normal(size=(nb, len(w)))) / (1 + w.kinetic_energy)
              for w in system.wave_spheres]
    tc = _run(system, veff, blocks, nb, True)
    simt = _run(system, veff, blocks, nb, False)
    off = 0
    for ik, (w, b) in enumerate(zip(system.wave_spheres, blocks)):
        ref = hamiltonian_apply(b, w.miller, system.grid.shape, w.kinetic_energy, veff[0],
                                system.projectors[ik].matrix, system.projectors[ik].dij)
        scale = np.max(np.abs(ref))
        got_tc = tc[off:off + b.size].reshape(b.shape)
        got_simt = simt[off:off + b.size].reshape(b.shape)
        off += b.size
        assert np.max(np.abs(got_simt - ref)) / scale < 2e-5
        assert np.max(np.abs(got_tc - ref)) / scale < 2e-5
        assert np.max(np.abs(got_tc - got_simt)) / scale < 2e-5


@pytest.mark.parametrize("nb", [5, 16, 37])
def test_tc_nonlocal_mini(mini_system, nb):
    _check(mini_system, nb, 10 + nb)


def test_tc_nonlocal_si64(si_pseudo):
    from amaterasu_b200.cells import workload
    from amaterasu_b200.system import build_system
    structure, ecut, ks, _ = workload("si64_hpsi")
    system = build_system(structure, {"Si": si_pseudo}, ecut, 4 * ecut, kpoints=ks, nbands=160)
    _check(system, 160, 7)
