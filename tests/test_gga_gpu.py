"""GGA on the GPU (csrc/xc_gga.cu, the spectral gradient and divergence of csrc/engine.cu)
against the oracle and the reference's goldens (tests/golden/gga.npz).

Tolerances: gradient and divergence 1e-12 of the field's scale; E_xc 1e-12 relative and
v_xc 1e-10 Ha against the reference on the mini grid (PBE, PBEsol, spin-split); the Si2 PBE
SCF with the per-k FP64 Davidson as in test_scf_gpu.py (total energy 1e-9 Ha/atom, terms
1e-7 Ha, eigenvalues 1e-8 Ha, forces 1e-7 Ha/Bohr and stress 1e-8 Ha/Bohr^3 per term)."""
import numpy as np
import pytest
import torch

from conftest import golden
from oracle.xc_gga import divergence, gradient

pytestmark = pytest.mark.gpu


def test_gradient_and_divergence_match_the_oracle(mini_system):
    from amaterasu_b200._lib import call
    from amaterasu_b200.engine import ptr, stream_ptr
    from amaterasu_b200.potential import grid_ops
    import ctypes as ct
    s = mini_system
    ops = grid_ops(s)
    rng = np.random.default_rng(3)
    f = s.initial_density()[0] + 0.01 * rng.normal(size=s.grid.shape)
    cell = np.ascontiguousarray(s.grid.cell, dtype=np.float64)
    cptr = cell.ctypes.data_as(ct.c_void_p)
    fin = torch.from_numpy(f.ravel()).cuda()
    out = torch.empty((3, fin.numel()), dtype=torch.float64, device="cuda")
    call("ama_grid_gradient", ops.engine.handle, cptr, ptr(fin), 2.0, ptr(out), stream_ptr())
    ref = gradient(f, cell)
    got = out.cpu().numpy().reshape(3, *s.grid.shape)
    scale = np.abs(ref).max()
    for a in range(3):
        assert np.abs(got[a] - 2.0 * ref[..., a]).max() < 1e-12 * 2.0 * scale
    vec = rng.normal(size=(*s.grid.shape, 3))
    vin = torch.from_numpy(np.ascontiguousarray(np.moveaxis(vec, -1, 0)).reshape(3, -1)).cuda()
    acc = torch.from_numpy(f.ravel()).cuda()
    call("ama_grid_divergence", ops.engine.handle, cptr, ptr(vin), -0.5, 1.0, ptr(acc), stream_ptr())
    ref = f - 0.5 * divergence(vec, cell)
    assert np.abs(acc.cpu().numpy().reshape(s.grid.shape) - ref).max() < 1e-12 * np.abs(ref).max()


@pytest.mark.parametrize("functional", ["PBE", "PBEsol"])
def test_gga_on_grid_matches_reference(mini_system, functional):
    from amaterasu_b200.potential import grid_ops
    g = golden("gga.npz")
    ops = grid_ops(mini_system)
    e, v, outer = ops.gga(torch.from_numpy(g["mini_rho0"].reshape(1, -1)), functional)
    np.testing.assert_allclose(float(e), float(g[f"mini_{functional}_energy"]), rtol=1e-12)
    ref = g[f"mini_{functional}_potential"].reshape(1, -1)
    assert np.abs(v.cpu().numpy() - ref).max() < 1e-10
    assert outer.shape == (3, 3) and np.allclose(outer.cpu().numpy(), outer.cpu().numpy().T)


def test_spin_polarised_gga_matches_reference(mini_system):
    from amaterasu_b200.potential import grid_ops
    g = golden("gga.npz")
    ops = grid_ops(mini_system)
    rho0 = g["mini_rho0"][0].ravel()
    e, v, _ = ops.gga(torch.from_numpy(np.stack([0.6 * rho0, 0.4 * rho0])), "PBE")
    np.testing.assert_allclose(float(e), float(g["mini_pol_energy"]), rtol=1e-12)
    assert np.abs(v.cpu().numpy() - g["mini_pol_potential"].reshape(2, -1)).max() < 1e-10


def test_si2_pbe_scf_matches_reference(si_pseudo):
    from amaterasu_b200 import kpoints as kp
    from amaterasu_b200.cells import si2_primitive
    from amaterasu_b200.config import Config
    from amaterasu_b200.properties import compute_forces, compute_stress
    from amaterasu_b200.scf import run_scf
    from amaterasu_b200.system import build_system
    g = golden("gga.npz")
    ks = kp.monkhorst_pack((2, 2, 2), (0.5, 0.5, 0.5))
    s = build_system(si2_primitive(), {"Si": si_pseudo}, 10.0, 40.0, kpoints=ks, nbands=8, xc="PBE")
    assert tuple(s.grid.shape) == tuple(g["scf_grid"])
    np.testing.assert_allclose(s.kpoints.points, g["scf_kpoints"], atol=1e-14)
    c = Config()
    c.engine.batched = False
    c.engine.precision = "complex128"
    c.occupations.scheme = "fixed"
    c.occupations.nbands = 8
    c.scf.tol_energy = 1e-8
    c.scf.tol_density = 1e-8
    res = run_scf(s, c, logger=print)
    assert res.converged
    e = res.energies
    assert abs(e.total - float(g["scf_e_total"])) / s.natoms < 1e-9
    for name in ("kinetic", "local", "hartree", "xc", "ewald"):
        assert abs(getattr(e, name) - float(g[f"scf_e_{name}"])) < 1e-7, name
    assert abs(e.nonlocal_ - float(g["scf_e_nonlocal"])) < 1e-7
    np.testing.assert_allclose(res.eigenvalues, g["scf_eigenvalues"], rtol=0, atol=1e-8)
    forces = compute_forces(s, res.density, res.wavefunctions, res.occupations,
                            eigenvalues=res.eigenvalues, decompose=True)
    for name, value in forces.items():
        if f"scf_force_{name}" in g:
            np.testing.assert_allclose(value, g[f"scf_force_{name}"], rtol=0, atol=1e-7, err_msg=name)
    stress = compute_stress(s, res.density, res.wavefunctions, res.occupations,
                            eigenvalues=res.eigenvalues, decompose=True)
    for name, value in stress.items():
        if f"scf_stress_{name}" in g:
            np.testing.assert_allclose(value, g[f"scf_stress_{name}"], rtol=0, atol=1e-8, err_msg=name)
    assert "xc" in stress
