"""Restarting the SCF from a saved result (amaterasu scf/driver.py:267-274, io/results.py):
a converged Si2 run is written with its orbitals, read back, and run_scf(density=...,
wavefunctions=...) from it converges again within three iterations to the same free energy
(1e-9 Ha/atom) and eigenvalues (1e-8 Ha)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_restart_from_saved_result_converges_at_once(tmp_path, si_pseudo):
    from amaterasu_b200.cells import workload
    from amaterasu_b200.config import Config
    from amaterasu_b200.properties import compute_forces, compute_stress
    from amaterasu_b200.results import read_scf, write_scf
    from amaterasu_b200.scf import run_scf
    from amaterasu_b200.system import build_system
    from amaterasu_b200.units import HARTREE_IN_EV
    structure, ecut, ks, nb = workload("si2_scf")
    s = build_system(structure, {"Si": si_pseudo}, ecut, 4 * ecut, kpoints=ks, nbands=nb)
    c = Config()
    c.occupations.scheme = "fixed"
    c.scf.tol_energy = 1e-8
    c.scf.tol_density = 1e-8
    c.engine.batched = False
    first = run_scf(s, c)
    assert first.converged
    forces = compute_forces(s, first.density, first.wavefunctions, first.occupations)
    stress = compute_stress(s, first.density, first.wavefunctions, first.occupations)
    path = write_scf(tmp_path / "si2.npz", s, first, forces=forces, stress=stress, save_wavefunctions=True)
    saved = read_scf(path)
    np.testing.assert_allclose(saved["scf"]["energies"]["@free_energy"], first.energies.free_energy * HARTREE_IN_EV)
    again = run_scf(s, c, density=saved["density_internal"], wavefunctions=saved["wavefunctions"])
    assert again.converged and again.iterations <= 3
    assert abs(again.energies.free_energy - first.energies.free_energy) / s.natoms < 1e-9
    np.testing.assert_allclose(again.eigenvalues, first.eigenvalues, rtol=0, atol=1e-8)
