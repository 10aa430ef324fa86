"""Full SCF on the GPU against the reference's own run (Si2 fcc, 30 Ry, shifted 4x4x4 ->
32 k-points, 8 bands, LDA-PZ, fixed occupations, tol 1e-8 eV/atom and 1e-8 density).

Tolerances against the reference (FP64 numpy): plain FP64 engine -- total energy 1e-9
Ha/atom, eigenvalues 1e-8 Ha, density integral |dn|/N 1e-8; mixed precision (complex64 bulk,
complex128 refinement) -- |dE| < 1e-5 eV/atom, eigenvalues 1e-6 Ha, density 1e-6.

With this synthetic dataset and fixed occupations the fourth and fifth bands are split by
only ~2e-4 Ha at some k-points, so the SCF has two symmetry-equivalent fixed points (images
of each other under a crystal symmetry: equal energies, densities that are a permutation of
the grid, eigenvalue sets exchanged between equivalent k-points, forces and stress rotated).
Which one a run reaches depends on rounding inside the eigensolver. The plain FP64 engine
with the per-k Davidson follows the reference's arithmetic closely enough to reach the
reference's own fixed point and is compared element by element; the other runs are compared
through quantities that are invariant under the symmetry: every energy term, the sorted
eigenvalue multiset (all k-points carry the same weight), the sorted density values, the
force magnitudes per atom and the principal stresses.
"""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def si2_system(si_pseudo):
    from amaterasu_b200.cells import workload
    from amaterasu_b200.system import build_system
    structure, ecut, ks, nb = workload("si2_scf")
    return build_system(structure, {"Si": si_pseudo}, ecut, 4 * ecut, kpoints=ks, nbands=nb)


def _config(precision, batched=True):
    from amaterasu_b200.config import Config
    c = Config()
    c.engine.batched = batched
    c.occupations.scheme = "fixed"
    c.occupations.nbands = 8
    c.scf.tol_energy = 1e-8
    c.scf.tol_density = 1e-8
    c.engine.precision = precision
    return c


@pytest.mark.parametrize("precision,batched", [("complex128", True), ("mixed", True), ("complex128", False)])
def test_si2_scf_matches_reference(si2_system, precision, batched):
    from amaterasu_b200.scf import run_scf
    from amaterasu_b200.units import HARTREE_IN_EV
    g = golden("si2_scf.npz")
    s = si2_system
    res = run_scf(s, _config(precision, batched), logger=print)
    assert res.converged
    e = res.energies
    natoms = s.natoms
    elementwise = precision == "complex128" and not batched
    assert np.allclose(g["weights"], g["weights"][0])  # the sorted multisets below need equal weights
    eig = res.eigenvalues if elementwise else np.sort(res.eigenvalues.ravel())
    eig_ref = g["eigenvalues"] if elementwise else np.sort(g["eigenvalues"].ravel())
    rho = res.density.ravel() if elementwise else np.sort(res.density.ravel())
    rho_ref = g["density"].ravel() if elementwise else np.sort(g["density"].ravel())
    dn = np.sum(np.abs(rho - rho_ref)) * s.grid.cell_volume_per_point / s.nelectrons
    if precision == "complex128":
        assert abs(e.total - float(g["e_total"])) / natoms < 1e-9
        for name in ("kinetic", "local", "hartree", "xc", "ewald"):
            assert abs(getattr(e, name) - float(g[f"e_{name}"])) < 1e-7, name
        assert abs(e.nonlocal_ - float(g["e_nonlocal"])) < 1e-7
        np.testing.assert_allclose(eig, eig_ref, rtol=0, atol=1e-8)
        assert dn < 1e-8
        assert abs(res.history[-1][2]) < 1e-9  # eigenvalue-sum identity (Ha)
    else:
        assert "complex64" in res.precision_trace and res.precision_trace[-1] == "complex128"
        assert abs(e.total - float(g["e_total"])) * HARTREE_IN_EV / natoms < 1e-5
        np.testing.assert_allclose(eig, eig_ref, rtol=0, atol=1e-6)
        assert dn < 1e-6
    assert abs(res.electron_count - s.nelectrons) < 1e-9

    from amaterasu_b200.properties import compute_forces, compute_stress
    from amaterasu_b200.units import HARTREE_PER_BOHR_IN_EV_PER_ANG
    forces = compute_forces(s, res.density, res.wavefunctions, res.occupations, decompose=True)
    stress = compute_stress(s, res.density, res.wavefunctions, res.occupations, decompose=True)
    f_tot = sum(forces.values())
    s_tot = sum(stress.values())
    if elementwise:
        for name, value in forces.items():
            np.testing.assert_allclose(value, g[f"force_{name}"], rtol=0, atol=1e-7, err_msg=name)
        for name, value in stress.items():
            np.testing.assert_allclose(value, g[f"stress_{name}"], rtol=0, atol=1e-8, err_msg=name)
    elif precision == "complex128":
        np.testing.assert_allclose(np.linalg.norm(f_tot, axis=1), np.linalg.norm(g["forces"], axis=1),
                                   rtol=0, atol=1e-7)
        np.testing.assert_allclose(np.linalg.eigvalsh(s_tot), np.linalg.eigvalsh(g["stress"]), rtol=0, atol=1e-8)
    else:
        df = np.abs(np.linalg.norm(f_tot, axis=1) - np.linalg.norm(g["forces"], axis=1))
        assert np.max(df) * HARTREE_PER_BOHR_IN_EV_PER_ANG < 1e-4
        assert np.max(np.abs(np.linalg.eigvalsh(s_tot) - np.linalg.eigvalsh(g["stress"]))) < 1e-6
