"""The two large benchmark configurations pinned to the reference's own numbers
(tests/golden/si215.npz and si8_scf1.npz, written by tests/golden/make_golden.py running the
reference), plus the Ewald sum on every golden cell.

Si215 (3x3x3 conventional cell, one vacancy, displaced, Gamma, 30 Ry, 108^3 grid, 80,797
plane waves, 860 projectors): sphere order by SHA-256 of the Miller indices, projector norms
and rows (1e-12), Ewald energy/forces/stress (1e-10 relative / 1e-10 Ha/Bohr / 1e-12
Ha/Bohr^3), the starting density and v_eff at 400 seeded grid points (1e-10), the seeded
starting orbitals (1e-10), and H.psi of three bands: complex128 to 1e-11 and complex64 to 2e-5
of max |H psi|, as for the other H.psi goldens.

Si8 with 260 k-points (40 Ry, 20 bands, Fermi-Dirac 0.01 Ha): the first SCF iteration from the
reference's own start. The per-k FP64 Davidson is the reference's algorithm and is compared
at 1e-8 Ha (every eigenvalue), 1e-9 Ha/atom (free energy), 1e-8 Ha (each energy term) and
the density at 400 grid points. The batched Davidson (all k in lockstep, the production
path) has not converged every band of every k-point after the first iteration's 40 steps from
the random start (measured: the top empty bands 16-19 of some k-points off by up to 2e-3 Ha,
62 of 5200 eigenvalues; three of the 4160 occupied ones by up to 2.1e-6 Ha; later SCF
iterations converge them), so it is compared on the occupied bands at 1e-5 Ha (FP64 and the
mixed policy's complex64 iteration alike), the empty ones at 5e-3 Ha, the energy terms at
1e-4 Ha (measured: kinetic 3.2e-5, the terms compensating in the variational free energy)
and the free energy at 1e-6 Ha/atom (FP64 and mixed; measured 5.6e-7 in FP64, which 80
Davidson steps bring to 1e-7).
"""
import hashlib

import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


# ------------------------------------------------------------------------------------ Ewald
def test_ewald_matches_reference_on_every_golden_cell(mini_system, si_pseudo):
    from amaterasu_b200.cells import workload
    from amaterasu_b200.ewald import ewald
    from amaterasu_b200.system import build_system
    np.testing.assert_allclose(mini_system.ewald, float(golden("mini.npz")["ewald"]), rtol=1e-13)
    g = golden("si2_scf.npz")
    structure, ecut, ks, nb = workload("si2_scf")
    s = build_system(structure, {"Si": si_pseudo}, ecut, 4 * ecut, kpoints=ks, nbands=nb,
                     build_projector_matrices=False)
    res = ewald(s.cell, s.positions, np.full(s.natoms, 4.0))
    np.testing.assert_allclose(res.energy, float(g["ewald"]), rtol=1e-13)
    np.testing.assert_allclose(res.forces, g["force_ewald"], rtol=0, atol=1e-11)
    np.testing.assert_allclose(res.stress, g["stress_ewald"], rtol=0, atol=1e-12)
    g = golden("si215.npz")
    res = ewald(g["cell"], g["positions"], np.full(len(g["positions"]), 4.0))
    np.testing.assert_allclose(res.energy, float(g["ewald_energy"]), rtol=1e-12)
    np.testing.assert_allclose(res.forces, g["ewald_forces"], rtol=0, atol=1e-10)
    np.testing.assert_allclose(res.stress, g["ewald_stress"], rtol=0, atol=1e-12)
    # the splitting parameter only moves work between the two sums
    other = ewald(g["cell"], g["positions"], np.full(len(g["positions"]), 4.0), eta=0.09)
    np.testing.assert_allclose(other.energy, res.energy, rtol=1e-12)
    np.testing.assert_allclose(other.forces, res.forces, rtol=0, atol=1e-9)


# ----------------------------------------------------------------------------------- Si215
@pytest.fixture(scope="module")
def si215_system(si_pseudo):
    from amaterasu_b200.cells import workload
    from amaterasu_b200.system import build_system
    structure, ecut, ks, nb = workload("si215_gamma")
    return build_system(structure, {"Si": si_pseudo}, ecut, 4 * ecut, kpoints=ks, nbands=nb)


def test_si215_setup_and_potential_match_reference(si215_system):
    from amaterasu_b200.potential import effective_potential
    g = golden("si215.npz")
    s = si215_system
    assert tuple(s.grid.shape) == tuple(g["grid"]) == (108, 108, 108)
    sphere = s.wave_spheres[0]
    assert len(sphere) == int(g["npw"][0]) == 80797
    assert hashlib.sha256(np.ascontiguousarray(sphere.miller.astype(np.int64)).tobytes()).hexdigest() == \
        str(g["miller_sha"][0])
    B = s.projectors[0].matrix
    assert B.shape[0] == int(g["nproj"]) == 860
    np.testing.assert_allclose(np.linalg.norm(B, axis=1), g["proj_norms"], rtol=0, atol=1e-12)
    np.testing.assert_allclose(B[0, :64], g["proj_row0"], rtol=0, atol=1e-12)
    np.testing.assert_allclose(B[-1, :64], g["proj_row859"], rtol=0, atol=1e-12)
    np.testing.assert_allclose(s.ewald, float(g["ewald"]), rtol=1e-12)
    probe = g["probe"]
    rho0 = s.initial_density()
    np.testing.assert_allclose(rho0.ravel()[probe], g["rho0_probe"], rtol=0, atol=1e-12)
    np.testing.assert_allclose(rho0.sum(), float(g["rho0_sum"]), rtol=1e-12)
    np.testing.assert_allclose(s.v_local.ravel()[probe], g["vloc_probe"], rtol=0, atol=1e-10)
    veff, e_h, e_xc = effective_potential(s, rho0)
    veff = veff.cpu().numpy()
    np.testing.assert_allclose(e_h, float(g["e_hartree0"]), rtol=1e-11)
    np.testing.assert_allclose(e_xc, float(g["e_xc0"]), rtol=1e-11)
    np.testing.assert_allclose(veff.ravel()[probe], g["veff_probe"], rtol=0, atol=1e-10)
    np.testing.assert_allclose(veff.sum(), float(g["veff_sum"]), rtol=1e-11)
    np.testing.assert_allclose((veff ** 2).sum(), float(g["veff_sq"]), rtol=1e-11)


def test_si215_starting_orbitals_match_reference(si215_system):
    """The seeded random_bands start (12345), drawn with the reference's generator and
    orthonormalised by the engine's own inverse Cholesky factor."""
    from amaterasu_b200.scf import starting_orbitals
    g = golden("si215.npz")
    x = starting_orbitals(si215_system, 0, 0).cpu().numpy()
    np.testing.assert_allclose(x[0, :256], g["start_row0"], rtol=0, atol=1e-10)
    np.testing.assert_allclose(x[-1, :256], g["start_row_last"], rtol=0, atol=1e-10)
    np.testing.assert_allclose(np.linalg.norm(x[:, :512], axis=0), g["start_col_norms"], rtol=0, atol=1e-10)


@pytest.mark.parametrize("precision,tol", [("complex128", 1e-11), ("complex64", 2e-5)])
def test_si215_hpsi_matches_reference(si215_system, precision, tol):
    from amaterasu_b200.hamiltonian import Hamiltonian
    from amaterasu_b200.potential import effective_potential
    g = golden("si215.npz")
    s = si215_system
    veff, _, _ = effective_potential(s, s.initial_density())
    H = Hamiltonian(s, veff.cpu().numpy(), precision=precision)
    sphere = s.wave_spheres[0]
    rng = np.random.default_rng(2150)
    psi = (rng.normal(size=(3, len(sphere))) + 1j * rng.normal(size=(3, len(sphere)))) / (1.0 + sphere.kinetic_energy)
    assert _rel(H.apply(psi, 0), g["hpsi"]) < tol
    # every stage B (x stage A/C for complex64) variant compiled for the 108^3 grid
    variants = []
    for v in (0, 1, 2, 3, 4):
        try:
            H.engine.set_stage_b_variant(precision, v)
        except NotImplementedError:
            continue
        variants.append(v)
        for a in ((0, 1) if precision == "complex64" else (None,)):
            if a is not None:
                H.engine.set_stage_ac_variant(a)
            assert _rel(H.apply(psi, 0), g["hpsi"]) < tol, (v, a)
    assert variants == ([0, 3, 4] if precision == "complex64" else [0, 4])
    H.engine.set_stage_b_variant(precision, 0)
    if precision == "complex64":
        H.engine.set_stage_ac_variant(0)


# ------------------------------------------------------------------------- Si8, 260 k-points
@pytest.fixture(scope="module")
def si8_system(si_pseudo):
    from amaterasu_b200.cells import workload
    from amaterasu_b200.system import build_system
    structure, ecut, ks, nb = workload("si8_batched")
    return build_system(structure, {"Si": si_pseudo}, ecut, 4 * ecut, kpoints=ks, nbands=nb)


def _first_iteration(system, precision, batched):
    from amaterasu_b200.config import Config
    from amaterasu_b200.scf import run_scf
    c = Config()
    c.engine.batched = batched
    c.engine.precision = precision
    c.engine.c64_tolerance_cap = 1e-6  # the reference's Davidson tolerance, not the policy's looser start
    c.occupations.scheme = "fermi-dirac"
    c.occupations.smearing = "0.01 Ha"
    c.scf.max_steps = 1
    return run_scf(system, c)


@pytest.mark.parametrize("precision,batched", [("complex128", False), ("complex128", True), ("mixed", True)])
def test_si8_260k_first_scf_iteration_matches_reference(si8_system, precision, batched):
    from amaterasu_b200.units import HARTREE_IN_EV
    g = golden("si8_scf1.npz")
    s = si8_system
    assert len(s.wave_spheres) == 260 and tuple(s.grid.shape) == tuple(g["grid"])
    np.testing.assert_array_equal([len(w) for w in s.wave_spheres], g["npw"])
    res = _first_iteration(s, precision, batched)
    e = res.energies
    natoms = s.natoms
    occupied = int(round(s.nelectrons / 2))
    if batched:  # the empty top bands may still be converging after 40 steps (see above)
        np.testing.assert_allclose(res.eigenvalues[..., occupied:], g["eigenvalues"][..., occupied:], rtol=0,
                                   atol=5e-3)
    if precision == "complex128":
        eig_tol, e_tol, dn_tol, term_tol = (1e-8, 1e-9, 1e-8, 1e-8) if not batched else (1e-5, 1e-6, 1e-4, 1e-4)
        bands = slice(None) if not batched else slice(0, occupied)
        np.testing.assert_allclose(res.eigenvalues[..., bands], g["eigenvalues"][..., bands], rtol=0, atol=eig_tol)
        assert abs(e.free_energy - float(g["e_free"])) / natoms < e_tol
        for name in ("kinetic", "local", "hartree", "xc", "entropy"):
            assert abs(getattr(e, name) - float(g[f"e_{name}"])) < term_tol, name
        assert abs(e.nonlocal_ - float(g["e_nonlocal"])) < term_tol
        np.testing.assert_allclose(res.fermi_level, float(g["fermi"]), rtol=0, atol=eig_tol)
        rho = res.density.ravel()
        np.testing.assert_allclose(rho.sum(), float(g["density_sum"]), rtol=1e-12)
        scale = np.abs(g["density_probe"]).max()
        np.testing.assert_allclose(rho[g["probe"]], g["density_probe"], rtol=0, atol=dn_tol * scale * 100)
    else:
        np.testing.assert_allclose(res.eigenvalues[..., :occupied], g["eigenvalues"][..., :occupied], rtol=0,
                                   atol=1e-5 if batched else 2e-5)
        # the batched first iteration's convergence limit (as for FP64 above), not the precision
        assert abs(e.free_energy - float(g["e_free"])) / natoms < (1e-6 if batched else 1e-5 / HARTREE_IN_EV)
