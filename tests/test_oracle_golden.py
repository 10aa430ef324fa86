"""Pin the CPU oracle (oracle/) against the reference's own outputs."""
import numpy as np

from conftest import golden
from oracle.hamiltonian import hamiltonian_apply


def test_oracle_hpsi_matches_reference_mini(mini_system):
    g = golden("mini.npz")
    s = mini_system
    for ik, sphere in enumerate(s.wave_spheres):
        psi = g[f"psi{ik}"]
        out = hamiltonian_apply(psi, sphere.miller, s.grid.shape, sphere.kinetic_energy,
                                g["veff"][0], s.projectors[ik].matrix, s.projectors[ik].dij)
        np.testing.assert_allclose(out, g[f"hpsi{ik}"], rtol=0, atol=1e-12)


def test_oracle_hartree_and_lda_match_reference(mini_system):
    from oracle.potential import hartree, xc_on_grid
    g = golden("mini.npz")
    s = mini_system
    sph = s.density_sphere
    e_h, v_h = hartree(g["density"][0], s.grid.shape, sph.miller, sph.g2, s.grid.volume)
    np.testing.assert_allclose(e_h, float(g["hartree_e"]), rtol=1e-13)
    np.testing.assert_allclose(v_h, g["hartree_v"], rtol=0, atol=1e-13)
    e_xc, v_xc = xc_on_grid(g["density"], s.grid.cell_volume_per_point)
    np.testing.assert_allclose(e_xc, float(g["xc_e"]), rtol=1e-13)
    np.testing.assert_allclose(v_xc, g["xc_v"], rtol=0, atol=1e-13)
    # effective potential of the starting density (scf/driver.py:330-357)
    e_h0, v_h0 = hartree(g["rho0"][0], s.grid.shape, sph.miller, sph.g2, s.grid.volume)
    e_xc0, v_xc0 = xc_on_grid(g["rho0"], s.grid.cell_volume_per_point)
    np.testing.assert_allclose(s.v_local + v_h0 + v_xc0[0], g["veff"][0], rtol=0, atol=1e-12)
    np.testing.assert_allclose([e_h0, e_xc0], [float(g["e_hartree0"]), float(g["e_xc0"])], rtol=1e-13)


def _mini_h(s, g, ik):
    sphere = s.wave_spheres[ik]
    return lambda b: hamiltonian_apply(b, sphere.miller, s.grid.shape, sphere.kinetic_energy,
                                       g["veff"][0], s.projectors[ik].matrix, s.projectors[ik].dij)


def test_oracle_davidson_pieces_match_reference(mini_system):
    from oracle.eigen import davidson, orthonormalize, random_bands, rayleigh_ritz, teter_payne_allan
    g = golden("mini.npz")
    s = mini_system
    for ik, sphere in enumerate(s.wave_spheres):
        guess = random_bands(len(sphere), s.nbands, sphere.kinetic_energy, seed=12345 + ik)
        np.testing.assert_allclose(guess, g[f"guess{ik}"], rtol=0, atol=1e-14)
        basis = orthonormalize(g[f"psi{ik}"][:4])
        np.testing.assert_allclose(basis, g[f"ortho{ik}"], rtol=0, atol=1e-12)
        e, _, _ = rayleigh_ritz(basis, _mini_h(s, g, ik)(basis), 3)
        np.testing.assert_allclose(e, g[f"rr_eig{ik}"], rtol=0, atol=1e-12)
        out = teter_payne_allan(g[f"tpa_in{ik}"], sphere.kinetic_energy, g[f"tpa_ref{ik}"])
        np.testing.assert_allclose(out, g[f"tpa_out{ik}"], rtol=0, atol=1e-14)
        res = davidson(_mini_h(s, g, ik), g[f"guess{ik}"], sphere.kinetic_energy, tolerance=1e-9,
                       max_iterations=60)
        np.testing.assert_allclose(res.eigenvalues, g[f"dav_eig{ik}"], rtol=0, atol=1e-9)


def test_oracle_density_occupations_match_reference(mini_system):
    from oracle.scf import compute_density, compute_occupations
    g = golden("mini.npz")
    s = mini_system
    eig = np.array([[g["dav_eig0"], g["dav_eig1"]]])
    occ, fermi, ent, gap = compute_occupations(eig, s.kpoints.weights, s.nelectrons, "gaussian",
                                               0.1 / 27.211386, nspin=1)
    np.testing.assert_allclose(occ, g["occ"], rtol=0, atol=1e-12)
    np.testing.assert_allclose(fermi, float(g["fermi"]), rtol=0, atol=1e-11)
    wfs = [[g["dav_vec0"], g["dav_vec1"]]]
    millers = [w.miller for w in s.wave_spheres]
    d = compute_density(s.grid.shape, s.grid.volume, millers, s.kpoints.weights, wfs, g["occ"])
    np.testing.assert_allclose(d, g["density"], rtol=0, atol=1e-13)
    d2 = compute_density(s.grid.shape, s.grid.volume, millers, s.kpoints.weights, wfs, g["occ"], clip=False)
    np.testing.assert_allclose(d2, g["density_nosym"], rtol=0, atol=1e-13)


def test_oracle_mixers_match_reference(mini_system):
    from oracle.scf import Kerker, Mixer
    g = golden("mini.npz")
    s = mini_system
    for algo in ("linear", "pulay", "broyden", "anderson"):
        mixer = Mixer(algo, 0.4, 8, Kerker(s.grid.gvectors_cartesian(), 1.5))
        target = g[f"mix_{algo}_target"]
        x = g["rho0"].copy()
        for step, ref in enumerate(g[f"mix_{algo}_seq"]):
            out = 0.5 * x + 0.5 * target + 0.002 * np.sin(step + x)
            x = mixer(x, out)
            np.testing.assert_allclose(x, ref, rtol=0, atol=1e-12, err_msg=f"{algo} step {step}")
