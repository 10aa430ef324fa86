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
