"""The GGA oracle (oracle/xc_gga.py: PBE and PBEsol from the published forms, derivatives
by complex step) pinned to the reference's own outputs (tests/golden/gga.npz, written by
tests/golden/make_golden.py running amaterasu xc/gga.py and xc/driver.py).

Tolerances: eps 1e-13 relative, vrho 1e-12 relative, vsigma 1e-9 relative (the reference's
closed-form chain rule loses a few digits at large reduced gradients); on the grid the
energy to 1e-12 relative and the potential to 1e-10 Ha."""
import numpy as np
import pytest

from conftest import golden
from oracle.xc_gga import gga_on_grid, gga_point


def _rel(a, b):
    scale = np.maximum(np.abs(b), 1e-12 * np.max(np.abs(b)))
    return float(np.max(np.abs(a - b) / scale))


@pytest.mark.parametrize("functional", ["PBE", "PBEsol"])
def test_pointwise_oracle_matches_reference(functional):
    g = golden("gga.npz")
    eps, vrho, vsigma = gga_point(g["rho"], g["sigma"], functional)
    assert _rel(eps, g[f"{functional}_eps"]) < 1e-13
    assert _rel(vrho, g[f"{functional}_vrho"]) < 1e-12
    assert _rel(vsigma, g[f"{functional}_vsigma"]) < 1e-9


@pytest.mark.parametrize("functional", ["PBE", "PBEsol"])
def test_grid_oracle_matches_reference(functional):
    g = golden("gga.npz")
    e, v = gga_on_grid(g["mini_rho0"], g["mini_cell"], functional)
    np.testing.assert_allclose(e, float(g[f"mini_{functional}_energy"]), rtol=1e-12)
    np.testing.assert_allclose(v, g[f"mini_{functional}_potential"], rtol=0, atol=1e-10)


def test_spin_polarised_grid_oracle_matches_reference():
    g = golden("gga.npz")
    rho0 = g["mini_rho0"][0]
    e, v = gga_on_grid(np.stack([0.6 * rho0, 0.4 * rho0]), g["mini_cell"], "PBE")
    np.testing.assert_allclose(e, float(g["mini_pol_energy"]), rtol=1e-12)
    np.testing.assert_allclose(v, g["mini_pol_potential"], rtol=0, atol=1e-10)


def test_unknown_functional_is_refused():
    with pytest.raises(ValueError):
        gga_point(np.ones((1, 2)), np.zeros((1, 3)), "BLYP")
