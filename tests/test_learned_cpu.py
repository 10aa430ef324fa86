"""Host-side pieces of the learned start: Fourier resampling and strain bookkeeping."""
import numpy as np


def test_fourier_resample_is_band_limited_and_conserves_charge():
    from amaterasu_b200.learned import fourier_resample
    rng = np.random.default_rng(0)
    n = 35
    x = np.arange(n) / n
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    f = 1.0 + 0.3 * np.cos(2 * np.pi * (2 * X + Y)) + 0.1 * np.sin(2 * np.pi * (3 * Z - X))
    g = fourier_resample(f, (36, 36, 36))
    back = fourier_resample(g, (n, n, n))
    np.testing.assert_allclose(back, f, atol=1e-12)
    np.testing.assert_allclose(g.mean(), f.mean(), rtol=1e-14)
    h = fourier_resample(f, (40, 36, 35))
    assert h.shape == (40, 36, 35)
    np.testing.assert_allclose(h.mean(), f.mean(), rtol=1e-14)


def test_strain_of_recovers_symmetric_strain():
    from amaterasu_b200.learned import strain_of
    from amaterasu_b200.learned_pipeline import make_cell
    s, ref = make_cell(7)
    e = strain_of(s.cell, ref)
    full = np.array([[e[0], e[5], e[4]], [e[5], e[1], e[3]], [e[4], e[3], e[2]]])
    np.testing.assert_allclose(ref @ (np.eye(3) + full), s.cell, atol=1e-12)
    assert np.all(np.abs(e) <= 0.03 + 1e-12)
