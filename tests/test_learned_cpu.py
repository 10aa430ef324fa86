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


def test_working_grid_keeps_the_training_spacing():
    from amaterasu_b200.learned import working_grid
    spacing = 10.86 / 40
    assert working_grid(np.eye(3) * 10.86, spacing) == 40
    assert working_grid(np.eye(3) * 16.29, spacing) == 60
    assert working_grid(np.eye(3) * 5.43, 5.43 / 36) == 36
    assert working_grid(np.eye(3) * 16.29, spacing) % 4 == 0


def test_si64_family_cells():
    from amaterasu_b200.learned import strain_of
    from amaterasu_b200.learned_pipeline import make_cell
    a, ref = make_cell(1000, "si64")
    b, _ = make_cell(1001, "si64")
    assert {len(a.symbols), len(b.symbols)} == {63, 64}  # a vacancy in every second cell
    e = strain_of(a.cell, ref)
    assert np.all(np.abs(e) <= 0.01 + 1e-12)
    again, _ = make_cell(1000, "si64")
    np.testing.assert_array_equal(again.positions, a.positions)


def test_dataset_shards_cover_every_seed_once_and_keep_seed_order(tmp_path, monkeypatch):
    """generate() splits seeds into interleaved shards (one per worker process) and writes the
    samples in seed order; here one worker and a stand-in for the cell convergence."""
    from amaterasu_b200 import learned_pipeline as lp
    seeds = list(range(1000, 1011))
    shards = lp._shards(seeds, 4)
    assert sorted(s for part in shards for s in part) == seeds
    assert [len(p) for p in shards] == [3, 3, 3, 2]
    assert lp._shards(seeds[:2], 4) == [[1000], [1001]]  # no empty shard (no idle process)

    def fake_cell(seed, pseudo, **kw):
        grid = np.full((2, 2, 2), float(seed), dtype=np.float32)
        return dict(seed=seed, grid=[2, 2, 2], iterations=seed % 7, converged=True, free_energy=-1.0,
                    seconds=0.5, n0=grid, nconv=grid + 1, strain=np.full(6, seed * 1e-6))

    monkeypatch.setattr(lp, "run_cell", fake_cell)
    monkeypatch.setattr(lp, "_pseudo", lambda: None)
    order = [1004, 1001, 1003]
    lp.generate(order, tmp_path / "d.npz")
    data = np.load(tmp_path / "d.npz")
    np.testing.assert_array_equal(data["seeds"], order)
    np.testing.assert_array_equal(data["n0"][:, 0, 0, 0], order)
    np.testing.assert_array_equal(data["iterations"], [s % 7 for s in order])
