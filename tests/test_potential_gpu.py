"""FP64 grid kernels (Hartree filter, LDA-PZ, density accumulation) against the oracle."""
import numpy as np
import pytest
import torch

from conftest import golden

pytestmark = pytest.mark.gpu


def test_hartree_lda_veff_match_reference(mini_system):
    from amaterasu_b200.potential import effective_potential, grid_ops
    g = golden("mini.npz")
    s = mini_system
    ops = grid_ops(s)
    e_h, v_h = ops.hartree(torch.from_numpy(g["density"][0]))
    np.testing.assert_allclose(float(e_h), float(g["hartree_e"]), rtol=1e-12)
    np.testing.assert_allclose(v_h.cpu().numpy().reshape(s.grid.shape), g["hartree_v"], rtol=0, atol=1e-12)
    e_xc, v_xc = ops.lda(torch.from_numpy(g["density"].reshape(1, -1)))
    np.testing.assert_allclose(float(e_xc), float(g["xc_e"]), rtol=1e-12)
    np.testing.assert_allclose(v_xc.cpu().numpy().reshape(g["xc_v"].shape), g["xc_v"], rtol=0, atol=1e-12)
    veff, e_h0, e_xc0 = effective_potential(s, g["rho0"])
    np.testing.assert_allclose(veff.cpu().numpy(), g["veff"], rtol=0, atol=1e-11)


def test_lda_spin_polarised_and_vacuum_points():
    from amaterasu_b200.potential import GridOps  # noqa: F401  (loads the library)
    from amaterasu_b200._lib import call
    from amaterasu_b200.engine import ptr, stream_ptr
    from oracle.potential import lda_pz
    rng = np.random.default_rng(1)
    n = 4096
    rho = np.abs(rng.normal(size=(2, n))) * 10.0 ** rng.uniform(-8, 1, size=(2, n))
    rho[:, :5] = 0.0
    rho[0, 5:10] = 0.0  # fully polarised points
    d = torch.from_numpy(rho).cuda()
    eps = torch.empty(n, dtype=torch.float64, device="cuda")
    v = torch.empty((2, n), dtype=torch.float64, device="cuda")
    call("ama_lda_pz", ptr(d), n, ptr(eps), ptr(v), stream_ptr())
    e_ref, v_ref = lda_pz(rho.T)
    np.testing.assert_allclose(eps.cpu().numpy(), e_ref, rtol=1e-13, atol=1e-300)
    np.testing.assert_allclose(v.cpu().numpy(), v_ref.T, rtol=1e-12, atol=1e-300)


@pytest.mark.parametrize("precision,tol", [("complex128", 1e-12), ("complex64", 1e-5)])
def test_density_accumulate_matches_reference(mini_system, precision, tol):
    from amaterasu_b200.engine import engine_for
    g = golden("mini.npz")
    s = mini_system
    eng = engine_for(s)
    dtype = torch.complex128 if precision == "complex128" else torch.complex64
    wfs = [g["dav_vec0"], g["dav_vec1"]]
    occ = g["occ"]
    nb = wfs[0].shape[0]
    packed = torch.from_numpy(np.concatenate([w.ravel() for w in wfs])).to("cuda", dtype)
    w = 2.0 * s.kpoints.weights[:, None] * occ[0]
    weights = torch.from_numpy(np.ascontiguousarray(w.ravel())).cuda()
    rho = torch.zeros(int(np.prod(s.grid.shape)), dtype=torch.float64, device="cuda")
    eng.density_accumulate(packed, weights, rho, k_first=0, k_count=2, nbands=nb)
    rho = rho.cpu().numpy().reshape(s.grid.shape) / s.grid.volume
    ref = g["density_nosym"][0]
    assert np.max(np.abs(rho - ref)) / np.max(np.abs(ref)) < tol


def test_structure_sums_on_the_gpu_match_the_host_form(si_pseudo):
    """ama_structure_sum (used by the set-up's superposed density and local potential) against
    the host phase-matrix form, on a displaced 64-atom cell: 1e-12 of max|coefficient|."""
    import amaterasu_b200.local as local
    from amaterasu_b200.cells import si_supercell
    from amaterasu_b200.formfactors import density_form_factor
    from amaterasu_b200.system import build_system
    s = build_system(si_supercell(2, sigma=0.05, seed=3), {"Si": si_pseudo}, 6.0, 24.0,
                     build_projector_matrices=False)
    sph = s.density_sphere
    radial = {"Si": density_form_factor(si_pseudo.grid, si_pseudo.valence_density, np.sqrt(sph.g2))}
    dev = local._device_structure_sum(sph, s.positions, s.symbols, radial, 1.0 / s.grid.volume)
    assert dev is not None
    phases = local.structure_factors(sph, s.positions)
    host = (radial["Si"][None, :] * phases).sum(0) / s.grid.volume
    assert np.max(np.abs(dev - host)) < 1e-12 * np.max(np.abs(host))


@pytest.mark.parametrize("algo", ["linear", "pulay", "broyden", "anderson"])
@pytest.mark.parametrize("bare_grid", [False, True])
def test_mixers_match_reference_sequences(mini_system, algo, bare_grid):
    """The device mixers (grid-vector kernels + Kerker grid filter) reproduce the reference's
    six-step mixing sequences (mini.npz) to 1e-12, created the reference's way from the FFT
    grid alone (create_mixer(config, grid)); the bare-grid case builds a grid-only engine."""
    from amaterasu_b200.basis import FFTGrid
    from amaterasu_b200.config import MixingConfig
    from amaterasu_b200.mixing import create_mixer
    from amaterasu_b200.potential import grid_ops
    g = golden("mini.npz")
    s = mini_system
    if bare_grid:
        grid = FFTGrid(shape=tuple(s.grid.shape), cell=np.array(s.grid.cell))
    else:
        grid_ops(s)
        grid = s.grid
    mixer = create_mixer(MixingConfig(algorithm=algo), grid)
    target = g[f"mix_{algo}_target"]
    x = g["rho0"].copy()
    for step, ref in enumerate(g[f"mix_{algo}_seq"]):
        out = 0.5 * x + 0.5 * target + 0.002 * np.sin(step + x)
        x = mixer(x, out)
        np.testing.assert_allclose(x, ref, rtol=0, atol=1e-12, err_msg=f"{algo} step {step}")
