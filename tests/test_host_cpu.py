"""Host-side option handling (no GPU): engine option overrides and their types."""
import pytest


def test_engine_option_overrides_are_typed_like_the_defaults():
    from amaterasu_b200.scf_benchmark import parse_engine_options
    opts = parse_engine_options(["c64_tolerance_floor=5e-7", "refine_max_iterations=2", "tc_subspace=false",
                                 "autotune=1", "tc_min_npw=2048"])
    assert opts == {"c64_tolerance_floor": 5e-7, "refine_max_iterations": 2, "tc_subspace": False,
                    "autotune": True, "tc_min_npw": 2048}
    assert isinstance(opts["refine_max_iterations"], int)
    with pytest.raises(ValueError):
        parse_engine_options(["no_such_option=1"])


def test_scf_benchmark_config_applies_overrides():
    from amaterasu_b200.scf_benchmark import _config
    c = _config("si215_gamma", "mixed", {"refine_max_iterations": 3})
    assert c.engine.precision == "mixed" and c.engine.refine_max_iterations == 3
    assert c.occupations.scheme == "gaussian" and c.scf.tol_energy == 1e-5


def test_device_timeout_is_raised_not_ignored(monkeypatch):
    """A timed-out device wait (device error word != 0) must stop the SCF step: the check
    reads the tensor-core and eigensolver status words and raises; with every word clear
    it returns quietly."""
    import ctypes as ct

    from amaterasu_b200 import engine as E

    words = {"ama_tc_status": 0, "ama_subspace_tc_status": 0, "ama_solver_status": 0}

    def fake_call(name, *args):
        out = args[-1]  # ctypes byref(c_int32)
        ct.cast(out, ct.POINTER(ct.c_int32))[0] = words[name]

    monkeypatch.setattr(E, "call", fake_call)

    class FakeEngine:
        handle = ct.c_void_p(1)

    E.check_device_status(FakeEngine())
    words["ama_subspace_tc_status"] = 3
    with pytest.raises(E.DeviceTimeout, match="subspace tensor-core"):
        E.check_device_status(FakeEngine())
    words.update(ama_subspace_tc_status=0, ama_tc_status=2)
    with pytest.raises(E.DeviceTimeout, match="nonlocal"):
        E.check_device_status(FakeEngine())
    words.update(ama_tc_status=0, ama_solver_status=1)
    with pytest.raises(E.DeviceTimeout, match="eigensolver"):
        E.check_device_status(FakeEngine())


@pytest.mark.parametrize("scheme", ["fermi-dirac", "gaussian", "methfessel-paxton", "marzari-vanderbilt"])
@pytest.mark.parametrize("order", [1, 2, 3])
def test_smearing_functions_match_the_oracle(scheme, order):
    """The published closed forms (Methfessel-Paxton's A_n H_{2n-1} sum and A_N H_2N entropy,
    Marzari-Vanderbilt, a log-free Fermi-Dirac entropy) against the oracle's restatement of
    the reference's recursions, to 1e-14."""
    import numpy as np
    from amaterasu_b200 import occupations as occ
    from oracle import scf as o
    x = np.linspace(-12.0, 12.0, 2001)
    np.testing.assert_allclose(occ.occupation_function(x, scheme, order), o.occupation_function(x, scheme, order),
                               rtol=0, atol=1e-14)
    np.testing.assert_allclose(occ.entropy_function(x, scheme, order), o.entropy_function(x, scheme, order),
                               rtol=0, atol=1e-14)


@pytest.mark.parametrize("scheme,smearing", [("gaussian", 0.01), ("fermi-dirac", 0.005), ("methfessel-paxton", 0.02),
                                             ("marzari-vanderbilt", 0.02), ("fixed", 0.0)])
def test_occupations_match_the_oracle(scheme, smearing):
    import numpy as np
    from amaterasu_b200.occupations import compute_occupations
    from oracle.scf import compute_occupations as oracle_occupations
    rng = np.random.default_rng(4)
    eig = np.sort(rng.uniform(-0.3, 0.6, size=(1, 7, 12)), axis=2)
    w = rng.uniform(0.5, 1.5, 7)
    w /= w.sum()
    res = compute_occupations(eig, w, 13.0, scheme=scheme, smearing=smearing)
    occ, fermi, ent, gap = oracle_occupations(eig, w, 13.0, scheme, smearing)
    np.testing.assert_allclose(res.occupations, occ, rtol=0, atol=1e-11)
    np.testing.assert_allclose(res.fermi_level, fermi, rtol=0, atol=1e-11)
    np.testing.assert_allclose(res.entropy_term, ent, rtol=0, atol=1e-12)


def test_occupations_match_reference_golden(mini_system):
    import numpy as np
    from conftest import golden
    from amaterasu_b200.occupations import compute_occupations
    g = golden("mini.npz")
    eig = np.array([[g["dav_eig0"], g["dav_eig1"]]])
    res = compute_occupations(eig, mini_system.kpoints.weights, mini_system.nelectrons, scheme="gaussian",
                              smearing=0.1 / 27.211386, nspin=1)
    np.testing.assert_allclose(res.occupations, g["occ"], rtol=0, atol=1e-12)
    np.testing.assert_allclose(res.fermi_level, float(g["fermi"]), rtol=0, atol=1e-11)
    with pytest.raises(ValueError, match="not one of"):
        compute_occupations(eig, mini_system.kpoints.weights, 8.0, scheme="bogus", smearing=0.01)


def test_engine_tables_from_a_reference_system(mini_system):
    """The drop-in boundary with the reference's own objects: the AmaSystemDesc host tables
    (grid, plane-wave counts, Miller indices in sphere order, kinetic energies, projector
    matrices, D) that the engine builds from the reference's PlaneWaveSystem equal the ones
    from this package's system, so Hamiltonian(reference_system, v_eff) sets up the same
    engine. Needs the reference source tree (skipped where it is absent)."""
    import sys

    import numpy as np
    from conftest import GOLDEN
    sys.path.insert(0, str(GOLDEN))
    import make_golden
    from amaterasu_b200.engine import system_tables
    ref_system = make_golden.reference_mini_system()
    if ref_system is None:
        pytest.skip("the reference source tree is not available here")
    ours, theirs = system_tables(mini_system), system_tables(ref_system)
    assert ours["grid"] == theirs["grid"] and ours["nproj"] == theirs["nproj"] and ours["nspin"] == theirs["nspin"]
    np.testing.assert_array_equal(ours["npw"], theirs["npw"])
    np.testing.assert_array_equal(ours["miller"], theirs["miller"])
    np.testing.assert_allclose(ours["kinetic"], theirs["kinetic"], rtol=0, atol=1e-13)
    np.testing.assert_allclose(ours["projectors"], theirs["projectors"], rtol=0, atol=1e-12)
    np.testing.assert_array_equal(ours["dij"], theirs["dij"])


def test_results_round_trip_in_output_units(tmp_path, mini_system):
    """write_scf / read_scf: the reference's groups and output units (eV, Angstrom, eV/A,
    eV/A^3 positive under compression), and the restart fields back in internal units."""
    import numpy as np
    from amaterasu_b200.results import read_scf, write_scf
    from amaterasu_b200.scf import Energies, SCFResult
    from amaterasu_b200.units import BOHR_IN_ANG, HARTREE_IN_EV
    s = mini_system
    rng = np.random.default_rng(0)
    dens = np.abs(rng.normal(size=(1, *s.grid.shape)))
    wfs = [[rng.normal(size=(6, len(w))) + 1j * rng.normal(size=(6, len(w))) for w in s.wave_spheres]]
    res = SCFResult(converged=True, iterations=7, energies=Energies(kinetic=1.0, local=-2.0, hartree=0.5, xc=-0.7,
                                                                    nonlocal_=0.3, ewald=-8.0, entropy=0.01),
                    eigenvalues=rng.normal(size=(1, 2, 6)), occupations=rng.random((1, 2, 6)), fermi_level=0.2,
                    gap=None, magnetization=0.0, density=dens, wavefunctions=wfs, history=[(1.0, 0.1, 0.0)],
                    electron_count=8.0)
    stress = np.diag([1e-4, 2e-4, 3e-4])
    path = write_scf(tmp_path / "r.npz", s, res, forces=np.ones((2, 3)) * 1e-3, stress=stress,
                     save_wavefunctions=True)
    out = read_scf(path)
    assert out["@format_version"] == 2 and out["@stress_convention"] == "positive_under_compression"
    np.testing.assert_allclose(out["scf"]["energies"]["@free_energy"], res.energies.free_energy * HARTREE_IN_EV)
    np.testing.assert_allclose(out["scf"]["eigenvalues"], res.eigenvalues * HARTREE_IN_EV)
    np.testing.assert_allclose(out["structure"]["cell"], s.cell * BOHR_IN_ANG)
    assert np.all(np.diag(out["stress"]) < 0)  # tensile internal stress is negative under compression
    assert out["@pressure_GPa"] < 0
    np.testing.assert_allclose(out["density_internal"], dens, rtol=1e-14)
    for a, b in zip(out["wavefunctions"][0], wfs[0]):
        np.testing.assert_array_equal(a, b)


def test_davidson_tolerance_schedule():
    """The reference's clip(1e-3 r, 1e-11, 1e-6) in FP64; the complex64 phase floored at the
    FP32 noise and capped at c64_tolerance_cap."""
    from amaterasu_b200.config import EngineConfig
    from amaterasu_b200.scf import davidson_tolerance
    e = EngineConfig()
    assert davidson_tolerance(0.5, False, e) == 1e-6
    assert davidson_tolerance(1e-5, False, e) == 1e-8
    assert davidson_tolerance(1e-12, False, e) == 1e-11
    e.c64_tolerance_cap = 1e-6
    assert davidson_tolerance(0.5, True, e) == e.c64_tolerance_floor  # cap below the floor
    e.c64_tolerance_cap = 1e-4
    assert davidson_tolerance(0.5, True, e) == 1e-4
    assert abs(davidson_tolerance(1e-2, True, e) - 1e-5) < 1e-20
    assert davidson_tolerance(1e-4, True, e) == e.c64_tolerance_floor
