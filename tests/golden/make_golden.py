"""Generate the golden fixtures under ``tests/golden/`` by running the reference itself.

The reference (amaterasu 0.1.0a2) is pure numpy/scipy and is imported from its source
tree with the minimal ``ase``/``spglib`` stand-ins in ``tests/golden/shim`` (symmetry off,
time-reversal-only k-point reduction). Nothing here runs on the GPU box: the fixtures it
writes are committed, and the tests read only those.

    python tests/golden/make_golden.py [--reference PATH] [--only NAME ...]

Fixtures (``*.npz``):
  mini.npz      small Si2 system (two explicit k-points): set-up arrays, H.psi, Davidson,
                density, Hartree, LDA, mixing, occupations on full arrays
  si2_scf.npz   Si2 fcc 30 Ry, shifted 4x4x4 (32 k), 8 bands, LDA-PZ, fixed occupations:
                full SCF energies, eigenvalues, density, forces, stress
  si64.npz      Si64 40 Ry, Gamma + 3 random k: sphere and projector pins, v_eff
                checksums, H.psi of a few bands
  si8_k.npz     Si8 displaced, 8x8x8 Gamma mesh: k-points, weights, plane-wave counts
  si8_scf1.npz  the same Si8 cell at 40 Ry, 260 k-points, 20 bands, Fermi-Dirac 0.01 Ha:
                the first SCF iteration from the reference's own start (eigenvalues at
                every k, energy terms, output-density checksums and probes)
  si215.npz     Si215 (3x3x3 conventional, one vacancy, displaced), Gamma, 30 Ry, 440
                bands: sphere and projector pins, Ewald energy/forces/stress, v_eff
                checksums and probes, starting-orbital pins, H.psi of a few bands
  gga.npz       PBE / PBEsol: pointwise outputs at seeded points, the grid functional on
                the mini system's start density (unpolarised and spin-split), and a Si2
                PBE SCF (20 Ry, shifted 2x2x2, 8 bands) with forces and stress
"""
from __future__ import annotations

import argparse
import hashlib
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parent.parent


DEFAULT_REFERENCE = "/root/reference"


def reference_mini_system():
    """The reference's own PlaneWaveSystem for the mini configuration (Si2, two explicit
    k-points, 8 Ha), or None when the reference is not at DEFAULT_REFERENCE."""
    if not Path(DEFAULT_REFERENCE, "amaterasu").is_dir():
        return None
    _import_reference(DEFAULT_REFERENCE)
    from amaterasu_b200.cells import si2_primitive
    with tempfile.TemporaryDirectory() as tmp:
        pseudo, _ = _upf(tmp)
    kpts = [[0.0, 0.0, 0.0], [0.125, -0.25, 0.375]]
    cfg = _config(kpoints__scheme="explicit", kpoints__points=kpts, occupations__nbands=6,
                  occupations__scheme="gaussian", occupations__smearing=0.1)
    return _system(si2_primitive(), cfg, pseudo, 8.0)


def _import_reference(path: str):
    sys.path.insert(0, str(HERE / "shim"))
    sys.path.insert(0, path)
    sys.path.insert(0, str(REPO))
    import amaterasu  # noqa: F401  (the reference package)
    return amaterasu


def _atoms(structure):
    from ase import Atoms
    return Atoms(structure.symbols, structure.positions, structure.cell)


def _config(**kw):
    from amaterasu.config.schema import Config
    c = Config(structure="-")
    c.xc.functional = "LDA-PZ"
    for key, value in kw.items():
        section, name = key.split("__")
        setattr(getattr(c, section), name, value)
    return c


def _sha(array) -> str:
    return hashlib.sha256(np.ascontiguousarray(array).tobytes()).hexdigest()


def _upf(tmp):
    from amaterasu_b200.pseudo import write_synthetic_upf
    from amaterasu.pseudo.readers import read_pseudopotential
    path = write_synthetic_upf(Path(tmp) / "Si.synthetic.upf")
    return read_pseudopotential(str(path)), path


def _system(structure, config, pseudo, ecut):
    from amaterasu.hamiltonian.system import build_system
    return build_system(_atoms(structure), config, {"Si": pseudo}, ecut, 4.0 * ecut)


def damped_noise(npw, nbands, kinetic, seed):
    """Un-orthonormalised N(0,1)+iN(0,1) over (1+T_G): exactly reproducible anywhere."""
    rng = np.random.default_rng(seed)
    block = rng.normal(size=(nbands, npw)) + 1j * rng.normal(size=(nbands, npw))
    return block / (1.0 + kinetic)


# --------------------------------------------------------------------------- mini
def make_mini(pseudo, out):
    from amaterasu.hamiltonian.operator import Hamiltonian
    from amaterasu.hamiltonian.hartree import hartree
    from amaterasu.scf.density import compute_density
    from amaterasu.scf.driver import effective_potential
    from amaterasu.scf.eigen import davidson, random_bands, rayleigh_ritz, orthonormalize
    from amaterasu.scf.eigen.precond import teter_payne_allan
    from amaterasu.scf.mixing import create_mixer
    from amaterasu.scf.occupations import compute_occupations
    from amaterasu.xc.driver import XCFunctional
    from amaterasu_b200.cells import si2_primitive

    kpts = [[0.0, 0.0, 0.0], [0.125, -0.25, 0.375]]
    cfg = _config(kpoints__scheme="explicit", kpoints__points=kpts, occupations__nbands=6,
                  occupations__scheme="gaussian", occupations__smearing=0.1)
    system = _system(si2_primitive(), cfg, pseudo, 8.0)
    rho0 = system.initial_density()
    veff, e_h, e_xc, _ = effective_potential(system, rho0)
    H = Hamiltonian(system, veff)
    d = dict(grid=np.array(system.grid.shape), kpoints=system.kpoints.points,
             weights=system.kpoints.weights, nbands=system.nbands, ewald=system.ewald,
             v_local=system.v_local, rho0=rho0, veff=veff, e_hartree0=e_h, e_xc0=e_xc,
             density_miller=system.density_sphere.miller)
    for ik, sphere in enumerate(system.wave_spheres):
        d[f"miller{ik}"] = sphere.miller
        d[f"kinetic{ik}"] = sphere.kinetic_energy
        d[f"proj{ik}"] = system.projectors[ik].matrix
        d[f"dij{ik}"] = system.projectors[ik].dij
        psi = damped_noise(len(sphere), 7, sphere.kinetic_energy, 100 + ik)
        d[f"psi{ik}"] = psi
        d[f"hpsi{ik}"] = H.apply(psi, ik)
        guess = random_bands(len(sphere), system.nbands, sphere.kinetic_energy, seed=12345 + ik)
        d[f"guess{ik}"] = guess
        res = davidson(lambda b, ik=ik: H.apply(b, ik), guess, sphere.kinetic_energy,
                       tolerance=1e-9, max_iterations=60)
        d[f"dav_eig{ik}"] = res.eigenvalues
        d[f"dav_vec{ik}"] = res.coefficients
        d[f"dav_iters{ik}"] = res.iterations
        # single-step pins of the subspace pieces
        basis = orthonormalize(psi[:4])
        d[f"ortho{ik}"] = basis
        e, x, hx = rayleigh_ritz(basis, H.apply(basis, ik), 3)
        d[f"rr_eig{ik}"] = e
        r = hx - e[:, None] * x
        t_band = np.einsum("ng,g->n", np.abs(x) ** 2, sphere.kinetic_energy)
        d[f"tpa_in{ik}"] = r
        d[f"tpa_ref{ik}"] = t_band
        d[f"tpa_out{ik}"] = teter_payne_allan(r, sphere.kinetic_energy, t_band)
    wfs = [[d["dav_vec0"], d["dav_vec1"]]]
    eig = np.array([[d["dav_eig0"], d["dav_eig1"]]])
    occ = compute_occupations(eig, system.kpoints.weights, system.nelectrons,
                              scheme="gaussian", smearing=0.1 / 27.211386, nspin=1)
    d["occ"] = occ.occupations
    d["fermi"] = occ.fermi_level
    d["density"] = compute_density(system, wfs, occ.occupations)
    d["density_nosym"] = compute_density(system, wfs, occ.occupations, symmetrize=False)
    e_h2, v_h2 = hartree(system.grid, system.density_sphere, d["density"][0])
    d["hartree_e"] = e_h2
    d["hartree_v"] = v_h2
    xcr = XCFunctional("LDA-PZ").evaluate_on_grid(d["density"], system.grid)
    d["xc_e"] = xcr.energy
    d["xc_v"] = xcr.potential
    # mixing sequences: a contractive linear map n -> A n + b with the grid's shape
    rng = np.random.default_rng(5)
    shape = (1, *system.grid.shape)
    n_in = rho0.copy()
    for algo in ("linear", "pulay", "broyden", "anderson"):
        from amaterasu.config.schema import MixingConfig
        mixer = create_mixer(MixingConfig(algorithm=algo), system.grid)
        target = rho0 + 0.01 * rng.normal(size=shape)
        x = n_in.copy()
        seq = []
        for step in range(6):
            out_ = 0.5 * x + 0.5 * target + 0.002 * np.sin(step + x)
            x = mixer(x, out_)
            seq.append(x.copy())
        d[f"mix_{algo}_target"] = target
        d[f"mix_{algo}_seq"] = np.array(seq)
    np.savez_compressed(out / "mini.npz", **d)


# ------------------------------------------------------------------------ si2_scf
def make_si2(pseudo, out):
    from amaterasu.scf.driver import run_scf
    from amaterasu.properties.forces import compute_forces
    from amaterasu.properties.stress import compute_stress
    from amaterasu_b200.cells import si2_primitive

    cfg = _config(kpoints__grid=[4, 4, 4], kpoints__shift=[0.5, 0.5, 0.5],
                  occupations__scheme="fixed", occupations__nbands=8,
                  scf__tol_energy=1e-8, scf__tol_density=1e-8)
    t0 = time.perf_counter()
    system = _system(si2_primitive(), cfg, pseudo, 15.0)
    setup = time.perf_counter() - t0
    result = run_scf(system, cfg, logger=print)
    forces = compute_forces(system, result.density, result.wavefunctions, result.occupations,
                            eigenvalues=result.eigenvalues, decompose=True)
    stress = compute_stress(system, result.density, result.wavefunctions, result.occupations,
                            eigenvalues=result.eigenvalues, decompose=True)
    e = result.energies
    d = dict(grid=np.array(system.grid.shape), kpoints=system.kpoints.points,
             weights=system.kpoints.weights, npw=np.array([len(s) for s in system.wave_spheres]),
             miller_sha=np.array([_sha(s.miller.astype(np.int64)) for s in system.wave_spheres]),
             ewald=system.ewald, v_local=system.v_local, rho0=system.initial_density(),
             converged=result.converged, iterations=result.iterations,
             e_kinetic=e.kinetic, e_local=e.local, e_hartree=e.hartree, e_xc=e.xc,
             e_nonlocal=e.nonlocal_, e_ewald=e.ewald, e_entropy=e.entropy,
             e_total=e.total, e_free=e.free_energy,
             eigenvalues=result.eigenvalues, occupations=result.occupations,
             fermi=result.fermi_level, density=result.density,
             history=np.array(result.history), seconds_setup=setup, seconds_scf=result.seconds)
    for name, value in forces.items():
        d[f"force_{name}"] = value
    d["forces"] = sum(forces.values())
    for name, value in stress.items():
        d[f"stress_{name}"] = value
    d["stress"] = sum(stress.values())
    np.savez_compressed(out / "si2_scf.npz", **d)


# -------------------------------------------------------------------------- si64
def make_si64(pseudo, out):
    from amaterasu.hamiltonian.operator import Hamiltonian
    from amaterasu.scf.driver import effective_potential
    from amaterasu_b200.cells import hpsi_bench_kpoints, si_supercell

    kset = hpsi_bench_kpoints()
    cfg = _config(kpoints__scheme="explicit", kpoints__points=kset.points.tolist(),
                  occupations__nbands=160)
    t0 = time.perf_counter()
    system = _system(si_supercell(2), cfg, pseudo, 20.0)
    setup = time.perf_counter() - t0
    rho0 = system.initial_density()
    veff, e_h, e_xc, _ = effective_potential(system, rho0)
    rng = np.random.default_rng(11)
    probe = rng.integers(0, veff.size, size=200)
    d = dict(grid=np.array(system.grid.shape), kpoints=system.kpoints.points,
             npw=np.array([len(s) for s in system.wave_spheres]),
             miller_sha=np.array([_sha(s.miller.astype(np.int64)) for s in system.wave_spheres]),
             nproj=len(system.projectors[0]), ewald=system.ewald, seconds_setup=setup,
             e_hartree0=e_h, e_xc0=e_xc, probe=probe, veff_probe=veff.ravel()[probe],
             veff_sum=float(veff.sum()), veff_sq=float((veff**2).sum()),
             vloc_probe=system.v_local.ravel()[probe], rho0_probe=rho0.ravel()[probe])
    for ik, sphere in enumerate(system.wave_spheres):
        B = system.projectors[ik].matrix
        d[f"proj_norms{ik}"] = np.linalg.norm(B, axis=1)
        d[f"proj_row0_{ik}"] = B[0, :64]
        d[f"proj_row5_{ik}"] = B[5, :64]
    H = Hamiltonian(system, veff)
    for ik, nb in ((0, 2), (1, 1)):
        sphere = system.wave_spheres[ik]
        psi = damped_noise(len(sphere), nb, sphere.kinetic_energy, 300 + ik)
        t0 = time.perf_counter()
        d[f"hpsi{ik}"] = H.apply(psi, ik)
        d[f"seconds_hpsi{ik}"] = time.perf_counter() - t0
    np.savez_compressed(out / "si64.npz", **d)


# --------------------------------------------------------------------------- si8
def make_si8(pseudo, out):
    from amaterasu.system.kpoints import generate
    from amaterasu.basis.gvectors import GSphere
    from amaterasu.units import ANG_IN_BOHR
    from amaterasu_b200.cells import si_supercell

    s = si_supercell(1, sigma=0.05, seed=8)
    cfg = _config(kpoints__grid=[8, 8, 8])
    kset = generate(_atoms(s), cfg.kpoints)
    cell = np.asarray(s.cell) * ANG_IN_BOHR
    npw = np.array([len(GSphere.build(cell, 20.0, kpoint=k)) for k in kset.points])
    np.savez_compressed(out / "si8_k.npz", kpoints=kset.points, weights=kset.weights, npw=npw,
                        positions=s.positions)


# ---------------------------------------------------------------------- si8_scf1
def make_si8_scf1(pseudo, out):
    from amaterasu.scf.driver import run_scf
    from amaterasu_b200.cells import workload

    structure, ecut, _, nbands = workload("si8_batched")
    cfg = _config(kpoints__grid=[8, 8, 8], occupations__scheme="fermi-dirac",
                  occupations__smearing="0.01 Ha", occupations__nbands=nbands,
                  scf__max_steps=1)
    t0 = time.perf_counter()
    system = _system(structure, cfg, pseudo, ecut)
    setup = time.perf_counter() - t0
    result = run_scf(system, cfg, logger=print)
    e = result.energies
    rng = np.random.default_rng(81)
    probe = rng.integers(0, result.density.size, size=400)
    np.savez_compressed(
        out / "si8_scf1.npz", grid=np.array(system.grid.shape), kpoints=system.kpoints.points,
        weights=system.kpoints.weights, npw=np.array([len(s) for s in system.wave_spheres]),
        ewald=system.ewald, e_kinetic=e.kinetic, e_local=e.local, e_hartree=e.hartree,
        e_xc=e.xc, e_nonlocal=e.nonlocal_, e_entropy=e.entropy, e_free=e.free_energy,
        eigenvalues=result.eigenvalues, occupations=result.occupations, fermi=result.fermi_level,
        history=np.array(result.history), probe=probe, density_probe=result.density.ravel()[probe],
        density_sum=float(result.density.sum()), density_sq=float((result.density**2).sum()),
        seconds_setup=setup, seconds_scf=result.seconds)


# ------------------------------------------------------------------------- si215
def make_si215(pseudo, out):
    from amaterasu.hamiltonian.ewald import ewald
    from amaterasu.hamiltonian.operator import Hamiltonian
    from amaterasu.scf.driver import effective_potential
    from amaterasu.scf.eigen import random_bands
    from amaterasu_b200.cells import workload

    structure, ecut, _, nbands = workload("si215_gamma")
    cfg = _config(kpoints__scheme="gamma", occupations__scheme="gaussian",
                  occupations__smearing="0.005 Ha", occupations__nbands=nbands)
    t0 = time.perf_counter()
    system = _system(structure, cfg, pseudo, ecut)
    setup = time.perf_counter() - t0
    print(f"si215 set-up {setup:.1f} s", flush=True)
    charges = np.full(len(system.symbols), 4.0)
    ew = ewald(system.cell, system.positions, charges)
    rho0 = system.initial_density()
    veff, e_h, e_xc, _ = effective_potential(system, rho0)
    rng = np.random.default_rng(215)
    probe = rng.integers(0, veff.size, size=400)
    sphere = system.wave_spheres[0]
    B = system.projectors[0].matrix
    d = dict(grid=np.array(system.grid.shape), npw=np.array([len(sphere)]),
             miller_sha=np.array([_sha(sphere.miller.astype(np.int64))]), nproj=len(B),
             ewald=system.ewald, ewald_energy=ew.energy, ewald_forces=ew.forces, ewald_stress=ew.stress,
             positions=system.positions, cell=system.cell, seconds_setup=setup,
             e_hartree0=e_h, e_xc0=e_xc, probe=probe, veff_probe=veff.ravel()[probe],
             veff_sum=float(veff.sum()), veff_sq=float((veff**2).sum()),
             vloc_probe=system.v_local.ravel()[probe], rho0_probe=rho0.ravel()[probe],
             rho0_sum=float(rho0.sum()), proj_norms=np.linalg.norm(B, axis=1),
             proj_row0=B[0, :64], proj_row859=B[-1, :64])
    t0 = time.perf_counter()
    start = random_bands(len(sphere), nbands, sphere.kinetic_energy, seed=12345)
    d["seconds_random_bands"] = time.perf_counter() - t0
    d["start_row0"] = start[0, :256]
    d["start_row_last"] = start[-1, :256]
    d["start_col_norms"] = np.linalg.norm(start[:, :512], axis=0)
    del start
    H = Hamiltonian(system, veff)
    psi = damped_noise(len(sphere), 3, sphere.kinetic_energy, 2150)
    t0 = time.perf_counter()
    d["hpsi"] = H.apply(psi, 0)
    d["seconds_hpsi3"] = time.perf_counter() - t0
    np.savez_compressed(out / "si215.npz", **d)


# ------------------------------------------------------------------------------ gga
def make_gga(pseudo, out):
    """PBE / PBEsol: the pointwise functionals at seeded points, the grid functional on the
    mini system's starting density (unpolarised, and split 0.6 / 0.4 between the spins), and
    a small Si2 PBE SCF with forces and stress."""
    from amaterasu.properties.forces import compute_forces
    from amaterasu.properties.stress import compute_stress
    from amaterasu.scf.driver import run_scf
    from amaterasu.xc import gga
    from amaterasu.xc.driver import XCFunctional
    from amaterasu_b200.cells import si2_primitive

    rng = np.random.default_rng(2024)
    n = 600
    tot = 10.0 ** rng.uniform(-6, 1, n)
    zeta = rng.uniform(-0.95, 0.95, n)
    zeta[:100] = 0.0
    rho = np.stack([tot * (1 + zeta) / 2, tot * (1 - zeta) / 2], axis=-1)
    g = rng.normal(size=(n, 2, 3)) * tot[:, None, None] ** (4 / 3) * 10.0 ** rng.uniform(-3, 1, (n, 1, 1))
    g[:40] = 0.0
    sigma = np.stack([np.sum(g[:, 0] * g[:, 0], 1), np.sum(g[:, 0] * g[:, 1], 1), np.sum(g[:, 1] * g[:, 1], 1)], -1)
    d = dict(rho=rho, sigma=sigma)
    for name in ("PBE", "PBEsol"):
        ex, vx, sx = gga.exchange(rho, sigma, name)
        ec, vc, sc = gga.correlation(rho, sigma, name)
        d[f"{name}_eps"] = ex + ec
        d[f"{name}_vrho"] = vx + vc
        d[f"{name}_vsigma"] = sx + sc
    system = reference_mini_system()
    rho0 = system.initial_density()
    d["mini_cell"] = system.grid.cell
    d["mini_rho0"] = rho0
    for name in ("PBE", "PBEsol"):
        r = XCFunctional(name).evaluate_on_grid(rho0, system.grid)
        d[f"mini_{name}_energy"] = r.energy
        d[f"mini_{name}_potential"] = r.potential
    pol = np.stack([0.6 * rho0[0], 0.4 * rho0[0]])
    r = XCFunctional("PBE").evaluate_on_grid(pol, system.grid)
    d["mini_pol_energy"] = r.energy
    d["mini_pol_potential"] = r.potential
    cfg = _config(kpoints__grid=[2, 2, 2], kpoints__shift=[0.5, 0.5, 0.5], occupations__scheme="fixed",
                  occupations__nbands=8, scf__tol_energy=1e-8, scf__tol_density=1e-8)
    cfg.xc.functional = "PBE"
    system = _system(si2_primitive(), cfg, pseudo, 10.0)
    result = run_scf(system, cfg, logger=print)
    forces = compute_forces(system, result.density, result.wavefunctions, result.occupations,
                            eigenvalues=result.eigenvalues, decompose=True)
    stress = compute_stress(system, result.density, result.wavefunctions, result.occupations,
                            eigenvalues=result.eigenvalues, decompose=True)
    e = result.energies
    d.update(scf_grid=np.array(system.grid.shape), scf_kpoints=system.kpoints.points,
             scf_weights=system.kpoints.weights, scf_iterations=result.iterations,
             scf_converged=result.converged, scf_e_kinetic=e.kinetic, scf_e_local=e.local,
             scf_e_hartree=e.hartree, scf_e_xc=e.xc, scf_e_nonlocal=e.nonlocal_, scf_e_ewald=e.ewald,
             scf_e_total=e.total, scf_e_free=e.free_energy, scf_eigenvalues=result.eigenvalues,
             scf_density=result.density)
    for name, value in forces.items():
        d[f"scf_force_{name}"] = value
    for name, value in stress.items():
        d[f"scf_stress_{name}"] = value
    np.savez_compressed(out / "gga.npz", **d)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=DEFAULT_REFERENCE)
    ap.add_argument("--only", nargs="*", default=None)
    args = ap.parse_args()
    _import_reference(args.reference)
    jobs = {"mini": make_mini, "si8": make_si8, "si64": make_si64, "si2": make_si2,
            "si215": make_si215, "si8_scf1": make_si8_scf1, "gga": make_gga}
    with tempfile.TemporaryDirectory() as tmp:
        pseudo, _ = _upf(tmp)
        for name, job in jobs.items():
            if args.only and name not in args.only:
                continue
            t0 = time.perf_counter()
            job(pseudo, HERE)
            print(f"{name}: {time.perf_counter() - t0:.1f} s", flush=True)


if __name__ == "__main__":
    main()
