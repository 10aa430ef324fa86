"""SCF wall time of the engine's precision policies on one workload.

    python -m amaterasu_b200.scf_benchmark --workload si215_gamma \\
        --weights amaterasu_b200/data/density_net_si64.npz --forces --out scf_si215.json

Runs, on the same system and GPU, to |dF| < 1e-5 eV/atom and an integrated density
residual below 1e-7 per electron:

* ``plain``: the FP64 engine (complex128 H.psi, Davidson and density) from the superposed
  atomic density, the reference's start;
* ``mixed``: complex64 bulk with tensor-core subspace products, FP64 refinement, from the
  same start;
* ``mixed_ref_schedule``: the same with the reference's Davidson tolerance cap (1e-6) in the
  complex64 phase instead of the policy's looser one while the density is far from
  converged (``c64_tolerance_cap``), to show what that part of the policy contributes;
* ``learned+mixed`` (with ``--weights``): the mixed policy from the learned start density,
  the network run on a working grid with the spacing it was trained at (0.151 A).

Reported per run: SCF seconds (system set-up excluded, the same for every run: grids,
spheres, projectors, structure factors and the seeded starting orbitals),
iterations, free energy, |dF| per atom against the plain run, and the largest force
(eV/A) and stress (GPa) differences against the plain run when ``--forces`` / ``--stress``
are given.
"""
from __future__ import annotations

import argparse
import json
import tempfile
import time
from pathlib import Path

import numpy as np

HARTREE_PER_BOHR_IN_EV_PER_ANG = 27.211386245988 / 0.529177210903
HARTREE_PER_BOHR3_IN_GPA = 29421.015697
SMEARING = {"si215_gamma": ("gaussian", "0.005 Ha"), "si8_batched": ("fermi-dirac", "0.01 Ha"),
            "si2_scf": ("fixed", None), "si64_hpsi": ("gaussian", "0.005 Ha")}


def _system(workload: str):
    from .cells import workload as make
    from .pseudo import read_upf, write_synthetic_upf
    from .system import build_system
    with tempfile.TemporaryDirectory() as tmp:
        pseudo = read_upf(write_synthetic_upf(Path(tmp) / "Si.upf"))
    structure, ecut, kpts, nbands = make(workload)
    return build_system(structure, {"Si": pseudo}, ecut, 4 * ecut, kpoints=kpts, nbands=nbands)


def _config(workload: str, precision: str, engine_options=None):
    from .config import Config
    c = Config()
    for key, value in (engine_options or {}).items():
        setattr(c.engine, key, value)
    scheme, smearing = SMEARING[workload]
    c.occupations.scheme = scheme
    if smearing:
        c.occupations.smearing = smearing
    c.scf.tol_energy = 1e-5
    c.scf.tol_density = 1e-7
    c.scf.max_steps = 80
    c.engine.precision = precision
    return c


TRAINING_SPACING_A = 5.43 / 36  # working-grid spacing the committed nets were trained at


def run(workload: str, weights=None, forces=False, log=print, policies=("plain", "mixed", "learned+mixed"),
        engine_options=None, spacing=TRAINING_SPACING_A, stress=False, hook=None, after=None) -> dict:
    """Run the policies on one system; ``hook(name, "start"|"stop")`` brackets each timed run
    (the bench samples clocks there); ``after(system)``, when given, runs on the same system
    once the policies are done and its result is returned under "after"."""
    import torch
    from .learned import DensityNet, LearnedStart, working_grid
    from .scf import prepare_starting_orbitals, run_scf
    t0 = time.perf_counter()
    system = _system(workload)
    prepare_starting_orbitals(system)  # the seeded start is part of the system, same for every policy
    torch.cuda.synchronize()
    setup = time.perf_counter() - t0
    runs = [(p, {"plain": "complex128"}.get(p, "mixed"), None) for p in policies
            if p in ("plain", "mixed", "mixed_ref_schedule")]
    if weights and "learned+mixed" in policies:
        net = DensityNet.from_file(weights)
        cell = np.asarray(system.cell, float)
        learned = LearnedStart(net, cell, grid=working_grid(cell, spacing / 0.529177210903))
        runs.append(("learned+mixed", "mixed", learned))
    out = dict(workload=workload, setup_seconds=setup, natoms=system.natoms, runs={})
    results = {}
    for name, precision, start in runs:
        if hook:
            hook(name, "start")
        torch.cuda.synchronize()
        t = time.perf_counter()
        density = start.predict(system) if start is not None else None
        options = dict(engine_options or {})
        if name == "mixed_ref_schedule":
            options["c64_tolerance_cap"] = 1e-6
        res = run_scf(system, _config(workload, precision, options), density=density)
        torch.cuda.synchronize()
        seconds = time.perf_counter() - t
        if hook:
            hook(name, "stop")
        row = dict(seconds=seconds, iterations=res.iterations, converged=res.converged,
                   free_energy=res.energies.free_energy, precision_trace=res.precision_trace.count("complex64"))
        if start is not None:
            row["fallback"] = bool(start.stats.get("fallback", False))
        if forces:
            from .properties import compute_forces
            row["_forces"] = compute_forces(system, res.density, res.wavefunctions, res.occupations)
        if stress:
            from .properties import compute_stress
            row["_stress"] = compute_stress(system, res.density, res.wavefunctions, res.occupations)
        results[name] = row
        log(f"{name}: {seconds:.1f} s, {res.iterations} iterations, F = {res.energies.free_energy:.10f} Ha")
    plain = results.get("plain")
    for name, row in results.items():
        if plain is not None:
            row["dF_per_atom_eV"] = abs(row["free_energy"] - plain["free_energy"]) * 27.211386245988 / system.natoms
            row["speedup_vs_plain"] = plain["seconds"] / row["seconds"]
            if forces:
                row["max_force_diff_eV_per_A"] = float(np.abs(row["_forces"] - plain["_forces"]).max()
                                                       * HARTREE_PER_BOHR_IN_EV_PER_ANG)
            if stress:
                row["max_stress_diff_GPa"] = float(np.abs(row["_stress"] - plain["_stress"]).max()
                                                   * HARTREE_PER_BOHR3_IN_GPA)
        out["runs"][name] = row
    for row in results.values():
        row.pop("_forces", None)
        row.pop("_stress", None)
    if after is not None:
        out["after"] = after(system)
    return out


def parse_engine_options(items) -> dict:
    """KEY=VALUE strings -> EngineConfig overrides, typed like the defaults."""
    from .config import EngineConfig
    defaults = EngineConfig()
    options = {}
    for item in items:
        key, value = item.split("=", 1)
        if not hasattr(defaults, key):
            raise ValueError(f"unknown engine option {key!r}")
        kind = type(getattr(defaults, key))
        options[key] = value.lower() in ("1", "true", "yes") if kind is bool else kind(value)
    return options


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", default="si215_gamma", choices=sorted(SMEARING))
    ap.add_argument("--weights", default=None)
    ap.add_argument("--forces", action="store_true")
    ap.add_argument("--stress", action="store_true")
    ap.add_argument("--policies", default="plain,mixed,learned+mixed")
    ap.add_argument("--spacing", type=float, default=TRAINING_SPACING_A,
                    help="working-grid spacing (A) the network was trained at")
    ap.add_argument("--engine", action="append", default=[],
                    help="engine option override KEY=VALUE (e.g. c64_tolerance_floor=5e-7)")
    ap.add_argument("--out", default=None)
    args = ap.parse_args()
    result = run(args.workload, args.weights, args.forces, policies=tuple(args.policies.split(",")),
                 engine_options=parse_engine_options(args.engine), spacing=args.spacing, stress=args.stress)
    text = json.dumps(result, indent=1)
    print(text, flush=True)
    if args.out:
        Path(args.out).write_text(text)


if __name__ == "__main__":
    main()
