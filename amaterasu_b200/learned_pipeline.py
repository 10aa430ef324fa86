"""Data generation, training and evaluation of the learned start density.

    python -m amaterasu_b200.learned_pipeline all --train 48 --test 12 --out DIR

Cells: the 8-atom conventional silicon cell (a = 5.43 A) under a seeded random symmetric
strain (components uniform in +-3 %) with seeded N(0, 0.1 A) atomic displacements, the
synthetic norm-conserving dataset, ecut 30 Ry, an unshifted 4x4x4 mesh reduced by time
reversal, LDA-PZ, Gaussian smearing 0.01 Ha. Each cell is converged by the engine
(mixed precision with FP64 refinement) from the superposed atomic density; the pair
(n0, strain) -> n_conv, resampled to the 36^3 working grid, is one training sample.
Evaluation converges held-out cells from both starts and reports iterations, time and the
final-energy difference (the fixed point must not move: |dE| < 1e-6 Ha).
"""
from __future__ import annotations

import argparse
import json
import tempfile
import time
from pathlib import Path

import numpy as np

A_SI = 5.43


def make_cell(seed: int):
    from .cells import _DIAMOND
    from .system import Structure
    rng = np.random.default_rng(seed)
    e = rng.uniform(-0.03, 0.03, size=(3, 3))
    e = 0.5 * (e + e.T)
    ref = np.eye(3) * A_SI
    cell = ref @ (np.eye(3) + e)
    pos = _DIAMOND @ cell + rng.normal(scale=0.1, size=(8, 3))
    return Structure(["Si"] * 8, pos, cell), ref


def _pseudo():
    from .pseudo import read_upf, write_synthetic_upf
    with tempfile.TemporaryDirectory() as tmp:
        return read_upf(write_synthetic_upf(Path(tmp) / "Si.upf"))


def _config(precision="mixed"):
    from .config import Config
    c = Config()
    c.occupations.scheme = "gaussian"
    c.occupations.smearing = "0.01 Ha"
    c.scf.tol_energy = 1e-6
    c.scf.tol_density = 1e-7
    c.scf.max_steps = 60
    c.engine.precision = precision
    return c


def build(structure, pseudo, kmesh=(4, 4, 4), ecut=15.0):
    from . import kpoints as kp
    from .system import build_system
    return build_system(structure, {"Si": pseudo}, ecut, 4 * ecut, kpoints=kp.monkhorst_pack(kmesh), nbands=20)


def run_cell(seed, pseudo, *, kmesh=(4, 4, 4), ecut=15.0, density=None, precision="mixed"):
    import torch
    from .learned import WORK_GRID, fourier_resample, strain_of
    from .scf import run_scf
    structure, ref = make_cell(seed)
    system = build(structure, pseudo, kmesh, ecut)
    n0 = system.initial_density()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    start = n0 if density is None else density(system)
    res = run_scf(system, _config(precision), density=start)
    torch.cuda.synchronize()
    seconds = time.perf_counter() - t0
    work = (WORK_GRID,) * 3
    return dict(seed=seed, grid=list(system.grid.shape), iterations=res.iterations, converged=res.converged,
                free_energy=res.energies.free_energy, seconds=seconds,
                n0=fourier_resample(n0.sum(0), work).astype(np.float32),
                nconv=fourier_resample(res.density.sum(0), work).astype(np.float32),
                strain=strain_of(system.cell, ref * (1.0 / 0.529177210903)))


def generate(seeds, out_file, **kw):
    pseudo = _pseudo()
    rows = []
    for s in seeds:
        r = run_cell(s, pseudo, **kw)
        rows.append(r)
        print(f"cell {s}: grid {r['grid']} {r['iterations']} iterations {r['seconds']:.1f} s", flush=True)
    np.savez_compressed(out_file, n0=np.stack([r["n0"] for r in rows]), nconv=np.stack([r["nconv"] for r in rows]),
                        strain=np.stack([r["strain"] for r in rows]), seeds=np.array(seeds),
                        iterations=np.array([r["iterations"] for r in rows]),
                        seconds=np.array([r["seconds"] for r in rows]))
    return rows


def samples(data):
    from .learned import network_input
    x = np.stack([network_input(np.maximum(n0, 1e-12), st) for n0, st in zip(data["n0"], data["strain"])])
    t = np.log(np.maximum(data["nconv"], 1e-12) / np.maximum(data["n0"], 1e-12))[:, None].astype(np.float32)
    return x, t


def fit(dataset, weights_out, epochs=200, seed=0):
    from .learned import DensityNet, train
    data = np.load(dataset)
    x, t = samples(data)
    net = DensityNet(seed=seed)
    hist = train(net, x, t, epochs=epochs, log=lambda m: print(m, flush=True))
    net.save(weights_out)
    return hist


def evaluate(weights, seeds, **kw):
    from .learned import DensityNet, LearnedStart
    pseudo = _pseudo()
    net = DensityNet.from_file(weights)
    learned = LearnedStart(net, np.eye(3) * A_SI / 0.529177210903)
    rows = []
    for s in seeds:
        base = run_cell(s, pseudo, **kw)
        pred = run_cell(s, pseudo, density=learned.predict, **kw)
        rows.append(dict(seed=s, iterations_superposition=base["iterations"], iterations_learned=pred["iterations"],
                         seconds_superposition=base["seconds"], seconds_learned=pred["seconds"],
                         energy_difference=abs(base["free_energy"] - pred["free_energy"]),
                         fallback=learned.stats.get("fallback", False)))
        print(json.dumps(rows[-1]), flush=True)
    return rows


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("stage", choices=["generate", "fit", "evaluate", "all"])
    ap.add_argument("--train", type=int, default=48)
    ap.add_argument("--test", type=int, default=12)
    ap.add_argument("--epochs", type=int, default=200)
    ap.add_argument("--kmesh", type=int, nargs=3, default=[4, 4, 4])
    ap.add_argument("--out", default="learned_out")
    args = ap.parse_args()
    out = Path(args.out)
    out.mkdir(parents=True, exist_ok=True)
    train_seeds = list(range(1000, 1000 + args.train))
    test_seeds = list(range(5000, 5000 + args.test))
    kw = dict(kmesh=tuple(args.kmesh))
    if args.stage in ("generate", "all"):
        generate(train_seeds, out / "dataset.npz", **kw)
    if args.stage in ("fit", "all"):
        fit(out / "dataset.npz", out / "density_net.npz", epochs=args.epochs)
    if args.stage in ("evaluate", "all"):
        rows = evaluate(out / "density_net.npz", test_seeds, **kw)
        summary = dict(cells=len(rows),
                       mean_iterations_superposition=float(np.mean([r["iterations_superposition"] for r in rows])),
                       mean_iterations_learned=float(np.mean([r["iterations_learned"] for r in rows])),
                       mean_seconds_superposition=float(np.mean([r["seconds_superposition"] for r in rows])),
                       mean_seconds_learned=float(np.mean([r["seconds_learned"] for r in rows])),
                       max_energy_difference=float(np.max([r["energy_difference"] for r in rows])),
                       rows=rows)
        (out / "evaluation.json").write_text(json.dumps(summary, indent=1))
        print(json.dumps({k: v for k, v in summary.items() if k != "rows"}), flush=True)


if __name__ == "__main__":
    main()
