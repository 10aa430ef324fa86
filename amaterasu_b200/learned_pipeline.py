"""Data generation, training and evaluation of the learned start density.

    python -m amaterasu_b200.learned_pipeline all --family si8 --train 2000 --test 200 --workers 8 --out DIR
    python -m amaterasu_b200.learned_pipeline all --family si64 --train 32 --test 4 --out DIR
    python -m amaterasu_b200.learned_pipeline all --family si215 --train 16 --test 2 --init W --out DIR

Cell families (synthetic norm-conserving dataset, ecut 30 Ry, LDA-PZ):

* ``si8``: the 8-atom conventional silicon cell (a = 5.43 A) under a seeded random
  symmetric strain (components uniform in +-3 %) with seeded N(0, 0.1 A) displacements,
  an unshifted 4x4x4 mesh reduced by time reversal, Gaussian smearing 0.01 Ha, 20 bands,
  working grid 36^3.
* ``si64``: the 2x2x2 conventional supercell (a = 10.86 A) with strain in +-1 %, N(0,
  0.05 A) displacements and, in every second cell, a vacancy; Gamma only, Gaussian smearing
  0.005 Ha, 144 bands, working grid 72^3 (0.151 A, the spacing of the si8 grid and of the
  3x3x3 supercell's 108^3 grid: the net trained here starts that cell). Its fit starts from
  the si8 weights (``fit --init``).
* ``si215``: the 3x3x3 conventional supercell (a = 16.29 A) with the first site vacant and
  N(0, 0.05 A) displacements, no strain (the distribution of the Si215 benchmark cell, whose
  own seed is not among the training or test seeds); Gamma only, Gaussian smearing 0.005 Ha,
  440 bands, working grid 108^3 (the system grid). Its fit starts from the si64 weights.

A coarser working grid than the system grid truncates the converged density's Fourier
series and the ringing makes log(n_conv / n0) meaningless in low-density regions, so the
working grids keep the system grid's spacing.

Each cell is converged by the engine (mixed precision with FP64 refinement) from the
superposed atomic density; the pair (n0, strain) -> n_conv on the working grid is one
training sample. Evaluation converges held-out cells from both starts and reports
iterations, time and the final-energy difference (the fixed point must not move:
|dE| < 1e-6 Ha).
"""
from __future__ import annotations

import argparse
import json
import tempfile
import time
from pathlib import Path

import numpy as np

A_SI = 5.43
BOHR_IN_ANGSTROM = 0.529177210903

FAMILIES = {
    "si8": dict(supercell=1, strain=0.03, sigma=0.1, vacancy_every=0, kmesh=(4, 4, 4), smearing="0.01 Ha",
                nbands=20, grid=36),
    "si64": dict(supercell=2, strain=0.01, sigma=0.05, vacancy_every=2, kmesh=None, smearing="0.005 Ha",
                 nbands=144, grid=72),
    "si215": dict(supercell=3, strain=0.0, sigma=0.05, vacancy_every=1, kmesh=None, smearing="0.005 Ha",
                  nbands=440, grid=108),
}


def reference_cell(family: str) -> np.ndarray:
    """Unstrained cell of a family, Angstrom."""
    return np.eye(3) * A_SI * FAMILIES[family]["supercell"]


def make_cell(seed: int, family: str = "si8"):
    from .cells import _DIAMOND
    from .system import Structure
    f = FAMILIES[family]
    n = f["supercell"]
    rng = np.random.default_rng(seed)
    e = rng.uniform(-f["strain"], f["strain"], size=(3, 3))
    e = 0.5 * (e + e.T)
    ref = reference_cell(family)
    cell = ref @ (np.eye(3) + e)
    frac = np.vstack([(_DIAMOND + np.array([i, j, k])) / n for i in range(n) for j in range(n) for k in range(n)])
    if f["vacancy_every"] and seed % f["vacancy_every"] == 0:
        frac = frac[1:]
    pos = frac @ cell + rng.normal(scale=f["sigma"], size=(len(frac), 3))
    return Structure(["Si"] * len(pos), pos, cell), ref


def _pseudo():
    from .pseudo import read_upf, write_synthetic_upf
    with tempfile.TemporaryDirectory() as tmp:
        return read_upf(write_synthetic_upf(Path(tmp) / "Si.upf"))


def _config(family: str, precision="mixed"):
    from .config import Config
    c = Config()
    c.occupations.scheme = "gaussian"
    c.occupations.smearing = FAMILIES[family]["smearing"]
    c.scf.tol_energy = 1e-6
    c.scf.tol_density = 1e-7
    c.scf.max_steps = 60
    c.engine.precision = precision
    return c


def build(structure, pseudo, family: str, ecut=15.0):
    from . import kpoints as kp
    from .system import build_system
    f = FAMILIES[family]
    kpts = kp.monkhorst_pack(f["kmesh"]) if f["kmesh"] else kp.gamma_only()
    return build_system(structure, {"Si": pseudo}, ecut, 4 * ecut, kpoints=kpts, nbands=f["nbands"])


def run_cell(seed, pseudo, *, family="si8", ecut=15.0, density=None, precision="mixed"):
    import torch
    from .learned import fourier_resample, strain_of
    from .scf import run_scf
    structure, ref = make_cell(seed, family)
    system = build(structure, pseudo, family, ecut)
    # timed: the start density (superposition or prediction) and the SCF
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    start = system.initial_density() if density is None else density(system)
    res = run_scf(system, _config(family, precision), density=start)
    torch.cuda.synchronize()
    seconds = time.perf_counter() - t0
    n0 = system.initial_density() if density is not None else start
    work = (FAMILIES[family]["grid"],) * 3
    return dict(seed=seed, grid=list(system.grid.shape), iterations=res.iterations, converged=res.converged,
                free_energy=res.energies.free_energy, seconds=seconds,
                n0=fourier_resample(n0.sum(0), work).astype(np.float32),
                nconv=fourier_resample(res.density.sum(0), work).astype(np.float32),
                strain=strain_of(system.cell, ref / BOHR_IN_ANGSTROM))


def _save_dataset(out_file, rows):
    np.savez_compressed(out_file, n0=np.stack([r["n0"] for r in rows]), nconv=np.stack([r["nconv"] for r in rows]),
                        strain=np.stack([r["strain"] for r in rows]), seeds=np.array([r["seed"] for r in rows]),
                        iterations=np.array([r["iterations"] for r in rows]),
                        seconds=np.array([r["seconds"] for r in rows]))


def _generate_rows(seeds, kw):
    pseudo = _pseudo()
    rows = []
    for s in seeds:
        r = run_cell(s, pseudo, **kw)
        rows.append(r)
        print(f"cell {s}: grid {r['grid']} {r['iterations']} iterations {r['seconds']:.1f} s", flush=True)
    return rows


def _shards(seeds, workers):
    return [list(seeds[i::workers]) for i in range(workers) if seeds[i::workers]]


def _pool_map(fn, shards, kw):
    """fn(shard, kw) for every shard, each in its own spawned process (one CUDA context each,
    all on the current device: the cells are small, so several SCFs share the GPU)."""
    import multiprocessing as mp
    with mp.get_context("spawn").Pool(len(shards)) as pool:
        return pool.starmap(fn, [(s, kw) for s in shards])


def generate(seeds, out_file, workers=1, **kw):
    """Converge every seed's cell; write the (n0, strain) -> n_conv samples to out_file in
    seed order. ``workers`` > 1 runs that many processes over interleaved seed shards."""
    seeds = list(seeds)
    if workers > 1:
        rows = [r for part in _pool_map(_generate_rows, _shards(seeds, workers), kw) for r in part]
    else:
        rows = _generate_rows(seeds, kw)
    rows.sort(key=lambda r: seeds.index(r["seed"]))
    _save_dataset(out_file, rows)
    return rows


def samples(data):
    from .learned import network_input
    x = np.stack([network_input(np.maximum(n0, 1e-12), st) for n0, st in zip(data["n0"], data["strain"])])
    t = np.log(np.maximum(data["nconv"], 1e-12) / np.maximum(data["n0"], 1e-12))[:, None].astype(np.float32)
    return x, t


def fit(dataset, weights_out, epochs=200, seed=0, lr=2e-3, init=None):
    from .learned import DensityNet, train
    data = np.load(dataset)
    x, t = samples(data)
    net = DensityNet.from_file(init) if init else DensityNet(seed=seed)
    hist = train(net, x, t, epochs=epochs, lr=lr, log=lambda m: print(m, flush=True))
    net.save(weights_out)
    return hist


def learned_start(weights, family: str):
    from .learned import DensityNet, LearnedStart
    net = DensityNet.from_file(weights)
    return LearnedStart(net, reference_cell(family) / BOHR_IN_ANGSTROM, grid=FAMILIES[family]["grid"])


def _evaluate_rows(seeds, kw):
    kw = dict(kw)
    return evaluate(kw.pop("weights"), seeds, **kw)


def evaluate(weights, seeds, *, family="si8", workers=1, **kw):
    """Converge every held-out cell from the superposition and from the network's start.
    ``workers`` > 1 runs that many processes over interleaved seed shards; the rows come
    back in seed order."""
    seeds = list(seeds)
    if workers > 1:
        parts = _pool_map(_evaluate_rows, _shards(seeds, workers), dict(kw, weights=str(weights), family=family))
        return sorted((r for part in parts for r in part), key=lambda r: seeds.index(r["seed"]))
    pseudo = _pseudo()
    learned = learned_start(weights, family)
    rows = []
    for s in seeds:
        base = run_cell(s, pseudo, family=family, **kw)
        pred = run_cell(s, pseudo, family=family, density=learned.predict, **kw)
        rows.append(dict(seed=s, iterations_superposition=base["iterations"], iterations_learned=pred["iterations"],
                         seconds_superposition=base["seconds"], seconds_learned=pred["seconds"],
                         energy_difference=abs(base["free_energy"] - pred["free_energy"]),
                         fallback=learned.stats.get("fallback", False)))
        print(json.dumps(rows[-1]), flush=True)
    return rows


def summarize(rows) -> dict:
    return dict(cells=len(rows),
                mean_iterations_superposition=float(np.mean([r["iterations_superposition"] for r in rows])),
                mean_iterations_learned=float(np.mean([r["iterations_learned"] for r in rows])),
                mean_seconds_superposition=float(np.mean([r["seconds_superposition"] for r in rows])),
                mean_seconds_learned=float(np.mean([r["seconds_learned"] for r in rows])),
                max_energy_difference=float(np.max([r["energy_difference"] for r in rows])),
                rows=rows)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("stage", choices=["generate", "fit", "evaluate", "all"])
    ap.add_argument("--family", choices=sorted(FAMILIES), default="si8")
    ap.add_argument("--train", type=int, default=48)
    ap.add_argument("--test", type=int, default=12)
    ap.add_argument("--epochs", type=int, default=200)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--init", default=None, help="start the fit from these weights")
    ap.add_argument("--out", default="learned_out")
    ap.add_argument("--workers", type=int, default=1, help="processes converging cells side by side")
    args = ap.parse_args()
    out = Path(args.out)
    out.mkdir(parents=True, exist_ok=True)
    train_seeds = list(range(1000, 1000 + args.train))
    test_seeds = list(range(5000, 5000 + args.test))
    if args.stage in ("generate", "all"):
        generate(train_seeds, out / "dataset.npz", workers=args.workers, family=args.family)
    if args.stage in ("fit", "all"):
        fit(out / "dataset.npz", out / "density_net.npz", epochs=args.epochs, lr=args.lr, init=args.init)
    if args.stage in ("evaluate", "all"):
        summary = summarize(evaluate(out / "density_net.npz", test_seeds, family=args.family, workers=args.workers))
        summary["family"] = args.family
        (out / "evaluation.json").write_text(json.dumps(summary, indent=1))
        print(json.dumps({k: v for k, v in summary.items() if k != "rows"}), flush=True)


if __name__ == "__main__":
    main()
