#!/usr/bin/env python
"""H.psi throughput (bands/s) of the B200 plane-wave engine on the Si64 workload.

Workload (one step): H.psi for 160 bands at each of 4 k-points (Gamma + 3 seeded random
k) of the 64-atom simple-cubic Si supercell (a = 10.86 A, synthetic analytic
norm-conserving dataset, ecut 40 Ry, 84^3 grid, ~37k plane waves, 256 projectors), all
four k-points in one batched call, psi and V_eff resident in HBM. psi is
orthonormalised seeded N(0,1)/(1+|k+G|^2/2) noise; V_eff is built from the superposed
atomic density. The per-step working set (~1.7 GB) exceeds L2, so no flush is needed.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line (rank 0). `--impl reference` times the CPU oracle (a numpy/scipy
FP64 restatement of the reference's Hamiltonian.apply) on the host cores instead.
Under torchrun each rank runs the same workload on its own GPU (k-point sets are
independent; no collective on the data path) and the value is the total over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO))

WORKLOAD = "si64_hpsi"
# DRAM bytes of one complex64 all-k call, measured by ncu (sum over the call's kernels of
# dram__bytes_read.sum + dram__bytes_write.sum on the one-k case, times 4 k-points)
TRAFFIC_PER_CALL = 9.73e9
METRIC = "Hpsi bands/s (Si64 40 Ry 84^3, 4 k x 160 bands)"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--precision", choices=["complex64", "complex128"], default="complex64")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--kpoints", type=int, default=4, help="k-points of the workload to include (profiling)")
    ap.add_argument("--no-extras", action="store_true", help="skip the e2e and complex128 legs (profiling)")
    ap.add_argument("--no-autotune", action="store_true", help="keep the engine's default kernel variants")
    ap.add_argument("--scf", action="store_true",
                    help="also time the Si215 Gamma SCF (plain FP64, mixed, learned+mixed; several minutes)")
    return ap.parse_args()


def build_system_for_bench(kpoints: int = 4):
    from amaterasu_b200 import kpoints as kp
    from amaterasu_b200.cells import workload
    from amaterasu_b200.pseudo import read_upf, write_synthetic_upf
    from amaterasu_b200.system import build_system
    with tempfile.TemporaryDirectory() as tmp:
        pseudo = read_upf(write_synthetic_upf(Path(tmp) / "Si.upf"))
    structure, ecut, kset, nbands = workload(WORKLOAD)
    if kpoints < len(kset):
        kset = kp.explicit(kset.points[:kpoints])
    system = build_system(structure, {"Si": pseudo}, ecut, 4 * ecut, kpoints=kset, nbands=nbands)
    return system, nbands


def orthonormal_bands(npw, nbands, kinetic, seed):
    """random_bands of the reference (scf/eigen/subspace.py:79-88): damped noise,
    Cholesky-orthonormalised."""
    import scipy.linalg as sla
    rng = np.random.default_rng(seed)
    block = (rng.normal(size=(nbands, npw)) + 1j * rng.normal(size=(nbands, npw))) / (1.0 + kinetic)
    factor = sla.cholesky(block @ block.conj().T, lower=True)
    return sla.solve_triangular(factor, block, lower=True)


def algorithmic_bytes(system, nbands, itemsize):
    """Per all-k H.psi launch: per band 2*npw*s + 4*N*s, per launch N*4 (V) and
    nproj*npw*s per k (projectors)."""
    N = int(np.prod(system.grid.shape))
    nproj = len(system.projectors[0])
    total = 0
    for w in system.wave_spheres:
        npw = len(w)
        total += nbands * (2 * npw * itemsize + 4 * N * itemsize) + nproj * npw * itemsize
    return total + N * 4


class ClockSampler:
    """SM clock and throttle reasons during the timed region: one `nvidia-smi -lms 200`
    process started (and seen to answer) before the region, stopped after it. A fresh
    nvidia-smi per sample initialises NVML each time, which was seen to stall the GPU for
    tens of milliseconds inside short timed regions."""

    def __init__(self, index):
        self.index = index
        self.lines = []
        self._proc = None
        self._t = None

    def start(self, wait_s: float = 5.0):
        q = ("--query-gpu=clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self._proc = subprocess.Popen(["nvidia-smi", q, "--format=csv,noheader,nounits", "-i", str(self.index),
                                           "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                                          text=True)
        except Exception:
            self._proc = None
            return

        def reader():
            for line in self._proc.stdout:
                self.lines.append([x.strip() for x in line.strip().split(",")])
        self._t = threading.Thread(target=reader, daemon=True)
        self._t.start()
        t0 = time.time()
        while not self.lines and time.time() - t0 < wait_s and self._proc.poll() is None:
            time.sleep(0.05)

    def mark(self):
        """Index of the next sample (samples from here on are inside the timed region)."""
        return len(self.lines)

    def stop(self, first: int = 0):
        if self._proc is not None:
            time.sleep(0.25)  # at least one sample after the region
            self._proc.terminate()
            try:
                self._proc.wait(timeout=5)
            except Exception:
                self._proc.kill()
        if self._t:
            self._t.join(timeout=5)
        samples = self.lines[max(0, first - 1):] or self.lines
        if not samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in samples if len(s) >= 6 and s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in samples if len(s) >= 6 and s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in samples if len(s) >= 6
                          for i in range(4) if s[2 + i].strip() == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(samples)}


def cpu_hpsi_sample(system, veff, nbands_sample, seconds, threads):
    """Time the oracle's FP64 H.psi on a bounded sample of the workload: blocks of
    `nbands_sample` bands cycling over the k-points until `seconds` have passed."""
    from threadpoolctl import threadpool_limits
    from oracle.hamiltonian import hamiltonian_apply
    blocks = []
    for ik, w in enumerate(system.wave_spheres):
        rng = np.random.default_rng(1000 + ik)
        psi = (rng.normal(size=(nbands_sample, len(w))) + 1j * rng.normal(size=(nbands_sample, len(w))))
        blocks.append(psi / (1.0 + w.kinetic_energy))
    done = 0
    t0 = time.perf_counter()
    with threadpool_limits(limits=threads):
        while True:
            for ik, w in enumerate(system.wave_spheres):
                p = system.projectors[ik]
                hamiltonian_apply(blocks[ik], w.miller, system.grid.shape, w.kinetic_energy, veff,
                                  p.matrix, p.dij, workers=threads)
                done += nbands_sample
            if time.perf_counter() - t0 > seconds:
                break
    elapsed = time.perf_counter() - t0
    return done / elapsed, done, elapsed


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from oracle.potential import hartree, xc_on_grid
    system, nbands = build_system_for_bench()
    rho0 = system.initial_density()
    sph = system.density_sphere
    _, v_h = hartree(rho0[0], system.grid.shape, sph.miller, sph.g2, system.grid.volume)
    _, v_xc = xc_on_grid(rho0, system.grid.cell_volume_per_point)
    veff = system.v_local + v_h + v_xc[0]
    threads = os.cpu_count() or 1
    per_step = []
    sample_bands = 8
    for step in range(args.warmup + args.steps):
        rate, done, elapsed = cpu_hpsi_sample(system, veff, sample_bands, 0.0, threads)
        if step >= args.warmup:
            per_step.append((done, elapsed))
    done = sum(d for d, _ in per_step)
    elapsed = sum(e for _, e in per_step)
    value = done / elapsed
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "bands/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * elapsed / max(args.steps, 1), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "complex128", "data": "synthetic",
        "config": {"workload": WORKLOAD, "cell": "Si64 sc a=10.86 A", "ecut_ry": 40,
                   "grid": list(system.grid.shape), "kpoints": 4, "bands_per_k": nbands,
                   "sample": f"{sample_bands} bands at each of the 4 k-points per step"},
        "cpu_baseline": {"value": value, "unit": "bands/s", "cores": threads, "kind": "port",
                         "sample": f"{sample_bands} bands x 4 k per step, oracle FP64 H.psi, "
                                   f"scipy.fft workers={threads}, BLAS threads={threads}"},
        "e2e": {"value": value, "unit": "bands/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))

    from amaterasu_b200.engine import engine_for
    from amaterasu_b200.hamiltonian import Hamiltonian
    from amaterasu_b200.potential import effective_potential

    system, nbands = build_system_for_bench(args.kpoints)
    nk = len(system.wave_spheres)
    veff, _, _ = effective_potential(system, system.initial_density())
    prec = args.precision
    cdtype = torch.complex64 if prec == "complex64" else torch.complex128
    itemsize = 8 if prec == "complex64" else 16
    H = Hamiltonian(system, veff, precision=prec)
    eng = engine_for(system)
    blocks = [orthonormal_bands(len(w), nbands, w.kinetic_energy, 12345 + ik)
              for ik, w in enumerate(system.wave_spheres)]
    host = np.concatenate([b.ravel() for b in blocks]).astype(np.complex64 if prec == "complex64"
                                                              else np.complex128)
    psi = torch.from_numpy(host).cuda().to(cdtype)
    out = torch.empty_like(psi)
    eng.reserve(prec, nk * nbands)
    stream = torch.cuda.current_stream()

    # kernel variants chosen by timing them on this workload (amaterasu_b200.autotune)
    from amaterasu_b200.autotune import autotune_hpsi
    tuned = {"stage_b": "default", "nonlocal_tc": True} if args.no_autotune else autotune_hpsi(H, nbands)

    def step():
        H.apply_all(psi, nbands, out=out)

    for _ in range(max(args.warmup, 3)):
        step()
    torch.cuda.synchronize()

    sampler = ClockSampler(local)
    sampler.start()
    first_sample = sampler.mark()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for _ in range(args.steps):
        step()
    stop.record(stream)
    torch.cuda.synchronize()
    ms = start.elapsed_time(stop)

    # end-to-end through the public API: pinned host psi -> H.psi -> pinned host, the
    # per-k copies overlapped with the compute (Hamiltonian.apply_host)
    e2e_ms = float("nan")
    if not args.no_extras:
        pinned_in = torch.from_numpy(host).pin_memory()
        pinned_out = torch.empty_like(pinned_in).pin_memory()
        dev_in = torch.empty_like(psi)
        for _ in range(2):
            H.apply_host(pinned_in, pinned_out, nbands, dev_in=dev_in, dev_out=out)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            H.apply_host(pinned_in, pinned_out, nbands, dev_in=dev_in, dev_out=out)
        e1.record(stream)
        torch.cuda.synchronize()
        e2e_ms = e0.elapsed_time(e1)
    clocks = sampler.stop(first_sample)

    t = torch.tensor([ms, e2e_ms], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms, e2e_ms = float(t[0]), float(t[1])
    bands_step = nk * nbands
    value = world * bands_step * args.steps / (ms / 1e3)
    e2e_value = world * bands_step * args.steps / (e2e_ms / 1e3)

    # second precision for the record (same workload, complex128)
    extra = {}
    if prec == "complex64" and not args.no_extras:
        H2 = Hamiltonian(system, veff, precision="complex128")
        psi2 = torch.from_numpy(np.concatenate([b.ravel() for b in blocks])).cuda()
        out2 = torch.empty_like(psi2)
        for _ in range(3):
            H2.apply_all(psi2, nbands, out=out2)
        torch.cuda.synchronize()
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        n2 = max(3, args.steps // 2)
        a0.record(stream)
        for _ in range(n2):
            H2.apply_all(psi2, nbands, out=out2)
        a1.record(stream)
        torch.cuda.synchronize()
        ms2 = a0.elapsed_time(a1) / n2
        peak_c128 = algorithmic_bytes(system, nbands, 16) / (ms2 / 1e3) / 1e9
        extra["complex128"] = {"value": bands_step / (ms2 / 1e3), "unit": "bands/s",
                               "ms_per_step": ms2, "achieved_gbs": peak_c128}
        del H2, psi2, out2

    peaks = {}
    try:
        peaks = json.loads((REPO / "MEASURED_PEAKS.json").read_text())
    except Exception:
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    per_launch_s = ms / 1e3 / args.steps
    alg = algorithmic_bytes(system, nbands, itemsize)
    achieved = alg / per_launch_s / 1e9
    line = {
        "metric": METRIC, "value": value, "unit": "bands/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "c64" if prec == "complex64" else "c128",
        "data": "synthetic",
        "config": {"workload": WORKLOAD, "cell": "Si64 sc a=10.86 A, synthetic NC dataset",
                   "ecut_ry": 40, "grid": list(system.grid.shape),
                   "npw": [len(w) for w in system.wave_spheres], "nproj": len(system.projectors[0]),
                   "kpoints": nk, "bands_per_k": nbands, "batched": "all k in one call",
                   "l2": "working set > L2 (no flush)", "parallelism": f"replicas x{world}",
                   "autotune": {"stage_b": tuned["stage_b"], "nonlocal_tc": tuned["nonlocal_tc"]}},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak,
                     "traffic": TRAFFIC_PER_CALL if (prec == "complex64" and nk == 4 and nbands == 160) else None,
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of the call's 7 kernels, "
                                       "one-k capture x 4 (profiles/hpsi_si64_c64_kernels.md)",
                     "what": "whole H.psi call (stages A/B/C + projector GEMMs), algorithmic bytes",
                     "peak_source": "MEASURED_PEAKS.json hbm_gbs" if peaks else "fallback"},
        "e2e": {"value": e2e_value, "unit": "bands/s",
                "h2d_bytes_per_step": int(host.nbytes), "d2h_bytes_per_step": int(host.nbytes)},
        # per call: stages A, B, C + (complex64, tensor cores) psi split, project, reduce, apply
        # or (SIMT) project, its split-K reduce, apply
        "gpu_launches": args.steps * (7 if (prec == "complex64" and tuned["nonlocal_tc"]) else 6),
        "clocks": clocks,
        **extra,
    }
    if args.scf and world == 1:
        from amaterasu_b200.scf_benchmark import run as scf_run
        weights = REPO / "amaterasu_b200" / "data" / "density_net_si64.npz"
        line["scf"] = scf_run("si215_gamma", str(weights) if weights.exists() else None, forces=True,
                              log=lambda *_: None)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle.potential import hartree, xc_on_grid  # noqa: F401
        veff_np = veff[0].cpu().numpy()
        rate, done, elapsed = cpu_hpsi_sample(system, veff_np, 4, 10.0, 1)
        line["cpu_baseline"] = {"value": rate, "unit": "bands/s", "cores": 1, "kind": "port",
                                "sample": f"{done} bands (4-band blocks cycling over the 4 k-points, "
                                          f"{elapsed:.1f} s), oracle FP64 H.psi, scipy.fft workers=1, BLAS 1 thread"}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
