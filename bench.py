#!/usr/bin/env python
"""The B200 plane-wave engine's headline numbers: H.psi throughput (bands/s) on the Si64
workload and the Si215 SCF time of the precision policies.

H.psi (one step): H.psi for 160 bands at each of 4 k-points (Gamma + 3 seeded random k) of
the 64-atom simple-cubic Si supercell (a = 10.86 A, synthetic analytic norm-conserving
dataset, ecut 40 Ry, 84^3 grid, ~37k plane waves, 256 projectors), all four k-points in one
batched call, psi and V_eff resident in HBM. psi is orthonormalised seeded
N(0,1)/(1+|k+G|^2/2) noise; V_eff is built from the superposed atomic density. The
per-step working set (~1.7 GB) exceeds L2, so no flush is needed. After timing, a sample of
the timed call's output bands is checked against the CPU oracle's FP64 H.psi (the run fails
on a miss).

SCF (the ``scf`` block, 1 GPU): the Si215 Gamma cell (one vacancy, displaced, 30 Ry, 108^3,
440 bands) converged to |dF| < 1e-5 eV/atom by the plain FP64 engine, the mixed-precision
engine and the mixed engine from the learned start density; seconds, iterations, |dF| per
atom and the largest force difference against the plain run, clocks sampled per policy.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--no-scf]
    python bench.py --cpu-baselines      # CPU oracle on configs 1, 3 and 5 (bounded)

Prints one JSON line (rank 0). `--impl reference` times the CPU oracle (a numpy/scipy
FP64 restatement of the reference's Hamiltonian.apply) on the host cores instead, without
loading the CUDA engine. Under torchrun each rank runs the same H.psi workload on its own
GPU (k-point sets are independent; no collective on the data path) and the value is the
total over ranks.
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
METRIC = "Hpsi bands/s (Si64 40 Ry 84^3, 4 k x 160 bands)"
# ncu DRAM bytes of one all-k call, written by the profiling recipe in profiles/ together with
# a hash of the CUDA sources they were measured on; used only while the sources match
TRAFFIC_FILE = REPO / "profiles" / "hpsi_si64_traffic.json"
HPSI_SOURCES = ("common.cuh", "dft.cuh", "twiddles.h", "twiddles_line.h", "engine_impl.cuh", "engine.cu",
                "gemm.cuh", "nl_tc.cu", "tc_chain.cuh", "tc_gemm.cuh")


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
    ap.add_argument("--variants", default=None, metavar="B,AC,TC[,B128]",
                    help="force the complex64 kernel variants (stage B, stages A/C, tensor-core nonlocal 0/1; "
                         "with --config5-hpsi also the complex128 stage B) instead of timing them: profiling "
                         "runs reproduce a timed run's choice with it")
    ap.add_argument("--no-scf", action="store_true",
                    help="skip the Si215 Gamma SCF block (plain FP64, mixed, learned+mixed; ~2 minutes)")
    ap.add_argument("--density-only", action="store_true",
                    help="time only the density accumulation (profiling)")
    ap.add_argument("--config5-hpsi", action="store_true",
                    help="time only the Si215 (108^3, 440 bands) H.psi in both precisions (profiling)")
    ap.add_argument("--cpu-baselines", action="store_true",
                    help="time the CPU oracle on configs 1, 3 and 5 (bounded samples; minutes) and exit")
    return ap.parse_args()


def source_hash() -> str:
    """SHA-256 of the CUDA sources the H.psi call compiles from (what a DRAM-traffic
    measurement belongs to)."""
    import hashlib
    h = hashlib.sha256()
    for name in HPSI_SOURCES:
        p = REPO / "amaterasu_b200" / "csrc" / name
        h.update(name.encode())
        h.update(p.read_bytes())
    return h.hexdigest()[:16]


def measured_traffic(precision: str):
    """DRAM bytes per all-k call from the committed ncu summary, or None when it was taken on
    other sources."""
    try:
        rec = json.loads(TRAFFIC_FILE.read_text())
    except Exception:
        return None, "no committed ncu measurement"
    entry = rec.get(precision)
    if not entry:
        return None, "no committed ncu measurement for this precision"
    if rec.get("sources") != source_hash():
        return None, "the committed ncu measurement belongs to other CUDA sources"
    return float(entry["bytes_per_call"]), entry.get("how", "ncu")


def cpu_model() -> str:
    try:
        for line in Path("/proc/cpuinfo").read_text().splitlines():
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except Exception:
        pass
    return "unknown"


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


def check_against_oracle(system, veff_np, packed, nbands, bands=(0, 77, 159), tol=None):
    """Compare a few bands of every k-point of the timed call's output with the CPU oracle's
    FP64 H.psi of the same input (the oracle is only the checker here). Returns the largest
    relative error; raises when it is above tol."""
    from oracle.hamiltonian import hamiltonian_apply
    psi_all, out_all = packed
    worst = 0.0
    off = 0
    for ik, w in enumerate(system.wave_spheres):
        n = len(w)
        blk_in = psi_all[off:off + nbands * n].reshape(nbands, n)
        blk_out = out_all[off:off + nbands * n].reshape(nbands, n)
        off += nbands * n
        rows = [b for b in bands if b < nbands]
        p = system.projectors[ik]
        ref = hamiltonian_apply(blk_in[rows].astype(np.complex128), w.miller, system.grid.shape, w.kinetic_energy,
                                veff_np, p.matrix, p.dij)
        err = float(np.max(np.abs(blk_out[rows] - ref)) / np.max(np.abs(ref)))
        worst = max(worst, err)
    if tol is not None and not worst < tol:
        raise SystemExit(f"bench: the timed H.psi output differs from the CPU oracle by {worst:.3e} (> {tol:g})")
    return worst


def _common_config(system, nbands):
    return {"workload": WORKLOAD, "cell": "Si64 sc a=10.86 A, synthetic NC dataset", "ecut_ry": 40,
            "grid": list(system.grid.shape), "npw": [len(w) for w in system.wave_spheres],
            "nproj": len(system.projectors[0]), "kpoints": len(system.wave_spheres), "bands_per_k": nbands,
            "batched": "all k in one call", "l2": "working set > L2 (no flush)"}


def run_reference(args):
    """The reference arm: the CPU oracle's FP64 H.psi with every host thread, on a bounded
    sample of the same workload per step. The inputs are built on the host only (the engine
    library is never loaded in this process)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import amaterasu_b200.local as local_setup
    local_setup._device_structure_sum = lambda *a, **k: None  # host structure sums: no CUDA engine here
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
        "config": {**_common_config(system, nbands), "parallelism": f"replicas x{args.gpus}"},
        "cpu_baseline": {"value": value, "unit": "bands/s", "cores": threads, "kind": "port",
                         "cpu": cpu_model(),
                         "sample": f"{sample_bands} bands at each of the 4 k-points per step, oracle FP64 "
                                   f"H.psi, scipy.fft workers={threads}, BLAS threads={threads}"},
        "e2e": {"value": value, "unit": "bands/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def time_calls(fn, steps, stream):
    import torch
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1)


def hpsi_leg(system, veff, blocks, nbands, prec, steps, warmup, stream, autotune, with_e2e, peak):
    """Device-resident and host-to-host timing of the all-k H.psi call in one precision;
    returns (record, timed output as numpy, input as numpy)."""
    import torch
    from amaterasu_b200.engine import engine_for
    from amaterasu_b200.hamiltonian import Hamiltonian
    cdtype = torch.complex64 if prec == "complex64" else torch.complex128
    itemsize = 8 if prec == "complex64" else 16
    nk = len(system.wave_spheres)
    H = Hamiltonian(system, veff, precision=prec)
    eng = engine_for(system)
    host = np.concatenate([b.ravel() for b in blocks]).astype(np.complex64 if prec == "complex64" else np.complex128)
    psi = torch.from_numpy(host).cuda()
    out = torch.empty_like(psi)
    eng.reserve(prec, nk * nbands)
    if isinstance(autotune, tuple) and prec == "complex64":
        b, ac, tc = autotune
        eng.set_stage_b_variant(prec, b)
        eng.set_stage_ac_variant(ac)
        eng.set_tensor_core_nonlocal(bool(tc))
        tuned = {"stage_b": b, "stage_ac": ac, "nonlocal_tc": bool(tc), "forced": True}
    elif autotune:
        from amaterasu_b200.autotune import autotune_hpsi
        tuned = autotune_hpsi(H, nbands)
    else:
        tuned = {"stage_b": "default", "nonlocal_tc": prec == "complex64"}

    def step():
        H.apply_all(psi, nbands, out=out)

    for _ in range(max(warmup, 3)):
        step()
    torch.cuda.synchronize()
    ms = time_calls(step, steps, stream)
    out_np = out.cpu().numpy()
    e2e_ms = float("nan")
    if with_e2e:
        pinned_in = torch.from_numpy(host).pin_memory()
        pinned_out = torch.empty_like(pinned_in).pin_memory()
        dev_in = torch.empty_like(psi)
        for _ in range(2):
            H.apply_host(pinned_in, pinned_out, nbands, dev_in=dev_in, dev_out=out)
        torch.cuda.synchronize()
        e2e_ms = time_calls(lambda: H.apply_host(pinned_in, pinned_out, nbands, dev_in=dev_in, dev_out=out),
                            steps, stream)
    per_launch_s = ms / 1e3 / steps
    alg = algorithmic_bytes(system, nbands, itemsize)
    traffic, traffic_how = measured_traffic(prec)
    rec = {
        "ms": ms, "e2e_ms": e2e_ms, "tuned": tuned, "bytes": int(host.nbytes),
        "roofline": {"bound": "hbm", "achieved": alg / per_launch_s / 1e9, "peak": peak["value"], "unit": "GB/s",
                     "frac": alg / per_launch_s / 1e9 / peak["value"],
                     "achieved_on_traffic": None if traffic is None else traffic / per_launch_s / 1e9,
                     "frac_on_traffic": None if traffic is None else traffic / per_launch_s / 1e9 / peak["value"],
                     "traffic": traffic, "traffic_source": traffic_how, "algorithmic_bytes": alg,
                     "what": "whole all-k H.psi call (stages A/B/C + projector GEMMs), algorithmic bytes "
                             "(2 npw s + 4 N s per band, N*4 + nproj npw s per call)",
                     "peak_source": peak["source"]},
        # per call: stages A, B, C + (complex64, tensor cores) psi split, project, reduce, apply
        # or (SIMT / complex128) project, its split-K reduce, apply
        "launches_per_call": 7 if (prec == "complex64" and tuned["nonlocal_tc"]) else 6,
    }
    del H
    return rec, out_np, host


def density_leg(system, blocks, nbands, steps, stream, peak):
    """The occupation-weighted density accumulation (``ama_density_accumulate``) over the whole
    4 k x 160 band set, both precisions: device time and the roofline on algorithmic bytes
    (per band npw s read + 2 N s for the slot planes' write and read back, per k-point the FP64
    density read and written)."""
    import torch
    from amaterasu_b200.engine import engine_for
    eng = engine_for(system)
    nk = len(system.wave_spheres)
    N = int(np.prod(system.grid.shape))
    out = {}
    for prec, cdt, s_ in (("complex64", torch.complex64, 8), ("complex128", torch.complex128, 16)):
        psi = torch.from_numpy(np.concatenate([b.ravel() for b in blocks])).cuda().to(cdt)
        w = torch.full((nk * nbands,), 2.0 / (nk * nbands), dtype=torch.float64, device="cuda")
        rho = torch.zeros(N, dtype=torch.float64, device="cuda")
        eng.reserve(prec, nbands)

        def step():
            eng.density_accumulate(psi, w, rho, k_first=0, k_count=nk, nbands=nbands)

        for _ in range(3):
            step()
        torch.cuda.synchronize()
        ms = time_calls(step, steps, stream) / steps
        alg = sum(nbands * (len(wv) * s_ + 2 * N * s_) + 2 * N * 8 for wv in system.wave_spheres)
        out[prec] = {"ms_per_call": ms, "bands_per_s": nk * nbands / (ms / 1e3),
                     "roofline": {"bound": "hbm", "achieved": alg / (ms / 1e3) / 1e9, "peak": peak["value"],
                                  "unit": "GB/s", "frac": alg / (ms / 1e3) / 1e9 / peak["value"],
                                  "algorithmic_bytes": alg, "peak_source": peak["source"]}}
        del psi, rho
    return out


def hpsi_config5(system, peak, steps=10, variants=None):
    """H.psi of the Si215 Gamma configuration (108^3 grid, 440 bands, 80,797 plane waves)
    in both precisions on the SCF's own system: device-timed all-band calls after the
    kernel-variant autotune, with the roofline on the algorithmic bytes and the measured
    copy bandwidth."""
    import torch
    from amaterasu_b200.autotune import autotune_hpsi
    from amaterasu_b200.hamiltonian import Hamiltonian
    from amaterasu_b200.potential import effective_potential
    nb = int(system.nbands)
    veff, _, _ = effective_potential(system, system.initial_density())
    veff = veff.cpu().numpy()
    w = system.wave_spheres[0]
    rng = np.random.default_rng(5)
    block = (rng.normal(size=(nb, len(w))) + 1j * rng.normal(size=(nb, len(w)))) / (1.0 + w.kinetic_energy)
    stream = torch.cuda.current_stream()
    out = {"workload": "si215_gamma", "bands": nb, "plane_waves": len(w), "grid": list(system.grid.shape)}
    for prec, itemsize in (("complex64", 8), ("complex128", 16)):
        H = Hamiltonian(system, veff, precision=prec)
        psi = torch.from_numpy(block.astype(np.complex64 if prec == "complex64" else np.complex128).ravel()).cuda()
        res = torch.empty_like(psi)
        if variants is not None and prec == "complex64":
            H.engine.set_stage_b_variant(prec, variants[0])
            H.engine.set_stage_ac_variant(variants[1])
            H.engine.set_tensor_core_nonlocal(bool(variants[2]))
            tuned = {"stage_b": variants[0], "stage_ac": variants[1], "nonlocal_tc": bool(variants[2])}
        elif variants is not None:
            H.engine.set_stage_b_variant(prec, variants[3] if len(variants) > 3 else 0)
            tuned = {"stage_b": variants[3] if len(variants) > 3 else 0}
        else:
            tuned = autotune_hpsi(H, nb)
        for _ in range(3):
            H.apply_all(psi, nb, out=res)
        torch.cuda.synchronize()
        ms = time_calls(lambda: H.apply_all(psi, nb, out=res), steps, stream) / steps
        alg = algorithmic_bytes(system, nb, itemsize)
        achieved = alg / (ms / 1e3) / 1e9
        out[prec] = {"ms_per_call": ms, "bands_per_s": nb / (ms / 1e3),
                     "autotune": {k: tuned[k] for k in ("stage_b", "stage_ac", "nonlocal_tc") if k in tuned},
                     "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak["value"], "unit": "GB/s",
                                  "frac": achieved / peak["value"], "algorithmic_bytes": alg,
                                  "peak_source": peak["source"]}}
    return out


def scf_block(log=lambda *_: None, peak=None):
    """Si215 SCF policies with a clock record per policy, then the Si215 H.psi figures."""
    from amaterasu_b200.scf_benchmark import run as scf_run
    weights = REPO / "amaterasu_b200" / "data" / "density_net_si64.npz"
    samplers = {}

    def hook(name, phase):
        if phase == "start":
            samplers[name] = ClockSampler(0)
            samplers[name].start()
            samplers[name]._first = samplers[name].mark()
        else:
            samplers[name] = samplers[name].stop(samplers[name]._first)

    after = (lambda system: hpsi_config5(system, peak)) if peak is not None else None
    out = scf_run("si215_gamma", str(weights) if weights.exists() else None, forces=True, log=log, hook=hook,
                  after=after, policies=("plain", "mixed", "learned+mixed", "mixed_ref_schedule"))
    if "after" in out:
        out["hpsi_config5"] = out.pop("after")
    for name, row in out["runs"].items():
        row["clocks"] = samplers.get(name)
    plain, best = out["runs"].get("plain"), out["runs"].get("learned+mixed") or out["runs"].get("mixed")
    out["target"] = "learned+mixed at least 3x faster than plain FP64 to |dF| < 1e-5 eV/atom, forces within 1e-4 eV/A"
    if plain and best:
        out["speedup_learned_mixed_vs_plain"] = plain["seconds"] / out["runs"]["learned+mixed"]["seconds"] \
            if "learned+mixed" in out["runs"] else None
        out["speedup_mixed_vs_plain"] = plain["seconds"] / out["runs"]["mixed"]["seconds"]
    return out


def main():
    args = parse()
    if args.cpu_baselines:
        run_cpu_baselines()
        return
    if args.impl == "reference":
        run_reference(args)
        return
    import torch
    import torch.distributed as dist

    if args.config5_hpsi:  # profiling: the Si215 H.psi legs alone
        from amaterasu_b200.scf_benchmark import _system
        peaks = json.loads((REPO / "MEASURED_PEAKS.json").read_text()) if (REPO / "MEASURED_PEAKS.json").exists() else {}
        peak = {"value": float(peaks.get("hbm_gbs", 6650.0)),
                "source": "MEASURED_PEAKS.json hbm_gbs (measured)" if "hbm_gbs" in peaks else "fallback 6650 GB/s"}
        variants = tuple(int(x) for x in args.variants.split(",")) if args.variants else None
        print(json.dumps(hpsi_config5(_system("si215_gamma"), peak, steps=args.steps, variants=variants)), flush=True)
        return

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))

    from amaterasu_b200.potential import effective_potential

    system, nbands = build_system_for_bench(args.kpoints)
    nk = len(system.wave_spheres)
    veff, _, _ = effective_potential(system, system.initial_density())
    blocks = [orthonormal_bands(len(w), nbands, w.kinetic_energy, 12345 + ik)
              for ik, w in enumerate(system.wave_spheres)]
    stream = torch.cuda.current_stream()
    peaks = {}
    try:
        peaks = json.loads((REPO / "MEASURED_PEAKS.json").read_text())
    except Exception:
        pass
    peak = {"value": float(peaks.get("hbm_gbs", 6650.0)),
            "source": "MEASURED_PEAKS.json hbm_gbs (measured)" if "hbm_gbs" in peaks else "fallback 6650 GB/s"}
    prec = args.precision
    if args.density_only:
        print(json.dumps({"density": density_leg(system, blocks, nbands, args.steps, stream, peak)}), flush=True)
        return

    sampler = ClockSampler(local)
    sampler.start()
    first_sample = sampler.mark()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    tune = tuple(int(x) for x in args.variants.split(",")) if args.variants else not args.no_autotune
    main_rec, out_np, host = hpsi_leg(system, veff, blocks, nbands, prec, args.steps, args.warmup, stream,
                                      tune, not args.no_extras, peak)
    clocks = sampler.stop(first_sample)

    t = torch.tensor([main_rec["ms"], main_rec["e2e_ms"]], dtype=torch.float64, device="cuda")
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms, e2e_ms = float(t[0]), float(t[1])
    bands_step = nk * nbands
    value = world * bands_step * args.steps / (ms / 1e3)
    e2e_value = world * bands_step * args.steps / (e2e_ms / 1e3)

    veff_np = veff[0].cpu().numpy()
    parity = check_against_oracle(system, veff_np, (host, out_np), nbands,
                                  tol=2e-5 if prec == "complex64" else 1e-11)

    extra = {}
    if prec == "complex64" and not args.no_extras:  # the plain FP64 engine's H.psi on the same workload
        rec2, out2, host2 = hpsi_leg(system, veff, blocks, nbands, "complex128", max(3, args.steps // 2),
                                     args.warmup, stream, False, True, peak)
        n2 = max(3, args.steps // 2)
        parity2 = check_against_oracle(system, veff_np, (host2, out2), nbands, tol=1e-11)
        extra["complex128"] = {
            "value": bands_step / (rec2["ms"] / 1e3 / n2), "unit": "bands/s", "ms_per_step": rec2["ms"] / n2,
            "steps": n2, "roofline": rec2["roofline"],
            "e2e": {"value": bands_step * n2 / (rec2["e2e_ms"] / 1e3), "unit": "bands/s",
                    "h2d_bytes_per_step": rec2["bytes"], "d2h_bytes_per_step": rec2["bytes"]},
            "oracle_max_rel_err": parity2, "oracle_tolerance": 1e-11}
        del out2, host2

    line = {
        "metric": METRIC, "value": value, "unit": "bands/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "c64" if prec == "complex64" else "c128",
        "data": "synthetic",
        "config": {**_common_config(system, nbands), "parallelism": f"replicas x{world}"},
        "autotune": {k: main_rec["tuned"][k] for k in ("stage_b", "stage_ac", "nonlocal_tc") if k in main_rec["tuned"]},
        "roofline": main_rec["roofline"],
        "e2e": {"value": e2e_value, "unit": "bands/s",
                "h2d_bytes_per_step": main_rec["bytes"], "d2h_bytes_per_step": main_rec["bytes"]},
        "gpu_launches": args.steps * main_rec["launches_per_call"],
        "clocks": clocks,
        "parity": {"oracle_max_rel_err": parity, "oracle_tolerance": 2e-5 if prec == "complex64" else 1e-11,
                   "checked": "bands 0, 77, 159 of every k-point of the timed call's output vs the CPU oracle"},
        **extra,
    }
    if not args.no_extras:
        line["density"] = density_leg(system, blocks, nbands, max(3, args.steps // 2), stream, peak)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        rate, done, elapsed = cpu_hpsi_sample(system, veff_np, 8, 10.0, threads)
        line["cpu_baseline"] = {"value": rate, "unit": "bands/s", "cores": threads, "kind": "port",
                                "cpu": cpu_model(),
                                "sample": f"{done} bands (8-band blocks cycling over the 4 k-points, {elapsed:.1f} s), "
                                          f"oracle FP64 H.psi, scipy.fft workers={threads}, BLAS {threads} threads"}
    if world == 1 and not args.no_scf:
        line["scf"] = scf_block(peak=peak)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def run_cpu_baselines():
    """The CPU oracle (FP64 numpy/scipy, the reference's algorithm) on configs 1, 3 and 5,
    bounded so that the whole run takes minutes; extrapolations are labelled as such.
    The engine library is not loaded."""
    import amaterasu_b200.local as local_setup
    local_setup._device_structure_sum = lambda *a, **k: None
    from oracle.eigen import davidson, random_bands
    from oracle.hamiltonian import hamiltonian_apply
    from oracle.potential import hartree, xc_on_grid
    from oracle.scf import run_scf as oracle_scf
    from amaterasu_b200.cells import workload
    from amaterasu_b200.pseudo import read_upf, write_synthetic_upf
    from amaterasu_b200.system import build_system
    with tempfile.TemporaryDirectory() as tmp:
        pseudo = read_upf(write_synthetic_upf(Path(tmp) / "Si.upf"))
    threads = os.cpu_count() or 1
    out = {"impl": "cpu-oracle", "cpu": cpu_model(), "nproc": threads,
           "note": "scipy.fft workers=1 as the reference ships; BLAS default threads"}

    def arrays(system):
        sph = system.density_sphere
        return dict(shape=system.grid.shape, volume=system.grid.volume, natoms=system.natoms,
                    nelectrons=system.nelectrons, nbands=system.nbands, weights=system.kpoints.weights,
                    spheres=[dict(miller=w.miller, kinetic=w.kinetic_energy, proj=p.matrix, dij=p.dij)
                             for w, p in zip(system.wave_spheres, system.projectors)],
                    v_local=system.v_local, rho0=system.initial_density(), ewald=0.0,  # timing only
                    density_miller=sph.miller, density_g2=sph.g2,
                    gvectors=system.grid.gvectors_cartesian())

    # config 1: full SCF
    structure, ecut, ks, nb = workload("si2_scf")
    s1 = build_system(structure, {"Si": pseudo}, ecut, 4 * ecut, kpoints=ks, nbands=nb)
    t0 = time.perf_counter()
    r1 = oracle_scf(arrays(s1), occupation_scheme="fixed", tol_energy_ev=1e-8 * 27.211386245988, tol_density=1e-8)
    out["config1_si2_scf"] = {"seconds": time.perf_counter() - t0, "iterations": r1["iterations"],
                              "what": "full SCF to 1e-8 Ha/atom and 1e-8 density (32 k, 8 bands, 25^3)"}
    print(json.dumps(out), flush=True)

    # config 3: the first SCF iteration's Davidson on 8 of the 260 k-points, extrapolated
    structure, ecut, ks, nb = workload("si8_batched")
    s3 = build_system(structure, {"Si": pseudo}, ecut, 4 * ecut, kpoints=ks, nbands=nb)
    rho0 = s3.initial_density()
    sph = s3.density_sphere
    _, v_h = hartree(rho0[0], s3.grid.shape, sph.miller, sph.g2, s3.grid.volume)
    _, v_xc = xc_on_grid(rho0, s3.grid.cell_volume_per_point)
    veff = s3.v_local + v_h + v_xc[0]
    sample = list(range(0, 260, 33))
    t0 = time.perf_counter()
    for ik in sample:
        w, p = s3.wave_spheres[ik], s3.projectors[ik]
        guess = random_bands(len(w), nb, w.kinetic_energy, seed=12345 + ik)
        davidson(lambda b: hamiltonian_apply(b, w.miller, s3.grid.shape, w.kinetic_energy, veff, p.matrix, p.dij),
                 guess, w.kinetic_energy, tolerance=1e-6, max_iterations=40)
    per_k = (time.perf_counter() - t0) / len(sample)
    out["config3_si8_260k"] = {"seconds_per_k_first_iteration": per_k, "k_sampled": len(sample),
                               "extrapolated_first_iteration_seconds": per_k * 260,
                               "what": "first SCF iteration's Davidson (tol 1e-6, <= 40 steps) on 8 of the 260 "
                                       "k-points, extrapolated x260/8 (label: extrapolated)"}
    print(json.dumps(out), flush=True)

    # config 5: H.psi of a band sample at 108^3, 440 bands; per-band cost
    structure, ecut, ks, nb = workload("si215_gamma")
    s5 = build_system(structure, {"Si": pseudo}, ecut, 4 * ecut, kpoints=ks, nbands=nb)
    rho0 = s5.initial_density()
    sph = s5.density_sphere
    _, v_h = hartree(rho0[0], s5.grid.shape, sph.miller, sph.g2, s5.grid.volume)
    _, v_xc = xc_on_grid(rho0, s5.grid.cell_volume_per_point)
    veff = s5.v_local + v_h + v_xc[0]
    w, p = s5.wave_spheres[0], s5.projectors[0]
    rng = np.random.default_rng(5)
    psi = (rng.normal(size=(8, len(w))) + 1j * rng.normal(size=(8, len(w)))) / (1.0 + w.kinetic_energy)
    t0 = time.perf_counter()
    hamiltonian_apply(psi, w.miller, s5.grid.shape, w.kinetic_energy, veff, p.matrix, p.dij)
    per_band = (time.perf_counter() - t0) / 8
    out["config5_si215"] = {"hpsi_seconds_per_band": per_band, "hpsi_bands_per_s": 1.0 / per_band,
                            "extrapolated_hpsi_440_bands_seconds": 440 * per_band,
                            "what": "oracle FP64 H.psi of 8 bands at 108^3 (80,797 plane waves, 860 projectors); "
                                    "one 440-band H.psi extrapolated (label: extrapolated)"}
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
