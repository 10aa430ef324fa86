"""Run-time choice of the H.psi kernel variants by timing them on the caller's shapes.

The engine compiles several variants of the x-transform stage ("stage B": shared-memory
slabs; register-resident x columns for short x lines; register-resident with the spheres'
x-plane set fixed at compile time, for the benchmark grid; register-resident with two
threads per column, for even x lengths up to 108; shared-memory slabs split in two along z,
for the long lines of a 108^3 grid), two variants of the stages around it
(y transforms in shared memory or in registers with four lanes per column) and two paths
for the complex64 nonlocal products (tcgen05 split-TF32 GEMMs or SIMT GEMMs). Which is
fastest depends on the grid, the band count and the number of k-points of a call.
``autotune_hpsi`` times every stage combination on the caller's Hamiltonian and block shape
(CUDA events on the current stream after one warm-up call each), and the SIMT nonlocal
alternative only with the fastest stage pair, the two parts' times being additive; it
leaves the engine set to the fastest and returns the measurements. Results are cached per
(precision, nbands, k-point range) on the engine. All variants compute the same H.psi (``tests/test_autotune_gpu.py``).
"""
from __future__ import annotations

import torch

from .engine import TORCH_DTYPE, precision_code


def _variants(eng, prec_code):
    """Stage B variants the engine has for this precision (probe by selecting them)."""
    out = []
    for v in (0, 1, 2, 3, 4):
        try:
            eng.set_stage_b_variant(prec_code, v)
            out.append(v)
        except NotImplementedError:
            pass
    return out


def _ac_variants(eng, prec_code):
    """complex64 stage A/C variants the engine has (complex128 has only the first)."""
    if prec_code != 0:
        return [0]
    out = []
    for v in (0, 1):
        try:
            eng.set_stage_ac_variant(v)
            out.append(v)
        except NotImplementedError:
            pass
    return out


def autotune_hpsi(H, nbands: int, *, k_first: int = 0, k_count: int | None = None, reps: int = 3,
                  force: bool = False) -> dict:
    """Time the stage B variants x stage A/C variants x nonlocal paths for ``H.apply_all`` on
    blocks of ``nbands`` bands at k-points k_first .. k_first + k_count - 1, select the fastest
    on H's engine and return ``{"stage_b": v, "stage_ac": a, "nonlocal_tc": bool, "ms": {...}}``."""
    eng = H.engine
    prec = precision_code(H.precision)
    k_count = eng.nk - k_first if k_count is None else k_count
    key = (prec, nbands, k_first, k_count)
    cache = getattr(eng, "_autotune", None)
    if cache is None:
        cache = eng._autotune = {}
    if key in cache and not force:
        choice = cache[key]
        eng.set_stage_b_variant(prec, choice["stage_b"])
        if prec == 0:
            eng.set_stage_ac_variant(choice["stage_ac"])
        eng.set_tensor_core_nonlocal(choice["nonlocal_tc"])
        return choice
    n = int(eng.pw_off[k_first + k_count] - eng.pw_off[k_first]) * nbands
    g = torch.Generator(device=eng.device).manual_seed(7)
    psi = torch.randn(n, dtype=TORCH_DTYPE[prec], device=eng.device, generator=g)
    out = torch.empty_like(psi)
    times = {}
    stream = torch.cuda.current_stream(eng.device)

    def time_call(v, a, tc):
        eng.set_stage_b_variant(prec, v)
        if prec == 0:
            eng.set_stage_ac_variant(a)
        eng.set_tensor_core_nonlocal(tc)
        H.apply_all(psi, nbands, k_first=k_first, k_count=k_count, out=out)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            H.apply_all(psi, nbands, k_first=k_first, k_count=k_count, out=out)
        e1.record(stream)
        torch.cuda.synchronize(eng.device)
        times[(v, a, tc)] = e0.elapsed_time(e1) / reps

    # The FFT stages and the nonlocal products are separate launches in stream order, so
    # their times add: time every stage pair with the tensor-core products, then the SIMT
    # products only with the fastest stage pair.
    for v in _variants(eng, prec):
        for a in _ac_variants(eng, prec):
            time_call(v, a, True)
    if prec == 0 and eng.nproj > 0:
        v, a, _ = min(times, key=times.get)
        time_call(v, a, False)
    best = min(times, key=times.get)
    eng.set_stage_b_variant(prec, best[0])
    if prec == 0:
        eng.set_stage_ac_variant(best[1])
    eng.set_tensor_core_nonlocal(best[2])
    choice = {"stage_b": best[0], "stage_ac": best[1], "nonlocal_tc": best[2],
              "ms": {f"stage_b={v},stage_ac={a},nonlocal_tc={int(tc)}": ms for (v, a, tc), ms in times.items()}}
    cache[key] = choice
    return choice
