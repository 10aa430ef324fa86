"""Throughput of the Davidson subspace products at the Si215 shape.

    python -m amaterasu_b200.subspace_benchmark [--reps 3] [--m 1320] [--npw 80797]

One k-point with npw plane waves (Si215 at 30 Ry: 80,797), a basis of m = 3 x 440 rows
(a Davidson subspace three blocks deep) and its H image:

* NC  P = B HB^H (m x m, reduction over the plane waves: Gram / Rayleigh-Ritz),
* NN  X = R B   (440 x npw, reduction over the m basis rows: rotation),

through ``ama_kbatch_zgemm`` (SIMT, complex128 and complex64) and
``ama_kbatch_zgemm_tc`` (tensor cores, complex64). Prints ms per product and the complex
flop rate 8 m n k / t, CUDA-event timed after one warm-up call.
"""
from __future__ import annotations

import argparse
import ctypes as ct

import numpy as np
import torch

from ._lib import AMA_C64, AMA_C128, AmaKOperand, call, load


def _cx(v):
    return (ct.c_double * 2)(float(np.real(v)), float(np.imag(v)))


def _op(t, rows_per_k=0, ragged=True, ld=0, kstride=0):
    return AmaKOperand(ct.c_void_p(t.data_ptr()), rows_per_k, 0, 1 if ragged else 0, ld, kstride)


def run(m=1320, npw=80797, nrot=440, reps=3, log=print):
    load()
    npw_t = torch.tensor([npw], dtype=torch.int32, device="cuda")
    off = torch.tensor([0], dtype=torch.int64, device="cuda")
    stream = ct.c_void_p(torch.cuda.current_stream().cuda_stream)
    p_npw, p_off = ct.c_void_p(npw_t.data_ptr()), ct.c_void_p(off.data_ptr())
    results = []
    for dtype, prec, tc in ((torch.complex128, AMA_C128, False), (torch.complex64, AMA_C64, False),
                            (torch.complex64, AMA_C64, True)):
        g = torch.Generator(device="cuda").manual_seed(1)
        basis = torch.randn(m * npw, dtype=dtype, device="cuda", generator=g)
        hbasis = torch.randn(m * npw, dtype=dtype, device="cuda", generator=g)
        p = torch.zeros((1, m, m), dtype=dtype, device="cuda")
        rot = torch.randn((1, nrot, m), dtype=dtype, device="cuda", generator=g)
        x = torch.zeros(nrot * npw, dtype=dtype, device="cuda")

        def nc():
            a, b, c = _op(basis, m), _op(hbasis, m), _op(p, ragged=False, ld=m, kstride=m * m)
            if tc:
                call("ama_kbatch_zgemm_tc", 1, 1, m, m, -1, p_npw, p_off, ct.byref(a), ct.byref(b), ct.byref(c),
                     _cx(1), _cx(0), npw, stream)
            else:
                call("ama_kbatch_zgemm", prec, 1, 1, m, m, -1, p_npw, p_off, ct.byref(a), ct.byref(b), ct.byref(c),
                     _cx(1), _cx(0), m, m, stream)

        def nn():
            a, b, c = _op(rot, ragged=False, ld=m, kstride=nrot * m), _op(basis, m), _op(x, nrot)
            if tc:
                call("ama_kbatch_zgemm_tc", 0, 1, nrot, -1, m, p_npw, p_off, ct.byref(a), ct.byref(b), ct.byref(c),
                     _cx(1), _cx(0), npw, stream)
            else:
                call("ama_kbatch_zgemm", prec, 0, 1, nrot, -1, m, p_npw, p_off, ct.byref(a), ct.byref(b), ct.byref(c),
                     _cx(1), _cx(0), nrot, npw, stream)

        for name, fn, flops in (("NC", nc, 8.0 * m * m * npw), ("NN", nn, 8.0 * nrot * m * npw)):
            fn()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(reps):
                fn()
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / reps
            row = dict(form=name, dtype=str(dtype).replace("torch.", ""), tensor_cores=tc, ms=ms,
                       tflops=flops / ms / 1e9)
            results.append(row)
            log(f"{row['dtype']:10s} tc={str(tc):5s} {name}: {ms:8.2f} ms {row['tflops']:8.1f} TFLOP/s")
        del basis, hbasis, p, rot, x
        torch.cuda.empty_cache()
    return results


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--m", type=int, default=1320)
    ap.add_argument("--npw", type=int, default=80797)
    ap.add_argument("--reps", type=int, default=3)
    args = ap.parse_args()
    run(args.m, args.npw, reps=args.reps)


if __name__ == "__main__":
    main()
