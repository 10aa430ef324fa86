"""ctypes binding of ``libama.so`` (the CUDA engine's C-ABI, ``include/ama.h``).

The library is built in-tree (``amaterasu_b200/libama.so``). There is no CPU fallback:
if the library is missing, or no CUDA device is present when a kernel is called,
the call raises.
"""
from __future__ import annotations

import ctypes as ct
import os
from pathlib import Path

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "libama.so"

AMA_OK, AMA_ERR_SHAPE, AMA_ERR_CUDA, AMA_ERR_NOT_CONVERGED = 0, 1, 2, 3
AMA_ERR_TIMEOUT, AMA_ERR_NOT_SPD, AMA_ERR_ARG, AMA_ERR_UNSUPPORTED = 4, 5, 6, 7
AMA_C64, AMA_C128 = 0, 1


class AmaError(RuntimeError):
    """A CUDA-side failure reported by the engine."""


class NotConvergedError(AmaError):
    pass


class AmaKOperand(ct.Structure):
    _fields_ = [("base", ct.c_void_p), ("rows_per_k", ct.c_int64), ("row0", ct.c_int64),
                ("ragged", ct.c_int32), ("ld", ct.c_int64), ("kstride", ct.c_int64)]


class AmaSystemDesc(ct.Structure):
    _fields_ = [
        ("n1", ct.c_int32), ("n2", ct.c_int32), ("n3", ct.c_int32),
        ("nk", ct.c_int32),
        ("npw", ct.POINTER(ct.c_int32)),
        ("miller", ct.POINTER(ct.c_int32)),
        ("kinetic", ct.POINTER(ct.c_double)),
        ("nproj", ct.c_int32),
        ("projectors", ct.POINTER(ct.c_double)),
        ("dij", ct.POINTER(ct.c_double)),
        ("nspin", ct.c_int32),
        ("precisions", ct.c_uint32),
    ]


_P = ct.c_void_p
_I32, _I64, _D = ct.c_int32, ct.c_int64, ct.c_double
SIGNATURES = {
    "ama_last_error": (ct.c_char_p, []),
    "ama_version": (ct.c_int, []),
    "ama_engine_create": (ct.c_int, [ct.POINTER(AmaSystemDesc), ct.POINTER(_P)]),
    "ama_engine_destroy": (ct.c_int, [_P]),
    "ama_grid_gradient": (ct.c_int, [_P, _P, _P, ct.c_double, _P, _P]),
    "ama_grid_divergence": (ct.c_int, [_P, _P, _P, ct.c_double, ct.c_double, _P, _P]),
    "ama_xc_gga": (ct.c_int, [_P, _I32, _I32, _P, _P, _P, _P, _P]),
    "ama_davidson": (ct.c_int, [_P, _I32, _I32, _I32, _P, _D, _I32, _I32, _P, _P, _P, _P, _P]),
    "ama_davidson_graph_stats": (ct.c_int, [ct.POINTER(_I64), ct.POINTER(_I64), ct.POINTER(_I64), _I32]),
    "ama_engine_option": (ct.c_int, [_P, _I32, _I32]),
    "ama_tc_status": (ct.c_int, [_P, ct.POINTER(ct.c_int32)]),
    "ama_set_potential": (ct.c_int, [_P, _P, _I32, _P]),
    "ama_reserve": (ct.c_int, [_P, _I32, _I64]),
    "ama_hpsi": (ct.c_int, [_P, _I32, _I32, _I32, _I32, _I32, _P, _P, _P]),
    "ama_density_accumulate": (ct.c_int, [_P, _I32, _I32, _I32, _I32, _P, _P, _P, _P]),
    "ama_project": (ct.c_int, [_P, _I32, _I32, _I32, _P, _P, _P]),
    "ama_zgemm": (ct.c_int, [_I32, _I32, _I32, _I32, _I32, _P, _P, _I64, _I64, _P, _I64, _I64,
                             _P, _P, _I64, _I64, _I32, _P]),
    "ama_residual_precondition": (ct.c_int, [_I32, _I32, _I32, _P, _P, _P, _P, _P, _P, _I32, _P, _P]),
    "ama_lda_pz": (ct.c_int, [_P, _I64, _P, _P, _P]),
    "ama_kbatch_zgemm": (ct.c_int, [_I32, _I32, _I32, _I32, _I32, _I32, _P, _P, _P, _P, _P, _P, _P, _I32, _I32,
                                    _P]),
    "ama_kbatch_zgemm_tc": (ct.c_int, [_I32, _I32, _I32, _I32, _I32, _P, _P, _P, _P, _P, _P, _P, _I32, _P]),
    "ama_subspace_tc_status": (ct.c_int, [ct.POINTER(ct.c_int32)]),
    "ama_kbatch_residual": (ct.c_int, [_I32, _I32, _I32, _P, _P, _P, _P, _P, _P, _P, _P, _I32, _P, _P]),
    "ama_kbatch_copy_rows": (ct.c_int, [_I32, _I32, _I32, _P, _P, _P, _I64, _I64, _P, _I64, _I64, _P]),
    "ama_set_grid_filter": (ct.c_int, [_P, _I32, _P]),
    "ama_grid_filter": (ct.c_int, [_P, _I32, _I32, _P, _P, _P, _P]),
    "ama_grid_fft_forward": (ct.c_int, [_P, _P, _P, _P]),
    "ama_grid_filter_noalloc": (ct.c_int, [_P, _I32, _I32, _P, _P, _P, _P]),
    "ama_heev": (ct.c_int, [_I32, _P, _P, _I32, _P]),
    "ama_heev_lowest": (ct.c_int, [_I32, _I32, _P, _P, _I32, _P]),
    "ama_solver_status": (ct.c_int, [ct.POINTER(ct.c_int32)]),
    "ama_vec_gram": (ct.c_int, [_I32, _P, _I32, _P, _P, _I64, _P, _P]),
    "ama_vec_lincomb": (ct.c_int, [_I32, _P, _P, _I64, _P, _P]),
    "ama_vec_reduce": (ct.c_int, [_I32, _I64, _P, _P, _D, _I32, _P, _P]),
    "ama_density_floor": (ct.c_int, [_I32, _I64, _D, _P, _P]),
    "ama_band_kinetic": (ct.c_int, [_I32, _I32, _I32, _P, _P, _P, _P, _P, _P]),
    "ama_rowdot": (ct.c_int, [_I32, _I32, _P, _P, _P, _P]),
    "ama_ewald": (ct.c_int, [_I32, _P, _P, _P, _I32, _P, _I32, _D, _D, _D, _P, _P, _P]),
    "ama_structure_sum": (ct.c_int, [_P, _I32, _P, _P, _I32, _P, ct.c_double, _P, _P]),
    "ama_potrf_inv": (ct.c_int, [_I32, _P, _I32, _P]),
    "ama_heev_small": (ct.c_int, [_I32, _P, _P, _I32, _P]),
    "ama_conv3d_fwd_bf16": (ct.c_int, [_P, _P, _P, _P, _I32, _I32, _I32, _I32, _I32, _P]),
    "ama_conv3d_bwd_data_bf16": (ct.c_int, [_P, _P, _P, _I32, _I32, _I32, _I32, _I32, _P]),
    "ama_conv3d_bwd_weight_bf16": (ct.c_int, [_P, _P, _P, _P, _I32, _I32, _I32, _I32, _I32, _P]),
    "ama_silu_fwd_bf16": (ct.c_int, [_P, _P, _I64, _P]),
    "ama_silu_bwd": (ct.c_int, [_P, _P, _P, _I64, _P]),
    "ama_upsample2_fwd_bf16": (ct.c_int, [_P, _P, _I64, _I32, _P]),
    "ama_upsample2_bwd": (ct.c_int, [_P, _P, _I64, _I32, _P]),
}

_lib = None


def load() -> ct.CDLL:
    """Load the engine library (once); raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    path = Path(os.environ.get("AMA_LIBRARY", LIB_PATH))
    if not path.exists():
        raise ImportError(
            f"{path} is missing: build the CUDA engine with `python -m amaterasu_b200.build` "
            "(there is no CPU fallback)")
    lib = ct.CDLL(str(path))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(rc: int) -> None:
    if rc == AMA_OK:
        return
    msg = load().ama_last_error().decode(errors="replace")
    if rc == AMA_ERR_SHAPE:
        raise ValueError(msg)
    if rc == AMA_ERR_ARG:
        raise ValueError(msg)
    if rc == AMA_ERR_UNSUPPORTED:
        raise NotImplementedError(msg)
    if rc == AMA_ERR_NOT_CONVERGED:
        raise NotConvergedError(msg)
    raise AmaError(f"[{rc}] {msg}")


def call(name: str, *args) -> None:
    check(getattr(load(), name)(*args))
