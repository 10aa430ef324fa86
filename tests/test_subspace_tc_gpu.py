"""Tensor-core (split-TF32) subspace products against FP64 products of the same complex64
operands: the NC form (A B^H over the plane waves: Gram, Rayleigh-Ritz, projections) and
the NN form (small matrix times basis block: rotations, projection updates), on one
k-point with odd plane-wave counts and on ragged per-k batches.

Tolerance: max |C - C_fp64| <= 4e-6 * max |C_fp64| (the FP32 bar of the complex64 engine;
inputs are exactly representable, so the FP64 product is the reference).
"""
import ctypes as ct

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _setup(npw_list):
    from amaterasu_b200._lib import load
    load()
    npw = torch.tensor(npw_list, dtype=torch.int32, device="cuda")
    off = np.concatenate([[0], np.cumsum(npw_list)])
    pw_off = torch.tensor(off[:-1], dtype=torch.int64, device="cuda")
    return npw, pw_off, off


def _rand(shape, seed):
    g = torch.Generator(device="cpu").manual_seed(seed)
    x = torch.randn(shape + (2,), generator=g, dtype=torch.float32)
    return torch.view_as_complex(x).contiguous().cuda()


def _op(t, rows_per_k=0, row0=0, ragged=True, ld=0, kstride=0):
    from amaterasu_b200._lib import AmaKOperand
    return AmaKOperand(ct.c_void_p(t.data_ptr()), rows_per_k, row0, 1 if ragged else 0, ld, kstride)


def _status():
    from amaterasu_b200._lib import call
    code = ct.c_int32(0)
    call("ama_subspace_tc_status", ct.byref(code))
    return code.value


def _cplx(a, b):
    return (ct.c_double * 2)(float(np.real(a)), float(np.imag(a))), (ct.c_double * 2)(float(np.real(b)),
                                                                                       float(np.imag(b)))


@pytest.mark.parametrize("npw_list,m,n,row0", [([20011], 300, 200, 0), ([1000, 1237, 999], 40, 33, 3),
                                                ([80797], 130, 140, 0)])
def test_nc_matches_fp64(npw_list, m, n, row0):
    from amaterasu_b200._lib import call
    npw, pw_off, off = _setup(npw_list)
    nk = len(npw_list)
    rows_a, rows_b = m + row0, n
    a = _rand((rows_a * int(off[-1]),), 1)
    b = _rand((rows_b * int(off[-1]),), 2)
    c = torch.zeros((nk, m, n), dtype=torch.complex64, device="cuda")
    al, be = _cplx(1.0, 0.0)
    call("ama_kbatch_zgemm_tc", 1, nk, m, n, -1, ct.c_void_p(npw.data_ptr()), ct.c_void_p(pw_off.data_ptr()),
         ct.byref(_op(a, rows_a, row0)), ct.byref(_op(b, rows_b, 0)), ct.byref(_op(c, ragged=False, ld=n, kstride=m * n)),
         al, be, max(npw_list), ct.c_void_p(torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    assert _status() == 0
    for k in range(nk):
        p = int(npw_list[k])
        ak = a[rows_a * int(off[k]):rows_a * int(off[k + 1])].view(rows_a, p)[row0:row0 + m].to(torch.complex128)
        bk = b[rows_b * int(off[k]):rows_b * int(off[k + 1])].view(rows_b, p).to(torch.complex128)
        ref = ak @ bk.conj().T
        err = (c[k].to(torch.complex128) - ref).abs().max().item() / ref.abs().max().item()
        assert err < 4e-6, (k, err)


@pytest.mark.parametrize("npw_list,m,kdim,beta", [([20011], 70, 150, 0.0), ([1000, 1237, 999], 20, 45, 1.0),
                                                  ([80797], 440, 1000, 0.0)])
def test_nn_matches_fp64(npw_list, m, kdim, beta):
    from amaterasu_b200._lib import call
    npw, pw_off, off = _setup(npw_list)
    nk = len(npw_list)
    r = _rand((nk, m, kdim), 3)
    basis_rows = kdim + 2
    bas = _rand((basis_rows * int(off[-1]),), 4)
    out0 = _rand((m * int(off[-1]),), 5)
    out = out0.clone()
    alpha = -1.0 if beta else 1.0
    al, be = _cplx(alpha, beta)
    call("ama_kbatch_zgemm_tc", 0, nk, m, -1, kdim, ct.c_void_p(npw.data_ptr()), ct.c_void_p(pw_off.data_ptr()),
         ct.byref(_op(r, ragged=False, ld=kdim, kstride=m * kdim)), ct.byref(_op(bas, basis_rows, 0)),
         ct.byref(_op(out, m, 0)), al, be, max(npw_list), ct.c_void_p(torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    assert _status() == 0
    for k in range(nk):
        p = int(npw_list[k])
        bk = bas[basis_rows * int(off[k]):basis_rows * int(off[k + 1])].view(basis_rows, p)[:kdim]
        ref = alpha * (r[k].to(torch.complex128) @ bk.to(torch.complex128))
        if beta:
            ref = ref + beta * out0[m * int(off[k]):m * int(off[k + 1])].view(m, p).to(torch.complex128)
        got = out[m * int(off[k]):m * int(off[k + 1])].view(m, p).to(torch.complex128)
        err = (got - ref).abs().max().item() / ref.abs().max().item()
        assert err < 4e-6, (k, err)


def test_rejects_unsupported_shapes():
    from amaterasu_b200._lib import call
    npw, pw_off, _ = _setup([100])
    a = _rand((100 * 4,), 1)
    c = torch.zeros((4, 4), dtype=torch.complex64, device="cuda")
    al, be = _cplx(1.0, 0.0)
    with pytest.raises(ValueError):
        call("ama_kbatch_zgemm_tc", 1, 1, 4, 4, 8, ct.c_void_p(npw.data_ptr()), ct.c_void_p(pw_off.data_ptr()),
             ct.byref(_op(a, 4, 0)), ct.byref(_op(a, 4, 0)), ct.byref(_op(c, ragged=False, ld=4, kstride=16)),
             al, be, 100, ct.c_void_p(0))
    with pytest.raises(NotImplementedError):
        call("ama_kbatch_zgemm_tc", 2, 1, 4, 4, -1, ct.c_void_p(npw.data_ptr()), ct.c_void_p(pw_off.data_ptr()),
             ct.byref(_op(a, 4, 0)), ct.byref(_op(a, 4, 0)), ct.byref(_op(c, ragged=False, ld=4, kstride=16)),
             al, be, 100, ct.c_void_p(0))
