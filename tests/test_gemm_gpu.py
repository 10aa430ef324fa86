"""SIMT complex GEMMs (ama_zgemm, ama_kbatch_zgemm) against FP64 products of the same
operands, every form (NN, NC, CN), both precisions, odd sizes, every tile shape of the
FP64 tensor-core kernel, split-K and ragged per-k batches, with alpha/beta.

Tolerances: complex128 1e-13, complex64 2e-6 of max|C| (the FP32 sums are flushed into FP64
every 128 products, so the error does not grow with the reduction length).
"""
import ctypes as ct

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _rand(shape, seed, dtype):
    g = torch.Generator(device="cpu").manual_seed(seed)
    x = torch.view_as_complex(torch.randn(tuple(shape) + (2,), generator=g, dtype=torch.float64))
    return x.to(dtype).contiguous().cuda()


def _cx(v):
    return (ct.c_double * 2)(float(np.real(v)), float(np.imag(v)))


def _tol(dtype):
    return 1e-13 if dtype == torch.complex128 else 2e-6


@pytest.mark.parametrize("dtype", [torch.complex64, torch.complex128])
@pytest.mark.parametrize("form", [0, 1, 2])
# complex128 tile shapes: 64 x 64 (the first three and (33, 20)), 32 x 32 (m <= 32, n <= 64;
# split-K at (20, 40)), 32 x 128 (m <= 32, n > 64)
@pytest.mark.parametrize("m,n,k,batch", [(37, 53, 29, 3), (70, 65, 40000, 1), (128, 64, 600, 2), (33, 20, 50, 2),
                                         (20, 40, 4615, 5), (32, 64, 1000, 1), (1, 1, 5, 1), (17, 300, 77, 2),
                                         (32, 129, 4000, 1)])
def test_zgemm_forms(dtype, form, m, n, k, batch):
    from amaterasu_b200._lib import AMA_C64, AMA_C128, call, load
    load()
    prec = AMA_C64 if dtype == torch.complex64 else AMA_C128
    a = _rand((batch, k, m) if form == 2 else (batch, m, k), 1, dtype)
    b = _rand((batch, n, k) if form == 1 else (batch, k, n), 2, dtype)
    c0 = _rand((batch, m, n), 3, dtype)
    c = c0.clone()
    alpha, beta = 0.7 - 0.2j, 0.5 + 0.1j
    lda = a.shape[2]
    ldb = b.shape[2]
    call("ama_zgemm", prec, form, m, n, k, _cx(alpha), ct.c_void_p(a.data_ptr()), lda, a[0].numel(),
         ct.c_void_p(b.data_ptr()), ldb, b[0].numel(), _cx(beta), ct.c_void_p(c.data_ptr()), n, m * n, batch,
         ct.c_void_p(torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    A, B = a.to(torch.complex128), b.to(torch.complex128)
    if form == 1:
        B = B.conj().transpose(1, 2)
    if form == 2:
        A = A.conj().transpose(1, 2)
    ref = alpha * (A @ B) + beta * c0.to(torch.complex128)
    err = (c.to(torch.complex128) - ref).abs().max().item() / ref.abs().max().item()
    assert err < _tol(dtype), err


@pytest.mark.parametrize("dtype", [torch.complex64, torch.complex128])
def test_kbatch_ragged_nc_and_nn(dtype):
    from amaterasu_b200._lib import AMA_C64, AMA_C128, AmaKOperand, call, load
    load()
    prec = AMA_C64 if dtype == torch.complex64 else AMA_C128
    npw_list = [301, 1777, 45]
    off = np.concatenate([[0], np.cumsum(npw_list)])
    npw = torch.tensor(npw_list, dtype=torch.int32, device="cuda")
    pw_off = torch.tensor(off[:-1], dtype=torch.int64, device="cuda")
    nk, rows, m, n = 3, 12, 10, 7
    X = _rand((rows * int(off[-1]),), 4, dtype)
    Y = _rand((rows * int(off[-1]),), 5, dtype)
    G = torch.zeros((nk, m, n), dtype=dtype, device="cuda")

    def op(t, rpk=0, row0=0, ragged=True, ld=0, ks=0):
        return AmaKOperand(ct.c_void_p(t.data_ptr()), rpk, row0, 1 if ragged else 0, ld, ks)

    s = ct.c_void_p(torch.cuda.current_stream().cuda_stream)
    # NC: G[k] = X[k][2:2+m] . Y[k][:n]^H over each k's plane waves
    call("ama_kbatch_zgemm", prec, 1, nk, m, n, -1, ct.c_void_p(npw.data_ptr()), ct.c_void_p(pw_off.data_ptr()),
         ct.byref(op(X, rows, 2)), ct.byref(op(Y, rows, 0)), ct.byref(op(G, ragged=False, ld=n, ks=m * n)),
         _cx(1.0), _cx(0.0), m, n, s)
    # NN: Z[k] = R[k] (n x m) . X[k][2:2+m]  -> per-k block of n rows
    R = _rand((nk, n, m), 6, dtype)
    Z = torch.zeros((n * int(off[-1]),), dtype=dtype, device="cuda")
    call("ama_kbatch_zgemm", prec, 0, nk, n, -1, m, ct.c_void_p(npw.data_ptr()), ct.c_void_p(pw_off.data_ptr()),
         ct.byref(op(R, ragged=False, ld=m, ks=n * m)), ct.byref(op(X, rows, 2)), ct.byref(op(Z, n, 0)),
         _cx(1.0), _cx(0.0), n, max(npw_list), s)
    torch.cuda.synchronize()
    for k in range(nk):
        p = npw_list[k]
        xk = X[rows * int(off[k]):rows * int(off[k + 1])].view(rows, p).to(torch.complex128)
        yk = Y[rows * int(off[k]):rows * int(off[k + 1])].view(rows, p).to(torch.complex128)
        ref = xk[2:2 + m] @ yk[:n].conj().T
        err = (G[k].to(torch.complex128) - ref).abs().max().item() / ref.abs().max().item()
        assert err < _tol(dtype), ("NC", k, err)
        refz = R[k].to(torch.complex128) @ xk[2:2 + m]
        got = Z[n * int(off[k]):n * int(off[k + 1])].view(n, p).to(torch.complex128)
        err = (got - refz).abs().max().item() / refz.abs().max().item()
        assert err < _tol(dtype), ("NN", k, err)
