"""Density mixing on the GPU in FP64: Kerker preconditioning plus linear, Pulay (DIIS),
Anderson and Broyden updates, keeping the reference's API (amaterasu ``scf/mixing.py``:
``KerkerPreconditioner`` :48-105, the ``Mixer`` family :131-260, ``create_mixer`` :271-285).

Every mixer here produces the new input density in the same form,

    n_new = sum_j a_j n_in[j] + beta K( sum_j b_j r[j] ),     r[j] = n_out[j] - n_in[j],

over its stored history, so one step is: the overlap matrix of the residual combinations it
needs (``ama_vec_gram``, one pass over the history), a solve of at most history x history
numbers on the host, two combinations (``ama_vec_lincomb``), one Kerker filter (the grid
filter kernel) and one final combination. The history vectors stay on the device. Because
the Kerker filter is linear, Broyden's per-pair preconditioned input differences are folded
into one filtered combination.

Which combination each mixer takes follows the reference, as the SCF iteration counts and
fixed points are compared against it:
  * Pulay: the coefficients minimise |sum c_j r_j| with sum c_j = 1 (Pulay, Chem. Phys.
    Lett. 73, 393 (1980)): the bordered linear system with the overlaps scaled by their mean
    diagonal, dropping the oldest entry until it has a finite solution bounded by 1e4;
  * Anderson: Pulay with two history entries;
  * Broyden: Johnson's modified Broyden (Phys. Rev. B 38, 12807 (1988)) with weights 1 and
    w0 = 0.01 on the normalised residual differences.
"""
from __future__ import annotations

import ctypes as ct

import numpy as np
import torch

from ._lib import call
from .engine import ptr, stream_ptr
from .potential import grid_ops_for_grid

__all__ = ["AndersonMixer", "BroydenMixer", "KerkerPreconditioner", "LinearMixer", "Mixer", "PulayMixer",
           "create_mixer"]

_MAX_HISTORY = 16


def _dptrs(vectors):
    arr = (ct.c_void_p * len(vectors))(*[t.data_ptr() for t in vectors])
    return ct.cast(arr, ct.c_void_p), arr


def _lincomb(vectors, coefs, out=None) -> torch.Tensor:
    """out = sum_j coefs[j] vectors[j] (flat FP64 device vectors) on the grid-vector kernel."""
    v0 = vectors[0]
    out = torch.empty_like(v0) if out is None else out
    p, keep = _dptrs(vectors)
    c = (ct.c_double * len(coefs))(*[float(x) for x in coefs])
    call("ama_vec_lincomb", len(vectors), p, c, v0.numel(), ptr(out), stream_ptr())
    return out


def _gram(vectors, combos, extra=None) -> np.ndarray:
    """Overlaps of the rows of combos @ vectors (and of ``extra``), on the host."""
    ncomb = len(combos)
    nout = ncomb + (extra is not None)
    out = torch.empty(nout * nout, dtype=torch.float64, device=vectors[0].device)
    p, keep = _dptrs(vectors)
    flat = np.ascontiguousarray(np.asarray(combos, dtype=np.float64).reshape(ncomb, len(vectors)))
    c = flat.ctypes.data_as(ct.c_void_p) if ncomb else ct.cast((ct.c_double * 1)(0.0), ct.c_void_p)
    call("ama_vec_gram", len(vectors), p, ncomb, c, ptr(extra) if extra is not None else None,
         vectors[0].numel(), ptr(out), stream_ptr())
    return out.cpu().numpy().reshape(nout, nout)


class KerkerPreconditioner:
    """K r = G^2/(G^2 + q0^2) r over every grid frequency, G = 0 weighted by
    ``uniform_factor`` (0, or 1 when the total charge floats); charge channel only."""

    def __init__(self, grid, q0: float, uniform_factor: float = 0.0):
        self.ops = grid_ops_for_grid(getattr(grid, "grid", grid))
        self.q0 = q0
        self.uniform_factor = uniform_factor

    def _filter(self, field: torch.Tensor) -> torch.Tensor:
        self.ops.set_kerker(self.q0, self.uniform_factor)
        return self.ops.kerker(field).reshape(field.shape)

    def __call__(self, residual: torch.Tensor) -> torch.Tensor:
        if self.q0 <= 0:
            return residual
        if residual.shape[0] == 1:
            return self._filter(residual[0])[None]
        up, down = residual[0].reshape(-1), residual[1].reshape(-1)
        charge = self._filter(_lincomb([up, down], [1.0, 1.0]))
        moment = _lincomb([up, down], [0.5, -0.5])
        out = torch.empty_like(residual)
        _lincomb([charge, moment], [0.5, 1.0], out=out[0].reshape(-1))
        _lincomb([charge, moment], [0.5, -1.0], out=out[1].reshape(-1))
        return out


def _identity(r):
    return r


class Mixer:
    """Linear mixing n_in + beta K r, and the history store the other mixers read."""

    def __init__(self, beta: float = 0.4, history: int = 8, precondition=None):
        if history > _MAX_HISTORY:
            raise ValueError(f"mixing history of at most {_MAX_HISTORY} entries is supported")
        self.beta = beta
        self.history = history
        self.precondition = precondition or _identity
        self.inputs: list = []
        self.residuals: list = []

    def reset(self):
        self.inputs.clear()
        self.residuals.clear()

    def _record(self, n_in, n_out):
        flat_in, flat_out = n_in.reshape(-1), n_out.reshape(-1)
        self.inputs.append(_lincomb([flat_in], [1.0]))
        self.residuals.append(_lincomb([flat_out, flat_in], [1.0, -1.0]))
        while len(self.inputs) > self.history:
            del self.inputs[0]
            del self.residuals[0]

    def _combine(self, a, b, shape) -> torch.Tensor:
        """sum_j a_j inputs[j] + beta K(sum_j b_j residuals[j])."""
        base = _lincomb(self.inputs, a)
        res = _lincomb(self.residuals, b).reshape(shape)
        filtered = self.precondition(res).reshape(-1)
        return _lincomb([base, filtered], [1.0, self.beta]).reshape(shape)

    def _mix(self, n_in, n_out):
        self._record(n_in, n_out)
        h = len(self.inputs)
        last = np.zeros(h)
        last[-1] = 1.0
        return self._combine(last, last, n_in.shape)

    def __call__(self, density_in, density_out):
        as_numpy = not isinstance(density_in, torch.Tensor)
        if as_numpy:
            dev = torch.device("cuda", torch.cuda.current_device())
            density_in = torch.from_numpy(np.asarray(density_in, dtype=float)).to(dev)
            density_out = torch.from_numpy(np.asarray(density_out, dtype=float)).to(dev)
        out = self._mix(density_in.to(torch.float64).contiguous(), density_out.to(torch.float64).contiguous())
        return out.cpu().numpy() if as_numpy else out


class LinearMixer(Mixer):
    pass


class PulayMixer(Mixer):
    def _coefficients(self) -> np.ndarray:
        """DIIS weights of the stored residuals (oldest entries dropped while the bordered
        system has no acceptable solution)."""
        overlap = _gram(self.residuals, np.eye(len(self.residuals)))
        while True:
            h = len(self.residuals)
            if h == 1:
                return np.ones(1)
            s = overlap[-h:, -h:]
            bordered = np.zeros((h + 1, h + 1))
            bordered[:h, :h] = s / (np.trace(s) / h)
            bordered[:h, h] = bordered[h, :h] = 1.0
            rhs = np.zeros(h + 1)
            rhs[h] = 1.0
            try:
                sol = np.linalg.solve(bordered, rhs)[:h]
            except np.linalg.LinAlgError:
                sol = None
            if sol is not None and np.all(np.isfinite(sol)) and np.max(np.abs(sol)) < 1e4:
                return sol
            del self.inputs[0]
            del self.residuals[0]

    def _mix(self, n_in, n_out):
        self._record(n_in, n_out)
        c = self._coefficients()
        return self._combine(c, c, n_in.shape)


class AndersonMixer(PulayMixer):
    def __init__(self, beta: float = 0.4, history: int = 2, precondition=None):
        super().__init__(beta=beta, history=min(history, 2), precondition=precondition)


class BroydenMixer(Mixer):
    def __init__(self, beta: float = 0.4, history: int = 8, precondition=None, w0: float = 0.01,
                 weight: float = 1.0):
        super().__init__(beta, history, precondition)
        self.w0 = w0
        self.weight = weight

    def _mix(self, n_in, n_out):
        self._record(n_in, n_out)
        h = len(self.residuals)
        last = np.zeros(h)
        last[-1] = 1.0
        if h < 2:
            return self._combine(last, last, n_in.shape)
        steps = np.zeros((h - 1, h))  # residual differences r_{i+1} - r_i
        for i in range(h - 1):
            steps[i, i + 1], steps[i, i] = 1.0, -1.0
        g = _gram(self.residuals, steps, extra=self.residuals[-1].reshape(-1))
        norms = np.sqrt(np.maximum(np.diag(g)[:h - 1], 0.0))
        kept = [i for i in range(h - 1) if norms[i] >= 1e-30]
        if not kept:
            return self._combine(last, last, n_in.shape)
        nrm = norms[kept]
        overlap = g[np.ix_(kept, kept)] / np.outer(nrm, nrm)
        system = self.weight ** 2 * overlap + self.w0 ** 2 * np.eye(len(kept))
        rhs = self.weight * g[kept, h - 1] / nrm
        gamma = np.linalg.solve(system, rhs) * self.weight
        # n_new = n_in + beta K r - sum_i gamma_i (dn_i + beta K dr_i) / |dr_i|
        a, b = last.copy(), last.copy()
        for gi, i, ni in zip(gamma, kept, nrm):
            a -= gi / ni * steps[i]
            b -= gi / ni * steps[i]
        return self._combine(a, b, n_in.shape)


_MIXERS = {"linear": LinearMixer, "anderson": AndersonMixer, "pulay": PulayMixer, "broyden": BroydenMixer}


def create_mixer(config, grid, *, floating_charge: bool = False) -> Mixer:
    """The mixer named by ``config.algorithm`` with its Kerker preconditioner on ``grid`` (an
    FFT grid; a system is accepted for its grid)."""
    factory = _MIXERS.get(config.algorithm)
    if factory is None:
        raise ValueError(f"unknown mixing algorithm {config.algorithm!r}")
    mixer = factory(beta=config.beta, history=config.history)
    if config.preconditioner == "kerker":
        mixer.precondition = KerkerPreconditioner(grid, config.kerker_q0,
                                                  uniform_factor=1.0 if floating_charge else 0.0)
    return mixer
