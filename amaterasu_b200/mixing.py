"""Density mixing on the GPU (FP64 vectors): Kerker preconditioning plus linear, Pulay,
Anderson and Broyden updates.

Mirrors amaterasu ``scf/mixing.py``: Kerker G^2/(G^2+q0^2) over every grid frequency,
G=0 factor 0 (or 1 with a floating charge), charge channel only (:48-105); the history
bookkeeping of ``Mixer`` (:131-160); Pulay's bordered DIIS system, scaled by the mean
diagonal and solved in FP64, dropping the oldest entry until the solution is finite and
bounded by 1e4 (:163-201); Anderson = Pulay with history 2 (:204-213); Johnson's
modified Broyden with w0 = 0.01 (:216-260). Vectors stay on the device; the Gram
matrices (at most history x history) are solved on the host.
"""
from __future__ import annotations

import numpy as np
import torch

from .potential import grid_ops

__all__ = ["AndersonMixer", "BroydenMixer", "KerkerPreconditioner", "LinearMixer", "Mixer", "PulayMixer",
           "create_mixer"]


class KerkerPreconditioner:
    def __init__(self, system, q0: float, uniform_factor: float = 0.0):
        self.ops = grid_ops(system)
        self.q0 = q0
        self.uniform_factor = uniform_factor
        if q0 > 0:
            self.ops.set_kerker(q0, uniform_factor)

    def _filter(self, field: torch.Tensor) -> torch.Tensor:
        self.ops.set_kerker(self.q0, self.uniform_factor)
        return self.ops.kerker(field).reshape(field.shape)

    def __call__(self, residual: torch.Tensor) -> torch.Tensor:
        if self.q0 <= 0:
            return residual
        if residual.shape[0] == 1:
            return self._filter(residual[0])[None]
        charge = self._filter(residual[0] + residual[1])
        moment = residual[0] - residual[1]
        return torch.stack([0.5 * (charge + moment), 0.5 * (charge - moment)])


def _identity(r):
    return r


class Mixer:
    """Linear mixing and the history store the other mixers extend."""

    def __init__(self, beta: float = 0.4, history: int = 8, precondition=None):
        self.beta = beta
        self.history = history
        self.precondition = precondition or _identity
        self.inputs: list = []
        self.residuals: list = []

    def reset(self):
        self.inputs.clear()
        self.residuals.clear()

    def _record(self, n_in, n_out):
        r = n_out - n_in
        self.inputs.append(n_in.clone())
        self.residuals.append(r)
        if len(self.inputs) > self.history:
            del self.inputs[0]
            del self.residuals[0]
        return r

    def _mix(self, n_in, n_out):
        r = self._record(n_in, n_out)
        return n_in + self.beta * self.precondition(r)

    def __call__(self, density_in, density_out):
        as_numpy = not isinstance(density_in, torch.Tensor)
        if as_numpy:
            dev = torch.device("cuda", torch.cuda.current_device())
            density_in = torch.from_numpy(np.asarray(density_in, dtype=float)).to(dev)
            density_out = torch.from_numpy(np.asarray(density_out, dtype=float)).to(dev)
        out = self._mix(density_in.to(torch.float64), density_out.to(torch.float64))
        return out.cpu().numpy() if as_numpy else out


class LinearMixer(Mixer):
    pass


class PulayMixer(Mixer):
    def _coefficients(self) -> np.ndarray:
        while True:
            size = len(self.residuals)
            if size == 1:
                return np.ones(1)
            flat = torch.stack([r.reshape(-1) for r in self.residuals])
            overlap = (flat @ flat.T).cpu().numpy()
            scale = float(np.trace(overlap)) / size
            m = np.ones((size + 1, size + 1))
            m[:size, :size] = overlap / scale
            m[size, size] = 0.0
            t = np.zeros(size + 1)
            t[size] = 1.0
            try:
                sol = np.linalg.solve(m, t)
            except np.linalg.LinAlgError:
                pass
            else:
                if np.all(np.isfinite(sol)) and np.max(np.abs(sol[:size])) < 1e4:
                    return sol[:size]
            del self.inputs[0]
            del self.residuals[0]

    def _mix(self, n_in, n_out):
        self._record(n_in, n_out)
        c = torch.from_numpy(self._coefficients()).to(n_in.device)
        mixed_in = torch.einsum("i,i...->...", c, torch.stack(self.inputs))
        mixed_res = torch.einsum("i,i...->...", c, torch.stack(self.residuals))
        return mixed_in + self.beta * self.precondition(mixed_res)


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
        r = self._record(n_in, n_out)
        step = self.beta * self.precondition(r)
        if len(self.residuals) < 2:
            return n_in + step
        dfs, dns = [], []
        for i in range(len(self.residuals) - 1):
            d = self.residuals[i + 1] - self.residuals[i]
            nrm = float(torch.linalg.vector_norm(d))
            if nrm < 1e-30:
                continue
            dfs.append(d.reshape(-1) / nrm)
            dns.append((self.inputs[i + 1] - self.inputs[i] + self.beta * self.precondition(d)).reshape(-1) / nrm)
        if not dfs:
            return n_in + step
        df = torch.stack(dfs)
        dn = torch.stack(dns)
        m = self.weight**2 * (df @ df.T).cpu().numpy() + self.w0**2 * np.eye(len(dfs))
        ov = self.weight * (df @ r.reshape(-1)).cpu().numpy()
        gamma = np.linalg.solve(m, ov) * self.weight
        corr = (torch.from_numpy(gamma).to(dn.device) @ dn).reshape(n_in.shape)
        return n_in + step - corr


_MIXERS = {"linear": LinearMixer, "anderson": AndersonMixer, "pulay": PulayMixer, "broyden": BroydenMixer}


def create_mixer(config, system, *, floating_charge: bool = False) -> Mixer:
    """The mixer named by ``config.algorithm`` with its Kerker preconditioner."""
    factory = _MIXERS.get(config.algorithm)
    if factory is None:
        raise ValueError(f"unknown mixing algorithm {config.algorithm!r}")
    mixer = factory(beta=config.beta, history=config.history)
    if config.preconditioner == "kerker":
        mixer.precondition = KerkerPreconditioner(system, config.kerker_q0,
                                                  uniform_factor=1.0 if floating_charge else 0.0)
    return mixer
