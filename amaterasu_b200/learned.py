"""Learned SCF start density: a small periodic 3D convolution network.

The network maps the superposed atomic density n0 (the reference's start density,
amaterasu ``hamiltonian/local.py:77-106``) and the cell strain to a correction
Delta(r); the start density is n0 exp(Delta), renormalised to the electron count and
floored at zero exactly like the superposition (``local.py:102-105``), so a poor prediction
can only cost SCF iterations, never move the fixed point: the converged SCF decides.

Architecture (36^3 working grid, circular padding, 3x3x3 kernels, SiLU):
  enc1  8 -> 16 -> 16            (36^3)
  enc2  16 -> 32 (stride 2) -> 32 (18^3)
  enc3  32 -> 64 (stride 2) -> 64 (9^3)
  dec2  up x2, 64 -> 32, + enc2, 32 -> 32
  dec1  up x2, 32 -> 16, + enc1, 16 -> 16, 16 -> 1 (linear)
Input channels: n0 / mean(n0), the six strain components (xx, yy, zz, yz, xz, xy), zero.
Every convolution, activation and upsampling runs in the engine's hand-written kernels
(``csrc/convnet.cu``: BF16 operands, FP32 accumulation, forward and backward); the
trainer keeps FP32 master weights and runs Adam. Densities move between the system grid
and the 36^3 working grid by Fourier interpolation (zero-padding or truncating the
coefficients), which conserves the G=0 component.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from pathlib import Path

import numpy as np
import torch

from ._lib import call
from .engine import ptr, require_cuda, stream_ptr

WORK_GRID = 36
IN_CHANNELS = 8

# (name, ci, co, stride)
LAYERS = [
    ("e1a", 8, 16, 1), ("e1b", 16, 16, 1),
    ("e2a", 16, 32, 2), ("e2b", 32, 32, 1),
    ("e3a", 32, 64, 2), ("e3b", 64, 64, 1),
    ("u2", 64, 32, 1), ("d2", 32, 32, 1),
    ("u1", 32, 16, 1), ("d1", 16, 16, 1),
    ("out", 16, 1, 1),
]


# ------------------------------------------------------------------ kernel wrappers
def conv_fwd(x_bf16, w_bf16, bias, stride):
    b, ci, d = x_bf16.shape[0], x_bf16.shape[1], x_bf16.shape[2]
    co = w_bf16.shape[0]
    dout = d // stride
    y = torch.empty((b, co, dout, dout, dout), dtype=torch.float32, device=x_bf16.device)
    call("ama_conv3d_fwd_bf16", ptr(x_bf16), ptr(w_bf16), ptr(bias), ptr(y), b, ci, co, d, stride, stream_ptr())
    return y


def conv_bwd(dy, x_bf16, w_bf16, stride, need_dx=True):
    b, ci, d = x_bf16.shape[0], x_bf16.shape[1], x_bf16.shape[2]
    co = w_bf16.shape[0]
    dw = torch.empty((co, ci, 3, 3, 3), dtype=torch.float32, device=dy.device)
    db = torch.empty(co, dtype=torch.float32, device=dy.device)
    call("ama_conv3d_bwd_weight_bf16", ptr(dy), ptr(x_bf16), ptr(dw), ptr(db), b, ci, co, d, stride, stream_ptr())
    dx = None
    if need_dx:
        dx = torch.empty((b, ci, d, d, d), dtype=torch.float32, device=dy.device)
        call("ama_conv3d_bwd_data_bf16", ptr(dy), ptr(w_bf16), ptr(dx), b, ci, co, d, stride, stream_ptr())
    return dx, dw, db


def silu_fwd(z):
    a = torch.empty(z.shape, dtype=torch.bfloat16, device=z.device)
    call("ama_silu_fwd_bf16", ptr(z), ptr(a), z.numel(), stream_ptr())
    return a


def silu_bwd(z, da):
    dz = torch.empty_like(z)
    call("ama_silu_bwd", ptr(z), ptr(da.contiguous()), ptr(dz), z.numel(), stream_ptr())
    return dz


def up_fwd(x_bf16):
    b, c, d = x_bf16.shape[0], x_bf16.shape[1], x_bf16.shape[2]
    y = torch.empty((b, c, 2 * d, 2 * d, 2 * d), dtype=torch.bfloat16, device=x_bf16.device)
    call("ama_upsample2_fwd_bf16", ptr(x_bf16), ptr(y), b * c, d, stream_ptr())
    return y


def up_bwd(dy):
    b, c, d2 = dy.shape[0], dy.shape[1], dy.shape[2]
    d = d2 // 2
    dx = torch.empty((b, c, d, d, d), dtype=torch.float32, device=dy.device)
    call("ama_upsample2_bwd", ptr(dy.contiguous()), ptr(dx), b * c, d, stream_ptr())
    return dx


# ------------------------------------------------------------------------ network
class DensityNet:
    def __init__(self, seed: int = 0, device=None):
        self.device = device or require_cuda()
        g = torch.Generator().manual_seed(seed)
        self.params = {}
        for name, ci, co, stride in LAYERS:
            std = (2.0 / (ci * 27)) ** 0.5 * (0.1 if name == "out" else 1.0)
            w = torch.randn((co, ci, 3, 3, 3), generator=g) * std
            self.params[name] = [w.to(self.device), torch.zeros(co, device=self.device)]
        self._m = None
        self._v = None
        self._t = 0

    # weights as used by the kernels
    def _w16(self, name):
        return self.params[name][0].to(torch.bfloat16).contiguous()

    def forward(self, x: torch.Tensor, keep: bool = False):
        """x: [B][8][n][n][n] FP32 (n a multiple of 4) -> Delta [B][1][n]^3 FP32."""
        cache = {}
        w = {name: self._w16(name) for name, *_ in LAYERS}
        b = {name: self.params[name][1] for name, *_ in LAYERS}

        def conv_act(name, inp, stride):
            z = conv_fwd(inp, w[name], b[name], stride)
            a = silu_fwd(z)
            if keep:
                cache[name] = (inp, z)
            return a

        x16 = x.to(torch.bfloat16).contiguous()
        e1 = conv_act("e1b", conv_act("e1a", x16, 1), 1)
        e2 = conv_act("e2b", conv_act("e2a", e1, 2), 1)
        e3 = conv_act("e3b", conv_act("e3a", e2, 2), 1)
        u2 = up_fwd(e3)
        s2 = (conv_act("u2", u2, 1).float() + e2.float()).to(torch.bfloat16)
        d2 = conv_act("d2", s2, 1)
        u1 = up_fwd(d2)
        s1 = (conv_act("u1", u1, 1).float() + e1.float()).to(torch.bfloat16)
        d1 = conv_act("d1", s1, 1)
        out = conv_fwd(d1, w["out"], b["out"], 1)
        if keep:
            cache["out"] = (d1, None)
            cache["_w"] = w
        return out, cache

    def backward(self, dout: torch.Tensor, cache) -> dict:
        """Gradients of every parameter for dL/dDelta = dout."""
        w = cache["_w"]
        grads = {}

        def back(name, stride, da, need_dx=True):
            inp, z = cache[name]
            dz = silu_bwd(z, da) if z is not None else da.contiguous()
            dx, dw, db = conv_bwd(dz, inp, w[name], stride, need_dx)
            grads[name] = (dw, db)
            return dx

        g_d1 = back("out", 1, dout)
        g_s1 = back("d1", 1, g_d1)
        g_u1 = back("u1", 1, g_s1)          # through the conv of the skip branch
        g_e1 = g_s1.clone()                 # skip: identity
        g_d2 = up_bwd(g_u1)
        g_s2 = back("d2", 1, g_d2)
        g_u2 = back("u2", 1, g_s2)
        g_e2 = g_s2.clone()
        g_e3 = up_bwd(g_u2)
        g_e3a = back("e3b", 1, g_e3)
        g_e2 = g_e2 + back("e3a", 2, g_e3a)
        g_e2a = back("e2b", 1, g_e2)
        g_e1 = g_e1 + back("e2a", 2, g_e2a)
        g_e1a = back("e1b", 1, g_e1)
        back("e1a", 1, g_e1a, need_dx=False)
        return grads

    def adam_step(self, grads, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8, weight_decay=0.0):
        if self._m is None:
            self._m = {k: [torch.zeros_like(p) for p in v] for k, v in self.params.items()}
            self._v = {k: [torch.zeros_like(p) for p in v] for k, v in self.params.items()}
        self._t += 1
        c1 = 1 - beta1**self._t
        c2 = 1 - beta2**self._t
        for name, (dw, db) in grads.items():
            for i, g in enumerate((dw, db)):
                p = self.params[name][i]
                if weight_decay and i == 0:
                    g = g + weight_decay * p
                m, v = self._m[name][i], self._v[name][i]
                m.mul_(beta1).add_(g, alpha=1 - beta1)
                v.mul_(beta2).addcmul_(g, g, value=1 - beta2)
                p.addcdiv_(m / c1, (v / c2).sqrt_().add_(eps), value=-lr)

    def state(self) -> dict:
        out = {}
        for name, (w, b) in self.params.items():
            out[f"{name}.w"] = w.cpu().numpy()
            out[f"{name}.b"] = b.cpu().numpy()
        return out

    def load(self, state: dict):
        for name in self.params:
            self.params[name][0] = torch.from_numpy(np.asarray(state[f"{name}.w"], dtype=np.float32)).to(self.device)
            self.params[name][1] = torch.from_numpy(np.asarray(state[f"{name}.b"], dtype=np.float32)).to(self.device)

    def save(self, path):
        np.savez_compressed(path, **self.state())

    @classmethod
    def from_file(cls, path):
        net = cls()
        net.load(dict(np.load(path)))
        return net


# ---------------------------------------------------------------- grids and inputs
def fourier_resample(field: np.ndarray, shape) -> np.ndarray:
    """Band-limited interpolation of a real periodic field to another grid shape."""
    src = np.asarray(field, dtype=float)
    coeff = np.fft.fftn(src) / src.size
    out = np.zeros(shape, dtype=complex)
    idx_src, idx_dst = [], []
    for ns, nd in zip(src.shape, shape):
        nmax = (min(ns, nd) - 1) // 2
        m = np.concatenate([np.arange(0, nmax + 1), np.arange(-nmax, 0)])
        idx_src.append(m % ns)
        idx_dst.append(m % nd)
    out[np.ix_(*idx_dst)] = coeff[np.ix_(*idx_src)]
    return np.real(np.fft.ifftn(out) * np.prod(shape))


def strain_of(cell, reference_cell) -> np.ndarray:
    """Symmetric strain eps with cell = reference (I + eps) (rows), Voigt-ordered."""
    f = np.linalg.solve(np.asarray(reference_cell, float), np.asarray(cell, float)) - np.eye(3)
    e = 0.5 * (f + f.T)
    return np.array([e[0, 0], e[1, 1], e[2, 2], e[1, 2], e[0, 2], e[0, 1]])


def network_input(n0_work: np.ndarray, strain: np.ndarray) -> np.ndarray:
    """[8][n]^3 input channels from n0 on the working grid and the strain."""
    x = np.zeros((IN_CHANNELS, *n0_work.shape), dtype=np.float32)
    x[0] = n0_work / max(float(n0_work.mean()), 1e-30)
    for i in range(6):
        x[1 + i] = 10.0 * strain[i]  # strains of a few percent -> O(0.1) inputs
    return x


def finalize(density: np.ndarray, nelectrons: float, dv: float) -> np.ndarray:
    """Floor at 1e-12 and rescale to the electron count (local.py:102-105)."""
    d = np.maximum(np.asarray(density, float), 1e-12)
    return d * (nelectrons / (float(d.sum()) * dv))


def working_grid(cell, spacing: float) -> int:
    """Edge of the cubic working grid whose point spacing along the longest cell vector is
    closest to ``spacing`` (same length unit as ``cell``), rounded to a multiple of 4 (two
    stride-2 levels). The network is fully convolutional, so a net trained at one spacing
    runs on larger cells at the same spacing."""
    length = float(np.max(np.linalg.norm(np.asarray(cell, float), axis=1)))
    return max(4, int(round(length / spacing / 4.0)) * 4)


@dataclass
class LearnedStart:
    """Predicts a start density for a system; falls back to the superposition.

    ``grid`` is the working-grid edge (``WORK_GRID`` for the cells the net was trained on;
    :func:`working_grid` keeps the training spacing on a larger cell)."""

    net: DensityNet
    reference_cell: np.ndarray
    stats: dict = field(default_factory=dict)
    grid: int = WORK_GRID

    def predict(self, system) -> np.ndarray:
        n0 = system.initial_density()  # (nspin, ...)
        total0 = n0.sum(axis=0)
        try:
            same = tuple(system.grid.shape) == (self.grid,) * 3
            if same:  # the resampling is a band limit: one grid-filter pass on the device
                from .potential import grid_ops
                ops = grid_ops(system)
                work = ops.band_limit(torch.from_numpy(total0)).reshape(total0.shape).cpu().numpy()
            else:
                work = fourier_resample(total0, (self.grid,) * 3)
            strain = strain_of(system.cell, self.reference_cell)
            x = torch.from_numpy(network_input(np.maximum(work, 1e-12), strain)[None]).to(self.net.device)
            delta, _ = self.net.forward(x)
            delta = torch.clamp(delta[0, 0].to(torch.float64), -5.0, 5.0)
            if same:
                log_corr = ops.band_limit(delta).reshape(total0.shape).cpu().numpy()
            else:
                log_corr = fourier_resample(delta.cpu().numpy(), tuple(system.grid.shape))
            pred = finalize(total0 * np.exp(log_corr), system.nelectrons, system.grid.cell_volume_per_point)
            if not np.all(np.isfinite(pred)):
                raise FloatingPointError("non-finite prediction")
            self.stats["fallback"] = False
        except Exception as exc:  # the superposition is the fallback
            self.stats["fallback"] = True
            self.stats["reason"] = repr(exc)
            return n0
        if system.nspin == 1:
            return pred[None]
        return np.stack([0.5 * pred, 0.5 * pred])


def train(net: DensityNet, inputs: np.ndarray, targets: np.ndarray, *, epochs: int = 200, batch: int = 4,
          lr: float = 2e-3, seed: int = 0, log=None, density_weighted: bool = True) -> list:
    """Fit Delta to log(n_conv / n0) on the working grid.

    The loss is the mean squared error weighted by n0 / mean(n0) (input channel 0): the
    start density's error is n0 * dDelta to first order, so low-density regions (vacancies,
    interstitials), where log(n_conv / n0) is large but carries little charge, do not
    dominate the fit. ``density_weighted=False`` gives the plain mean squared error."""
    rng = np.random.default_rng(seed)
    x_all = torch.from_numpy(np.asarray(inputs, dtype=np.float32)).to(net.device)
    t_all = torch.from_numpy(np.asarray(targets, dtype=np.float32)).to(net.device)
    n = len(x_all)
    history = []
    for epoch in range(epochs):
        order = rng.permutation(n)
        total = 0.0
        for s in range(0, n, batch):
            idx = torch.from_numpy(order[s:s + batch]).to(net.device)
            x, t = x_all[idx], t_all[idx]
            out, cache = net.forward(x, keep=True)
            diff = out - t
            w = x[:, :1] if density_weighted else torch.ones_like(diff)
            loss = float((w * diff * diff).mean())
            dout = (2.0 / diff.numel()) * w * diff
            grads = net.backward(dout.contiguous(), cache)
            step_lr = lr * 0.5 * (1 + np.cos(np.pi * epoch / max(epochs, 1)))
            net.adam_step(grads, lr=step_lr)
            total += loss * len(idx)
        history.append(total / n)
        if log and (epoch % 20 == 0 or epoch == epochs - 1):
            log(f"epoch {epoch:4d} loss {history[-1]:.4e}")
    return history
