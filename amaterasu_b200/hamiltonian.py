"""Drop-in ``Hamiltonian``: the reference's Python API over the CUDA engine.

Mirrors amaterasu ``hamiltonian/operator.py:37-95``: same constructor (system, effective
potential of shape (nspin, n1, n2, n3) or (n1, n2, n3), ValueError on a mismatch), same
``apply(coefficients, ik, spin)`` for one band (npw,) or a block (nbands, npw), identity
``apply_overlap`` for norm-conserving datasets and ``local_energy``. numpy input returns
numpy (host<->device copies at the boundary); CUDA tensors stay on the device.
``apply_all`` is the batched form: every k-point in one set of launches.
"""
from __future__ import annotations

import numpy as np
import torch

from .engine import TORCH_DTYPE, engine_for, precision_code, require_cuda


class Hamiltonian:
    """A Kohn-Sham Hamiltonian at one fixed effective potential, applied on the GPU."""

    def __init__(self, system, effective_potential, coupling=None, *, precision="complex128"):
        if coupling is not None:
            raise NotImplementedError("PAW couplings are not supported by this engine")
        self.system = system
        self.precision = precision_code(precision)
        if isinstance(effective_potential, torch.Tensor):
            pot = effective_potential.to(torch.float64)
        else:
            pot = torch.from_numpy(np.asarray(effective_potential, dtype=float))
        if pot.ndim == 3:
            pot = pot[None, ...]
        expected = (system.nspin, *system.grid.shape)
        if tuple(pot.shape) != tuple(expected):
            raise ValueError(f"effective potential has shape {tuple(pot.shape)}, expected {expected}")
        self.device = require_cuda()
        self.effective_potential = pot.to(self.device).contiguous()
        self.engine = engine_for(system)
        self._bind()

    def _bind(self):
        # The engine holds one potential at a time; rebind before every use so several
        # Hamiltonian objects of one system can be alive together.
        if getattr(self.engine, "_bound", None) is not self:
            self.engine.set_potential(self.effective_potential)
            self.engine._bound = self

    @property
    def overlap_operator(self):
        return None

    def apply(self, coefficients, ik: int, spin: int = 0):
        """``H |psi>`` for one band or a block of bands at k-point ``ik``."""
        npw = int(self.engine.npw[ik])
        as_numpy = not isinstance(coefficients, torch.Tensor)
        if as_numpy:
            arr = np.asarray(coefficients)
            psi = torch.from_numpy(np.ascontiguousarray(arr, dtype=np.complex128))
        else:
            psi = coefficients
        single = psi.ndim == 1
        if single:
            psi = psi[None, :]
        if psi.ndim != 2 or psi.shape[1] != npw:
            raise ValueError(f"coefficients have shape {tuple(psi.shape)}, expected (nbands, {npw})")
        dtype = TORCH_DTYPE[self.precision]
        dev = psi.to(self.device, dtype).contiguous()
        out = torch.empty_like(dev)
        if dev.shape[0] > 0:
            self._bind()
            self.engine.hpsi(dev, out, k_first=ik, k_count=1, nbands=dev.shape[0], spin=spin)
        if single:
            out = out[0]
        if as_numpy:
            return out.to(torch.complex128).cpu().numpy()
        return out.to(coefficients.dtype) if out.dtype != coefficients.dtype else out

    def apply_all(self, psi: torch.Tensor, nbands: int, spin: int = 0, *, k_first: int = 0,
                  k_count: int | None = None, out: torch.Tensor | None = None) -> torch.Tensor:
        """Batched H.psi over k-points: ``psi`` packs one (nbands, npw_k) block per k."""
        k_count = self.engine.nk - k_first if k_count is None else k_count
        out = torch.empty_like(psi) if out is None else out
        self._bind()
        return self.engine.hpsi(psi, out, k_first=k_first, k_count=k_count, nbands=nbands, spin=spin)

    def apply_host(self, host_in: torch.Tensor, host_out: torch.Tensor, nbands: int, spin: int = 0, *,
                   dev_in: torch.Tensor | None = None, dev_out: torch.Tensor | None = None,
                   chunks_per_k: int = 1) -> None:
        """Batched H.psi from host memory to host memory, pipelined over band chunks.

        ``host_in``/``host_out`` pack one (nbands, npw_k) block per k (pinned CPU tensors
        for asynchronous copies). Each k block is cut into ``chunks_per_k`` runs of bands; the
        copy of chunk i+1 in, the H.psi of chunk i and the copy of chunk i-1 out overlap on
        three streams, so only one chunk's copies are exposed at the start and the end. The
        call returns with the work queued on the current stream (synchronise before reading
        ``host_out``).
        """
        eng = self.engine
        offsets = eng.block_offsets(nbands)
        if host_in.numel() != int(offsets[-1]) or host_out.numel() != int(offsets[-1]):
            raise ValueError(f"host blocks hold {host_in.numel()} coefficients, expected {int(offsets[-1])}")
        dtype = TORCH_DTYPE[self.precision]
        if dev_in is None:
            dev_in = torch.empty(host_in.shape, dtype=dtype, device=self.device)
        if dev_out is None:
            dev_out = torch.empty_like(dev_in)
        if not hasattr(self, "_copy_streams"):
            self._copy_streams = (torch.cuda.Stream(self.device), torch.cuda.Stream(self.device))
        s_in, s_out = self._copy_streams
        compute = torch.cuda.current_stream(self.device)
        s_in.wait_stream(compute)
        s_out.wait_stream(compute)
        self._bind()
        per = max(1, -(-nbands // max(1, int(chunks_per_k))))
        for k in range(eng.nk):
            npw = int(eng.npw[k])
            for r0 in range(0, nbands, per):
                r1 = min(nbands, r0 + per)
                a, b = int(offsets[k]) + r0 * npw, int(offsets[k]) + r1 * npw
                with torch.cuda.stream(s_in):
                    dev_in[a:b].copy_(host_in[a:b], non_blocking=True)
                compute.wait_stream(s_in)
                eng.hpsi(dev_in[a:b], dev_out[a:b], k_first=k, k_count=1, nbands=r1 - r0, spin=spin)
                s_out.wait_stream(compute)
                with torch.cuda.stream(s_out):
                    host_out[a:b].copy_(dev_out[a:b], non_blocking=True)
        compute.wait_stream(s_out)

    def apply_overlap(self, coefficients, ik: int):
        return coefficients

    def local_energy(self, density) -> float:
        d = density if isinstance(density, torch.Tensor) else torch.from_numpy(np.asarray(density, float))
        d = d.to(self.device, torch.float64)
        return float((self.effective_potential * d).sum()) * self.system.grid.cell_volume_per_point
