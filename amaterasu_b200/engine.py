"""Device engine for one :class:`~amaterasu_b200.system.PlaneWaveSystem`.

Owns the C-ABI handle (``AmaEngine``) that holds the sphere<->grid maps, kinetic
energies, projector matrices and D.B in HBM, and exposes the batched device calls on
torch tensors. Every call runs on torch's current CUDA stream.
"""
from __future__ import annotations

import ctypes as ct

import numpy as np
import torch

from . import _lib
from ._lib import AMA_C64, AMA_C128, call

PRECISIONS = {"complex64": AMA_C64, "complex128": AMA_C128, torch.complex64: AMA_C64,
              torch.complex128: AMA_C128, np.complex64: AMA_C64, np.complex128: AMA_C128}
TORCH_DTYPE = {AMA_C64: torch.complex64, AMA_C128: torch.complex128}


def precision_code(p) -> int:
    if isinstance(p, int) and p in (AMA_C64, AMA_C128):
        return p
    if isinstance(p, np.dtype):
        p = p.type
    try:
        return PRECISIONS[p]
    except KeyError:
        raise ValueError(f"unsupported precision {p!r}; use complex64 or complex128") from None


def require_cuda() -> torch.device:
    if not torch.cuda.is_available():
        raise RuntimeError("amaterasu_b200 needs a CUDA device (sm_100a); there is no CPU fallback")
    return torch.device("cuda", torch.cuda.current_device())


def stream_ptr() -> ct.c_void_p:
    return ct.c_void_p(torch.cuda.current_stream().cuda_stream)


def ptr(t: torch.Tensor) -> ct.c_void_p:
    return ct.c_void_p(t.data_ptr())


def system_tables(system) -> dict:
    """The host arrays of an ``AmaSystemDesc`` for a plane-wave system: grid shape, plane
    waves per k, Miller indices (sphere order, k-major), kinetic energies, projector
    matrices (k-major, row-major (nproj, npw_k)) and D. Works on this package's
    ``PlaneWaveSystem`` and on the reference's (amaterasu ``hamiltonian/system.py:71-122``):
    both expose ``grid.shape``, ``wave_spheres[k].miller / .kinetic_energy``,
    ``projectors[k].matrix / .dij`` and ``nspin``."""
    spheres = system.wave_spheres
    projs = system.projectors
    nproj = 0 if projs[0] is None else int(np.asarray(projs[0].matrix).shape[0])
    tables = {
        "grid": tuple(int(n) for n in system.grid.shape),
        "npw": np.array([len(s.miller) for s in spheres], dtype=np.int32),
        "miller": np.ascontiguousarray(np.concatenate([s.miller for s in spheres]).astype(np.int32)),
        "kinetic": np.ascontiguousarray(np.concatenate([s.kinetic_energy for s in spheres]), dtype=np.float64),
        "nproj": nproj,
        "nspin": int(system.nspin),
    }
    if nproj:
        tables["projectors"] = np.ascontiguousarray(
            np.concatenate([np.asarray(p.matrix, dtype=np.complex128).ravel() for p in projs])).view(np.float64)
        tables["dij"] = np.ascontiguousarray(projs[0].dij, dtype=np.float64)
    else:
        tables["projectors"] = np.zeros(2)
        tables["dij"] = np.zeros(1)
    return tables


class DeviceEngine:
    """The C-ABI engine of a system, plus per-k offsets for packed band blocks."""

    def __init__(self, system, precisions=("complex128", "complex64")):
        self.device = require_cuda()
        lib = _lib.load()
        self.system = system
        spheres = system.wave_spheres
        t = system_tables(system)
        self.npw = t["npw"]
        self.pw_off = np.concatenate([[0], np.cumsum(self.npw.astype(np.int64))])
        self.nk = len(spheres)
        self.grid_shape = t["grid"]
        self.N = int(np.prod(self.grid_shape))
        self.nspin = t["nspin"]
        miller, kinetic = t["miller"], t["kinetic"]
        self.kinetic = [torch.from_numpy(np.ascontiguousarray(s.kinetic_energy)).to(self.device)
                        for s in spheres]
        self.nproj = t["nproj"]
        pmat, dij = t["projectors"], t["dij"]
        mask = 0
        for p in precisions:
            mask |= 1 << precision_code(p)
        self.precisions = mask
        desc = _lib.AmaSystemDesc(
            n1=self.grid_shape[0], n2=self.grid_shape[1], n3=self.grid_shape[2], nk=self.nk,
            npw=self.npw.ctypes.data_as(ct.POINTER(ct.c_int32)),
            miller=miller.ctypes.data_as(ct.POINTER(ct.c_int32)),
            kinetic=kinetic.ctypes.data_as(ct.POINTER(ct.c_double)),
            nproj=self.nproj,
            projectors=pmat.ctypes.data_as(ct.POINTER(ct.c_double)),
            dij=dij.ctypes.data_as(ct.POINTER(ct.c_double)),
            nspin=self.nspin, precisions=mask)
        handle = ct.c_void_p()
        with torch.cuda.device(self.device):
            call("ama_engine_create", ct.byref(desc), ct.byref(handle))
        self.handle = handle
        self._lib = lib
        self._potential_set = False

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                self._lib.ama_engine_destroy(h)
            except Exception:  # pragma: no cover - interpreter shutdown
                pass
            self.handle = None

    def set_tensor_core_nonlocal(self, enabled: bool) -> None:
        """Route the complex64 projector products to the tcgen05 split-TF32 GEMM (default)
        or to the SIMT GEMM."""
        call("ama_engine_option", self.handle, 0, 1 if enabled else 0)

    def set_stage_b_variant(self, precision, variant: int) -> None:
        """Select the stage B kernel (x transforms and V): 0 shared-memory slabs, 1 register-
        resident x columns, 2 register-resident with the compile-time x-plane set, 3 register-
        resident with two threads per column, 4 shared-memory slabs split in two along z.
        Raises NotImplementedError when the variant is not compiled for this grid."""
        option = 1 if precision_code(precision) == AMA_C64 else 2
        call("ama_engine_option", self.handle, option, int(variant))

    def set_stage_ac_variant(self, variant: int) -> None:
        """Select the complex64 stages A and C (y and z transforms with the sphere scatter and
        gather): 0 shared-memory y passes, 1 y transforms in registers with four lanes per
        column. Raises NotImplementedError when the variant is not compiled for this grid."""
        call("ama_engine_option", self.handle, 3, int(variant))

    def set_davidson_graphs(self, on: bool) -> None:
        """ama_davidson on this engine: replay recurring iteration segments as CUDA graphs
        (True, the default) or launch every kernel (False). The results are the same."""
        call("ama_engine_option", self.handle, 4, 1 if on else 0)

    def tc_status(self) -> int:
        code = ct.c_int32(0)
        call("ama_tc_status", self.handle, ct.byref(code))
        return int(code.value)

    def block_offsets(self, nbands: int, k_first: int = 0, k_count: int | None = None):
        """Element offsets of each k's (nbands, npw_k) block in a packed all-k array."""
        k_count = self.nk - k_first if k_count is None else k_count
        sizes = self.npw[k_first:k_first + k_count].astype(np.int64) * nbands
        return np.concatenate([[0], np.cumsum(sizes)])

    def set_potential(self, v: torch.Tensor) -> None:
        v = v.to(self.device, torch.float64).contiguous()
        if v.shape != (self.nspin, *self.grid_shape):
            raise ValueError(f"effective potential has shape {tuple(v.shape)}, "
                             f"expected {(self.nspin, *self.grid_shape)}")
        call("ama_set_potential", self.handle, ptr(v), self.nspin, stream_ptr())
        self._v = v  # keep alive until the stream consumes it
        self._potential_set = True

    def reserve(self, precision, max_bands: int) -> None:
        call("ama_reserve", self.handle, precision_code(precision), int(max_bands))

    def hpsi(self, psi: torch.Tensor, out: torch.Tensor, *, k_first: int, k_count: int,
             nbands: int, spin: int = 0) -> torch.Tensor:
        prec = precision_code(psi.dtype)
        expected = int(self.pw_off[k_first + k_count] - self.pw_off[k_first]) * nbands
        if psi.numel() != expected or out.numel() != expected:
            raise ValueError(f"packed psi has {psi.numel()} coefficients, expected {expected}")
        call("ama_hpsi", self.handle, prec, k_first, k_count, nbands, spin, ptr(psi), ptr(out), stream_ptr())
        return out

    def density_accumulate(self, psi: torch.Tensor, weights: torch.Tensor, rho: torch.Tensor, *,
                           k_first: int, k_count: int, nbands: int) -> None:
        prec = precision_code(psi.dtype)
        expected = int(self.pw_off[k_first + k_count] - self.pw_off[k_first]) * nbands
        if psi.numel() != expected:
            raise ValueError(f"packed psi has {psi.numel()} coefficients, expected {expected}")
        if weights.dtype != torch.float64 or weights.numel() != k_count * nbands:
            raise ValueError("weights must be float64 with k_count*nbands entries")
        if rho.dtype != torch.float64 or rho.numel() != self.N:
            raise ValueError("rho must be float64 with one value per grid point")
        call("ama_density_accumulate", self.handle, prec, k_first, k_count, nbands, ptr(psi),
             ptr(weights), ptr(rho), stream_ptr())

    def project(self, psi: torch.Tensor, k: int) -> torch.Tensor:
        prec = precision_code(psi.dtype)
        nb = psi.shape[0]
        out = torch.empty((nb, self.nproj), dtype=psi.dtype, device=psi.device)
        call("ama_project", self.handle, prec, k, nb, ptr(psi), ptr(out), stream_ptr())
        return out


class DeviceTimeout(_lib.AmaError):
    """A bounded device-side wait ran out: the kernel skipped the rest of its work, so the
    results of that launch (and everything computed from them) are wrong."""


def check_device_status(engine: "DeviceEngine | None" = None) -> None:
    """Raise :class:`DeviceTimeout` if a kernel recorded a timed-out wait.

    The tcgen05 kernels (nonlocal products of an engine, Davidson subspace products of the
    current device) bound every mbarrier wait, and the eigensolver's cooperative
    tridiagonalisation bounds every grid-barrier wait; one that runs out sets a device-side
    error word and the kernel returns without finishing. Reading the words costs one small
    synchronous device-to-host copy each, so callers check once per SCF step."""
    codes = []
    code = ct.c_int32(0)
    if engine is not None:
        call("ama_tc_status", engine.handle, ct.byref(code))
        codes.append(("nonlocal tensor-core products", int(code.value)))
    code = ct.c_int32(0)
    call("ama_subspace_tc_status", ct.byref(code))
    codes.append(("subspace tensor-core products", int(code.value)))
    code = ct.c_int32(0)
    call("ama_solver_status", ct.byref(code))
    codes.append(("subspace eigensolver", int(code.value)))
    bad = [f"{name} (wait code {value})" for name, value in codes if value]
    if bad:
        raise DeviceTimeout("a bounded device wait ran out in the " + " and ".join(bad)
                            + "; the results of that step are invalid")


class GridEngine:
    """A C-ABI engine for a bare FFT grid (one plane wave, no projectors): enough for the
    FP64 grid transforms and filters (Kerker, Hartree) when no system engine exists."""

    def __init__(self, shape):
        self.device = require_cuda()
        lib = _lib.load()
        self.grid_shape = tuple(int(n) for n in shape)
        self.N = int(np.prod(self.grid_shape))
        npw = np.ones(1, dtype=np.int32)
        miller = np.zeros(3, dtype=np.int32)
        kinetic = np.zeros(1)
        dij = np.zeros(1)
        self._keep = (npw, miller, kinetic, dij)
        desc = _lib.AmaSystemDesc(
            n1=self.grid_shape[0], n2=self.grid_shape[1], n3=self.grid_shape[2], nk=1,
            npw=npw.ctypes.data_as(ct.POINTER(ct.c_int32)), miller=miller.ctypes.data_as(ct.POINTER(ct.c_int32)),
            kinetic=kinetic.ctypes.data_as(ct.POINTER(ct.c_double)), nproj=0, projectors=None,
            dij=dij.ctypes.data_as(ct.POINTER(ct.c_double)), nspin=1, precisions=1 << AMA_C128)
        handle = ct.c_void_p()
        with torch.cuda.device(self.device):
            call("ama_engine_create", ct.byref(desc), ct.byref(handle))
        self.handle = handle
        self._lib = lib

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                self._lib.ama_engine_destroy(h)
            except Exception:  # pragma: no cover - interpreter shutdown
                pass
            self.handle = None


def engine_for(system, precisions=("complex128", "complex64")) -> DeviceEngine:
    """The system's engine, created on first use and cached on the system object."""
    eng = getattr(system, "_device_engine", None)
    if eng is None:
        eng = DeviceEngine(system, precisions)
        system._device_engine = eng
    return eng
