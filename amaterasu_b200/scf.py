"""The self-consistent field loop on the GPU (norm-conserving, symmetry off).

Mirrors amaterasu ``scf/driver.py:267-464`` (``run_scf``, mixing branch): per iteration
v_eff[n_in] (Hartree + LDA + local), Davidson at every (spin, k) with the tolerance
schedule clip(1e-3 min(residual, 1), 1e-11, 1e-6) and 40/20 iterations, occupations,
n_out, the Kohn-Sham energy at n_out, the eigenvalue-sum identity, the density residual
integral |n_out - n_in| / N_e, convergence when |dF| < tol_energy * natoms (eV -> Ha) and
the residual < tol_density (from the second iteration on), then mixing. Starting
orbitals are random_bands seeded 12345 + 991 spin + ik (driver.py:255-264).

Precision policy (``config.engine.precision``): "complex128" is the plain FP64 engine;
"mixed" runs H.psi, Davidson and the density in complex64 and switches the orbitals to
complex128 once the density residual falls below ``refine_below``, or earlier when the
complex64 iterations stop reducing it (best of the last ``stall_window`` iterations not
below ``stall_ratio`` times the best before them: the FP32 rounding floor of a large cell
can sit above ``refine_below``), so the fixed point is the FP64 one. The complex64
Davidson tolerance is 1e-3 of the density residual clipped to [``c64_tolerance_floor``,
``c64_tolerance_cap``] (the reference's clip to [1e-11, 1e-6] with the FP32 noise floor and a
looser cap while the density is far from converged); ``refine_max_iterations`` > 0 caps
the Davidson iterations per SCF step of the FP64 refinement (the orbitals are already
converged to the FP32 floor; the SCF convergence test itself is unchanged). Energies, densities, potentials and subspace eigensolves are FP64 always.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np
import torch

from .autotune import autotune_hpsi
from .batched import BatchedDavidson
from .config import Config, parse_energy
from .density import accumulate_packed, band_weights, finalize_density
from .eigen import davidson, random_bands
from ._lib import call
from .engine import check_device_status, engine_for, precision_code, ptr, require_cuda, stream_ptr
from .linalg import gemm_nn
from .hamiltonian import Hamiltonian
from .mixing import create_mixer
from .occupations import compute_occupations
from .potential import effective_potential, grid_ops
from .units import EV_IN_HARTREE, HARTREE_IN_EV

__all__ = ["Energies", "SCFResult", "prepare_starting_orbitals", "run_scf", "starting_orbitals"]


def davidson_tolerance(residual: float, complex64: bool, engine) -> float:
    """Davidson residual tolerance of an SCF step: the reference's clip(1e-3 min(residual, 1),
    1e-11, 1e-6) (scf/driver.py:334); in the complex64 phase of the mixed policy 1e-3 of the
    residual clipped to [c64_tolerance_floor, c64_tolerance_cap] instead: never below the FP32
    rounding noise, and only as tight as the density residual warrants."""
    x = 1e-3 * min(float(residual), 1.0)
    if complex64:
        lo = engine.c64_tolerance_floor
        return float(np.clip(x, lo, max(engine.c64_tolerance_cap, lo)))
    return float(np.clip(x, 1e-11, 1e-6))


@dataclass
class Energies:
    kinetic: float = 0.0
    local: float = 0.0
    hartree: float = 0.0
    xc: float = 0.0
    nonlocal_: float = 0.0
    ewald: float = 0.0
    entropy: float = 0.0

    @property
    def total(self) -> float:
        return self.kinetic + self.local + self.hartree + self.xc + self.nonlocal_ + self.ewald

    @property
    def free_energy(self) -> float:
        return self.total - self.entropy

    @property
    def extrapolated(self) -> float:
        return self.total - 0.5 * self.entropy


@dataclass
class SCFResult:
    converged: bool
    iterations: int
    energies: Energies
    eigenvalues: np.ndarray
    occupations: np.ndarray
    fermi_level: float
    gap: float | None
    magnetization: float
    density: np.ndarray
    wavefunctions: list
    history: list = field(default_factory=list)
    electron_count: float = 0.0
    seconds: float = 0.0
    precision_trace: list = field(default_factory=list)
    seconds_per_iteration: list = field(default_factory=list)


class _Orbitals:
    """All (spin, k) orbital blocks in one packed device buffer per spin."""

    def __init__(self, system, nbands, dtype, device):
        self.system = system
        self.nbands = nbands
        self.eng = engine_for(system)
        self.offsets = self.eng.block_offsets(nbands)
        self.dtype = dtype
        total = int(self.offsets[-1])
        self.packed = [torch.empty(total, dtype=dtype, device=device) for _ in range(system.nspin)]

    def block(self, spin, ik) -> torch.Tensor:
        a, b = int(self.offsets[ik]), int(self.offsets[ik + 1])
        return self.packed[spin][a:b].view(self.nbands, -1)

    def set(self, spin, ik, value):
        self.block(spin, ik).copy_(value)

    def to(self, dtype):
        self.packed = [p.to(dtype) for p in self.packed]
        self.dtype = dtype


def starting_orbitals(system, spin: int, ik: int) -> torch.Tensor:
    """The reference's seeded starting block of (spin, k): random_bands seeded
    12345 + 991 spin + ik (scf/driver.py:255-264), orthonormalised, complex128 on the device.

    It depends only on the system (plane-wave count, kinetic energies, band count), so it is
    drawn once per system and kept: every SCF run on the system, whatever its precision
    policy, starts from the same block without drawing it again. ``prepare_starting_orbitals``
    draws them all up front (part of the system set-up)."""
    cache = system.__dict__.setdefault("_start_orbitals", {})
    key = (spin, ik, system.nbands)
    block = cache.get(key)
    if block is None:
        sphere = system.wave_spheres[ik]
        k_global = ik + (system.kparts[system.krank][0] if hasattr(system, "kparts") else 0)  # a rank's shard
        block = random_bands(len(sphere), system.nbands, sphere.kinetic_energy, seed=12345 + 991 * spin + k_global,
                             dtype=torch.complex128)
        cache[key] = block
    return block


def prepare_starting_orbitals(system) -> None:
    """Draw every (spin, k) starting block of the system now (see starting_orbitals)."""
    for spin in range(system.nspin):
        for ik in range(system.nkpoints):
            starting_orbitals(system, spin, ik)


def _band_factors(system, occ, spin) -> torch.Tensor:
    g = 2.0 / system.nspin
    w = g * np.asarray(system.kpoints.weights)[:, None] * np.asarray(occ)[spin]
    return torch.from_numpy(np.ascontiguousarray(w.ravel(), dtype=np.float64))


def _weighted_sum(rows: torch.Tensor, weights: torch.Tensor, acc: torch.Tensor, accumulate: bool) -> None:
    call("ama_vec_reduce", 0, rows.numel(), ptr(rows), ptr(weights.to(rows.device)), 1.0, int(accumulate), ptr(acc),
         stream_ptr())


def _kinetic_energy(system, orb: _Orbitals, occ, kin_packed) -> float:
    """Local (this rank's k-points) kinetic energy: per-band sum_G |psi|^2 T_G on the device
    (``ama_band_kinetic``), weighted by 2/nspin w_k f_nk; occ holds this rank's k-points."""
    eng = orb.eng
    dev = orb.packed[0].device
    rows = torch.empty(eng.nk * orb.nbands, dtype=torch.float64, device=dev)
    acc = torch.zeros(1, dtype=torch.float64, device=dev)
    npw = torch.from_numpy(eng.npw.astype(np.int32)).to(dev)
    pw_off = torch.from_numpy(eng.pw_off[:-1].astype(np.int64)).to(dev)
    for spin in range(system.nspin):
        call("ama_band_kinetic", precision_code(orb.dtype), eng.nk, orb.nbands, ptr(npw), ptr(pw_off),
             ptr(orb.packed[spin]), ptr(kin_packed), ptr(rows), stream_ptr())
        _weighted_sum(rows, _band_factors(system, occ, spin), acc, spin > 0)
    return float(acc[0])


def _nonlocal_energy(system, orb: _Orbitals, occ, dij_dev) -> float:
    """sum over bands of f <beta|psi>^* D <beta|psi>: the projections of each k (engine GEMM),
    P D on the FP64 GEMM, and the per-band quadratic forms (``ama_rowdot``)."""
    eng = orb.eng
    if eng.nproj == 0:
        return 0.0
    dev = orb.packed[0].device
    nb = orb.nbands
    rows = torch.empty(eng.nk * nb, dtype=torch.float64, device=dev)
    acc = torch.zeros(1, dtype=torch.float64, device=dev)
    for spin in range(system.nspin):
        for ik in range(system.nkpoints):
            p = eng.project(orb.block(spin, ik), ik).to(torch.complex128).contiguous()
            q = gemm_nn(p, dij_dev)
            call("ama_rowdot", nb, eng.nproj, ptr(p), ptr(q), ptr(rows[ik * nb:(ik + 1) * nb]), stream_ptr())
        _weighted_sum(rows, _band_factors(system, occ, spin), acc, spin > 0)
    return float(acc[0])


def _grid_dot(a: torch.Tensor, b: torch.Tensor, op: int = 0) -> float:
    """sum a*b (op 0) or sum |a - b| (op 1) over flat FP64 device vectors."""
    out = torch.empty(1, dtype=torch.float64, device=a.device)
    call("ama_vec_reduce", op, a.numel(), ptr(a.contiguous()), ptr(b.contiguous()), 1.0, 0, ptr(out), stream_ptr())
    return float(out[0])


def _density_out(system, orb: _Orbitals, occ, comm=None) -> torch.Tensor:
    rho = torch.zeros((system.nspin, orb.eng.N), dtype=torch.float64, device=orb.packed[0].device)
    for spin in range(system.nspin):
        accumulate_packed(system, orb.packed[spin], orb.nbands, band_weights(system, occ, spin), rho[spin])
    if comm is not None:
        comm.allreduce_(rho)  # partial densities of the ranks' k-points
    return finalize_density(system, rho)


def run_scf(system, config: Config | None = None, *, logger=None, wavefunctions=None, density=None,
            comm=None) -> SCFResult:
    """Run the SCF loop to self-consistency on the GPU.

    With ``comm`` (a :class:`~amaterasu_b200.parallel.KpointComm` of several ranks) the
    system must be this rank's shard (:func:`~amaterasu_b200.parallel.shard_system`): the
    rank solves its own k-points and the density, eigenvalues and band energies are
    combined across ranks every iteration."""
    distributed = comm is not None and comm.world > 1
    if distributed and not hasattr(system, "kparts"):
        raise ValueError("a distributed SCF needs the rank's shard of the system (parallel.shard_system)")
    config = config or Config()
    if config.scf.method != "mixing":
        raise NotImplementedError(f"scf.method {config.scf.method!r}: only density mixing is implemented")
    log = logger or (lambda *_: None)
    dev = require_cuda()
    started = time.perf_counter()
    natoms = system.natoms
    smearing = 0.0 if config.occupations.scheme == "fixed" else parse_energy(config.occupations.smearing, "eV")
    policy = config.engine.precision
    wdtype = torch.complex64 if policy in ("mixed", "complex64") else torch.complex128
    nb = system.nbands
    eng = engine_for(system)
    ops = grid_ops(system)
    N = eng.N
    dv = system.grid.cell_volume_per_point

    if density is None:
        rho_in = torch.from_numpy(system.initial_density().reshape(system.nspin, -1)).to(dev)
    else:
        d = density if isinstance(density, torch.Tensor) else torch.from_numpy(np.asarray(density, float))
        rho_in = d.to(dev, torch.float64).reshape(system.nspin, -1).clone()
    orb = _Orbitals(system, nb, wdtype, dev)
    for spin in range(system.nspin):
        for ik, sphere in enumerate(system.wave_spheres):
            if wavefunctions is not None:
                w = wavefunctions[spin][ik]
                w = w if isinstance(w, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(w))
                orb.set(spin, ik, w.to(dev, wdtype))
            else:
                orb.set(spin, ik, starting_orbitals(system, spin, ik).to(wdtype))
    eng.reserve("complex128" if wdtype == torch.complex128 else "complex64", nb)
    kin_dev = [torch.from_numpy(s.kinetic_energy).to(dev) for s in system.wave_spheres]
    kin_packed = torch.cat(kin_dev).contiguous()
    dij_dev = torch.from_numpy(system.projectors[0].dij).to(dev, torch.complex128) if eng.nproj else None
    vloc = torch.from_numpy(system.v_local.ravel()).to(dev)
    mixer = create_mixer(config.scf.mixing, system.grid)

    threshold = config.scf.tol_energy * natoms * EV_IN_HARTREE
    history, trace, step_times = [], [], []
    previous = np.inf
    residual = np.inf
    converged = False
    energies = Energies(ewald=system.ewald)
    occ_result = None
    eigenvalues = np.zeros((system.nspin, system.nkpoints, nb))
    rho_out = rho_in
    iteration = 0
    res64 = []  # density residuals of the complex64 iterations
    for iteration in range(1, config.scf.max_steps + 1):
        t_step = time.perf_counter()
        w = config.engine.stall_window
        stalled = len(res64) > w and min(res64[-w:]) > config.engine.stall_ratio * min(res64[:-w])
        if policy == "mixed" and orb.dtype == torch.complex64 and (residual < config.engine.refine_below or stalled):
            # the complex64 fixed point differs from the FP64 one by the FP32 rounding floor:
            # restart the mixer so that its history does not pull towards the former
            mixer = create_mixer(config.scf.mixing, system.grid)
            orb.to(torch.complex128)
            eng.reserve("complex128", nb)
        prec_name = "complex64" if orb.dtype == torch.complex64 else "complex128"
        trace.append(prec_name)
        veff, _, _ = effective_potential(system, rho_in)
        H = Hamiltonian(system, veff, precision=prec_name)
        if config.engine.autotune:  # kernel variants timed once per precision on this system
            autotune_hpsi(H, nb)
        tol = davidson_tolerance(residual, orb.dtype == torch.complex64, config.engine)
        maxit = 40 if iteration == 1 else 20
        if policy == "mixed" and orb.dtype == torch.complex128 and config.engine.refine_max_iterations > 0:
            maxit = config.engine.refine_max_iterations  # FP64 refinement of converged complex64 orbitals
        eigenvalues = np.empty((system.nspin, system.nkpoints, nb))
        for spin in range(system.nspin):
            if config.engine.batched:
                # every k-point in lockstep: one launch per step over all k
                key = ("_batched_davidson", orb.dtype)
                bd = getattr(system, "_bd_cache", {}).get(key)
                if bd is None:
                    bd = BatchedDavidson(system, nb, orb.dtype, tensor_cores=config.engine.tc_subspace,
                                         tc_min_npw=config.engine.tc_min_npw)
                    system._bd_cache = {**getattr(system, "_bd_cache", {}), key: bd}
                bd.graphs = config.engine.davidson_graphs
                eps, X, _, _ = bd.run(H, orb.packed[spin], tolerance=tol, max_iterations=maxit, spin=spin)
                eigenvalues[spin] = eps
                orb.packed[spin].copy_(X)
                continue
            for ik, sphere in enumerate(system.wave_spheres):
                res = davidson(lambda b, ik=ik, spin=spin: H.apply(b, ik, spin), orb.block(spin, ik),
                               kin_dev[ik], tolerance=tol, max_iterations=maxit)
                eigenvalues[spin, ik] = res.eigenvalues.cpu().numpy()
                orb.set(spin, ik, res.coefficients)
        check_device_status(eng)  # a timed-out device wait must not go unnoticed
        if distributed:
            eig_all = comm.gather_eigenvalues(eigenvalues, system.kparts)
            weights_all = system.global_weights
        else:
            eig_all, weights_all = eigenvalues, system.kpoints.weights
        occ_result = compute_occupations(eig_all, weights_all, system.nelectrons,
                                         scheme=config.occupations.scheme, smearing=smearing,
                                         order=config.occupations.order, nspin=system.nspin)
        occ_all = occ_result.occupations
        if distributed:
            k0, kc = system.kparts[system.krank]
            occ = occ_all[:, k0:k0 + kc]
        else:
            occ = occ_all
        rho_out = _density_out(system, orb, occ, comm if distributed else None)
        e_h, _ = ops.hartree(rho_out.sum(0))
        xc_d = rho_out
        if system.core_density is not None:
            xc_d = rho_out + torch.from_numpy(system.core_density.ravel()).to(dev)[None] / system.nspin
        e_xc, _, _ = ops.xc(xc_d, system.xc)
        e_kin = _kinetic_energy(system, orb, occ, kin_packed)
        e_nl = _nonlocal_energy(system, orb, occ, dij_dev)
        if distributed:
            e_kin, e_nl = comm.allreduce_scalars([e_kin, e_nl])
        energies = Energies(
            kinetic=float(e_kin),
            local=_grid_dot(vloc, rho_out[0] if system.nspin == 1 else rho_out.sum(0)) * dv,
            hartree=float(e_h), xc=float(e_xc),
            nonlocal_=float(e_nl),
            ewald=system.ewald, entropy=occ_result.entropy_term)
        band_sum = 2.0 / system.nspin * float(np.einsum("k,skn,skn->", weights_all, occ_all, eig_all))
        local_e = _grid_dot(veff.reshape(-1), rho_out.reshape(-1)) * dv
        identity = band_sum - (energies.kinetic + local_e + energies.nonlocal_)
        residual = _grid_dot(rho_out.reshape(-1), rho_in.reshape(-1), op=1) * dv / system.nelectrons
        if orb.dtype == torch.complex64:
            res64.append(residual)
        energy = energies.free_energy
        delta = energy - previous
        history.append((energy, residual, identity))
        step_times.append(time.perf_counter() - t_step)
        log(f"  {iteration:4d} {energy * HARTREE_IN_EV:18.9f} {delta * HARTREE_IN_EV / natoms:14.2e} "
            f"{residual:13.3e} {identity * HARTREE_IN_EV:12.2e} {step_times[-1]:9.2f} {prec_name}")
        if iteration > 1 and abs(delta) < threshold and residual < config.scf.tol_density:
            if not (policy == "mixed" and orb.dtype == torch.complex64):
                converged = True
                break
        previous = energy
        rho_in = mixer(rho_in, rho_out)

    wfs = [[orb.block(spin, ik).clone() for ik in range(system.nkpoints)] for spin in range(system.nspin)]
    dens = rho_out.reshape(system.nspin, *system.grid.shape).cpu().numpy()
    return SCFResult(
        converged=converged, iterations=iteration, energies=energies, eigenvalues=eig_all,
        occupations=occ_all, fermi_level=occ_result.fermi_level, gap=occ_result.gap,
        magnetization=occ_result.magnetization, density=dens, wavefunctions=wfs, history=history,
        electron_count=float(dens.sum()) * dv, seconds=time.perf_counter() - started,
        precision_trace=trace, seconds_per_iteration=step_times)
