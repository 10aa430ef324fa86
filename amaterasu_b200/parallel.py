"""k-point sharding of the SCF over GPUs (one process per GPU, torch.distributed).

The Kohn-Sham problem is independent per (spin, k) inside an SCF iteration (amaterasu
``scf/driver.py:338-355`` loops over them serially), so each rank takes a contiguous block
of k-points, balanced by its share of sum_k npw_k * nbands (the H.psi work). Per SCF
iteration the ranks exchange:

* the partial densities (one all-reduce of nspin * N FP64 values, before the floor and
  rescale that need the total),
* the eigenvalues of all k-points (an all-gather, so every rank computes the same
  occupations and Fermi level by the same host arithmetic),
* the partial kinetic and nonlocal energies (one all-reduce of a few scalars).

Everything else (potential, mixing, convergence test) is replicated and deterministic, so
every rank takes the same collective steps in the same order. The backend is NCCL on GPUs;
with gloo (the CPU tests, and ranks sharing one GPU) device tensors are staged through host
memory around each collective.
"""
from __future__ import annotations

import numpy as np
import torch
import torch.distributed as dist


def partition_kpoints(npw, nbands: int, world: int):
    """Contiguous k blocks, one per rank, balanced by sum npw_k * nbands.

    Returns a list of (k_first, k_count); every rank gets at least one k-point when
    there are enough of them.
    """
    npw = np.asarray(npw, dtype=np.int64)
    nk = len(npw)
    if world < 1:
        raise ValueError("world must be positive")
    if world > nk:
        raise ValueError(f"{world} ranks for {nk} k-points: some ranks would be idle")
    cost = np.cumsum(npw * nbands)
    total = cost[-1]
    bounds = [0]
    for r in range(1, world):
        target = total * r / world
        b = int(np.searchsorted(cost, target, side="left")) + 1
        b = max(b, bounds[-1] + 1)
        b = min(b, nk - (world - r))
        bounds.append(b)
    bounds.append(nk)
    return [(bounds[r], bounds[r + 1] - bounds[r]) for r in range(world)]


class KpointComm:
    """The collectives of a k-sharded SCF on a process group."""

    def __init__(self, group=None):
        self.group = group
        self.world = dist.get_world_size(group) if dist.is_initialized() else 1
        self.rank = dist.get_rank(group) if dist.is_initialized() else 0

    def allreduce_(self, t: torch.Tensor) -> torch.Tensor:
        if self.world > 1:
            if t.is_cuda and dist.get_backend(self.group) != "nccl":  # gloo reduces host tensors
                host = t.cpu()
                dist.all_reduce(host, op=dist.ReduceOp.SUM, group=self.group)
                t.copy_(host)
            else:
                dist.all_reduce(t, op=dist.ReduceOp.SUM, group=self.group)
        return t

    def allreduce_scalars(self, values) -> np.ndarray:
        t = torch.tensor(np.asarray(values, dtype=np.float64))
        if self.world > 1:
            t = t.to(self._device())
            dist.all_reduce(t, op=dist.ReduceOp.SUM, group=self.group)
        return t.cpu().numpy()

    def gather_eigenvalues(self, local: np.ndarray, parts) -> np.ndarray:
        """local: (nspin, k_count_of_this_rank, nbands) -> (nspin, nk, nbands) on every rank."""
        if self.world == 1:
            return np.asarray(local)
        nspin, _, nb = local.shape
        width = max(c for _, c in parts)
        buf = torch.zeros((nspin, width, nb), dtype=torch.float64)
        buf[:, :local.shape[1]] = torch.from_numpy(np.asarray(local, dtype=np.float64))
        buf = buf.to(self._device())
        out = [torch.empty_like(buf) for _ in range(self.world)]
        dist.all_gather(out, buf, group=self.group)
        return np.concatenate([o.cpu().numpy()[:, :c] for o, (_, c) in zip(out, parts)], axis=1)

    def _device(self):
        backend = dist.get_backend(self.group)
        return torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")


def shard_system(system, parts, rank: int):
    """The rank's view of a system: its k-points (spheres, projectors, weights) only,
    plus the global weights and partition needed for the collectives. Shares every other
    field (grid, local potential, Ewald) with the global system."""
    import copy

    from . import kpoints as kp
    k0, kc = parts[rank]
    local = copy.copy(system)
    for attr in ("_device_engine", "_grid_ops", "_bd_cache", "_v_local_dev", "_sphere_tables", "_start_orbitals"):
        if hasattr(local, attr):
            delattr(local, attr)
    local.kpoints = kp.KPointSet(system.kpoints.points[k0:k0 + kc], system.kpoints.weights[k0:k0 + kc],
                                 system.kpoints.mesh, system.kpoints.shift)
    local.wave_spheres = system.wave_spheres[k0:k0 + kc]
    local.projectors = system.projectors[k0:k0 + kc]
    local.global_weights = np.asarray(system.kpoints.weights)
    local.kparts = list(parts)
    local.krank = rank
    return local
