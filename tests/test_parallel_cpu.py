"""k-point sharding logic on CPU: the partition, and the collectives of a sharded SCF
iteration run as two gloo ranks against the single-process result."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


def test_partition_is_contiguous_balanced_and_complete():
    from amaterasu_b200.parallel import partition_kpoints
    rng = np.random.default_rng(0)
    npw = rng.integers(4500, 4700, size=260)
    for world in (1, 2, 3, 4, 8):
        parts = partition_kpoints(npw, 20, world)
        assert len(parts) == world
        assert parts[0][0] == 0 and sum(c for _, c in parts) == 260
        for (a, ca), (b, _) in zip(parts, parts[1:]):
            assert a + ca == b
        loads = [npw[a:a + c].sum() for a, c in parts]
        assert max(loads) / min(loads) < 1.1
    with pytest.raises(ValueError):
        partition_kpoints(npw[:3], 20, 4)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from amaterasu_b200.occupations import compute_occupations
        from amaterasu_b200.parallel import KpointComm, partition_kpoints
        rng = np.random.default_rng(42)
        nk, nb, n = 7, 6, 1000
        npw = rng.integers(100, 140, size=nk)
        eig = np.sort(rng.normal(size=(1, nk, nb)), axis=2)
        weights = rng.random(nk)
        weights /= weights.sum()
        dens_k = rng.random((nk, n))  # per-k density contributions
        parts = partition_kpoints(npw, nb, world)
        comm = KpointComm()
        k0, kc = parts[rank]
        gathered = comm.gather_eigenvalues(eig[:, k0:k0 + kc], parts)
        occ = compute_occupations(gathered, weights, 9.0, scheme="gaussian", smearing=0.05)
        rho = torch.from_numpy(dens_k[k0:k0 + kc].sum(0).copy())
        comm.allreduce_(rho)
        e = comm.allreduce_scalars([float(weights[k0:k0 + kc].sum()), float(k0 + kc)])
        out[rank] = (np.array_equal(gathered, eig), occ.fermi_level, float(np.abs(rho.numpy() - dens_k.sum(0)).max()),
                     e.tolist())
    finally:
        dist.destroy_process_group()


def test_sharded_collectives_match_single_process():
    from amaterasu_b200.occupations import compute_occupations
    world = 2
    manager = mp.get_context("spawn").Manager()
    out = manager.dict()
    mp.spawn(_worker, args=(world, _free_port(), out), nprocs=world, join=True)
    rng = np.random.default_rng(42)
    nk, nb = 7, 6
    rng.integers(100, 140, size=nk)
    eig = np.sort(rng.normal(size=(1, nk, nb)), axis=2)
    weights = rng.random(nk)
    weights /= weights.sum()
    ref = compute_occupations(eig, weights, 9.0, scheme="gaussian", smearing=0.05)
    for rank in range(world):
        same, fermi, drho, sums = out[rank]
        assert same
        assert fermi == ref.fermi_level
        assert drho < 1e-12
        assert abs(sums[0] - 1.0) < 1e-12
