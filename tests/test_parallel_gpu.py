"""The k-sharded SCF (run_scf(comm=...)) run by two ranks that share one GPU, each with its
own CUDA context, exchanging densities, eigenvalues and band energies through gloo (host
tensors), against the single-process run on the same GPU. The ranks' kernels never wait on
one another; only the host collectives couple them.

Tolerances: the two runs start from the same seeded orbitals (global k index), run the same
per-k Davidson and differ only in the summation order of the partial densities and energies,
so the free energy agrees to
1e-10 Ha/atom, the eigenvalues to 1e-8 Ha and the density to 1e-8 (integrated |dn| per
electron)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _config():
    from amaterasu_b200.config import Config
    c = Config()
    c.occupations.scheme = "fixed"
    c.occupations.nbands = 8
    c.scf.tol_energy = 1e-8
    c.scf.tol_density = 1e-8
    c.engine.precision = "complex128"
    c.engine.batched = False  # per-k Davidson: each k-point's work is the same however they are split
    return c


def _system():
    import tempfile
    from pathlib import Path

    from amaterasu_b200.cells import workload
    from amaterasu_b200.pseudo import read_upf, write_synthetic_upf
    from amaterasu_b200.system import build_system
    with tempfile.TemporaryDirectory() as tmp:
        pseudo = read_upf(write_synthetic_upf(Path(tmp) / "Si.upf"))
    structure, ecut, ks, nb = workload("si2_scf")
    return build_system(structure, {"Si": pseudo}, ecut, 4 * ecut, kpoints=ks, nbands=nb)


def _rank(rank, world, port, out):
    from datetime import timedelta

    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    torch.cuda.set_device(0)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    try:
        from amaterasu_b200.parallel import KpointComm, partition_kpoints, shard_system
        from amaterasu_b200.scf import run_scf
        system = _system()
        parts = partition_kpoints([len(w) for w in system.wave_spheres], system.nbands, world)
        local = shard_system(system, parts, rank)
        res = run_scf(local, _config(), comm=KpointComm())
        out[rank] = (res.converged, res.iterations, res.energies.free_energy, res.eigenvalues, res.density)
    finally:
        dist.destroy_process_group()


def test_two_ranks_on_one_gpu_match_the_single_process_scf():
    from amaterasu_b200.scf import run_scf
    world = 2
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=600)
    for p in procs:
        if p.is_alive():
            p.kill()
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    system = _system()
    ref = run_scf(system, _config())
    natoms = system.natoms
    for rank in range(world):
        converged, iterations, free, eig, dens = out[rank]
        assert converged
        assert abs(free - ref.energies.free_energy) / natoms < 1e-10
        np.testing.assert_allclose(eig, ref.eigenvalues, rtol=0, atol=1e-8)
        dn = np.sum(np.abs(dens - ref.density)) * system.grid.cell_volume_per_point / system.nelectrons
        assert dn < 1e-8
