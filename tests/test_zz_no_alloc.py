"""ama_grid_filter_noalloc: the grid filter for callers that cannot let the library call
cudaMalloc (device memory already reserved by a framework allocator, or loops that must
not take cudaMalloc's device-wide synchronisation). It must give the same Hartree
potential and energy as ama_grid_filter, on consecutive calls that share its fixed work
array, and refuse grids larger than that array. Collected last on purpose."""
import ctypes as ct

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _filter(lib, handle, noalloc, rho, slot=0, energy_slot=0):
    from amaterasu_b200.engine import ptr, stream_ptr
    out = torch.empty_like(rho)
    energy = torch.zeros(1, dtype=torch.float64, device=rho.device)
    fn = lib.ama_grid_filter_noalloc if noalloc else lib.ama_grid_filter
    rc = fn(handle, slot, energy_slot, ptr(rho), ptr(out), ptr(energy), stream_ptr())
    assert rc == 0, lib.ama_last_error().decode()
    torch.cuda.synchronize()
    return out.cpu().numpy(), float(energy[0])


def test_noalloc_filter_matches_allocating_filter(mini_system):
    from amaterasu_b200 import _lib
    from amaterasu_b200.potential import grid_ops
    lib = _lib.load()
    ops = grid_ops(mini_system)  # sets the Hartree filter (slot 0) on the engine
    handle = ops.engine.handle
    rng = np.random.default_rng(42)
    n = int(np.prod(mini_system.grid.shape))
    for call in range(2):  # two calls in a row share the fixed array
        rho = torch.from_numpy(np.abs(rng.normal(size=n)) * (1 + call)).cuda()
        ref, e_ref = _filter(lib, handle, False, rho)
        got, e_got = _filter(lib, handle, True, rho)
        scale = np.max(np.abs(ref))
        assert np.max(np.abs(got - ref)) <= 1e-12 * scale
        assert abs(e_got - e_ref) <= 1e-12 * abs(e_ref)


def test_noalloc_filter_without_energy_allocates_nothing(si_pseudo):
    """energy_slot -1 with no energy pointer (the Kerker use), on a fresh engine whose grid
    differs from the allocating path's last one: same result as ama_grid_filter, and the
    device's free memory does not move across further calls (the call allocates nothing)."""
    from amaterasu_b200 import _lib
    from amaterasu_b200 import kpoints as kp
    from amaterasu_b200.cells import si2_primitive
    from amaterasu_b200.engine import ptr, stream_ptr
    from amaterasu_b200.potential import grid_ops
    from amaterasu_b200.system import build_system
    lib = _lib.load()
    s = build_system(si2_primitive(), {"Si": si_pseudo}, 6.0, 24.0, kpoints=kp.gamma_only(), nbands=4)
    ops = grid_ops(s)
    ops.set_kerker(1.5)  # slot 1
    handle = ops.engine.handle
    n = int(np.prod(s.grid.shape))
    rho = torch.from_numpy(np.random.default_rng(7).normal(size=n)).cuda()
    ref = torch.empty_like(rho)
    assert lib.ama_grid_filter(handle, 1, -1, ptr(rho), ptr(ref), None, stream_ptr()) == 0
    out = torch.empty_like(rho)
    assert lib.ama_grid_filter_noalloc(handle, 1, -1, ptr(rho), ptr(out), None, stream_ptr()) == 0
    torch.cuda.synchronize()
    scale = float(ref.abs().max())
    assert float((out - ref).abs().max()) <= 1e-12 * scale
    free_before, _ = torch.cuda.mem_get_info()
    for _ in range(3):
        assert lib.ama_grid_filter_noalloc(handle, 1, -1, ptr(rho), ptr(out), None, stream_ptr()) == 0
    torch.cuda.synchronize()
    free_after, _ = torch.cuda.mem_get_info()
    assert free_after == free_before
    assert float((out - ref).abs().max()) <= 1e-12 * scale


def test_noalloc_filter_rejects_grids_beyond_its_array():
    from amaterasu_b200 import _lib
    lib = _lib.load()
    n1, n2, n3 = 240, 240, 40  # 2,304,000 points > 128^3, planes still fit in shared memory
    npw = np.array([1], dtype=np.int32)
    miller = np.zeros(3, dtype=np.int32)
    kinetic = np.zeros(1)
    dij = np.zeros(1)
    desc = _lib.AmaSystemDesc(n1=n1, n2=n2, n3=n3, nk=1, npw=npw.ctypes.data_as(ct.POINTER(ct.c_int32)),
                              miller=miller.ctypes.data_as(ct.POINTER(ct.c_int32)),
                              kinetic=kinetic.ctypes.data_as(ct.POINTER(ct.c_double)), nproj=0,
                              projectors=None, dij=dij.ctypes.data_as(ct.POINTER(ct.c_double)), nspin=1,
                              precisions=1 << _lib.AMA_C128)
    handle = ct.c_void_p()
    assert lib.ama_engine_create(ct.byref(desc), ct.byref(handle)) == 0, lib.ama_last_error().decode()
    try:
        rho = torch.zeros(n1 * n2 * n3, dtype=torch.float64, device="cuda")
        out = torch.empty_like(rho)
        rc = lib.ama_grid_filter_noalloc(handle, 0, -1, ct.c_void_p(rho.data_ptr()), ct.c_void_p(out.data_ptr()),
                                         None, None)
        assert rc == _lib.AMA_ERR_SHAPE
        assert b"exceeds" in lib.ama_last_error()
    finally:
        lib.ama_engine_destroy(handle)
