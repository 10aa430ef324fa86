"""The run-time variant choice: every stage B variant and nonlocal path compiled for a grid
gives the reference's H.psi, and autotune_hpsi leaves the engine on the fastest one.

Tolerances as in test_hpsi_gpu.py: 1e-11 (complex128), 2e-5 (complex64) of max|H psi|."""
import numpy as np
import pytest
import torch

from conftest import golden
from oracle.hamiltonian import hamiltonian_apply

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def _available(eng, precision):
    out = []
    for v in (0, 1, 2, 3, 4):
        try:
            eng.set_stage_b_variant(precision, v)
            out.append(v)
        except NotImplementedError:
            pass
    return out


def _available_ac(eng):
    out = []
    for v in (0, 1):
        try:
            eng.set_stage_ac_variant(v)
            out.append(v)
        except NotImplementedError:
            pass
    return out


@pytest.mark.parametrize("precision,tol", [("complex128", 1e-11), ("complex64", 2e-5)])
def test_every_variant_matches_the_oracle(mini_system, precision, tol):
    from amaterasu_b200.autotune import autotune_hpsi
    from amaterasu_b200.hamiltonian import Hamiltonian
    s = mini_system
    rng = np.random.default_rng(5)
    veff = rng.normal(size=(1, *s.grid.shape))
    H = Hamiltonian(s, veff, precision=precision)
    eng = H.engine
    variants = _available(eng, precision)
    assert 0 in variants and (precision == "complex128" or 1 in variants)
    for v in variants:
        for tc in ((True, False) if precision == "complex64" else (True,)):
            eng.set_stage_b_variant(precision, v)
            eng.set_tensor_core_nonlocal(tc)
            for ik, w in enumerate(s.wave_spheres):
                psi = rng.normal(size=(3, len(w))) + 1j * rng.normal(size=(3, len(w)))
                ref = hamiltonian_apply(psi, w.miller, s.grid.shape, w.kinetic_energy, veff[0],
                                        s.projectors[ik].matrix, s.projectors[ik].dij)
                assert _rel(H.apply(psi, ik), ref) < tol, (v, tc, ik)
    choice = autotune_hpsi(H, 4)
    assert choice["stage_b"] in variants and len(choice["ms"]) >= len(variants)
    assert autotune_hpsi(H, 4) is choice  # cached
    eng.set_stage_b_variant(precision, 1 if precision == "complex64" else 0)
    eng.set_tensor_core_nonlocal(True)


def test_si64_variants_match_the_reference(si_pseudo):
    """84^3 grid: shared-memory, register, sparse register and two-lane register stage B
    (complex64), whole-slab and z-split shared-memory stage B (complex128), against the
    golden."""
    from amaterasu_b200.autotune import autotune_hpsi
    from amaterasu_b200.cells import workload
    from amaterasu_b200.hamiltonian import Hamiltonian
    from amaterasu_b200.potential import effective_potential
    from amaterasu_b200.system import build_system
    g = golden("si64.npz")
    structure, ecut, ks, nb = workload("si64_hpsi")
    s = build_system(structure, {"Si": si_pseudo}, ecut, 4 * ecut, kpoints=ks, nbands=nb)
    veff, _, _ = effective_potential(s, s.initial_density())
    H = Hamiltonian(s, veff.cpu().numpy(), precision="complex64")
    eng = H.engine
    variants = _available(eng, "complex64")
    assert variants == [0, 1, 2, 3]
    ac = _available_ac(eng)
    assert ac == [0, 1]
    for v in variants:
        eng.set_stage_b_variant("complex64", v)
        for a in ac:
            eng.set_stage_ac_variant(a)
            for ik, nbk in ((0, 2), (1, 1)):
                w = s.wave_spheres[ik]
                rng = np.random.default_rng(300 + ik)
                psi = (rng.normal(size=(nbk, len(w))) + 1j * rng.normal(size=(nbk, len(w)))) / (1.0 + w.kinetic_energy)
                assert _rel(H.apply(psi, ik), g[f"hpsi{ik}"]) < 2e-5, (v, a, ik)
    choice = autotune_hpsi(H, 32)
    print("autotune", choice)
    assert choice["stage_b"] in variants and choice["stage_ac"] in ac
    # complex128: the whole-slab and the z-split shared-memory stage B
    H2 = Hamiltonian(s, veff.cpu().numpy(), precision="complex128")
    v128 = _available(H2.engine, "complex128")
    assert v128 == [0, 4]
    for v in v128:
        H2.engine.set_stage_b_variant("complex128", v)
        for ik, nbk in ((0, 2), (1, 1)):
            w = s.wave_spheres[ik]
            rng = np.random.default_rng(300 + ik)
            psi = (rng.normal(size=(nbk, len(w))) + 1j * rng.normal(size=(nbk, len(w)))) / (1.0 + w.kinetic_energy)
            assert _rel(H2.apply(psi, ik), g[f"hpsi{ik}"]) < 1e-11, (v, ik)
    H2.engine.set_stage_b_variant("complex128", 0)
    torch.cuda.synchronize()


def test_si8_grid_variants_match_the_oracle(si_pseudo):
    """42^3 grid (the 260-k Si8 configuration's): every stage B variant of both precisions,
    on two k-points of its mesh with 20 bands, against the oracle's FP64 H.psi."""
    from amaterasu_b200 import kpoints as kp
    from amaterasu_b200.cells import workload
    from amaterasu_b200.hamiltonian import Hamiltonian
    from amaterasu_b200.system import build_system
    structure, ecut, ks, nb = workload("si8_batched")
    two = kp.KPointSet(ks.points[[0, 37]], ks.weights[[0, 37]], ks.mesh, ks.shift)
    s = build_system(structure, {"Si": si_pseudo}, ecut, 4 * ecut, kpoints=two, nbands=nb)
    assert tuple(s.grid.shape) == (42, 42, 42)
    rng = np.random.default_rng(42)
    veff = rng.normal(size=(1, *s.grid.shape))
    H = Hamiltonian(s, veff, precision="complex64")
    eng = H.engine
    variants = _available(eng, "complex64")
    assert variants == [0, 1, 3]
    for v in variants:
        eng.set_stage_b_variant("complex64", v)
        for ik, w in enumerate(s.wave_spheres):
            psi = (rng.normal(size=(nb, len(w))) + 1j * rng.normal(size=(nb, len(w)))) / (1.0 + w.kinetic_energy)
            ref = hamiltonian_apply(psi, w.miller, s.grid.shape, w.kinetic_energy, veff[0],
                                    s.projectors[ik].matrix, s.projectors[ik].dij)
            assert _rel(H.apply(psi, ik), ref) < 2e-5, (v, ik)
    H2 = Hamiltonian(s, veff, precision="complex128")
    assert _available(H2.engine, "complex128") == [0, 4]
    for v in (0, 4):
        H2.engine.set_stage_b_variant("complex128", v)
        for ik, w in enumerate(s.wave_spheres):
            psi = (rng.normal(size=(nb, len(w))) + 1j * rng.normal(size=(nb, len(w)))) / (1.0 + w.kinetic_energy)
            ref = hamiltonian_apply(psi, w.miller, s.grid.shape, w.kinetic_energy, veff[0],
                                    s.projectors[ik].matrix, s.projectors[ik].dij)
            assert _rel(H2.apply(psi, ik), ref) < 1e-11, (v, ik)
    H2.engine.set_stage_b_variant("complex128", 0)
