"""SCF results written to and read from disk, in the reference's output units and layout.

Replaces amaterasu ``io/results.py:71-241`` (``write_scf`` / ``read_scf``). The reference
writes HDF5 through h5py; this engine keeps the same groups, dataset names, units and
conventions, stored as the keys ``group/name`` of one compressed ``.npz`` archive (h5py is
not a dependency here): an attribute ``a`` of group ``g`` is the key ``g/@a``.

Units (the reference's output convention): energies eV, lengths Angstrom, forces eV/A,
stress eV/A^3 positive under compression (the opposite sign to the internal
sigma = (1/Omega) dE/d eps), pressure GPa, density electrons/A^3. Wavefunctions, when
saved, are the orbital coefficients of every (spin, k) block, unchanged, so that
``run_scf(system, config, density=..., wavefunctions=...)`` restarts from them.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np

from .units import BOHR_IN_ANG, HARTREE_IN_EV, HARTREE_PER_BOHR3_IN_GPA, HARTREE_PER_BOHR_IN_EV_PER_ANG

__all__ = ["FORMAT_VERSION", "read_scf", "write_scf"]

#: Layout version of the reference's result files that this one mirrors (forces and stress present).
FORMAT_VERSION = 2
_ENERGY_TERMS = ("kinetic", "local", "hartree", "xc", "nonlocal_", "ewald", "entropy")


def _host(x):
    return x.cpu().numpy() if hasattr(x, "cpu") else np.asarray(x)


def write_scf(path, system, result, *, forces=None, stress=None, save_wavefunctions: bool = False) -> Path:
    """Write ``result`` (an SCFResult of ``system``) to ``path`` (.npz)."""
    path = Path(path)
    d: dict[str, np.ndarray] = {
        "@format_version": np.array(FORMAT_VERSION),
        "@stress_convention": np.array("positive_under_compression"),
        "@solver": np.array("scf"),
        "@functional": np.array(str(system.xc)),
        "@converged": np.array(bool(result.converged)),
        "structure/cell": np.asarray(system.cell) * BOHR_IN_ANG,
        "structure/positions": np.asarray(system.positions) * BOHR_IN_ANG,
        "structure/symbols": np.array(list(system.symbols)),
        "basis/@ecut": np.array(system.ecut * HARTREE_IN_EV),
        "basis/@ecut_rho": np.array(system.ecut_rho * HARTREE_IN_EV),
        "basis/grid_shape": np.asarray(system.grid.shape),
        "basis/plane_waves": np.asarray([len(s) for s in system.wave_spheres]),
        "kpoints/points": np.asarray(system.kpoints.points),
        "kpoints/weights": np.asarray(system.kpoints.weights),
        "scf/@iterations": np.array(int(result.iterations)),
        "scf/@seconds": np.array(float(result.seconds)),
        "scf/@electron_count": np.array(float(result.electron_count)),
        "scf/@magnetization": np.array(float(result.magnetization)),
        "scf/@fermi_level": np.array(result.fermi_level * HARTREE_IN_EV),
        "scf/eigenvalues": _host(result.eigenvalues) * HARTREE_IN_EV,
        "scf/occupations": _host(result.occupations),
        "scf/history": np.asarray(result.history, dtype=float),
        "density": _host(result.density) / BOHR_IN_ANG ** 3,
    }
    if result.gap is not None:
        d["scf/@gap"] = np.array(result.gap * HARTREE_IN_EV)
    for name in _ENERGY_TERMS:
        d[f"scf/energies/@{name.rstrip('_')}"] = np.array(getattr(result.energies, name) * HARTREE_IN_EV)
    for name in ("total", "free_energy", "extrapolated"):
        d[f"scf/energies/@{name}"] = np.array(getattr(result.energies, name) * HARTREE_IN_EV)
    if forces is not None:
        d["forces"] = np.asarray(forces) * HARTREE_PER_BOHR_IN_EV_PER_ANG
    if stress is not None:
        s = np.asarray(stress)
        d["stress"] = -s * HARTREE_IN_EV / BOHR_IN_ANG ** 3
        d["@pressure_GPa"] = np.array(float(-np.trace(s) / 3.0 * HARTREE_PER_BOHR3_IN_GPA))
    if save_wavefunctions:
        for spin, blocks in enumerate(result.wavefunctions):
            for ik, block in enumerate(blocks):
                d[f"wavefunctions/spin{spin}/kpoint{ik}"] = _host(block)
    with open(path, "wb") as fh:
        np.savez_compressed(fh, **d)
    return path


def read_scf(path) -> dict:
    """The archive as a nested dict in output units, plus, for a restart, ``density_internal``
    (electrons/Bohr^3) and ``wavefunctions`` ([spin][k] arrays) when they were saved."""
    with np.load(path, allow_pickle=False) as z:
        flat = {k: z[k] for k in z.files}
    out: dict = {}
    for key, value in flat.items():
        node = out
        parts = key.split("/")
        for p in parts[:-1]:
            node = node.setdefault(p, {})
        leaf = parts[-1]
        node[leaf] = value.item() if value.shape == () else value
    out["density_internal"] = flat["density"] * BOHR_IN_ANG ** 3
    if "wavefunctions" in out:
        wf = out.pop("wavefunctions")
        nspin = len(wf)
        out["wavefunctions"] = [[wf[f"spin{s}"][f"kpoint{k}"] for k in range(len(wf[f"spin{s}"]))]
                                for s in range(nspin)]
    return out
