"""The fixed part of a plane-wave calculation: basis, k-points, projectors, local
potential, Ewald energy (host set-up, FP64).

Mirrors amaterasu ``hamiltonian/system.py`` for the norm-conserving path
(``build_system`` :215-379, ``PlaneWaveSystem`` :62-212, ``default_band_count`` :48-59)
with symmetry switched off: the grid multiple is 1 and the density is not symmetrised.
The device engine (``amaterasu_b200.engine``) is built from this object.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from . import kpoints as kpoint_module
from .basis import FFTGrid, GSphere
from .ewald import ewald_energy
from .local import atomic_core_density, atomic_valence_density, local_potential
from .projectors import ProjectorSet, build_projectors
from .units import ANG_IN_BOHR

__all__ = ["PlaneWaveSystem", "Structure", "build_system", "default_band_count"]


@dataclass
class Structure:
    """A periodic cell: rows of ``cell`` and ``positions`` in Angstrom."""

    symbols: list
    positions: np.ndarray
    cell: np.ndarray

    def __len__(self) -> int:
        return len(self.symbols)


def _structure_arrays(atoms):
    if isinstance(atoms, Structure):
        return list(atoms.symbols), np.asarray(atoms.positions, float), np.asarray(atoms.cell, float)
    # duck-typed ase.Atoms
    if hasattr(atoms, "pbc") and not all(np.atleast_1d(atoms.pbc)):
        raise ValueError("every direction must be periodic")
    return (list(atoms.get_chemical_symbols()), np.asarray(atoms.get_positions(), float),
            np.asarray(atoms.cell[:], float))


def default_band_count(nelectrons: float, nspin: int, moment: float = 0.0) -> int:
    occupied = 0.5 * nelectrons
    if nspin == 2:
        occupied += 0.5 * abs(moment)
    return max(math.ceil(occupied) + 4, math.ceil(1.2 * occupied))


@dataclass
class PlaneWaveSystem:
    cell: np.ndarray            # Bohr, rows
    positions: np.ndarray       # Bohr
    symbols: list
    pseudopotentials: dict
    xc: str
    ecut: float
    ecut_rho: float
    grid: FFTGrid
    density_sphere: GSphere
    kpoints: kpoint_module.KPointSet
    wave_spheres: list
    projectors: list
    nspin: int
    nbands: int
    nelectrons: float
    v_local: np.ndarray
    core_density: np.ndarray | None = None
    warnings: list = field(default_factory=list)
    _ewald: float | None = field(default=None, repr=False)

    @property
    def ewald(self) -> float:
        """Ion-ion Ewald energy (Ha), summed on the GPU the first time it is needed."""
        if self._ewald is None:
            charges = np.array([self.pseudopotentials[s].valence_charge for s in self.symbols])
            self._ewald = float(ewald_energy(self.cell, self.positions, charges))
        return self._ewald

    @property
    def volume(self) -> float:
        return self.grid.volume

    @property
    def nkpoints(self) -> int:
        return len(self.kpoints)

    @property
    def natoms(self) -> int:
        return len(self.symbols)

    def smooth_electron_count(self) -> float:
        return self.nelectrons

    def initial_density(self) -> np.ndarray:
        """Superposed atomic valence density, shape (nspin, n1, n2, n3)."""
        total = atomic_valence_density(self.grid, self.density_sphere, self.positions, self.symbols,
                                       self.pseudopotentials, total_electrons=self.nelectrons)
        if self.nspin == 1:
            return total[None, ...]
        return np.stack([0.5 * total, 0.5 * total])

    def symmetrize_density(self, density):
        return density


def build_system(atoms, pseudopotentials: dict, ecut: float, ecut_rho: float | None = None, *,
                 kpoints: kpoint_module.KPointSet | None = None, nbands: int | None = None,
                 nspin: int = 1, xc: str = "LDA-PZ", charge: float = 0.0,
                 build_projector_matrices: bool = True) -> PlaneWaveSystem:
    """Assemble the fixed part of a calculation; ``ecut``/``ecut_rho`` in Hartree."""
    from .potential import functional_key
    xc = {"LDA-PZ": "LDA-PZ", "PBE": "PBE", "PBESOL": "PBEsol"}[functional_key(xc)]
    ecut_rho = 4.0 * ecut if ecut_rho is None else ecut_rho
    symbols, pos_ang, cell_ang = _structure_arrays(atoms)
    cell = cell_ang * ANG_IN_BOHR
    positions = pos_ang * ANG_IN_BOHR
    missing = sorted(set(symbols) - set(pseudopotentials))
    if missing:
        raise ValueError(f"no pseudopotential supplied for {', '.join(missing)}")
    nelectrons = sum(pseudopotentials[s].valence_charge for s in symbols) - charge
    if nelectrons <= 0:
        raise ValueError(f"the cell holds {nelectrons:g} electrons")
    kpoints = kpoint_module.gamma_only() if kpoints is None else kpoints
    grid = FFTGrid(shape=FFTGrid.for_cutoff(cell, ecut_rho).shape, cell=cell)
    density_sphere = GSphere.build(cell, ecut_rho)
    wave_spheres = [GSphere.build(cell, ecut, kpoint=k) for k in kpoints.points]
    nbands = nbands or default_band_count(nelectrons, nspin)
    warnings = []
    smallest = min(len(s) for s in wave_spheres)
    if nbands > smallest:
        warnings.append(f"asked for {nbands} bands but the smallest k-point has {smallest} plane waves")
        nbands = smallest
    if build_projector_matrices:
        projectors = [build_projectors(s, positions, symbols, pseudopotentials, grid.volume)
                      for s in wave_spheres]
    else:
        projectors = [None] * len(wave_spheres)
    v_local = local_potential(grid, density_sphere, positions, symbols, pseudopotentials)
    core = atomic_core_density(grid, density_sphere, positions, symbols, pseudopotentials)
    return PlaneWaveSystem(
        cell=cell, positions=positions, symbols=symbols, pseudopotentials=pseudopotentials, xc=xc,
        ecut=float(ecut), ecut_rho=float(ecut_rho), grid=grid, density_sphere=density_sphere,
        kpoints=kpoints, wave_spheres=wave_spheres, projectors=projectors, nspin=nspin,
        nbands=int(nbands), nelectrons=float(nelectrons), v_local=v_local,
        core_density=core, warnings=warnings,
    )
