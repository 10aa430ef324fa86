"""Minimal stand-in for the parts of ``ase`` that the reference's SCF path imports.

Test infrastructure only: it lets ``tests/golden/make_golden.py`` import and run the
reference package in a container without ``ase``. Cells and positions are in Angstrom,
as ``ase.Atoms`` keeps them.
"""
import numpy as np

__all__ = ["Atoms"]


class _Cell:
    def __init__(self, matrix):
        self.array = np.asarray(matrix, dtype=float).reshape(3, 3)

    def __getitem__(self, key):
        return self.array[key]

    def __array__(self, dtype=None, copy=None):
        return self.array if dtype is None else self.array.astype(dtype)

    def reciprocal(self):
        # ase convention: rows b_i with a_i . b_j = delta_ij (no 2 pi)
        return np.linalg.inv(self.array).T


class Atoms:
    def __init__(self, symbols, positions=None, cell=None, pbc=True, magmoms=None):
        self._symbols = list(symbols)
        n = len(self._symbols)
        self.positions = np.zeros((n, 3)) if positions is None else np.asarray(positions, float)
        self.cell = _Cell(np.eye(3) if cell is None else cell)
        self.pbc = np.array([bool(pbc)] * 3) if np.isscalar(pbc) else np.asarray(pbc, bool)
        self._magmoms = np.zeros(n) if magmoms is None else np.asarray(magmoms, float)

    def __len__(self):
        return len(self._symbols)

    def copy(self):
        return Atoms(self._symbols, self.positions.copy(), self.cell.array.copy(),
                     self.pbc.copy(), self._magmoms.copy())

    def get_positions(self):
        return self.positions.copy()

    def get_chemical_symbols(self):
        return list(self._symbols)

    def get_initial_magnetic_moments(self):
        return self._magmoms.copy()

    def get_scaled_positions(self, wrap=True):
        return self.positions @ np.linalg.inv(self.cell.array)

    @property
    def numbers(self):
        from .data import atomic_numbers
        return np.array([atomic_numbers[s] for s in self._symbols])
