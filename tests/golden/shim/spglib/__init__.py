"""Stand-in for ``spglib`` with symmetry switched off.

``get_symmetry_dataset`` raises, so the reference builds its system without a space group
(grid multiple 1, no density symmetrisation). ``get_ir_reciprocal_mesh`` reduces a
Monkhorst-Pack mesh by time reversal alone: grid point g (mesh order i-major, as numpy's
``meshgrid(indexing="ij")``) is mapped to the lowest-index point equivalent to it under
k -> -k, where a half-step shift s makes the partner of g the point -g - s (mod mesh).
"""
import numpy as np


def get_symmetry_dataset(*args, **kwargs):
    raise RuntimeError("symmetry analysis disabled in the test shim")


def get_ir_reciprocal_mesh(mesh, cell, is_shift=(0, 0, 0), is_time_reversal=True, symprec=1e-5):
    mesh = np.asarray(mesh, dtype=int)
    shift = np.asarray(is_shift, dtype=int)
    axes = [np.arange(n) for n in mesh]
    grid = np.stack(np.meshgrid(*axes, indexing="ij"), axis=-1).reshape(-1, 3)
    mapping = np.arange(len(grid))
    if is_time_reversal:
        partner = np.mod(-grid - shift, mesh)
        partner_index = (partner[:, 0] * mesh[1] + partner[:, 1]) * mesh[2] + partner[:, 2]
        for index in range(len(grid)):
            other = partner_index[index]
            if other < index:
                mapping[index] = mapping[other]
    return mapping, grid
