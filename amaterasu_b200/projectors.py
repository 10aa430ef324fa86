"""Kleinman-Bylander projector matrices ``<k+G|beta_i>`` for one k-point (host set-up).

Restates amaterasu ``pseudo/kb.py:260-343``: rows are ordered atom -> channel -> m
(m = -l..l), each row is ``4 pi/sqrt(Omega) (-i)^l Y_lm(k+G) f_l(|k+G|) e^{-i(k+G).tau}``
with real spherical harmonics (``kb.py:52-97``), and ``D`` is block-diagonal per atom,
coupling rows of equal (l, m). The device engine keeps the matrix in HBM and applies it
with its own GEMM kernels.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .formfactors import projector_form_factor

MAX_L = 3


def real_spherical_harmonics(l: int, directions) -> np.ndarray:
    """Real Y_lm for m=-l..l on (n,3) directions; the zero vector maps to +z."""
    if not 0 <= l <= MAX_L:
        raise NotImplementedError(f"real spherical harmonics are implemented up to l={MAX_L}")
    d = np.atleast_2d(np.asarray(directions, dtype=float))
    norms = np.linalg.norm(d, axis=1)
    unit = np.zeros_like(d)
    unit[:, 2] = 1.0
    nz = norms > 1e-14
    unit[nz] = d[nz] / norms[nz, None]
    x, y, z = unit[:, 0], unit[:, 1], unit[:, 2]
    if l == 0:
        return np.full((1, len(unit)), 0.5 / np.sqrt(np.pi))
    if l == 1:
        return np.sqrt(0.75 / np.pi) * np.stack([y, z, x])
    if l == 2:
        c2 = 0.5 * np.sqrt(15.0 / np.pi)
        return np.stack([c2 * x * y, c2 * y * z, 0.25 * np.sqrt(5.0 / np.pi) * (3.0 * z**2 - 1.0),
                         c2 * x * z, 0.25 * np.sqrt(15.0 / np.pi) * (x**2 - y**2)])
    return np.stack([
        0.25 * np.sqrt(17.5 / np.pi) * y * (3.0 * x**2 - y**2),
        0.5 * np.sqrt(105.0 / np.pi) * x * y * z,
        0.25 * np.sqrt(10.5 / np.pi) * y * (5.0 * z**2 - 1.0),
        0.25 * np.sqrt(7.0 / np.pi) * z * (5.0 * z**2 - 3.0),
        0.25 * np.sqrt(10.5 / np.pi) * x * (5.0 * z**2 - 1.0),
        0.25 * np.sqrt(105.0 / np.pi) * z * (x**2 - y**2),
        0.25 * np.sqrt(17.5 / np.pi) * x * (x**2 - 3.0 * y**2),
    ])


def solid_harmonics(l: int, vectors) -> np.ndarray:
    """``|q|^l Y_lm(q_hat)``, homogeneous polynomials of degree l, shape (2l+1, n)."""
    q = np.atleast_2d(np.asarray(vectors, dtype=float))
    x, y, z = q[:, 0], q[:, 1], q[:, 2]
    r2 = x**2 + y**2 + z**2
    if l == 0:
        return np.full((1, len(q)), 0.5 / np.sqrt(np.pi))
    if l == 1:
        return np.sqrt(0.75 / np.pi) * np.stack([y, z, x])
    if l == 2:
        c = 0.5 * np.sqrt(15.0 / np.pi)
        return np.stack([c * x * y, c * y * z, 0.25 * np.sqrt(5.0 / np.pi) * (3.0 * z**2 - r2),
                         c * x * z, 0.25 * np.sqrt(15.0 / np.pi) * (x**2 - y**2)])
    if l == 3:
        return np.stack([
            0.25 * np.sqrt(17.5 / np.pi) * y * (3.0 * x**2 - y**2),
            0.5 * np.sqrt(105.0 / np.pi) * x * y * z,
            0.25 * np.sqrt(10.5 / np.pi) * y * (5.0 * z**2 - r2),
            0.25 * np.sqrt(7.0 / np.pi) * z * (5.0 * z**2 - 3.0 * r2),
            0.25 * np.sqrt(10.5 / np.pi) * x * (5.0 * z**2 - r2),
            0.25 * np.sqrt(105.0 / np.pi) * z * (x**2 - y**2),
            0.25 * np.sqrt(17.5 / np.pi) * x * (x**2 - 3.0 * y**2),
        ])
    raise NotImplementedError(f"solid harmonics are implemented up to l={MAX_L}")


def solid_harmonics_gradient(l: int, vectors) -> np.ndarray:
    """``dC_lm/dq_alpha``, shape (2l+1, n, 3); exact polynomial derivatives."""
    q = np.atleast_2d(np.asarray(vectors, dtype=float))
    x, y, z = q[:, 0], q[:, 1], q[:, 2]
    r2 = x**2 + y**2 + z**2
    o = np.zeros_like(x)
    one = np.ones_like(x)
    s = lambda a, b, c: np.stack([a, b, c], axis=-1)  # noqa: E731
    if l == 0:
        return np.zeros((1, len(q), 3))
    if l == 1:
        c = np.sqrt(0.75 / np.pi)
        return c * np.stack([s(o, one, o), s(o, o, one), s(one, o, o)])
    if l == 2:
        c = 0.5 * np.sqrt(15.0 / np.pi)
        cz = 0.25 * np.sqrt(5.0 / np.pi)
        cd = 0.25 * np.sqrt(15.0 / np.pi)
        return np.stack([c * s(y, x, o), c * s(o, z, y), cz * s(-2 * x, -2 * y, 4 * z),
                         c * s(z, o, x), cd * s(2 * x, -2 * y, o)])
    if l == 3:
        ca = 0.25 * np.sqrt(17.5 / np.pi)
        cb = 0.5 * np.sqrt(105.0 / np.pi)
        cc = 0.25 * np.sqrt(10.5 / np.pi)
        cdd = 0.25 * np.sqrt(7.0 / np.pi)
        ce = 0.25 * np.sqrt(105.0 / np.pi)
        return np.stack([
            ca * s(6 * x * y, 3 * (x**2 - y**2), o),
            cb * s(y * z, x * z, x * y),
            cc * s(-2 * x * y, 5 * z**2 - r2 - 2 * y**2, 8 * y * z),
            cdd * s(-6 * x * z, -6 * y * z, 9 * z**2 - 3 * r2),
            cc * s(5 * z**2 - r2 - 2 * x**2, -2 * x * y, 8 * x * z),
            ce * s(2 * x * z, -2 * y * z, x**2 - y**2),
            ca * s(3 * (x**2 - y**2), -6 * x * y, o),
        ])
    raise NotImplementedError(f"solid harmonics are implemented up to l={MAX_L}")


@dataclass
class ProjectorSet:
    """Projector matrix of one k-point: ``matrix`` (nproj, npw) complex, ``dij`` real."""

    matrix: np.ndarray
    dij: np.ndarray
    labels: list

    def __len__(self) -> int:
        return len(self.labels)


def projector_layout(symbols, pseudopotentials):
    """Row labels (atom, l, channel, m) and the block-diagonal D, shared by every k."""
    labels, blocks = [], []
    for atom, symbol in enumerate(symbols):
        pseudo = pseudopotentials[symbol]
        atom_labels = []
        for index, proj in enumerate(pseudo.projectors):
            for m_index in range(2 * proj.l + 1):
                atom_labels.append((atom, proj.l, index, m_index - proj.l))
        size = len(atom_labels)
        block = np.zeros((size, size))
        for row, (_, lr, cr, mr) in enumerate(atom_labels):
            for col, (_, lc, cc, mc) in enumerate(atom_labels):
                if lr != lc or mr != mc:
                    continue
                if pseudo.dij is not None:
                    block[row, col] = pseudo.dij[cr, cc]
                elif cr == cc:
                    block[row, col] = pseudo.projectors[cr].energy
        labels.extend(atom_labels)
        blocks.append(block)
    total = sum(len(b) for b in blocks)
    dij = np.zeros((total, total))
    offset = 0
    for b in blocks:
        dij[offset:offset + len(b), offset:offset + len(b)] = b
        offset += len(b)
    return labels, dij


def build_projectors(sphere, positions, symbols, pseudopotentials, volume) -> ProjectorSet:
    kg = sphere.cartesian
    q = np.sqrt(sphere.g2)
    prefactor = 4.0 * np.pi / np.sqrt(volume)
    radial, harmonics = {}, {}
    for symbol, pseudo in pseudopotentials.items():
        for proj in pseudo.projectors:
            radial[(symbol, proj.l, proj.index)] = projector_form_factor(pseudo.grid, proj, q)
            if proj.l not in harmonics:
                harmonics[proj.l] = real_spherical_harmonics(proj.l, kg)
    labels, dij = projector_layout(symbols, pseudopotentials)
    rows = []
    for atom, symbol in enumerate(symbols):
        pseudo = pseudopotentials[symbol]
        phase = np.exp(-1j * (kg @ positions[atom]))
        for proj in pseudo.projectors:
            f = radial[(symbol, proj.l, proj.index)]
            y = harmonics[proj.l]
            for m_index in range(2 * proj.l + 1):
                rows.append(prefactor * (-1j) ** proj.l * y[m_index] * f * phase)
    if not rows:
        return ProjectorSet(np.zeros((0, len(sphere)), dtype=complex), np.zeros((0, 0)), [])
    return ProjectorSet(np.asarray(rows), dij, labels)
