"""Norm-conserving pseudopotentials: the in-memory model, a UPF v2 reader, and the
synthetic analytic dataset the benchmark cells use.

Conventions follow the reference (amaterasu ``pseudo/base.py:1-40``): radii in Bohr,
energies in Hartree, projectors stored as ``r*beta_l(r)`` with ``integral p^2 dr = 1``,
densities stored as ``4 pi r^2 rho(r)``. UPF files are in Rydberg, so ``PP_LOCAL`` and
``PP_DIJ`` are halved on load (``pseudo/readers/upf.py:173-174,205``).
"""
from __future__ import annotations

import math
import xml.etree.ElementTree as ET
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np
from scipy.integrate import simpson
from scipy.special import erf

from .units import RYDBERG_IN_HARTREE

__all__ = [
    "NCPseudopotential",
    "Projector",
    "RadialGrid",
    "read_upf",
    "synthetic_silicon_upf",
    "write_synthetic_upf",
]


@dataclass(frozen=True)
class RadialGrid:
    """Radial mesh with the quadrature every radial integral uses.

    Simpson's rule over the index with ``dr/di`` as Jacobian when the file ships it,
    else Simpson in ``r`` (reference ``pseudo/base.py:130-144``).
    """

    r: np.ndarray
    dr_di: np.ndarray | None = None

    def __len__(self) -> int:
        return len(self.r)

    def integrate(self, values, axis: int = -1):
        values = np.asarray(values, dtype=float)
        if self.dr_di is not None and len(self.dr_di) == len(self.r):
            total = simpson(values * self.dr_di, dx=1.0, axis=axis)
        else:
            total = simpson(values, x=self.r, axis=axis)
        return float(total) if values.ndim == 1 else total

    def weights(self) -> np.ndarray:
        """Quadrature weights w with ``integrate(f) == sum(w * f)`` up to rounding."""
        n = len(self.r)
        eye = np.eye(n)
        return np.asarray(self.integrate(eye, axis=-1), dtype=float)


@dataclass(frozen=True)
class Projector:
    """One Kleinman-Bylander channel: ``r*beta_l(r)`` and its energy in Hartree."""

    l: int
    index: int
    energy: float
    values: np.ndarray


@dataclass
class NCPseudopotential:
    symbol: str
    valence_charge: float
    grid: RadialGrid
    local_potential: np.ndarray
    projectors: list[Projector]
    dij: np.ndarray | None = None
    valence_density: np.ndarray | None = None
    core_density: np.ndarray | None = None
    xc_functional: str | None = None
    source: str = ""
    extra: dict = field(default_factory=dict)

    @property
    def has_core_correction(self) -> bool:
        return self.core_density is not None

    @property
    def n_projector_rows(self) -> int:
        """Rows this species contributes to the projector matrix (sum of 2l+1)."""
        return sum(2 * p.l + 1 for p in self.projectors)


def _floats(element, name: str, source: str) -> np.ndarray:
    if element is None or element.text is None:
        raise ValueError(f"{source}: required block {name} is missing or empty")
    return np.array(element.text.split(), dtype=float)


def read_upf(path) -> NCPseudopotential:
    """Read the norm-conserving content of a UPF v2 file.

    Mirrors reference ``pseudo/readers/upf.py:132-264`` for the blocks the NC path uses:
    PP_MESH (PP_R, PP_RAB), PP_LOCAL (Ry), PP_BETA.n (``r*beta``), PP_DIJ (Ry),
    PP_RHOATOM (``4 pi r^2 rho``) and PP_NLCC (bare ``rho_c``).
    """
    path = Path(path)
    source = path.name
    root = ET.fromstring(path.read_text(encoding="utf-8"))
    if not root.tag.startswith("UPF"):
        raise ValueError(f"{source}: root element is <{root.tag}>, expected <UPF>")
    header = root.find("PP_HEADER")
    if header is None:
        raise ValueError(f"{source}: no PP_HEADER block")
    attrs = {k: v.strip() for k, v in header.attrib.items()}
    symbol = attrs.get("element", path.stem.split(".")[0]).strip()
    if attrs.get("has_so", "F").upper() in ("T", "TRUE", ".TRUE."):
        raise NotImplementedError(f"{source}: spin-orbit datasets are not supported")
    valence_charge = float(attrs["z_valence"])
    mesh = root.find("PP_MESH")
    radii = _floats(mesh.find("PP_R") if mesh is not None else None, "PP_MESH/PP_R", source)
    rab = mesh.find("PP_RAB") if mesh is not None else None
    dr_di = _floats(rab, "PP_MESH/PP_RAB", source) if rab is not None else None
    grid = RadialGrid(r=np.ascontiguousarray(radii), dr_di=dr_di)
    local = _floats(root.find("PP_LOCAL"), "PP_LOCAL", source) * RYDBERG_IN_HARTREE

    projectors: list[Projector] = []
    dij = None
    nonlocal_block = root.find("PP_NONLOCAL")
    if nonlocal_block is not None:
        betas = sorted(
            (e for e in nonlocal_block if e.tag.startswith("PP_BETA")),
            key=lambda e: int(e.tag.split(".")[-1]) if "." in e.tag else 0,
        )
        per_l: dict[int, int] = {}
        for element in betas:
            l = int(element.attrib.get("angular_momentum", 0))
            values = np.array(element.text.split(), dtype=float)
            if len(values) < len(radii):
                values = np.concatenate([values, np.zeros(len(radii) - len(values))])
            index = per_l.get(l, 0)
            per_l[l] = index + 1
            projectors.append(Projector(l, index, 0.0, np.ascontiguousarray(values[: len(radii)])))
        dij_element = nonlocal_block.find("PP_DIJ")
        if dij_element is not None and projectors:
            count = len(projectors)
            flat = _floats(dij_element, "PP_DIJ", source) * RYDBERG_IN_HARTREE
            if flat.size != count * count:
                raise ValueError(f"{source}: PP_DIJ holds {flat.size} numbers, expected {count}x{count}")
            dij = flat.reshape(count, count)
            projectors = [Projector(p.l, p.index, float(dij[i, i]), p.values)
                          for i, p in enumerate(projectors)]
    declared = int(attrs.get("number_of_proj", 0))
    if declared and declared != len(projectors):
        raise ValueError(f"{source}: PP_HEADER declares {declared} projectors, found {len(projectors)}")
    rho = root.find("PP_RHOATOM")
    valence_density = np.ascontiguousarray(_floats(rho, "PP_RHOATOM", source)) if rho is not None else None
    nlcc = root.find("PP_NLCC")
    core_density = (np.ascontiguousarray(_floats(nlcc, "PP_NLCC", source) * 4.0 * np.pi * radii**2)
                    if nlcc is not None else None)
    return NCPseudopotential(
        symbol=symbol, valence_charge=valence_charge, grid=grid,
        local_potential=np.ascontiguousarray(local), projectors=projectors, dij=dij,
        valence_density=valence_density, core_density=core_density,
        xc_functional=attrs.get("functional"), source=str(path),
    )


# --------------------------------------------------------------------- synthetic dataset
def synthetic_silicon_upf(*, z: float = 4.0, rloc: float = 0.44, rc: float = 1.0,
                          d_s: float = 3.0, d_p: float = 1.5, rmax: float = 12.0,
                          npoints: int = 1201, density_width2: float = 1.5) -> str:
    """UPF v2 text of the analytic silicon-like dataset the benchmark cells use.

    * local part ``V(r) = -Z erf(r/rloc)/r`` (limit ``-2Z/(sqrt(pi) rloc)`` at r=0);
    * one s and one p KB projector, ``beta_l(r) ~ r^l exp(-r^2/(2 rc^2))``, stored as
      ``r*beta`` normalised analytically to ``integral (r beta)^2 dr = 1``;
    * ``D_s``, ``D_p`` in Hartree (written in Rydberg, as UPF requires);
    * an atomic valence density ``4 pi r^2 rho = N r^2 exp(-r^2/w)`` normalised to Z.

    The radial mesh is uniform, ``r = 0 ... rmax`` with ``npoints`` points.
    """
    r = np.linspace(0.0, rmax, npoints)
    step = r[1] - r[0]
    safe = np.where(r > 0, r, 1.0)
    v = np.where(r > 0, -z * erf(r / rloc) / safe, -2.0 * z / (math.sqrt(math.pi) * rloc))
    betas = []
    for l in (0, 1):
        # integral_0^inf r^(2l+2) exp(-r^2/rc^2) dr = Gamma(l + 3/2)/2 * rc^(2l+3)
        norm2 = math.gamma(l + 1.5) / 2.0 * rc ** (2 * l + 3)
        betas.append(r ** (l + 1) * np.exp(-(r**2) / (2.0 * rc**2)) / math.sqrt(norm2))
    # integral r^2 exp(-r^2/w) dr = sqrt(pi)/4 * w^(3/2)
    rho = z * r**2 * np.exp(-(r**2) / density_width2) / (math.sqrt(math.pi) / 4.0 * density_width2**1.5)

    def block(values):
        return "\n".join("  ".join(f"{x:.16e}" for x in values[i:i + 4]) for i in range(0, len(values), 4))

    ry = 1.0 / RYDBERG_IN_HARTREE
    return f"""<UPF version="2.0.1">
  <PP_INFO>analytic silicon-like norm-conserving dataset (synthetic)</PP_INFO>
  <PP_HEADER element="Si" pseudo_type="NC" relativistic="scalar" is_ultrasoft="F" is_paw="F"
     has_so="F" core_correction="F" functional="SLA PZ NOGX NOGC" z_valence="{z}" l_max="1"
     l_local="-1" mesh_size="{npoints}" number_of_wfc="0" number_of_proj="2"/>
  <PP_MESH dx="{step}" mesh="{npoints}">
    <PP_R>
{block(r)}
    </PP_R>
    <PP_RAB>
{block(np.full_like(r, step))}
    </PP_RAB>
  </PP_MESH>
  <PP_LOCAL>
{block(v * ry)}
  </PP_LOCAL>
  <PP_NONLOCAL>
    <PP_BETA.1 index="1" angular_momentum="0" cutoff_radius_index="{npoints}">
{block(betas[0])}
    </PP_BETA.1>
    <PP_BETA.2 index="2" angular_momentum="1" cutoff_radius_index="{npoints}">
{block(betas[1])}
    </PP_BETA.2>
    <PP_DIJ>
{d_s * ry:.16e} 0.0 0.0 {d_p * ry:.16e}
    </PP_DIJ>
  </PP_NONLOCAL>
  <PP_RHOATOM>
{block(rho)}
  </PP_RHOATOM>
</UPF>
"""


def write_synthetic_upf(path, **kwargs) -> Path:
    path = Path(path)
    path.write_text(synthetic_silicon_upf(**kwargs), encoding="utf-8")
    return path
