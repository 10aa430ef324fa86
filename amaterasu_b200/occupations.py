"""Occupations, Fermi level and smearing entropy (host FP64; nspin*nk*nbands numbers).

Restates amaterasu ``scf/occupations.py:38-244``: Fermi-Dirac, Gaussian,
Methfessel-Paxton (Hermite recursion), Marzari-Vanderbilt and fixed filling; the Fermi
level by bisection to 1e-12 (at most 200 halvings) on [min - 20 sigma - 1, max + 20 sigma + 1];
the gap reported only when no state is partially filled.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
from scipy.special import erfc

_MAX = 200.0
SCHEMES = ("fermi-dirac", "gaussian", "methfessel-paxton", "marzari-vanderbilt", "tetrahedron", "fixed")


def _mp_terms(x, order):
    hp = np.exp(-np.minimum(_MAX, x**2))
    hd = np.zeros_like(x)
    ni = 0
    a = 1.0 / np.sqrt(np.pi)
    for i in range(1, order + 1):
        hd = 2.0 * x * hp - 2.0 * ni * hd
        ni += 1
        a = -a / (i * 4.0)
        prev = hp
        hp = 2.0 * x * hd - 2.0 * ni * hp
        ni += 1
        yield a, hd, hp, prev, ni


def occupation_function(x, scheme: str, order: int = 1):
    x = np.asarray(x, dtype=float)
    if scheme == "fermi-dirac":
        return 1.0 / (1.0 + np.exp(np.clip(x, -_MAX, _MAX)))
    if scheme == "marzari-vanderbilt":
        s = x + 1.0 / np.sqrt(2.0)
        return 0.5 * erfc(s) + np.exp(-np.minimum(_MAX, s**2)) / np.sqrt(2.0 * np.pi)
    if scheme in ("gaussian", "tetrahedron", "fixed"):
        return 0.5 * erfc(x)
    if scheme == "methfessel-paxton":
        out = 0.5 * erfc(x)
        for a, hd, _, _, _ in _mp_terms(-x, order):
            out = out - a * hd
        return out
    raise ValueError(f"unknown smearing scheme {scheme!r}; available: {', '.join(SCHEMES)}")


def entropy_function(x, scheme: str, order: int = 1):
    x = np.asarray(x, dtype=float)
    if scheme == "fermi-dirac":
        f = np.clip(occupation_function(x, scheme), 1e-300, 1.0 - 1e-16)
        return -(f * np.log(f) + (1.0 - f) * np.log1p(-f))
    if scheme == "marzari-vanderbilt":
        s = x + 1.0 / np.sqrt(2.0)
        return s * np.exp(-np.minimum(_MAX, s**2)) / np.sqrt(2.0 * np.pi)
    if scheme in ("gaussian", "tetrahedron", "fixed"):
        return 0.5 * np.exp(-np.minimum(_MAX, x**2)) / np.sqrt(np.pi)
    if scheme == "methfessel-paxton":
        n = -x
        out = 0.5 * np.exp(-np.minimum(_MAX, n**2)) / np.sqrt(np.pi)
        for a, _, hp, prev, ni in _mp_terms(n, order):
            out = out + a * (0.5 * hp + ni * prev)
        return out
    raise ValueError(f"unknown smearing scheme {scheme!r}; available: {', '.join(SCHEMES)}")


@dataclass
class OccupationResult:
    occupations: np.ndarray
    fermi_level: float
    entropy_term: float
    gap: float | None
    magnetization: float

    @property
    def is_metallic(self) -> bool:
        return self.gap is None


def compute_occupations(eigenvalues, weights, nelectrons, *, scheme="gaussian", smearing=0.0, order=1,
                        nspin=1, tolerance=1e-12) -> OccupationResult:
    eig = np.asarray(eigenvalues, dtype=float)
    if eig.ndim != 3:
        raise ValueError(f"eigenvalues must be (nspin, nk, nbands), got {eig.shape}")
    w = np.asarray(weights, dtype=float)
    g = 2.0 / nspin
    if scheme == "tetrahedron":
        raise NotImplementedError("the tetrahedron method is not implemented")
    if scheme == "fixed" or smearing <= 0.0:
        flat = eig.ravel()
        order_ = np.argsort(flat, kind="stable")
        sw = np.broadcast_to(w[None, :, None] * g, eig.shape).ravel()[order_]
        cum = np.cumsum(sw)
        occ = np.zeros_like(flat)
        full = cum <= nelectrons + 1e-12
        occ[order_[full]] = 1.0
        b = int(np.count_nonzero(full))
        if b < len(order_):
            rem = nelectrons - (cum[b - 1] if b else 0.0)
            occ[order_[b]] = max(0.0, rem / sw[b])
        homo = flat[order_[max(b - 1, 0)]]
        lumo = flat[order_[b]] if b < len(order_) else homo
        occupations, fermi, gap, ent = occ.reshape(eig.shape), 0.5 * (homo + lumo), lumo - homo, 0.0
    else:
        lo = float(eig.min()) - 20.0 * smearing - 1.0
        hi = float(eig.max()) + 20.0 * smearing + 1.0

        def count(mu):
            return g * float(np.einsum("k,skn->", w, occupation_function((eig - mu) / smearing, scheme, order)))

        if count(hi) < nelectrons - 1e-9:
            raise ValueError(f"only {count(hi):.4f} of {nelectrons:g} electrons fit in {eig.shape[2]} bands")
        for _ in range(200):
            mu = 0.5 * (lo + hi)
            if count(mu) < nelectrons:
                lo = mu
            else:
                hi = mu
            if hi - lo < tolerance:
                break
        fermi = 0.5 * (lo + hi)
        red = (eig - fermi) / smearing
        occupations = occupation_function(red, scheme, order)
        ent = smearing * g * float(np.einsum("k,skn->", w, entropy_function(red, scheme, order)))
        gap = None
        if float(np.max(np.minimum(occupations, 1.0 - occupations))) < 1e-6:
            filled, empty = eig[occupations > 0.5], eig[occupations <= 0.5]
            if filled.size and empty.size:
                gap = float(empty.min() - filled.max())
    per_spin = g * np.einsum("k,skn->s", w, occupations)
    mag = float(per_spin[0] - per_spin[1]) if nspin == 2 else 0.0
    return OccupationResult(occupations, float(fermi), float(ent),
                            None if gap is None or gap <= 0 else float(gap), mag)
