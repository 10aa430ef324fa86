"""Band occupations, Fermi level and smearing entropy (host FP64: nspin x nk x nbands numbers).

Stands in for amaterasu ``scf/occupations.py:157-244`` (``compute_occupations``). The
smearing functions are written from their published forms, with x = (e - mu) / sigma:

* Fermi-Dirac: f = 1 / (1 + e^x); the entropy term s = -[f ln f + (1 - f) ln(1 - f)],
  evaluated as |x| sigmoid(-|x|) + ln(1 + e^-|x|), which is exact and never takes ln 0;
* Gaussian: f = erfc(x) / 2, s = e^{-x^2} / (2 sqrt(pi));
* Methfessel-Paxton of order N (Phys. Rev. B 40, 3616 (1989)):
  f = erfc(x)/2 + sum_{n=1}^{N} A_n H_{2n-1}(x) e^{-x^2},  s = A_N H_{2N}(x) e^{-x^2} / 2,
  A_n = (-1)^n / (n! 4^n sqrt(pi)), H the physicists' Hermite polynomials;
* Marzari-Vanderbilt cold smearing (Phys. Rev. Lett. 82, 3296 (1999)), with u = x + 1/sqrt(2):
  f = erfc(u)/2 + e^{-u^2} / sqrt(2 pi),  s = u e^{-u^2} / sqrt(2 pi);
* fixed: bands filled in energy order (the state at the boundary fractionally).

The Fermi level solves N(mu) = N_e by bisection on [min e - 20 sigma - 1, max e + 20 sigma + 1]
to 1e-12 Ha (at most 200 halvings): the reference's bracket and tolerance, kept so that in a
gap, where N(mu) is flat, the level lands where the reference's does. A gap is reported when
no state is partially occupied (every occupation within 1e-6 of 0 or 1).
"""
from __future__ import annotations

from dataclasses import dataclass
from math import factorial, pi, sqrt

import numpy as np
from scipy.special import erfc, expit

SCHEMES = ("fermi-dirac", "gaussian", "methfessel-paxton", "marzari-vanderbilt", "tetrahedron", "fixed")
_SQRT_PI = sqrt(pi)


def _gauss(x):
    return np.exp(-np.minimum(x * x, 700.0))


def _hermite(n: int, x):
    """H_n(x) (physicists'), by the three-term recurrence H_{k+1} = 2x H_k - 2k H_{k-1}."""
    h_prev, h = np.ones_like(x), 2.0 * x
    if n == 0:
        return h_prev
    for k in range(1, n):
        h_prev, h = h, 2.0 * x * h - 2.0 * k * h_prev
    return h


def _mp_coefficient(n: int) -> float:
    return (-1.0) ** n / (factorial(n) * 4.0 ** n * _SQRT_PI)


def _unknown(scheme):
    return ValueError(f"smearing scheme {scheme!r} is not one of: {', '.join(SCHEMES)}")


def occupation_function(x, scheme: str, order: int = 1):
    x = np.asarray(x, dtype=float)
    if scheme == "fermi-dirac":
        return expit(-x)
    if scheme in ("gaussian", "tetrahedron", "fixed"):
        return 0.5 * erfc(x)
    if scheme == "methfessel-paxton":
        f = 0.5 * erfc(x)
        g = _gauss(x)
        for n in range(1, order + 1):
            f = f + _mp_coefficient(n) * _hermite(2 * n - 1, x) * g
        return f
    if scheme == "marzari-vanderbilt":
        u = x + 1.0 / sqrt(2.0)
        return 0.5 * erfc(u) + _gauss(u) / sqrt(2.0 * pi)
    raise _unknown(scheme)


def entropy_function(x, scheme: str, order: int = 1):
    """The dimensionless entropy term s(x); -TS = sigma * sum w s."""
    x = np.asarray(x, dtype=float)
    if scheme == "fermi-dirac":
        a = np.abs(x)
        return a * expit(-a) + np.log1p(np.exp(-a))
    if scheme in ("gaussian", "tetrahedron", "fixed"):
        return 0.5 * _gauss(x) / _SQRT_PI
    if scheme == "methfessel-paxton":
        return 0.5 * _mp_coefficient(order) * _hermite(2 * order, x) * _gauss(x)
    if scheme == "marzari-vanderbilt":
        u = x + 1.0 / sqrt(2.0)
        return u * _gauss(u) / sqrt(2.0 * pi)
    raise _unknown(scheme)


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


def _fixed_filling(eig, weights, nelectrons, degeneracy):
    """Aufbau filling in energy order; returns (occupations, Fermi level, HOMO-LUMO gap)."""
    flat = eig.ravel()
    order = np.argsort(flat, kind="stable")
    capacity = np.broadcast_to(weights[None, :, None] * degeneracy, eig.shape).ravel()[order]
    filled_to = np.cumsum(capacity)
    full = filled_to <= nelectrons + 1e-12
    occ = np.zeros_like(flat)
    occ[order[full]] = 1.0
    nfull = int(np.count_nonzero(full))
    if nfull < len(order):  # the boundary state takes what is left
        left = nelectrons - (filled_to[nfull - 1] if nfull else 0.0)
        occ[order[nfull]] = max(0.0, left / capacity[nfull])
    homo = flat[order[max(nfull - 1, 0)]]
    lumo = flat[order[nfull]] if nfull < len(order) else homo
    return occ.reshape(eig.shape), 0.5 * (homo + lumo), lumo - homo


def compute_occupations(eigenvalues, weights, nelectrons, *, scheme="gaussian", smearing=0.0, order=1,
                        nspin=1, tolerance=1e-12) -> OccupationResult:
    eig = np.asarray(eigenvalues, dtype=float)
    if eig.ndim != 3:
        raise ValueError(f"eigenvalues must be (nspin, nk, nbands), got {eig.shape}")
    w = np.asarray(weights, dtype=float)
    degeneracy = 2.0 / nspin
    if scheme == "tetrahedron":
        raise NotImplementedError("the tetrahedron method is not implemented; use a smearing scheme")
    if scheme not in SCHEMES:
        raise _unknown(scheme)
    if scheme == "fixed" or smearing <= 0.0:
        occupations, fermi, gap = _fixed_filling(eig, w, nelectrons, degeneracy)
        entropy = 0.0
    else:
        def count(mu):
            return degeneracy * float(np.sum(w[None, :, None] * occupation_function((eig - mu) / smearing,
                                                                                    scheme, order)))

        lo = float(eig.min()) - 20.0 * smearing - 1.0
        hi = float(eig.max()) + 20.0 * smearing + 1.0
        if count(hi) < nelectrons - 1e-9:
            raise ValueError(f"only {count(hi):.4f} of {nelectrons:g} electrons fit in {eig.shape[2]} bands; "
                             "raise occupations.nbands")
        halvings = 0
        while hi - lo >= tolerance and halvings < 200:
            mid = 0.5 * (lo + hi)
            if count(mid) < nelectrons:
                lo = mid
            else:
                hi = mid
            halvings += 1
        fermi = 0.5 * (lo + hi)
        x = (eig - fermi) / smearing
        occupations = occupation_function(x, scheme, order)
        entropy = smearing * degeneracy * float(np.sum(w[None, :, None] * entropy_function(x, scheme, order)))
        gap = None
        if float(np.max(np.minimum(occupations, 1.0 - occupations))) < 1e-6:
            occ_states, empty_states = eig[occupations > 0.5], eig[occupations <= 0.5]
            if occ_states.size and empty_states.size:
                gap = float(empty_states.min() - occ_states.max())
    per_spin = degeneracy * np.einsum("k,skn->s", w, occupations)
    magnetization = float(per_spin[0] - per_spin[1]) if nspin == 2 else 0.0
    return OccupationResult(occupations, float(fermi), float(entropy),
                            None if gap is None or gap <= 0 else float(gap), magnetization)
