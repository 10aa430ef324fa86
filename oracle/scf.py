"""Density, occupations, mixing and the SCF loop in FP64 numpy (the CPU oracle).

Follows amaterasu ``scf/density.py:35-84``, ``scf/occupations.py:38-244`` (Fermi-Dirac,
Gaussian, Methfessel-Paxton, Marzari-Vanderbilt, fixed), ``scf/mixing.py:48-285``
(Kerker, linear, Pulay, Anderson, Broyden) and ``scf/driver.py:267-464`` (run_scf, NC
branch, symmetry off).
"""
from __future__ import annotations

import numpy as np
import scipy.fft as sfft
from scipy.special import erfc

from .eigen import davidson, random_bands
from .hamiltonian import hamiltonian_apply, kb_energy, wave_to_real
from .potential import hartree, xc_on_grid

MAX_ARG = 200.0


# ------------------------------------------------------------------- density
def compute_density(shape, volume, spheres_miller, weights, wavefunctions, occupations, nspin=1,
                    clip=True):
    degeneracy = 2.0 / nspin
    density = np.zeros((nspin, *shape))
    for spin in range(nspin):
        for ik, (miller, w) in enumerate(zip(spheres_miller, weights)):
            factors = degeneracy * w * occupations[spin, ik]
            active = factors > 1e-12
            if not np.any(active):
                continue
            real = wave_to_real(wavefunctions[spin][ik][active], miller, shape)
            density[spin] += np.einsum("n,n...->...", factors[active], np.abs(real) ** 2)
    density /= volume
    if clip:
        before = density.sum(axis=(-3, -2, -1))
        clipped = np.maximum(density, 0.0)
        after = clipped.sum(axis=(-3, -2, -1))
        scale = np.where(after > 0, before / np.where(after > 0, after, 1.0), 1.0)
        density = clipped * scale[:, None, None, None]
    return density


# --------------------------------------------------------------- occupations
def _hermite_terms(x, order):
    arg = np.minimum(MAX_ARG, x**2)
    hp = np.exp(-arg)
    hd = np.zeros_like(x)
    ni = 0
    a = 1.0 / np.sqrt(np.pi)
    for i in range(1, order + 1):
        hd = 2.0 * x * hp - 2.0 * ni * hd
        ni += 1
        a = -a / (i * 4.0)
        previous = hp
        hp = 2.0 * x * hd - 2.0 * ni * hp
        ni += 1
        yield a, hd, hp, previous, ni


def occupation_function(x, scheme, order=1):
    x = np.asarray(x, dtype=float)
    if scheme == "fermi-dirac":
        return 1.0 / (1.0 + np.exp(np.clip(x, -MAX_ARG, MAX_ARG)))
    if scheme == "marzari-vanderbilt":
        s = x + 1.0 / np.sqrt(2.0)
        return 0.5 * erfc(s) + np.exp(-np.minimum(MAX_ARG, s**2)) / np.sqrt(2.0 * np.pi)
    if scheme in ("gaussian", "fixed"):
        return 0.5 * erfc(x)
    if scheme == "methfessel-paxton":
        r = 0.5 * erfc(x)
        for a, hd, _, _, _ in _hermite_terms(-x, order):
            r = r - a * hd
        return r
    raise ValueError(scheme)


def entropy_function(x, scheme, order=1):
    x = np.asarray(x, dtype=float)
    if scheme == "fermi-dirac":
        f = np.clip(occupation_function(x, scheme), 1e-300, 1.0 - 1e-16)
        return -(f * np.log(f) + (1.0 - f) * np.log1p(-f))
    if scheme == "marzari-vanderbilt":
        s = x + 1.0 / np.sqrt(2.0)
        return s * np.exp(-np.minimum(MAX_ARG, s**2)) / np.sqrt(2.0 * np.pi)
    if scheme in ("gaussian", "fixed"):
        return 0.5 * np.exp(-np.minimum(MAX_ARG, x**2)) / np.sqrt(np.pi)
    if scheme == "methfessel-paxton":
        n = -x
        r = 0.5 * np.exp(-np.minimum(MAX_ARG, n**2)) / np.sqrt(np.pi)
        for a, _, hp, prev, ni in _hermite_terms(n, order):
            r = r + a * (0.5 * hp + ni * prev)
        return r
    raise ValueError(scheme)


def compute_occupations(eigenvalues, weights, nelectrons, scheme="gaussian", smearing=0.0,
                        order=1, nspin=1, tolerance=1e-12):
    eig = np.asarray(eigenvalues, dtype=float)
    weights = np.asarray(weights, dtype=float)
    g = 2.0 / nspin
    if scheme == "fixed" or smearing <= 0.0:
        flat = eig.ravel()
        order_ = np.argsort(flat, kind="stable")
        sw = np.broadcast_to(weights[None, :, None] * g, eig.shape).ravel()[order_]
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
        gap = lumo - homo
        return occ.reshape(eig.shape), 0.5 * (homo + lumo), 0.0, (gap if gap > 0 else None)
    lower = float(eig.min()) - 20.0 * smearing - 1.0
    upper = float(eig.max()) + 20.0 * smearing + 1.0

    def electrons(mu):
        return g * float(np.einsum("k,skn->", weights, occupation_function((eig - mu) / smearing, scheme, order)))

    for _ in range(200):
        mu = 0.5 * (lower + upper)
        if electrons(mu) < nelectrons:
            lower = mu
        else:
            upper = mu
        if upper - lower < tolerance:
            break
    mu = 0.5 * (lower + upper)
    red = (eig - mu) / smearing
    occ = occupation_function(red, scheme, order)
    ent = smearing * g * float(np.einsum("k,skn->", weights, entropy_function(red, scheme, order)))
    gap = None
    if float(np.max(np.minimum(occ, 1.0 - occ))) < 1e-6:
        filled, empty = eig[occ > 0.5], eig[occ <= 0.5]
        if filled.size and empty.size:
            gap = float(empty.min() - filled.max())
    return occ, float(mu), float(ent), (gap if gap is not None and gap > 0 else None)


# -------------------------------------------------------------------- mixing
class Kerker:
    def __init__(self, gvectors, q0, uniform_factor=0.0):
        g2 = np.einsum("...i,...i->...", gvectors, gvectors)
        with np.errstate(invalid="ignore"):
            self.factor = np.where(g2 > 1e-12, g2 / (g2 + q0**2), float(uniform_factor))
        self.q0 = q0

    def _filter(self, f):
        return sfft.ifftn(sfft.fftn(f.astype(complex), norm="forward") * self.factor, norm="forward").real

    def __call__(self, residual):
        if self.q0 <= 0:
            return residual
        if residual.shape[0] == 1:
            return self._filter(residual[0])[None, ...]
        charge = self._filter(residual[0] + residual[1])
        moment = residual[0] - residual[1]
        return np.stack([0.5 * (charge + moment), 0.5 * (charge - moment)])


class Mixer:
    def __init__(self, algorithm="pulay", beta=0.4, history=8, precondition=None, w0=0.01):
        self.algorithm = algorithm
        self.beta = beta
        self.history = min(history, 2) if algorithm == "anderson" else history
        self.precondition = precondition or (lambda r: r)
        self.inputs, self.residuals = [], []
        self.w0 = w0

    def _record(self, n_in, n_out):
        r = n_out - n_in
        self.inputs.append(n_in.copy())
        self.residuals.append(r)
        if len(self.inputs) > self.history:
            del self.inputs[0]
            del self.residuals[0]
        return r

    def _pulay_coefficients(self):
        while True:
            size = len(self.residuals)
            if size == 1:
                return np.ones(1)
            flat = np.array([r.ravel() for r in self.residuals])
            ov = flat @ flat.T
            scale = float(np.trace(ov)) / size
            m = np.ones((size + 1, size + 1))
            m[:size, :size] = ov / scale
            m[size, size] = 0.0
            t = np.zeros(size + 1)
            t[size] = 1.0
            try:
                sol = np.linalg.solve(m, t)
            except np.linalg.LinAlgError:
                pass
            else:
                if np.all(np.isfinite(sol)) and np.max(np.abs(sol[:size])) < 1e4:
                    return sol[:size]
            del self.inputs[0]
            del self.residuals[0]

    def __call__(self, n_in, n_out):
        if self.algorithm == "linear":
            r = self._record(n_in, n_out)
            return n_in + self.beta * self.precondition(r)
        if self.algorithm in ("pulay", "anderson"):
            self._record(n_in, n_out)
            c = self._pulay_coefficients()
            mi = np.einsum("i,i...->...", c, np.array(self.inputs))
            mr = np.einsum("i,i...->...", c, np.array(self.residuals))
            return mi + self.beta * self.precondition(mr)
        if self.algorithm == "broyden":
            r = self._record(n_in, n_out)
            step = self.beta * self.precondition(r)
            if len(self.residuals) < 2:
                return n_in + step
            dfs, dns = [], []
            for i in range(len(self.residuals) - 1):
                d = self.residuals[i + 1] - self.residuals[i]
                nrm = float(np.linalg.norm(d))
                if nrm < 1e-30:
                    continue
                dfs.append(d.ravel() / nrm)
                dns.append((self.inputs[i + 1] - self.inputs[i] + self.beta * self.precondition(d)).ravel() / nrm)
            if not dfs:
                return n_in + step
            df, dn = np.array(dfs), np.array(dns)
            m = df @ df.T + self.w0**2 * np.eye(len(df))
            gamma = np.linalg.solve(m, df @ r.ravel())
            return n_in + step - np.einsum("i,i...->...", gamma, dn).reshape(n_in.shape)
        raise ValueError(self.algorithm)


# ------------------------------------------------------------------ SCF loop
def run_scf(system_arrays, *, occupation_scheme="fixed", smearing=0.0, tol_energy_ev=1e-6,
            tol_density=1e-7, max_steps=100, mixing="pulay", beta=0.4, history=8, q0=1.5,
            hartree_in_ev=27.211386024367243, log=None):
    """SCF on plain arrays (symmetry off, nspin=1, NC). ``system_arrays`` holds: shape,
    volume, natoms, nelectrons, nbands, kpoints_weights, spheres (list of dicts with miller,
    kinetic, proj, dij), v_local, rho0, ewald, density_miller, density_g2, gvectors."""
    s = system_arrays
    shape = tuple(s["shape"])
    dv = s["volume"] / np.prod(shape)
    rho = np.array(s["rho0"], dtype=float)
    nk = len(s["spheres"])
    wfs = [[random_bands(len(sp["kinetic"]), s["nbands"], sp["kinetic"], seed=12345 + ik)
            for ik, sp in enumerate(s["spheres"])]]
    mixer = Mixer(mixing, beta, history, Kerker(s["gvectors"], q0))
    threshold = tol_energy_ev * s["natoms"] / hartree_in_ev
    prev = np.inf
    residual = np.inf
    history_rows = []
    it = 0
    for it in range(1, max_steps + 1):
        e_h, v_h = hartree(rho[0], shape, s["density_miller"], s["density_g2"], s["volume"])
        e_xc, v_xc = xc_on_grid(rho, dv)
        veff = s["v_local"] + v_h + v_xc[0]
        tol = float(np.clip(1e-3 * min(residual, 1.0), 1e-11, 1e-6))
        maxit = 40 if it == 1 else 20
        eig = np.empty((1, nk, s["nbands"]))
        for ik, sp in enumerate(s["spheres"]):
            res = davidson(lambda b, sp=sp: hamiltonian_apply(b, sp["miller"], shape, sp["kinetic"], veff,
                                                              sp["proj"], sp["dij"]),
                           wfs[0][ik], sp["kinetic"], tolerance=tol, max_iterations=maxit)
            eig[0, ik] = res.eigenvalues
            wfs[0][ik] = res.coefficients
        occ, fermi, ent, gap = compute_occupations(eig, s["weights"], s["nelectrons"], occupation_scheme,
                                                   smearing)
        rho_out = compute_density(shape, s["volume"], [sp["miller"] for sp in s["spheres"]], s["weights"],
                                  wfs, occ)
        e_h2, _ = hartree(rho_out[0], shape, s["density_miller"], s["density_g2"], s["volume"])
        e_xc2, _ = xc_on_grid(rho_out, dv)
        kin = sum(2.0 * s["weights"][ik] * float(occ[0, ik] @ (np.abs(wfs[0][ik]) ** 2 @ sp["kinetic"]))
                  for ik, sp in enumerate(s["spheres"]))
        enl = sum(kb_energy(wfs[0][ik], sp["proj"], sp["dij"], 2.0 * s["weights"][ik] * occ[0, ik])
                  for ik, sp in enumerate(s["spheres"]))
        eloc = float(np.sum(s["v_local"] * rho_out[0])) * dv
        total = kin + eloc + e_h2 + e_xc2 + enl + s["ewald"]
        free = total - ent
        residual = float(np.sum(np.abs(rho_out - rho))) * dv / s["nelectrons"]
        delta = free - prev
        history_rows.append((free, residual))
        if log:
            log(f"{it:4d} {free:.12f} {delta:.3e} {residual:.3e}")
        if it > 1 and abs(delta) < threshold and residual < tol_density:
            break
        prev = free
        rho = mixer(rho, rho_out)
    return dict(iterations=it, free_energy=free, total=total, eigenvalues=eig, occupations=occ,
                fermi=fermi, density=rho_out, wavefunctions=wfs, history=history_rows,
                energies=dict(kinetic=kin, local=eloc, hartree=e_h2, xc=e_xc2, nonlocal_=enl,
                              ewald=s["ewald"], entropy=ent))
