"""PBE and PBEsol exchange-correlation in FP64 numpy: the oracle for the GPU GGA path.

Test infrastructure only (imported by tests/). It restates, from the published forms,

* the pointwise functionals of amaterasu ``xc/gga.py:112-254`` (exchange and correlation):
  PBE, J. P. Perdew, K. Burke and M. Ernzerhof, Phys. Rev. Lett. 77, 3865 (1996); PBEsol
  (mu = 10/81, beta = 0.046), Phys. Rev. Lett. 100, 136406 (2008); the local part is the
  Perdew-Wang 1992 correlation (Phys. Rev. B 45, 13244) with the extra-digit ("modified")
  coefficients that PBE is defined on;
* the grid layer of ``xc/driver.py:111-165``: gradients of each spin density, the contracted
  sigma = (grad n_u.grad n_u, grad n_u.grad n_d, grad n_d.grad n_d), and the potential
  v_s = d(n eps)/dn_s - div(2 vsigma_ss grad n_s + vsigma_ud grad n_s'), an unpolarised
  density being split n/2, n/2;
* the spectral gradient and divergence of ``basis/fft.py:288-304`` (multiplication by i G
  with the Nyquist frequency of every even axis set to zero).

The energy density n eps is written in closed form; its derivatives (vrho, vsigma) are taken
by complex-step differentiation, d f/dx = Im f(x + i h) / h, which is exact to rounding for
these analytic expressions and independent of the hand-derived chain rules in the CUDA
kernel. Everything is written in terms of s^2 and t^2 (never |grad n| itself), so the step
is analytic at sigma = 0 too.
"""
from __future__ import annotations

import numpy as np
import scipy.fft as sfft

THRESHOLD = 1e-24                               # vacuum: densities below give zero
C_X = 0.9305257363491000250020102180716672510262  # (3/8)(3/pi)^(1/3) 4^(2/3)
RS_C = 0.6203504908994000166680068120477781673508  # (3/(4 pi))^(1/3)
X2S = 0.1282782438530421943003109254455883701296   # 1 / (2 (6 pi^2)^(1/3))
GAMMA = 0.031090690869654895034                 # (1 - ln 2) / pi^2
KAPPA = 0.804
PARAMS = {"PBE": (0.2195149727645171, 0.06672455060314922),          # (mu, beta)
          "PBESOL": (10.0 / 81.0, 0.046)}
# modified PW92: (A, alpha1, beta1..beta4) for unpolarised, polarised and -alpha_c
PW92 = ((0.0310907, 0.21370, 7.5957, 3.5876, 1.6382, 0.49294),
        (0.01554535, 0.20548, 14.1189, 6.1977, 3.3662, 0.62517),
        (0.0168869, 0.11125, 10.357, 3.6231, 0.88026, 0.49671))
FZ20 = 1.709920934161365617563962776245          # f''(0)
_FZ_DEN = 2.0 ** (4.0 / 3.0) - 2.0


def _key(functional):
    k = functional.strip().upper().replace("-", "").replace("_", "")
    if k not in PARAMS:
        raise ValueError(f"GGA functional {functional!r} is not PBE or PBEsol")
    return k


def _pw92_g(rs, c):
    a, a1, b1, b2, b3, b4 = c
    srs = np.sqrt(rs)
    q = srs * (b1 + srs * (b2 + srs * (b3 + srs * b4)))
    return -2.0 * a * (1.0 + a1 * rs) * np.log1p(1.0 / (2.0 * a * q))


def _pow(x, p):
    return np.exp(p * np.log(x))


def _exchange(n_s, sig, mu):
    """One spin channel's exchange energy density, -C_X n_s^(4/3) F_x(s), with
    F_x = 1 + kappa mu s^2 / (kappa + mu s^2) and s^2 = X2S^2 sigma_ss / n_s^(8/3)
    (exact spin scaling: E_x[n_u, n_d] = (E_x[2 n_u] + E_x[2 n_d]) / 2)."""
    s2 = X2S * X2S * sig / _pow(n_s, 8.0 / 3.0)
    return -C_X * _pow(n_s, 4.0 / 3.0) * (1.0 + KAPPA * mu * s2 / (KAPPA + mu * s2))


def _correlation(nu, nd, sig_tot, beta):
    """n (eps_c^PW92(rs, zeta) + H(rs, zeta, t)) with
    H = gamma phi^3 ln(1 + (beta/gamma) t^2 (1 + A t^2) / (1 + A t^2 + A^2 t^4)),
    A = (beta/gamma) / (exp(-eps_c^PW92 / (gamma phi^3)) - 1), t = |grad n| / (2 phi k_s n)."""
    n = nu + nd
    rs = RS_C / _pow(n, 1.0 / 3.0)
    z = (nu - nd) / n
    fz = (_pow(1.0 + z, 4.0 / 3.0) + _pow(1.0 - z, 4.0 / 3.0) - 2.0) / _FZ_DEN
    g0, g1, g2 = (_pw92_g(rs, c) for c in PW92)
    z4 = z ** 4
    ec_lda = g0 * (1.0 - z4 * fz) + g1 * z4 * fz + g2 * fz * (z4 - 1.0) / FZ20
    phi = 0.5 * (_pow(1.0 + z, 2.0 / 3.0) + _pow(1.0 - z, 2.0 / 3.0))
    phi3 = phi ** 3
    # t^2 = sigma_tot / (n^(8/3) (4 2^(1/3) phi)^2 rs)
    t2 = sig_tot / (_pow(n, 8.0 / 3.0) * (4.0 * 2.0 ** (1.0 / 3.0) * phi) ** 2 * rs)
    A = (beta / GAMMA) / np.expm1(-ec_lda / (GAMMA * phi3))
    At2 = A * t2
    H = GAMMA * phi3 * np.log1p((beta / GAMMA) * t2 * (1.0 + At2) / (1.0 + At2 + At2 * At2))
    return n * (ec_lda + H)


def _dstep(f, args, i):
    """d f / d args[i] by a complex step."""
    x = args[i]
    h = 1e-20 * np.maximum(np.abs(x), 1e-30)
    a2 = list(args)
    a2[i] = x + 1j * h
    return f(*a2).imag / h


def gga_point(rho, sigma, functional="PBE"):
    """libxc layout: rho (npoints, 2), sigma (npoints, 3) -> (eps, vrho (npoints, 2),
    vsigma (npoints, 3)). Points with n <= 1e-24 give zeros; a spin channel at or below
    1e-24 carries no exchange. Derivatives are exact for |zeta| < 1 (both channels
    occupied)."""
    mu, beta = PARAMS[_key(functional)]
    rho = np.atleast_2d(np.asarray(rho, dtype=float))
    sigma = np.atleast_2d(np.asarray(sigma, dtype=float))
    n = rho[:, 0] + rho[:, 1]
    live = n > THRESHOLD
    e = np.zeros_like(n)
    vrho = np.zeros((len(n), 2))
    vsigma = np.zeros((len(n), 3))
    for s in range(2):
        on = live & (rho[:, s] > THRESHOLD)
        args = [np.maximum(rho[:, s], THRESHOLD), np.maximum(sigma[:, 2 * s], 0.0)]
        fx = lambda a, b: _exchange(a, b, mu)  # noqa: E731
        e += np.where(on, fx(*args), 0.0)
        vrho[:, s] += np.where(on, _dstep(fx, args, 0), 0.0)
        vsigma[:, 2 * s] += np.where(on, _dstep(fx, args, 1), 0.0)
    safe = np.where(live, 1.0, 0.0)
    nu = np.where(live, np.maximum(rho[:, 0], 0.0), 0.5)  # placeholders where dead
    nd = np.where(live, np.maximum(rho[:, 1], 0.0), 0.5)
    sig_tot = np.maximum(sigma[:, 0] + 2.0 * sigma[:, 1] + sigma[:, 2], 0.0)
    fc = lambda a, b, c: _correlation(a, b, c, beta)  # noqa: E731
    args = [nu, nd, sig_tot]
    e += safe * fc(*args)
    vrho[:, 0] += safe * _dstep(fc, args, 0)
    vrho[:, 1] += safe * _dstep(fc, args, 1)
    vc = safe * _dstep(fc, args, 2)
    vsigma += np.stack([vc, 2.0 * vc, vc], axis=-1)
    eps = np.where(live, e / np.where(live, n, 1.0), 0.0)
    return eps, vrho, vsigma


def gvectors(shape, cell):
    """Cartesian G of every grid point (natural FFT order), Nyquist frequency zeroed."""
    recip = 2.0 * np.pi * np.linalg.inv(np.asarray(cell, dtype=float)).T
    freqs = []
    for n in shape:
        f = np.fft.fftfreq(n, d=1.0 / n)
        if n % 2 == 0:
            f[n // 2] = 0.0
        freqs.append(f)
    m = np.stack(np.meshgrid(*freqs, indexing="ij"), axis=-1)
    return m @ recip


def gradient(field, cell):
    g = gvectors(field.shape, cell)
    f = sfft.fftn(field)
    return np.stack([sfft.ifftn(1j * g[..., a] * f).real for a in range(3)], axis=-1)


def divergence(vec, cell):
    g = gvectors(vec.shape[:3], cell)
    acc = sum(1j * g[..., a] * sfft.fftn(vec[..., a]) for a in range(3))
    return sfft.ifftn(acc).real


def gga_on_grid(density, cell, functional="PBE"):
    """(E_xc, v_xc (nspin, n1, n2, n3)) for density (nspin, n1, n2, n3) in electrons/Bohr^3."""
    density = np.asarray(density, dtype=float)
    nspin = density.shape[0]
    shape = density.shape[1:]
    spin = np.stack([density[0] / 2, density[0] / 2]) if nspin == 1 else density
    grads = [gradient(spin[s], cell) for s in range(2)]
    flat = [g.reshape(-1, 3) for g in grads]
    sigma = np.stack([np.sum(flat[0] * flat[0], axis=1), np.sum(flat[0] * flat[1], axis=1),
                      np.sum(flat[1] * flat[1], axis=1)], axis=-1)
    rho = spin.reshape(2, -1).T
    eps, vrho, vsigma = gga_point(rho, sigma, functional)
    dv = abs(np.linalg.det(np.asarray(cell, dtype=float))) / np.prod(shape)
    energy = float(np.sum(eps * (rho[:, 0] + rho[:, 1])) * dv)
    pot = vrho.T.reshape(2, *shape).copy()
    vs = vsigma.T.reshape(3, *shape)
    for s in range(2):
        flux = 2.0 * vs[2 * s][..., None] * grads[s] + vs[1][..., None] * grads[1 - s]
        pot[s] -= divergence(flux, cell)
    return energy, pot[:nspin]
