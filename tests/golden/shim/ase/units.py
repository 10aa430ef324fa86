"""Unit constants derived from the CODATA 2014 recommended values, the way ``ase.units``
derives them, so that the reference's ``units.py`` sees the numbers it expects."""
from math import pi

__codata_version__ = "2014"
_c = 299792458.0
_mu0 = 4.0e-7 * pi
_eps0 = 1.0 / _mu0 / _c**2
_hplanck = 6.626070040e-34
_hbar = _hplanck / (2.0 * pi)
_e = 1.6021766208e-19
_me = 9.10938356e-31
_k = 1.38064852e-23
_amu = 1.660539040e-27

Ang = Angstrom = 1.0
eV = 1.0
Bohr = 4.0e10 * pi * _eps0 * _hbar**2 / _me / _e**2
Hartree = Ha = _me * _e**3 / 16.0 / pi**2 / _eps0**2 / _hbar**2
Ry = Rydberg = Hartree / 2.0
J = 1.0 / _e
Pascal = (1.0 / _e) / 1e30
GPa = 1e9 * Pascal
kB = _k / _e
