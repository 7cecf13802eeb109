"""CGS units and constants of hammurabiX (include/hamunits.h:10-67).

Every value is computed with the same double-precision expression as the
reference header, so Python-side parameter parsing produces bit-identical
CGS values.
"""
import math

erg = 1.
cm = 1.
sec = 1.
Kelvin = 1.

pi = 3.141592653589793238462643383279502884197
halfpi = 1.570796326794896619231321691639751442099
twopi = 6.283185307179586476925286766559005768394
rad = (pi / 180.)
esu = math.sqrt(erg * cm)
m = (1.e2 * cm)
km = (1.e5 * cm)
pc = (3.0856775806e+18 * cm)
kpc = (3.0856775806e+21 * cm)
eV = (1.60217733e-12 * erg)
GeV = (1.e9 * eV)
Hz = (1. / sec)
GHz = (1.e9 * Hz)
MHz = (1.e6 * Hz)
Gauss = math.sqrt(erg / (cm * cm * cm))
muGauss = (1.e-6 * Gauss)
ccm = (cm * cm * cm)
c_light = (2.99792458e+10 * cm / sec)
h_planck = (6.626075540e-27 * erg * sec)
qe = (4.80320425e-10 * esu)
mec2 = (0.51099907e-3 * GeV)
mec = (mec2 / c_light)
kB = (1.380622e-16 * erg / Kelvin)
