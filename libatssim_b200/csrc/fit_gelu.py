"""Generates the GELU polynomial of the warm-start network (ats_gelu.cuh).

The network's activation is defined as
    g(z) = z (1/2 + z S(x)),   x = 2 z^2 / c^2 - 1,   |z| < c = 4.5
    g(z) = z for z >= c,  0 for z <= -c,
with S a degree-8 polynomial in x: the least-squares Chebyshev fit of
(Phi(z) - 1/2) / z, Phi the standard normal CDF, over z in (0, c] weighted by z^2
(the error of g, not of S), converted to powers of x. g is within 1.2e-4 of the
exact GELU z Phi(z) everywhere (the tanh approximation of GELU is within 5e-4), and
its jump at +-c is 1.5e-5. It costs FMAs only. Run
    python libatssim_b200/csrc/fit_gelu.py
to print the coefficient table and the fit's error.
"""
import math

import numpy as np
from numpy.polynomial import chebyshev as C
from numpy.polynomial import polynomial as P

CUT, DEG = 4.5, 8


def phi(z):
    return 0.5 * (1.0 + np.array([math.erf(v / math.sqrt(2.0)) for v in np.atleast_1d(z)]))


def coefficients():
    z = np.linspace(1e-6, CUT, 40001)
    x = 2.0 * z * z / (CUT * CUT) - 1.0
    w = np.maximum(z * z, 1e-3)
    cf = C.chebfit(x, (phi(z) - 0.5) / z, DEG, w=w)
    return np.float32(C.cheb2poly(cf)).astype(np.float64)  # lowest power first, FP32 values


def gelu(z, coef):
    s = P.polyval(z * z * float(np.float32(2.0 / (CUT * CUT))) - 1.0, coef)
    return np.where(z >= CUT, z, np.where(z <= -CUT, 0.0, z * (0.5 + z * s)))


if __name__ == "__main__":
    c = coefficients()
    z = np.linspace(-8.0, 8.0, 160001)
    print("// max |g - z Phi(z)| = %.2e" % np.max(np.abs(gelu(z, c) - z * phi(z))))
    print("static __constant__ float kGeluPoly[kGeluDeg + 1] = {")
    print(",\n".join("    %.9ef" % v for v in c) + "};")
