"""Independent FP64 growth check — TEST INFRASTRUCTURE ONLY (see oracle/pm.py).

For flat LCDM (w = -1) the growing mode has the closed form
  D(a) ~ E(a) * int_0^a da' / (a' E(a'))^3,
and the kick derivative dGf/da follows from the growth ODE as 3/2 Om D / (a^2 E)
(the relation the reference's test mock spells out, tests/conftest.py:64-86). These
check the product's tabulated ODE solution (jfli_b200.cosmology) to interpolation
accuracy. The normalisation of the fork's tables is parity unpinned.
"""

from __future__ import annotations

import math

import numpy as np
from scipy.integrate import quad


def E(om, a):
    return math.sqrt(om / a**3 + (1.0 - om))


def growth_unnormalised(om, a):
    val = quad(lambda x: 1.0 / (x * E(om, x)) ** 3 if x > 0 else 0.0, 0.0, a, epsabs=0, epsrel=1e-12, limit=200)[0]
    return 2.5 * om * E(om, a) * val


def growth(om, a):
    return growth_unnormalised(om, a) / growth_unnormalised(om, 1.0)


def growth_rate(om, a, h=1e-5):
    return (math.log(growth(om, a * (1 + h))) - math.log(growth(om, a * (1 - h)))) / (
        math.log(1 + h) - math.log(1 - h))


def dGfa(om, a):
    return 1.5 * om * growth(om, a) / (a * a * E(om, a))


def chi(om, a, rh=2997.92458):
    return rh * quad(lambda x: 1.0 / (x * x * E(om, x)), a, 1.0, epsabs=0, epsrel=1e-12)[0]
