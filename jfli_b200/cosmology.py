"""FP64 host-side cosmology: background, linear growth (1st and 2nd order), comoving
distances and the Eisenstein-Hu linear matter power spectrum.

These are the coefficient tables the particle-mesh kernels consume (growth and
time-step factors, P_lin). The reference takes them from forks of jax_cosmo and JaxPM
(`jaxpm.growth.{E, Gf, dGfa, gp, growth_factor}` imported at pm/solvers.py:8-9 and
pm/interp.py:13-14; `jc.power.linear_matter_power` at initial.py:172;
`jc.background.{radial_comoving_distance, a_of_chi}` at pm/_resolve_geometry.py:78 and
utils.py:228). This module restates the published algorithms those packages implement:

* flat w0-wa CDM background without radiation, E(a)^2 = Om a^-3 + Ok a^-2 + Ode a^f(a);
* the linear growth ODE in the scale factor, D'' + q D' - r D = 0 with
  q = (2 - (Om(a) + (1 + 3 w) Ode(a)) / 2) / a and r = 3/2 Om(a) / a^2, and the
  second-order one D2'' + q D2' - r D2 = -r D1^2, integrated from matter domination
  (D1 = a, D2 = -3/7 a^2) on a table of 128 log-spaced scale factors in [1e-3, 1],
  normalised to 1 at a = 1 and read back by linear interpolation;
* the FastPM time-integration factors Gp = D, gp = dD/da, Gf = a^3 E dD/da and
  dGfa = dGf/da (the growth ODE itself), as the test mock at tests/conftest.py:64-86
  spells out;
* chi(a) = c/H0 * int_a^1 da' / (a'^2 E(a')) on 256 log-spaced scale factors;
* Eisenstein & Hu (1998, ApJ 496, 605) transfer function with baryon oscillations,
  P(k) = A k^ns T(k)^2 D(a)^2 normalised to sigma8 with a top-hat of 8 Mpc/h.

Everything here is NumPy float64 and runs once per cosmology (results are cached).
"""

from __future__ import annotations

import dataclasses
import functools
import math

import numpy as np
from scipy.integrate import odeint

RH = 2997.92458  # Hubble radius c/H0 in Mpc/h
TCMB = 2.7255


@dataclasses.dataclass(frozen=True)
class Cosmology:
    """Cosmological parameters (jax_cosmo.Cosmology field names)."""

    Omega_c: float
    Omega_b: float
    h: float
    n_s: float
    sigma8: float
    Omega_k: float = 0.0
    w0: float = -1.0
    wa: float = 0.0

    @property
    def Omega_m(self) -> float:
        return self.Omega_c + self.Omega_b

    @property
    def Omega_de(self) -> float:
        return 1.0 - self.Omega_m - self.Omega_k

    def replace(self, **kw) -> "Cosmology":
        return dataclasses.replace(self, **kw)


def Planck18(**overrides) -> Cosmology:
    """Planck 2018 parameters as in jax_cosmo.Planck18."""
    p = dict(Omega_c=0.2607, Omega_b=0.0490, h=0.6766, n_s=0.9665, sigma8=0.8102, Omega_k=0.0, w0=-1.0, wa=0.0)
    p.update(overrides)
    return Cosmology(**p)


# ----------------------------------------------------------------------------- background
def _f_de(c: Cosmology, a):
    a = np.asarray(a, dtype=np.float64)
    return -3.0 * (1.0 + c.w0 + c.wa) + 3.0 * c.wa * (a - 1.0) / np.log(a)


def w(c: Cosmology, a):
    a = np.asarray(a, dtype=np.float64)
    return c.w0 + c.wa * (1.0 - a)


def Esqr(c: Cosmology, a):
    a = np.asarray(a, dtype=np.float64)
    if c.wa == 0.0:
        de = c.Omega_de * a ** (-3.0 * (1.0 + c.w0))
    else:
        de = c.Omega_de * a ** _f_de(c, a)
    return c.Omega_m * a ** -3 + c.Omega_k * a ** -2 + de


def E(c: Cosmology, a):
    return np.sqrt(Esqr(c, a))


def dEa(c: Cosmology, a, eps: float = 1e-6):
    """dE/da (analytic for constant w, centred difference otherwise)."""
    a = np.asarray(a, dtype=np.float64)
    if c.wa == 0.0:
        de = -3.0 * (1.0 + c.w0) * c.Omega_de * a ** (-3.0 * (1.0 + c.w0) - 1.0)
        dE2 = -3.0 * c.Omega_m * a ** -4 - 2.0 * c.Omega_k * a ** -3 + de
        return 0.5 * dE2 / E(c, a)
    return (E(c, a * (1 + eps)) - E(c, a * (1 - eps))) / (2 * eps * a)


def Omega_m_a(c: Cosmology, a):
    a = np.asarray(a, dtype=np.float64)
    return c.Omega_m * a ** -3 / Esqr(c, a)


def Omega_de_a(c: Cosmology, a):
    a = np.asarray(a, dtype=np.float64)
    return (Esqr(c, a) - c.Omega_m * a ** -3 - c.Omega_k * a ** -2) / Esqr(c, a)


# ------------------------------------------------------------------- table interpolation
def interp(x, xp, fp):
    """Linear interpolation with linear extrapolation past both ends (jax_cosmo interp)."""
    x = np.asarray(x, dtype=np.float64)
    xp = np.asarray(xp, dtype=np.float64)
    fp = np.asarray(fp, dtype=np.float64)
    i = np.clip(np.searchsorted(xp, x) - 1, 0, len(xp) - 2)
    slope = (fp[i + 1] - fp[i]) / (xp[i + 1] - xp[i])
    return fp[i] + (x - xp[i]) * slope


# ----------------------------------------------------------------------------- growth
@dataclasses.dataclass(frozen=True)
class GrowthTable:
    a: np.ndarray
    g: np.ndarray  # D1 / D1(1)
    f: np.ndarray  # dlnD1/dlna
    g2: np.ndarray  # D2 / D2(1)
    f2: np.ndarray  # dlnD2/dlna
    d2g: np.ndarray  # d^2 (D1/D1(1)) / da^2


def _q_r_scalar(c: Cosmology, a: float):
    """Coefficients of the growth ODE at one scale factor (plain floats, no arrays)."""
    if c.wa == 0.0:
        de = c.Omega_de * a ** (-3.0 * (1.0 + c.w0))
    else:
        de = c.Omega_de * a ** (-3.0 * (1.0 + c.w0 + c.wa) + 3.0 * c.wa * (a - 1.0) / math.log(a))
    m = c.Omega_m / (a * a * a)
    e2 = m + c.Omega_k / (a * a) + de
    om = m / e2
    ode = de / e2
    wa = c.w0 + c.wa * (1.0 - a)
    return (2.0 - 0.5 * (om + (1.0 + 3.0 * wa) * ode)) / a, 1.5 * om / (a * a)


@functools.lru_cache(maxsize=1024)
def growth_table(c: Cosmology, log10_amin: float = -3.0, steps: int = 128) -> GrowthTable:
    atab = np.logspace(log10_amin, 0.0, steps)

    def q_r(a):
        om = Omega_m_a(c, a)
        ode = Omega_de_a(c, a)
        q = (2.0 - 0.5 * (om + (1.0 + 3.0 * w(c, a)) * ode)) / a
        r = 1.5 * om / (a * a)
        return q, r

    def rhs(y, a):
        g1, d1, g2, d2 = y
        q, r = _q_r_scalar(c, a)
        return [d1, -q * d1 + r * g1, d2, -q * d2 + r * g2 - r * g1 * g1]

    a0 = atab[0]
    y0 = [a0, 1.0, -3.0 / 7.0 * a0 * a0, -6.0 / 7.0 * a0]
    sol = odeint(rhs, y0, atab, rtol=1e-12, atol=1e-15)  # LSODA
    g1, d1, g2, d2 = sol.T
    q, r = q_r(atab)
    dd1 = -q * d1 + r * g1
    gtab = g1 / g1[-1]
    g2tab = g2 / g2[-1]
    ftab = d1 / g1[-1] * atab / gtab
    f2tab = d2 / g2[-1] * atab / g2tab
    return GrowthTable(a=atab, g=gtab, f=ftab, g2=g2tab, f2=f2tab, d2g=dd1 / g1[-1])


def growth_factor(c: Cosmology, a):
    t = growth_table(c)
    return np.clip(interp(a, t.a, t.g), 0.0, 1.0)


def growth_rate(c: Cosmology, a):
    t = growth_table(c)
    return interp(a, t.a, t.f)


def growth_factor_second(c: Cosmology, a):
    t = growth_table(c)
    return interp(a, t.a, t.g2)


def growth_rate_second(c: Cosmology, a):
    t = growth_table(c)
    return interp(a, t.a, t.f2)


def Gp(c: Cosmology, a):
    """Drift growth: Gp = D1."""
    return growth_factor(c, a)


def gp(c: Cosmology, a):
    """dGp/da = f D1 / a."""
    a = np.asarray(a, dtype=np.float64)
    return growth_rate(c, a) * growth_factor(c, a) / a


def Gf(c: Cosmology, a):
    """Kick growth: Gf = f D1 a^2 E = a^3 E dD1/da."""
    a = np.asarray(a, dtype=np.float64)
    return growth_rate(c, a) * growth_factor(c, a) * a ** 2 * E(c, a)


def dGfa(c: Cosmology, a):
    """dGf/da = D1' E' a^3 + 3 a^2 E D1' + a^3 E D1'' with tabulated D1''."""
    a = np.asarray(a, dtype=np.float64)
    t = growth_table(c)
    d1p = growth_rate(c, a) * growth_factor(c, a) / a
    d1pp = interp(a, t.a, t.d2g)
    Ea = E(c, a)
    return d1p * dEa(c, a) * a ** 3 + 3.0 * a ** 2 * Ea * d1p + a ** 3 * Ea * d1pp


# ----------------------------------------------------------------------------- distances
@dataclasses.dataclass(frozen=True)
class DistanceTable:
    a: np.ndarray
    chi: np.ndarray


@functools.lru_cache(maxsize=1024)
def distance_table(c: Cosmology, log10_amin: float = -3.0, steps: int = 256) -> DistanceTable:
    atab = np.logspace(log10_amin, 0.0, steps)
    # d chi / d ln a = 1 / (a E): composite Simpson on 16 sub-intervals per table interval
    sub = 16
    x = np.linspace(np.log(atab[0]), 0.0, (steps - 1) * sub + 1)
    a = np.exp(x)
    f = 1.0 / (a * E(c, a))
    h = x[1] - x[0]
    seg = f[:-1].reshape(steps - 1, sub)
    fe = np.append(f[sub::sub], [])  # right ends
    # Simpson over each table interval: h/3 [f0 + 4 f_odd + 2 f_even + f_end]
    odd = seg[:, 1::2].sum(axis=1)
    even = seg[:, 2::2].sum(axis=1)
    piece = h / 3.0 * (seg[:, 0] + 4.0 * odd + 2.0 * even + fe)
    chi = np.concatenate([np.cumsum(piece[::-1])[::-1], [0.0]])
    return DistanceTable(a=atab, chi=RH * chi)


def radial_comoving_distance(c: Cosmology, a):
    t = distance_table(c)
    return np.clip(interp(a, t.a, t.chi), 0.0, 1e6)


def a_of_chi(c: Cosmology, chi):
    t = distance_table(c)
    return interp(chi, t.chi[::-1], t.a[::-1])


def a2z(a):
    return 1.0 / np.asarray(a, dtype=np.float64) - 1.0


def z2a(z):
    return 1.0 / (1.0 + np.asarray(z, dtype=np.float64))


# ----------------------------------------------------------------------------- power
def eisenstein_hu_transfer(c: Cosmology, k):
    """Eisenstein & Hu (1998) transfer function with baryon oscillations; k in h/Mpc."""
    k = np.asarray(k, dtype=np.float64) * c.h  # 1/Mpc
    om = c.Omega_m * c.h ** 2
    ob = c.Omega_b * c.h ** 2
    fb = c.Omega_b / c.Omega_m
    fc = c.Omega_c / c.Omega_m
    th = TCMB / 2.7
    z_eq = 2.50e4 * om * th ** -4
    k_eq = 7.46e-2 * om * th ** -2
    b1 = 0.313 * om ** -0.419 * (1.0 + 0.607 * om ** 0.674)
    b2 = 0.238 * om ** 0.223
    z_d = 1291.0 * om ** 0.251 / (1.0 + 0.659 * om ** 0.828) * (1.0 + b1 * ob ** b2)
    R_eq = 31.5 * ob * th ** -4 * (z_eq / 1e3) ** -1
    R_d = 31.5 * ob * th ** -4 * (z_d / 1e3) ** -1
    s = 2.0 / (3.0 * k_eq) * math.sqrt(6.0 / R_eq) * math.log(
        (math.sqrt(1.0 + R_d) + math.sqrt(R_d + R_eq)) / (1.0 + math.sqrt(R_eq))
    )
    k_silk = 1.6 * ob ** 0.52 * om ** 0.73 * (1.0 + (10.4 * om) ** -0.95)
    q = k / (13.41 * k_eq)

    a1 = (46.9 * om) ** 0.670 * (1.0 + (32.1 * om) ** -0.532)
    a2 = (12.0 * om) ** 0.424 * (1.0 + (45.0 * om) ** -0.582)
    alpha_c = a1 ** -fb * a2 ** (-(fb ** 3))
    bb1 = 0.944 / (1.0 + (458.0 * om) ** -0.708)
    bb2 = (0.395 * om) ** -0.0266
    beta_c = 1.0 / (1.0 + bb1 * (fc ** bb2 - 1.0))

    def t0(alpha, beta):
        L = np.log(np.e + 1.8 * beta * q)
        C = 14.2 / alpha + 386.0 / (1.0 + 69.9 * q ** 1.08)
        return L / (L + C * q * q)

    f = 1.0 / (1.0 + (k * s / 5.4) ** 4)
    Tc = f * t0(1.0, beta_c) + (1.0 - f) * t0(alpha_c, beta_c)

    y = (1.0 + z_eq) / (1.0 + z_d)
    sq = math.sqrt(1.0 + y)
    G = y * (-6.0 * sq + (2.0 + 3.0 * y) * math.log((sq + 1.0) / (sq - 1.0)))
    alpha_b = 2.07 * k_eq * s * (1.0 + R_d) ** -0.75 * G
    beta_node = 8.41 * om ** 0.435
    beta_b = 0.5 + fb + (3.0 - 2.0 * fb) * math.sqrt((17.2 * om) ** 2 + 1.0)
    ks = k * s
    s_tilde = s / (1.0 + (beta_node / np.maximum(ks, 1e-300)) ** 3) ** (1.0 / 3.0)
    x = k * s_tilde
    j0 = np.where(x > 1e-8, np.sin(x) / np.where(x > 1e-8, x, 1.0), 1.0)
    Tb = (t0(1.0, 1.0) / (1.0 + (ks / 5.2) ** 2) + alpha_b / (1.0 + (beta_b / np.maximum(ks, 1e-300)) ** 3)
          * np.exp(-((k / k_silk) ** 1.4))) * j0
    return fb * Tb + fc * Tc


@functools.lru_cache(maxsize=1024)
def _sigma_r8_unnormalised(c: Cosmology) -> float:
    """sigma^2(8 Mpc/h) of k^ns T(k)^2 (Simpson on a dense log-k grid; depends on
    everything but sigma8, so sigma8 alone rescales without recomputation)."""
    R = 8.0
    lnk = np.linspace(math.log(1e-5), math.log(1e3), 16385)
    k = np.exp(lnk)
    x = k * R
    small = x < 1e-4
    xs = np.where(small, 1.0, x)
    wt = np.where(small, 1.0 - x * x / 10.0, 3.0 * (np.sin(xs) - xs * np.cos(xs)) / xs ** 3)
    f = k ** 3 * k ** c.n_s * eisenstein_hu_transfer(c, k) ** 2 * wt * wt / (2.0 * math.pi ** 2)
    h = lnk[1] - lnk[0]
    return float(h / 3.0 * (f[0] + 4.0 * f[1:-1:2].sum() + 2.0 * f[2:-1:2].sum() + f[-1]))


def _sigma8_norm(c: Cosmology) -> float:
    return c.sigma8 ** 2 / _sigma_r8_unnormalised(c.replace(sigma8=1.0))


def linear_matter_power(c: Cosmology, k, a=1.0):
    """Linear P(k) in (Mpc/h)^3 at scale factor a, k in h/Mpc."""
    k = np.asarray(k, dtype=np.float64)
    return _sigma8_norm(c) * k ** c.n_s * eisenstein_hu_transfer(c, k) ** 2 * growth_factor(c, a) ** 2


def pk_table(c: Cosmology, n: int = 128):
    """(k, P_lin(k)) on logspace(-4, 1, n), the table jax-fli interpolates for its ICs
    (128 points at initial.py:171, 256 points at infer/dist.py:50)."""
    k = np.logspace(-4, 1, n)
    return k, linear_matter_power(c, k)
