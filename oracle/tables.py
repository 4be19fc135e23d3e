"""Closed-form 1-D integral tables of the screened-Poisson bases (FP64).

TEST INFRASTRUCTURE / ORACLE ONLY.  Nothing in the product imports this
module; the product package derives the same tables with its own code
(``jspsr/bases/tables.py``) and the tests compare the two.

The reference loads these tables from ``jspsr/data/bezier_integrals.pkl``
(``jspsr/bases/bezier_tensor.py:26-34``), a file that was never published.
They are re-derived here from their definitions:

* ``_integrate_ff``     -- ``jspsr/bases/additive.py:17-28`` (theta, theta-dot)
* ``_integrate_f``      -- ``jspsr/bases/additive.py:31-40`` (rho, rho-dot)
* ``_integrate_f_inv``  -- ``jspsr/bases/additive.py:43-52``
* index conventions     -- ``jspsr/bases/bezier_tensor.py:75-121``,
  ``jspsr/bases/additive.py:188-246``.

Every integrand is piecewise smooth with known breakpoints; each smooth piece
is integrated with 24-point Gauss-Legendre, which is exact (to rounding) for
the piecewise polynomials of the Bezier / Power components and converges to
machine precision for the sinusoid components.

Convention shared with the reference (chosen so that ``BezierTensorBasis``
equals ``AdditiveBasis([Bezier()], [1.0])``, ``additive.py:406-409``):

* ``ff[m][i]  = int q_s(y + dx) q_t(y / M) dy``,  ``dx = -1.5M - 0.5 + i``,
  ``i in [0, 3M + 2)``, ``M = 2**m``                       (``additive.py:202-203``)
* ``dfdf[m][i] = int d/dy[q_s(y + dx)] d/dy[q_t(y / M)] dy`` (with the 1/M chain factor)
* ``f[m][i]   = int_{ra}^{ra+1} q(x / M) dx``, ``ra = 1.5M - 1 - i``, ``i in [0, 3M)``
  (``additive.py:227-233``: ``insert(0, ...)`` reverses the order)
* ``df[m][i]  = int_{ra}^{ra+1} d/dx[q(x / M)] dx``
* ``f_inv[m-1][i] = int_{lb}^{ub} q(x) dx``, ``ra = 0.5 - i``, ``lb = max(ra, -1.5)``,
  ``ub = min(ra + M, 1.5)``, ``i in [0, M + 2)``, ``m >= 1`` (``additive.py:238-244``)
* ``df_inv[m-1][i] = int_{lb}^{ub} q'(x) dx``

The Bezier-specific tables of ``bezier_tensor.py`` then are
``SHIFTED_SELF_INTEGRAL = ff``, ``SHIFTED_DERIVATIVE_INTEGRAL = M * dfdf``,
``DERIVATIVE_PARTIAL_INTEGRAL = f``, ``PARTIAL_INTEGRAL = M * df``,
``INV_DERIVATIVE_PARTIAL_INTEGRAL = f_inv``, ``INV_PARTIAL_INTEGRAL = df_inv``
(see the ``const_val`` / ``integral_val`` scalings at ``bezier_tensor.py:86-90,115-116``).
"""
import math

import numpy as np

_GL_X, _GL_W = np.polynomial.legendre.leggauss(24)
SUPPORT = 1.5


class Component:
    """A 1-D function q(x) supported on [-1.5, 1.5), with derivative and breakpoints."""

    def __init__(self, name, f, df, breaks):
        self.name, self.f, self.df, self.breaks = name, f, df, tuple(breaks)

    def __repr__(self):
        return self.name


def bezier():
    """Quadratic B-spline scaled by 2 (``bezier_tensor.py:17-22``, ``additive_components.py:102-131``)."""
    def f(x):
        return np.where((x >= -1.5) & (x < -0.5), (x + 1.5) ** 2,
               np.where((x >= -0.5) & (x < 0.5), -2 * x ** 2 + 1.5,
               np.where((x >= 0.5) & (x < 1.5), (x - 1.5) ** 2, 0.0)))

    def df(x):
        return np.where((x >= -1.5) & (x < -0.5), 2 * x + 3,
               np.where((x >= -0.5) & (x < 0.5), -4 * x,
               np.where((x >= 0.5) & (x < 1.5), 2 * x - 3, 0.0)))
    return Component("Bezier()", f, df, (-1.5, -0.5, 0.5, 1.5))


def power(p):
    """q(x) = x**p on [-1.5, 1.5) (``additive_components.py:73-99``)."""
    def f(x):
        return np.where((x >= -1.5) & (x < 1.5), x ** p if p > 0 else np.ones_like(x), 0.0)

    def df(x):
        if p == 0:
            return np.zeros_like(x)
        return np.where((x >= -1.5) & (x < 1.5), p * x ** (p - 1) if p > 1 else np.ones_like(x), 0.0)
    return Component(f"Power({p:.2f})", f, df, (-1.5, 1.5))


def sin_peaks(n):
    """q(x) = sin(beta x + gamma), beta = pi n / 3, gamma = pi - pi n / 2 (``additive_components.py:134-164``)."""
    beta, gamma = math.pi * n / 3, -0.5 * math.pi * n + math.pi

    def f(x):
        return np.where((x >= -1.5) & (x < 1.5), np.sin(beta * x + gamma), 0.0)

    def df(x):
        return np.where((x >= -1.5) & (x < 1.5), beta * np.cos(beta * x + gamma), 0.0)
    return Component(f"SinPeaks({n})", f, df, (-1.5, 1.5))


def _integrate(fn, lo, hi, breaks):
    """Piecewise Gauss-Legendre integral of fn over [lo, hi] split at ``breaks``."""
    if hi <= lo:
        return 0.0
    pts = sorted({lo, hi, *[b for b in breaks if lo < b < hi]})
    total = 0.0
    for a, b in zip(pts[:-1], pts[1:]):
        xm, xr = 0.5 * (a + b), 0.5 * (b - a)
        total += xr * float(np.sum(_GL_W * fn(xm + xr * _GL_X)))
    return total


def ff_tables(cs: Component, ct: Component, n_mult: int):
    """theta / theta-dot of ``additive.py:17-28`` for every ratio M = 2**m, m < n_mult."""
    ff, dfdf = [], []
    for m in range(n_mult):
        M = 2 ** m
        row_f, row_d = [], []
        for i in range(3 * M + 2):
            dx = -1.5 * M - 0.5 + i
            br = [b - dx for b in cs.breaks] + [b * M for b in ct.breaks]
            lo, hi = -SUPPORT * M - abs(dx) - 2, SUPPORT * M + abs(dx) + 2
            row_f.append(_integrate(lambda y: cs.f(y + dx) * ct.f(y / M), lo, hi, br))
            row_d.append(_integrate(lambda y: cs.df(y + dx) * ct.df(y / M) / M, lo, hi, br))
        ff.append(np.asarray(row_f))
        dfdf.append(np.asarray(row_d))
    return ff, dfdf


def f_tables(c: Component, n_mult: int):
    """rho / rho-dot (``additive.py:31-52``): forward tables for m < n_mult, inverse for 1 <= m < n_mult."""
    f, df, f_inv, df_inv = [], [], [], []
    for m in range(n_mult):
        M = 2 ** m
        rf, rd = [], []
        for i in range(3 * M):
            ra = 1.5 * M - 1 - i
            br = [b * M for b in c.breaks]
            rf.append(_integrate(lambda x: c.f(x / M), ra, ra + 1, br))
            rd.append(_integrate(lambda x: c.df(x / M) / M, ra, ra + 1, br))
        f.append(np.asarray(rf))
        df.append(np.asarray(rd))
    for m in range(1, n_mult):
        M = 2 ** m
        rf, rd = [], []
        for i in range(M + 2):
            ra = 0.5 - i
            lb, ub = max(ra, -1.5), min(ra + M, 1.5)
            rf.append(_integrate(c.f, lb, ub, c.breaks))
            rd.append(_integrate(c.df, lb, ub, c.breaks))
        f_inv.append(np.asarray(rf))
        df_inv.append(np.asarray(rd))
    return f, df, f_inv, df_inv


def bezier_tables(n_mult: int):
    """The eight Bezier tables in the order of ``bezier_tensor.py:31-34``."""
    b = bezier()
    ff, dfdf = ff_tables(b, b, n_mult)
    f, df, f_inv, df_inv = f_tables(b, n_mult)
    mults = [2 ** m for m in range(n_mult)]
    return {
        "PARTIAL_INTEGRAL": [M * t for M, t in zip(mults, df)],
        "DERIVATIVE_PARTIAL_INTEGRAL": f,
        "INV_PARTIAL_INTEGRAL": df_inv,
        "INV_DERIVATIVE_PARTIAL_INTEGRAL": f_inv,
        "SHIFTED_SELF_INTEGRAL": ff,
        "SHIFTED_DERIVATIVE_INTEGRAL": [M * t for M, t in zip(mults, dfdf)],
        # The two tables below are not in the reference pickle; they are the
        # self-integrals used by nothing but kept for completeness of the order.
        "SHIFTED_SELF_DERIV_INTEGRAL": [np.zeros_like(t) for t in ff],
        "INV_SHIFTED_SELF_DERIV_INTEGRAL": [np.zeros_like(t) for t in f_inv],
    }


BEZIER_PICKLE_ORDER = ("PARTIAL_INTEGRAL", "DERIVATIVE_PARTIAL_INTEGRAL",
                       "INV_PARTIAL_INTEGRAL", "INV_DERIVATIVE_PARTIAL_INTEGRAL",
                       "SHIFTED_SELF_INTEGRAL", "SHIFTED_DERIVATIVE_INTEGRAL",
                       "SHIFTED_SELF_DERIV_INTEGRAL", "INV_SHIFTED_SELF_DERIV_INTEGRAL")
