"""1-D integral tables of the quadratic B-spline basis, derived exactly.

The reference ships these as ``jspsr/data/bezier_integrals.pkl``
(``jspsr/bases/bezier_tensor.py:26-34``), a file that was never published.  The
tables follow from the basis definition (``bezier_tensor.py:17-22``) and the
index conventions of ``bezier_tensor.py:75-121``; every entry is the integral
of a piecewise polynomial, evaluated here in closed form (antiderivatives of the
polynomial pieces between consecutive knots, in a variable local to each interval).  Level ratios beyond the
reference's 16 (``n_multiples=5``) follow from the same formulas.

Names and meaning (M = 2**m is the stride ratio of the two levels):

* ``ssi[m][i] = int B(y + dx) B(y / M) dy``,             ``dx = -1.5M - 0.5 + i``
* ``sdi[m][i] = int B'(y + dx) B'(y / M) dy``            (no chain factor; the caller divides by the coarse stride)
* ``dpi[m][i] = int_{ra}^{ra+1} B(x / M) dx``,           ``ra = 1.5M - 1 - i``
* ``pi[m][i]  = int_{ra}^{ra+1} B'(x / M) dx``           (no chain factor)
* ``idpi[m-1][i] = int_{max(ra,-1.5)}^{min(ra+M,1.5)} B(x) dx``,  ``ra = 0.5 - i``
* ``ipi[m-1][i]  = int ... B'(x) dx``
"""
from __future__ import annotations

from functools import lru_cache

import numpy as np
from numpy.polynomial import polynomial as P

# B-spline pieces on [-1.5,-0.5), [-0.5,0.5), [0.5,1.5): coefficients in ascending powers.
_KNOTS = (-1.5, -0.5, 0.5, 1.5)
_PIECES = (np.array([2.25, 3.0, 1.0]), np.array([1.5, 0.0, -2.0]), np.array([2.25, -3.0, 1.0]))


def _piece(x_lo, x_hi, scale=1.0, shift=0.0, deriv=False):
    """Pieces of B(scale * y + shift) (or d/du B(u) at u = scale*y + shift) on the y line: each piece is
    (y_lo, y_hi, polynomial in u, scale, shift).  The polynomial stays in the spline's own variable u,
    whose range is the knot span: integrals are taken in a variable local to each interval, never by
    evaluating antiderivatives at large y (at a level ratio M = 1024 the y range reaches 1.5M, and an
    antiderivative expanded in y loses every digit of the small entries to cancellation)."""
    out = []
    for (a, b), c in zip(zip(_KNOTS[:-1], _KNOTS[1:]), _PIECES):
        poly = P.polyder(c) if deriv else c
        out.append(((a - shift) / scale, (b - shift) / scale, poly, scale, shift))
    return out


def _local(piece, y0):
    """The piece as a polynomial in t = y - y0 (u = scale * y0 + shift + scale * t)."""
    _, _, poly, scale, shift = piece
    u0 = scale * y0 + shift
    comp = np.zeros(1)
    for k, ck in enumerate(poly):
        comp = P.polyadd(comp, ck * P.polypow([u0, scale], k))
    return comp


_ONE = ((-np.inf, np.inf, np.array([1.0]), 1.0, 0.0),)


def _integrate_product(f_pieces, g_pieces=None, lo=-np.inf, hi=np.inf):
    total = 0.0
    if g_pieces is None:
        g_pieces = _ONE
    for fpc in f_pieces:
        for gpc in g_pieces:
            a, b = max(fpc[0], gpc[0], lo), min(fpc[1], gpc[1], hi)
            if b <= a:
                continue
            # integrate over t = y - a in [0, b - a]
            anti = P.polyint(P.polymul(_local(fpc, a), _local(gpc, a)))
            total += P.polyval(b - a, anti)
    return total


@lru_cache(maxsize=None)
def shifted(m: int):
    """(ssi[m], sdi[m]) as float64 arrays of length 3M + 2."""
    M = 2 ** m
    ssi, sdi = [], []
    for i in range(3 * M + 2):
        dx = -1.5 * M - 0.5 + i
        ssi.append(_integrate_product(_piece(0, 0, 1.0, dx), _piece(0, 0, 1.0 / M, 0.0)))
        sdi.append(_integrate_product(_piece(0, 0, 1.0, dx, True), _piece(0, 0, 1.0 / M, 0.0, True)))
    return np.array(ssi), np.array(sdi)


@lru_cache(maxsize=None)
def partial(m: int):
    """(dpi[m], pi[m]) as float64 arrays of length 3M."""
    M = 2 ** m
    dpi, pi = [], []
    for i in range(3 * M):
        ra = 1.5 * M - 1 - i
        dpi.append(_integrate_product(_piece(0, 0, 1.0 / M, 0.0), None, ra, ra + 1))
        pi.append(_integrate_product(_piece(0, 0, 1.0 / M, 0.0, True), None, ra, ra + 1))
    return np.array(dpi), np.array(pi)


@lru_cache(maxsize=None)
def inverse_partial(m: int):
    """(idpi[m-1], ipi[m-1]) for m >= 1 as float64 arrays of length M + 2."""
    assert m >= 1
    M = 2 ** m
    f, df = [], []
    for i in range(M + 2):
        ra = 0.5 - i
        lb, ub = max(ra, -1.5), min(ra + M, 1.5)
        f.append(_integrate_product(_piece(0, 0), None, lb, ub) if ub > lb else 0.0)
        df.append(_integrate_product(_piece(0, 0, deriv=True), None, lb, ub) if ub > lb else 0.0)
    return np.array(f), np.array(df)


def ratio_log2(m_ratio: int) -> int:
    m = int(m_ratio).bit_length() - 1
    assert 2 ** m == m_ratio, m_ratio
    return m


# ----------------------------------------------------------------------------- kernel-ready tables
def stencil125(stride: int) -> np.ndarray:
    """Same-level stiffness of the 125 lexicographic offsets (dx, dy, dz) in [-2, 2]^3."""
    ssi, sdi = shifted(0)
    c = ssi * stride
    g = sdi / stride
    out = np.zeros(125)
    o = 0
    for dx in range(-2, 3):
        for dy in range(-2, 3):
            for dz in range(-2, 3):
                ix, iy, iz = dx + 2, dy + 2, dz + 2
                out[o] = g[ix] * c[iy] * c[iz] + c[ix] * g[iy] * c[iz] + c[ix] * c[iy] * g[iz]
                o += 1
    return out


def correction_tables(fine_stride: int, coarse_stride: int):
    """(tc, tg) for K(fine, coarse): tc = ssi * s_fine, tg = sdi / s_coarse (length 3M + 2)."""
    ssi, sdi = shifted(ratio_log2(coarse_stride // fine_stride))
    return ssi * fine_stride, sdi / coarse_stride


def rhs_tables(data_stride: int, target_stride: int):
    """(tc, tg) for the divergence RHS of a data level onto a target level."""
    if target_stride >= data_stride:
        M = target_stride // data_stride
        dpi, pi = partial(ratio_log2(M))
        return dpi * data_stride, pi * (data_stride / target_stride)
    M = data_stride // target_stride
    idpi, ipi = inverse_partial(ratio_log2(M))
    return idpi * target_stride, ipi


def reference_pickle_tables(n_mult: int = 5):
    """The eight tables in the order of the reference's pickle (bezier_tensor.py:31-34)."""
    sh = [shifted(m) for m in range(n_mult)]
    pa = [partial(m) for m in range(n_mult)]
    inv = [inverse_partial(m) for m in range(1, n_mult)]
    return ([p[1] for p in pa], [p[0] for p in pa], [p[1] for p in inv], [p[0] for p in inv],
            [s[0] for s in sh], [s[1] for s in sh], [np.zeros_like(s[0]) for s in sh],
            [np.zeros_like(p[0]) for p in inv])


# ----------------------------------------------------------------------------- general 1-D components
_GL_X, _GL_W = np.polynomial.legendre.leggauss(40)


def _gl(fn, lo, hi, breaks):
    """Gauss-Legendre (40 nodes) on each smooth piece of [lo, hi] between breakpoints."""
    if hi <= lo:
        return 0.0
    pts = sorted({lo, hi, *[b for b in breaks if lo < b < hi]})
    tot = 0.0
    for a, b in zip(pts[:-1], pts[1:]):
        m, h = 0.5 * (a + b), 0.5 * (b - a)
        tot += h * float(np.dot(_GL_W, fn(m + h * _GL_X)))
    return tot


def component_pair_tables(ci, cj, n_mult: int):
    """theta / theta-dot tables of two additive components (the integrals of
    ``jspsr/bases/additive.py:17-28``): lists over m < n_mult of arrays of length 3*2^m + 2."""
    ff, dfdf = [], []
    for m in range(n_mult):
        M = 2 ** m
        rf, rd = [], []
        for i in range(3 * M + 2):
            dx = -1.5 * M - 0.5 + i
            br = [b - dx for b in ci.breaks] + [b * M for b in cj.breaks]
            lo, hi = max(-1.5 - dx, -1.5 * M), min(1.5 - dx, 1.5 * M)
            rf.append(_gl(lambda y: ci.f(y + dx) * cj.f(y / M), lo, hi, br))
            rd.append(_gl(lambda y: ci.df(y + dx) * cj.df(y / M) / M, lo, hi, br))
        ff.append(np.asarray(rf))
        dfdf.append(np.asarray(rd))
    return ff, dfdf


def component_tables(c, n_mult: int):
    """rho / rho-dot tables of one component (``jspsr/bases/additive.py:31-52``):
    forward f, df (m < n_mult, length 3*2^m) and inverse f_inv, df_inv (1 <= m < n_mult, length 2^m + 2)."""
    f, df, fi, dfi = [], [], [], []
    for m in range(n_mult):
        M = 2 ** m
        br = [b * M for b in c.breaks]
        f.append(np.asarray([_gl(lambda x: c.f(x / M), 1.5 * M - 1 - i, 1.5 * M - i, br) for i in range(3 * M)]))
        df.append(np.asarray([_gl(lambda x: c.df(x / M) / M, 1.5 * M - 1 - i, 1.5 * M - i, br) for i in range(3 * M)]))
    for m in range(1, n_mult):
        M = 2 ** m
        rows_f, rows_d = [], []
        for i in range(M + 2):
            ra = 0.5 - i
            lb, ub = max(ra, -1.5), min(ra + M, 1.5)
            rows_f.append(_gl(c.f, lb, ub, c.breaks))
            rows_d.append(_gl(c.df, lb, ub, c.breaks))
        fi.append(np.asarray(rows_f))
        dfi.append(np.asarray(rows_d))
    return f, df, fi, dfi
