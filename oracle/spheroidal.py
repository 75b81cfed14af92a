"""ORACLE — test infrastructure only (never imported by the product).

Prolate spheroidal wave function psi_{alpha,0}(c, eta), normalised to 1 at
eta = 0, as used by yandasoft's gridders through
``scimath::SpheroidalFunction(pi*support, alpha)``.

That class lives in the un-vendored base-scimath library (tags/1.9.0).  Its
call sites are askap/gridding/SphFuncVisGridder.cc:47 (construction) and
SphFuncVisGridder.h:101 (``grdsf(nu) = itsSphFunc(nu)``).  The published
method it implements is documented in the reference's own research code,
apps/gridderExperiments.cc:180-260 (``fillHelperMatrix``, ``legendreCoeffs``,
``sumLegendreSeries``, ``sphFunc``): expand S_{m,0}(c, eta) in normalised
associated Legendre functions P_{m+2k}^m, take the eigenvector of the
symmetric tridiagonal matrix that belongs to the smallest eigenvalue, sum the
series, normalise by its value at eta = 0, and multiply by
(1 - eta^2)^(-alpha/2).  m = int(alpha).

This restatement builds the same matrix, solves it with numpy's symmetric
eigen-solver and evaluates the Legendre series with a stable upward
recurrence of orthonormal associated Legendre functions (any l-independent
normalisation cancels in the ratio).  It is written independently of the
product's C++ implementation so that the two check each other.
"""
from __future__ import annotations

import math

import numpy as np

NTERMS_DEFAULT = 16


def _helper_matrix(c: float, m: int, nterms: int) -> np.ndarray:
    """Symmetric tridiagonal matrix of the spheroidal equation in the basis of
    orthonormal associated Legendre functions P_{m+2k}^m (gridderExperiments.cc:262-280)."""
    c2 = c * c
    b = np.zeros((nterms, nterms))
    for row in range(nterms):
        l = 2 * row + m
        b[row, row] = l * (l + 1) + c2 * ((2 * l + 3) * (l + m) * (l - m)
                                          + (2 * l - 1) * (l + m + 1) * (l - m + 1)) / (
            (2 * l + 1) * (2 * l - 1) * (2 * l + 3))
        if row >= 1:
            b[row, row - 1] = c2 / (2 * l - 1) * math.sqrt(
                (l + m) * (l + m - 1) * (l - m) * (l - m - 1) / ((2 * l + 1) * (2 * l - 3)))
        if row + 1 < nterms:
            b[row, row + 1] = c2 / (2 * l + 3) * math.sqrt(
                (l + m + 1) * (l + m + 2) * (l - m + 1) * (l - m + 2) / ((2 * l + 1) * (2 * l + 5)))
    return b


def _norm_legendre(lmax: int, m: int, x: np.ndarray) -> np.ndarray:
    """Orthonormal associated Legendre functions Pbar_l^m(x) for l = m..lmax.

    Pbar_l^m = sqrt((2l+1)/2 (l-m)!/(l+m)!) P_l^m; the standard three-term
    recurrence in l for the normalised functions.  Returns (lmax-m+1, len(x))."""
    x = np.asarray(x, dtype=np.float64)
    out = np.zeros((lmax - m + 1,) + x.shape)
    s = np.sqrt(np.maximum(0.0, 1.0 - x * x))
    # Pbar_m^m = (-1)^m sqrt((2m+1)/2 * (2m)!/(2^m m!)^2) * (1-x^2)^(m/2)
    pmm = np.full_like(x, math.sqrt(0.5))
    for k in range(1, m + 1):
        pmm = -pmm * math.sqrt((2.0 * k + 1.0) / (2.0 * k)) * s
    out[0] = pmm
    if lmax == m:
        return out
    pm1 = x * math.sqrt(2.0 * m + 3.0) * pmm
    out[1] = pm1
    for l in range(m + 2, lmax + 1):
        a = math.sqrt((4.0 * l * l - 1.0) / (l * l - m * m))
        bcoef = math.sqrt(((l - 1.0) ** 2 - m * m) / (4.0 * (l - 1.0) ** 2 - 1.0))
        pl = a * (x * pm1 - bcoef * pmm)
        out[l - m] = pl
        pmm, pm1 = pm1, pl
    return out


class SpheroidalFunction:
    """psi_{alpha,0}(c, eta) normalised to 1 at eta = 0; zero for |eta| >= 1."""

    def __init__(self, c: float, alpha: float, nterms: int = NTERMS_DEFAULT):
        self.c = float(c)
        self.alpha = float(alpha)
        self.m = int(alpha)
        self.nterms = int(nterms)
        b = _helper_matrix(self.c, self.m, self.nterms)
        vals, vecs = np.linalg.eigh(b)
        self.coeffs = vecs[:, int(np.argmin(vals))].copy()
        self.sum0 = self._series(np.array([0.0]))[0]

    def _series(self, eta: np.ndarray) -> np.ndarray:
        lmax = self.m + 2 * (self.nterms - 1)
        p = _norm_legendre(lmax, self.m, eta)
        # only even r = l - m enter the expansion
        return np.tensordot(self.coeffs, p[0::2], axes=(0, 0))

    def __call__(self, nu):
        nu = np.asarray(nu, dtype=np.float64)
        scalar = nu.ndim == 0
        nu = np.atleast_1d(nu)
        out = np.zeros_like(nu)
        inside = np.abs(nu) < 1.0
        if np.any(inside):
            e = nu[inside]
            res = self._series(e) / self.sum0
            out[inside] = res * np.power(1.0 - e * e, -self.alpha / 2.0)
        return out[0] if scalar else out


def grdsf_factory(support: int = 3, alpha: float = 1.0):
    """grdsf of SphFuncVisGridder (itsSphFunc(C::pi*support, alpha))."""
    return SpheroidalFunction(math.pi * support, alpha)


def schwab_grdsf(nu):
    """Schwab's rational approximation for m = 6, alpha = 1 (published method,
    F. Schwab, Indirect Imaging 1984; quoted in SphFuncVisGridder.cc:268-333).
    Used only as an independent cross-check of the Legendre expansion."""
    p = [[8.203343e-2, -3.644705e-1, 6.278660e-1, -5.335581e-1, 2.312756e-1],
         [4.028559e-3, -3.697768e-2, 1.021332e-1, -1.201436e-1, 6.412774e-2]]
    q = [[1.0, 8.212018e-1, 2.078043e-1], [1.0, 9.599102e-1, 2.918724e-1]]
    nu = np.atleast_1d(np.asarray(nu, dtype=np.float64))
    out = np.zeros_like(nu)
    for i, v in enumerate(nu):
        if 0.0 <= v < 0.75:
            part, nuend = 0, 0.75
        elif 0.75 <= v <= 1.0:
            part, nuend = 1, 1.0
        else:
            continue
        d = v * v - nuend * nuend
        top = sum(p[part][k] * d ** k for k in range(5))
        bot = sum(q[part][k] * d ** k for k in range(3))
        out[i] = max(top / bot, 0.0) if bot != 0 else 0.0
    return out
