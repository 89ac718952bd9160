# -*- coding: utf-8 -*-
"""Gauss quadratures by the Golub-Welsch eigenvalue method.

Same rules as frfs/quadratures.py:6-50 (Gauss-Jacobi and
Gauss-Lobatto-Jacobi nodes and weights on [-1, 1]); used for the radial
velocity quadrature (frfs/solvers/dgfs/velocitymesh.py:112-126) and for the
element point sets.
"""

from math import gamma

import numpy as np


def jacobi_recurrence(n, a, b):
    """Three-term recurrence coefficients of the monic Jacobi polynomials;
    rb[0] is the integral of the weight (1-x)^a (1+x)^b over [-1, 1]."""
    ra, rb = np.zeros(n), np.zeros(n)
    s = 2.0 + a + b
    ra[0] = (b - a)/s
    rb[0] = 2.0**(a + b + 1)*gamma(a + 1.0)*gamma(b + 1.0)/gamma(s)
    if n > 1:
        rb[1] = 4.0*(a + 1.0)*(b + 1.0)/((s + 1.0)*s*s)
    s += 2
    for i in range(1, n - 1):
        ra[i] = (b*b - a*a)/((s - 2.0)*s)
        rb[i + 1] = (4.0*(i + 1)*(i + 1 + a)*(i + 1 + b)*(i + 1 + a + b) /
                     ((s*s - 1)*s*s))
        s += 2
    if n > 1:
        ra[n - 1] = (b*b - a*a)/((s - 2.0)*s)
    return ra, rb


def _golub_welsch(ra, rb):
    mu0 = rb[0]
    J = np.diag(ra) + np.diag(np.sqrt(rb[1:]), -1)
    z, V = np.linalg.eigh(J)
    order = np.argsort(z)
    z, V = z[order], V[:, order]
    return z, mu0*V[0, :]**2


def zwgj(n, a=0.0, b=0.0):
    """n-point Gauss-Jacobi rule."""
    return _golub_welsch(*jacobi_recurrence(n, a, b))


def zwglj(n, a=0.0, b=0.0):
    """n-point Gauss-Lobatto-Jacobi rule (endpoints included)."""
    m = n - 2
    ra, rb = jacobi_recurrence(n, a, b)
    apb1 = a + b + 1.0
    ra[n - 1] = (a - b)/(2.0*m + apb1 + 1.0)
    rb[n - 1] = (4.0*(m + a + 1.0)*(m + b + 1.0)*(m + apb1) /
                 ((2.0*m + apb1)*(2*m + apb1 + 1)**2))
    return _golub_welsch(ra, rb)


def gauss_legendre(n):
    return zwgj(n, 0.0, 0.0)


def gauss_legendre_lobatto(n):
    """GLL points: endpoints plus the Gauss-Jacobi(1,1) nodes; weights
    2/(n(n-1) P_{n-1}(x)^2)."""
    if n == 1:
        return np.array([0.0]), np.array([2.0])
    if n == 2:
        return np.array([-1.0, 1.0]), np.array([1.0, 1.0])
    zi, _ = zwgj(n - 2, 1.0, 1.0)
    z = np.concatenate(([-1.0], zi, [1.0]))
    P = np.polynomial.legendre.legval(z, [0]*(n - 1) + [1])
    w = 2.0/(n*(n - 1)*P*P)
    return z, w
