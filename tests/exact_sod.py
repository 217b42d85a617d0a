"""Exact solution of the Sod shock tube for the known-answer tests.

Restates the shock-tube equation and wave structure of the reference's IDL
solver FX/Simulation/SimulationMain/Sod/shocktube.pro (after B. Fryxell):
states 1 (left, at rest) and 5 (right, at rest), rarefaction into 1, contact,
shock into 5.  f(p4) = p1*(1 - (g-1)/(2g)*(c5/c1)*z/sqrt(1+(g+1)/(2g)*z))^(2g/(g-1)) - p4
with z = p4/p5 - 1.
"""
import math

import numpy as np


def _f(p4, p1, p5, r1, r5, g):
    z = p4 / p5 - 1.0
    c1 = math.sqrt(g * p1 / r1)
    c5 = math.sqrt(g * p5 / r5)
    gm1, gp1, g2 = g - 1.0, g + 1.0, 2.0 * g
    fact = gm1 / g2 * (c5 / c1) * z / math.sqrt(1.0 + gp1 / g2 * z)
    fact = (1.0 - fact) ** (g2 / gm1)
    return p1 * fact - p4


def sod_exact(x, t, x0=0.5, r1=1.0, p1=1.0, r5=0.125, p5=0.1, g=1.4):
    """rho, u, p at positions x (1-D along the tube normal) and time t."""
    lo, hi = p5, p1
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if _f(mid, p1, p5, r1, r5, g) > 0.0:
            lo = mid
        else:
            hi = mid
    p4 = 0.5 * (lo + hi)
    c1 = math.sqrt(g * p1 / r1)
    c5 = math.sqrt(g * p5 / r5)
    z = p4 / p5 - 1.0
    gm1, gp1, g2 = g - 1.0, g + 1.0, 2.0 * g
    gmfac1 = 0.5 * gm1 / g
    gmfac2 = 0.5 * gp1 / g
    fact = math.sqrt(1.0 + gmfac2 * z)
    u4 = c5 * z / (g * fact)
    r4 = r5 * (1.0 + gmfac2 * z) / (1.0 + gmfac1 * z)
    w = c5 * fact                       # shock speed
    p3, u3 = p4, u4
    r3 = r1 * (p3 / p1) ** (1.0 / g)
    c3 = math.sqrt(g * p3 / r3)
    x1 = x0 - c1 * t                    # rarefaction head
    x2 = x0 + (u3 - c3) * t             # rarefaction tail
    x3 = x0 + u3 * t                    # contact
    x4 = x0 + w * t                     # shock
    x = np.asarray(x, dtype=float)
    rho = np.empty_like(x); u = np.empty_like(x); p = np.empty_like(x)
    m = x < x1
    rho[m], u[m], p[m] = r1, 0.0, p1
    m = (x >= x1) & (x < x2)
    uf = 2.0 / gp1 * (c1 + (x[m] - x0) / t)
    cf = c1 - 0.5 * gm1 * uf
    rho[m] = r1 * (cf / c1) ** (2.0 / gm1)
    u[m] = uf
    p[m] = p1 * (cf / c1) ** (2.0 * g / gm1)
    m = (x >= x2) & (x < x3)
    rho[m], u[m], p[m] = r3, u3, p3
    m = (x >= x3) & (x < x4)
    rho[m], u[m], p[m] = r4, u4, p4
    m = x >= x4
    rho[m], u[m], p[m] = r5, 0.0, p5
    return rho, u, p
