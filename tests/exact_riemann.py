"""Exact solution of the 1D Riemann problem for an ideal gas (Toro,
"Riemann Solvers and Numerical Methods for Fluid Dynamics", ch. 4: pressure
function, Newton iteration for p*, then sampling of the self-similar fan).
Used as an analytic pin for the Sod configuration."""
from __future__ import annotations

import numpy as np


def _f(p, rho, pk, ck, g):
    if p > pk:  # shock
        A = 2.0 / ((g + 1.0) * rho)
        B = (g - 1.0) / (g + 1.0) * pk
        return (p - pk) * np.sqrt(A / (p + B)), np.sqrt(A / (B + p)) * (1.0 - 0.5 * (p - pk) / (B + p))
    # rarefaction
    e = (g - 1.0) / (2.0 * g)
    return 2.0 * ck / (g - 1.0) * ((p / pk) ** e - 1.0), 1.0 / (rho * ck) * (p / pk) ** (-(g + 1.0) / (2.0 * g))


def star_state(rl, ul, pl, rr, ur, pr, g=1.4):
    cl, cr = np.sqrt(g * pl / rl), np.sqrt(g * pr / rr)
    p = max(1e-12, 0.5 * (pl + pr) - 0.125 * (ur - ul) * (rl + rr) * (cl + cr))
    for _ in range(100):
        fl, dl = _f(p, rl, pl, cl, g)
        fr, dr = _f(p, rr, pr, cr, g)
        dp = (fl + fr + ur - ul) / (dl + dr)
        pn = max(1e-14, p - dp)
        if abs(pn - p) < 1e-15 * (pn + p):
            p = pn
            break
        p = pn
    fl, _ = _f(p, rl, pl, cl, g)
    fr, _ = _f(p, rr, pr, cr, g)
    u = 0.5 * (ul + ur + fr - fl)
    return p, u


def sample(x, t, x0, left, right, g=1.4):
    """(rho, u, p) at positions x and time t for the initial jump at x0."""
    rl, ul, pl = left
    rr, ur, pr = right
    ps, us = star_state(rl, ul, pl, rr, ur, pr, g)
    cl, cr = np.sqrt(g * pl / rl), np.sqrt(g * pr / rr)
    s = (np.asarray(x, dtype=float) - x0) / t
    rho = np.empty_like(s); u = np.empty_like(s); p = np.empty_like(s)
    gm = (g - 1.0) / (g + 1.0)
    for n, si in enumerate(s):
        if si <= us:  # left of contact
            if ps > pl:  # left shock
                sl = ul - cl * np.sqrt((g + 1) / (2 * g) * ps / pl + (g - 1) / (2 * g))
                if si <= sl:
                    rho[n], u[n], p[n] = rl, ul, pl
                else:
                    rho[n] = rl * (ps / pl + gm) / (gm * ps / pl + 1.0)
                    u[n], p[n] = us, ps
            else:  # left rarefaction
                shl = ul - cl
                cls = cl * (ps / pl) ** ((g - 1) / (2 * g))
                stl = us - cls
                if si <= shl:
                    rho[n], u[n], p[n] = rl, ul, pl
                elif si >= stl:
                    rho[n] = rl * (ps / pl) ** (1.0 / g)
                    u[n], p[n] = us, ps
                else:
                    c = 2.0 / (g + 1) * (cl + (g - 1) / 2 * (ul - si))
                    u[n] = 2.0 / (g + 1) * (cl + (g - 1) / 2 * ul + si)
                    rho[n] = rl * (c / cl) ** (2.0 / (g - 1))
                    p[n] = pl * (c / cl) ** (2.0 * g / (g - 1))
        else:  # right of contact
            if ps > pr:
                sr = ur + cr * np.sqrt((g + 1) / (2 * g) * ps / pr + (g - 1) / (2 * g))
                if si >= sr:
                    rho[n], u[n], p[n] = rr, ur, pr
                else:
                    rho[n] = rr * (ps / pr + gm) / (gm * ps / pr + 1.0)
                    u[n], p[n] = us, ps
            else:
                shr = ur + cr
                crs = cr * (ps / pr) ** ((g - 1) / (2 * g))
                str_ = us + crs
                if si >= shr:
                    rho[n], u[n], p[n] = rr, ur, pr
                elif si <= str_:
                    rho[n] = rr * (ps / pr) ** (1.0 / g)
                    u[n], p[n] = us, ps
                else:
                    c = 2.0 / (g + 1) * (cr - (g - 1) / 2 * (ur - si))
                    u[n] = 2.0 / (g + 1) * (-cr + (g - 1) / 2 * ur + si)
                    rho[n] = rr * (c / cr) ** (2.0 / (g - 1))
                    p[n] = pr * (c / cr) ** (2.0 * g / (g - 1))
    return rho, u, p


def sod_exact(x, t):
    return sample(x, t, 0.5, (1.0, 0.0, 1.0), (0.125, 0.0, 0.1))
