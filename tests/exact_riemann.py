"""Exact solution of the 1-D Riemann problem for an ideal gas (Toro, "Riemann
Solvers and Numerical Methods for Fluid Dynamics", 3rd ed., ch. 4): a Newton
solve for the star pressure, then self-similar sampling.  Independent of the
solver under test; used as the Sod reference."""
from __future__ import annotations

import math


def _f_side(p, rho_k, p_k, a_k, g):
    if p > p_k:  # shock branch
        A = 2.0 / ((g + 1.0) * rho_k)
        B = (g - 1.0) / (g + 1.0) * p_k
        q = math.sqrt(A / (B + p))
        return (p - p_k) * q, q * (1.0 - 0.5 * (p - p_k) / (B + p))
    # rarefaction branch
    r = p / p_k
    f = 2.0 * a_k / (g - 1.0) * (r ** ((g - 1.0) / (2.0 * g)) - 1.0)
    df = 1.0 / (rho_k * a_k) * r ** (-(g + 1.0) / (2.0 * g))
    return f, df


def star(rho_l, u_l, p_l, rho_r, u_r, p_r, g):
    a_l, a_r = math.sqrt(g * p_l / rho_l), math.sqrt(g * p_r / rho_r)
    p = max(0.5 * (p_l + p_r), 1e-6)
    for _ in range(100):
        fl, dfl = _f_side(p, rho_l, p_l, a_l, g)
        fr, dfr = _f_side(p, rho_r, p_r, a_r, g)
        p_new = max(p - (fl + fr + (u_r - u_l)) / (dfl + dfr), 1e-9)
        done = abs(2.0 * (p_new - p) / (p_new + p)) < 1e-12
        p = p_new
        if done:
            break
    fl, _ = _f_side(p, rho_l, p_l, a_l, g)
    fr, _ = _f_side(p, rho_r, p_r, a_r, g)
    return p, 0.5 * (u_l + u_r) + 0.5 * (fr - fl)


def density(s, rho_l, u_l, p_l, rho_r, u_r, p_r, g, p_s=None, u_s=None):
    """Exact density at similarity coordinate s = (x - x0)/t."""
    if p_s is None:
        p_s, u_s = star(rho_l, u_l, p_l, rho_r, u_r, p_r, g)
    a_l, a_r = math.sqrt(g * p_l / rho_l), math.sqrt(g * p_r / rho_r)
    g1 = (g - 1.0) / (g + 1.0)
    if s <= u_s:
        if p_s > p_l:
            sl = u_l - a_l * math.sqrt((g + 1.0) / (2.0 * g) * p_s / p_l + (g - 1.0) / (2.0 * g))
            return rho_l if s <= sl else rho_l * (p_s / p_l + g1) / (g1 * p_s / p_l + 1.0)
        if s <= u_l - a_l:
            return rho_l
        a_st = a_l * (p_s / p_l) ** ((g - 1.0) / (2.0 * g))
        if s >= u_s - a_st:
            return rho_l * (p_s / p_l) ** (1.0 / g)
        a = 2.0 / (g + 1.0) * (a_l + (g - 1.0) / 2.0 * (u_l - s))
        return rho_l * (a / a_l) ** (2.0 / (g - 1.0))
    if p_s > p_r:
        sr = u_r + a_r * math.sqrt((g + 1.0) / (2.0 * g) * p_s / p_r + (g - 1.0) / (2.0 * g))
        return rho_r if s >= sr else rho_r * (p_s / p_r + g1) / (g1 * p_s / p_r + 1.0)
    if s >= u_r + a_r:
        return rho_r
    a_st = a_r * (p_s / p_r) ** ((g - 1.0) / (2.0 * g))
    if s <= u_s + a_st:
        return rho_r * (p_s / p_r) ** (1.0 / g)
    a = 2.0 / (g + 1.0) * (a_r - (g - 1.0) / 2.0 * (u_r - s))
    return rho_r * (a / a_r) ** (2.0 / (g - 1.0))
