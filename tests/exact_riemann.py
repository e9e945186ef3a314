"""Exact solution of the 1D Riemann problem of the Euler equations for an
ideal gas, from the mathematics in E. F. Toro, "Riemann Solvers and Numerical
Methods for Fluid Dynamics" (1999), chapter 4: the star-region pressure is
the root of f(p) = f_L(p) + f_R(p) + (u_R - u_L) with shock (Rankine-Hugoniot)
or rarefaction (isentropic) branches, found by Newton iteration; the solution
is then sampled along x/t.  Used to validate the oracle (known-answer Sod).
"""
from __future__ import annotations

import numpy as np


def _f_k(p, rho_k, p_k, gamma):
    a_k = np.sqrt(gamma * p_k / rho_k)
    if p > p_k:  # shock
        A = 2.0 / ((gamma + 1.0) * rho_k)
        B = (gamma - 1.0) / (gamma + 1.0) * p_k
        f = (p - p_k) * np.sqrt(A / (p + B))
        df = np.sqrt(A / (B + p)) * (1.0 - (p - p_k) / (2.0 * (B + p)))
    else:  # rarefaction
        e = (gamma - 1.0) / (2.0 * gamma)
        f = 2.0 * a_k / (gamma - 1.0) * ((p / p_k) ** e - 1.0)
        df = 1.0 / (rho_k * a_k) * (p / p_k) ** (-(gamma + 1.0) / (2.0 * gamma))
    return f, df


def star_state(rho_l, u_l, p_l, rho_r, u_r, p_r, gamma):
    """Pressure and velocity of the star region."""
    a_l = np.sqrt(gamma * p_l / rho_l)
    a_r = np.sqrt(gamma * p_r / rho_r)
    if 2.0 * (a_l + a_r) / (gamma - 1.0) <= u_r - u_l:
        raise ValueError("vacuum is generated")
    p = max(1e-12, 0.5 * (p_l + p_r) - 0.125 * (u_r - u_l) * (rho_l + rho_r) * (a_l + a_r))
    for _ in range(200):
        fl, dfl = _f_k(p, rho_l, p_l, gamma)
        fr, dfr = _f_k(p, rho_r, p_r, gamma)
        f = fl + fr + (u_r - u_l)
        p_new = max(1e-14, p - f / (dfl + dfr))
        if abs(p_new - p) <= 1e-14 * 0.5 * (p_new + p):
            p = p_new
            break
        p = p_new
    fl, _ = _f_k(p, rho_l, p_l, gamma)
    fr, _ = _f_k(p, rho_r, p_r, gamma)
    u = 0.5 * (u_l + u_r) + 0.5 * (fr - fl)
    return p, u


def sample(x, t, x0, left, right, gamma):
    """rho, u, p at positions x and time t > 0 for the split at x0."""
    rho_l, u_l, p_l = left
    rho_r, u_r, p_r = right
    p_s, u_s = star_state(rho_l, u_l, p_l, rho_r, u_r, p_r, gamma)
    a_l = np.sqrt(gamma * p_l / rho_l)
    a_r = np.sqrt(gamma * p_r / rho_r)
    g1, gp = gamma - 1.0, gamma + 1.0
    out = np.zeros((3, len(x)))
    for n, xi in enumerate(x):
        s = (xi - x0) / t
        if s <= u_s:  # left of the contact
            if p_s > p_l:  # left shock
                sl = u_l - a_l * np.sqrt(gp / (2 * gamma) * p_s / p_l + g1 / (2 * gamma))
                if s <= sl:
                    out[:, n] = (rho_l, u_l, p_l)
                else:
                    r = rho_l * ((p_s / p_l + g1 / gp) / (g1 / gp * p_s / p_l + 1.0))
                    out[:, n] = (r, u_s, p_s)
            else:  # left rarefaction
                shl = u_l - a_l
                a_sl = a_l * (p_s / p_l) ** (g1 / (2 * gamma))
                stl = u_s - a_sl
                if s <= shl:
                    out[:, n] = (rho_l, u_l, p_l)
                elif s >= stl:
                    out[:, n] = (rho_l * (p_s / p_l) ** (1.0 / gamma), u_s, p_s)
                else:
                    c = 2.0 / gp + g1 / (gp * a_l) * (u_l - s)
                    out[:, n] = (rho_l * c ** (2.0 / g1),
                                 2.0 / gp * (a_l + g1 / 2.0 * u_l + s),
                                 p_l * c ** (2.0 * gamma / g1))
        else:  # right of the contact
            if p_s > p_r:  # right shock
                sr = u_r + a_r * np.sqrt(gp / (2 * gamma) * p_s / p_r + g1 / (2 * gamma))
                if s >= sr:
                    out[:, n] = (rho_r, u_r, p_r)
                else:
                    r = rho_r * ((p_s / p_r + g1 / gp) / (g1 / gp * p_s / p_r + 1.0))
                    out[:, n] = (r, u_s, p_s)
            else:  # right rarefaction
                shr = u_r + a_r
                a_sr = a_r * (p_s / p_r) ** (g1 / (2 * gamma))
                str_ = u_s + a_sr
                if s >= shr:
                    out[:, n] = (rho_r, u_r, p_r)
                elif s <= str_:
                    out[:, n] = (rho_r * (p_s / p_r) ** (1.0 / gamma), u_s, p_s)
                else:
                    c = 2.0 / gp - g1 / (gp * a_r) * (u_r - s)
                    out[:, n] = (rho_r * c ** (2.0 / g1),
                                 2.0 / gp * (-a_r + g1 / 2.0 * u_r + s),
                                 p_r * c ** (2.0 * gamma / g1))
    return out
