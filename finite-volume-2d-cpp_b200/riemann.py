"""Exact solution of the 1D Euler Riemann problem (ideal gas), following the
published exact solver of E. F. Toro, "Riemann Solvers and Numerical Methods
for Fluid Dynamics", 3rd ed., chapter 4: a Newton iteration on the star
pressure with the two-wave pressure functions, then sampling of the wave
pattern (shock or rarefaction on either side).

Used to measure the discretisation error of the batched Riemann-strip
workload (each strip is a 1D Riemann problem in x) in density and pressure,
so that FP32-bulk and FP64 runs can be compared at equal final L2 error.
"""
import numpy as np


def _pressure_function(p, rho_k, p_k, c_k, gamma):
    """f_K(p) and its derivative (Toro eqs. 4.6-4.7, 4.37)."""
    if p > p_k:  # shock
        a = 2.0 / ((gamma + 1.0) * rho_k)
        b = (gamma - 1.0) / (gamma + 1.0) * p_k
        s = np.sqrt(a / (p + b))
        return (p - p_k) * s, s * (1.0 - 0.5 * (p - p_k) / (b + p))
    # rarefaction
    r = (p / p_k) ** ((gamma - 1.0) / (2.0 * gamma))
    return 2.0 * c_k / (gamma - 1.0) * (r - 1.0), 1.0 / (rho_k * c_k) * (p / p_k) ** (-(gamma + 1.0) / (2.0 * gamma))


def star_state(left, right, gamma=1.4, tol=1e-14, max_iter=200):
    """(p*, u*) of the Riemann problem with primitive states (rho, u, p)."""
    rl, ul, pl = left
    rr, ur, pr = right
    cl, cr = np.sqrt(gamma * pl / rl), np.sqrt(gamma * pr / rr)
    du = ur - ul
    if 2.0 * (cl + cr) / (gamma - 1.0) <= du:
        raise ValueError("the initial data generate a vacuum")
    # two-rarefaction guess (Toro eq. 4.46), kept positive
    z = (gamma - 1.0) / (2.0 * gamma)
    p = ((cl + cr - 0.5 * (gamma - 1.0) * du) / (cl / pl ** z + cr / pr ** z)) ** (1.0 / z)
    p = max(p, tol)
    for _ in range(max_iter):
        fl, dl = _pressure_function(p, rl, pl, cl, gamma)
        fr, dr = _pressure_function(p, rr, pr, cr, gamma)
        p_new = max(p - (fl + fr + du) / (dl + dr), tol)
        if abs(p_new - p) <= tol * 0.5 * (p_new + p):
            p = p_new
            break
        p = p_new
    fl, _ = _pressure_function(p, rl, pl, cl, gamma)
    fr, _ = _pressure_function(p, rr, pr, cr, gamma)
    return p, 0.5 * (ul + ur) + 0.5 * (fr - fl)


def sample(x, t, left, right, gamma=1.4, x0=0.5):
    """Density, velocity and pressure at positions x and time t > 0 (Toro 4.5)."""
    rl, ul, pl = left
    rr, ur, pr = right
    cl, cr = np.sqrt(gamma * pl / rl), np.sqrt(gamma * pr / rr)
    ps, us = star_state(left, right, gamma)
    g1 = (gamma - 1.0) / (gamma + 1.0)
    s = (np.asarray(x, np.float64) - x0) / t
    rho = np.empty_like(s); u = np.empty_like(s); p = np.empty_like(s)

    def side(mask, rk, uk, pk, ck, sign):
        # sign = -1: left wave family, +1: right wave family; mask = points on that side of the contact
        sm = s[mask]
        rr_, uu, pp = np.empty_like(sm), np.empty_like(sm), np.empty_like(sm)
        if ps > pk:  # shock
            speed = uk + sign * ck * np.sqrt((gamma + 1.0) / (2.0 * gamma) * ps / pk + (gamma - 1.0) / (2.0 * gamma))
            rho_star = rk * (ps / pk + g1) / (g1 * ps / pk + 1.0)
            outside = sm * sign > speed * sign
            rr_[outside], uu[outside], pp[outside] = rk, uk, pk
            rr_[~outside], uu[~outside], pp[~outside] = rho_star, us, ps
        else:  # rarefaction
            rho_star = rk * (ps / pk) ** (1.0 / gamma)
            c_star = ck * (ps / pk) ** ((gamma - 1.0) / (2.0 * gamma))
            head, tail = uk + sign * ck, us + sign * c_star
            outside = sm * sign > head * sign
            inside = (~outside) & (sm * sign > tail * sign)
            star = ~(outside | inside)
            rr_[outside], uu[outside], pp[outside] = rk, uk, pk
            rr_[star], uu[star], pp[star] = rho_star, us, ps
            si = sm[inside]
            c = 2.0 / (gamma + 1.0) * (ck - sign * (gamma - 1.0) / 2.0 * (uk - si))
            uu[inside] = 2.0 / (gamma + 1.0) * (-sign * ck + (gamma - 1.0) / 2.0 * uk + si)
            rr_[inside] = rk * (c / ck) ** (2.0 / (gamma - 1.0))
            pp[inside] = pk * (c / ck) ** (2.0 * gamma / (gamma - 1.0))
        rho[mask], u[mask], p[mask] = rr_, uu, pp

    lm = s <= us
    side(lm, rl, ul, pl, cl, -1.0)
    side(~lm, rr, ur, pr, cr, +1.0)
    return rho, u, p
