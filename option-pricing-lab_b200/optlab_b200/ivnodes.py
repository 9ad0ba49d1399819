"""Vegas on the implied-vol nodes of the reference's risk grid, from the adjoint's gradient of the local-variance table.

The reference's node vega (packages/risk/src/optlab/risk/greeks.py:217-226) bumps the implied volatility of one name by
a tent of its risk grid, sigma'(k, T) = sigma(k, T) + h phi_i(k, T) psi_j(T), re-tabulates Dupire's local variance of
the bumped surface per step (packages/risk/src/optlab/risk/surfaces.py:95-167, on the base's grid in k) and revalues:
vega_ij = (V(h) - V(0)) 0.01 / h, per implied vol point. The adjoint gives dV / d(table entry); here the chain rule
maps it onto the nodes with the exact derivative of each table entry with respect to the tent's amplitude, so one
backward pass gives every node vega:

    vega_ij = 0.01 sum_{step r, point x} dV/dL[r, x] dL[r, x]/dH_ij.

The grid (packages/risk/src/optlab/risk/grid.py:1-26, restated here): strikes at forward moneyness 60 % .. 140 %
(log-moneyness nodes), tenors 1m .. 5y. Tenor tents are a partition of unity in T whose weight passes between
neighbouring tenors along the smootherstep s(u) = u^3 (10 - 15 u + 6 u^2), flat at one beyond the end tenors. Strike
tents are the hats of the log-strike nodes (flat beyond the end nodes) smoothed by a Gaussian of width
l(k, T) = c(k) sqrt(max(T, 1/52)), c(k) = c_wing - (c_wing - c_atm) exp(-k^2 / a^2): a hat is a constant plus ramps
c_m (k - k_m)_+, and a smoothed ramp is u Phi(u / l) + l n(u / l) with u = k - k_m.

The table entry at (k, T) is L = clip(w_T / max(g, 1e-6), 1e-4, 4) of the total variance w = T sigma'^2 (T floored at a
day), with Gatheral's g(w, w_k, w_kk, k). With a = h phi psi the bump field, w moves by dw = 2 T sigma da, w_k by
2 T (sigma_k da + sigma da_k), w_kk by 2 T (2 sigma_k da_k + sigma_kk da + sigma da_kk), w_T by
2 sigma da + 2 T (sigma_T da + sigma da_T); so dL = (dw_T - L dg) / g where L is inside its clip and g above its floor,
and 0 elsewhere: a linear combination c0 da + c1 da_k + c2 da_kk + c3 da_T with coefficients of the base surface.
"""

from __future__ import annotations

import numpy as np
from scipy.special import ndtr

STRIKES = (0.6, 0.7, 0.8, 0.9, 0.95, 1.0, 1.05, 1.1, 1.2, 1.4)  # forward moneyness K / F
TENORS = (1 / 12, 0.25, 0.5, 1.0, 1.5, 2.0, 3.0, 5.0)  # years
LOG_STRIKES = np.log(np.array(STRIKES))
WIDTH_ATM, WIDTH_WING, WIDTH_SCALE = 0.04, 0.12, 0.15  # c(k) at the money, in the wings, and the scale a
WIDTH_T_FLOOR = 1.0 / 52
MIN_EXPIRY = 1.0 / 365
G_FLOOR, LV_FLOOR, LV_CAP = 1e-6, 1e-4, 4.0
PER_POINT = 0.01  # vegas per implied vol point


def _smootherstep(u):
    u = np.clip(u, 0.0, 1.0)
    return u**3 * (10.0 - 15.0 * u + 6.0 * u * u), 30.0 * u * u * (1.0 - u) ** 2


def tenor_tents(T):
    """(psi, dpsi/dT), each (n_tenors, *T.shape)."""
    T = np.asarray(T, dtype=float)
    nodes = np.asarray(TENORS)
    psi = np.zeros((len(nodes), *T.shape))
    dpsi = np.zeros_like(psi)
    psi[0] = T <= nodes[0]
    psi[-1] = T >= nodes[-1]
    j = np.clip(np.searchsorted(nodes, T, side="right") - 1, 0, len(nodes) - 2)
    a, b = nodes[j], nodes[j + 1]
    strictly = (T > a) & (T < b)
    s, ds = _smootherstep((T - a) / (b - a))
    for n in range(len(nodes) - 1):
        sel = strictly & (j == n)
        psi[n] += np.where(sel, 1.0 - s, 0.0)
        psi[n + 1] += np.where(sel, s, 0.0)
        dpsi[n] += np.where(sel, -ds / (b - a), 0.0)
        dpsi[n + 1] += np.where(sel, ds / (b - a), 0.0)
    for n in range(1, len(nodes) - 1):  # exactly on an inner tenor: that tent alone
        psi[n] = np.where(T == nodes[n], 1.0, psi[n])
    return psi, dpsi


def _hat_ramps():
    """Per strike node, its hat as (constant, [(knot, slope change), ...]): sum of c (k - knot)_+ plus the constant."""
    x = LOG_STRIKES
    n = len(x)
    out = []
    for i in range(n):
        if i == 0:
            d = x[1] - x[0]
            out.append((1.0, ((x[0], -1 / d), (x[1], 1 / d))))
        elif i == n - 1:
            d = x[-1] - x[-2]
            out.append((0.0, ((x[-2], 1 / d), (x[-1], -1 / d))))
        else:
            dl, dr = x[i] - x[i - 1], x[i + 1] - x[i]
            out.append((0.0, ((x[i - 1], 1 / dl), (x[i], -1 / dl - 1 / dr), (x[i + 1], 1 / dr))))
    return out


_HATS = _hat_ramps()


def smoothing_width(k, T):
    """l(k, T) and its derivatives l_k, l_kk, l_T."""
    k, T = np.asarray(k, dtype=float), np.asarray(T, dtype=float)
    root = np.sqrt(np.maximum(T, WIDTH_T_FLOOR))
    span, a2 = WIDTH_WING - WIDTH_ATM, WIDTH_SCALE**2
    e = np.exp(-k * k / a2)
    c, ck, ckk = WIDTH_WING - span * e, span * e * 2 * k / a2, span * e * (2 / a2 - 4 * k * k / a2**2)
    return c * root, ck * root, ckk * root, np.where(T < WIDTH_T_FLOOR, 0.0, 0.5 * c / root)


def strike_tents(k, T):
    """(phi, dphi/dk, d2phi/dk2, dphi/dT), each (n_strikes, *shape): the smoothed hats. A smoothed ramp
    R = u Phi(z) + l n(z) (z = u / l) has R_k = Phi(z) + n(z) l_k, R_kk = n(z) ((1 - z l_k)^2 / l + l_kk) and
    R_T = n(z) l_T (dR/dl = n(z))."""
    k, T = np.broadcast_arrays(np.asarray(k, dtype=float), np.asarray(T, dtype=float))
    ell, lk, lkk, lT = smoothing_width(k, T)
    knots = np.unique(np.concatenate([[kn for kn, _ in r] for _, r in _HATS]))
    ramp = {}
    for kn in knots:
        u = k - kn
        z = u / ell
        pdf = np.exp(-0.5 * z * z) / np.sqrt(2 * np.pi)
        cdf = ndtr(z)
        ramp[kn] = (u * cdf + ell * pdf, cdf + pdf * lk, pdf * ((1 - z * lk) ** 2 / ell + lkk), pdf * lT)
    out = np.zeros((4, len(_HATS), *k.shape))
    for i, (const, parts) in enumerate(_HATS):
        out[0, i] = const
        for kn, c in parts:
            for q in range(4):
                out[q, i] += c * ramp[kn][q]
    return out[0], out[1], out[2], out[3]


def _g_and_partials(w, wk, wkk, k):
    A = 1.0 - k * wk / (2.0 * w)
    g = A * A - 0.25 * wk * wk * (1.0 / w + 0.25) + 0.5 * wkk
    g_w = A * k * wk / (w * w) + 0.25 * wk * wk / (w * w)
    g_wk = -A * k / w - 0.5 * wk * (1.0 / w + 0.25)
    return g, g_w, g_wk


def table_sensitivity(surface, t0, n_x: int, sd_range=(-8.0, 6.0)):
    """The per-step local-variance table of `surface` (the reference's tabulation: n_x points over sd_range ATM
    standard deviations at each step start) and the coefficients (c0, c1, c2, c3) of dL in the bump field's
    (a, a_k, a_kk, a_T): returns (k, T, L, c), k and T (steps, n_x), c (4, steps, n_x)."""
    t0 = np.asarray(t0, dtype=float)
    T1 = np.maximum(t0, MIN_EXPIRY)
    sd = np.sqrt(np.asarray(surface.w(np.zeros_like(T1), T1), dtype=float))
    lo, hi = sd_range[0] * sd, sd_range[1] * sd
    k = lo[:, None] + np.arange(n_x)[None, :] * ((hi - lo) / (n_x - 1))[:, None]
    k[:, -1] = hi
    T = np.broadcast_to(T1[:, None], k.shape)
    w, wk, wkk, wT = (np.asarray(a, dtype=float) for a in surface.derivatives(k, T))
    s = np.sqrt(np.maximum(w, 1e-300) / T)
    sk = wk / (2 * T * s)
    skk = (wkk - 2 * T * sk**2) / (2 * T * s)
    sT = (wT - s**2) / (2 * T * s)
    g, g_w, g_wk = _g_and_partials(w, wk, wkk, k)
    gf = np.maximum(g, G_FLOOR)
    raw = wT / gf
    L = np.clip(raw, LV_FLOOR, LV_CAP)
    live = (g > G_FLOOR) & (raw > LV_FLOOR) & (raw < LV_CAP)
    c0 = (2 * s + 2 * T * sT - L * (2 * T * s * g_w + 2 * T * sk * g_wk + T * skk)) / gf
    c1 = -L * (2 * T * s * g_wk + 2 * T * sk) / gf
    c2 = -L * T * s / gf
    c3 = 2 * T * s / gf
    c = np.where(live[None], np.stack([c0, c1, c2, c3]), 0.0)
    return k, T, L, c


def node_table_derivative(surface, t0, n_x: int, i: int, j: int, sd_range=(-8.0, 6.0)):
    """dL/dH_ij over the whole per-step table (steps, n_x): the table's derivative in node (i, j)'s amplitude."""
    k, T, _, c = table_sensitivity(surface, t0, n_x, sd_range)
    phi, phik, phikk, phiT = strike_tents(k, T)
    psi, dpsi = tenor_tents(T[:, 0])
    pj, dpj = psi[j][:, None], dpsi[j][:, None]
    return c[0] * phi[i] * pj + c[1] * phik[i] * pj + c[2] * phikk[i] * pj + c[3] * (phiT[i] * pj + phi[i] * dpj)


def node_jacobian_contract(grad, surface, t0, n_x: int, sd_range=(-8.0, 6.0)):
    """Node vegas (n_strikes, n_tenors) per implied vol point of one name: sum over the name's table of
    grad[r, x] dL[r, x]/dH_ij, times 0.01. grad: (steps, n_x), dV/d(table entry) for the rows of t0."""
    k, T, _, c = table_sensitivity(surface, t0, n_x, sd_range)
    phi, phik, phikk, phiT = strike_tents(k, T)  # (n_strikes, steps, n_x)
    psi, dpsi = tenor_tents(T[:, 0])  # (n_tenors, steps)
    G = np.asarray(grad, dtype=float)
    # sum_x G (c0 phi + c1 phi_k + c2 phi_kk + c3 phi_T) per (strike, step): the part that multiplies psi_j
    A = np.einsum("rx,irx->ir", G * c[0], phi) + np.einsum("rx,irx->ir", G * c[1], phik)
    A += np.einsum("rx,irx->ir", G * c[2], phikk) + np.einsum("rx,irx->ir", G * c[3], phiT)
    B = np.einsum("rx,irx->ir", G * c[3], phi)  # multiplies dpsi_j / dT
    return PER_POINT * (A @ psi.T + B @ dpsi.T)


# The reference's skew move (packages/structured/src/optlab/structured/surfaces.py:10-50): a rotation of the implied
# vols around the forward, -skew c sqrt(1 / max(T, 1m)) tanh(k / 0.3), with c such that the 90 % - 110 % vol gap at one
# year rises by exactly `skew`; it saturates at a few 0.3 of log-moneyness.
SKEW_WIDTH, SKEW_T_FLOOR = 0.3, 1.0 / 12
SKEW_NORM = 1.0 / (np.tanh(-np.log(0.9) / SKEW_WIDTH) + np.tanh(np.log(1.1) / SKEW_WIDTH))


def skew_rotation(k, T, skew: float):
    """The skew move in implied vol at (k, T) and its derivatives in k, k twice and T."""
    k, T = np.broadcast_arrays(np.asarray(k, dtype=float), np.asarray(T, dtype=float))
    if not skew:
        z = np.zeros(k.shape)
        return z, z, z, z
    Tf = np.maximum(T, SKEW_T_FLOOR)
    scale = np.sqrt(1.0 / Tf)
    dscale = np.where(T < SKEW_T_FLOOR, 0.0, -0.5 * scale / Tf)
    amp = -skew * SKEW_NORM
    th = np.tanh(k / SKEW_WIDTH)
    sech2 = 1.0 - th * th
    return (amp * scale * th, amp * scale * sech2 / SKEW_WIDTH, -2.0 * amp * scale * th * sech2 / SKEW_WIDTH**2,
            amp * dscale * th)


def moved_derivatives(surface, k, T, parallel: float = 0.0, relative: float = 0.0, skew: float = 0.0, nodes=None):
    """w, w_k, w_kk, w_T of the surface with its implied vols moved as the reference's risk scenarios move them
    (packages/risk/src/optlab/risk/surfaces.py:95-204): sigma' = sigma (1 + relative) + parallel + skew rotation
    + sum_ij nodes[i, j] phi_i psi_j, each term with its exact derivatives, and w' = T sigma'^2."""
    k, T = np.broadcast_arrays(np.asarray(k, dtype=float), np.asarray(T, dtype=float))
    w, wk, wkk, wT = (np.asarray(a, dtype=float) for a in surface.derivatives(k, T))
    s = np.sqrt(np.maximum(w, 1e-300) / T)
    sk = wk / (2 * T * s)
    skk = (wkk - 2 * T * sk**2) / (2 * T * s)
    sT = (wT - s**2) / (2 * T * s)
    a, ak, akk, aT = skew_rotation(k, T, skew)
    a = a + parallel
    if nodes is not None and np.any(nodes):
        H = np.asarray(nodes, dtype=float)
        phi, phik, phikk, phiT = strike_tents(k, T)
        psi, dpsi = tenor_tents(T)
        a = a + np.einsum("ij,i...,j...->...", H, phi, psi)
        ak = ak + np.einsum("ij,i...,j...->...", H, phik, psi)
        akk = akk + np.einsum("ij,i...,j...->...", H, phikk, psi)
        aT = aT + np.einsum("ij,i...,j...->...", H, phiT, psi) + np.einsum("ij,i...,j...->...", H, phi, dpsi)
    g1 = 1.0 + relative
    s2, sk2, skk2, sT2 = s * g1 + a, sk * g1 + ak, skk * g1 + akk, sT * g1 + aT
    return T * s2**2, 2 * T * s2 * sk2, 2 * T * (sk2**2 + s2 * skk2), s2**2 + 2 * T * s2 * sT2


def moved_local_var(surface, k, T, **moves):
    """Dupire's local variance of the moved surface (moved_derivatives), read at no earlier expiry than a day, as the
    reference's bumped surfaces read theirs: clip(w_T / max(g, 1e-6), 1e-4, 4)."""
    T = np.maximum(np.asarray(T, dtype=float), MIN_EXPIRY)
    w, wk, wkk, wT = moved_derivatives(surface, k, T, **moves)
    g, _, _ = _g_and_partials(w, wk, wkk, np.broadcast_to(np.asarray(k, dtype=float), w.shape))
    return np.clip(wT / np.maximum(g, G_FLOOR), LV_FLOOR, LV_CAP)


def grid_points(lo, inv_dx, n_x: int):
    """The n_x log-moneyness points of uniform rows (lo, inv_dx), (rows, n_x)."""
    lo, inv = np.asarray(lo, dtype=float), np.asarray(inv_dx, dtype=float)
    hi = lo + (n_x - 1) / inv
    k = lo[:, None] + np.arange(n_x)[None, :] * ((hi - lo) / (n_x - 1))[:, None]
    k[:, -1] = hi
    return k


def bumped_table(surface, t0, n_x: int, nodes, sd_range=(-8.0, 6.0)):
    """The per-step table of the surface with its implied vols moved by sum_ij nodes[i, j] phi_i psi_j, exactly (not
    linearised), on the base's grid: the reference's TentBumpedSurface.local_var_rows. For parity checks."""
    t0 = np.asarray(t0, dtype=float)
    T1 = np.maximum(t0, MIN_EXPIRY)
    sd = np.sqrt(np.asarray(surface.w(np.zeros_like(T1), T1), dtype=float))
    lo, hi = sd_range[0] * sd, sd_range[1] * sd
    k = lo[:, None] + np.arange(n_x)[None, :] * ((hi - lo) / (n_x - 1))[:, None]
    k[:, -1] = hi
    T = np.broadcast_to(T1[:, None], k.shape)
    return lo, (n_x - 1) / (hi - lo), moved_local_var(surface, k, T, nodes=nodes)
