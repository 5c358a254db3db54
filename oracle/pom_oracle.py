"""CPU oracle for the NeuralPOM physical time step -- TEST INFRASTRUCTURE ONLY.

This module restates, in numpy, the arithmetic of the two reference POM cores
(`src/neuralpom/cores/explicit/` and `src/neuralpom/cores/implicit_p0_fixed/`)
so that the CUDA implementation in ``neuralpom_b200`` can be checked against it
on seeded inputs of any size.  Only ``tests/``, ``__graft_entry__.smoke()`` and
``bench.py``'s CPU-baseline leg may import it; the product never does.

Parity pinning: the restatement is checked against golden vectors produced by
running the reference core itself (``tests/golden/make_golden.py``) and, when the
reference sources are present, directly against the reference operators
(``tests/test_oracle_reference.py``).

Conventions follow the reference: C-contiguous ``(im, jm, kb)`` arrays with the
sigma level ``k`` fastest, float32 by default (float64 when the state is
float64), Python-float constants folded in double precision before they meet an
array (numpy 2 weak-scalar rules match torch's here).  Every function cites the
reference lines it restates.
"""
from __future__ import annotations

import math

import numpy as np


# ---------------------------------------------------------------------------
# small helpers
# ---------------------------------------------------------------------------

def _b(a2):
    """(im, jm) -> (im, jm, 1) broadcast view."""
    return a2[:, :, None]


def _cumsum_k(inc):
    """Cumulative sum over the last axis, accumulated in float64 and rounded
    per element, which is what torch's CPU ``cumsum`` does for float32
    (``at::acc_type<float, false>`` is double)."""
    return np.cumsum(inc.astype(np.float64), axis=-1).astype(inc.dtype)


def _sum_k(a):
    """Sum over the last axis (torch.sum(..., dim=2) in the reference)."""
    return a.sum(axis=-1, dtype=a.dtype)


# ---------------------------------------------------------------------------
# surface forcing
# ---------------------------------------------------------------------------

def surface_fluxes(S, P):
    """Inner-domain surface fluxes shared by both cores.

    Restates ``explicit/time_loop.py:118-164`` and
    ``implicit_p0_fixed/forcing/surface.py:20-68`` (identical arithmetic):
    e_atmos/vfluxf/swrad cleared on the interior, w(:,:,0)=vfluxf,
    wtsurf += vfluxf*(tatm-t-tbias), wssurf = vfluxf*(0-s-sbias).
    """
    im, jm = P.im, P.jm
    I, J = slice(1, im - 1), slice(1, jm - 1)
    for name in ("e_atmos", "vfluxf", "swrad"):
        S[name] = S[name].copy()
        S[name][I, J] = 0.0
    w = S["w"].copy()
    w[I, J, 0] = S["vfluxf"][I, J]
    S["w"] = w
    t_surf = S["t"][I, J, 0]
    tatm = t_surf + P.tbias
    delta = S["vfluxf"][I, J] * (tatm - t_surf - P.tbias)
    wt = S["wtsurf"].copy()
    wt[I, J] = wt[I, J] + delta
    S["wtsurf"] = wt
    s_surf = S["s"][I, J, 0]
    ws = S["wssurf"].copy()
    ws[I, J] = S["vfluxf"][I, J] * (0.0 - s_surf - P.sbias)
    S["wssurf"] = ws


def double_gyre_wind(S, P):
    """Implicit-core wind forcing rewritten before every step.

    Restates ``implicit_p0_fixed/forcing/surface.py:70-84``:
    wusurf = -(tau0/rhoref)*(1-cos(2*pi*(north_e-30)/20))*dum, wvsurf = 0.
    """
    tau0 = float(getattr(P, "double_gyre_wind_stress_pa", 0.1))
    kf = tau0 / P.rhoref
    arg = 2.0 * P.pi * (S["north_e"] - 30.0) / 20.0
    S["wusurf"] = -kf * (1.0 - np.cos(arg)) * S["dum"]
    S["wvsurf"] = np.zeros_like(S["wvsurf"])


# ---------------------------------------------------------------------------
# 3-D momentum advection (ADVCT)
# ---------------------------------------------------------------------------

def advct(S, P):
    """Horizontal momentum advection/diffusion with curvature terms.

    Restates ``explicit/baroclinic.py:14-260`` (the implicit copy
    ``implicit_p0_fixed/baroclinic.py:15-265`` only adds identity flux hooks
    for the closed basin).  Returns (curv, advx, advy).
    """
    u, v, ub, vb, aam = S["u"], S["v"], S["ub"], S["vb"], S["aam"]
    dt, dx, dy, aru, arv = S["dt"], S["dx"], S["dy"], S["aru"], S["arv"]
    im, jm, kb = u.shape
    K = slice(0, kb - 1)
    z3 = np.zeros_like(u)
    curv, advx, advy = z3.copy(), z3.copy(), z3.copy()

    i, j = slice(1, im - 1), slice(1, jm - 1)
    ip, imn = slice(2, im), slice(0, im - 2)
    jp, jmn = slice(2, jm), slice(0, jm - 2)
    t1 = (v[i, jp, K] + v[i, j, K]) * _b(dy[ip, j] - dy[imn, j])
    t2 = (u[ip, j, K] + u[i, j, K]) * _b(dx[i, jp] - dx[i, jmn])
    curv[i, j, K] = 0.25 * (t1 - t2) / (_b(dx[i, j] * dy[i, j]) + 1e-20)

    # --- x-momentum fluxes
    xflux, yflux = z3.copy(), z3.copy()
    xi, xip, xim = slice(1, im - 1), slice(2, im), slice(0, im - 2)
    tu1 = (_b(dt[xip, :]) + _b(dt[xi, :])) * u[xip, :, K]
    tu2 = (_b(dt[xi, :]) + _b(dt[xim, :])) * u[xi, :, K]
    xflux[xi, :, K] = 0.125 * (tu1 + tu2) * (u[xip, :, K] + u[xi, :, K])

    yi, yim, yj, yjm = slice(1, im), slice(0, im - 1), slice(1, jm), slice(0, jm - 1)
    tv1 = (_b(dt[yi, yj]) + _b(dt[yi, yjm])) * v[yi, yj, K]
    tv2 = (_b(dt[yim, yj]) + _b(dt[yim, yjm])) * v[yim, yj, K]
    yflux[yi, yj, K] = 0.125 * (tv1 + tv2) * (u[yi, yj, K] + u[yi, yjm, K])

    si, sim, sip = slice(1, im - 1), slice(0, im - 2), slice(2, im)
    sj, sjm = slice(1, jm), slice(0, jm - 1)
    grad_u = (ub[sip, sj, K] - ub[si, sj, K]) / (_b(dx[si, sj]) + 1e-20)
    xflux[si, sj, K] = xflux[si, sj, K] - _b(dt[si, sj]) * aam[si, sj, K] * 2.0 * grad_u
    dt_avg = 0.25 * (dt[si, sj] + dt[sim, sj] + dt[si, sjm] + dt[sim, sjm])
    aam_sum = aam[si, sj, K] + aam[sim, sj, K] + aam[si, sjm, K] + aam[sim, sjm, K]
    dtaam = _b(dt_avg) * aam_sum
    den_dy = _b(dy[si, sj] + dy[sim, sj] + dy[si, sjm] + dy[sim, sjm])
    den_dx = _b(dx[si, sj] + dx[sim, sj] + dx[si, sjm] + dx[sim, sjm])
    du_dy = (ub[si, sj, K] - ub[si, sjm, K]) / (den_dy + 1e-20)
    dv_dx = (vb[si, sj, K] - vb[sim, sj, K]) / (den_dx + 1e-20)
    yflux[si, sj, K] = yflux[si, sj, K] - dtaam * (du_dy + dv_dx)
    xflux[si, sj, K] *= _b(dy[si, sj])
    dx_sum = dx[si, sj] + dx[sim, sj] + dx[si, sjm] + dx[sim, sjm]
    yflux[si, sj, K] *= _b(0.25 * dx_sum)

    i, im1 = slice(1, im - 1), slice(0, im - 2)
    j, jp1 = slice(1, jm - 1), slice(2, jm)
    advx[i, j, K] = xflux[i, j, K] - xflux[im1, j, K] + yflux[i, jp1, K] - yflux[i, j, K]
    ic, icm = slice(2, im - 1), slice(1, im - 2)
    tc1 = curv[ic, j, K] * _b(dt[ic, j]) * (v[ic, jp1, K] + v[ic, j, K])
    tc2 = curv[icm, j, K] * _b(dt[icm, j]) * (v[icm, jp1, K] + v[icm, j, K])
    advx[ic, j, K] -= _b(aru[ic, j]) * 0.25 * (tc1 + tc2)

    # --- y-momentum fluxes
    xflux, yflux = z3.copy(), z3.copy()
    si, sim, sj, sjm = slice(1, im), slice(0, im - 1), slice(1, jm), slice(0, jm - 1)
    tu1 = (_b(dt[si, sj]) + _b(dt[sim, sj])) * u[si, sj, K]
    tu2 = (_b(dt[si, sjm]) + _b(dt[sim, sjm])) * u[si, sjm, K]
    xflux[si, sj, K] = 0.125 * (tu1 + tu2) * (v[si, sj, K] + v[sim, sj, K])

    sj, sjp, sjm = slice(1, jm - 1), slice(2, jm), slice(0, jm - 2)
    tv1 = (_b(dt[:, sjp]) + _b(dt[:, sj])) * v[:, sjp, K]
    tv2 = (_b(dt[:, sj]) + _b(dt[:, sjm])) * v[:, sj, K]
    yflux[:, sj, K] = 0.125 * (tv1 + tv2) * (v[:, sjp, K] + v[:, sj, K])

    si, sim = slice(1, im), slice(0, im - 1)
    dt_avg = 0.25 * (dt[si, sj] + dt[sim, sj] + dt[si, sjm] + dt[sim, sjm])
    aam_sum = aam[si, sj, K] + aam[sim, sj, K] + aam[si, sjm, K] + aam[sim, sjm, K]
    dtaam = _b(dt_avg) * aam_sum
    den_dy = _b(dy[si, sj] + dy[sim, sj] + dy[si, sjm] + dy[sim, sjm])
    den_dx = _b(dx[si, sj] + dx[sim, sj] + dx[si, sjm] + dx[sim, sjm])
    du_dy = (ub[si, sj, K] - ub[si, sjm, K]) / (den_dy + 1e-20)
    dv_dx = (vb[si, sj, K] - vb[sim, sj, K]) / (den_dx + 1e-20)
    xflux[si, sj, K] = xflux[si, sj, K] - dtaam * (du_dy + dv_dx)
    grad_v = (vb[si, sjp, K] - vb[si, sj, K]) / (_b(dy[si, sj]) + 1e-20)
    yflux[si, sj, K] = yflux[si, sj, K] - _b(dt[si, sj]) * aam[si, sj, K] * 2.0 * grad_v
    dy_sum = dy[si, sj] + dy[sim, sj] + dy[si, sjm] + dy[sim, sjm]
    xflux[si, sj, K] *= _b(0.25 * dy_sum)
    yflux[si, sj, K] *= _b(dx[si, sj])

    i, ip1 = slice(1, im - 1), slice(2, im)
    j, jm1 = slice(1, jm - 1), slice(0, jm - 2)
    advy[i, j, K] = xflux[ip1, j, K] - xflux[i, j, K] + yflux[i, j, K] - yflux[i, jm1, K]
    jc, jcm = slice(2, jm - 1), slice(1, jm - 2)
    tc1 = curv[i, jc, K] * _b(dt[i, jc]) * (u[ip1, jc, K] + u[i, jc, K])
    tc2 = curv[i, jcm, K] * _b(dt[i, jcm]) * (u[ip1, jcm, K] + u[i, jcm, K])
    advy[i, jc, K] += _b(arv[i, jc]) * 0.25 * (tc1 + tc2)
    return curv, advx, advy


# ---------------------------------------------------------------------------
# baroclinic pressure gradient (BAROPG)
# ---------------------------------------------------------------------------

def baropg(S, P):
    """Sigma-coordinate baroclinic pressure gradient.

    Restates ``explicit/momentum.py:543-700``.  Returns (rho_out, drhox,
    drhoy) where rho_out = (rho - rmean) + rmean carries the reference's
    round trip.
    """
    rho = S["rho"] - S["rmean"]
    dt, dx, dy, zz = S["dt"], S["dx"], S["dy"], S["zz"]
    im, jm, kb = rho.shape
    kbm1 = kb - 1
    g = P.grav
    drhox = np.zeros_like(rho)
    drhoy = np.zeros_like(rho)
    i, im1, j, jm1 = slice(1, im - 1), slice(0, im - 2), slice(1, jm - 1), slice(0, jm - 2)
    ks, km = slice(1, kbm1), slice(0, kbm1 - 1)
    zzk = zz[ks][None, None, :]
    zzkm = zz[km][None, None, :]
    kf = slice(0, kbm1)

    for (a_i, a_j, b_i, b_j, area_d, mask, out) in (
        (i, j, im1, j, dy, S["dum"], drhox),
        (i, j, i, jm1, dx, S["dvm"], drhoy),
    ):
        term_dt = dt[a_i, a_j] + dt[b_i, b_j]
        drho = rho[a_i, a_j, 0] - rho[b_i, b_j, 0]
        out[a_i, a_j, 0] = 0.5 * g * (-zz[0]) * term_dt * drho
        r_k, r_bk = rho[a_i, a_j, ks], rho[b_i, b_j, ks]
        r_km, r_bkm = rho[a_i, a_j, km], rho[b_i, b_j, km]
        term1 = g * 0.25 * (zzkm - zzk) * _b(term_dt) * ((r_k - r_bk) + (r_km - r_bkm))
        dt_diff = dt[a_i, a_j] - dt[b_i, b_j]
        term2 = g * 0.25 * (zzkm + zzk) * _b(dt_diff) * ((r_k + r_bk) - (r_km + r_bkm))
        out[a_i, a_j, ks] = _b(out[a_i, a_j, 0]) + _cumsum_k(term1 + term2)
        scale = 0.25 * term_dt * mask[a_i, a_j] * (area_d[a_i, a_j] + area_d[b_i, b_j])
        out[a_i, a_j, kf] *= _b(scale)
    drhox *= P.ramp
    drhoy *= P.ramp
    return rho + S["rmean"], drhox, drhoy


# ---------------------------------------------------------------------------
# Smagorinsky viscosity
# ---------------------------------------------------------------------------

def _smag_terms(S, P):
    u, v, dx, dy = S["u"], S["v"], S["dx"], S["dy"]
    im, jm, kb = u.shape
    K = slice(0, kb - 1)
    i, ip, imn = slice(1, im - 1), slice(2, im), slice(0, im - 2)
    j, jp, jmn = slice(1, jm - 1), slice(2, jm), slice(0, jm - 2)
    dxs, dys = _b(dx[i, j]), _b(dy[i, j])
    du_dx = (u[ip, j, K] - u[i, j, K]) / dxs
    dv_dy = (v[i, jp, K] - v[i, j, K]) / dys
    u_term = 0.25 * (u[i, jp, K] + u[ip, jp, K] - u[i, jmn, K] - u[ip, jmn, K]) / dys
    v_term = 0.25 * (v[ip, j, K] + v[ip, jp, K] - v[imn, j, K] - v[imn, jp, K]) / dxs
    return du_dx, dv_dy, u_term, v_term, dxs, dys, (i, j, K)


def smagorinsky_explicit(S, P):
    """aam = horcon*dx*dy*||(du/dx, dv/dy, (u_y+v_x)/sqrt2)||.

    Restates ``explicit/time_loop.py:10-16,193-233`` (vector_norm of the
    stacked components).  The norm is evaluated as sqrt(a^2+b^2+c^2) with the
    squares summed in order.
    """
    du_dx, dv_dy, u_term, v_term, dxs, dys, sl = _smag_terms(S, P)
    c = (u_term + v_term) * np.float32(math.sqrt(0.5)).astype(du_dx.dtype)
    mag = np.sqrt(du_dx * du_dx + dv_dy * dv_dy + c * c)
    aam = S["aam"].copy()
    aam[sl] = P.horcon * dxs * dys * mag
    return aam


def smagorinsky_implicit(S, P):
    """aam = horcon*dx*dy*sqrt(ux^2 + vy^2 + 0.5*(uy+vx)^2).

    Restates ``implicit_p0_fixed/time_loop.py:153-199`` with
    ``autograd.py:5-29`` (exact sqrt forward); aam_min clamp when positive.
    """
    du_dx, dv_dy, u_term, v_term, dxs, dys, sl = _smag_terms(S, P)
    term1 = (du_dx) ** 2
    term2 = (dv_dy) ** 2
    term3 = 0.5 * (u_term + v_term) ** 2
    smag = P.horcon * dxs * dys * np.sqrt(term1 + term2 + term3)
    aam_min = float(getattr(P, "aam_min", 0.0) or 0.0)
    if aam_min > 0.0:
        smag = np.maximum(smag, aam_min)
    aam = S["aam"].copy()
    aam[sl] = smag
    return aam


# ---------------------------------------------------------------------------
# 2-D advection (ADVAVE, mode 3)
# ---------------------------------------------------------------------------

def advave(S, P, fluxua, fluxva, tps):
    """2-D advection/diffusion of the depth-mean velocity (mode 3).

    Restates ``explicit/baroclinic.py:262-494``.  ``fluxua``, ``fluxva`` and
    ``tps`` are updated in place exactly where the reference writes them
    (the stale rows/columns it leaves untouched keep their values).  Returns
    (advua, advva).
    """
    d, ua, va, uab, vab = S["d"], S["ua"], S["va"], S["uab"], S["vab"]
    dx, dy, aam2d = S["dx"], S["dy"], S["aam2d"]
    im, jm = d.shape
    advua = np.zeros_like(d)
    si, sj = slice(1, im), slice(1, jm)
    sim, sjm = slice(0, im - 1), slice(0, jm - 1)
    iu, iup, ium = slice(1, im - 1), slice(2, im), slice(0, im - 2)

    t1 = (d[iup, sj] + d[iu, sj]) * ua[iup, sj]
    t2 = (d[iu, sj] + d[ium, sj]) * ua[iu, sj]
    fluxua[iu, sj] = 0.125 * (t1 + t2) * (ua[iup, sj] + ua[iu, sj])
    t1 = (d[si, sj] + d[si, sjm]) * va[si, sj]
    t2 = (d[sim, sj] + d[sim, sjm]) * va[sim, sj]
    fluxva[si, sj] = 0.125 * (t1 + t2) * (ua[si, sj] + ua[si, sjm])
    diff_u = (uab[iup, sj] - uab[iu, sj]) / dx[iu, sj]
    fluxua[iu, sj] -= d[iu, sj] * 2.0 * aam2d[iu, sj] * diff_u
    d_sum = d[si, sj] + d[sim, sj] + d[si, sjm] + d[sim, sjm]
    aam_sum = aam2d[si, sj] + aam2d[si, sjm] + aam2d[sim, sj] + aam2d[sim, sjm]
    dy_sum = dy[si, sj] + dy[sim, sj] + dy[si, sjm] + dy[sim, sjm]
    dx_sum = dx[si, sj] + dx[sim, sj] + dx[si, sjm] + dx[sim, sjm]
    du_dy = (uab[si, sj] - uab[si, sjm]) / dy_sum
    dv_dx = (vab[si, sj] - vab[sim, sj]) / dx_sum
    tps[si, sj] = 0.25 * d_sum * aam_sum * (du_dy + dv_dx)
    fluxua[si, sj] *= dy[si, sj]
    fluxva[si, sj] = (fluxva[si, sj] - tps[si, sj]) * 0.25 * dx_sum
    ia, iam, ja, jap = slice(1, im - 1), slice(0, im - 2), slice(1, jm - 1), slice(2, jm)
    advua[ia, ja] = fluxua[ia, ja] - fluxua[iam, ja] + fluxva[ia, jap] - fluxva[ia, ja]

    advva = np.zeros_like(d)
    t1 = (d[si, sj] + d[sim, sj]) * ua[si, sj]
    t2 = (d[si, sjm] + d[sim, sjm]) * ua[si, sjm]
    fluxua[si, sj] = 0.125 * (t1 + t2) * (va[sim, sj] + va[si, sj])
    jv, jvp, jvm = slice(1, jm - 1), slice(2, jm), slice(0, jm - 2)
    t1 = (d[si, jvp] + d[si, jv]) * va[si, jvp]
    t2 = (d[si, jv] + d[si, jvm]) * va[si, jv]
    fluxva[si, jv] = 0.125 * (t1 + t2) * (va[si, jvp] + va[si, jv])
    diff_v = (vab[si, jvp] - vab[si, jv]) / dy[si, jv]
    fluxva[si, jv] -= d[si, jv] * 2.0 * aam2d[si, jv] * diff_v
    fluxva[si, sj] *= dx[si, sj]
    dy_sum = dy[si, sj] + dy[sim, sj] + dy[si, sjm] + dy[sim, sjm]
    fluxua[si, sj] = (fluxua[si, sj] - tps[si, sj]) * 0.25 * dy_sum
    ip1, jm1 = slice(2, im), slice(0, jm - 2)
    advva[ia, ja] = fluxua[ip1, ja] - fluxua[ia, ja] + fluxva[ia, ja] - fluxva[ia, jm1]
    return advua, advva


def vertical_means(S, P):
    """Depth integrals sum_k f*dz over the active levels.

    Restates ``explicit/time_loop.py:240-258``; returns
    (adx2d, ady2d, drx2d, dry2d, aam2d)."""
    kbm1 = P.kb - 1
    dz = S["dz"][:kbm1][None, None, :]
    return tuple(_sum_k(S[n][:, :, :kbm1] * dz) for n in ("advx", "advy", "drhox", "drhoy", "aam"))


# ---------------------------------------------------------------------------
# boundary conditions
# ---------------------------------------------------------------------------

def _copy_edges_2d(a):
    im, jm = a.shape[:2]
    a[im - 1, :] = a[im - 2, :]
    a[0, :] = a[1, :]
    a[:, jm - 1] = a[:, jm - 2]
    a[:, 0] = a[:, 1]


def bcond_explicit(S, P, idx, F):
    """Explicit double-gyre lateral boundary conditions.

    Restates ``explicit/baroclinic.py:496-928``.  ``F`` maps the names
    elf/uaf/vaf/uf/vf/w to the arrays being conditioned; it is updated with
    the returned (possibly new) arrays.
    """
    im, jm, kb = P.im, P.jm, P.kb
    kbm1 = kb - 1
    fsm = S["fsm"]
    if idx == 1:
        elf = F["elf"]
        _copy_edges_2d(elf)
        F["elf"] = elf * fsm
        return
    if idx == 2:
        uaf, vaf = F["uaf"], F["vaf"]
        h, el, g, ramp = S["h"], S["el"], P.grav, P.ramp
        J = slice(1, jm - 1)
        I = slice(1, im - 1)

        def rad(h_edge):
            return np.sqrt(np.maximum(g / np.maximum(h_edge, 1e-8), 1e-8))

        te = P.rfe * rad(h[im - 2, J]) * (el[im - 2, J] - S["ele"][J])
        uaf[im - 1, J] = (S["uabe"][J] + te) * ramp
        vaf[im - 1, J] = 0.0
        tw = P.rfw * rad(h[1, J]) * (el[1, J] - S["elw"][J])
        uaf[1, J] = (S["uabw"][J] - tw) * ramp
        uaf[0, J] = uaf[1, J]
        vaf[0, J] = 0.0
        tn = P.rfn * rad(h[I, jm - 2]) * (el[I, jm - 2] - S["eln"][I])
        vaf[I, jm - 1] = (S["vabn"][I] + tn) * ramp
        uaf[I, jm - 1] = 0.0
        ts = P.rfs * rad(h[I, 1]) * (el[I, 1] - S["els"][I])
        vaf[I, 1] = (S["vabs"][I] - ts) * ramp
        vaf[I, 0] = vaf[I, 1]
        uaf[I, 0] = 0.0
        F["uaf"] = uaf * S["dum"]
        F["vaf"] = vaf * S["dvm"]
        return
    if idx == 3:
        uf, vf = F["uf"], F["vf"]
        u, v, h, hmax = S["u"], S["v"], S["h"], P.hmax
        K = slice(0, kbm1)
        J, Jm, Jp = slice(1, jm - 1), slice(0, jm - 2), slice(2, jm)
        I, Im, Ip = slice(1, im - 1), slice(0, im - 2), slice(2, im)

        def ga_of(hh):
            return np.sqrt(np.maximum(hh / hmax, 1e-8))[:, None]

        def smooth_j(a, i):
            return 0.25 * a[i, Jm, K] + 0.50 * a[i, J, K] + 0.25 * a[i, Jp, K]

        def smooth_i(a, j):
            return 0.25 * a[Im, j, K] + 0.50 * a[I, j, K] + 0.25 * a[Ip, j, K]

        ga = ga_of(h[im - 1, J])
        uf[im - 1, J, K] = ga * smooth_j(u, im - 2) + (1.0 - ga) * smooth_j(u, im - 1)
        vf[im - 1, J, K] = 0.0
        ga = ga_of(h[0, J])
        uf[1, J, K] = ga * smooth_j(u, 2) + (1.0 - ga) * smooth_j(u, 1)
        uf[0, J, K] = uf[1, J, K]
        vf[0, J, K] = 0.0
        ga = ga_of(h[I, jm - 1])
        vf[I, jm - 1, K] = ga * smooth_i(v, jm - 2) + (1.0 - ga) * smooth_i(v, jm - 1)
        uf[I, jm - 1, K] = 0.0
        ga = ga_of(h[I, 0])
        vf[I, 1, K] = ga * smooth_i(v, 2) + (1.0 - ga) * smooth_i(v, 1)
        vf[I, 0, K] = vf[I, 1, K]
        uf[I, 0, K] = 0.0
        F["uf"] = uf * _b(S["dum"])
        F["vf"] = vf * _b(S["dvm"])
        return
    if idx == 4:
        uf, vf = F["uf"], F["vf"]
        t, s, u, v, w, zz, dt = S["t"], S["s"], S["u"], S["v"], S["w"], S["zz"], S["dt"]
        dx, dy, dti = S["dx"], S["dy"], P.dti
        K = slice(0, kbm1)
        km_, kmn, kp = slice(1, kbm1 - 1), slice(0, kbm1 - 2), slice(2, kbm1)
        dzz_ = (zz[kmn] - zz[kp])[None, :]
        # east
        u1 = 2.0 * u[im - 1, :, K] * dti / (dx[im - 1, :] + dx[im - 2, :])[:, None]
        inflow = u1 <= 0.0
        tc, sc, ti, si_ = t[im - 1, :, K], s[im - 1, :, K], t[im - 2, :, K], s[im - 2, :, K]
        te, se = S["tbe"][:, K], S["sbe"][:, K]
        uf[im - 1, :, K] = np.where(inflow, tc - u1 * (te - tc), tc - u1 * (tc - ti))
        vf[im - 1, :, K] = np.where(inflow, sc - u1 * (se - sc), sc - u1 * (sc - si_))
        if kbm1 > 2:
            wm = 0.5 * (w[im - 2, :, km_] + w[im - 2, :, kp]) * dti / (dzz_ * dt[im - 2, :][:, None])
            out = u1[:, km_] > 0.0
            uf[im - 1, :, km_] = np.where(out, uf[im - 1, :, km_] - wm * (t[im - 2, :, kmn] - t[im - 2, :, kp]), uf[im - 1, :, km_])
            vf[im - 1, :, km_] = np.where(out, vf[im - 1, :, km_] - wm * (s[im - 2, :, kmn] - s[im - 2, :, kp]), vf[im - 1, :, km_])
        # west
        u1 = 2.0 * u[1, :, K] * dti / (dx[0, :] + dx[1, :])[:, None]
        inflow = u1 >= 0.0
        tc, sc, ti, si_ = t[0, :, K], s[0, :, K], t[1, :, K], s[1, :, K]
        te, se = S["tbw"][:, K], S["sbw"][:, K]
        uf[0, :, K] = np.where(inflow, tc - u1 * (tc - te), tc - u1 * (ti - tc))
        vf[0, :, K] = np.where(inflow, sc - u1 * (sc - se), sc - u1 * (si_ - sc))
        if kbm1 > 2:
            wm = 0.5 * (w[1, :, km_] + w[1, :, kp]) * dti / (dzz_ * dt[1, :][:, None])
            out = u1[:, km_] < 0.0
            uf[0, :, km_] = np.where(out, uf[0, :, km_] - wm * (t[1, :, kmn] - t[1, :, kp]), uf[0, :, km_])
            vf[0, :, km_] = np.where(out, vf[0, :, km_] - wm * (s[1, :, kmn] - s[1, :, kp]), vf[0, :, km_])
        # north
        u1 = 2.0 * v[:, jm - 1, K] * dti / (dy[:, jm - 1] + dy[:, jm - 2])[:, None]
        inflow = u1 <= 0.0
        tc, sc, ti, si_ = t[:, jm - 1, K], s[:, jm - 1, K], t[:, jm - 2, K], s[:, jm - 2, K]
        te, se = S["tbn"][:, K], S["sbn"][:, K]
        uf[:, jm - 1, K] = np.where(inflow, tc - u1 * (te - tc), tc - u1 * (tc - ti))
        vf[:, jm - 1, K] = np.where(inflow, sc - u1 * (se - sc), sc - u1 * (sc - si_))
        if kbm1 > 2:
            wm = 0.5 * (w[:, jm - 2, km_] + w[:, jm - 2, kp]) * dti / (dzz_ * dt[:, jm - 2][:, None])
            out = u1[:, km_] > 0.0
            uf[:, jm - 1, km_] = np.where(out, uf[:, jm - 1, km_] - wm * (t[:, jm - 2, kmn] - t[:, jm - 2, kp]), uf[:, jm - 1, km_])
            vf[:, jm - 1, km_] = np.where(out, vf[:, jm - 1, km_] - wm * (s[:, jm - 2, kmn] - s[:, jm - 2, kp]), vf[:, jm - 1, km_])
        # south
        u1 = 2.0 * v[:, 1, K] * dti / (dy[:, 0] + dy[:, 1])[:, None]
        inflow = u1 >= 0.0
        tc, sc, ti, si_ = t[:, 0, K], s[:, 0, K], t[:, 1, K], s[:, 1, K]
        te, se = S["tbs"][:, K], S["sbs"][:, K]
        uf[:, 0, K] = np.where(inflow, tc - u1 * (tc - te), tc - u1 * (ti - tc))
        vf[:, 0, K] = np.where(inflow, sc - u1 * (sc - se), sc - u1 * (si_ - sc))
        if kbm1 > 2:
            wm = 0.5 * (w[:, 1, km_] + w[:, 1, kp]) * dti / (dzz_ * dt[:, 1][:, None])
            out = u1[:, km_] < 0.0
            uf[:, 0, km_] = np.where(out, uf[:, 0, km_] - wm * (t[:, 1, kmn] - t[:, 1, kp]), uf[:, 0, km_])
            vf[:, 0, km_] = np.where(out, vf[:, 0, km_] - wm * (s[:, 1, kmn] - s[:, 1, kp]), vf[:, 0, km_])
        F["uf"] = uf * _b(fsm)
        F["vf"] = vf * _b(fsm)
        return
    if idx == 5:
        w = F["w"]
        w[:, :, :kbm1] = w[:, :, :kbm1] * _b(fsm)
        return
    if idx == 6:
        uf, vf = F["uf"], F["vf"]
        q2, q2l, u, v = S["q2"], S["q2l"], S["u"], S["v"]
        dx, dy, dti, small = S["dx"], S["dy"], P.dti, P.small
        # east
        u1 = 2.0 * u[im - 1, :] * dti / (dx[im - 1, :] + dx[im - 2, :])[:, None]
        inflow = u1 <= 0.0
        uf[im - 1, :] = np.where(inflow, q2[im - 1, :] - u1 * (small - q2[im - 1, :]),
                                 q2[im - 1, :] - u1 * (q2[im - 1, :] - q2[im - 2, :]))
        vf[im - 1, :] = np.where(inflow, q2l[im - 1, :] - u1 * (small - q2l[im - 1, :]),
                                 q2l[im - 1, :] - u1 * (q2l[im - 1, :] - q2l[im - 2, :]))
        # west
        u1 = 2.0 * u[1, :] * dti / (dx[0, :] + dx[1, :])[:, None]
        inflow = u1 >= 0.0
        uf[0, :] = np.where(inflow, q2[0, :] - u1 * (q2[0, :] - small), q2[0, :] - u1 * (q2[1, :] - q2[0, :]))
        vf[0, :] = np.where(inflow, q2l[0, :] - u1 * (q2l[0, :] - small), q2l[0, :] - u1 * (q2l[1, :] - q2l[0, :]))
        # north
        u1 = 2.0 * v[:, jm - 1] * dti / (dy[:, jm - 1] + dy[:, jm - 2])[:, None]
        inflow = u1 <= 0.0
        uf[:, jm - 1] = np.where(inflow, q2[:, jm - 1] - u1 * (small - q2[:, jm - 1]),
                                 q2[:, jm - 1] - u1 * (q2[:, jm - 1] - q2[:, jm - 2]))
        vf[:, jm - 1] = np.where(inflow, q2l[:, jm - 1] - u1 * (small - q2l[:, jm - 1]),
                                 q2l[:, jm - 1] - u1 * (q2l[:, jm - 1] - q2l[:, jm - 2]))
        # south
        u1 = 2.0 * v[:, 1] * dti / (dy[:, 0] + dy[:, 1])[:, None]
        inflow = u1 >= 0.0
        uf[:, 0] = np.where(inflow, q2[:, 0] - u1 * (q2[:, 0] - small), q2[:, 0] - u1 * (q2[:, 1] - q2[:, 0]))
        vf[:, 0] = np.where(inflow, q2l[:, 0] - u1 * (q2l[:, 0] - small), q2l[:, 0] - u1 * (q2l[:, 1] - q2l[:, 0]))
        F["uf"] = uf * _b(fsm) + 1.0e-10
        F["vf"] = vf * _b(fsm) + 1.0e-10
        return
    raise ValueError(f"Invalid bcond index: {idx}")


def _zero_ring(a):
    a[0] = 0.0
    a[-1] = 0.0
    a[:, 0] = 0.0
    a[:, -1] = 0.0


# ---------------------------------------------------------------------------
# periodic-x halo (no counterpart in the reference, whose only lateral
# boundaries are walls and open edges)
# ---------------------------------------------------------------------------

# per-edge open-boundary arrays and the 1-D vertical grid: not planes of the grid
_NOT_PLANES = frozenset(("z", "zz", "dz", "dzz", "ele", "elw", "eln", "els", "uabe", "uabw", "vabn", "vabs",
                         "tbe", "sbe", "tbw", "sbw", "tbn", "sbn", "tbs", "sbs"))


def wrap_x(a):
    """Halo columns of a periodic-x plane (2-D or 3-D, i first), two on
    each side: columns 0, 1 are copies of im-4, im-3 and columns im-2,
    im-1 of 2, 3, so the unique columns are 2..im-3 (period im-4).  Two
    columns because the reference's operators compute some intermediates
    (advct's x-fluxes, the curvature term of advx) only from column 1 or
    2 on: with two halo columns every unique column is computed exactly as
    an interior column of a wider basin.  A u-point column i is the west
    face of cell i, so the same copy serves every staggering."""
    im = a.shape[0]
    a[0] = a[im - 4]
    a[1] = a[im - 3]
    a[im - 2] = a[2]
    a[im - 1] = a[3]


def periodic_fill(S, P, *extra):
    """The periodic-x halo fill after a phase of the step: every plane of
    the state (and the phase's extra planes) gets wrap_x.  Nothing when
    the core is not periodic in x."""
    if not getattr(P, "periodic_x", False):
        return
    im, jm = P.im, P.jm
    for name, a in S.items():
        if name in _NOT_PLANES or not isinstance(a, np.ndarray) or a.ndim not in (2, 3):
            continue
        if a.shape[:2] == (im, jm):
            wrap_x(a)
    for a in extra:
        wrap_x(a)


def _pcg_ring(a, periodic):
    """The ring of a PCG vector: zero (the Dirichlet ring), or with
    periodic x zero on the j walls and the halo columns wrapped."""
    if not periodic:
        _zero_ring(a)
        return
    a[:, 0] = 0.0
    a[:, -1] = 0.0
    wrap_x(a)


def bcond_implicit(S, P, idx, F):
    """Closed-basin boundary policy of the implicit core.

    Restates ``implicit_p0_fixed/boundary/closed_basin.py:27-87``.
    """
    fsm = S["fsm"]
    if idx == 1:
        elf = F["elf"] * fsm
        _zero_ring(elf)
        F["elf"] = elf
        return
    if idx == 2:
        uaf = F["uaf"] * S["dum"]
        vaf = F["vaf"] * S["dvm"]
        _zero_ring(uaf)
        _zero_ring(vaf)
        F["uaf"], F["vaf"] = uaf, vaf
        return
    if idx == 3:
        uf = F["uf"] * _b(S["dum"])
        vf = F["vf"] * _b(S["dvm"])
        _zero_ring(uf)
        _zero_ring(vf)
        F["uf"], F["vf"] = uf, vf
        return
    if idx == 4:
        _copy_edges_2d_rows_then_cols(F["uf"])
        _copy_edges_2d_rows_then_cols(F["vf"])
        return
    if idx == 5:
        F["w"] = F["w"] * _b(fsm)
        return
    if idx == 6:
        F["uf"] = F["uf"] * _b(fsm)
        F["vf"] = F["vf"] * _b(fsm)
        return
    raise ValueError(f"Invalid bcond index: {idx}")


def _copy_edges_2d_rows_then_cols(a):
    """closed_basin.py:290-297 order: west, east, south, north."""
    im, jm = a.shape[:2]
    a[0] = a[1]
    a[im - 1] = a[im - 2]
    a[:, 0] = a[:, 1]
    a[:, jm - 1] = a[:, jm - 2]


# ---------------------------------------------------------------------------
# vertical velocity (VERTVL)
# ---------------------------------------------------------------------------

def vertvl(S, P):
    """w from continuity.  Restates ``explicit/baroclinic.py:930-1040``.
    Returns the updated w (a copy)."""
    u, v, dt, dx, dy, dz = S["u"], S["v"], S["dt"], S["dx"], S["dy"], S["dz"]
    im, jm, kb = u.shape
    kbm1 = kb - 1
    K = slice(0, kbm1)
    xflux = np.zeros_like(u)
    yflux = np.zeros_like(u)
    si, sim, sj, sjm = slice(1, im), slice(0, im - 1), slice(1, jm), slice(0, jm - 1)
    xflux[si, sj, K] = 0.25 * _b(dy[si, sj] + dy[sim, sj]) * _b(dt[si, sj] + dt[sim, sj]) * u[si, sj, K]
    yflux[si, sj, K] = 0.25 * _b(dx[si, sj] + dx[si, sjm]) * _b(dt[si, sj] + dt[si, sjm]) * v[si, sj, K]
    w = S["w"].copy()
    I, J = slice(1, im - 1), slice(1, jm - 1)
    Ip, Jp = slice(2, im), slice(2, jm)
    w[I, J, 0] = 0.5 * (S["vfluxb"][I, J] + S["vfluxf"][I, J])
    div = xflux[Ip, J, K] - xflux[I, J, K] + yflux[I, Jp, K] - yflux[I, J, K]
    inc = div / _b(dx[I, J] * dy[I, J]) + _b((S["etf"][I, J] - S["etb"][I, J]) / P.dti2)
    inc = inc * dz[K][None, None, :]
    w[I, J, 1:kbm1 + 1] = w[I, J, 0][:, :, None] + _cumsum_k(inc)
    return w


# ---------------------------------------------------------------------------
# turbulence advection (ADVQ)
# ---------------------------------------------------------------------------

def advq(S, P, qb, q, qf):
    """Advection/diffusion of q2 or q2l on w-levels, leapfrog to qf.

    Restates ``explicit/tracers.py:14-156``.  ``qf`` is written in place on
    the interior and returned.
    """
    u, v, w, aam, h = S["u"], S["v"], S["w"], S["aam"], S["h"]
    dt, dx, dy, dz, art = S["dt"], S["dx"], S["dy"], S["dz"], S["art"]
    dum, dvm, etb, etf = S["dum"], S["dvm"], S["etb"], S["etf"]
    im, jm, kb = q.shape
    kbm1 = kb - 1
    ks, km = slice(1, kbm1), slice(0, kbm1 - 1)
    si, sim, sj, sjm = slice(1, im), slice(0, im - 1), slice(1, jm), slice(0, jm - 1)
    xflux = np.zeros_like(q)
    yflux = np.zeros_like(q)
    xflux[si, sj, ks] = 0.125 * (q[si, sj, ks] + q[sim, sj, ks]) * _b(dt[si, sj] + dt[sim, sj]) * (u[si, sj, ks] + u[si, sj, km])
    yflux[si, sj, ks] = 0.125 * (q[si, sj, ks] + q[si, sjm, ks]) * _b(dt[si, sj] + dt[si, sjm]) * (v[si, sj, ks] + v[si, sj, km])
    aam_sum = aam[si, sj, ks] + aam[sim, sj, ks] + aam[si, sj, km] + aam[sim, sj, km]
    xflux[si, sj, ks] -= 0.25 * aam_sum * _b(h[si, sj] + h[sim, sj]) * (qb[si, sj, ks] - qb[sim, sj, ks]) * _b(dum[si, sj]) / _b(dx[si, sj] + dx[sim, sj])
    aam_sum = aam[si, sj, ks] + aam[si, sjm, ks] + aam[si, sj, km] + aam[si, sjm, km]
    yflux[si, sj, ks] -= 0.25 * aam_sum * _b(h[si, sj] + h[si, sjm]) * (qb[si, sj, ks] - qb[si, sjm, ks]) * _b(dvm[si, sj]) / _b(dy[si, sj] + dy[si, sjm])
    xflux[si, sj, ks] *= 0.5 * _b(dy[si, sj] + dy[sim, sj])
    yflux[si, sj, ks] *= 0.5 * _b(dx[si, sj] + dx[si, sjm])

    I, Ip, J, Jp = slice(1, im - 1), slice(2, im), slice(1, jm - 1), slice(2, jm)
    kp = slice(2, kbm1 + 1)
    dz_sum = (dz[ks] + dz[km])[None, None, :]
    vert = (w[I, J, km] * q[I, J, km] - w[I, J, kp] * q[I, J, kp]) * _b(art[I, J]) / dz_sum
    horiz = xflux[Ip, J, ks] - xflux[I, J, ks] + yflux[I, Jp, ks] - yflux[I, J, ks]
    qf[I, J, ks] = vert + horiz
    tb = _b((h[I, J] + etb[I, J]) * art[I, J])
    tf = _b((h[I, J] + etf[I, J]) * art[I, J])
    qf[I, J, ks] = (tb * qb[I, J, ks] - P.dti2 * qf[I, J, ks]) / (tf + 1e-20)
    return qf


# ---------------------------------------------------------------------------
# Mellor-Yamada 2.5 (PROFQ)
# ---------------------------------------------------------------------------

def profq(S, P, uf, vf, implicit_variant):
    """Mellor-Yamada 2.5 turbulence closure with two tridiagonal solves.

    Restates ``explicit/tracers.py:158-431``; ``implicit_variant`` selects the
    epsilon forms of ``implicit_p0_fixed/tracers.py:156-430`` (wall function
    ``1/(|dz|+1e-8)``).  ``uf``/``vf`` hold the advected q2/q2l forecasts.
    Returns dict with l, kq, km, kh, uf, vf, cc.
    """
    t, s, rho, u, v = S["t"], S["s"], S["rho"], S["u"], S["v"]
    q2, q2b, q2lb = S["q2"], S["q2b"], S["q2lb"]
    km_in, kh_in, kq_in = S["km"], S["kh"], S["kq"]
    h, etf, dt, fsm = S["h"], S["etf"], S["dt"], S["fsm"]
    dz, dzz, zz, z = S["dz"], S["dzz"], S["zz"], S["z"]
    im, jm, kb = q2.shape
    kbm1 = kb - 1
    dti2, umol, grav, kappa, small = P.dti2, P.umol, P.grav, P.kappa, P.small
    dt_ = q2.dtype
    a1, b1, a2, b2, c1 = 0.92, 16.6, 0.74, 10.1, 0.08
    e1, e2, sef = 1.8, 1.33, 1.0
    cbcnst, surfl, shiw = 100.0, 2.0e5, 0.0

    dh = h + etf
    A = np.zeros_like(q2)
    C = np.zeros_like(q2)
    for k in range(1, kbm1):
        den_a = dzz[k - 1] * dz[k] * dh * dh
        den_c = dzz[k - 1] * dz[k - 1] * dh * dh
        A[:, :, k] = -dti2 * (kq_in[:, :, k + 1] + kq_in[:, :, k] + 2.0 * umol) * 0.5 / den_a
        C[:, :, k] = -dti2 * (kq_in[:, :, k - 1] + kq_in[:, :, k] + 2.0 * umol) * 0.5 / den_c

    const1 = (16.6 ** (2.0 / 3.0)) * sef
    si, sip, sj, sjp = slice(0, im - 1), slice(1, im), slice(0, jm - 1), slice(1, jm)
    us = 0.5 * (S["wusurf"][si, sj] + S["wusurf"][sip, sj])
    vs = 0.5 * (S["wvsurf"][si, sj] + S["wvsurf"][si, sjp])
    utau2 = np.sqrt(us ** 2 + vs ** 2 + 1e-8)
    l0 = np.zeros_like(h)
    l0[si, sj] = surfl * utau2 / grav
    ub_ = 0.5 * (S["wubot"][si, sj] + S["wubot"][sip, sj])
    vb_ = 0.5 * (S["wvbot"][si, sj] + S["wvbot"][si, sjp])
    uf_bottom = np.zeros_like(h)
    uf_bottom[si, sj] = np.sqrt(ub_ ** 2 + vb_ ** 2 + 1e-8) * const1

    tp = t[:, :, :kbm1] + P.tbias
    sp = s[:, :, :kbm1] + P.sbias
    p = grav * P.rhoref * (-zz[:kbm1][None, None, :] * _b(dh)) * 1.0e-4
    cc = 1449.1 + 0.00821 * p + 4.55 * tp - 0.045 * (tp ** 2) + 1.34 * (sp - 35.0)
    cc = np.where(np.abs(cc) < 1e-6, np.asarray(1e-6, dtype=dt_), cc)
    rad = (1.0 - 0.01642 * p / cc) * (1.0 - 0.40 * p / (cc ** 2))
    cc = cc / np.sqrt(np.maximum(rad, 1e-8))

    boygr = np.zeros_like(q2)
    for k in range(1, kbm1):
        term1 = grav * (rho[:, :, k - 1] - rho[:, :, k]) / (dzz[k - 1] * dh)
        term2 = (grav ** 2) * 2.0 / (cc[:, :, k - 1] ** 2 + cc[:, :, k] ** 2)
        boygr[:, :, k] = term1 + term2

    q2b_abs = np.abs(q2b)
    q2lb_abs = np.abs(q2lb)
    l = np.zeros_like(q2)
    l[:, :, 1:kbm1] = q2lb_abs[:, :, 1:kbm1] / (q2b_abs[:, :, 1:kbm1] + 1e-20)
    surf = (z[:kbm1] > -0.5)[None, None, :]
    lsl = l[:, :, :kbm1].copy()
    l[:, :, :kbm1] = np.where(surf, np.maximum(lsl, kappa * _b(l0)), lsl)
    gh = np.zeros_like(q2)
    gh[:, :, 1:kbm1] = (l[:, :, 1:kbm1] ** 2) * boygr[:, :, 1:kbm1] / (q2b_abs[:, :, 1:kbm1] + 1e-20)
    gh = np.minimum(gh, 0.028)
    l[:, :, 0] = kappa * l0
    l[:, :, kb - 1] = 0.0
    gh[:, :, 0] = 0.0
    gh[:, :, kb - 1] = 0.0

    kn = np.zeros_like(q2)
    I, Ip, J, Jp = slice(1, im - 1), slice(2, im), slice(1, jm - 1), slice(2, jm)
    for k in range(1, kbm1):
        du = (u[I, J, k] - u[I, J, k - 1] + u[Ip, J, k] - u[Ip, J, k - 1]) ** 2
        dv = (v[I, J, k] - v[I, J, k - 1] + v[I, Jp, k] - v[I, Jp, k - 1]) ** 2
        den = (dzz[k - 1] * dh[I, J]) ** 2
        kn[I, J, k] = km_in[I, J, k] * 0.25 * sef * (du + dv) / den
        kn[I, J, k] = kn[I, J, k] - shiw * km_in[I, J, k] * boygr[I, J, k] + kh_in[I, J, k] * boygr[I, J, k]

    dtef = np.sqrt(q2b_abs + 1e-8) * 1.0 / (b1 * l + small)
    # q2 sweep
    ee = np.zeros((im, jm), dtype=dt_)
    gg = np.zeros((im, jm), dtype=dt_)
    gg[si, sj] = (15.8 * cbcnst) ** (2.0 / 3.0) * utau2
    EE, GG = [ee], [gg]
    for k in range(1, kbm1):
        den = A[:, :, k] + C[:, :, k] * (1.0 - EE[k - 1]) - (2.0 * dti2 * dtef[:, :, k] + 1.0)
        EE.append(A[:, :, k] / (den + 1e-20))
        GG.append((-2.0 * dti2 * kn[:, :, k] + C[:, :, k] * GG[k - 1] - uf[:, :, k]) / (den + 1e-20))
    q2f = [None] * kb
    q2f[kb - 1] = uf_bottom
    for k in range(kbm1 - 1, -1, -1):
        q2f[k] = EE[k] * q2f[k + 1] + GG[k]
    uf_out = np.stack(q2f, axis=2)

    # q2l sweep
    EE = [np.zeros((im, jm), dtype=dt_)]
    GG = [np.zeros((im, jm), dtype=dt_)]
    z_surf, z_bot = z[0], z[kb - 1]
    for k in range(1, kbm1):
        if implicit_variant:
            wall = (1.0 / (np.abs(z[k] - z_surf) + 1e-8) + 1.0 / (np.abs(z[k] - z_bot) + 1e-8))
            wall = np.broadcast_to(wall, dh.shape)
        else:
            one = np.ones_like(dh)
            wall = one / (np.abs(z[k] - z_surf) + 1e-20) + one / (np.abs(z[k] - z_bot) + 1e-20)
        wall = wall * l[:, :, k] / (dh * kappa)
        dtef_k = dtef[:, :, k] * (1.0 + e2 * (wall ** 2))
        den = A[:, :, k] + C[:, :, k] * (1.0 - EE[k - 1]) - (dti2 * dtef_k + 1.0)
        EE.append(A[:, :, k] / (den + 1e-20))
        GG.append((dti2 * (-kn[:, :, k] * l[:, :, k] * e1) + C[:, :, k] * GG[k - 1] - vf[:, :, k]) / (den + 1e-20))
    q2lf = [None] * kb
    q2lf[kb - 1] = np.zeros((im, jm), dtype=dt_)
    for k in range(kbm1 - 1, -1, -1):
        q2lf[k] = EE[k] * q2lf[k + 1] + GG[k]
    vf_out = np.stack(q2lf, axis=2)

    ks = slice(1, kbm1)
    mask = (uf_out[:, :, ks] <= small) | (vf_out[:, :, ks] <= small)
    uf_fin = uf_out.copy()
    vf_fin = vf_out.copy()
    if implicit_variant:
        uf_fin[:, :, ks] = np.where(mask, uf_out[:, :, ks] * 0.0 + small, uf_out[:, :, ks])
    else:
        uf_fin[:, :, ks] = np.where(mask, np.asarray(small, dtype=dt_), uf_out[:, :, ks])
    vf_fin[:, :, ks] = np.where(mask, 0.1 * _b(dt) * small, vf_out[:, :, ks])

    coef4 = 18.0 * a1 * a1 + 9.0 * a1 * a2
    coef5 = 9.0 * a1 * a2
    coef1 = a2 * (1.0 - 6.0 * a1 / b1)
    coef2 = 3.0 * a2 * b2 + 18.0 * a1 * a2
    coef3 = a1 * (1.0 - 3.0 * c1 - 6.0 * a1 / b1)
    sh = coef1 / ((1.0 - coef2 * gh) + 1e-20)
    sm = (coef3 + sh * coef4 * gh) / ((1.0 - coef5 * gh) + 1e-20)
    knf = l * np.sqrt(np.abs(q2) + 1e-8)
    kq_out = (knf * 0.41 * sh + kq_in) * 0.5
    km_out = (knf * sm + km_in) * 0.5
    kh_out = (knf * sh + kh_in) * 0.5
    for arr in (km_out, kh_out):
        arr[im - 1] = arr[im - 2] * fsm[im - 1][:, None]
        arr[0] = arr[1] * fsm[0][:, None]
        arr[:, jm - 1] = arr[:, jm - 2] * fsm[:, jm - 1][:, None]
        arr[:, 0] = arr[:, 1] * fsm[:, 0][:, None]
    return dict(l=l, kq=kq_out, km=km_out, kh=kh_out, uf=uf_fin, vf=vf_fin, cc=cc,
                a=A, c=C)


def profq_pom08(S, P, uf, vf):
    """The POM08-WAD closure of the reference's case policies.

    Restates ``cores/case_adapters/fortran_compat.py:26-147`` (``profq``
    bound by ``install``, ``:147-161``, with the default reference pressure
    and ``zsh``): sound speed from the fixed pressure of -zz*max(h, 0),
    buoyancy over h + et, exact stress norms, |q2b| / |q2lb| on the interior
    levels (returned as the new q2b / q2lb, which the time loop keeps),
    reciprocal pivots, Dirichlet q2l values on the second and penultimate
    levels, |q2| / |q2l| forecasts, kn = (kappa*zsh + l)*sqrt|q2|,
    kq = (0.20*kn + kq)*0.5, and km/kh edges with the north/south copies
    first.  Returns the dict of ``profq`` plus q2b and q2lb."""
    t, s, rho, u, v = S["t"], S["s"], S["rho"], S["u"], S["v"]
    q2, q2b, q2lb = S["q2"], S["q2b"], S["q2lb"]
    km_in, kh_in, kq_in = S["km"], S["kh"], S["kq"]
    h, etf, et, fsm = S["h"], S["etf"], S["et"], S["fsm"]
    dz, dzz, zz, z = S["dz"], S["dzz"], S["zz"], S["z"]
    im, jm, kb = q2.shape
    kbm1 = kb - 1
    dti2, umol, grav, kappa, small = P.dti2, P.umol, P.grav, P.kappa, P.small
    zsh = float(getattr(P, "zsh", 0.01))
    zero = np.zeros_like(h)
    dh = h + etf
    aa = np.zeros_like(q2)
    ca = np.zeros_like(q2)
    for k in range(1, kbm1):
        aa[:, :, k] = -dti2 * (kq_in[:, :, k + 1] + kq_in[:, :, k] + 2 * umol) * .5 / (dzz[k - 1] * dz[k] * dh * dh)
        ca[:, :, k] = -dti2 * (kq_in[:, :, k - 1] + kq_in[:, :, k] + 2 * umol) * .5 / (dzz[k - 1] * dz[k - 1] * dh * dh)
    us = .5 * (S["wusurf"][:-1, :-1] + S["wusurf"][1:, :-1])
    vs = .5 * (S["wvsurf"][:-1, :-1] + S["wvsurf"][:-1, 1:])
    ub = .5 * (S["wubot"][:-1, :-1] + S["wubot"][1:, :-1])
    vb = .5 * (S["wvbot"][:-1, :-1] + S["wvbot"][:-1, 1:])
    utau2 = np.sqrt(us * us + vs * vs)
    btau2 = np.sqrt(ub * ub + vb * vb)
    l0 = zero.copy()
    l0[:-1, :-1] = 2.e5 * utau2 / grav
    surface_q = zero.copy()
    surface_q[:-1, :-1] = (15.8 * 100.) ** (2. / 3.) * utau2
    bottom = uf[:, :, -1].copy()
    bottom[:-1, :-1] = btau2 * (16.6 ** (2. / 3.))
    pdens = grav * P.rhoref * (-zz[None, None, :] * np.maximum(h[:, :, None], 0.)) * 1.e-5
    pdens = pdens.astype(q2.dtype)
    p = pdens[:, :, :kbm1] * 10.
    tp = t[:, :, :kbm1] + P.tbias
    sp = s[:, :, :kbm1] + P.sbias
    sound = 1449.1 + .00821 * p + 4.55 * tp - .045 * (tp * tp) + 1.34 * (sp - 35.)
    sound = sound / np.sqrt((1. - .01642 * p / sound) * (1. - .40 * p / (sound * sound)))
    qb = q2b.copy()
    qlb = q2lb.copy()
    qb[:, :, 1:kbm1] = np.abs(q2b[:, :, 1:kbm1])
    qlb[:, :, 1:kbm1] = np.abs(q2lb[:, :, 1:kbm1])
    boygr = np.zeros_like(q2)
    l_out = np.zeros_like(q2)
    gh = np.zeros_like(q2)
    l_out[:, :, 0] = kappa * l0
    depth = h + et
    for k in range(1, kbm1):
        b = grav * (rho[:, :, k - 1] - rho[:, :, k]) / (dzz[k - 1] * depth)
        b = b + grav ** 2 * 2. / (sound[:, :, k - 1] * sound[:, :, k - 1] + sound[:, :, k] * sound[:, :, k])
        ll = np.abs(qlb[:, :, k] / qb[:, :, k])
        if z[k] > -.5:
            ll = np.maximum(ll, kappa * l0)
        boygr[:, :, k] = b
        l_out[:, :, k] = ll
        gh[:, :, k] = np.minimum((ll * ll) * b / qb[:, :, k], .028)
    prod = np.zeros_like(q2)
    for k in range(1, kbm1):
        du = u[1:-1, 1:-1, k] - u[1:-1, 1:-1, k - 1] + u[2:, 1:-1, k] - u[2:, 1:-1, k - 1]
        dv = v[1:-1, 1:-1, k] - v[1:-1, 1:-1, k - 1] + v[1:-1, 2:, k] - v[1:-1, 2:, k - 1]
        den = dzz[k - 1] * dh[1:-1, 1:-1]
        pr = km_in[1:-1, 1:-1, k] * .25 * (du * du + dv * dv) / (den * den)
        prod[1:-1, 1:-1, k] = pr + kh_in[1:-1, 1:-1, k] * boygr[1:-1, 1:-1, k]
    diss = np.sqrt(np.abs(qb)) / (16.6 * l_out + small)
    e = [zero]
    g = [surface_q]
    for k in range(1, kbm1):
        inv = 1. / (aa[:, :, k] + ca[:, :, k] * (1. - e[k - 1]) - (2. * dti2 * diss[:, :, k] + 1.))
        e.append(aa[:, :, k] * inv)
        g.append((-2. * dti2 * prod[:, :, k] + ca[:, :, k] * g[k - 1] - uf[:, :, k]) * inv)
    usol = np.zeros_like(q2)
    usol[:, :, kb - 1] = bottom
    for k in range(kbm1 - 1, -1, -1):
        usol[:, :, k] = e[k] * usol[:, :, k + 1] + g[k]
    e2 = [zero, zero]
    g2 = [zero, (-kappa * z[1]) * dh * q2[:, :, 1]]
    for k in range(2, kbm1):
        wall = (1. / np.abs(z[k] - z[0]) + 1. / np.abs(z[k] - z[-1])) * l_out[:, :, k] / (dh * kappa)
        ds = diss[:, :, k] * (1. + 1.33 * (wall * wall))
        inv = 1. / (aa[:, :, k] + ca[:, :, k] * (1. - e2[k - 1]) - (dti2 * ds + 1.))
        e2.append(aa[:, :, k] * inv)
        rhs = (kappa * (1. + z[kbm1 - 1])) * dh * q2[:, :, kbm1 - 1] if k == kbm1 - 1 else vf[:, :, k]
        g2.append((dti2 * (-prod[:, :, k] * l_out[:, :, k] * 1.8) + ca[:, :, k] * g2[k - 1] - rhs) * inv)
    vsol = np.zeros_like(q2)
    for k in range(kbm1 - 1, 0, -1):
        vsol[:, :, k] = e2[k] * vsol[:, :, k + 1] + g2[k]
    usol[:, :, 1:kbm1] = np.abs(usol[:, :, 1:kbm1])
    vsol[:, :, 1:kbm1] = np.abs(vsol[:, :, 1:kbm1])
    coef1 = .74 * (1. - 6. * .92 / 16.6)
    coef2 = 3. * .74 * 10.1 + 18. * .92 * .74
    coef3 = .92 * (1. - 3. * .08 - 6. * .92 / 16.6)
    coef4 = 18. * .92 * .92 + 9. * .92 * .74
    coef5 = 9. * .92 * .74
    sh = coef1 / (1. - coef2 * gh)
    sm = (coef3 + sh * coef4 * gh) / (1. - coef5 * gh)
    kn = (kappa * zsh + l_out) * np.sqrt(np.abs(q2))
    kq_out = (kn * .20 + kq_in) * .5
    km_out = (kn * sm + km_in) * .5
    kh_out = (kn * sh + kh_in) * .5
    for arr in (km_out, kh_out):
        # north/south first, then east/west (fortran_compat.py:19-24)
        arr[:, 0] = arr[:, 1] * fsm[:, 0][:, None]
        arr[:, jm - 1] = arr[:, jm - 2] * fsm[:, jm - 1][:, None]
        arr[0] = arr[1] * fsm[0][:, None]
        arr[im - 1] = arr[im - 2] * fsm[im - 1][:, None]
    return dict(l=l_out, kq=kq_out, km=km_out, kh=kh_out, uf=usol, vf=vsol, cc=sound, a=aa, c=ca,
                q2b=qb, q2lb=qlb)


# ---------------------------------------------------------------------------
# tracer advection (ADVT1) and vertical diffusion (PROFT)
# ---------------------------------------------------------------------------

def advt1(S, P, fb, f, fclim):
    """Centred horizontal advection + diffusion, vertical flux, leapfrog.

    Restates ``explicit/tracers.py:433-569``.  Returns (fb', f', ff) where the
    primed inputs carry the ghost-level copy f[..., kb-1] = f[..., kb-2].
    """
    u, v, w, aam, h = S["u"], S["v"], S["w"], S["aam"], S["h"]
    dt, dx, dy, dz, art = S["dt"], S["dx"], S["dy"], S["dz"], S["art"]
    dum, dvm, etb, etf = S["dum"], S["dvm"], S["etb"], S["etf"]
    f = f.copy()
    fb = fb.copy()
    im, jm, kb = f.shape
    kbm1 = kb - 1
    f[:, :, kb - 1] = f[:, :, kbm1 - 1]
    fb[:, :, kb - 1] = fb[:, :, kbm1 - 1]
    K = slice(0, kbm1)
    si, sim, sj, sjm = slice(1, im), slice(0, im - 1), slice(1, jm), slice(0, jm - 1)
    xflux = np.zeros_like(f)
    yflux = np.zeros_like(f)
    zflux = np.zeros_like(f)
    ff = np.zeros_like(f)
    xflux[si, sj, K] = 0.25 * _b(dt[si, sj] + dt[sim, sj]) * (f[si, sj, K] + f[sim, sj, K]) * u[si, sj, K]
    yflux[si, sj, K] = 0.25 * _b(dt[si, sj] + dt[si, sjm]) * (f[si, sj, K] + f[si, sjm, K]) * v[si, sj, K]
    fa = fb - fclim
    aam_avg = 0.5 * (aam[si, sj, K] + aam[sim, sj, K])
    xflux[si, sj, K] -= aam_avg * _b(h[si, sj] + h[sim, sj]) * P.tprni * (fa[si, sj, K] - fa[sim, sj, K]) * _b(dum[si, sj]) / _b(dx[si, sj] + dx[sim, sj])
    xflux[si, sj, K] *= _b(0.5 * (dy[si, sj] + dy[sim, sj]))
    aam_avg = 0.5 * (aam[si, sj, K] + aam[si, sjm, K])
    yflux[si, sj, K] -= aam_avg * _b(h[si, sj] + h[si, sjm]) * P.tprni * (fa[si, sj, K] - fa[si, sjm, K]) * _b(dvm[si, sj]) / _b(dy[si, sj] + dy[si, sjm])
    yflux[si, sj, K] *= _b(0.5 * (dx[si, sj] + dx[si, sjm]))
    I, J, Ip, Jp = slice(1, im - 1), slice(1, jm - 1), slice(2, im), slice(2, jm)
    zflux[I, J, 0] = f[I, J, 0] * w[I, J, 0] * art[I, J]
    zflux[I, J, kb - 1] = 0.0
    ks, km = slice(1, kbm1), slice(0, kbm1 - 1)
    zflux[I, J, ks] = 0.5 * (f[I, J, km] + f[I, J, ks]) * w[I, J, ks] * _b(art[I, J])
    kp = slice(1, kbm1 + 1)
    horiz = xflux[Ip, J, K] - xflux[I, J, K] + yflux[I, Jp, K] - yflux[I, J, K]
    vert = (zflux[I, J, K] - zflux[I, J, kp]) / dz[K][None, None, :]
    ff[I, J, K] = horiz + vert
    tb = _b((h[I, J] + etb[I, J]) * art[I, J])
    tf = _b((h[I, J] + etf[I, J]) * art[I, J])
    ff[I, J, K] = (tb * fb[I, J, K] - P.dti2 * ff[I, J, K]) / (tf + 1e-20)
    return fb, f, ff


_IRR = {"R": [0.58, 0.62, 0.67, 0.77, 0.78], "AD1": [0.35, 0.60, 1.00, 1.50, 1.40],
        "AD2": [0.23, 20.0, 17.0, 14.0, 7.90]}


def proft(f, wfsurf, fsurf, nbc, h, etf, dti2, dz, dzz, swrad, ntp, kh, umol, z):
    """Implicit vertical diffusion of a tracer column (Thomas algorithm).

    Restates ``explicit/tracers.py:890-1010`` for any kb >= 3 and nbc 1-4.
    Returns (f_out, dh) with f_out[..., kb-1] = f[..., kb-1].
    """
    im, jm, kb = f.shape
    kbm1, kbm2 = kb - 1, kb - 2
    out = f.copy()
    a = np.zeros_like(f)
    c = np.zeros_like(f)
    ee = np.zeros_like(f)
    gg = np.zeros_like(f)
    idx = int(ntp) - 1
    r, ad1, ad2 = _IRR["R"][idx], _IRR["AD1"][idx], _IRR["AD2"][idx]
    dh = h + etf
    rad = np.zeros_like(f)
    for k in range(1, kbm1):
        dh2 = dh ** 2
        num = -dti2 * (kh[:, :, k] + umol)
        a[:, :, k - 1] = num / (dz[k - 1] * dzz[k - 1] * dh2)
        c[:, :, k] = num / (dz[k] * dzz[k - 1] * dh2)
    if nbc in (2, 4):
        for k in range(kbm1):
            zt = z[k] * dh
            rad[:, :, k] = swrad * (r * np.exp(zt / ad1) + (1.0 - r) * np.exp(zt / ad2))
    if nbc == 1:
        den = a[:, :, 0] - 1.0
        ee[:, :, 0] = a[:, :, 0] / den
        gprev = (-dti2 * wfsurf / (-dz[0] * dh) - f[:, :, 0]) / den
    elif nbc == 2:
        den = a[:, :, 0] - 1.0
        ee[:, :, 0] = a[:, :, 0] / den
        gprev = (dti2 * (wfsurf + (rad[:, :, 0] - rad[:, :, 1])) / (dz[0] * dh) - f[:, :, 0]) / den
    else:
        ee[:, :, 0] = 0.0
        gprev = fsurf
    gg[:, :, 0] = gprev
    for k in range(1, kbm2):
        den = a[:, :, k] + c[:, :, k] * (1.0 - ee[:, :, k - 1]) - 1.0
        inv = 1.0 / (den + 1e-20)
        ee[:, :, k] = a[:, :, k] * inv
        rt = dti2 * (rad[:, :, k] - rad[:, :, k + 1]) / (dh * dz[k])
        gprev = (c[:, :, k] * gprev - f[:, :, k] + rt) * inv
        gg[:, :, k] = gprev
    kbt = kbm1 - 1
    rt = dti2 * (rad[:, :, kbt] - rad[:, :, kbt + 1]) / (dh * dz[kbt])
    num = c[:, :, kbt] * gg[:, :, kbt - 1] - f[:, :, kbt] + rt
    den = c[:, :, kbt] * (1.0 - ee[:, :, kbt - 1]) - 1.0
    nxt = num / (den + 1e-20)
    out[:, :, kbt] = nxt
    for k in range(kbm1 - 2, -1, -1):
        nxt = ee[:, :, k] * nxt + gg[:, :, k]
        out[:, :, k] = nxt
    return out, dh


# ---------------------------------------------------------------------------
# equation of state (DENS)
# ---------------------------------------------------------------------------

def dens(S, P):
    """Mellor (1991) EOS.  Restates ``explicit/momentum.py:467-541``; returns
    a new rho with levels < kb-1 replaced."""
    kbm1 = P.kb - 1
    tr = S["t"][:, :, :kbm1] + P.tbias
    sr = S["s"][:, :, :kbm1] + P.sbias
    tr2 = tr * tr
    tr3 = tr2 * tr
    tr4 = tr3 * tr
    p = P.grav * P.rhoref * (-S["zz"][:kbm1][None, None, :] * _b(S["h"])) * 1.0e-5
    rhor = -0.157406 + 6.793952e-2 * tr - 9.095290e-3 * tr2 + 1.001685e-4 * tr3 - 1.120083e-6 * tr4 + 6.536332e-9 * tr4 * tr
    rhor = rhor + (0.824493 - 4.0899e-3 * tr + 7.6438e-5 * tr2 - 8.2467e-7 * tr3 + 5.3875e-9 * tr4) * sr
    rhor = rhor + (-5.72466e-3 + 1.0227e-4 * tr - 1.6546e-6 * tr2) * np.power(np.maximum(np.abs(sr), 1e-8), 1.5)
    rhor = rhor + 4.8314e-4 * sr * sr
    cr = 1449.1 + 0.0821 * p + 4.55 * tr - 0.045 * tr2 + 1.34 * (sr - 35.0)
    cr2 = cr * cr
    tp = 1.0e5 * p / cr2
    rhor = rhor + tp * (1.0 - 2.0 * p / cr2)
    rho = S["rho"].copy()
    rho[:, :, :kbm1] = (rhor / P.rhoref) * _b(S["fsm"])
    return rho


# ---------------------------------------------------------------------------
# internal momentum (ADVU/ADVV) and vertical viscosity (PROFU/PROFV)
# ---------------------------------------------------------------------------

def advu(S, P):
    """Restates ``explicit/momentum.py:14-131``; returns uf."""
    u, v, w, ub, advx, drhox = S["u"], S["v"], S["w"], S["ub"], S["advx"], S["drhox"]
    aru, cor, dt, dy, h, dz = S["aru"], S["cor"], S["dt"], S["dy"], S["h"], S["dz"]
    egf, egb, etf, etb, ea = S["egf"], S["egb"], S["etf"], S["etb"], S["e_atmos"]
    im, jm, kb = u.shape
    kbm1 = kb - 1
    uf = np.zeros_like(u)
    vflux = np.zeros_like(u)
    ks, km = slice(1, kbm1), slice(0, kbm1 - 1)
    si, sim = slice(1, im), slice(0, im - 1)
    vflux[si, :, ks] = 0.25 * (w[si, :, ks] + w[sim, :, ks]) * (u[si, :, ks] + u[si, :, km])
    K, Kp = slice(0, kbm1), slice(1, kbm1 + 1)
    i, im1, j, jp1 = slice(1, im - 1), slice(0, im - 2), slice(1, jm - 1), slice(2, jm)
    vdiv = (vflux[i, j, K] - vflux[i, j, Kp]) * _b(aru[i, j]) / dz[K][None, None, :]
    ct1 = _b(cor[i, j] * dt[i, j]) * (v[i, jp1, K] + v[i, j, K])
    ct2 = _b(cor[im1, j] * dt[im1, j]) * (v[im1, jp1, K] + v[im1, j, K])
    corio = -_b(aru[i, j]) * 0.25 * (ct1 + ct2)
    grad_eg = (egf[i, j] - egf[im1, j]) + (egb[i, j] - egb[im1, j])
    grad_pa = 2.0 * (ea[i, j] - ea[im1, j])
    press = P.grav * 0.125 * _b((dt[i, j] + dt[im1, j]) * (grad_eg + grad_pa) * (dy[i, j] + dy[im1, j]))
    uf[i, j, K] = advx[i, j, K] + vdiv + corio + press + drhox[i, j, K]
    hs = h[i, j] + h[im1, j]
    den = _b((hs + etf[i, j] + etf[im1, j]) * aru[i, j])
    old = _b((hs + etb[i, j] + etb[im1, j]) * aru[i, j]) * ub[i, j, K]
    uf[i, j, K] = (old - 2.0 * P.dti2 * uf[i, j, K]) / (den + 1e-20)
    return uf


def advv(S, P):
    """Restates ``explicit/momentum.py:133-248``; returns vf."""
    u, v, w, vb, advy, drhoy = S["u"], S["v"], S["w"], S["vb"], S["advy"], S["drhoy"]
    arv, cor, dt, dx, h, dz = S["arv"], S["cor"], S["dt"], S["dx"], S["h"], S["dz"]
    egf, egb, etf, etb, ea = S["egf"], S["egb"], S["etf"], S["etb"], S["e_atmos"]
    im, jm, kb = u.shape
    kbm1 = kb - 1
    vf = np.zeros_like(v)
    vflux = np.zeros_like(v)
    ks, km = slice(1, kbm1), slice(0, kbm1 - 1)
    sj, sjm = slice(1, jm), slice(0, jm - 1)
    vflux[:, sj, ks] = 0.25 * (w[:, sj, ks] + w[:, sjm, ks]) * (v[:, sj, ks] + v[:, sj, km])
    K, Kp = slice(0, kbm1), slice(1, kbm1 + 1)
    i, ip1, j, jm1 = slice(1, im - 1), slice(2, im), slice(1, jm - 1), slice(0, jm - 2)
    vdiv = (vflux[i, j, K] - vflux[i, j, Kp]) * _b(arv[i, j]) / dz[K][None, None, :]
    ct1 = _b(cor[i, j] * dt[i, j]) * (u[ip1, j, K] + u[i, j, K])
    ct2 = _b(cor[i, jm1] * dt[i, jm1]) * (u[ip1, jm1, K] + u[i, jm1, K])
    corio = _b(arv[i, j]) * 0.25 * (ct1 + ct2)
    grad_eg = (egf[i, j] - egf[i, jm1]) + (egb[i, j] - egb[i, jm1])
    grad_pa = 2.0 * (ea[i, j] - ea[i, jm1])
    press = P.grav * 0.125 * _b((dt[i, j] + dt[i, jm1]) * (grad_eg + grad_pa) * (dx[i, j] + dx[i, jm1]))
    vf[i, j, K] = advy[i, j, K] + vdiv + corio + press + drhoy[i, j, K]
    hs = h[i, j] + h[i, jm1]
    den = _b((hs + etf[i, j] + etf[i, jm1]) * arv[i, j])
    old = _b((hs + etb[i, j] + etb[i, jm1]) * arv[i, j]) * vb[i, j, K]
    vf[i, j, K] = (old - 2.0 * P.dti2 * vf[i, j, K]) / (den + 1e-20)
    return vf


def profuv(S, P, comp):
    """Implicit vertical viscosity of u ('u') or v ('v').

    Restates ``explicit/momentum.py:250-357`` (PROFU) and ``:359-465``
    (PROFV).  Returns (f_out, wbot, tps)."""
    im, jm, kb = P.im, P.jm, P.kb
    kbm1, kbm2 = kb - 1, kb - 2
    dti2, umol = P.dti2, P.umol
    dz, dzz, h, etf, km, cbc = S["dz"], S["dzz"], S["h"], S["etf"], S["km"], S["cbc"]
    ub, vb = S["ub"], S["vb"]
    if comp == "u":
        fin, wsurf, mask, wbot = S["uf"], S["wusurf"], S["dum"], S["wubot"]
        si, sj, so_i, so_j = slice(1, im), slice(1, jm), slice(0, im - 1), slice(1, jm)
    else:
        fin, wsurf, mask, wbot = S["vf"], S["wvsurf"], S["dvm"], S["wvbot"]
        si, sj, so_i, so_j = slice(1, im), slice(1, jm), slice(1, im), slice(0, jm - 1)
    fout = fin.copy()
    wbot = wbot.copy()
    a = np.zeros_like(fin)
    c = np.zeros_like(fin)
    ee = np.zeros_like(fin)
    gg = np.zeros_like(fin)
    tps = np.zeros_like(h)
    dhf = 0.5 * (h[si, sj] + etf[si, sj] + h[so_i, so_j] + etf[so_i, so_j])
    kmf = np.zeros_like(km)
    kmf[si, sj, :] = 0.5 * (km[si, sj, :] + km[so_i, so_j, :])
    dh2 = dhf ** 2
    for k in range(1, kbm1):
        num = -dti2 * (kmf[si, sj, k] + umol)
        a[si, sj, k - 1] = num / (dz[k - 1] * dzz[k - 1] * dh2)
        c[si, sj, k] = num / (dz[k] * dzz[k - 1] * dh2)
    den = a[si, sj, 0] - 1.0
    ee[si, sj, 0] = a[si, sj, 0] / (den + 1e-20)
    term = -dti2 * wsurf[si, sj] / (-dz[0] * dhf)
    gprev = (term - fin[si, sj, 0]) / (den + 1e-20)
    gg[si, sj, 0] = gprev
    for k in range(1, kbm2):
        den = a[si, sj, k] + c[si, sj, k] * (1.0 - ee[si, sj, k - 1]) - 1.0
        inv = 1.0 / (den + 1e-20)
        ee[si, sj, k] = a[si, sj, k] * inv
        gprev = (c[si, sj, k] * gprev - fin[si, sj, k]) * inv
        gg[si, sj, k] = gprev
    I, J = slice(1, im - 1), slice(1, jm - 1)
    kbt = kbm1 - 1
    if comp == "u":
        Im, Jp = slice(0, im - 2), slice(2, jm)
        cbc_avg = 0.5 * (cbc[I, J] + cbc[Im, J])
        u_sq = ub[I, J, kbt] ** 2
        vsum = vb[I, J, kbt] + vb[I, Jp, kbt] + vb[Im, J, kbt] + vb[Im, Jp, kbt]
        mag = np.sqrt(u_sq + (0.25 * vsum) ** 2 + 1e-8)
    else:
        Jm, Ip = slice(0, jm - 2), slice(2, im)
        cbc_avg = 0.5 * (cbc[I, J] + cbc[I, Jm])
        v_sq = vb[I, J, kbt] ** 2
        usum = ub[I, J, kbt] + ub[Ip, J, kbt] + ub[I, Jm, kbt] + ub[Ip, Jm, kbt]
        mag = np.sqrt((0.25 * usum) ** 2 + v_sq + 1e-8)
    tps[I, J] = cbc_avg * mag
    fric = tps[I, J] * dti2 / (-dz[kbt] * dhf[0:im - 2, 0:jm - 2])
    den = fric - 1.0 - (ee[I, J, kbt - 1] - 1.0) * c[I, J, kbt]
    num = c[I, J, kbt] * gg[I, J, kbt - 1] - fin[I, J, kbt]
    nxt = num / (den + 1e-20) * mask[I, J]
    fout[I, J, kbt] = nxt
    for k in range(kbt - 1, -1, -1):
        nxt = (ee[I, J, k] * nxt + gg[I, J, k]) * mask[I, J]
        fout[I, J, k] = nxt
    wbot[I, J] = -tps[I, J] * fout[I, J, kbt]
    return fout, wbot, tps


# ---------------------------------------------------------------------------
# implicit barotropic mode
# ---------------------------------------------------------------------------

def implicit_coefficients(S, P):
    """Cached elliptic-operator geometry.  Restates
    ``implicit_p0_fixed/core.py:121-199``."""
    dx, dy, dum, dvm, art = S["dx"], S["dy"], S["dum"], S["dvm"], S["art"]
    im, jm = dx.shape
    i, j = slice(1, im - 1), slice(1, jm - 1)
    ip, imn, jp, jmn = slice(2, im), slice(0, im - 2), slice(2, jm), slice(0, jm - 2)
    dx_e = 0.5 * (dx[ip, j] + dx[i, j])
    dx_w = 0.5 * (dx[i, j] + dx[imn, j])
    dy_e = 0.5 * (dy[ip, j] + dy[i, j])
    dy_w = 0.5 * (dy[i, j] + dy[imn, j])
    dy_n = 0.5 * (dy[i, jp] + dy[i, j])
    dy_s = 0.5 * (dy[i, j] + dy[i, jmn])
    dx_n = 0.5 * (dx[i, jp] + dx[i, j])
    dx_s = 0.5 * (dx[i, j] + dx[i, jmn])
    return dict(
        ce=dy_e / (dx_e + 1e-20), cw=dy_w / (dx_w + 1e-20),
        cn=dx_n / (dy_n + 1e-20), cs=dx_s / (dy_s + 1e-20),
        me=dum[ip, j], mw=dum[i, j], mn=dvm[i, jp], ms=dvm[i, j],
        inv_art=1.0 / (art[i, j] + 1e-20),
        coeff=4.0 * (P.dti ** 2) * P.grav * P.alpha,
    )


def elliptic_apply(eta, d, C):
    """out = eta - coeff*div(D grad eta)/art on the interior, eta elsewhere.
    Restates ``implicit_p0_fixed/core.py:591-639``."""
    im, jm = eta.shape
    i, j = slice(1, im - 1), slice(1, jm - 1)
    ip, imn, jp, jmn = slice(2, im), slice(0, im - 2), slice(2, jm), slice(0, jm - 2)
    he = 0.5 * (d[ip, j] + d[i, j])
    hw = 0.5 * (d[i, j] + d[imn, j])
    hn = 0.5 * (d[i, jp] + d[i, j])
    hs = 0.5 * (d[i, j] + d[i, jmn])
    fe = he * (eta[ip, j] - eta[i, j]) * C["ce"] * C["me"]
    fw = hw * (eta[i, j] - eta[imn, j]) * C["cw"] * C["mw"]
    fn = hn * (eta[i, jp] - eta[i, j]) * C["cn"] * C["mn"]
    fs = hs * (eta[i, j] - eta[i, jmn]) * C["cs"] * C["ms"]
    div = (fe - fw + fn - fs) * C["inv_art"]
    out = eta.copy()
    out[i, j] = eta[i, j] - C["coeff"] * div
    return out


def jacobi_diag(d, C):
    """Restates ``implicit_p0_fixed/core.py:677-700``."""
    im, jm = d.shape
    i, j = slice(1, im - 1), slice(1, jm - 1)
    ip, imn, jp, jmn = slice(2, im), slice(0, im - 2), slice(2, jm), slice(0, jm - 2)
    he = 0.5 * (d[ip, j] + d[i, j])
    hw = 0.5 * (d[i, j] + d[imn, j])
    hn = 0.5 * (d[i, jp] + d[i, j])
    hs = 0.5 * (d[i, j] + d[i, jmn])
    diag = np.ones_like(d)
    diag[i, j] = 1.0 + C["coeff"] * C["inv_art"] * (
        he * C["ce"] * C["me"] + hw * C["cw"] * C["mw"] + hn * C["cn"] * C["mn"] + hs * C["cs"] * C["ms"])
    return diag


def dst1_matrix(n, dtype=np.float64):
    """S[k, m] = 2*sin(pi*(k+1)*(m+1)/(n+1)): the DST-I that
    ``implicit_p0_fixed/core.py:713-728`` evaluates through an FFT of the odd
    extension (-imag of the first n bins of fft([0, x, 0, -flip(x)]))."""
    k = np.arange(1, n + 1, dtype=np.float64)
    return (2.0 * np.sin(np.pi * np.outer(k, k) / (n + 1))).astype(dtype)


def hartley_matrix(n):
    """H[k, m] = cas(2 pi k m / n) = cos + sin: symmetric, H H = n I, and
    H C H = n diag(lambda) for a symmetric circulant C (the periodic second
    difference: lambda_k = 4 sin^2(pi k / n)).  No counterpart in the
    reference, which has no periodic boundary."""
    k = np.arange(n, dtype=np.float64)
    t = 2.0 * np.pi * np.outer(k, k) / n
    return np.cos(t) + np.sin(t)


def spectral_cache(S, P, C):
    """Restates ``implicit_p0_fixed/core.py:730-760`` (median spacings and
    depth of the interior, eigenvalues of the constant-coefficient
    operator).  With ``P.periodic_x`` the rows are the unique columns
    2..im-3 and the x transform is the Hartley matrix of the period (its
    eigenvalues 4 sin^2(pi k / n) / dx^2, scale n * 2(nj+1))."""
    dx, dy, h = S["dx"], S["dy"], S["h"]
    im, jm = dx.shape
    periodic = bool(getattr(P, "periodic_x", False))
    i, j = (slice(2, im - 2) if periodic else slice(1, im - 1)), slice(1, jm - 1)
    ni, nj = (im - 4 if periodic else im - 2), jm - 2
    dt_ = dx.dtype

    def tmedian(a):
        # torch.median returns the lower of the two middle values
        flat = np.sort(a.reshape(-1))
        return flat[(flat.size - 1) // 2]

    dx0, dy0, h0 = tmedian(dx[i, j]), tmedian(dy[i, j]), tmedian(h[i, j])
    ky = np.arange(1, nj + 1, dtype=dt_).reshape(1, -1)
    if periodic:
        kx = np.arange(0, ni, dtype=dt_).reshape(-1, 1)
        lam_x = 4.0 * np.square(np.sin(np.pi * kx / ni)) / (dx0 * dx0 + 1e-30)
    else:
        kx = np.arange(1, ni + 1, dtype=dt_).reshape(-1, 1)
        lam_x = 4.0 * np.square(np.sin(np.pi * kx / (2.0 * (ni + 1)))) / (dx0 * dx0 + 1e-30)
    lam_y = 4.0 * np.square(np.sin(np.pi * ky / (2.0 * (nj + 1)))) / (dy0 * dy0 + 1e-30)
    inv_eigs = 1.0 / (1.0 + C["coeff"] * h0 * (lam_x + lam_y))
    sx = hartley_matrix(ni) if periodic else dst1_matrix(ni)
    scale = 2.0 * ni * (nj + 1) if periodic else 4.0 * (ni + 1) * (nj + 1)
    return dict(inv_eigs=inv_eigs.astype(dt_), inverse_scale=scale, sx=sx, sy=dst1_matrix(nj), rows=i)


def spectral_apply(r, SC):
    """z = DST(DST(r_int) * inv_eigs) / (4(ni+1)(nj+1)) on the interior
    (the rows of ``SC['rows']``; Hartley along a periodic x).
    Restates ``implicit_p0_fixed/core.py:762-773``."""
    im, jm = r.shape
    i, j = SC.get("rows", slice(1, im - 1)), slice(1, jm - 1)
    dt_ = r.dtype
    x = r[i, j].astype(np.float64)
    coef = (SC["sx"] @ x @ SC["sy"]).astype(dt_)
    coef = coef * SC["inv_eigs"]
    inner = (SC["sx"] @ coef.astype(np.float64) @ SC["sy"]).astype(dt_) / SC["inverse_scale"]
    z = np.zeros_like(r)
    z[i, j] = inner
    return z


def pcg_solve(rhs, d, x0, S, P, C, SC, max_iter, tol, rel_tol, precond, dot_dtype=np.float64, periodic=False):
    """Preconditioned CG for the implicit free surface (Dirichlet ring).

    Restates ``implicit_p0_fixed/core.py:460-589`` (non-graph branch): stop
    when rs <= tol^2, rs <= rel_tol^2*max(rs0, 1e-30) or rs <= 1e-30.  Dot
    products are accumulated in ``dot_dtype`` (float64 here; the reference's
    are float32).  With ``periodic`` (periodic x) the ring of the iterated
    vectors is wrapped in i instead of zeroed (``_pcg_ring``), which makes
    the operator periodic; the unknowns are then the unique columns
    2..im-3 (the dot products run over them only).  Returns (x,
    iterations).
    """
    im, jm = rhs.shape
    I, J = slice(1, im - 1), slice(1, jm - 1)
    # the unknowns: the interior, or the unique columns 2..im-3 when periodic
    IU = slice(2, im - 2) if periodic else I

    def dot(a, b):
        return float(np.sum(a[IU, J].astype(dot_dtype) * b[IU, J].astype(dot_dtype)))

    x = x0.copy()
    _pcg_ring(x, periodic)
    rw = rhs.copy()
    _zero_ring(rw)
    ap = elliptic_apply(x, d, C)
    r = rw - ap
    if precond == "spectral":
        z = spectral_apply(r, SC)
    else:
        diag = jacobi_diag(d, C)
        z = r.copy()
        z[I, J] = r[I, J] / (diag[I, J] + 1e-30)
    p = z.copy()
    rho_old = dot(r, z)
    rs0 = dot(r, r)
    tol_sq = tol * tol
    rel_sq = rel_tol ** 2 * max(rs0, 1e-30)
    its = 0
    dt_ = rhs.dtype
    for it in range(1, max_iter + 1):
        _pcg_ring(p, periodic)
        ap = elliptic_apply(p, d, C)
        denom = dot(p, ap)
        alpha = rho_old / (denom + 1e-30)
        x = x + np.asarray(alpha, dtype=dt_) * p
        _pcg_ring(x, periodic)
        r = r - np.asarray(alpha, dtype=dt_) * ap
        rs = dot(r, r)
        its = it
        if rs <= tol_sq or rs <= rel_sq or rs <= 1e-30:
            break
        if precond == "spectral":
            z = spectral_apply(r, SC)
        else:
            z = r.copy()
            z[I, J] = r[I, J] / (diag[I, J] + 1e-30)
        rho_new = dot(r, z)
        beta = rho_new / (rho_old + 1e-30)
        p = p * np.asarray(beta, dtype=dt_) + z
        _pcg_ring(p, periodic)
        rho_old = rho_new
    _pcg_ring(x, periodic)
    return x, its


def eta_depth_adjoint(eta, lam_eta, d, C):
    """d/dd of <lam_eta, A(d) eta> with the sign of the reference, i.e. the
    array that ``_ImplicitEtaSolveFunction.backward`` negates.  Restates
    ``implicit_p0_fixed/core.py:645-675``; the eight scatter-adds run in the
    reference's statement order (their rounding depends on it)."""
    im, jm = eta.shape
    i, j = slice(1, im - 1), slice(1, jm - 1)
    ip, imn, jp, jmn = slice(2, im), slice(0, im - 2), slice(2, jm), slice(0, jm - 2)
    grad = np.zeros_like(d)
    lam = lam_eta[i, j] * C["coeff"] * C["inv_art"]
    east = 0.5 * lam * (eta[ip, j] - eta[i, j]) * C["ce"] * C["me"]
    west = 0.5 * lam * (eta[i, j] - eta[imn, j]) * C["cw"] * C["mw"]
    north = 0.5 * lam * (eta[i, jp] - eta[i, j]) * C["cn"] * C["mn"]
    south = 0.5 * lam * (eta[i, j] - eta[i, jmn]) * C["cs"] * C["ms"]
    grad[ip, j] += -east
    grad[i, j] += -east
    grad[i, j] += west
    grad[imn, j] += west
    grad[i, jp] += -north
    grad[i, j] += -north
    grad[i, j] += south
    grad[i, jmn] += south
    return grad


def eta_adjoint(g, x, d, S, P, C, SC, max_iter, tol, rel_tol, precond, dot_dtype=np.float64):
    """Backward of the free-surface solve x = A(d)^-1 rhs for the cotangent
    g = dJ/dx.  Restates ``implicit_p0_fixed/core.py:24-59`` (the autograd
    function) and ``:231-252`` (A^-T = M A^-1 M^-1 with relative cell
    areas, the right-hand side scaled by max|rhs| clamped to 1 and the
    absolute tolerance by the same factor, zero initial guess).  Returns
    (dJ/drhs, dJ/dd, adjoint iterations)."""
    dt_ = g.dtype
    area = np.ones_like(g)
    area[1:-1, 1:-1] = S["art"][1:-1, 1:-1] / S["art"][1, 1]
    rhs = g / area
    scale = np.asarray(max(np.max(np.abs(rhs)), dt_.type(1.0)), dtype=dt_)
    nrhs = rhs / scale
    sol, its = pcg_solve(nrhs, d, np.zeros_like(g), S, P, C, SC, max_iter, float(tol) / float(scale), rel_tol,
                         precond, dot_dtype=dot_dtype)
    lam = sol * area * scale
    return lam, -eta_depth_adjoint(x, lam, d, C), its


def barotropic_predictor(S, P):
    """Restates ``implicit_p0_fixed/core.py:795-845``; returns
    (u_star, v_star, denom_u, denom_v) before the velocity BC."""
    ua, va, el, elb, d, cor = S["ua"], S["va"], S["el"], S["elb"], S["d"], S["cor"]
    dx, dy, h, aru, arv = S["dx"], S["dy"], S["h"], S["aru"], S["arv"]
    ea, g, al, dti = S["e_atmos"], P.grav, P.alpha, P.dti
    im, jm = ua.shape
    i, j = slice(1, im - 1), slice(1, jm - 1)
    imn, jmn, ip, jp = slice(0, im - 2), slice(0, jm - 2), slice(2, im), slice(2, jm)
    cor_u = 0.25 * (cor[i, j] * d[i, j] * (va[i, jp] + va[i, j]) + cor[imn, j] * d[imn, j] * (va[imn, jp] + va[imn, j]))
    cor_v = 0.25 * (cor[i, j] * d[i, j] * (ua[ip, j] + ua[i, j]) + cor[i, jmn] * d[i, jmn] * (ua[ip, jmn] + ua[i, jmn]))
    gu = 0.25 * g * (dy[i, j] + dy[imn, j]) * (d[i, j] + d[imn, j]) * (
        (1.0 - 2.0 * al) * (el[i, j] - el[imn, j]) + al * (elb[i, j] - elb[imn, j]) + ea[i, j] - ea[imn, j])
    gv = 0.25 * g * (dx[i, j] + dx[i, jmn]) * (d[i, j] + d[i, jmn]) * (
        (1.0 - 2.0 * al) * (el[i, j] - el[i, jmn]) + al * (elb[i, j] - elb[i, jmn]) + ea[i, j] - ea[i, jmn])
    uprov = S["adx2d"][i, j] + S["advua"][i, j] - aru[i, j] * cor_u + gu + S["drx2d"][i, j] - aru[i, j] * (-S["wusurf"][i, j] + S["wubot"][i, j])
    vprov = S["ady2d"][i, j] + S["advva"][i, j] + arv[i, j] * cor_v + gv + S["dry2d"][i, j] - arv[i, j] * (-S["wvsurf"][i, j] + S["wvbot"][i, j])
    us, vs = ua.copy(), va.copy()
    den_u = (h[i, j] + el[i, j] + h[imn, j] + el[imn, j]) * aru[i, j]
    num_u = (h[i, j] + elb[i, j] + h[imn, j] + elb[imn, j]) * aru[i, j] * S["uab"][i, j] - 4.0 * dti * uprov
    den_v = (h[i, j] + el[i, j] + h[i, jmn] + el[i, jmn]) * arv[i, j]
    num_v = (h[i, j] + elb[i, j] + h[i, jmn] + elb[i, jmn]) * arv[i, j] * S["vab"][i, j] - 4.0 * dti * vprov
    us[i, j] = (num_u / (den_u + 1e-20)) * S["dum"][i, j]
    vs[i, j] = (num_v / (den_v + 1e-20)) * S["dvm"][i, j]
    return us, vs, den_u, den_v


def barotropic_rhs(S, P, us, vs):
    """Restates ``implicit_p0_fixed/core.py:858-891``; returns (fluxua,
    fluxva, rhs) on the full grid."""
    d, dx, dy, art, elb = S["d"], S["dx"], S["dy"], S["art"], S["elb"]
    im, jm = d.shape
    sf, sfm, tf, tfm = slice(1, im), slice(0, im - 1), slice(1, jm), slice(0, jm - 1)
    fu = 0.25 * (d[sf, tf] + d[sfm, tf]) * (dy[sf, tf] + dy[sfm, tf]) * us[sf, tf]
    fv = 0.25 * (d[sf, tf] + d[sf, tfm]) * (dx[sf, tf] + dx[sf, tfm]) * vs[sf, tf]
    div = fu[1:, :-1] - fu[:-1, :-1] + fv[:-1, 1:] - fv[:-1, :-1]
    i, j = slice(1, im - 1), slice(1, jm - 1)
    rhs = elb.copy()
    rhs[i, j] = elb[i, j] - 2.0 * P.dti * (div / (art[i, j] + 1e-20) + S["vfluxf"][i, j])
    fluxua = np.zeros_like(d)
    fluxva = np.zeros_like(d)
    fluxua[1:, 1:] = fu
    fluxva[1:, 1:] = fv
    return fluxua, fluxva, rhs


def barotropic_shapiro(elf, S, gamma):
    """Restates ``implicit_p0_fixed/core.py:893-911``."""
    im, jm = elf.shape
    i, j = slice(1, im - 1), slice(1, jm - 1)
    ip, imn, jp, jmn = slice(2, im), slice(0, im - 2), slice(2, jm), slice(0, jm - 2)
    sm = elf[i, j] + (gamma / 4.0) * (elf[ip, j] + elf[imn, j] + elf[i, jp] + elf[i, jmn] - 4.0 * elf[i, j])
    out = elf.copy()
    out[i, j] = sm * S["fsm"][i, j]
    return out


def barotropic_corrector(S, P, us, vs, den_u, den_v):
    """Restates ``implicit_p0_fixed/core.py:918-934``; returns interior
    (uaf, vaf)."""
    elf, d, dx, dy, h = S["elf"], S["d"], S["dx"], S["dy"], S["h"]
    aru, arv, g, al, dti = S["aru"], S["arv"], P.grav, P.alpha, P.dti
    im, jm = elf.shape
    i, j, imn, jmn = slice(1, im - 1), slice(1, jm - 1), slice(0, im - 2), slice(0, jm - 2)
    gu = 0.25 * g * (dy[i, j] + dy[imn, j]) * (d[i, j] + d[imn, j]) * al * (elf[i, j] - elf[imn, j])
    gv = 0.25 * g * (dx[i, j] + dx[i, jmn]) * (d[i, j] + d[i, jmn]) * al * (elf[i, j] - elf[i, jmn])
    dfu = (h[i, j] + elf[i, j] + h[imn, j] + elf[imn, j]) * aru[i, j]
    dfv = (h[i, j] + elf[i, j] + h[i, jmn] + elf[i, jmn]) * arv[i, j]
    uaf = (us[i, j] * den_u - 4.0 * dti * gu) / (dfu + 1e-20) * S["dum"][i, j]
    vaf = (vs[i, j] * den_v - 4.0 * dti * gv) / (dfv + 1e-20) * S["dvm"][i, j]
    return uaf, vaf


# ---------------------------------------------------------------------------
# parameters
# ---------------------------------------------------------------------------

class Params:
    """Scalar settings of a core (the Python attributes of the reference's
    ``BaseCore``, ``explicit/base.py:9-189``)."""

    def __init__(self, **kw):
        self.__dict__.update(kw)

    def copy(self):
        return Params(**self.__dict__)


# ---------------------------------------------------------------------------
# explicit external subcycle and time step
# ---------------------------------------------------------------------------

class VmaxExceeded(FloatingPointError):
    pass


def _barotropic_fix(S, P):
    """Restates ``explicit/time_loop.py:440-477`` (identical in the implicit
    loop ``time_loop.py:396-433``)."""
    kbm1, im, jm = P.kb - 1, P.im, P.jm
    dz = S["dz"][:kbm1][None, None, :]
    for name, tb, tf, ax in (("u", "utb", "utf", 0), ("v", "vtb", "vtf", 1)):
        f = S[name]
        tps = _sum_k(f[:, :, :kbm1] * dz)
        if ax == 0:
            dts = S["dt"][1:im, :] + S["dt"][0:im - 1, :]
            corr = (S[tb][1:im, :] + S[tf][1:im, :]) / (dts + 1e-20)
            new = f.copy()
            new[1:im, :, :kbm1] = (f[1:im, :, :kbm1] - tps[1:im, :, None]) + corr[:, :, None]
        else:
            dts = S["dt"][:, 1:jm] + S["dt"][:, 0:jm - 1]
            corr = (S[tb][:, 1:jm] + S[tf][:, 1:jm]) / (dts + 1e-20)
            new = f.copy()
            new[:, 1:jm, :kbm1] = (f[:, 1:jm, :kbm1] - tps[:, 1:jm, None]) + corr[:, :, None]
        S[name] = new


def _internal_velocity_filter(S, P, shapiro=None):
    """Restates ``explicit/time_loop.py:632-678`` (explicit) and
    ``implicit_p0_fixed/time_loop.py:585-639`` (implicit, with the Shapiro
    filter and masks of ``numerics/double_gyre.py:147-184``)."""
    kbm1 = P.kb - 1
    dz = S["dz"][:kbm1][None, None, :]
    out = {}
    for f, ff, fb in (("u", "uf", "ub"), ("v", "vf", "vb")):
        term = S[ff][:, :, :kbm1] + S[fb][:, :, :kbm1] - 2.0 * S[f][:, :, :kbm1]
        tps = _sum_k(term * dz)
        filt = S[f].copy()
        filt[:, :, :kbm1] = S[f][:, :, :kbm1] + 0.5 * P.smoth * (term - tps[:, :, None])
        out[f] = filt
    if shapiro is not None:
        uf_, vf_ = out["u"], out["v"]
        gamma = shapiro
        for name, mask in (("u", "dum"), ("v", "dvm")):
            a = out[name]
            sh = a.copy()
            if gamma > 0.0:
                im, jm = P.im, P.jm
                I, J, K = slice(1, im - 1), slice(1, jm - 1), slice(0, kbm1)
                sh[I, J, K] = a[I, J, K] + (gamma / 4.0) * (a[2:im, J, K] + a[0:im - 2, J, K] + a[I, 2:jm, K] + a[I, 0:jm - 2, K] - 4.0 * a[I, J, K])
            out[name] = sh * _b(S[mask])
    S["ub"] = out["u"]
    S["u"] = S["uf"].copy()
    S["vb"] = out["v"]
    S["v"] = S["vf"].copy()


def step_explicit(S, P):
    """One internal step of the explicit mode-split core.

    Restates ``explicit/time_loop.py:75-709`` for the non-fast path (the
    generation fast path computes the same values in place).  Raises
    VmaxExceeded where the reference would print 'Abnormal end' and return.
    """
    im, jm, kb = P.im, P.jm, P.kb
    kbm1 = kb - 1
    P.iint += 1
    iint = P.iint
    P.time = P.dti * iint * 1.0 / 86400.0 + P.time0
    if P.lramp:
        P.ramp = min(P.time / P.period, 1.0)
    else:
        P.ramp = 1.0
    I, J = slice(1, im - 1), slice(1, jm - 1)
    Im, Jm = slice(0, im - 2), slice(0, jm - 2)
    Ip, Jp = slice(2, im), slice(2, jm)

    surface_fluxes(S, P)
    curv, advx, advy = advct(S, P)
    S["curv"], S["advx"], S["advy"] = curv, advx, advy
    S["rho"], S["drhox"], S["drhoy"] = baropg(S, P)
    S["aam"] = smagorinsky_explicit(S, P)
    S["adx2d"], S["ady2d"], S["drx2d"], S["dry2d"], S["aam2d"] = vertical_means(S, P)
    fluxua, fluxva, tps = S["fluxua"].copy(), S["fluxva"].copy(), S["tps"].copy()
    S["advua"], S["advva"] = advave(S, P, fluxua, fluxva, tps)
    S["fluxua"], S["fluxva"], S["tps"] = fluxua, fluxva, tps
    S["adx2d"] = S["adx2d"] - S["advua"]
    S["ady2d"] = S["ady2d"] - S["advva"]

    S["egf"] = S["el"] * P.ispi
    d = S["d"]
    utf = S["utf"].copy()
    vtf = S["vtf"].copy()
    utf[1:im, :] = S["ua"][1:im, :] * (d[1:im, :] + d[0:im - 1, :]) * P.isp2i
    vtf[:, 1:jm] = S["va"][:, 1:jm] * (d[:, 1:jm] + d[:, 0:jm - 1]) * P.isp2i
    S["utf"], S["vtf"] = utf, vtf

    vamax = 0.0
    exceeded = False
    F = {}
    for iext in range(1, P.isplit + 1):
        d = S["d"]
        dx, dy = S["dx"], S["dy"]
        fu, fv = S["fluxua"], S["fluxva"]
        fu[1:, 1:] = 0.25 * (d[1:, 1:] + d[:-1, 1:]) * (dy[1:, 1:] + dy[:-1, 1:]) * S["ua"][1:, 1:]
        fv[1:, 1:] = 0.25 * (d[1:, 1:] + d[1:, :-1]) * (dx[1:, 1:] + dx[1:, :-1]) * S["va"][1:, 1:]
        div = fu[Ip, J] - fu[I, J] + fv[I, Jp] - fv[I, J]
        elf = S["elf"].copy()
        elf[I, J] = S["elb"][I, J] + P.dte2 * (-(div / S["art"][I, J]) - S["vfluxf"][I, J])
        F["elf"] = elf
        bcond_explicit(S, P, 1, F)
        S["elf"] = F["elf"]
        if iext % P.ispadv == 0:
            S["advua"], S["advva"] = advave(S, P, S["fluxua"], S["fluxva"], S["tps"])
        el, elb, elf, ea = S["el"], S["elb"], S["elf"], S["e_atmos"]
        cor, h, al, g = S["cor"], S["h"], P.alpha, P.grav
        aru, arv, ua, va = S["aru"], S["arv"], S["ua"], S["va"]
        cor_u = 0.25 * (cor[I, J] * d[I, J] * (va[I, Jp] + va[I, J]) + cor[Im, J] * d[Im, J] * (va[Im, Jp] + va[Im, J]))
        gu = 0.25 * g * (dy[I, J] + dy[Im, J]) * (d[I, J] + d[Im, J]) * (
            (1.0 - 2.0 * al) * (el[I, J] - el[Im, J]) + al * (elb[I, J] - elb[Im, J] + elf[I, J] - elf[Im, J]) + ea[I, J] - ea[Im, J])
        uaf = S["uaf"].copy()
        uaf[I, J] = S["adx2d"][I, J] + S["advua"][I, J] - aru[I, J] * cor_u + gu + S["drx2d"][I, J] - aru[I, J] * (-S["wusurf"][I, J] + S["wubot"][I, J])
        den = (h[I, J] + elf[I, J] + h[Im, J] + elf[Im, J]) * aru[I, J]
        num = (h[I, J] + elb[I, J] + h[Im, J] + elb[Im, J]) * aru[I, J] * S["uab"][I, J] - 4.0 * P.dte * uaf[I, J]
        uaf[I, J] = num / (den + 1e-20)
        cor_v = 0.25 * (cor[I, J] * d[I, J] * (ua[Ip, J] + ua[I, J]) + cor[I, Jm] * d[I, Jm] * (ua[Ip, Jm] + ua[I, Jm]))
        gv = 0.25 * g * (dx[I, J] + dx[I, Jm]) * (d[I, J] + d[I, Jm]) * (
            (1.0 - 2.0 * al) * (el[I, J] - el[I, Jm]) + al * (elb[I, J] - elb[I, Jm] + elf[I, J] - elf[I, Jm]) + ea[I, J] - ea[I, Jm])
        vaf = S["vaf"].copy()
        vaf[I, J] = S["ady2d"][I, J] + S["advva"][I, J] + arv[I, J] * cor_v + gv + S["dry2d"][I, J] - arv[I, J] * (-S["wvsurf"][I, J] + S["wvbot"][I, J])
        den = (h[I, J] + elf[I, J] + h[I, Jm] + elf[I, Jm]) * arv[I, J]
        num = (h[I, J] + elb[I, J] + h[I, Jm] + elb[I, Jm]) * arv[I, J] * S["vab"][I, J] - 4.0 * P.dte * vaf[I, J]
        vaf[I, J] = num / (den + 1e-20)
        F["uaf"], F["vaf"] = uaf, vaf
        bcond_explicit(S, P, 2, F)
        S["uaf"], S["vaf"] = F["uaf"], F["vaf"]
        etf = S["etf"].copy()
        if iext == P.isplit - 2:
            etf[:] = 0.25 * P.smoth * S["elf"]
        elif iext == P.isplit - 1:
            etf[:] += 0.5 * (1.0 - 0.5 * P.smoth) * S["elf"]
        elif iext == P.isplit:
            etf[:] = (etf + 0.5 * S["elf"]) * S["fsm"]
        S["etf"] = etf
        vamax = float(np.max(np.abs(S["vaf"])))
        if vamax <= P.vmaxl:
            S["ua"] = S["ua"] + 0.5 * P.smoth * (S["uab"] - 2.0 * S["ua"] + S["uaf"])
            S["va"] = S["va"] + 0.5 * P.smoth * (S["vab"] - 2.0 * S["va"] + S["vaf"])
            S["el"] = S["el"] + 0.5 * P.smoth * (S["elb"] - 2.0 * S["el"] + S["elf"])
            S["elb"] = S["el"].copy()
            S["el"] = S["elf"].copy()
            S["d"] = S["h"] + S["el"]
            S["uab"] = S["ua"].copy()
            S["ua"] = S["uaf"].copy()
            S["vab"] = S["va"].copy()
            S["va"] = S["vaf"].copy()
            if iext != P.isplit:
                S["egf"] = S["egf"] + S["el"] * P.ispi
                d = S["d"]
                S["utf"][1:im, :] = S["utf"][1:im, :] + S["ua"][1:im, :] * (d[1:im, :] + d[0:im - 1, :]) * P.isp2i
                S["vtf"][:, 1:jm] = S["vtf"][:, 1:jm] + S["va"][:, 1:jm] * (d[:, 1:jm] + d[:, 0:jm - 1]) * P.isp2i
        else:
            exceeded = True

    if vamax <= P.vmaxl and (iint != 1 or P.time0 != 0.0) and P.mode != 2:
        _barotropic_fix(S, P)
        S["w"] = vertvl(S, P)
        F = {"w": S["w"]}
        bcond_explicit(S, P, 5, F)
        S["w"] = F["w"]
        uf = np.zeros_like(S["u"])
        vf = np.zeros_like(S["u"])
        uf = advq(S, P, S["q2b"], S["q2"], uf)
        vf = advq(S, P, S["q2lb"], S["q2l"], vf)
        S["uf"], S["vf"] = uf, vf
        if getattr(P, "profq_form", "production") == "pom08":
            R = profq_pom08(S, P, uf, vf)
            S["q2b"], S["q2lb"] = R["q2b"], R["q2lb"]
        else:
            R = profq(S, P, uf, vf, implicit_variant=False)
        S["l"], S["kq"], S["km"], S["kh"] = R["l"], R["kq"], R["km"], R["kh"]
        S["dtef"] = R["cc"]
        F = {"uf": R["uf"], "vf": R["vf"]}
        bcond_explicit(S, P, 6, F)
        S["uf"], S["vf"] = F["uf"], F["vf"]
        q2 = S["q2"] + 0.5 * P.smoth * (S["uf"] + S["q2b"] - 2.0 * S["q2"])
        q2l = S["q2l"] + 0.5 * P.smoth * (S["vf"] + S["q2lb"] - 2.0 * S["q2l"])
        S["q2b"], S["q2"], S["q2lb"], S["q2l"] = q2, S["uf"].copy(), q2l, S["vf"].copy()
        if P.mode != 4:
            S["tb"], S["t"], uf = advt1(S, P, S["tb"], S["t"], S["tclim"])
            S["sb"], S["s"], vf = advt1(S, P, S["sb"], S["s"], S["sclim"])
            uf, _ = proft(uf, S["wtsurf"], S["tsurf"], P.nbct, S["h"], S["etf"], P.dti2, S["dz"], S["dzz"],
                          S["swrad"], P.ntp, S["kh"], P.umol, S["z"])
            vf, dh = proft(vf, S["wssurf"], S["ssurf"], P.nbcs, S["h"], S["etf"], P.dti2, S["dz"], S["dzz"],
                           S["swrad"], P.ntp, S["kh"], P.umol, S["z"])
            S["tps"] = dh
            F = {"uf": uf, "vf": vf}
            bcond_explicit(S, P, 4, F)
            S["uf"], S["vf"] = F["uf"], F["vf"]
            t = S["t"] + 0.5 * P.smoth * (S["uf"] + S["tb"] - 2.0 * S["t"])
            s = S["s"] + 0.5 * P.smoth * (S["vf"] + S["sb"] - 2.0 * S["s"])
            S["tb"], S["t"], S["sb"], S["s"] = t, S["uf"].copy(), s, S["vf"].copy()
            S["rho"] = dens(S, P)
        S["uf"] = advu(S, P)
        S["vf"] = advv(S, P)
        S["uf"], S["wubot"], _ = profuv(S, P, "u")
        S["vf"], S["wvbot"], S["tps"] = profuv(S, P, "v")
        F = {"uf": S["uf"], "vf": S["vf"]}
        bcond_explicit(S, P, 3, F)
        S["uf"], S["vf"] = F["uf"], F["vf"]
        _internal_velocity_filter(S, P, shapiro=None)

    S["egb"] = S["egf"].copy()
    S["etb"] = S["et"].copy()
    S["et"] = S["etf"].copy()
    S["dt"] = S["h"] + S["et"]
    S["utb"] = S["utf"].copy()
    S["vtb"] = S["vtf"].copy()
    S["vfluxb"] = S["vfluxf"].copy()
    if vamax > P.vmaxl:
        raise VmaxExceeded(f"Barotropic velocity {vamax} exceeds limit {P.vmaxl} at time {P.time}")
    return exceeded


# ---------------------------------------------------------------------------
# implicit time step
# ---------------------------------------------------------------------------

def step_implicit(S, P, C=None, SC=None, dot_dtype=np.float64):
    """One internal step of the semi-implicit free-surface core.

    Restates ``implicit_p0_fixed/time_loop.py:105-688`` with the closed-basin
    boundary, double-gyre wind forcing and numerics plugins
    (``boundary/closed_basin.py``, ``forcing/surface.py``,
    ``numerics/double_gyre.py``).  ``S['_eta_prev']`` (optional) plays the
    role of ``_eta_prev_solution``.  Returns the PCG iteration count.

    With ``P.periodic_x`` the x edges are periodic instead of walls (the
    reference has no periodic boundary): after each phase of the CUDA step
    (A1, A2, A3, the η-solve, I5, B1-B9; the comments below name them)
    every plane gets the halo fill ``periodic_fill``, and the η-solve's
    operator wraps in x (``pcg_solve(periodic=True)``).
    """
    im, jm, kb = P.im, P.jm, P.kb
    kbm1 = kb - 1
    if C is None:
        C = implicit_coefficients(S, P)
    if SC is None and P.eta_solver_preconditioner == "spectral":
        SC = spectral_cache(S, P, C)
    P.iint += 1
    iint = P.iint
    P.time = P.dti * iint * 1.0 / 86400.0 + P.time0
    if P.lramp:
        P.ramp = min(P.time / P.period, 1.0)
    else:
        P.ramp = 1.0

    if getattr(P, "wind_forcing", True):
        double_gyre_wind(S, P)
    surface_fluxes(S, P)
    curv, advx, advy = advct(S, P)
    S["curv"], S["advx"], S["advy"] = curv, advx, advy
    periodic_fill(S, P)  # A1
    S["rho"], S["drhox"], S["drhoy"] = baropg(S, P)
    S["aam"] = smagorinsky_implicit(S, P)
    S["adx2d"], S["ady2d"], S["drx2d"], S["dry2d"], S["aam2d"] = vertical_means(S, P)
    periodic_fill(S, P)  # A2
    fluxua, fluxva, tps = S["fluxua"].copy(), S["fluxva"].copy(), S["tps"].copy()
    S["advua"], S["advva"] = advave(S, P, fluxua, fluxva, tps)
    S["fluxua"], S["fluxva"], S["tps"] = fluxua, fluxva, tps
    S["adx2d"] = S["adx2d"] - S["advua"]
    S["ady2d"] = S["ady2d"] - S["advva"]

    S["egf"] = S["el"] * P.ispi
    d_baro = S["h"] + S["elb"]
    d = S["d"]
    utf = S["utf"].copy()
    vtf = S["vtf"].copy()
    utf[1:im, :] = S["ua"][1:im, :] * (d[1:im, :] + d[0:im - 1, :]) * P.isp2i
    vtf[:, 1:jm] = S["va"][:, 1:jm] * (d[:, 1:jm] + d[:, 0:jm - 1]) * P.isp2i
    S["utf"], S["vtf"] = utf, vtf

    us, vs, den_u, den_v = barotropic_predictor(S, P)
    F = {"uaf": us, "vaf": vs}
    bcond_implicit(S, P, 2, F)
    us, vs = F["uaf"], F["vaf"]
    periodic_fill(S, P, us, vs)  # A3 (den_u, den_v: interior arrays, pointwise)
    S["fluxua"], S["fluxva"], rhs = barotropic_rhs(S, P, us, vs)
    prev = S.get("_eta_prev")
    x0 = 2.0 * S["elf"] - prev if prev is not None else S["elf"]
    elf, its = pcg_solve(rhs, S["d"], x0, S, P, C, SC, int(P.eta_solver_max_iter), float(P.eta_solver_tol),
                         float(P.eta_solver_rel_tol), P.eta_solver_preconditioner, dot_dtype=dot_dtype,
                         periodic=bool(getattr(P, "periodic_x", False)))
    elf = barotropic_shapiro(elf, S, float(P.barotropic_shapiro))
    F = {"elf": elf}
    bcond_implicit(S, P, 1, F)
    S["elf"] = F["elf"]
    S["d"] = S["h"] + S["elf"]
    periodic_fill(S, P)  # the η-solve
    ui, vi = barotropic_corrector(S, P, us, vs, den_u, den_v)
    uaf, vaf = S["uaf"].copy(), S["vaf"].copy()
    uaf[1:im - 1, 1:jm - 1] = ui
    vaf[1:im - 1, 1:jm - 1] = vi
    F = {"uaf": uaf, "vaf": vaf}
    bcond_implicit(S, P, 2, F)
    S["uaf"], S["vaf"] = F["uaf"], F["vaf"]
    S["etf"] = S["elf"] * S["fsm"]
    vamax = float(np.max(np.abs(S["vaf"])))
    ok = vamax <= P.vmaxl
    if ok:
        S["ua"] = S["ua"] + 0.5 * P.smoth * (S["uab"] - 2.0 * S["ua"] + S["uaf"])
        S["va"] = S["va"] + 0.5 * P.smoth * (S["vab"] - 2.0 * S["va"] + S["vaf"])
        S["el"] = S["el"] + 0.5 * P.smoth * (S["elb"] - 2.0 * S["el"] + S["elf"])
        S["elb"] = S["el"].copy()
        S["el"] = S["elf"].copy()
        S["d"] = S["h"] + S["el"]
        S["uab"] = S["ua"].copy()
        S["ua"] = S["uaf"].copy()
        S["vab"] = S["va"].copy()
        S["va"] = S["vaf"].copy()
        S["egf"] = (S["elb"] + S["el"]) * 0.5
        d = S["d"]
        c = 0.25
        utf = S["utf"].copy()
        vtf = S["vtf"].copy()
        utf[1:im, :] = c * (S["uab"][1:im, :] * (d_baro[1:im, :] + d_baro[0:im - 1, :]) + S["ua"][1:im, :] * (d[1:im, :] + d[0:im - 1, :]))
        vtf[:, 1:jm] = c * (S["vab"][:, 1:jm] * (d_baro[:, 1:jm] + d_baro[:, 0:jm - 1]) + S["va"][:, 1:jm] * (d[:, 1:jm] + d[:, 0:jm - 1]))
        S["utf"], S["vtf"] = utf, vtf
    periodic_fill(S, P)  # I5

    if ok and (iint != 1 or P.time0 != 0.0) and P.mode != 2:
        _barotropic_fix(S, P)
        periodic_fill(S, P)  # B1
        S["w"] = vertvl(S, P)
        F = {"w": S["w"]}
        bcond_implicit(S, P, 5, F)
        S["w"] = F["w"]
        periodic_fill(S, P)  # B2A
        uf = advq(S, P, S["q2b"], S["q2"], np.zeros_like(S["u"]))
        vf = advq(S, P, S["q2lb"], S["q2l"], np.zeros_like(S["u"]))
        S["uf"], S["vf"] = uf, vf
        periodic_fill(S, P)  # B2B
        if getattr(P, "profq_form", "production") == "pom08":
            R = profq_pom08(S, P, uf, vf)
            S["q2b"], S["q2lb"] = R["q2b"], R["q2lb"]
        else:
            R = profq(S, P, uf, vf, implicit_variant=True)
        S["l"], S["kq"], S["km"], S["kh"] = R["l"], R["kq"], R["km"], R["kh"]
        S["dtef"] = R["cc"]
        S["uf"], S["vf"] = R["uf"], R["vf"]
        periodic_fill(S, P)  # B3
        F = {"uf": S["uf"], "vf": S["vf"]}
        bcond_implicit(S, P, 6, F)
        S["uf"], S["vf"] = F["uf"], F["vf"]
        periodic_fill(S, P)  # B4
        q2 = S["q2"] + 0.5 * P.smoth * (S["uf"] + S["q2b"] - 2.0 * S["q2"])
        q2l = S["q2l"] + 0.5 * P.smoth * (S["vf"] + S["q2lb"] - 2.0 * S["q2l"])
        S["q2b"], S["q2"], S["q2lb"], S["q2l"] = q2, S["uf"].copy(), q2l, S["vf"].copy()
        vmix = getattr(P, "vertical_mixing_max", None)
        if vmix is not None:
            for n in ("kh", "km", "kq"):
                S[n] = np.clip(S[n], 0.0, float(vmix))
        if P.mode != 4:
            S["tb"], S["t"], uf = advt1(S, P, S["tb"], S["t"], S["tclim"])
            S["sb"], S["s"], vf = advt1(S, P, S["sb"], S["s"], S["sclim"])
            periodic_fill(S, P, uf, vf)  # B5
            uf, _ = proft(uf, S["wtsurf"], S["tsurf"], P.nbct, S["h"], S["etf"], P.dti2, S["dz"], S["dzz"],
                          S["swrad"], P.ntp, S["kh"], P.umol, S["z"])
            vf, dh = proft(vf, S["wssurf"], S["ssurf"], P.nbcs, S["h"], S["etf"], P.dti2, S["dz"], S["dzz"],
                           S["swrad"], P.ntp, S["kh"], P.umol, S["z"])
            S["tps"] = dh
            periodic_fill(S, P, uf, vf)  # B6
            F = {"uf": uf, "vf": vf}
            bcond_implicit(S, P, 4, F)
            uf, vf = F["uf"], F["vf"]
            t = S["t"] + 0.5 * P.smoth * (uf + S["tb"] - 2.0 * S["t"])
            s = S["s"] + 0.5 * P.smoth * (vf + S["sb"] - 2.0 * S["s"])
            gamma = float(P.tracer_shapiro)
            ts, ss = uf.copy(), vf.copy()
            if gamma > 0.0:
                I, J, K = slice(1, im - 1), slice(1, jm - 1), slice(0, kbm1)
                for src, dst in ((uf, ts), (vf, ss)):
                    dst[I, J, K] = src[I, J, K] + (gamma / 4.0) * (src[2:im, J, K] + src[0:im - 2, J, K] + src[I, 2:jm, K] + src[I, 0:jm - 2, K] - 4.0 * src[I, J, K])
            uf, vf = ts * _b(S["fsm"]), ss * _b(S["fsm"])
            S["uf"], S["vf"] = uf, vf
            S["tb"], S["t"], S["sb"], S["s"] = t, uf.copy(), s, vf.copy()
            S["rho"] = dens(S, P)
            periodic_fill(S, P)  # B7
        S["uf"] = advu(S, P)
        S["vf"] = advv(S, P)
        S["uf"], S["wubot"], _ = profuv(S, P, "u")
        S["vf"], S["wvbot"], S["tps"] = profuv(S, P, "v")
        F = {"uf": S["uf"], "vf": S["vf"]}
        bcond_implicit(S, P, 3, F)
        S["uf"], S["vf"] = F["uf"], F["vf"]
        periodic_fill(S, P)  # B8
        _internal_velocity_filter(S, P, shapiro=float(P.velocity_shapiro))

    S["egb"] = S["egf"].copy()
    S["etb"] = S["et"].copy()
    S["et"] = S["etf"].copy()
    S["dt"] = S["h"] + S["et"]
    S["utb"] = S["utf"].copy()
    S["vtb"] = S["vtf"].copy()
    S["vfluxb"] = S["vfluxf"].copy()
    periodic_fill(S, P)  # B9
    if vamax > P.vmaxl:
        raise VmaxExceeded(f"Barotropic velocity {vamax} exceeds limit {P.vmaxl} at time {P.time}")
    return its


def run(S, P, steps, core):
    """Advance ``steps`` internal steps from the current clock, as
    ``SparsePhysics.advance`` does (``hybrid/sparse_physics.py:193-206``):
    time0 = time, iint restarts at 0.  Returns PCG iterations per step for
    the implicit core."""
    P.time0 = float(P.time)
    P.iint = 0
    hist = []
    for _ in range(steps):
        if core == "explicit":
            step_explicit(S, P)
        else:
            hist.append(step_implicit(S, P))
    return hist
