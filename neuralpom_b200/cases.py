"""Initial states of the cores (set-up, not the timed step).

``double_gyre`` rebuilds the reference's production case
(``cores/explicit/cases.py:30-164`` + ``initialization.py:10-99``) in numpy
float32, so a core can be created without the reference package.  The
synthetic workloads (``seamount``, ``noise_basin``) follow the recipes of the
benchmark configurations: a closed 90x82x16 basin with a Gaussian seamount
for the semi-implicit core, and a 64x64x16 noisy-bathymetry double gyre for
the explicit core.

Every builder returns ``(arrays, scalars)``: float32 arrays keyed by the
reference attribute names and the scalar attributes of the core.
"""
from __future__ import annotations

import math

import numpy as np

from . import _abi, state

F32 = np.float32


def _zeros(im, jm, kb):
    return {n: np.zeros(_abi.field_shape(n, im, jm, kb), F32) for n in _abi.FIELD_NAMES}


def sigma_levels(kb):
    """Uniform sigma levels (cases.py:76-87): z, zz, dz, dzz ('Approx')."""
    z = np.array([-float(k) / float(kb - 1) for k in range(kb)], F32)
    dz = np.zeros(kb, F32)
    zz = np.zeros(kb, F32)
    for k in range(kb - 1):
        dz[k] = z[k] - z[k + 1]
        zz[k] = F32(0.5) * (z[k] + z[k + 1])
    dzz = dz.copy()
    dz[kb - 1] = 0.0
    dzz[kb - 1] = 0.0
    zz[kb - 1] = F32(2.0) * zz[kb - 2] - zz[kb - 3]
    return z, zz, dz, dzz


def areas_masks(A):
    """grid.py:113-166: art, aru, arv, fsm (h > 1), dum, dvm."""
    dx, dy, h = A["dx"], A["dy"], A["h"]
    A["art"] = dx * dy
    aru = np.zeros_like(dx)
    arv = np.zeros_like(dx)
    aru[1:, 1:] = 0.25 * (dx[1:, 1:] + dx[:-1, 1:]) * (dy[1:, 1:] + dy[:-1, 1:])
    arv[1:, 1:] = 0.25 * (dx[1:, 1:] + dx[1:, :-1]) * (dy[1:, 1:] + dy[1:, :-1])
    aru[0, :] = aru[1, :]
    arv[0, :] = arv[1, :]
    aru[:, 0] = aru[:, 1]
    arv[:, 0] = arv[:, 1]
    A["aru"], A["arv"] = aru, arv
    fsm = np.where(h > 1.0, F32(1.0), F32(0.0)).astype(F32)
    dum = np.zeros_like(fsm)
    dvm = np.zeros_like(fsm)
    dum[1:, 1:] = fsm[1:, 1:] * fsm[:-1, 1:]
    dvm[1:, 1:] = fsm[1:, 1:] * fsm[1:, :-1]
    dum[0, :] = dum[1, :]
    dvm[0, :] = dvm[1, :]
    dum[:, 0] = dum[:, 1]
    dvm[:, 0] = dvm[:, 1]
    A["fsm"], A["dum"], A["dvm"] = fsm, dum, dvm


def dens_np(t, s, h, zz, fsm, s_):
    """Mellor (1991) EOS on levels < kb-1 (momentum.py:467-541)."""
    kbm1 = t.shape[2] - 1
    tr = t[:, :, :kbm1] + s_["tbias"]
    sr = s[:, :, :kbm1] + s_["sbias"]
    tr2 = tr * tr
    tr3 = tr2 * tr
    tr4 = tr3 * tr
    p = s_["grav"] * s_["rhoref"] * (-zz[:kbm1][None, None, :] * h[:, :, None]) * 1.0e-5
    rhor = -0.157406 + 6.793952e-2 * tr - 9.095290e-3 * tr2 + 1.001685e-4 * tr3 - 1.120083e-6 * tr4 + 6.536332e-9 * tr4 * tr
    rhor = rhor + (0.824493 - 4.0899e-3 * tr + 7.6438e-5 * tr2 - 8.2467e-7 * tr3 + 5.3875e-9 * tr4) * sr
    rhor = rhor + (-5.72466e-3 + 1.0227e-4 * tr - 1.6546e-6 * tr2) * np.power(np.maximum(np.abs(sr), 1e-8), 1.5)
    rhor = rhor + 4.8314e-4 * sr * sr
    cr = 1449.1 + 0.0821 * p + 4.55 * tr - 0.045 * tr2 + 1.34 * (sr - 35.0)
    cr2 = cr * cr
    rhor = rhor + (1.0e5 * p / cr2) * (1.0 - 2.0 * p / cr2)
    out = np.zeros_like(t)
    out[:, :, :kbm1] = (rhor / s_["rhoref"]) * fsm[:, :, None]
    return out.astype(F32)


def finish_initialization(A, s, core):
    """run_initialization (initialization.py:10-99) after the case set-up:
    clocks, d/dt, turbulence fields, the rest state of u/v/t/s, EOS, cbc and
    the CFL field tps.  (BAROPG at ramp 0 gives drhox = drhoy = 0.)"""
    im, jm, kb = A["u"].shape
    kbm1 = kb - 1
    mid_i, mid_j = im // 2, jm // 2
    cor_val = np.abs(A["cor"][mid_i, mid_j]) + F32(1e-20)
    A["period"] = np.asarray(F32(2.0 * s["pi"]) / cor_val / F32(86400.0), F32)
    s["period"] = float(A["period"])
    s["time0"] = 0.0
    s["time"] = 0.0
    A["ua"] = A["uab"].copy()
    A["va"] = A["vab"].copy()
    A["el"] = A["elb"].copy()
    A["et"] = A["etb"].copy()
    A["etf"] = A["et"].copy()
    A["d"] = A["h"] + A["el"]
    A["dt"] = A["h"] + A["et"]
    A["w"][:, :, 0] = A["vfluxf"]
    l = np.broadcast_to((F32(0.1) * A["dt"])[:, :, None], (im, jm, kb)).astype(F32)
    A["l"] = l.copy()
    q2b_val = F32(s.get("q2_init", s["small"]))
    A["q2b"] = np.full((im, jm, kb), q2b_val, F32)
    A["q2lb"] = (l * A["q2b"]).astype(F32)
    A["kh"] = (l * np.sqrt(A["q2b"] + F32(1e-8))).astype(F32)
    A["km"] = A["kh"].copy()
    A["kq"] = A["kh"].copy()
    A["aam"] = np.full((im, jm, kb), F32(s["aam_init"]), F32)
    for dst, src in (("q2", "q2b"), ("q2l", "q2lb"), ("t", "tb"), ("s", "sb"), ("u", "ub"), ("v", "vb")):
        A[dst][:, :, :kbm1] = A[src][:, :, :kbm1]
    A["rho"] = dens_np(A["t"], A["s"], A["h"], A["zz"], A["fsm"], s)
    A["drhox"][:] = 0.0
    A["drhoy"][:] = 0.0
    zz_val = A["zz"][kbm1 - 1]
    term = np.maximum((F32(1.0) + zz_val) * A["h"] / F32(s["z0b"]), F32(1e-12))
    raw = np.square(F32(s["kappa"]) / np.log(term))
    A["cbc"] = np.clip(raw, F32(s["cbcmin"]), F32(s["cbcmax"])).astype(F32)
    dxs = np.maximum(A["dx"], F32(1e-6))
    dys = np.maximum(A["dy"], F32(1e-6))
    geom = np.sqrt(F32(1.0) / (dxs * dxs) + F32(1.0) / (dys * dys))
    gt = np.sqrt(F32(s["grav"]) * (A["h"] + F32(s["small"])))
    A["tps"] = ((F32(0.5) / geom) / gt * A["fsm"]).astype(F32)
    for k in list(A):
        A[k] = np.ascontiguousarray(A[k], dtype=F32) if np.ndim(A[k]) else np.asarray(A[k], F32)
    return A, s


def _vertical_interp(z_src, val_src, z_dst):
    """cases.py:10-28 (descending source profile, torch.bucketize)."""
    zf = z_src[::-1].copy()
    vf = val_src[::-1].copy()
    idx = np.searchsorted(zf, z_dst, side="left")
    idx = np.clip(idx, 1, z_src.shape[0] - 1)
    z0, z1, v0, v1 = zf[idx - 1], zf[idx], vf[idx - 1], vf[idx]
    den = z1 - z0
    den = np.where(np.abs(den) < 1e-6, F32(1.0), den)
    wgt = (z_dst - z0) / den
    return (v0 * (F32(1.0) - wgt) + v1 * wgt).astype(F32)


def double_gyre(im, jm, core="implicit_p0_fixed", kb=16):
    """The reference's production double gyre (cases.py:30-164) followed by
    run_initialization, with the production clock of core_spec."""
    s = state.default_scalars(core)
    A = _zeros(im, jm, kb)
    deg2rad = s["pi"] / 180.0
    re, omega = 6371.0e3, 7.2921e-5
    dlat = (50.0 - 30.0) / float(jm - 2)
    dlon = (22.0 - 0.0) / float(im - 2)
    j_idx = np.broadcast_to(np.arange(jm, dtype=F32)[None, :], (im, jm))
    i_idx = np.broadcast_to(np.arange(im, dtype=F32)[:, None], (im, jm))
    A["north_e"] = (30.0 + (j_idx - F32(1.0)) * F32(dlat)).astype(F32)
    A["dy"] = np.full((im, jm), F32(re * dlat * deg2rad), F32)
    A["dx"] = (F32(re) * np.cos(A["north_e"] * F32(deg2rad)) * F32(dlon) * F32(deg2rad)).astype(F32)
    A["cor"] = (F32(2.0 * omega) * np.sin(A["north_e"] * F32(deg2rad))).astype(F32)
    _ = i_idx
    h = np.full((im, jm), F32(2500.0), F32)
    h[0, :] = 1.0
    h[im - 1, :] = 1.0
    h[:, 0] = 1.0
    h[:, jm - 1] = 1.0
    A["h"] = h
    hmax_real = float(h.max())
    A["z"], A["zz"], A["dz"], A["dzz"] = sigma_levels(kb)
    areas_masks(A)
    A["sb"][:] = 35.0
    z_ref = np.linspace(0, -(hmax_real + 100.0), 1000, dtype=F32)
    t_ref = (F32(2.0) + F32(30.0 - 2.0) * np.exp(z_ref / F32(800.0))).astype(F32)
    depths = (A["z"][None, None, :] * h[:, :, None]).astype(F32)
    A["tb"] = _vertical_interp(z_ref, t_ref, depths)
    A["tclim"] = A["tb"].copy()
    A["sclim"] = A["sb"].copy()
    # the reference evaluates DENS here on the still-zero t/s (cases.py:132)
    A["rho"] = dens_np(A["t"], A["s"], h, A["zz"], A["fsm"], s)
    A["rmean"] = A["rho"].copy()
    kf = 0.1 / s["rhoref"]
    arg = F32(2.0 * s["pi"]) * (A["north_e"] - F32(30.0)) / F32(20.0)
    A["wusurf"] = (F32(-kf) * (F32(1.0) - np.cos(arg)) * A["dum"]).astype(F32)
    s["horcon"] = 0.05
    return finish_initialization(A, s, core)


def _noise(shape, sigma, seed):
    from scipy.ndimage import gaussian_filter
    g = np.random.default_rng(seed)
    n = gaussian_filter(g.standard_normal(shape), sigma, mode="reflect")
    return n / np.max(np.abs(n))


def _with_profile(A, s, t_of_z, salinity):
    im, jm, kb = A["u"].shape
    depths = (A["z"][None, None, :] * A["h"][:, :, None]).astype(F32)
    A["tb"] = t_of_z(depths).astype(F32)
    A["sb"][:] = F32(salinity)
    A["tclim"] = A["tb"].copy()
    A["sclim"] = A["sb"].copy()
    A["rho"] = dens_np(A["tb"], A["sb"], A["h"], A["zz"], A["fsm"], s)
    A["rmean"] = A["rho"].copy()


def seamount(im=90, jm=82, kb=16, dti=300.0, isplit=30, dx=5.0e3, u0=0.1, eta_tol=1e-10, periodic_x=False):
    """Semi-implicit benchmark basin: flat 4500 m bottom with a Gaussian
    seamount (height 4000 m, e-folding 25 km) at the centre, dx = dy = 5 km,
    closed walls (the reference's ClosedBasinBoundary), f-plane at 40N,
    T = 10 + 10 exp(z/1000 m), S = 35, uniform initial inflow u0, no wind.

    periodic_x: a channel periodic in x with walls in y instead (the
    reference has no periodic boundary).  The unique columns are 2..im-3
    (period (im-4) dx); columns 0, 1 and im-2, im-1 are halo copies
    (``wrap_x``); the seamount sits at the centre of the unique columns
    with its distance measured to the nearest periodic image; the η-solve's
    spectral preconditioner is Hartley along x times DST-I along y."""
    core = "implicit_p0_fixed"
    s = state.default_scalars(core)
    s.update(dte=dti / isplit, isplit=isplit)
    state.derived_time(s)
    s.update(eta_solver_tol=eta_tol, eta_solver_rel_tol=eta_tol, double_gyre_wind_stress_pa=0.0, hmax=4500.0)
    A = _zeros(im, jm, kb)
    A["dx"][:] = dx
    A["dy"][:] = dx
    A["north_e"][:] = 40.0
    A["cor"][:] = F32(2.0 * 7.2921e-5 * math.sin(math.radians(40.0)))
    y = (np.arange(jm, dtype=np.float64) - (jm - 1) / 2.0) * dx
    if periodic_x:
        period = (im - 4) * dx
        x = (np.arange(im, dtype=np.float64) - 2.0 - (im - 5) / 2.0) * dx
        x = x - period * np.round(x / period)
    else:
        x = (np.arange(im, dtype=np.float64) - (im - 1) / 2.0) * dx
    r2 = x[:, None] ** 2 + y[None, :] ** 2
    h = (4500.0 - 4000.0 * np.exp(-r2 / (25.0e3 ** 2))).astype(F32)
    if not periodic_x:
        h[0, :] = 1.0
        h[-1, :] = 1.0
    h[:, 0] = 1.0
    h[:, -1] = 1.0
    A["h"] = h
    A["z"], A["zz"], A["dz"], A["dzz"] = sigma_levels(kb)
    if periodic_x:
        wrap_x(A["h"])
    areas_masks(A)
    if periodic_x:
        for n in ("aru", "arv", "fsm", "dum", "dvm"):
            wrap_x(A[n])
        s["periodic_x"] = True
    _with_profile(A, s, lambda z: 10.0 + 10.0 * np.exp(z / 1000.0), 35.0)
    A["ub"][:, :, : kb - 1] = F32(u0) * A["dum"][:, :, None]
    A["uab"][:] = F32(u0) * A["dum"]
    A, s = finish_initialization(A, s, core)
    if periodic_x:
        for n, a in A.items():
            if np.ndim(a) >= 2 and a.shape[:2] == (im, jm):
                wrap_x(a)
    return A, s


def seamount_channel(im=90, jm=82, kb=16, **kw):
    """The benchmark seamount as a channel periodic in x (walls in y):
    ``seamount(periodic_x=True)``; at 90x82 the unique columns are 2..87."""
    return seamount(im, jm, kb, periodic_x=True, **kw)


def wrap_x(a):
    """Halo columns of a periodic-x plane (i first), two on each side:
    columns 0, 1 take im-4, im-3 and columns im-2, im-1 take 2, 3.  A
    u-point column i is the west face of cell i, so the copy serves every
    staggering."""
    n = a.shape[0]
    a[0] = a[n - 4]
    a[1] = a[n - 3]
    a[n - 2] = a[2]
    a[n - 1] = a[3]


def noise_basin(im=64, jm=64, kb=16, dte=6.0, isplit=30, dx=20.0e3, seed=0, core="explicit"):
    """Explicit benchmark basin: closed 64x64 cells, dx = dy = 20 km,
    h = 4000 - 500 n (n: seeded Gaussian-filtered noise, sigma 4 cells,
    max |n| = 1), tau_x = -0.1 cos(2 pi y / Ly) N/m2, T = 5 + 15 exp(z/800 m),
    S = 35, q2 = q2l = 1e-8, the reference's latitude/Coriolis formula."""
    s = state.default_scalars(core)
    s.update(dte=dte, isplit=isplit, hmax=4500.0, q2_init=1e-8)
    state.derived_time(s)
    A = _zeros(im, jm, kb)
    A["dx"][:] = dx
    A["dy"][:] = dx
    dlat = (50.0 - 30.0) / float(jm - 2)
    A["north_e"] = np.broadcast_to((30.0 + (np.arange(jm) - 1.0) * dlat).astype(F32)[None, :], (im, jm)).astype(F32)
    A["cor"] = (F32(2.0 * 7.2921e-5) * np.sin(A["north_e"] * F32(math.pi / 180.0))).astype(F32)
    h = (4000.0 - 500.0 * _noise((im, jm), 4.0, seed)).astype(F32)
    h[0, :] = 1.0
    h[-1, :] = 1.0
    h[:, 0] = 1.0
    h[:, -1] = 1.0
    A["h"] = h
    A["z"], A["zz"], A["dz"], A["dzz"] = sigma_levels(kb)
    areas_masks(A)
    _with_profile(A, s, lambda z: 5.0 + 15.0 * np.exp(z / 800.0), 35.0)
    ly = dx * (jm - 2)
    y = (np.arange(jm, dtype=np.float64) - 1.0) * dx
    taux = -0.1 * np.cos(2.0 * np.pi * y / ly)
    A["wusurf"] = (np.broadcast_to((-taux / s["rhoref"]).astype(F32)[None, :], (im, jm)) * A["dum"]).astype(F32)
    if core != "explicit":
        s["wind_forcing"] = False
    return finish_initialization(A, s, core)


def tide_elevation(time_days, amplitude=1.0, period_h=12.42):
    """M2 boundary elevation a cos(2 pi t / T) at time t (days)."""
    return float(amplitude * math.cos(2.0 * math.pi * time_days * 24.0 / period_h))


def coastal_tide(im=354, jm=322, kb=16, dte=2.0, isplit=30, dx=500.0, seed=4, land_fraction=0.35,
                 amplitude=1.0, lat=30.0):
    """Coastal basin for the explicit core with one open boundary: dx = dy =
    500 m; land where seeded Gaussian-filtered noise (sigma 12 cells) is
    below its land_fraction quantile (h = 1, so fsm = 0); water depth 2 m at
    the coast growing to 60 m with the distance from it; west, east and
    north edges closed; the south edge open through the explicit core's
    Flather condition (rfs = 1) with the M2 elevation els = amplitude at
    t = 0 (``tide_elevation`` gives it at later times); T = 15 degC,
    S = 31 psu + 1 psu per 10 m of depth, no wind, f-plane at ``lat``."""
    from scipy.ndimage import distance_transform_edt
    core = "explicit"
    s = state.default_scalars(core)
    s.update(dte=dte, isplit=isplit, hmax=60.0, rfs=1.0)
    state.derived_time(s)
    A = _zeros(im, jm, kb)
    A["dx"][:] = dx
    A["dy"][:] = dx
    A["north_e"][:] = lat
    A["cor"][:] = F32(2.0 * 7.2921e-5 * math.sin(math.radians(lat)))
    n = _noise((im, jm), 12.0, seed)
    land = n < np.quantile(n, land_fraction)
    land[0, :] = True
    land[-1, :] = True
    land[:, -1] = True
    land[:, 0] = land[:, 1]          # the open row continues the first interior row
    water = ~land
    dist = distance_transform_edt(water)
    h = np.where(water, 2.0 + 58.0 * np.minimum(dist / max(float(dist[water].max()), 1.0), 1.0), 1.0)
    A["h"] = h.astype(F32)
    A["z"], A["zz"], A["dz"], A["dzz"] = sigma_levels(kb)
    areas_masks(A)
    depths = (A["z"][None, None, :] * A["h"][:, :, None]).astype(F32)
    A["tb"][:] = F32(15.0)
    A["sb"] = (F32(31.0) - F32(0.1) * depths).astype(F32)
    A["tclim"] = A["tb"].copy()
    A["sclim"] = A["sb"].copy()
    A["rho"] = dens_np(A["tb"], A["sb"], A["h"], A["zz"], A["fsm"], s)
    A["rmean"] = A["rho"].copy()
    A["els"][:] = F32(amplitude)
    A["tbs"] = A["tb"][:, 0, :].copy()
    A["sbs"] = A["sb"][:, 0, :].copy()
    return finish_initialization(A, s, core)


def seamount_policy(A, s, core="explicit"):
    """The seamount case policy's set-up on a state (cores/case_adapters/
    seamount_runtime.py:6-25): the exterior elevations, transports and T/S
    profiles taken from the current state's edge rows and columns, rf = 1,
    alpha and smoth of the explicit core, the POM08-WAD closure (zsh =
    0.01 m) and the seamount boundary (``obc_form``)."""
    A = dict(A)
    A["uabe"], A["uabw"] = A["uab"][-2, :].copy(), A["uab"][1, :].copy()
    A["vabn"], A["vabs"] = A["va"][:, -2].copy(), A["va"][:, 1].copy()
    A["ele"], A["elw"] = A["el"][-1, :].copy(), A["el"][0, :].copy()
    A["eln"], A["els"] = A["el"][:, -1].copy(), A["el"][:, 0].copy()
    for key, name, axis, index in (("tbe", "t", 0, -1), ("tbw", "t", 0, 0), ("sbe", "s", 0, -1), ("sbw", "s", 0, 0),
                                   ("tbn", "t", 1, -1), ("tbs", "t", 1, 0), ("sbn", "s", 1, -1), ("sbs", "s", 1, 0)):
        A[key] = np.ascontiguousarray(A[name][index, :, :] if axis == 0 else A[name][:, index, :]).copy()
    alpha, smoth = (0.225, 0.1) if core == "explicit" else (0.333, 0.15)
    s = dict(s, rfe=1.0, rfw=1.0, rfn=1.0, rfs=1.0, alpha=alpha, smoth=smoth, profq_form="pom08", zsh=0.01,
             obc_form="seamount")
    return A, s


def open_seamount(im=65, jm=49, kb=16, dte=5.0, isplit=30, dx=5.0e3, u0=0.1, lat=40.0, core="explicit"):
    """Explicit seamount with open east and west edges, the geometry the
    seamount case policy serves (registered at 65x49x16 with dtE/dtI = 5/150
    s): flat 4500 m with a Gaussian seamount (height 4000 m, e-folding 25
    km) at the centre, dx = dy, walls on the north and south edges, water
    on the east and west edges, T = 10 + 10 exp(z/1000 m), S = 35, uniform
    inflow u0, f-plane at ``lat``, no wind; with ``seamount_policy``
    applied.  ``core`` "implicit_p0_fixed" gives the semi-implicit core's
    scalars (dti = dte * isplit)."""
    s = state.default_scalars(core)
    s.update(dte=dte, isplit=isplit, hmax=4500.0)
    state.derived_time(s)
    A = _zeros(im, jm, kb)
    A["dx"][:] = dx
    A["dy"][:] = dx
    A["north_e"][:] = lat
    A["cor"][:] = F32(2.0 * 7.2921e-5 * math.sin(math.radians(lat)))
    x = (np.arange(im, dtype=np.float64) - (im - 1) / 2.0) * dx
    y = (np.arange(jm, dtype=np.float64) - (jm - 1) / 2.0) * dx
    r2 = x[:, None] ** 2 + y[None, :] ** 2
    h = (4500.0 - 4000.0 * np.exp(-r2 / (25.0e3 ** 2))).astype(F32)
    h[:, 0] = 1.0
    h[:, -1] = 1.0
    A["h"] = h
    A["z"], A["zz"], A["dz"], A["dzz"] = sigma_levels(kb)
    areas_masks(A)
    _with_profile(A, s, lambda z: 10.0 + 10.0 * np.exp(z / 1000.0), 35.0)
    A["ub"][:, :, : kb - 1] = F32(u0) * A["dum"][:, :, None]
    A["uab"][:] = F32(u0) * A["dum"]
    A, s = finish_initialization(A, s, core)
    return seamount_policy(A, s, core=core)


def coastal_policy(A, s, tide_i, tide_j, tide_amp, tide_phase, core="explicit"):
    """The coastal tide policy's set-up on a state (cores/case_adapters/
    coastal_boundary.py:55-65 and coastal_compat.py:12-23, registry.py:
    137-138): the tide table (0-based cells, amplitude in m, phase in
    degrees), rf = 1, alpha and smoth of the core (0.225 / 0.1 explicit,
    0.333 / 0.15 semi-implicit), the POM08-WAD closure (zsh = 0.01 m) and
    the coastal boundary (``obc_form``)."""
    A = dict(A)
    A["tide_i"] = np.asarray(tide_i, F32)
    A["tide_j"] = np.asarray(tide_j, F32)
    A["tide_amp"] = np.asarray(tide_amp, F32)
    A["tide_phase"] = np.asarray(tide_phase, F32)
    alpha, smoth = (0.225, 0.1) if core == "explicit" else (0.333, 0.15)
    s = dict(s, rfe=1.0, rfw=1.0, rfn=1.0, rfs=1.0, alpha=alpha, smoth=smoth, profq_form="pom08", zsh=0.01,
             obc_form="coastal")
    return A, s


def tidal_inlet(im=40, jm=30, kb=5, dte=1.0, isplit=10, dx=500.0, lat=30.0, amplitude=1.0, core="explicit"):
    """The geometry the coastal tide policy serves (registered at 161x101x5,
    dtE/dtI = 1/10 s, from data that is not in the repository): a shelf
    closed on the west, north and south, depth 2 m at the west wall growing
    to 60 m at the open east edge, T = 15 degC, S = 31 psu + 1 psu per 10 m,
    f-plane at ``lat``, no wind; with ``coastal_policy`` applied and the
    tide table of the registered case's layout: every interior cell of the
    column next to the east edge, here with amplitude ``amplitude`` scaled
    by 0.8-1.0 along the column and a phase of 2 degrees per row.  ``core``
    "implicit_p0_fixed" gives the semi-implicit core's scalars (its
    dti = dte * isplit, the policy's own spatial filters off)."""
    s = state.default_scalars(core)
    s.update(dte=dte, isplit=isplit, hmax=60.0)
    state.derived_time(s)
    A = _zeros(im, jm, kb)
    A["dx"][:] = dx
    A["dy"][:] = dx
    A["north_e"][:] = lat
    A["cor"][:] = F32(2.0 * 7.2921e-5 * math.sin(math.radians(lat)))
    x = np.arange(im, dtype=np.float64) / (im - 1)
    h = np.broadcast_to((2.0 + 58.0 * x)[:, None], (im, jm)).astype(F32).copy()
    h[0, :] = 1.0
    h[:, 0] = 1.0
    h[:, -1] = 1.0
    A["h"] = h
    A["z"], A["zz"], A["dz"], A["dzz"] = sigma_levels(kb)
    areas_masks(A)
    depths = (A["z"][None, None, :] * A["h"][:, :, None]).astype(F32)
    A["tb"][:] = F32(15.0)
    A["sb"] = (F32(31.0) - F32(0.1) * depths).astype(F32)
    A["tclim"] = A["tb"].copy()
    A["sclim"] = A["sb"].copy()
    A["rho"] = dens_np(A["tb"], A["sb"], A["h"], A["zz"], A["fsm"], s)
    A["rmean"] = A["rho"].copy()
    A, s = finish_initialization(A, s, core)
    rows = np.arange(1, jm - 1)
    amp = amplitude * (0.8 + 0.2 * rows / max(jm - 2, 1))
    return coastal_policy(A, s, np.full(rows.shape, im - 2), rows, amp, 2.0 * rows, core=core)


def jzb_policy(A, s, tide_i, tide_j, tide_amp, tide_phase, core="explicit"):
    """The Jiaozhou Bay tide policy's set-up on a state
    (cores/case_adapters/jzb_boundary.py:200-215 and jzb_compat.py:30-70):
    the tide table (0-based cells, amplitude in m, phase in degrees), rf = 1,
    alpha and smoth of the explicit core, the bay's settings (mode 4, a
    3-day ramp, horcon 0.1, hmax 60 m, tprni 0.2, umol 2e-5), the POM08-WAD
    closure (zsh = 0.01 m) and the bay's boundary (``obc_form``)."""
    A = dict(A)
    A["tide_i"] = np.asarray(tide_i, F32)
    A["tide_j"] = np.asarray(tide_j, F32)
    A["tide_amp"] = np.asarray(tide_amp, F32)
    A["tide_phase"] = np.asarray(tide_phase, F32)
    A["period"] = np.asarray(F32(3.0))
    alpha, smoth = (0.225, 0.1) if core == "explicit" else (0.333, 0.15)
    s = dict(s, rfe=1.0, rfw=1.0, rfn=1.0, rfs=1.0, alpha=alpha, smoth=smoth, profq_form="pom08", zsh=0.01,
             obc_form="jzb", mode=4, lramp=True, period=3.0, horcon=0.1, hmax=60.0, tprni=0.2, umol=2.0e-5)
    return A, s


def bay(im=40, jm=30, kb=16, dte=1.0, isplit=10, dx=500.0, lat=36.0, amplitude=1.0, core="explicit"):
    """The geometry the Jiaozhou Bay policy serves (registered at 312x213x17,
    dtE/dtI = 1/10 s, from data that is not in the repository): a bay closed
    on the west, east and north, open to the sea on the south edge, depth 2 m
    at the head growing to 40 m at the mouth, T = 15 degC, S = 31 psu + 1 psu
    per 10 m, f-plane at ``lat``, no wind, horizontal viscosity 50 m^2/s at
    rest; with ``jzb_policy`` applied and a tide table of the registered
    layout: every interior cell of the row next to the open edge, with
    amplitude ``amplitude`` scaled by 0.8-1.0 along the row and a phase of
    1.5 degrees per column.  ``core`` "implicit_p0_fixed" gives the
    semi-implicit core's scalars."""
    s = state.default_scalars(core)
    s.update(dte=dte, isplit=isplit, hmax=60.0, aam_init=50.0)
    state.derived_time(s)
    A = _zeros(im, jm, kb)
    A["dx"][:] = dx
    A["dy"][:] = dx
    A["north_e"][:] = lat
    A["cor"][:] = F32(2.0 * 7.2921e-5 * math.sin(math.radians(lat)))
    y = np.arange(jm, dtype=np.float64) / (jm - 1)
    h = np.broadcast_to((40.0 - 38.0 * y)[None, :], (im, jm)).astype(F32).copy()
    h[0, :] = 1.0
    h[-1, :] = 1.0
    h[:, -1] = 1.0
    A["h"] = h
    A["z"], A["zz"], A["dz"], A["dzz"] = sigma_levels(kb)
    areas_masks(A)
    depths = (A["z"][None, None, :] * A["h"][:, :, None]).astype(F32)
    A["tb"][:] = F32(15.0)
    A["sb"] = (F32(31.0) - F32(0.1) * depths).astype(F32)
    A["tclim"] = A["tb"].copy()
    A["sclim"] = A["sb"].copy()
    A["rho"] = dens_np(A["tb"], A["sb"], A["h"], A["zz"], A["fsm"], s)
    A["rmean"] = A["rho"].copy()
    A, s = finish_initialization(A, s, core)
    cols = np.arange(1, im - 1)
    amp = amplitude * (0.8 + 0.2 * cols / max(im - 2, 1))
    return jzb_policy(A, s, cols, np.full(cols.shape, 1), amp, 1.5 * cols, core=core)
