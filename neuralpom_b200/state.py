"""Scalar settings and solver caches of a core, shared by the torch host
layer (``core.py``) and the tests.

The scalar names are the reference core's Python attributes
(``src/neuralpom/cores/explicit/base.py:37-120`` and
``cores/implicit_p0_fixed/base.py``/``core.py:78-119``); the production
values are pinned by ``src/neuralpom/v1/core_spec.py:22-47``.
"""
from __future__ import annotations

import math

import numpy as np

from . import _abi

# Attributes of BaseCore (explicit/base.py) before any case or spec override.
BASE_SCALARS = dict(
    small=1e-9, pi=math.atan(1.0) * 4.0, mode=3, nadv=1, nitera=2, sw=0.5, lramp=True, rhoref=1035.0,
    hmax=2000.0, dte=30.0, isplit=30, grav=9.806, kappa=0.40, z0b=0.010, cbcmin=0.0025, cbcmax=1.0,
    horcon=0.20, tprni=0.20, umol=2e-5, vmaxl=100.0, slmax=2.0, ntp=2, nbct=1, nbcs=1, ispadv=5,
    tbias=0.0, sbias=0.0, rfe=0.0, rfw=0.0, rfn=0.0, rfs=0.0, ramp=0.0, aam_init=500.0,
)
EXPLICIT_DEFAULTS = dict(smoth=0.10, alpha=0.225)
IMPLICIT_DEFAULTS = dict(smoth=0.15, alpha=0.333, aam_min=0.0, eta_solver_rel_tol=1e-5,
                         eta_solver_preconditioner="spectral", eta_solver_max_iter=200,
                         eta_solver_tol=1.0e-12, barotropic_shapiro=0.0, tracer_shapiro=0.0,
                         velocity_shapiro=0.0)

# core_spec.py:42-47 production settings (dti=600, dte=20, isplit=30)
PRODUCTION = {
    "explicit": dict(dte=20.0, isplit=30, alpha=0.225, smoth=0.10, horcon=0.05),
    "implicit_p0_fixed": dict(dte=20.0, isplit=30, alpha=0.333, smoth=0.15, horcon=0.05,
                              eta_solver_rel_tol=1e-5, eta_solver_preconditioner="spectral",
                              barotropic_shapiro=0.0, tracer_shapiro=0.0, velocity_shapiro=0.0),
}


def derived_time(s):
    """base.py:111-120 derived clock values."""
    s["dti"] = s["dte"] * s["isplit"]
    s["dte2"] = s["dte"] * 2.0
    s["dti2"] = s["dti"] * 2.0
    s["ispi"] = 1.0 / s["isplit"]
    s["isp2i"] = 1.0 / (2.0 * s["isplit"])
    return s


def default_scalars(core):
    s = dict(BASE_SCALARS)
    s.update(EXPLICIT_DEFAULTS if core == "explicit" else IMPLICIT_DEFAULTS)
    s.update(PRODUCTION[core])
    return derived_time(s)


def host_array(v):
    """numpy copy of an array or a tensor (on any device)."""
    if hasattr(v, "detach"):
        return v.detach().cpu().numpy()
    return np.asarray(v)


def host_scalar(v):
    """float of a Python number or a one-element tensor.  A device tensor
    (the reference keeps ``period`` as one) is read back once and the value
    kept on the tensor with its version counter, so later reads (the step's
    host bookkeeping) do not wait for the work queued on the device; an
    in-place write to the tensor bumps the version and forces a new read."""
    if not hasattr(v, "detach"):
        return float(np.asarray(v, dtype=np.float64).reshape(-1)[0])
    hit = getattr(v, "_npom_host_value", None)
    if hit is not None and hit[0] == v._version:
        return hit[1]
    val = float(v.detach().reshape(-1)[0].cpu().item())
    try:
        v._npom_host_value = (v._version, val)
    except (AttributeError, RuntimeError):
        pass
    return val


def make_params(s, im, jm, kb, core, device=0):
    """npom_params from a mapping (or object) of the reference scalars."""
    get = (lambda k, d=None: s.get(k, d)) if isinstance(s, dict) else (lambda k, d=None: getattr(s, k, d))
    p = _abi.NpomParams()
    p.device = int(device)
    p.im, p.jm, p.kb = int(im), int(jm), int(kb)
    implicit = core != "explicit"
    p.core = _abi.CORE_IMPLICIT if implicit else _abi.CORE_EXPLICIT
    p.isplit = int(get("isplit"))
    p.ispadv = int(get("ispadv", 5))
    p.nbct, p.nbcs, p.ntp = int(get("nbct", 1)), int(get("nbcs", 1)), int(get("ntp", 2))
    p.mode, p.nadv = int(get("mode", 3)), int(get("nadv", 1))
    if p.nadv not in (1, 2):
        raise ValueError("tracer advection: nadv=1 (centred) or nadv=2 (MPDATA)")
    p.nitera, p.sw = int(get("nitera", 2)), float(get("sw", 0.5))
    if p.nitera < 1:
        raise ValueError("nitera must be positive")
    p.eta_max_iter = int(get("eta_solver_max_iter", 200) or 200)
    pre = str(get("eta_solver_preconditioner", "spectral") or "spectral").strip().lower()
    if implicit and pre not in ("spectral", "jacobi"):
        raise ValueError(f"unknown eta preconditioner {pre!r}")
    p.eta_precond = _abi.PRECOND_SPECTRAL if pre == "spectral" else _abi.PRECOND_JACOBI
    p.wind_forcing = 1 if (implicit and get("wind_forcing", True)) else 0
    vmix = get("vertical_mixing_max", None)
    p.has_vmix = 1 if vmix is not None else 0
    p.vmix = float(vmix) if vmix is not None else 0.0
    p.lramp = 1 if get("lramp", True) else 0
    for k in ("dti", "dte", "dti2", "dte2", "ispi", "isp2i", "alpha", "smoth", "horcon", "grav", "umol", "tprni",
              "small", "kappa", "rhoref", "tbias", "sbias", "vmaxl", "hmax", "rfe", "rfw", "rfn", "rfs", "pi"):
        setattr(p, k, float(get(k)))
    p.aam_min = float(get("aam_min", 0.0) or 0.0)
    p.eta_tol = float(get("eta_solver_tol", 1.0e-12))
    p.eta_rel_tol = float(get("eta_solver_rel_tol", 1e-5))
    p.barotropic_shapiro = float(get("barotropic_shapiro", 0.0) or 0.0)
    p.tracer_shapiro = float(get("tracer_shapiro", 0.0) or 0.0)
    p.velocity_shapiro = float(get("velocity_shapiro", 0.0) or 0.0)
    if p.velocity_shapiro != 0.0:
        raise ValueError("a non-zero internal-velocity Shapiro filter is not implemented (production uses 0)")
    tau0 = get("double_gyre_wind_stress_pa", None)
    p.wind_tau0 = 0.1 if tau0 is None else float(tau0)
    p.period = host_scalar(get("period", 1.0))
    p.inverse_scale = 4.0 * (im - 1) * (jm - 1)
    form = str(get("profq_form", "production") or "production").strip().lower()
    if form not in ("production", "pom08"):
        raise ValueError(f"unknown profq form {form!r} (production or pom08)")
    p.profq_form = _abi.PROFQ_POM08 if form == "pom08" else _abi.PROFQ_PRODUCTION
    p.zsh = float(get("zsh", 0.01))
    obc = str(get("obc_form", "native") or "native").strip().lower()
    if obc not in ("native", "seamount", "coastal", "jzb"):
        raise ValueError(f"unknown boundary policy {obc!r} (native, seamount, coastal or jzb)")
    if obc != "native" and implicit and float(get("barotropic_shapiro", 0.0) or 0.0) != 0.0:
        raise ValueError(f"the {obc} policy runs the semi-implicit core with its Shapiro filter off")
    p.obc_form = {"native": _abi.OBC_NATIVE, "seamount": _abi.OBC_SEAMOUNT, "coastal": _abi.OBC_COASTAL,
                  "jzb": _abi.OBC_JZB}[obc]
    # periodic x: two halo columns on each side, unique columns 2..im-3
    # (no counterpart in the reference, whose lateral boundaries are walls
    # and open edges)
    periodic = bool(get("periodic_x", False))
    if periodic:
        if not implicit:
            raise ValueError("periodic x is built for the semi-implicit core")
        if obc != "native" or int(p.nadv) != 1 or im < 8:
            raise ValueError("periodic x needs native boundaries, nadv 1 and im >= 8")
        # Hartley along the period (im-4 unique columns) times DST-I in y
        p.inverse_scale = 2.0 * (im - 4) * (jm - 1)
    p.periodic_x = 1 if periodic else 0
    tuning = get("tuning", None) or {}
    for k, v in dict(tuning).items():
        if k not in _abi.TUNING_FIELDS:
            raise ValueError(f"unknown tuning field {k!r}")
        setattr(p.tuning, k, int(v))
    return p


def spectral_setup(dx, dy, h, dti, grav, alpha, dtype=np.float32, periodic_x=False):
    """DST-I matrices and inverse eigenvalues of the spectral preconditioner
    (``implicit_p0_fixed/core.py:730-760``; torch.median picks the lower
    middle value).

    periodic_x (no counterpart in the reference): the rows are the n = im-4
    unique columns and Sx is the Hartley matrix cas(2 pi k m / n) =
    cos + sin, which is symmetric with Sx Sx = n I and diagonalises the
    periodic second difference with the eigenvalues 4 sin^2(pi k / n) --
    so z = Sx ((Sx r Sy) * inv_eigs) Sy / (2 n (nj + 1)) is the same
    symmetric two-sided product as the DST-I form.  The medians are taken
    over the unique columns."""
    im, jm = dx.shape
    rows = slice(2, im - 2) if periodic_x else slice(1, im - 1)
    ni, nj = (im - 4 if periodic_x else im - 2), jm - 2

    def tmedian(a):
        flat = np.sort(np.asarray(a, dtype=dtype).reshape(-1))
        return flat[(flat.size - 1) // 2]

    dx0, dy0, h0 = tmedian(dx[rows, 1:-1]), tmedian(dy[rows, 1:-1]), tmedian(h[rows, 1:-1])
    coeff = 4.0 * (dti ** 2) * grav * alpha
    ky = np.arange(1, nj + 1, dtype=dtype).reshape(1, -1)
    if periodic_x:
        kx = np.arange(0, ni, dtype=dtype).reshape(-1, 1)
        lam_x = 4.0 * np.square(np.sin(np.pi * kx / ni)) / (dx0 * dx0 + 1e-30)
    else:
        kx = np.arange(1, ni + 1, dtype=dtype).reshape(-1, 1)
        lam_x = 4.0 * np.square(np.sin(np.pi * kx / (2.0 * (ni + 1)))) / (dx0 * dx0 + 1e-30)
    lam_y = 4.0 * np.square(np.sin(np.pi * ky / (2.0 * (nj + 1)))) / (dy0 * dy0 + 1e-30)
    inv_eigs = (1.0 / (1.0 + coeff * h0 * (lam_x + lam_y))).astype(dtype)

    def sine(n):
        k = np.arange(1, n + 1, dtype=np.float64)
        return (2.0 * np.sin(np.pi * np.outer(k, k) / (n + 1))).astype(dtype)

    sx = hartley(ni, dtype) if periodic_x else sine(ni)
    return sx, sine(nj), np.ascontiguousarray(inv_eigs)


def hartley(n, dtype=np.float32):
    """The n x n Hartley matrix cas(2 pi k m / n) = cos + sin (symmetric,
    its square is n I)."""
    k = np.arange(n, dtype=np.float64)
    t = 2.0 * np.pi * np.outer(k, k) / n
    return (np.cos(t) + np.sin(t)).astype(dtype)


def fill_flat(buf, arr):
    """Write arr row-major into the first arr.size elements of the flat
    buffer buf (numpy array or torch tensor): the periodic-x preconditioner
    arrays are smaller than the workspace planes sized for the interior."""
    n = int(np.asarray(arr).size)
    if hasattr(buf, "view") and not isinstance(buf, np.ndarray):
        import torch
        buf.view(-1)[:n].copy_(torch.from_numpy(np.ascontiguousarray(arr).reshape(-1)))
    else:
        buf.reshape(-1)[:n] = np.asarray(arr).reshape(-1)


def tide_planes(im, jm, tide_i, tide_j, amp, phase):
    """The coastal tide policy's table (0-based cell indices, amplitudes in
    m, phases in degrees; coastal_boundary.py:55-65 reads them 1-based from
    its data file) as the three im x jm planes of ``npom_workspace.tide``:
    1 at the tide cells, their amplitude, their phase.  A repeated cell
    keeps its last entry, as the policy's indexed assignment does."""
    out = np.zeros((3, im, jm), np.float32)
    for i, j, a, p in zip(np.asarray(tide_i).astype(np.int64).ravel(), np.asarray(tide_j).astype(np.int64).ravel(),
                          np.asarray(amp, np.float32).ravel(), np.asarray(phase, np.float32).ravel()):
        out[0, i, j] = 1.0
        out[1, i, j] = a
        out[2, i, j] = p
    return out
