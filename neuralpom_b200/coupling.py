"""Corrector coupling around the B200 step: the endpoint correction a
neural model applies between physics intervals, with the reference's API
(``src/neuralpom/hybrid/sparse_coupling.py:10-82``).

The state updates, budget projections and limits are a few reductions once
per interval and stay in PyTorch (differentiable by autograd).  The two
physics operators inside -- the equation of state and the baroclinic
pressure gradient -- run as CUDA kernels with hand-written adjoints
(``npom_dens``/``npom_dens_adjoint``, ``npom_baropg``/
``npom_baropg_adjoint``).  The cores' ``dens()`` and ``baropg()`` methods
use the same kernels, so the reference's own coupling functions also accept
a B200 core.
"""
from __future__ import annotations

import ctypes

import torch

from . import _abi

OUTPUT_FIELDS = ("u", "v", "t", "s")
LEVELS = 15
OUTPUT_CHANNELS = 4 * LEVELS


def _call(core):
    lib = _abi.load_library()
    if core.device.type != "cuda":
        raise RuntimeError("the B200 operators run on CUDA devices only")
    fa, keep = core._fields_readonly()
    return lib, core.params(), fa, keep, torch.cuda.current_stream(core.device)


def _vol(core, x):
    return x.detach().to(device=core.device, dtype=torch.float32).reshape(core.im, core.jm, core.kb).contiguous()


class _DensFunction(torch.autograd.Function):
    """rho = DENS(t, s) on levels < kb-1, the ghost level from rho_prev
    (explicit/momentum.py:467-541, as ``eos`` evaluates it on a copy of the
    core)."""

    @staticmethod
    def forward(ctx, core, t, s, rho_prev):
        lib, p, fa, keep, st = _call(core)
        t_, s_ = _vol(core, t), _vol(core, s)
        fields = _abi.FieldArray(*fa)
        rho_prev_c = _vol(core, rho_prev)
        fields[_abi.FIELD_NAMES.index("rho")] = rho_prev_c.data_ptr()
        out = torch.empty_like(t_)
        _abi.check(lib.npom_dens(ctypes.byref(p), ctypes.byref(fields), ctypes.c_void_p(t_.data_ptr()),
                                 ctypes.c_void_p(s_.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                 ctypes.c_void_p(st.cuda_stream)), "npom_dens")
        ctx.core = core
        ctx.save_for_backward(t_, s_)
        return out

    @staticmethod
    def backward(ctx, g):
        t_, s_ = ctx.saved_tensors
        core = ctx.core
        lib, p, fa, keep, st = _call(core)
        g_ = _vol(core, g)
        gt, gs, gr = torch.empty_like(g_), torch.empty_like(g_), torch.empty_like(g_)
        _abi.check(lib.npom_dens_adjoint(ctypes.byref(p), ctypes.byref(fa), ctypes.c_void_p(t_.data_ptr()),
                                         ctypes.c_void_p(s_.data_ptr()), ctypes.c_void_p(g_.data_ptr()),
                                         ctypes.c_void_p(gt.data_ptr()), ctypes.c_void_p(gs.data_ptr()),
                                         ctypes.c_void_p(gr.data_ptr()), ctypes.c_void_p(st.cuda_stream)),
                   "npom_dens_adjoint")
        return None, gt, gs, gr


class _BaropgFunction(torch.autograd.Function):
    """(rho, drhox, drhoy) = BAROPG of rho against rmean at the core's ramp
    and depth dt (explicit/momentum.py:543-700)."""

    @staticmethod
    def forward(ctx, core, rho, rmean, dt):
        lib, p, fa, keep, st = _call(core)
        rho_, rm_ = _vol(core, rho), _vol(core, rmean)
        fields = _abi.FieldArray(*fa)
        dt_ = dt.detach().to(device=core.device, dtype=torch.float32).reshape(core.im, core.jm).contiguous()
        fields[_abi.FIELD_NAMES.index("dt")] = dt_.data_ptr()
        ramp = float(core.ramp)
        rho_out, dx, dy = torch.empty_like(rho_), torch.empty_like(rho_), torch.empty_like(rho_)
        _abi.check(lib.npom_baropg(ctypes.byref(p), ctypes.byref(fields), ctypes.c_void_p(rho_.data_ptr()),
                                   ctypes.c_void_p(rm_.data_ptr()), ctypes.c_double(ramp),
                                   ctypes.c_void_p(rho_out.data_ptr()), ctypes.c_void_p(dx.data_ptr()),
                                   ctypes.c_void_p(dy.data_ptr()), ctypes.c_void_p(st.cuda_stream)), "npom_baropg")
        ctx.core, ctx.ramp = core, ramp
        ctx.save_for_backward(rho_, rm_, dt_)
        return rho_out, dx, dy

    @staticmethod
    def backward(ctx, g_rho, g_dx, g_dy):
        rho_, rm_, dt_ = ctx.saved_tensors
        core = ctx.core
        lib, p, fa, keep, st = _call(core)
        fields = _abi.FieldArray(*fa)
        fields[_abi.FIELD_NAMES.index("dt")] = dt_.data_ptr()
        gr = torch.zeros_like(rho_)
        gd = torch.zeros_like(dt_)
        zero = torch.zeros_like(rho_)
        gx = _vol(core, g_dx) if g_dx is not None else zero
        gy = _vol(core, g_dy) if g_dy is not None else zero
        _abi.check(lib.npom_baropg_adjoint(ctypes.byref(p), ctypes.byref(fields), ctypes.c_void_p(rho_.data_ptr()),
                                           ctypes.c_void_p(rm_.data_ptr()), ctypes.c_double(ctx.ramp),
                                           ctypes.c_void_p(gx.data_ptr()), ctypes.c_void_p(gy.data_ptr()),
                                           ctypes.c_void_p(gr.data_ptr()), ctypes.c_void_p(gd.data_ptr()),
                                           ctypes.c_void_p(st.cuda_stream)), "npom_baropg_adjoint")
        g_rmean = -gr
        if g_rho is not None:
            gr = gr + _vol(core, g_rho)  # the round trip (rho - rmean) + rmean
        return None, gr, g_rmean, gd


def eos(core, t, s):
    """The core's equation of state on (t, s) with its ghost rule
    (sparse_coupling.py:10-15): DENS on levels < kb-1, the ghost level of
    the core's rho."""
    return _DensFunction.apply(core, t, s, core.rho)


def volume_weights(core, field="t"):
    """Cell volumes of the corrected levels (sparse_coupling.py:18-20)."""
    mask = core.dum if field in ("u", "ub") else (core.dvm if field in ("v", "vb") else core.fsm)
    return (core.art * mask * (core.h + core.et))[:, :, None] * core.dz[:LEVELS][None, None, :]


def weighted_mse(x, y, w):
    return ((x - y).square() * w).sum() / w.expand_as(x).sum().clamp_min(1e-20)


def budget_project(increment, weights):
    """Remove the volume-weighted mean of each level on the wet cells, so
    the increment moves tracer within a layer and the physics keeps the
    vertical budget (sparse_coupling.py:27-32)."""
    level_mean = (increment * weights).sum((0, 1), keepdim=True) / weights.sum((0, 1), keepdim=True).clamp_min(1e-20)
    return (increment - level_mean) * (weights > 0)


def paired_limit(increments, scales, cap):
    """One common factor for a pair of increments so that neither exceeds
    cap scale units (sparse_coupling.py:35-39); returns the scaled pair and
    the factor."""
    peak = torch.stack([(x / sc).abs().amax() for x, sc in zip(increments, scales)]).amax()
    factor = (cap / peak.clamp_min(cap)).clamp(max=1.0)
    return [factor * x for x in increments], factor


def apply_joint_correction(core, raw, scales, cap=5.0):
    """Add a network's raw (60, im, jm) output to u, v, T, S and their
    previous time levels (sparse_coupling.py:42-67): per-field scales,
    depth-mean-free velocity increments, layer-budget-free tracer
    increments, paired limits, then the EOS refresh.  Differentiable in
    raw and in the state."""
    if core.kbm1 != LEVELS or tuple(raw.shape) != (OUTPUT_CHANNELS, core.im, core.jm):
        raise ValueError(f"Unexpected grid/output contract: {core.kbm1}, {tuple(raw.shape)}")
    inc = {f: raw[n * LEVELS:(n + 1) * LEVELS].permute(1, 2, 0) * scales[f] for n, f in enumerate(OUTPUT_FIELDS)}
    dz = core.dz[:LEVELS].view(1, 1, -1)
    for f, mask in (("u", core.dum), ("v", core.dvm)):
        inc[f] = (inc[f] - (inc[f] * dz).sum(2, keepdim=True) / dz.sum()) * mask[:, :, None]
    w = volume_weights(core)
    for f in ("t", "s"):
        inc[f] = budget_project(inc[f], w)
    (inc["t"], inc["s"]), factor = paired_limit([inc["t"], inc["s"]], [scales["t"], scales["s"]], cap)
    (inc["u"], inc["v"]), _ = paired_limit([inc["u"], inc["v"]], [scales["u"], scales["v"]], cap)
    for f, prev in (("u", "ub"), ("v", "vb"), ("t", "tb"), ("s", "sb")):
        for name in (f, prev):
            x = getattr(core, name)
            # the ghost level keeps the core's value
            setattr(core, name, torch.cat((x[:, :, :LEVELS] + inc[f], x[:, :, LEVELS:]), dim=2))
    core.rho = eos(core, core.t, core.s)
    return {"ts_limit_factor": factor, "t_budget": (w * inc["t"]).sum() / w.sum(),
            "s_budget": (w * inc["s"]).sum() / w.sum()}


def pressure_velocity_error(core, reference_t, reference_s):
    """Velocity kick of the baroclinic pressure-gradient difference between
    the core's (t, s) and a reference (t, s) on the core's geometry
    (sparse_coupling.py:70-82): BAROPG is linear in rho at fixed geometry,
    so it is evaluated once on the density difference with rmean = 0."""
    drho = eos(core, core.t, core.s) - eos(core, reference_t, reference_s)
    _, px, py = _BaropgFunction.apply(core, drho, torch.zeros_like(core.rmean), core.dt)
    depth = core.h + core.etf
    du = (depth + torch.roll(depth, 1, 0)) * core.aru
    dv = (depth + torch.roll(depth, 1, 1)) * core.arv
    kick_u = -2.0 * core.dti2 * px[:, :, :LEVELS] / du[:, :, None].clamp_min(1e-20)
    kick_v = -2.0 * core.dti2 * py[:, :, :LEVELS] / dv[:, :, None].clamp_min(1e-20)
    return kick_u * core.dum[:, :, None], kick_v * core.dvm[:, :, None]
