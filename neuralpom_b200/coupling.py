"""The two physics operators of the corrector coupling on the B200 library:
the equation of state and the baroclinic pressure gradient, as CUDA kernels
with hand-written adjoints (``npom_dens``/``npom_dens_adjoint``,
``npom_baropg``/``npom_baropg_adjoint``) behind ``torch.autograd.Function``.

The cores' operator methods ``dens()`` and ``baropg()`` use them, which is
all the reference's own coupling module needs: its ``eos``,
``apply_joint_correction`` and ``pressure_velocity_error``
(``src/neuralpom/hybrid/sparse_coupling.py:10-82``) run unchanged on a B200
core and differentiate through these operators.  The rest of that module
(increment scaling, budget projections, limits) is a few reductions per
physics interval and stays the reference's PyTorch code.
"""
from __future__ import annotations

import ctypes

import torch

from . import _abi

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
