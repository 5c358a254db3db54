"""The no-allocation PCG entry point (npom_pcg_solve_static) against the
allocating one (npom_pcg_solve), both called through the C ABI.  The file is
named to be collected last; its tests also pass on their own."""
import ctypes

import numpy as np
import pytest
import torch

from golden_io import rel_err


def _lib():
    from neuralpom_b200 import _abi, build
    build.build()
    return _abi, _abi.load_library()


def test_static_solve_rejects_grids_above_the_scratch_limit():
    """im*jm above NPOM_STATIC_MAX_CELLS is refused before any CUDA call."""
    _abi, lib = _lib()
    p = _abi.NpomParams()
    p.core, p.im, p.jm, p.kb, p.device = _abi.CORE_IMPLICIT, 200, 200, 16, 0
    p.eta_precond = _abi.PRECOND_JACOBI
    assert 200 * 200 > _abi.STATIC_MAX_CELLS
    fields = _abi.FieldArray()
    rc = lib.npom_pcg_solve_static(ctypes.byref(p), ctypes.byref(fields), ctypes.c_void_p(16), None, None, None,
                                   None, None, None)
    assert _abi.STATUS_NAMES[rc] == "NPOM_ERR_TOO_LARGE"


def _case(im, jm, precond="spectral"):
    from neuralpom_b200 import cases, resolve_core_class
    A, Sc = cases.seamount(im, jm)
    Sc = dict(Sc, eta_solver_preconditioner=precond)
    core = resolve_core_class("implicit_p0_fixed").from_state(A, Sc, device="cuda")
    g = torch.Generator(device="cpu").manual_seed(1000 * im + jm)
    fsm = core.fsm
    rhs = (0.01 * torch.randn((im, jm), generator=g)).cuda() * fsm
    x0 = (0.001 * torch.randn((im, jm), generator=g)).cuda() * fsm
    return core, rhs.contiguous(), x0.contiguous()


def _fields_with_elf(_abi, core, x):
    fields = _abi.FieldArray(*core._fields())
    fields[_abi.FIELD_NAMES.index("elf")] = x.data_ptr()
    return fields


def _solve_allocating(_abi, lib, core, rhs, x0):
    p, ws = core.params(), core._workspace()
    x = x0.clone()
    ws["bufs"]["rhs"].copy_(rhs)
    fields = _fields_with_elf(_abi, core, x)
    st = torch.cuda.current_stream()
    ws["ctrl"][4].zero_()
    _abi.check(lib.npom_pcg_solve(ctypes.byref(p), ctypes.byref(fields), ctypes.byref(ws["struct"]),
                                  ctypes.c_void_p(st.cuda_stream)), "npom_pcg_solve")
    torch.cuda.synchronize()
    status = int(ws["ctrl"][4].item())
    ws["ctrl"][4].zero_()
    return x, int(ws["ctrl"][8].item()), status


def _solve_static(_abi, lib, core, rhs, x0):
    p, ws = core.params(), core._workspace()     # ws only supplies the spectral operator inputs
    b = ws["bufs"]
    # the Jacobi preconditioner needs no spectral inputs: pass null for them
    spectral = p.eta_precond == _abi.PRECOND_SPECTRAL
    sx, sy, ie = ((b["sx"].data_ptr(), b["sy"].data_ptr(), b["inv_eigs"].data_ptr()) if spectral
                  else (None, None, None))
    x = x0.clone()
    fields = _fields_with_elf(_abi, core, x)
    out = torch.full((2,), -1, dtype=torch.int32, device="cuda")
    st = torch.cuda.current_stream()
    rc = lib.npom_pcg_solve_static(ctypes.byref(p), ctypes.byref(fields), ctypes.c_void_p(rhs.data_ptr()),
                                   ctypes.c_void_p(sx), ctypes.c_void_p(sy), ctypes.c_void_p(ie),
                                   ctypes.c_void_p(out.data_ptr()),
                                   ctypes.c_void_p(out.data_ptr() + 4), ctypes.c_void_p(st.cuda_stream))
    _abi.check(rc, "npom_pcg_solve_static")
    torch.cuda.synchronize()
    return x, int(out[0].item()), int(out[1].item())


# 90x82: the cluster PCG; 150x150 (148 interior rows): the grid-barrier PCG;
# each with the spectral preconditioner and with Jacobi (null spectral inputs)
@pytest.mark.gpu
@pytest.mark.parametrize("precond", ["spectral", "jacobi"])
@pytest.mark.parametrize("im,jm", [(90, 82), (150, 150)])
def test_static_solve_equals_allocating_solve_on_two_consecutive_calls(im, jm, precond):
    _abi, lib = _lib()
    core, rhs, x0 = _case(im, jm, precond)
    rhs_before = rhs.clone()
    xa, ia, status_a = _solve_allocating(_abi, lib, core, rhs, x0)
    assert ia > 0
    # the Jacobi-preconditioned solve of this case stops at the iteration
    # cap (status NPOM_DEV_PCG_MAXIT) in both entry points
    assert status_a in (0, _abi.DEV_PCG_MAXIT)
    for _ in range(2):
        xs, its, status = _solve_static(_abi, lib, core, rhs, x0)
        assert status == status_a
        assert its == ia
        # same kernels on the same inputs: equal within the parity bound
        assert rel_err(xs.cpu().numpy(), xa.cpu().numpy()) < 1e-6
        assert np.array_equal(xs[0].cpu().numpy(), np.zeros(jm, np.float32))
    assert torch.equal(rhs, rhs_before)
