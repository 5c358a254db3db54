"""CPU harness around tests/emul/npom_emul.cu (test infrastructure).

Builds the host-only emulation of the device phase bodies and drives it on
numpy arrays with the same field/workspace/parameter structs as the CUDA
library, so the phase logic can be compared with the oracle without a GPU.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "emul", "npom_emul.cu")
OUT = os.path.join(ROOT, "tests", "emul", "_build", "libnpom_emul.so")
DEPS = [SRC] + [os.path.join(ROOT, "neuralpom_b200", "csrc", f) for f in
                ("npom_ctx.cuh", "npom_phases_a.cuh", "npom_phases_ext.cuh", "npom_phases_int.cuh", "npom_host.cuh",
                 "npom_adjoint.cuh", "npom_mpdata.cuh", "npom_mpdata_adjoint.cuh")]

_LIB = None


def build_emul():
    global _LIB
    if _LIB is not None:
        return _LIB
    stale = not os.path.exists(OUT) or any(os.path.getmtime(d) > os.path.getmtime(OUT) for d in DEPS)
    if stale:
        os.makedirs(os.path.dirname(OUT), exist_ok=True)
        cmd = ["nvcc", "-O2", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "--fmad=false",
               "-Xcompiler", "-fPIC,-ffp-contract=off", "-shared", "-I", os.path.join(ROOT, "include"), SRC,
               "-o", OUT + ".tmp"]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(res.stdout + res.stderr)
        os.replace(OUT + ".tmp", OUT)
    from neuralpom_b200 import _abi
    lib = ctypes.CDLL(OUT)
    P = ctypes.POINTER
    lib.emul_run_phase.restype = ctypes.c_int
    lib.emul_run_phase.argtypes = [P(_abi.NpomParams), P(_abi.FieldArray), P(_abi.NpomWorkspace), ctypes.c_int,
                                   ctypes.c_double]
    lib.emul_steps.restype = ctypes.c_int
    lib.emul_step_adjoint.restype = ctypes.c_int
    lib.emul_step_adjoint.argtypes = [P(_abi.NpomParams), P(_abi.FieldArray), P(_abi.NpomWorkspace), P(_abi.NpomClock),
                                      P(_abi.FieldArray), P(_abi.FieldArray), ctypes.c_void_p, ctypes.c_size_t,
                                      ctypes.c_int]
    lib.emul_adjoint_plan.restype = ctypes.c_int
    lib.emul_adjoint_plan.argtypes = [P(_abi.NpomParams), ctypes.c_int, P(ctypes.c_size_t)]
    lib.emul_steps.argtypes = [P(_abi.NpomParams), P(_abi.FieldArray), P(_abi.NpomWorkspace), P(_abi.NpomClock)]
    _LIB = lib
    return lib


class EmulCore:
    """Numpy-backed state driven by the emulated phases."""

    def __init__(self, arrays, scalars, core):
        from neuralpom_b200 import _abi, state
        self.core = core
        im, jm, kb = arrays["u"].shape
        self.im, self.jm, self.kb = im, jm, kb
        self.F = {}
        for n in _abi.FIELD_NAMES:
            shp = _abi.field_shape(n, im, jm, kb)
            a = arrays.get(n)
            self.F[n] = np.ascontiguousarray(np.zeros(shp, np.float32) if a is None else a, dtype=np.float32).copy()
        self.W = {n: np.zeros(_abi.ws_shape(n, im, jm), np.float32) for n in _abi.WS_NAMES}
        s = dict(scalars)
        if "period" in arrays:
            s["period"] = float(np.asarray(arrays["period"]))
        self.scalars = s
        self.params = state.make_params(s, im, jm, kb, core)
        if core != "explicit":
            sx, sy, ie = state.spectral_setup(self.F["dx"], self.F["dy"], self.F["h"], s["dti"], s["grav"],
                                              s["alpha"], periodic_x=bool(s.get("periodic_x", False)))
            for n, a in (("sx", sx), ("sy", sy), ("inv_eigs", ie)):
                state.fill_flat(self.W[n], a)
        self.partials = np.zeros(4 * _abi.MAX_COOP_BLOCKS, np.float64)
        self.sync = np.zeros(4, np.uint32)
        self.status = np.zeros(1, np.uint32)
        self.cg_iters = np.zeros(4096, np.int32)
        self.mp3d = np.zeros(12 * im * jm * kb, np.float32)
        self.fa = _abi.FieldArray(*[self.F[n].ctypes.data for n in _abi.FIELD_NAMES])
        self.ws = _abi.NpomWorkspace()
        for i, n in enumerate(_abi.WS_NAMES):
            self.ws.buf[i] = self.W[n].ctypes.data
        self.ws.partials = self.partials.ctypes.data
        self.ws.sync = self.sync.ctypes.data
        self.ws.status = self.status.ctypes.data
        self.ws.cg_iters = self.cg_iters.ctypes.data
        if str(s.get("obc_form", "native")).lower() in ("coastal", "jzb"):
            self.tide = state.tide_planes(im, jm, arrays["tide_i"], arrays["tide_j"], arrays["tide_amp"],
                                          arrays["tide_phase"])
            self.ws.tide = self.tide.ctypes.data
        self.ws.mp3d = self.mp3d.ctypes.data
        self.robin = np.zeros(5 * im * jm, np.float64)
        self.ws.robin = self.robin.ctypes.data
        self.time = float(s.get("time", 0.0))

    def steps(self, n):
        from neuralpom_b200 import _abi
        clk = _abi.NpomClock(self.time, 1, n)
        rc = build_emul().emul_steps(ctypes.byref(self.params), ctypes.byref(self.fa), ctypes.byref(self.ws),
                                     ctypes.byref(clk))
        assert rc == 0
        self.time = self.time + n * self.params.dti / 86400.0
        return list(self.cg_iters[:n])

    def adjoint_step(self, grads, stop_after=-1):
        """Vector-Jacobian product of one internal step from the current
        state (which is restored afterwards): ``grads`` maps field names to
        the cotangents after the step; returns the cotangents before it."""
        from neuralpom_b200 import _abi
        lib = build_emul()
        need = ctypes.c_size_t(0)
        lib.emul_adjoint_plan(ctypes.byref(self.params), 1, ctypes.byref(need))
        save = np.zeros(max(int(need.value), 1), np.float32)
        G = {n: np.zeros_like(self.F[n]) for n in _abi.FIELD_NAMES}
        for n, g in grads.items():
            G[n][...] = g
        Lm = {n: np.zeros_like(self.F[n]) for n in _abi.FIELD_NAMES}
        ga = _abi.FieldArray(*[G[n].ctypes.data for n in _abi.FIELD_NAMES])
        la = _abi.FieldArray(*[Lm[n].ctypes.data for n in _abi.FIELD_NAMES])
        clk = _abi.NpomClock(self.time, 1, 1)
        rc = lib.emul_step_adjoint(ctypes.byref(self.params), ctypes.byref(self.fa), ctypes.byref(self.ws),
                                   ctypes.byref(clk), ctypes.byref(ga), ctypes.byref(la), save.ctypes.data,
                                   save.size, int(stop_after))
        assert rc == 0, rc
        return G

    def phase(self, ph, ramp=1.0):
        rc = build_emul().emul_run_phase(ctypes.byref(self.params), ctypes.byref(self.fa), ctypes.byref(self.ws),
                                         ph, ramp)
        assert rc == 0


def multi_step_adjoint(arrays, scalars, cot, nsteps, core="explicit"):
    """Reverse mode of ``nsteps`` emulated steps with a checkpoint per step:
    forward saving each step's start state, then the step adjoints in
    reverse order.  Returns the cotangents of the start state."""
    E = EmulCore(arrays, scalars, core)
    starts = []
    for _ in range(nsteps):
        starts.append(({n: v.copy() for n, v in E.F.items()}, E.time))
        E.steps(1)
    G = dict(cot)
    for F0, t0 in reversed(starts):
        for n, v in F0.items():
            E.F[n][...] = v
        E.time = t0
        G = E.adjoint_step(G)
    return G
