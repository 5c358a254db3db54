"""Drop-in POM cores whose physical time step runs on the B200 library.

``ExplicitCore`` and ``ImplicitCore`` expose the attribute set of the
reference ``POM2K_Core`` classes (``src/neuralpom/cores/explicit/core.py:17``,
``cores/implicit_p0_fixed/core.py:62``): the same tensor names and shapes
(``explicit/base.py:129-195``), the same scalar attributes, and the step
function ``run_time_loop()`` that advances ``iend`` internal steps from
``time0`` and leaves ``iint``/``time``/``ramp`` as the reference does
(``explicit/time_loop.py:75-88``).  The arithmetic runs in
``libnpom_b200.so`` (sm_100a) through the C ABI of ``include/npom.h``; there
is no CPU path.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _abi, cases, state

NUMERICS_VERSION = {
    "explicit": "explicit-dg-v2-split-smag-v2align-closure",
    "implicit_p0_fixed": "implicit-dg-v2-aligned-1e5-p0-barotropic-coupling-fixed",
}
MAX_STEPS_PER_CALL = 4096


class B200Core:
    """Common state container and C-ABI driver of both cores."""

    core_name = None

    def __init__(self, im, jm, problem_id=4, settings_overrides=None, case_name=None, device=None, kb=16):
        if problem_id != 4:
            raise ValueError(f"Only the Double-gyre problem_id=4 is supported; got {problem_id}.")
        self.device = torch.device(device if device is not None else "cuda")
        self.im, self.jm, self.kb = int(im), int(jm), int(kb)
        self.iproblem = problem_id
        self.case_name = case_name
        for k, v in state.default_scalars(self.core_name).items():
            setattr(self, k, v)
        self._refresh_derived()
        self.time = 0.0
        self.time0 = 0.0
        self.iint = 0
        self.iend = 2
        for n in _abi.FIELD_NAMES:
            setattr(self, n, torch.zeros(_abi.field_shape(n, self.im, self.jm, self.kb), dtype=torch.float32,
                                         device=self.device))
        self.period = torch.ones((), dtype=torch.float32, device=self.device)
        for k, v in dict(settings_overrides or {}).items():
            setattr(self, k, v)
        self._refresh_derived()
        self._ws = None
        self._ws_key = None
        self._ws_geo = None
        # launch shapes of the step (npom_tuning fields; None: the library's
        # rules), e.g. from neuralpom_b200.autotune
        self.tuning = None
        self._eta_solver_iteration_history = []
        self._eta_adjoint_iteration_history = []

    # -- reference-compatible helpers ------------------------------------
    @property
    def NUMERICS_VERSION(self):
        return NUMERICS_VERSION[self.core_name]

    def _refresh_derived(self):
        self.imm1, self.imm2 = self.im - 1, self.im - 2
        self.jmm1, self.jmm2 = self.jm - 1, self.jm - 2
        self.kbm1, self.kbm2 = self.kb - 1, self.kb - 2
        state.derived_time(self.__dict__)

    def load_state(self, arrays, scalars=None):
        """Overwrite tensors (and scalars) from numpy arrays / tensors."""
        for k, v in (scalars or {}).items():
            setattr(self, k, v)
        self._refresh_derived()
        for k, v in arrays.items():
            t = torch.as_tensor(np.ascontiguousarray(v) if isinstance(v, np.ndarray) else v)
            setattr(self, k, t.to(device=self.device, dtype=torch.float32).contiguous().clone())
        self._ws_key = None
        return self

    @classmethod
    def from_state(cls, arrays, scalars, device=None):
        im, jm, kb = np.asarray(arrays["u"]).shape
        core = cls(im, jm, device=device, kb=kb)
        return core.load_state(arrays, scalars)

    def run_initialization(self):
        """The reference double gyre set-up (cases.py:30 + initialization.py:10)."""
        arrays, scalars = cases.double_gyre(self.im, self.jm, self.core_name, self.kb)
        self.load_state(arrays, scalars)

    def state_arrays(self):
        return {n: getattr(self, n).detach().cpu().numpy().copy() for n in _abi.FIELD_NAMES}

    # -- workspace ---------------------------------------------------------
    def _workspace(self):
        # the spectral operator depends on dx, dy and h: a tensor replaced by
        # another one (a new object, even at a recycled address with a fresh
        # version counter) or modified in place (a new version) rebuilds it.
        # The key holds the objects' ids and _ws_geo keeps the objects alive,
        # so an id in the key cannot be recycled by a new tensor.
        geo = tuple((n, id(getattr(self, n)), getattr(self, n).data_ptr(), getattr(self, n)._version)
                    for n in ("dx", "dy", "h"))
        key = (self.im, self.jm, self.kb, self.device, geo, float(self.dti), float(self.alpha),
               bool(getattr(self, "periodic_x", False)))
        if self._ws is not None and self._ws_key == key:
            return self._ws
        im, jm, dev = self.im, self.jm, self.device
        if self._ws is None or self._ws["shape"] != (im, jm):
            bufs = {n: torch.zeros(_abi.ws_shape(n, im, jm), dtype=torch.float32, device=dev) for n in _abi.WS_NAMES}
            ws = {"shape": (im, jm), "bufs": bufs,
                  "partials": torch.zeros(4 * _abi.MAX_COOP_BLOCKS, dtype=torch.float64, device=dev),
                  # ctrl = [sync x4 | status | pad x3 | cg iterations ...]
                  "ctrl": torch.zeros(8 + MAX_STEPS_PER_CALL, dtype=torch.int32, device=dev)}
            s = _abi.NpomWorkspace()
            for i, n in enumerate(_abi.WS_NAMES):
                s.buf[i] = bufs[n].data_ptr()
            base = ws["ctrl"].data_ptr()
            s.partials = ws["partials"].data_ptr()
            s.sync = base
            s.status = base + 4 * 4
            s.cg_iters = base + 8 * 4
            ws["struct"] = s
            self._ws = ws
        if str(getattr(self, "obc_form", "native")).lower() in ("coastal", "jzb") and "tide" not in self._ws:
            # the coastal tide policy's table as three planes (flag, amplitude, phase)
            planes = state.tide_planes(im, jm, *(state.host_array(getattr(self, n))
                                                 for n in ("tide_i", "tide_j", "tide_amp", "tide_phase")))
            self._ws["tide"] = torch.from_numpy(planes).to(dev).contiguous()
            self._ws["struct"].tide = self._ws["tide"].data_ptr()
        if (str(getattr(self, "obc_form", "native")).lower() == "seamount" and self.core_name != "explicit"
                and "robin" not in self._ws):
            # the semi-implicit seamount policy's FP64 Robin solve: 5 planes
            self._ws["robin"] = torch.zeros(5 * im * jm, dtype=torch.float64, device=dev)
            self._ws["struct"].robin = self._ws["robin"].data_ptr()
        if int(getattr(self, "nadv", 1)) == 2 and "mp3d" not in self._ws:
            # MPDATA scratch: mass fluxes and fluxes of T and S
            self._ws["mp3d"] = torch.zeros(12 * im * jm * self.kb, dtype=torch.float32, device=dev)
            self._ws["struct"].mp3d = self._ws["mp3d"].data_ptr()
        if self.core_name != "explicit":
            sx, sy, ie = state.spectral_setup(self.dx.detach().cpu().numpy(), self.dy.detach().cpu().numpy(),
                                              self.h.detach().cpu().numpy(), float(self.dti), float(self.grav),
                                              float(self.alpha), periodic_x=bool(getattr(self, "periodic_x", False)))
            b = self._ws["bufs"]
            for n, a in (("sx", sx), ("sy", sy), ("inv_eigs", ie)):
                state.fill_flat(b[n], a)
        self._ws_key = key
        self._ws_geo = tuple(getattr(self, n) for n in ("dx", "dy", "h"))
        return self._ws

    def _fields(self):
        ptrs = []
        for n in _abi.FIELD_NAMES:
            t = getattr(self, n)
            shp = _abi.field_shape(n, self.im, self.jm, self.kb)
            if not torch.is_tensor(t):
                raise TypeError(f"{n} must be a tensor")
            if t.requires_grad:
                raise NotImplementedError(
                    f"{n} requires grad: the differentiable advance is not provided by the B200 core")
            if (tuple(t.shape) != shp or t.dtype != torch.float32 or t.device != self.device
                    or not t.is_contiguous()):
                t = t.detach().to(device=self.device, dtype=torch.float32).reshape(shp).contiguous()
                setattr(self, n, t)
            ptrs.append(t.data_ptr())
        return _abi.FieldArray(*ptrs)

    def _fields_readonly(self):
        """Field pointers for operators that only read the state (the
        coupling's DENS/BAROPG): detached, converted copies where needed;
        returns (FieldArray, tensors to keep alive)."""
        keep, ptrs = [], []
        for n in _abi.FIELD_NAMES:
            t = getattr(self, n).detach()
            shp = _abi.field_shape(n, self.im, self.jm, self.kb)
            if tuple(t.shape) != shp or t.dtype != torch.float32 or t.device != self.device or not t.is_contiguous():
                t = t.to(device=self.device, dtype=torch.float32).reshape(shp).contiguous()
            keep.append(t)
            ptrs.append(t.data_ptr())
        return _abi.FieldArray(*ptrs), keep

    def params(self):
        return state.make_params(self, self.im, self.jm, self.kb, self.core_name,
                                 self.device.index if self.device.index is not None else torch.cuda.current_device())

    # -- the step ----------------------------------------------------------
    def launch_steps(self, nsteps, time0, first_iint=1, stream=None):
        """Enqueue ``nsteps`` internal steps on ``stream`` without waiting."""
        lib = _abi.load_library()
        if self.device.type != "cuda":
            raise RuntimeError("the B200 core runs on CUDA devices only")
        p = self.params()
        fa = self._fields()
        ws = self._workspace()
        st = stream if stream is not None else torch.cuda.current_stream(self.device)
        fn = lib.npom_step_explicit if self.core_name == "explicit" else lib.npom_step_implicit
        done = 0
        while done < nsteps:
            n = min(MAX_STEPS_PER_CALL, nsteps - done)
            clk = _abi.NpomClock(float(time0), int(first_iint + done), int(n))
            _abi.check(fn(ctypes.byref(p), ctypes.byref(fa), ctypes.byref(ws["struct"]), ctypes.byref(clk),
                          ctypes.c_void_p(st.cuda_stream)), "npom step")
            done += n
        return ws

    def read_status(self, nsteps=0):
        """(status bits, PCG iterations of the last call) -- one device sync."""
        ws = self._ws
        if ws is None:
            return 0, []
        n = min(int(nsteps), MAX_STEPS_PER_CALL)
        ctrl = ws["ctrl"][4:8 + n].cpu()
        bits = int(ctrl[0])
        ws["ctrl"][4].zero_()
        return bits, [int(v) for v in ctrl[4:4 + n]]

    def run_time_loop(self):
        """Advance ``iend`` internal steps from ``time0`` (reference
        run_time_loop semantics); raises FloatingPointError when the
        barotropic velocity exceeds vmaxl or the elevation is not finite.
        When grad mode is on and a state tensor requires grad, the advance
        is one differentiable node whose backward is the hand-written step
        adjoint; the state attributes are rebound to its outputs, as the
        reference's autograd path rebinds them.

        With ``status_deferred`` set the call only enqueues: the device
        status is not read back (no host synchronisation, so the members of
        an ensemble on their own streams overlap) and accumulates until
        ``check_deferred_status()``; no PCG iteration history is recorded."""
        nsteps = int(self.iend)
        if nsteps < 0:
            raise ValueError("iend must be non-negative")
        deferred = getattr(self, "status_deferred", False)
        if self._differentiable_call():
            policy = (str(getattr(self, "profq_form", "production")).lower() != "production" or
                      str(getattr(self, "obc_form", "native")).lower() != "native")
            if policy:
                # as the reference's case-policy registry does
                # (cores/case_adapters/registry.py:38-41)
                raise RuntimeError("Registered case policies require advancement inside torch.no_grad(); "
                                   "their training adjoints are unvalidated.")
            if bool(getattr(self, "periodic_x", False)):
                raise RuntimeError("periodic x is forward only: advance inside torch.no_grad()")
            outs = _StepsFunction.apply(self, nsteps, float(self.time0),
                                        *[getattr(self, f) for f in _abi.ADJ_STATE_FIELDS])
            for f, o in zip(_abi.ADJ_STATE_FIELDS, outs):
                setattr(self, f, o)
        else:
            with torch.no_grad():
                self.launch_steps(nsteps, float(self.time0))
        bits, its = (0, []) if deferred else self.read_status(nsteps)
        self._finish_advance(nsteps, bits, its)

    def check_deferred_status(self):
        """Reads and clears the status accumulated by the advances made with
        ``status_deferred`` set (after the work of every stream on the
        device); raises for it like ``run_time_loop``."""
        if self.device.type == "cuda":
            torch.cuda.synchronize(self.device)
        bits, _ = self.read_status(0)
        self._raise_for(bits)

    def _finish_advance(self, nsteps, bits, its):
        """Clock, ramp and PCG history after ``nsteps`` steps from time0;
        raises for the device status bits."""
        self.iint = nsteps
        self.time = self.dti * nsteps * 1.0 / 86400.0 + self.time0
        if self.lramp:
            r = float(np.float32(self.time) / np.float32(state.host_scalar(self.period)))
            self.ramp = 1.0 if r > 1.0 else r
        else:
            self.ramp = 1.0
        if self.core_name != "explicit":
            self._eta_solver_iteration_history.extend(its)
        self._raise_for(bits)

    # -- operator methods (override points of the reference cores) ----------
    def dens(self):
        """DENS (explicit/momentum.py:467-541): rho on levels < kb-1 from
        (t, s), returned like the reference as (s, t, rho)."""
        from .coupling import eos
        self.rho = eos(self, self.t, self.s)
        return self.s, self.t, self.rho

    def baropg(self):
        """BAROPG (explicit/momentum.py:543-700): returns (rho, drhox,
        drhoy) at the core's ramp; rho goes through the reference's
        (rho - rmean) + rmean round trip."""
        from .coupling import _BaropgFunction
        self.rho, drhox, drhoy = _BaropgFunction.apply(self, self.rho, self.rmean, self.dt)
        return self.rho, drhox, drhoy

    def _differentiable_call(self):
        if not torch.is_grad_enabled():
            return False
        return any(torch.is_tensor(getattr(self, f)) and getattr(self, f).requires_grad for f in _abi.FIELD_NAMES)

    def _raise_for(self, bits):
        if bits & _abi.DEV_TIMEOUT:
            raise RuntimeError("B200 step: a grid barrier timed out (device status 0x%x)" % bits)
        if bits & (_abi.DEV_VMAX | _abi.DEV_NONFINITE):
            raise FloatingPointError(
                f"Barotropic velocity exceeds limit {self.vmaxl} or elevation not finite at time {self.time}")


class ExplicitCore(B200Core):
    """Explicit mode-split core (reference ``cores/explicit``)."""
    core_name = "explicit"


class _StateBuffer:
    """One flat float32 device buffer holding the given fields back to back,
    with a view per field (a checkpoint of them is one copy)."""

    def __init__(self, names, im, jm, kb, device):
        self.names = tuple(names)
        self.shapes = [_abi.field_shape(n, im, jm, kb) for n in self.names]
        sizes = [int(np.prod(s)) for s in self.shapes]
        self.flat = torch.zeros(sum(sizes), dtype=torch.float32, device=device)
        self.views = {}
        off = 0
        for n, shp, sz in zip(self.names, self.shapes, sizes):
            self.views[n] = self.flat[off:off + sz].view(shp)
            off += sz


class _StepsFunction(torch.autograd.Function):
    """``nsteps`` internal steps as one autograd node: inputs and outputs
    are the state fields ``_abi.ADJ_STATE_FIELDS``.  The forward keeps one
    checkpoint of the state per step; the backward recomputes each step
    from its checkpoint and runs the step adjoint
    (``npom_step_explicit_adjoint`` / ``npom_step_implicit_adjoint``) in
    reverse step order (per-internal-step checkpointing with recomputation,
    like the reference's ``_checkpoint_chunk``, sparse_physics.py:108-149,
    under torch autograd)."""

    @staticmethod
    def forward(ctx, core, nsteps, time0, *state):
        # outputs without a cotangent reach backward as None (no zero fills)
        ctx.set_materialize_grads(False)
        dev = core.device
        im, jm, kb = core.im, core.jm, core.kb
        dyn = _StateBuffer(_abi.ADJ_STATE_FIELDS, im, jm, kb, dev)
        for n, t in zip(_abi.ADJ_STATE_FIELDS, state):
            dyn.views[n].copy_(t.detach().reshape(dyn.views[n].shape))
            setattr(core, n, dyn.views[n])
        ckpt = torch.empty((max(nsteps, 1), dyn.flat.numel()), dtype=torch.float32, device=dev)
        # the call's structs once: the fields live in dyn for the whole call
        lib = _abi.load_library()
        p, fa, ws = core.params(), core._fields(), core._workspace()
        implicit = core.core_name != "explicit"
        fn = lib.npom_step_implicit if implicit else lib.npom_step_explicit
        st = ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
        # semi-implicit core: the raw solution of every step's free-surface
        # solve (workspace plane x), so the step adjoint replays the solve
        xck = torch.empty((max(nsteps, 1), im * jm) if implicit else (1, 1), dtype=torch.float32, device=dev)
        for n in range(nsteps):
            ckpt[n].copy_(dyn.flat)
            clk = _abi.NpomClock(float(time0), n + 1, 1)
            _abi.check(fn(ctypes.byref(p), ctypes.byref(fa), ctypes.byref(ws["struct"]), ctypes.byref(clk), st),
                       "npom step")
            if implicit:
                xck[n].copy_(ws["bufs"]["x"].reshape(-1))
        ctx.core, ctx.nsteps, ctx.time0 = core, nsteps, time0
        ctx.save_for_backward(ckpt, xck)
        outs = tuple(dyn.views[n].clone() for n in _abi.ADJ_STATE_FIELDS)
        for n, o in zip(_abi.ADJ_STATE_FIELDS, outs):
            setattr(core, n, o)
        return outs

    @staticmethod
    def backward(ctx, *grads):
        ckpt, xck = ctx.saved_tensors
        core = ctx.core
        lib = _abi.load_library()
        dev = core.device
        im, jm, kb = core.im, core.jm, core.kb
        names = _abi.FIELD_NAMES
        # the working state: every field, the dynamic ones reloaded from
        # each step's checkpoint
        work = _StateBuffer(_abi.ADJ_STATE_FIELDS + tuple(n for n in names if n not in _abi.ADJ_STATE_FIELDS),
                            im, jm, kb, dev)
        for n in names:
            if n not in _abi.ADJ_STATE_FIELDS:
                work.views[n].copy_(getattr(core, n).detach().reshape(work.views[n].shape))
        ndyn = ckpt.shape[1]
        G = _StateBuffer(names, im, jm, kb, dev)
        Lm = _StateBuffer(names, im, jm, kb, dev)
        for n, g in zip(_abi.ADJ_STATE_FIELDS, grads):
            if g is not None:
                G.views[n].copy_(g.reshape(G.views[n].shape))
        p = core.params()
        save = torch.empty(max(int(lib.npom_adjoint_save_floats(ctypes.byref(p))), 1), dtype=torch.float32,
                           device=dev)
        aws = _abi.NpomAdjointWs()
        for i, n in enumerate(names):
            aws.lam[i] = Lm.views[n].data_ptr()
        aws.save = save.data_ptr()
        aws.save_floats = save.numel()
        implicit = core.core_name != "explicit"
        xfix = torch.empty(im * jm if implicit else 1, dtype=torch.float32, device=dev)
        aws.pcg_x = xfix.data_ptr() if implicit else None
        fa = _abi.FieldArray(*[work.views[n].data_ptr() for n in names])
        ga = _abi.FieldArray(*[G.views[n].data_ptr() for n in names])
        ws = core._workspace()
        st = torch.cuda.current_stream(dev)
        fn = lib.npom_step_explicit_adjoint if core.core_name == "explicit" else lib.npom_step_implicit_adjoint
        for n in reversed(range(ctx.nsteps)):
            work.flat[:ndyn].copy_(ckpt[n])
            if implicit:
                xfix.copy_(xck[n])
            clk = _abi.NpomClock(float(ctx.time0), int(n + 1), 1)
            status = fn(ctypes.byref(p), ctypes.byref(fa), ctypes.byref(ws["struct"]), ctypes.byref(clk),
                        ctypes.byref(ga), ctypes.byref(aws), ctypes.c_void_p(st.cuda_stream))
            if status == 3:
                ws["ctrl"][4].zero_()
                raise FloatingPointError("step adjoint: non-finite cotangent of the free-surface solve")
            _abi.check(status, "step adjoint")
        return (None, None, None) + tuple(G.views[n].clone() for n in _abi.ADJ_STATE_FIELDS)


class _EtaSolveFunction(torch.autograd.Function):
    """The free-surface solve as an autograd node, like the reference's
    ``_ImplicitEtaSolveFunction`` (``implicit_p0_fixed/core.py:24-59``):
    gradients flow to ``rhs`` and ``d_2d``; the backward is the CUDA adjoint
    ``npom_pcg_adjoint``."""

    @staticmethod
    def forward(ctx, core, rhs, d_2d, max_iter, tol, initial_guess):
        x = core._eta_solve(rhs, d_2d, max_iter, tol, initial_guess)
        ctx.core = core
        ctx.max_iter, ctx.tol = max_iter, tol
        ctx.save_for_backward(x, d_2d)
        return x

    @staticmethod
    def backward(ctx, grad_x):
        x, d_2d = ctx.saved_tensors
        lam, grad_d = ctx.core._eta_adjoint(grad_x, x, d_2d, ctx.max_iter, ctx.tol)
        return None, lam, grad_d, None, None, None


class ImplicitCore(B200Core):
    """Semi-implicit free-surface core (reference ``cores/implicit_p0_fixed``)."""
    core_name = "implicit_p0_fixed"

    def solve_implicit_eta_cg(self, rhs, d_2d, max_iter=200, tol=1e-7, print_cg_residual=True, initial_guess=None):
        """One free-surface solve A(d_2d) x = rhs on the device, drop-in for
        ``implicit_p0_fixed/core.py:775``: warm start ``2 el - elb`` unless an
        initial guess is given, Dirichlet ring, the core's relative tolerance
        and preconditioner, iterations appended to
        ``_eta_solver_iteration_history``.  Differentiable in ``rhs`` and
        ``d_2d`` when either requires grad."""
        if torch.is_grad_enabled() and (rhs.requires_grad or d_2d.requires_grad):
            return _EtaSolveFunction.apply(self, rhs, d_2d, max_iter, tol, initial_guess)
        return self._eta_solve(rhs, d_2d, max_iter, tol, initial_guess)

    def _solver_call(self, max_iter, tol):
        lib = _abi.load_library()
        if self.device.type != "cuda":
            raise RuntimeError("the B200 core runs on CUDA devices only")
        p = self.params()
        p.eta_max_iter = int(max_iter)
        p.eta_tol = float(tol)
        return lib, p, self._fields(), self._workspace(), torch.cuda.current_stream(self.device)

    def _plane(self, t):
        return t.detach().to(device=self.device, dtype=torch.float32).reshape(self.im, self.jm).contiguous()

    def _eta_solve(self, rhs, d_2d, max_iter, tol, initial_guess):
        lib, p, fa, ws, st = self._solver_call(max_iter, tol)
        if initial_guess is not None:
            x = self._plane(initial_guess).clone()
        else:
            x = self._plane(2.0 * self.el.detach() - self.elb.detach())
        d = self._plane(d_2d)
        ws["bufs"]["rhs"].copy_(self._plane(rhs))
        fields = _abi.FieldArray(*fa)
        fields[_abi.FIELD_NAMES.index("elf")] = x.data_ptr()
        fields[_abi.FIELD_NAMES.index("d")] = d.data_ptr()
        _abi.check(lib.npom_pcg_solve(ctypes.byref(p), ctypes.byref(fields), ctypes.byref(ws["struct"]),
                                      ctypes.c_void_p(st.cuda_stream)), "npom_pcg_solve")
        self._eta_solver_iteration_history.append(int(ws["ctrl"][8].item()))
        return x

    def _eta_adjoint(self, grad_x, x, d_2d, max_iter, tol):
        lib, p, fa, ws, st = self._solver_call(max_iter, tol)
        g, xs, d = self._plane(grad_x), self._plane(x), self._plane(d_2d)
        lam = torch.empty_like(g)
        grad_d = torch.empty_like(g)
        status = lib.npom_pcg_adjoint(ctypes.byref(p), ctypes.byref(fa), ctypes.byref(ws["struct"]),
                                      ctypes.c_void_p(g.data_ptr()), ctypes.c_void_p(xs.data_ptr()),
                                      ctypes.c_void_p(d.data_ptr()), ctypes.c_void_p(lam.data_ptr()),
                                      ctypes.c_void_p(grad_d.data_ptr()), ctypes.c_void_p(st.cuda_stream))
        if status == 3:
            ws["ctrl"][4].zero_()
            raise FloatingPointError("free-surface adjoint: non-finite cotangent")
        _abi.check(status, "npom_pcg_adjoint")
        self._eta_adjoint_iteration_history.append(int(ws["ctrl"][8].item()))
        return lam, grad_d


CORE_REGISTRY = {"explicit": ExplicitCore, "implicit_p0_fixed": ImplicitCore}


def resolve_core_class(name):
    """Mirror of ``src/neuralpom/core_factory.py:resolve_core_class``."""
    if name not in CORE_REGISTRY:
        raise ValueError(f"Unsupported production core {name!r}; choose from {sorted(CORE_REGISTRY)}.")
    return CORE_REGISTRY[name]
