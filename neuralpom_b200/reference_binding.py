"""The reference's own core classes with their time step on the B200 library.

A maintainer who keeps NeuralPOM's classes, executor and training loops
binds the step here: ``bound_core_class(name)`` is a subclass of the
reference's ``POM2K_Core`` (``cores/implicit_p0_fixed/core.py:62`` or
``cores/explicit/core.py:17``) whose ``run_time_loop`` runs
``npom_step_implicit`` / ``npom_step_explicit`` (and, under autograd, the
hand-written step adjoints) on the core's own tensors.  Everything else --
the constructor, set-up, operator methods, ``SparsePhysics``,
``Runtime``, restart capture -- is the reference's code.

The reference's executor picks an acceleration variant by rebinding the
instance's class (``hybrid/sparse_physics.py:74-79`` sets ``core.__class__``
to ``POM2K_Core`` or one of its compiled subclasses on every ``advance``).
That would silently put the PyTorch step back.  A bound core therefore keeps
its class when such an assignment names a class that is not itself bound:
the B200 step replaces every one of those variants, and the other settings
``_configure`` makes (solver backend, fast-path flags) concern only the
PyTorch step.  ``unbind(core)`` returns a core to the plain reference class.

Usage (the reference package must be importable)::

    from neuralpom_b200 import reference_binding as rb
    rb.register()                      # CORE_REGISTRY of core_factory.py:5 -> bound classes
    core = resolve_core_class("implicit_p0_fixed")(90, 82)   # reference constructor
    SparsePhysics("cuda").advance(core, steps=6)              # runs on the B200 library

or ``rb.bind(core)`` for a core that already exists.
"""
from __future__ import annotations

from . import _abi, state
from .core import CORE_REGISTRY as _B200_CORES

_REFERENCE_CLASSES = {
    "implicit_p0_fixed": ("neuralpom.cores.implicit_p0_fixed", "POM2K_Core"),
    "explicit": ("neuralpom.cores.explicit", "POM2K_Core"),
}
_BOUND = {}
# internal steps advanced on the device through bound cores, in this process
# (the executor runs copies of a core, so the count is kept here)
_STEPS_ON_DEVICE = [0]


class _B200StepMixin:
    """``run_time_loop`` of a reference core on the B200 library.  The
    tensors stay the reference core's attributes: a B200 host core (the
    "shadow", kept on the instance) is pointed at them for the call, and
    whatever it rebinds (the differentiable path's outputs, converted
    copies) is written back, with the clock (``iint``, ``time``, ``ramp``)
    and the PCG iteration history."""

    npom_native_step = True
    _npom_core_name = None

    def __setattr__(self, name, value):
        if name == "__class__" and isinstance(value, type) and not getattr(value, "npom_native_step", False):
            # the executor's acceleration variant: the B200 step replaces it
            return
        super().__setattr__(name, value)

    def _npom_shadow(self):
        cname = self._npom_core_name
        cls = _B200_CORES[cname]
        sh = self.__dict__.get("_npom_shadow_core")
        if sh is None:
            sh = cls.__new__(cls)
            sh.__dict__.update(state.default_scalars(cname))
            sh._ws = sh._ws_key = sh._ws_geo = None
            sh._eta_solver_iteration_history = []
            sh._eta_adjoint_iteration_history = []
            self.__dict__["_npom_shadow_core"] = sh
        for k, v in vars(self).items():
            if isinstance(v, (bool, int, float, str)) and not k.startswith("_"):
                sh.__dict__[k] = v
        sh.device = self.el.device
        sh.im, sh.jm, sh.kb = int(self.im), int(self.jm), int(self.kb)
        for n in _abi.FIELD_NAMES:
            sh.__dict__[n] = getattr(self, n)
        sh.period = self.period
        return sh

    def run_time_loop(self):
        """Advance ``iend`` internal steps from ``time0`` on the B200
        library: the reference's ``run_time_loop`` contract
        (``explicit/time_loop.py:20``, ``implicit_p0_fixed/time_loop.py:38``),
        including its exceptions and its differentiable behaviour."""
        sh = self._npom_shadow()
        sh._eta_solver_iteration_history = []
        sh.run_time_loop()
        for n in _abi.FIELD_NAMES:
            t = sh.__dict__[n]
            if t is not self.__dict__.get(n):
                setattr(self, n, t)
        self.iint, self.time, self.ramp = sh.iint, sh.time, sh.ramp
        hist = self.__dict__.get("_eta_solver_iteration_history")
        if isinstance(hist, list):
            hist.extend(sh._eta_solver_iteration_history)
        _STEPS_ON_DEVICE[0] += int(sh.iint)


def reference_core_class(core_name):
    """The reference's own core class of ``core_name``."""
    import importlib
    if core_name not in _REFERENCE_CLASSES:
        raise ValueError(f"Unsupported production core {core_name!r}; choose from {sorted(_REFERENCE_CLASSES)}.")
    mod, attr = _REFERENCE_CLASSES[core_name]
    return getattr(importlib.import_module(mod), attr)


def bound_core_class(core_name):
    """Subclass of the reference's core class whose step runs on the B200
    library (made once per core kind)."""
    if core_name not in _BOUND:
        base = reference_core_class(core_name)
        cls_name = {"implicit_p0_fixed": "B200BoundImplicitCore", "explicit": "B200BoundExplicitCore"}[core_name]
        _BOUND[core_name] = type(cls_name, (_B200StepMixin, base),
                                 {"_npom_core_name": core_name, "__module__": __name__,
                                  "__doc__": f"{base.__module__}.{base.__name__} with its run_time_loop on the "
                                             f"B200 library."})
    return _BOUND[core_name]


def bind(core):
    """Rebind an existing reference core (of either kind) to its B200-bound
    class; returns the core."""
    for name in _REFERENCE_CLASSES:
        base = reference_core_class(name)
        if isinstance(core, base):
            object.__setattr__(core, "__class__", bound_core_class(name))
            return core
    raise TypeError(f"not a reference POM core: {type(core).__name__}")


def unbind(core):
    """Return a bound core to the reference's plain class (its PyTorch step)."""
    if not isinstance(core, _B200StepMixin):
        return core
    object.__setattr__(core, "__class__", reference_core_class(core._npom_core_name))
    core.__dict__.pop("_npom_shadow_core", None)
    return core


def register():
    """Point the reference's ``CORE_REGISTRY`` (``core_factory.py:5``) at the
    bound classes, so ``resolve_core_class`` and everything built on it
    (``build_initialized_core``, ``core_spec``) make B200-bound cores."""
    import importlib
    factory = importlib.import_module("neuralpom.core_factory")
    for name in _REFERENCE_CLASSES:
        factory.CORE_REGISTRY[name] = bound_core_class(name)
    return factory.CORE_REGISTRY


def steps_on_device():
    """Internal steps that bound cores have advanced on the B200 library in
    this process (forward calls, recomputations included)."""
    return _STEPS_ON_DEVICE[0]


__all__ = ["bound_core_class", "bind", "unbind", "register", "reference_core_class", "steps_on_device"]
