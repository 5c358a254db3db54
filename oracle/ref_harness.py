"""Drive the unmodified reference PyTorch core -- TEST INFRASTRUCTURE ONLY.

Used to (a) generate the golden vectors under ``tests/golden/`` and (b) time
the reference's own CPU implementation in ``bench.py --impl reference``.  The
reference package is imported from a source tree (``<ref>/src``) or from a
``pip install --target`` directory; its modules import ``netCDF4`` without
using it, so an empty stand-in module is registered when the real one is
missing.
"""
from __future__ import annotations

import importlib
import os
import sys
import types

import numpy as np


def import_reference(path):
    """Make ``neuralpom`` importable from ``path`` (a ``src`` dir or a pip
    ``--target`` dir) and return the module."""
    if "netCDF4" not in sys.modules:
        try:
            importlib.import_module("netCDF4")
        except ModuleNotFoundError:
            sys.modules["netCDF4"] = types.ModuleType("netCDF4")
    if path not in sys.path:
        sys.path.insert(0, path)
    return importlib.import_module("neuralpom")


def default_reference_path():
    """The reference package location: ``NPOM_REFERENCE_SRC`` (a ``src``
    directory of the reference sources) if set, else the ``pip install
    --target baseline/_ref`` copy next to this repository; None if neither
    holds the ``neuralpom`` package."""
    for cand in (os.environ.get("NPOM_REFERENCE_SRC", ""),
                 os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "baseline", "_ref")):
        if cand and os.path.isdir(os.path.join(cand, "neuralpom")):
            return cand
    return None


SCALAR_NAMES = (
    "im", "jm", "kb", "dti", "dte", "dti2", "dte2", "isplit", "ispi", "isp2i", "alpha", "smoth",
    "horcon", "grav", "umol", "tprni", "small", "kappa", "rhoref", "tbias", "sbias", "ramp", "vmaxl",
    "hmax", "rfe", "rfw", "rfn", "rfs", "nbct", "nbcs", "ntp", "mode", "nadv", "ispadv", "period",
    "lramp", "time", "time0", "iint", "aam_min", "pi",
)
IMPLICIT_SCALARS = ("eta_solver_rel_tol", "eta_solver_preconditioner", "barotropic_shapiro",
                    "tracer_shapiro", "velocity_shapiro")


def build_reference_core(name, im, jm, device="cpu"):
    """Reference core built and configured like production
    (``hybrid/core_pool.py:build_initialized_core`` + ``v1/core_spec.py``)."""
    import torch
    from neuralpom.hybrid import build_initialized_core
    from neuralpom.v1.core_spec import core_spec
    spec = core_spec(name)
    core = build_initialized_core(spec.core_class, torch.device(device), im, jm)
    spec.configure(core)
    return core


def extract_state(core):
    """Float tensor attributes as float numpy arrays, plus scalars."""
    import torch
    arrays = {}
    for k, v in vars(core).items():
        if torch.is_tensor(v) and v.is_floating_point() and not k.startswith("_"):
            arrays[k] = v.detach().cpu().numpy().copy()
    # the coastal tide policy's table (coastal_boundary.py:55-65), 0-based
    for k in ("_tide_i", "_tide_j", "_tide_amp", "_tide_phase"):
        if torch.is_tensor(getattr(core, k, None)):
            arrays[k[1:]] = getattr(core, k).detach().cpu().numpy().astype(np.float32)
    scalars = {}
    # case-policy settings a harness puts on a core (the POM08-WAD closure)
    for k in SCALAR_NAMES + IMPLICIT_SCALARS + ("profq_form", "zsh", "obc_form"):
        if hasattr(core, k):
            val = getattr(core, k)
            if isinstance(val, (bool, int, float, str)):
                scalars[k] = val
    return arrays, scalars


def load_state(core, arrays, scalars=None):
    """Overwrite the reference core's tensors (and scalars) with ``arrays``."""
    import torch
    dev = core.device
    for k, v in arrays.items():
        cur = getattr(core, k, None)
        dtype = cur.dtype if torch.is_tensor(cur) else torch.float32
        setattr(core, k, torch.as_tensor(np.ascontiguousarray(v), dtype=dtype, device=dev).clone())
    for k, v in (scalars or {}).items():
        setattr(core, k, v)
    # caches derived from geometry must be rebuilt for the implicit core
    if hasattr(core, "_accel_cache_ready"):
        core._accel_cache_ready = False
        core._spectral_eta_preconditioner_cache = None
        if hasattr(core, "_build_acceleration_cache"):
            core._build_acceleration_cache()


def advance(core, name, steps, differentiable=False, device="cpu", **physics_kw):
    """``SparsePhysics.advance`` with the production options of each core."""
    from neuralpom.hybrid.sparse_physics import SparsePhysics
    kw = dict(core_name="explicit", compiled_kernels=()) if name == "explicit" else {}
    kw.update(physics_kw)
    SparsePhysics(device, **kw).advance(core, steps=steps, differentiable=differentiable)


class ReferenceFloat64:
    """Context in which the reference core computes in float64: the
    default dtype is float64 and the float32 scratch its step allocates
    explicitly (explicit/momentum.py:25-28,144-147,555-556 and the tracer
    routines) is allocated as float64 instead.  The core's own tensors are
    promoted by ``promote``."""

    NAMES = ("zeros", "ones", "empty", "full", "tensor", "arange", "linspace", "zeros_like", "ones_like",
             "empty_like", "full_like", "as_tensor")

    def __enter__(self):
        import torch
        self.torch = torch
        self.saved = {n: getattr(torch, n) for n in self.NAMES}

        def wrap(fn):
            def alloc(*a, **k):
                if k.get("dtype") is torch.float32:
                    k["dtype"] = torch.float64
                return fn(*a, **k)
            return alloc
        self.prev = torch.get_default_dtype()
        for n in self.NAMES:
            setattr(torch, n, wrap(self.saved[n]))
        torch.set_default_dtype(torch.float64)
        return self

    def __exit__(self, *exc):
        for n, fn in self.saved.items():
            setattr(self.torch, n, fn)
        self.torch.set_default_dtype(self.prev)

    @staticmethod
    def promote(core):
        import torch
        for k, v in list(vars(core).items()):
            if torch.is_tensor(v) and v.dtype == torch.float32:
                setattr(core, k, v.to(torch.float64))
        # solver caches are rebuilt from the promoted geometry
        core._accel_cache_ready = False
        core._spectral_eta_preconditioner_cache = None
        core._cg_work = {}
