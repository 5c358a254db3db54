"""On-disk formats around the B200 cores: restart capture/restore and the
reference ensembles' NPZ states.

* ``capture``/``restore``/``save_restart``/``load_restart`` follow the
  reference's complete-state restart (``src/neuralpom/v1/checkpoint.py:51-95``):
  every tensor and scalar of the core is saved, only computational scratch
  (the CUDA workspace, solver histories) is rebuilt, and an attribute of an
  unknown type is an error rather than silently lost state.
* ``FixedCoreDataset`` reads the reference's downsampled ensemble layout
  (``src/neuralpom/v1/data.py:14-126``): a manifest and per-member provenance
  that must name the registered core and its numerics version, initial
  states ``checkpoint_DayNNNN.npz`` and intraday labels every 20 min over the
  first 4 h, each stamped with its model time.
* ``inject_core_state`` loads such a state into a core
  (``src/neuralpom/hybrid/state.py:228-306``): the 43 named fields, the
  previous-time-level fallbacks, and the checkpoint clock.
"""
from __future__ import annotations

import copy
import json
import os
from pathlib import Path

import numpy as np
import torch

from .core import NUMERICS_VERSION

# Attributes rebuilt on restore instead of saved.
SCRATCH = frozenset({"device", "_ws", "_ws_key", "_ws_geo", "tuning", "_eta_solver_iteration_history",
                     "_eta_adjoint_iteration_history"})


def _scratch(name):
    return name in SCRATCH


def capture(core, cpu=True):
    """Complete physical state of a core: {"tensors", "scalars", "objects",
    "complete": True}.  Raises TypeError on an attribute of unknown type."""
    tensors, scalars = {}, {}
    for name, value in vars(core).items():
        if _scratch(name):
            continue
        if torch.is_tensor(value):
            tensors[name] = value.detach().to("cpu" if cpu else value.device).clone()
        elif value is None or isinstance(value, (bool, int, float, str, np.generic)):
            scalars[name] = value.item() if isinstance(value, np.generic) else value
        else:
            raise TypeError(f"Unclassified physical state {name}: {type(value).__name__}")
    return {"tensors": tensors, "scalars": scalars, "objects": {}, "complete": True}


def restore(core, state):
    """Put a captured state back: attributes the state does not hold are
    removed, tensors go to the core's device, the workspace is rebuilt."""
    if state.get("complete") is not True:
        raise ValueError("Restart requires a complete physical state")
    device = core.device
    saved = set(state["tensors"]) | set(state["scalars"]) | set(state.get("objects", {}))
    for name in list(vars(core)):
        if not _scratch(name) and name not in saved:
            delattr(core, name)
    for name, value in state["tensors"].items():
        setattr(core, name, value.detach().to(device).clone())
    for section in ("scalars", "objects"):
        for name, value in state.get(section, {}).items():
            setattr(core, name, copy.deepcopy(value))
    core.device = device
    core._ws = None
    core._ws_key = None
    core._ws_geo = None
    core._eta_solver_iteration_history = []
    core._eta_adjoint_iteration_history = []


def _atomic(path, write):
    path = Path(path)
    path.parent.mkdir(parents=True, exist_ok=True)
    tmp = path.with_name(f"{path.name}.{os.getpid()}.tmp")
    write(tmp)
    os.replace(tmp, path)


def save_restart(path, core):
    """Capture to CPU and write atomically (temporary file + rename)."""
    state = capture(core, cpu=True)
    _atomic(path, lambda tmp: torch.save(state, tmp))


def load_restart(path, core):
    restore(core, torch.load(path, map_location="cpu", weights_only=False))


# ---------------------------------------------------------------------------
# reference ensemble states
# ---------------------------------------------------------------------------
CORE = "implicit_p0_fixed"
# model-time stamps of the fine-step source drift by ~1e-7 day by day 9000
NOMINAL_CLOCK_TOL_DAYS = 2e-7
LABEL_FIELDS = ("u", "ub", "v", "vb", "t", "s", "el", "ua", "uab", "va", "vab")
INITIAL_3D_FIELDS = ("u", "ub", "v", "vb", "t", "tb", "s", "sb", "q2", "q2b", "q2l", "q2lb", "km", "kh", "kq",
                     "aam", "rho", "w")
INITIAL_2D_FIELDS = ("el", "elb", "et", "etb", "etf", "ua", "uab", "va", "vab", "utf", "utb", "vtf", "vtb", "adx2d",
                     "ady2d", "drx2d", "dry2d", "vfluxf", "vfluxb", "wubot", "wvbot", "egb", "uaf", "vaf", "elf")
# explicit source trajectories: dtE = 5 s, isplit = 30, dtI = 150 s
EXPLICIT_SOURCE_CLOCK = {"dte_seconds": 5.0, "isplit": 30, "dti_seconds": 150.0}
SPEC = {"explicit": {"alpha": 0.225, "smoth": 0.10, "horcon": 0.05},
        "implicit_p0_fixed": {"alpha": 0.333, "smoth": 0.15, "horcon": 0.05}}


class FixedCoreDataset:
    """Initial states and labels of the reference's downsampled ensembles,
    indexed by model time (day d's initial state is the checkpoint written
    at the end of day d-1)."""

    def __init__(self, root, frequency_seconds=86400, core_name=CORE):
        if core_name not in NUMERICS_VERSION:
            raise ValueError(f"Unknown core {core_name!r}")
        self.root = Path(root)
        self.core_name = core_name
        self.numerics_version = NUMERICS_VERSION[core_name]
        self.frequency_seconds = int(frequency_seconds)
        if self.frequency_seconds not in (3600, 86400):
            raise ValueError("Correction interval must be 1 h or 1 day")
        m = json.loads((self.root / "manifest.json").read_text())
        self.manifest = m
        if (m.get("generation_core_requested") != core_name or
                m.get("generation_core_numerics_version") != self.numerics_version):
            raise ValueError("Dataset does not match the registered dynamical core")
        if core_name == CORE and str(m.get("implicit_spatial_shapiro_requested", "")).lower() not in (
                "0", "false", "off", "no"):
            raise ValueError("The implicit data must be generated with the spatial Shapiro filter off")
        if core_name == "explicit":
            integ = m.get("integration", {})
            if any(integ.get(k) != v for k, v in EXPLICIT_SOURCE_CLOCK.items()):
                raise ValueError("Explicit source trajectory has the wrong time split")
        down = m.get("downsampling", {})
        self.grid = tuple(down.get("coarse_grid", (90, 82))) + (16,)
        self.algorithm = down.get("algorithm")
        self._verified = set()

    def _member(self, member):
        if not isinstance(member, int) or not 0 <= member < 8:
            raise ValueError("Member must be an integer in [0, 7]")
        base = self.root / f"member_{member}_gpu{member}"
        if member in self._verified:
            return base
        prov = json.loads((base / "provenance.json").read_text())
        if (prov.get("member") != member or prov.get("core_requested") != self.core_name or
                prov.get("core_numerics_version") != self.numerics_version):
            raise ValueError(f"Member core provenance mismatch: {base}")
        num = prov.get("resolved_numerics", {})
        if self.core_name == CORE:
            gammas = ("barotropic_shapiro_gamma", "tracer_shapiro_gamma", "velocity_shapiro_gamma")
            if num.get("spatial_shapiro_enabled") is not False or any(num.get(k) != 0.0 for k in gammas):
                raise ValueError(f"Member data requires the spatial Shapiro filter off: {base}")
        else:
            want = dict(SPEC["explicit"], **EXPLICIT_SOURCE_CLOCK)
            if any(num.get(k) != v for k, v in want.items()):
                raise ValueError(f"Explicit member numerical settings mismatch: {base}")
        if self.algorithm is not None and prov.get("downsampling_algorithm") != self.algorithm:
            raise ValueError(f"Member downsampling differs from the dataset manifest: {base}")
        self._verified.add(member)
        return base

    def initial_path(self, member, model_day):
        if int(model_day) != model_day or not 1 <= model_day <= 9000:
            raise ValueError("Initial model day must be an integer in [1, 9000]")
        return self._member(member) / "checkpoints_lowres_consistent" / f"checkpoint_Day{int(model_day) - 1:04d}.npz"

    def label_path(self, member, model_day, lead_seconds):
        if int(model_day) != model_day or lead_seconds < 0 or int(lead_seconds) != lead_seconds:
            raise ValueError("Labels require integer model days and non-negative integer lead seconds")
        days, within = divmod(int(lead_seconds), 86400)
        day = int(model_day) + days
        if within == 0:
            return self.initial_path(member, day)
        if within > 14400 or within % 1200:
            raise ValueError("Intraday labels exist only every 20 min over the first 4 h")
        if not 0 <= day <= 8999:
            raise ValueError("Reference day outside the registered coverage")
        seg = within // 1200 - 1
        return self._member(member) / "reference_data_lowres_consistent" / f"ref_Day{day:04d}_seg{seg:02d}.npz"

    @staticmethod
    def _read(path, expected_time, map_location, fields=None):
        with np.load(path, allow_pickle=False) as z:
            if "time" not in z.files or abs(float(z["time"]) - expected_time) > NOMINAL_CLOCK_TOL_DAYS:
                raise ValueError(f"Reference clock mismatch: {path}; expected {expected_time}")
            keys = z.files if fields is None else (*fields, "time")
            out = {k: torch.as_tensor(z[k].copy(), device=map_location,
                                      dtype=torch.float64 if k == "time" else torch.float32) for k in keys}
        if not all(bool(torch.isfinite(v).all()) for v in out.values()):
            raise ValueError(f"Non-finite reference: {path}")
        return out

    def _check(self, state, initial):
        f3 = INITIAL_3D_FIELDS if initial else LABEL_FIELDS[:6]
        f2 = INITIAL_2D_FIELDS if initial else LABEL_FIELDS[6:]
        scal = ("time", "iint") if initial else ("time",)
        missing = set((*f3, *f2, *scal)) - set(state)
        if missing:
            raise ValueError(f"Missing required physical fields: {sorted(missing)}")
        for f in (*f3, *f2, *scal):
            want = self.grid if f in f3 else (self.grid[:2] if f in f2 else ())
            if tuple(state[f].shape) != want:
                raise ValueError(f"Physical field {f} shape {tuple(state[f].shape)} != {want}")
        return state

    def load_initial(self, member, model_day, map_location="cpu"):
        return self._check(self._read(self.initial_path(member, model_day), float(model_day), map_location), True)

    def load_target(self, member, model_day, lead_seconds, map_location="cpu"):
        s = self._read(self.label_path(member, model_day, lead_seconds), model_day + lead_seconds / 86400.0,
                       map_location, LABEL_FIELDS)
        return self._check(s, False)

    target = load_target


# Fields a state injection writes (target attribute, source key) and the
# previous-time-level fallbacks when a source holds only the current level.
INJECTION_FIELDS = ("u", "ub", "v", "vb", "t", "tb", "s", "sb", "el", "elb", "ua", "uab", "va", "vab", "q2", "q2b",
                    "q2l", "q2lb", "km", "kh", "kq", "rho", "w", "et", "etb", "etf", "utf", "utb", "vtf", "vtb",
                    "adx2d", "ady2d", "aam", "vfluxf", "vfluxb", "wubot", "wvbot", "egb", "drx2d", "dry2d", "uaf",
                    "vaf", "elf")
STATE_FALLBACKS = {"ub": "u", "vb": "v", "tb": "t", "sb": "s", "elb": "el", "uab": "ua", "vab": "va", "q2b": "q2",
                   "q2lb": "q2l"}
OPTIONAL_ZERO_FIELDS = frozenset({"drx2d", "dry2d"})


def inject_core_state(core, ics, sample_index=None, start_day=None):
    """Write the state ``ics`` (one state, or a batch with ``sample_index``)
    into the core in place and set its clock from the state's ``time`` (or
    ``start_day``), both in days."""
    for name in INJECTION_FIELDS:
        target = getattr(core, name, None)
        if target is None:
            continue
        key = name if name in ics else STATE_FALLBACKS.get(name)
        if key is None or key not in ics:
            if name in OPTIONAL_ZERO_FIELDS:
                setattr(core, name, torch.zeros_like(target))
            continue
        value = ics[key]
        if sample_index is not None and torch.is_tensor(value) and value.dim() > target.dim():
            value = value[sample_index]
        value = torch.as_tensor(value).detach().clone().to(core.device)
        if value.dim() > target.dim() and value.shape[0] == 1:
            value = value.squeeze(0)
        if value.shape != target.shape:
            if value.numel() != target.numel():
                continue
            value = value.view_as(target)
        if value.dtype == target.dtype and value.device == target.device:
            target.detach_()
            target.copy_(value)
        else:
            setattr(core, name, value)
    clock = ics.get("time")
    if clock is not None:
        if torch.is_tensor(clock):
            clock = clock.detach()
            if sample_index is not None and clock.dim() > 0:
                if sample_index >= clock.shape[0]:
                    raise IndexError(f"sample_index={sample_index} is out of range for the clock {tuple(clock.shape)}")
                clock = clock[sample_index]
            if clock.numel() != 1:
                raise ValueError(f"The clock must hold one value per sample, got {tuple(clock.shape)}")
            days = float(clock.item())
        else:
            days = float(clock)
    elif start_day is not None:
        days = float(start_day)
    else:
        days = None
    if days is not None:
        if not np.isfinite(days):
            raise ValueError(f"The clock must be finite, got {days}")
        core.time = days
        core.time0 = days
        core.iint = 0
