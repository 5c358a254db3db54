"""Launch-shape autotuner of the B200 step.

The step's kernels have several launch shapes that compute the same values
(``npom_tuning`` in ``include/npom.h``): point kernels or flux-once tiles
for A1 (advct) and B5 (advt1) with their rows per tile, 16 lanes or one
thread per column for the column phases, the explicit subcycle on one
cluster, a grid barrier or one launch per substep phase, the PCG's cluster
forms and CTA count or the cooperative grid, and for an ensemble the cap on
each member's cooperative-PCG blocks.  The library picks them by fixed
rules; this module measures the alternatives on the actual grid and device
and keeps the fastest.

* ``search(measure, space)`` -- coordinate descent: starting from the
  library's rules, each knob in turn takes every value of its range with the
  others fixed, and the fastest setting (by more than ``min_gain``) stays.
* ``tune(core)`` -- times ``steps`` internal steps of the core from its
  current state for every candidate (CUDA events, the median of ``reps``),
  restores the state after each, then checks the winner against the rules:
  the fields after the same steps must be equal bit for bit (every form in
  the search space computes the same values).
* The winners are cached in a JSON file keyed on device, core, grid and the
  settings that change the step's kernels (``NPOM_TUNING_CACHE``, default
  ``~/.cache/neuralpom_b200/tuning.json``); ``apply(core)`` gives a core its
  cached tuning, ``tuned(core)`` tunes on a cache miss.

The reference has no counterpart: its step is a sequence of PyTorch
operators with no launch shapes to choose.
"""
from __future__ import annotations

import json
import os
import statistics
import time

from . import _abi

# knob -> values tried (0 = the library's rule)
SPACE = {
    "a1_form": (0, 1, 2),
    "b5_form": (0, 1, 2),
    "tile_blocks_per_sm": (0, 8, 32),
    "column_form": (0, 1, 2),
    "subcycle_form": (0, 2, 3),
    # the cooperative-grid PCG (3) is left to the rules, which pick it where
    # no cluster layout fits: it sums its FP64 dot products over its blocks,
    # so it agrees with the cluster forms only to rounding
    "pcg_form": (0, 1, 2),
    "pcg_ctas": (0, 16),
}
BATCH_SPACE = dict(SPACE, batch_pcg_blocks=(0, 32, 40, 56, 64, 112))


def space_for(core, batch=False):
    """The knobs that change anything for this core's step."""
    space = dict(BATCH_SPACE if batch else SPACE)
    kb16 = int(core.kb) == 16
    explicit = core.core_name == "explicit"
    if not kb16:
        for k in ("a1_form", "b5_form", "tile_blocks_per_sm", "column_form"):
            space.pop(k)
    if explicit:
        for k in ("pcg_form", "pcg_ctas", "batch_pcg_blocks"):
            space.pop(k, None)
    else:
        space.pop("subcycle_form")
    if int(getattr(core, "nadv", 1)) == 2:
        space.pop("b5_form", None)
    return space


def search(measure, space, base=None, min_gain=0.02, log=None):
    """Coordinate descent over ``space`` ({knob: values}); ``measure(tuning)``
    returns a time.  Returns (best tuning, its time, time of ``base``)."""
    best = dict(base or {})
    t_base = t_best = measure(dict(best))
    if log is not None:
        log.append((dict(best), t_best))
    for knob, values in space.items():
        for v in values:
            if best.get(knob, 0) == v:
                continue
            cand = dict(best)
            if v:
                cand[knob] = v
            else:
                cand.pop(knob, None)
            t = measure(cand)
            if log is not None:
                log.append((dict(cand), t))
            if t < t_best * (1.0 - min_gain):
                best, t_best = cand, t
    return best, t_best, t_base


def _snapshot(core):
    return {n: getattr(core, n).detach().clone() for n in _abi.FIELD_NAMES}


def _restore(core, snap):
    import torch
    with torch.no_grad():
        for n, t in snap.items():
            getattr(core, n).copy_(t)


def _advance(core, steps, time0):
    import torch
    with torch.no_grad():
        core.launch_steps(steps, time0, 1, torch.cuda.current_stream(core.device))


def measure_core(core, tuning, steps=4, reps=3):
    """Median milliseconds per internal step of ``core`` under ``tuning``
    (CUDA events around ``steps`` steps, after one untimed call that builds
    the step's graph); the core's state is restored afterwards."""
    import torch
    snap = _snapshot(core)
    saved = getattr(core, "tuning", None)
    core.tuning = dict(tuning)
    t0 = float(core.time)
    try:
        _advance(core, steps, t0)
        times = []
        for _ in range(reps):
            _restore(core, snap)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            _advance(core, steps, t0)
            b.record()
            b.synchronize()
            times.append(a.elapsed_time(b) / steps)
        bits, _ = core.read_status(0)
        if bits & (_abi.DEV_TIMEOUT | _abi.DEV_VMAX | _abi.DEV_NONFINITE):
            return float("inf")
        return statistics.median(times)
    finally:
        _restore(core, snap)
        core.tuning = saved


def same_result(core, tuning, steps=4, rel_tol=None):
    """True if ``steps`` steps under ``tuning`` give the fields the library's
    rules give (bit for bit; within ``rel_tol`` of max|field| if given)."""
    import torch
    snap = _snapshot(core)
    saved = getattr(core, "tuning", None)
    t0 = float(core.time)
    outs = []
    try:
        for t in ({}, tuning):
            _restore(core, snap)
            core.tuning = dict(t)
            _advance(core, steps, t0)
            torch.cuda.synchronize(core.device)
            outs.append({n: getattr(core, n).detach().clone() for n in _abi.ADJ_STATE_FIELDS})
            core.read_status(0)
    finally:
        _restore(core, snap)
        core.tuning = saved
    for n in outs[0]:
        a, b = outs[0][n], outs[1][n]
        if rel_tol is None:
            if not torch.equal(a, b):
                return False
        else:
            den = float(a.abs().max())
            if den > 0 and float((a - b).abs().max()) > rel_tol * den:
                return False
    return True


def tune(core, steps=4, reps=3, min_gain=0.02, check=True):
    """Search the launch shapes of ``core``'s step; returns (tuning, report).
    The winner falls back to the rules if it does not reproduce them."""
    log = []
    best, t_best, t_base = search(lambda t: measure_core(core, t, steps, reps), space_for(core),
                                  min_gain=min_gain, log=log)
    checked = True
    if check and best:
        checked = same_result(core, best, steps)
        if not checked:
            best, t_best = {}, t_base
    return best, {"rule_ms_per_step": t_base, "tuned_ms_per_step": t_best, "candidates": len(log),
                  "reproduces_rules": checked, "tried": [[t, ms] for t, ms in log]}


# ---------------------------------------------------------------------------
# cache
# ---------------------------------------------------------------------------

def cache_path():
    return os.environ.get("NPOM_TUNING_CACHE") or os.path.join(os.path.expanduser("~"), ".cache", "neuralpom_b200",
                                                                 "tuning.json")


def device_name(device):
    import torch
    return torch.cuda.get_device_name(device)


def key_of(core, device=None):
    """Cache key: device name, core, grid and the settings that change the
    step's kernels."""
    dev = device_name(device if device is not None else core.device)
    pre = str(getattr(core, "eta_solver_preconditioner", "spectral")) if core.core_name != "explicit" else "-"
    return (f"{dev}|{core.core_name}|{core.im}x{core.jm}x{core.kb}|nadv{int(getattr(core, 'nadv', 1))}"
            f"|mode{int(getattr(core, 'mode', 3))}|{pre}")


def load(path=None):
    path = path or cache_path()
    try:
        with open(path) as f:
            data = json.load(f)
        return data if isinstance(data, dict) else {}
    except (OSError, ValueError):
        return {}


def store(key, tuning, report, path=None):
    """Write one entry (atomically: temporary file and rename)."""
    path = path or cache_path()
    data = load(path)
    data[key] = {"tuning": {k: int(v) for k, v in tuning.items()},
                 "rule_ms_per_step": report.get("rule_ms_per_step"),
                 "tuned_ms_per_step": report.get("tuned_ms_per_step"), "when": time.strftime("%Y-%m-%d %H:%M:%S")}
    os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
    tmp = f"{path}.{os.getpid()}.tmp"
    with open(tmp, "w") as f:
        json.dump(data, f, indent=1, sort_keys=True)
    os.replace(tmp, path)
    return data[key]


def lookup(key, path=None):
    entry = load(path).get(key)
    if not entry:
        return None
    tuning = entry.get("tuning", {})
    if not isinstance(tuning, dict) or any(k not in _abi.TUNING_FIELDS for k in tuning):
        return None
    return {k: int(v) for k, v in tuning.items()}


def apply(core, path=None):
    """Give ``core`` its cached tuning; returns it (None on a cache miss)."""
    tuning = lookup(key_of(core), path)
    if tuning is not None:
        core.tuning = tuning
    return tuning


def tuned(core, path=None, **kw):
    """The cached tuning of ``core``, tuned and stored on a miss; applied to
    the core and returned."""
    tuning = apply(core, path)
    if tuning is None:
        tuning, report = tune(core, **kw)
        store(key_of(core), tuning, report, path)
        core.tuning = tuning
    return tuning
