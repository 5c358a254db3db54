"""Ensembles on one GPU: members of one core, each with its own grid, state
and workspace, advanced together with one launch per phase of the internal
step (npom_step_batch) and the step replayed as one CUDA graph.

This replaces a Python loop of ``run_time_loop`` over ensemble members
(cores/explicit/time_loop.py:20, cores/implicit_p0_fixed/time_loop.py:38).
Each member computes what it computes when advanced alone: bitwise, except
semi-implicit members whose interior is too large for the one-cluster PCG
(their cooperative PCG sums its FP64 dot products over a different block
count, so they agree to rounding).
"""
from __future__ import annotations

import ctypes

import torch

from . import _abi

MAX_BATCH = 64


def _member_args(cores):
    if not cores:
        raise ValueError("an empty batch")
    if len(cores) > MAX_BATCH:
        raise ValueError(f"at most {MAX_BATCH} members per call, got {len(cores)}")
    kinds = {c.core_name for c in cores}
    devices = {c.device for c in cores}
    if len(kinds) != 1:
        raise ValueError(f"members of one core kind per call, got {sorted(kinds)}")
    if len(devices) != 1 or next(iter(devices)).type != "cuda":
        raise ValueError("members must live on one CUDA device")
    params = [c.params() for c in cores]
    fields = [c._fields() for c in cores]
    wss = [c._workspace()["struct"] for c in cores]
    return params, fields, wss


def launch_batch(cores, nsteps, time0, first_iint=1, stream=None):
    """Enqueue ``nsteps`` internal steps of every core in ``cores`` (one core
    kind, one device, one clock) on ``stream`` without waiting.  Steps are
    taken in calls of at most MAX_STEPS_PER_CALL (the length of each
    member's PCG iteration record).  Returns the number of kernels the
    calls launched."""
    from .core import MAX_STEPS_PER_CALL
    lib = _abi.load_library()
    params, fields, wss = _member_args(cores)
    n = len(cores)
    p_arr = (ctypes.c_void_p * n)(*[ctypes.addressof(p) for p in params])
    f_arr = (ctypes.c_void_p * n)(*[ctypes.addressof(f) for f in fields])
    w_arr = (ctypes.c_void_p * n)(*[ctypes.addressof(w) for w in wss])
    st = stream if stream is not None else torch.cuda.current_stream(cores[0].device)
    done, launches = 0, 0
    while done < nsteps:
        k = min(MAX_STEPS_PER_CALL, nsteps - done)
        clk = _abi.NpomClock(float(time0), int(first_iint + done), int(k))
        _abi.check(lib.npom_step_batch(n, p_arr, f_arr, w_arr, ctypes.byref(clk), ctypes.c_void_p(st.cuda_stream)),
                   "npom batch step")
        launches += int(lib.npom_batch_launches())
        done += k
    return launches


def run_batch(cores):
    """``run_time_loop`` of every member at once: each core advances its
    ``iend`` internal steps from ``time0`` (the members share both) and its
    clock, ramp and PCG history are updated as ``run_time_loop`` updates
    them; raises like ``run_time_loop`` for the first member whose status
    reports a velocity above vmaxl, a non-finite elevation or a timeout."""
    ends = {int(c.iend) for c in cores}
    starts = {float(c.time0) for c in cores}
    if len(ends) != 1 or len(starts) != 1:
        raise ValueError("batch members advance over one clock: iend and time0 must agree")
    steps, t0 = ends.pop(), starts.pop()
    if steps < 0:
        raise ValueError("iend must be non-negative")
    with torch.no_grad():
        launch_batch(cores, steps, t0)
    for c in cores:
        bits, its = c.read_status(steps)
        c._finish_advance(steps, bits, its)
