"""The Midtrain-shaped configuration (explicit core, 90x82x16 noise basin,
dtE = 6 s, isplit = 20, dtI = 120 s, T/S/u/v-perturbed member) at its own
size: the hand-written step adjoint against central differences of the
float64 oracle.

The window's loss is smooth only over a short horizon.  Measured on the
float64 oracle along one unit direction of (T, S, u, v): over 10 steps the
central difference is the same to 1e-7 for eps = 1e-7 and 1e-8; over 30
steps it still moves by 1e-3 between eps = 1e-6 and 1e-8, and by 40%
between eps = 1e-3 and 1e-5; over the full 90 steps eps = 1e-3 and 1e-5
give opposite signs.  The noise member drives the turbulence closure's
clamps and |.| terms and the limiters across their kinks at every
perturbation size, so a finite difference over the whole 3 h window does
not measure a derivative.  The check therefore runs the first 10 steps
(20 min, every phase of the step 10 times, 200 external substeps) at the
configuration's full size: 16 random unit directions, eps = 1e-7, within
2e-3 of the rms directional derivative (the float32 and float64 Jacobians
differ at that level), the bar of the smaller checks.
"""
import os
import tempfile

import numpy as np
import pytest
import torch

from oracle_days import fd_losses

pytestmark = pytest.mark.gpu


def test_gpu_midtrain_90x82_adjoint_matches_float64_differences():
    import bench
    from neuralpom_b200 import _abi, resolve_core_class
    A, Sc = bench.midtrain_case(0)
    im, jm, kb = A["u"].shape
    t0 = float(Sc["time"])
    steps = 10
    core = resolve_core_class("explicit").from_state(A, Sc, device="cuda")
    start = {f: getattr(core, f).detach().cpu().numpy().copy() for f in A}
    rng = np.random.default_rng(23)
    masks = {"t": start["fsm"][:, :, None], "s": start["fsm"][:, :, None], "u": start["dum"][:, :, None],
             "v": start["dvm"][:, :, None]}
    masks = {f: np.broadcast_to(m, start[f].shape).astype(np.float64) for f, m in masks.items()}
    scale = {"t": 1.0, "s": 0.1, "u": 0.01, "v": 0.01}
    target = {f: start[f] + 0.1 * scale[f] * rng.standard_normal(start[f].shape) * masks[f] for f in masks}
    leaves = {}
    for f in _abi.ADJ_STATE_FIELDS:
        leaves[f] = getattr(core, f).detach().clone().requires_grad_(True)
        setattr(core, f, leaves[f])
    core.time0, core.iend = t0, steps
    core.run_time_loop()
    loss = sum(((getattr(core, f).double() - torch.from_numpy(target[f]).cuda()) ** 2).mean() / scale[f] ** 2
               for f in target)
    loss.backward()
    grads = {f: leaves[f].grad.double().cpu().numpy() for f in target}
    dirs = []
    for _ in range(16):
        d = {f: rng.standard_normal(start[f].shape) * masks[f] * scale[f] for f in target}
        nrm = np.sqrt(sum((x ** 2).sum() for x in d.values()))
        dirs.append({f: x / nrm for f, x in d.items()})
    ads = np.array([sum(float((grads[f] * d[f]).sum()) for f in target) for d in dirs])
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "fd.npz")
        arrays = {f"start__{n}": v for n, v in start.items()}
        arrays.update({f"target__{f}": v for f, v in target.items()})
        arrays.update({f"scale__{f}": np.float64(v) for f, v in scale.items()})
        for i, d in enumerate(dirs):
            arrays.update({f"dir{i}__{f}": v for f, v in d.items()})
        np.savez(path, **arrays)
        scal = dict(Sc, im=im, jm=jm, kb=kb, time=t0, time0=t0)
        pairs = fd_losses(path, scal, "explicit", steps, len(dirs), 1e-7, workers=min(16, os.cpu_count() or 1))
    fds = np.array([(p - m) / 2e-7 for p, m in pairs])
    rms = float(np.sqrt((ads ** 2).mean()))
    err = np.abs(fds - ads) / rms
    print("midtrain 90x82 FD", fds, "adjoint", ads, "max err / rms", err.max(), "median", np.median(err))
    assert err.max() < 2e-3, (fds, ads)
