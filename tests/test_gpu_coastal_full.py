"""The coastal tide configuration (354x322x16, dx = 500 m, open southern
boundary with the Flather condition) at its own size: the hand-written step
adjoint against central differences of the float64 oracle.

From a developed state (three steps after the internal mode starts), two
differentiable steps, loss = MSE of u, v, T, S against a seeded target; the
CUDA gradient along 4 random unit directions of (T, S, u, v) against central
differences (eps = 1e-3) of the oracle in float64, within 2e-3 of the rms
directional derivative -- the bar of the 150x120 check, here on the full
grid (1.82 M cells per level set, the large-grid kernel forms throughout).
The adjoint through the open boundary has no reference counterpart (the
reference's adapters forbid gradients there), so differences of the float64
restatement are the check.
"""
import os
import tempfile

import numpy as np
import pytest
import torch

from oracle_days import fd_losses

pytestmark = pytest.mark.gpu


def test_gpu_coastal_354x322_step_adjoint_matches_float64_differences():
    from neuralpom_b200 import _abi, cases, resolve_core_class
    A, Sc = cases.coastal_tide(354, 322)
    Sc = dict(Sc, time=0.25, time0=0.25)
    im, jm, kb = A["u"].shape
    core = resolve_core_class("explicit").from_state(A, Sc, device="cuda")
    core.time0, core.iend = 0.25, 3
    with torch.no_grad():
        core.run_time_loop()
    t0 = float(core.time)
    start = {f: getattr(core, f).detach().cpu().numpy().copy() for f in A}
    rng = np.random.default_rng(11)
    masks = {"t": start["fsm"][:, :, None], "s": start["fsm"][:, :, None], "u": start["dum"][:, :, None],
             "v": start["dvm"][:, :, None]}
    masks = {f: np.broadcast_to(m, start[f].shape).astype(np.float64) for f, m in masks.items()}
    scale = {"t": 1.0, "s": 0.1, "u": 0.01, "v": 0.01}
    target = {f: start[f] + 0.1 * scale[f] * rng.standard_normal(start[f].shape) * masks[f] for f in masks}
    leaves = {}
    for f in _abi.ADJ_STATE_FIELDS:
        leaves[f] = getattr(core, f).detach().clone().requires_grad_(True)
        setattr(core, f, leaves[f])
    core.time0, core.iend = t0, 2
    core.run_time_loop()
    loss = sum(((getattr(core, f).double() - torch.from_numpy(target[f]).cuda()) ** 2).mean() / scale[f] ** 2
               for f in target)
    loss.backward()
    grads = {f: leaves[f].grad.double().cpu().numpy() for f in target}
    dirs = []
    for _ in range(4):
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
        pairs = fd_losses(path, scal, "explicit", 2, len(dirs), 1e-3, workers=min(8, os.cpu_count() or 1))
    fds = np.array([(p - m) / 2e-3 for p, m in pairs])
    rms = float(np.sqrt((ads ** 2).mean()))
    print("coastal 354x322 FD", fds, "adjoint", ads, "max err / rms", np.abs(fds - ads).max() / rms)
    assert np.abs(fds - ads).max() / rms < 2e-3, (fds, ads)
