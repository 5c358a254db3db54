"""The explicit step under torch autograd through the drop-in API
(``ExplicitCore.run_time_loop`` with state tensors that require grad; the
backward is the CUDA step adjoint ``npom_step_explicit_adjoint``): against
the reference's own autograd gradients (golden vectors) and against central
finite differences of the CUDA forward."""
import numpy as np
import pytest
import torch

from golden_io import directional_check, grad_check, load_adjoint_golden, load_directional_golden

pytestmark = pytest.mark.gpu



def _core(A, Sc, name="explicit"):
    from neuralpom_b200 import resolve_core_class
    return resolve_core_class(name).from_state(A, Sc, device="cuda")


def _differentiable_advance(core, nsteps, time0):
    """Leaves for every state field, ``nsteps`` steps, the leaves back."""
    from neuralpom_b200 import _abi
    leaves = {}
    for f in _abi.ADJ_STATE_FIELDS:
        leaves[f] = getattr(core, f).detach().clone().requires_grad_(True)
        setattr(core, f, leaves[f])
    core.time0 = time0
    core.iend = nsteps
    core.run_time_loop()
    return leaves


ADJOINT_CASES = [("step_adjoint_explicit_12x10.npz", "cluster"), ("step_adjoint_explicit_12x10.npz", "phases"),
                 ("step_adjoint_explicit_12x10.npz", "grid"),
                 ("step_adjoint_rest_12x10.npz", "cluster"), ("step_adjoint_rest_12x10.npz", "phases"),
                 ("step_adjoint_coastal_16x14.npz", "cluster"), ("step_adjoint_coastal_16x14.npz", "phases"),
                 ("step_adjoint_coastal_16x14.npz", "grid"),
                 ("step_adjoint_implicit_12x10.npz", "-"), ("step_adjoint_implicit_rest_12x10.npz", "-")]


def _core_name(fname):
    return "implicit_p0_fixed" if "implicit" in fname else "explicit"


@pytest.mark.parametrize("fname,ext", ADJOINT_CASES)
def test_gpu_step_adjoint_matches_reference_autograd(monkeypatch, fname, ext):
    """Both cores; for the explicit one every form of the external-subcycle
    adjoint (the two fused kernels on one thread-block cluster or as
    cooperative grid launches, one launch per substep phase)."""
    if ext != "-":
        monkeypatch.setenv("NPOM_ADJ_EXT", ext)
    A, Sc, cot, grads = load_adjoint_golden(fname)
    for n, ref in sorted(grads.items()):
        core = _core(A, Sc, _core_name(fname))
        leaves = _differentiable_advance(core, n, float(Sc["time"]))
        loss = sum((getattr(core, f) * torch.from_numpy(c).cuda()).sum() for f, c in cot.items())
        loss.backward()
        got = {f: (leaves[f].grad.cpu().numpy() if leaves[f].grad is not None else np.zeros_like(A[f]))
               for f in ref}
        assert grad_check(got, ref) == [], (fname, n, grad_check(got, ref))


@pytest.mark.parametrize("fname", ["step_adjoint_mpdata_12x10.npz", "step_adjoint_mpdata_implicit_12x10.npz"])
def test_gpu_mpdata_step_adjoint_matches_reference_float64_differences(fname):
    """MPDATA tracer advection (nadv = 2), both cores: the CUDA step adjoint
    of 1 and 3 steps (1 and 2 semi-implicit) along the golden's seeded
    directions against central differences of the reference's forward in
    float64, the bar of the emulated adjoint (of sum |g * d|: 2e-3 after
    one step, 2e-2 after more)."""
    A, Sc, cot, grads = load_adjoint_golden(fname)
    dirs = load_directional_golden(fname)
    assert int(Sc["nadv"]) == 2
    for n, per_field in sorted(dirs.items()):
        core = _core(A, Sc, _core_name(fname))
        leaves = _differentiable_advance(core, n, float(Sc["time"]))
        loss = sum((getattr(core, f) * torch.from_numpy(c).cuda()).sum() for f, c in cot.items())
        loss.backward()
        got = {f: (leaves[f].grad.cpu().numpy() if leaves[f].grad is not None else np.zeros_like(A[f]))
               for f in per_field}
        tol = 2e-3 if n == 1 else 2e-2
        assert directional_check(got, per_field, tol) == [], (n, directional_check(got, per_field, tol))
        for f in grads[n]:
            assert np.any(got[f] != 0), (n, f)


def test_gpu_step_adjoint_matches_finite_differences():
    """Midtrain-shaped check (three explicit steps of a developed double
    gyre, loss = MSE of u, v, T, S against a seeded target): the CUDA
    gradient with respect to the initial T, S, u, v along 16 random unit
    directions against central differences (eps = 1e-3) of the float64
    oracle step.  The float32 and float64 Jacobians differ slightly, so each
    error is taken relative to the rms of the 16 directional derivatives:
    bound 2e-3 (seen: below 1.5e-3), and the median error relative to its own
    derivative below 1e-3."""
    from neuralpom_b200 import cases
    from golden_io import oracle_params
    from oracle import pom_oracle as O
    A, Sc = cases.double_gyre(24, 20, "explicit")
    Sc = dict(Sc)
    Sc.update(time=0.5, time0=0.5)
    im, jm, kb = A["u"].shape
    core = _core(A, Sc)
    core.time0 = 0.5
    core.iend = 6
    with torch.no_grad():
        core.run_time_loop()  # develop the state
    t0 = float(core.time)
    start = {f: getattr(core, f).detach().cpu().numpy().copy() for f in A}
    rng = np.random.default_rng(7)
    masks = {"t": start["fsm"][:, :, None], "s": start["fsm"][:, :, None], "u": start["dum"][:, :, None],
             "v": start["dvm"][:, :, None]}
    masks = {f: np.broadcast_to(m, start[f].shape).astype(np.float64) for f, m in masks.items()}
    scale = {"t": 1.0, "s": 0.1, "u": 0.01, "v": 0.01}
    target = {f: start[f] + 0.1 * scale[f] * rng.standard_normal(start[f].shape) * masks[f] for f in masks}

    leaves = _differentiable_advance(core, 3, t0)
    loss = sum(((getattr(core, f).double() - torch.from_numpy(target[f]).cuda()) ** 2).mean() / scale[f] ** 2
               for f in target)
    loss.backward()
    grads = {f: leaves[f].grad.double().cpu().numpy() for f in target}

    P0 = oracle_params(dict(Sc, im=im, jm=jm, kb=kb, time=t0, time0=t0), start, "explicit")

    def run64(pert):
        S = {n: v.astype(np.float64).copy() for n, v in start.items()}
        for f, d in pert.items():
            S[f] += d
        P = P0.copy()
        P.time = t0
        O.run(S, P, 3, "explicit")
        return sum(((S[f] - target[f]) ** 2).mean() / scale[f] ** 2 for f in target)

    fds, ads = [], []
    eps = 1e-3
    for _ in range(16):
        dirs = {f: rng.standard_normal(start[f].shape) * masks[f] * scale[f] for f in target}
        nrm = np.sqrt(sum((d ** 2).sum() for d in dirs.values()))
        dirs = {f: d / nrm for f, d in dirs.items()}
        fds.append((run64({f: eps * d for f, d in dirs.items()}) - run64({f: -eps * d for f, d in dirs.items()}))
                   / (2 * eps))
        ads.append(sum(float((grads[f] * dirs[f]).sum()) for f in target))
    fds, ads = np.array(fds), np.array(ads)
    rms = float(np.sqrt((ads ** 2).mean()))
    assert np.abs(fds - ads).max() / rms < 2e-3, (fds, ads)
    assert np.median(np.abs(fds - ads) / np.maximum(np.abs(fds), np.abs(ads))) < 1e-3, (fds, ads)


def test_gpu_physics_differentiable_advance_in_chunks():
    """B200Physics.advance(differentiable=True) with chunk_steps = 2 over
    three steps (a chunk of 2 and one of 1, the reference's
    _checkpoint_chunk split) gives the reference's 3-step gradient."""
    from neuralpom_b200 import B200Physics, _abi
    A, Sc, cot, grads = load_adjoint_golden("step_adjoint_explicit_12x10.npz")
    core = _core(A, Sc)
    core.time = float(Sc["time"])
    leaves = {}
    for f in _abi.ADJ_STATE_FIELDS:
        leaves[f] = getattr(core, f).detach().clone().requires_grad_(True)
        setattr(core, f, leaves[f])
    B200Physics("cuda", chunk_steps=2, core_name="explicit").advance(core, steps=3, differentiable=True)
    assert core.iint == 1 and abs(core.time - (float(Sc["time"]) + 3 * core.dti / 86400.0)) < 1e-9
    loss = sum((getattr(core, f) * torch.from_numpy(c).cuda()).sum() for f, c in cot.items())
    loss.backward()
    got = {f: leaves[f].grad.cpu().numpy() for f in grads[3]}
    assert grad_check(got, grads[3]) == [], grad_check(got, grads[3])


def test_gpu_coastal_step_adjoint_large_grid_matches_float64_differences():
    """The large-grid forms (flux-once A1/B5 tiles and thread-per-column
    PROFT in the recomputation, the cooperative grid-barrier kernels of the
    external subcycle's adjoint: 150x120 = 18,000 cells) on the coastal basin with its open
    boundary: two steps from a developed state, loss = MSE of u, v, T, S
    against a seeded target, the CUDA gradient along 4 random unit
    directions of (T, S, u, v) against central differences (eps = 1e-3) of
    the float64 oracle; errors relative to the rms directional derivative
    below 2e-3 (7e-5 seen on the emulated 40x34 basin)."""
    from neuralpom_b200 import cases
    from golden_io import oracle_params
    from oracle import pom_oracle as O
    A, Sc = cases.coastal_tide(150, 120)
    Sc = dict(Sc)
    Sc.update(time=0.25, time0=0.25)
    im, jm, kb = A["u"].shape
    core = _core(A, Sc)
    core.time0 = 0.25
    core.iend = 3
    with torch.no_grad():
        core.run_time_loop()
    t0 = float(core.time)
    start = {f: getattr(core, f).detach().cpu().numpy().copy() for f in A}
    rng = np.random.default_rng(7)
    masks = {"t": start["fsm"][:, :, None], "s": start["fsm"][:, :, None], "u": start["dum"][:, :, None],
             "v": start["dvm"][:, :, None]}
    masks = {f: np.broadcast_to(m, start[f].shape).astype(np.float64) for f, m in masks.items()}
    scale = {"t": 1.0, "s": 0.1, "u": 0.01, "v": 0.01}
    target = {f: start[f] + 0.1 * scale[f] * rng.standard_normal(start[f].shape) * masks[f] for f in masks}
    leaves = _differentiable_advance(core, 2, t0)
    loss = sum(((getattr(core, f).double() - torch.from_numpy(target[f]).cuda()) ** 2).mean() / scale[f] ** 2
               for f in target)
    loss.backward()
    grads = {f: leaves[f].grad.double().cpu().numpy() for f in target}
    P0 = oracle_params(dict(Sc, im=im, jm=jm, kb=kb, time=t0, time0=t0), start, "explicit")

    def run64(pert):
        S = {n: v.astype(np.float64).copy() for n, v in start.items()}
        for f, d in pert.items():
            S[f] += d
        P = P0.copy()
        P.time = t0
        O.run(S, P, 2, "explicit")
        return sum(((S[f] - target[f]) ** 2).mean() / scale[f] ** 2 for f in target)

    fds, ads = [], []
    for _ in range(4):
        dirs = {f: rng.standard_normal(start[f].shape) * masks[f] * scale[f] for f in target}
        nrm = np.sqrt(sum((d ** 2).sum() for d in dirs.values()))
        dirs = {f: d / nrm for f, d in dirs.items()}
        fds.append((run64({f: 1e-3 * d for f, d in dirs.items()}) - run64({f: -1e-3 * d for f, d in dirs.items()}))
                   / 2e-3)
        ads.append(sum(float((grads[f] * dirs[f]).sum()) for f in target))
    fds, ads = np.array(fds), np.array(ads)
    assert np.abs(fds - ads).max() / np.sqrt((ads ** 2).mean()) < 2e-3, (fds, ads)


def test_gpu_implicit_adjoint_on_the_global_sy_cluster_layout(monkeypatch):
    """128x112 interiors solve on the 16-CTA cluster layout that reads Sy
    from global memory, in the forward and in the adjoint solve; the
    gradients of two differentiable steps agree with those of the
    grid-barrier PCG (a different rounding of the same solver) to 1e-3."""
    from neuralpom_b200 import cases, resolve_core_class
    A, Sc = cases.seamount(128, 112)
    Sc = dict(Sc, time=1.0, time0=1.0)
    grads = []
    for form in ("coop", "cluster"):
        monkeypatch.setenv("NPOM_PCG", form)
        c = resolve_core_class("implicit_p0_fixed").from_state(A, Sc, device="cuda")
        leaves = [getattr(c, f).requires_grad_(True) for f in ("t", "u", "el")]
        c.time0, c.iend = 1.0, 2
        c.run_time_loop()
        loss = (c.u ** 2).mean() + (c.v ** 2).mean() + 1e-2 * (c.t ** 2).mean()
        loss.backward()
        grads.append([t.grad.detach().cpu().numpy() for t in leaves])
    for x, y in zip(*grads):
        scale = float(np.abs(x).max())
        assert scale > 0 and float(np.abs(y - x).max()) <= 1e-3 * scale
