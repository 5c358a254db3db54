"""Ensembles on mixed grids advanced together (npom_step_batch: one launch
per phase over all members) against the same members advanced one at a
time by npom_step_explicit / npom_step_implicit."""
import numpy as np
import pytest
import torch

from golden_io import rel_err

pytestmark = pytest.mark.gpu


def _explicit_members():
    from neuralpom_b200 import cases
    return [cases.double_gyre(37, 45, "explicit"),
            cases.coastal_tide(60, 52),
            cases.noise_basin(90, 82, seed=1),
            # above one cluster: alone it runs the grid-barrier subcycle and
            # the flux-once A1/B5 tiles, in the batch the per-phase launches
            cases.noise_basin(180, 160, seed=2)]


def _implicit_members():
    from neuralpom_b200 import cases
    return [cases.seamount(40, 36),
            cases.seamount(90, 82),
            cases.double_gyre(64, 64, "implicit_p0_fixed"),
            # the 16-CTA cluster layout that reads Sy from global memory
            cases.seamount(128, 112),
            # interior too large for the one-cluster layout: cooperative PCG
            cases.seamount(177, 161)]


def _cores(members, name):
    from neuralpom_b200 import resolve_core_class
    return [resolve_core_class(name).from_state(A, Sc, device="cuda") for A, Sc in members]


def _snapshot(c):
    from neuralpom_b200 import _abi
    return {n: getattr(c, n).cpu().numpy().copy() for n in _abi.FIELD_NAMES}


def _run_both(members, name, time0, nsteps):
    from neuralpom_b200 import batch
    alone, together = _cores(members, name), _cores(members, name)
    stream = torch.cuda.current_stream()
    for c in alone:
        c.launch_steps(nsteps, time0, 1, stream)
    batch.launch_batch(together, nsteps, time0, 1, stream)
    torch.cuda.synchronize()
    out = []
    for a, b in zip(alone, together):
        sa = a.read_status(nsteps)
        sb = b.read_status(nsteps)
        out.append((_snapshot(a), _snapshot(b), sa, sb))
    return out


@pytest.mark.parametrize("time0,nsteps", [(0.25, 4), (0.0, 3)])
@pytest.mark.parametrize("subcycle", ["phases", "coop"])
def test_explicit_batch_is_bitwise_members_alone(monkeypatch, time0, nsteps, subcycle):
    monkeypatch.setenv("NPOM_BATCH_SUBCYCLE", subcycle)
    for m, (a, b, sa, sb) in enumerate(_run_both(_explicit_members(), "explicit", time0, nsteps)):
        assert sa[0] == 0 and sb[0] == 0, (m, sa, sb)
        for n in a:
            assert np.array_equal(a[n], b[n], equal_nan=True), (m, n, rel_err(b[n], a[n]))


@pytest.mark.parametrize("time0,nsteps", [(0.25, 3), (0.0, 3)])
def test_implicit_batch_matches_members_alone(time0, nsteps):
    """Members on the one-cluster PCG bitwise; the member on the
    cooperative PCG (177x161: its dot products are summed over fewer blocks
    than alone) to 1e-5 relative per field with iteration counts within
    one."""
    res = _run_both(_implicit_members(), "implicit_p0_fixed", time0, nsteps)
    for m, (a, b, sa, sb) in enumerate(res):
        assert sa[0] == 0 and sb[0] == 0, (m, sa, sb)
        if m < 4:
            assert sa[1] == sb[1], (m, sa, sb)
            for n in a:
                assert np.array_equal(a[n], b[n], equal_nan=True), (m, n, rel_err(b[n], a[n]))
        else:
            assert all(abs(x - y) <= 1 for x, y in zip(sa[1], sb[1])), (sa, sb)
            for n in a:
                if np.abs(a[n]).max() > 0:
                    assert rel_err(b[n], a[n]) <= 1e-5, (n, rel_err(b[n], a[n]))


def test_run_batch_updates_clock_like_run_time_loop():
    from neuralpom_b200 import batch
    members = _explicit_members()[:2]
    alone, together = _cores(members, "explicit"), _cores(members, "explicit")
    for c in alone + together:
        c.time0 = 0.25
        c.iend = 3
    for c in alone:
        c.run_time_loop()
    batch.run_batch(together)
    for a, b in zip(alone, together):
        assert a.time == b.time and a.iint == b.iint and a.ramp == b.ramp
        assert torch.equal(a.t, b.t) and torch.equal(a.elb, b.elb)


def test_batch_ensemble_of_equal_grids_is_bitwise():
    """Eight seeded members of one 90x82 explicit basin (the ensemble shape
    of the forward+adjoint Midtrain case): one call, each member bitwise."""
    from neuralpom_b200 import cases
    members = [cases.noise_basin(90, 82, seed=s) for s in range(8)]
    for m, (a, b, sa, sb) in enumerate(_run_both(members, "explicit", 0.25, 3)):
        assert sb[0] == 0
        for n in a:
            assert np.array_equal(a[n], b[n], equal_nan=True), (m, n)


def test_deferred_status_members_on_streams_match_sequential():
    """Differentiable advances of two members with ``status_deferred``, each
    on its own CUDA stream with no host synchronisation between intervals,
    give bitwise the outputs of the same members advanced one after the
    other with the status read after every call, and their gradients to
    1e-5 (the step adjoint scatters with atomic adds, whose order, and so
    the last bits, vary from run to run)."""
    from neuralpom_b200 import _abi, cases, resolve_core_class
    members = [cases.noise_basin(37, 45, seed=s) for s in (3, 4)]

    def run(deferred):
        main = torch.cuda.current_stream()
        streams = [torch.cuda.Stream() for _ in members]
        cores, leaves, losses = [], [], []
        for (A, Sc), st in zip(members, streams):
            c = resolve_core_class("explicit").from_state(A, dict(Sc, time=0.25, time0=0.25), device="cuda")
            c.status_deferred = deferred
            lv = [getattr(c, f).requires_grad_(True) for f in ("t", "u", "el")]
            go = torch.cuda.Event()
            go.record(main)
            st.wait_event(go)
            with torch.cuda.stream(st if deferred else main):
                for k in range(2):
                    c.time0, c.iend = 0.25 + k * 3 * float(c.dti) / 86400.0, 3
                    c.run_time_loop()
                loss = (c.t ** 2).mean() + (c.u ** 2).mean()
            main.wait_stream(st)
            loss.record_stream(main)
            cores.append(c)
            leaves.append(lv)
            losses.append(loss)
        torch.stack(losses).sum().backward()
        torch.cuda.synchronize()
        for c in cores:
            if deferred:
                c.check_deferred_status()
        return ([{f: getattr(c, f).detach().cpu().numpy() for f in ("t", "u", "el", "q2")} for c in cores],
                [[t.grad.cpu().numpy() for t in lv] for lv in leaves])

    outs0, grads0 = run(False)
    outs1, grads1 = run(True)
    for a, b in zip(outs0, outs1):
        for f in a:
            assert np.array_equal(a[f], b[f]), f
    for ga, gb in zip(grads0, grads1):
        for x, y in zip(ga, gb):
            assert np.abs(x).max() > 0 and rel_err(y, x) <= 1e-5, rel_err(y, x)


def test_mpdata_batch_is_bitwise_members_alone():
    """Members with MPDATA tracer advection (nadv = 2: the filter, ADVT2's
    passes, SMOL_ADIF) on two grids: the batched passes give bitwise what
    each member computes alone."""
    from neuralpom_b200 import cases
    members = []
    for im, jm, seed in ((37, 45, 5), (60, 52, 6)):
        A, Sc = cases.noise_basin(im, jm, seed=seed)
        members.append((A, dict(Sc, nadv=2)))
    res = _run_both(members, "explicit", 0.25, 3)
    for m, (a, b, sa, sb) in enumerate(res):
        assert sa[0] == 0 and sb[0] == 0, (m, sa, sb)
        for n in a:
            assert np.array_equal(a[n], b[n], equal_nan=True), (m, n, rel_err(b[n], a[n]))


@pytest.mark.parametrize("core", ["explicit", "implicit_p0_fixed"])
def test_batch_with_twelve_levels_is_bitwise_members_alone(core):
    """kb = 12: the batch runs every column phase one thread per column and
    A1/B5 as point kernels (the 16-lane and tile forms need kb = 16); each
    member bitwise what it computes alone."""
    from neuralpom_b200 import cases
    members = [cases.double_gyre(22, 20, core, kb=12), cases.double_gyre(30, 26, core, kb=12)]
    for m, (a, b, sa, sb) in enumerate(_run_both(members, core, 0.25, 3)):
        assert sa[0] == 0 and sb[0] == 0, (m, sa, sb)
        for n in a:
            assert np.array_equal(a[n], b[n], equal_nan=True), (m, n, rel_err(b[n], a[n]))


def test_batch_inside_the_ramp_period_is_bitwise_members_alone():
    """Members whose forcing ramp has not saturated (lramp with periods of
    0.5 and 2 days, from time 0.1): every step launches directly with each
    member's own ramp value; each member bitwise what it computes alone."""
    from neuralpom_b200 import cases
    members = []
    for (im, jm, seed), period in (((37, 45, 7), 0.5), ((48, 40, 8), 2.0)):
        A, Sc = cases.noise_basin(im, jm, seed=seed)
        members.append((A, dict(Sc, lramp=True, period=period)))
    for m, (a, b, sa, sb) in enumerate(_run_both(members, "explicit", 0.1, 3)):
        assert sa[0] == 0 and sb[0] == 0, (m, sa, sb)
        for n in a:
            assert np.array_equal(a[n], b[n], equal_nan=True), (m, n, rel_err(b[n], a[n]))
