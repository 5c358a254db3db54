"""Periodic x on the B200 (the benchmark seamount as a channel periodic in x
with walls in y, 90x82x16, dtI 300 s), through the drop-in API.

The reference has no periodic boundary: the bar is the oracle's periodic
step (float32, float32 with T moved by one ulp, float64), and the
properties only a periodic model has -- translation equivariance in x and
the conservation of the FP64 volume integral of the elevation.
"""
import numpy as np
import pytest
import torch

from golden_io import rel_err
from test_gpu_fullday import _check, compare_day

pytestmark = pytest.mark.gpu

CORE = "implicit_p0_fixed"


def _gpu(A, Sc, steps):
    from neuralpom_b200 import B200Physics, resolve_core_class
    c = resolve_core_class(CORE).from_state(A, Sc, device="cuda")
    B200Physics(core_name=CORE).advance(c, steps=steps)
    return c


def test_gpu_periodic_channel_matches_oracle_and_fp64():
    """48 steps (4 h) of the channel with its spectral preconditioner
    (Hartley along the period, DST-I across)."""
    rows, itg, it32 = compare_day("seamount_channel", 90, 82, CORE, 48)
    _check(rows)
    p = rows["pcg_iterations"]
    # the cooperative-grid solve sums its FP64 dot products in another
    # order than the oracle: counts within the 1-ulp run's own drift plus one
    assert abs(itg[0] - it32[0]) <= 1, p
    assert p["max_abs_step_diff"] <= p["ulp_max_abs_step_diff"] + 1, p


def test_gpu_periodic_channel_is_translation_equivariant_and_conserves_volume():
    from neuralpom_b200 import cases
    im, jm, m, steps = 90, 82, 29, 24
    A, Sc = cases.seamount_channel(im, jm)
    # the Jacobi preconditioner is pointwise, so the shifted run repeats the
    # same arithmetic (the Hartley transform is equivariant only to rounding)
    Sc = dict(Sc, eta_solver_preconditioner="jacobi", eta_solver_max_iter=1000)

    def roll(S):
        B = {k: np.array(v, copy=True) for k, v in S.items()}
        for k, a in S.items():
            if np.ndim(a) >= 2 and np.shape(a)[:2] == (im, jm):
                B[k][2:im - 2] = np.roll(np.asarray(a)[2:im - 2], m, axis=0)
                cases.wrap_x(B[k])
        return B

    c1 = _gpu(A, Sc, steps)
    c2 = _gpu(roll(A), Sc, steps)
    F = ("u", "v", "t", "s", "el", "q2", "km", "kh", "w", "rho", "ua", "va")
    S1 = {f: getattr(c1, f).cpu().numpy() for f in F}
    S2 = {f: getattr(c2, f).cpu().numpy() for f in F}
    R = roll(S1)
    for f in F:
        # the same arithmetic at every unique column; only the solve's FP64
        # dot products are summed over other blocks
        bound = 1e-3 if f == "w" else 1e-4
        assert rel_err(S2[f], R[f]) < bound, (f, rel_err(S2[f], R[f]))
    # the halo columns are copies of the unique ones
    for f in F:
        a = S1[f]
        assert np.array_equal(a[0], a[im - 4]) and np.array_equal(a[im - 1], a[3]), f
    # volume: the elevation integral over the unique columns moves only by
    # the solver's residual and float32 rounding (FP64 sums of the float32
    # state; the float32 oracle drifts by 4e-7 of the integral of |et| over
    # these 24 steps, a halo that leaked would move it by order one)
    U = slice(2, im - 2)
    w = (A["art"][U] * A["fsm"][U]).astype(np.float64)
    et = c1.et.double().cpu().numpy()[U]
    v0 = float((w * A["et"][U]).sum())
    assert abs(float((w * et).sum()) - v0) <= 1e-5 * float((w * np.abs(et)).sum())
    assert torch.isfinite(c1.el).all()
