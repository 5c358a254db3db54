"""Further GPU parity cases through the public API: the known answers of the
reference's own free-surface adjoint tests (tests/test_fixed_core_runtime.py
:156-200, restated here in FP32), and step parity against the oracle on the
paths the benchmark does not take (Jacobi preconditioner, kb != 16, a PCG
that stops at its iteration cap, non-contiguous / float64 attributes)."""
import numpy as np
import pytest
import torch

from golden_io import oracle_params, rel_err
from oracle import pom_oracle as O

pytestmark = pytest.mark.gpu


def _core(A, Sc, core="implicit_p0_fixed"):
    from neuralpom_b200 import resolve_core_class
    return resolve_core_class(core).from_state(A, Sc, device="cuda")


def _gyre_10x10():
    from neuralpom_b200 import cases
    A, Sc = cases.double_gyre(10, 10, "implicit_p0_fixed")
    Sc = dict(Sc)
    Sc.update(time=1000.0, time0=1000.0)
    return A, Sc


def test_gpu_eta_adjoint_equals_explicit_transpose_solve():
    """rhs.grad of <w, A^-1 rhs> equals A^-T w with A assembled column by
    column from the operator (reference test_fixed_core_runtime.py:156-181),
    and the forward residual is at the FP32 floor."""
    A, Sc = _gyre_10x10()
    core = _core(A, Sc)
    core.eta_solver_rel_tol = 1e-11
    rhs = torch.sin(torch.arange(100, dtype=torch.float32)).reshape(10, 10).cuda().requires_grad_(True)
    weight = torch.cos(torch.arange(100, dtype=torch.float32)).reshape(10, 10)
    weight[[0, -1], :] = 0
    weight[:, [0, -1]] = 0
    d = torch.tensor(A["d"], device="cuda")
    x = core.solve_implicit_eta_cg(rhs, d, max_iter=200, tol=1e-14, print_cg_residual=False,
                                   initial_guess=torch.zeros_like(d))
    (x * weight.cuda()).sum().backward()
    S64 = {k: (v.astype(np.float64) if isinstance(v, np.ndarray) and v.dtype == np.float32 else v)
           for k, v in A.items()}
    P = oracle_params(Sc, A, "implicit_p0_fixed")
    C = O.implicit_coefficients(S64, P)
    cols = []
    for idx in range(64):
        basis = np.zeros((10, 10))
        basis[1 + idx // 8, 1 + idx % 8] = 1.0
        cols.append(O.elliptic_apply(basis, S64["d"], C)[1:-1, 1:-1].reshape(-1))
    M = np.stack(cols, axis=1)
    expect = np.linalg.solve(M.T, weight.numpy()[1:-1, 1:-1].reshape(-1).astype(np.float64))
    got = rhs.grad.cpu().numpy()[1:-1, 1:-1].reshape(-1)
    assert rel_err(got, expect) < 2e-5, rel_err(got, expect)
    res = M @ x.detach().cpu().numpy()[1:-1, 1:-1].reshape(-1) - rhs.detach().cpu().numpy()[1:-1, 1:-1].reshape(-1)
    assert np.linalg.norm(res) / np.linalg.norm(rhs.detach().cpu().numpy()) < 1e-5


def test_gpu_eta_adjoint_of_a_huge_cotangent_stays_finite_and_linear():
    """Reference test_fixed_core_runtime.py:194-200: the right-hand-side
    scaling keeps a 1e20 cotangent finite and the adjoint linear."""
    A, Sc = _gyre_10x10()
    core = _core(A, Sc)
    g = torch.sin(torch.arange(100, dtype=torch.float32)).reshape(10, 10).cuda()
    d = torch.tensor(A["d"], device="cuda")
    x = torch.zeros_like(d)
    small, _ = core._eta_adjoint(g, x, d, 200, 1e-12)
    large, _ = core._eta_adjoint(g * 1e20, x, d, 200, 1e-12)
    assert bool(torch.isfinite(large).all())
    torch.testing.assert_close(large / 1e20, small, rtol=1e-4, atol=1e-6)


def _step_pair(A, Sc, core, steps, tweak=None):
    from neuralpom_b200 import B200Physics
    Sc = dict(Sc)
    im, jm, kb = A["u"].shape
    Sc.update(im=im, jm=jm, kb=kb)
    c = _core(A, Sc, core)
    S = {k: v.copy() for k, v in A.items()}
    P = oracle_params(Sc, A, core)
    if tweak:
        tweak(c, P)
    hist = []
    for _ in range(steps):
        B200Physics(core_name=core).advance(c, steps=1)
        hist.extend(O.run(S, P, 1, core) or [])
    return c, S, hist


FIELDS = ("u", "v", "t", "s", "el", "q2", "km", "kh", "w", "rho", "ua", "va")


def test_gpu_jacobi_preconditioner_step_matches_oracle():
    from neuralpom_b200 import cases
    A, Sc = cases.double_gyre(20, 18, "implicit_p0_fixed")
    Sc = dict(Sc)
    Sc.update(time=1000.0, time0=1000.0, eta_solver_preconditioner="jacobi")

    def tweak(c, P):
        P.eta_solver_preconditioner = "jacobi"

    c, S, hist = _step_pair(A, Sc, "implicit_p0_fixed", 2, tweak)
    assert c._eta_solver_iteration_history == hist
    for f in FIELDS:
        assert rel_err(getattr(c, f).cpu().numpy(), S[f]) < 1e-4, f


@pytest.mark.parametrize("core", ["implicit_p0_fixed", "explicit"])
def test_gpu_twelve_levels_match_oracle(core):
    """kb = 12 runs the thread-per-column bodies instead of the 16-lane
    kernels."""
    from neuralpom_b200 import cases
    A, Sc = cases.double_gyre(22, 20, core, kb=12)
    Sc = dict(Sc)
    Sc.update(time=1000.0, time0=1000.0)
    c, S, _ = _step_pair(A, Sc, core, 2)
    for f in FIELDS:
        assert rel_err(getattr(c, f).cpu().numpy(), S[f]) < 1e-4, f


def test_gpu_pcg_iteration_cap_is_reported_not_raised():
    """A solve that stops at eta_solver_max_iter ends the step normally, as
    in the reference; the cap shows in the iteration history."""
    from neuralpom_b200 import cases
    A, Sc = cases.seamount(40, 36)
    Sc = dict(Sc)
    Sc.update(eta_solver_max_iter=3)

    def tweak(c, P):
        P.eta_solver_max_iter = 3

    c, S, hist = _step_pair(A, Sc, "implicit_p0_fixed", 2, tweak)
    assert c._eta_solver_iteration_history == hist == [3, 3]
    for f in ("el", "ua", "va", "u", "t"):
        assert rel_err(getattr(c, f).cpu().numpy(), S[f]) < 1e-4, f


def test_gpu_accepts_noncontiguous_and_float64_attributes():
    """Attributes rebound to float64 or non-contiguous tensors (as callers of
    the reference do) are taken as float32 contiguous copies."""
    from neuralpom_b200 import B200Physics, cases
    A, Sc = cases.double_gyre(20, 18, "implicit_p0_fixed")
    Sc = dict(Sc)
    Sc.update(time=1000.0, time0=1000.0)
    ref = _core(A, Sc)
    B200Physics(core_name="implicit_p0_fixed").advance(ref, steps=2)
    c = _core(A, Sc)
    c.t = torch.tensor(A["t"], dtype=torch.float64, device="cuda")
    c.s = torch.tensor(np.ascontiguousarray(A["s"].transpose(1, 0, 2)), device="cuda").transpose(0, 1)
    assert not c.s.is_contiguous()
    B200Physics(core_name="implicit_p0_fixed").advance(c, steps=2)
    for f in ("t", "s", "u", "el", "kh"):
        assert torch.equal(getattr(c, f), getattr(ref, f)), f
