"""The free-surface solve and its CUDA adjoint (npom_pcg_adjoint) through the
drop-in API ``ImplicitCore.solve_implicit_eta_cg`` under torch autograd:
against the reference's own autograd gradients (golden vectors), against
the oracle, and against central finite differences."""
import numpy as np
import pytest
import torch

from golden_io import golden_path, oracle_params, rel_err
from oracle import pom_oracle as O

pytestmark = pytest.mark.gpu


def _case():
    z = np.load(golden_path("eta_adjoint_20x18.npz"))
    A = {k[4:]: z[k] for k in z.files if k.startswith("in__")}
    Sc = {k[8:]: (z[k].item() if z[k].dtype.kind in "biuf" else str(z[k])) for k in z.files
          if k.startswith("scalar__")}
    adj = {k[5:]: z[k] for k in z.files if k.startswith("adj__")}
    return A, Sc, adj


def _core(A, Sc):
    from neuralpom_b200 import resolve_core_class
    return resolve_core_class("implicit_p0_fixed").from_state(A, Sc, device="cuda")


def test_gpu_eta_solve_and_adjoint_match_reference_autograd():
    A, Sc, adj = _case()
    core = _core(A, Sc)
    rhs = torch.tensor(adj["rhs"], device="cuda", requires_grad=True)
    d2d = torch.tensor(adj["d2d"], device="cuda", requires_grad=True)
    x0 = torch.tensor(adj["x0"], device="cuda")
    tol = float(adj["tol"])
    core._eta_solver_iteration_history = []
    x = core.solve_implicit_eta_cg(rhs, d2d, max_iter=200, tol=tol, print_cg_residual=False, initial_guess=x0)
    assert core._eta_solver_iteration_history == [int(v) for v in adj["fwd_its"]]
    # forward: the step parity bound (1e-5 relative)
    assert rel_err(x.detach().cpu().numpy(), adj["x"]) < 1e-5
    (x * torch.tensor(adj["g"], device="cuda")).sum().backward()
    g_rhs, g_d = rhs.grad.cpu().numpy(), d2d.grad.cpu().numpy()
    # the adjoint solve stops at the same relative residual (1e-5) as the
    # reference's, from a different but equally converged iterate
    assert rel_err(g_rhs, adj["grad_rhs"]) < 1e-4, rel_err(g_rhs, adj["grad_rhs"])
    assert rel_err(g_d, adj["grad_d"]) < 1e-4, rel_err(g_d, adj["grad_d"])
    # and against the oracle's adjoint of the same forward solution
    P = oracle_params(Sc, A, "implicit_p0_fixed")
    C = O.implicit_coefficients(A, P)
    SC = O.spectral_cache(A, P, C)
    lam, gd, its = O.eta_adjoint(adj["g"], x.detach().cpu().numpy(), adj["d2d"], A, P, C, SC,
                                 int(P.eta_solver_max_iter), tol, float(P.eta_solver_rel_tol),
                                 P.eta_solver_preconditioner)
    assert rel_err(g_rhs, lam) < 1e-4
    assert rel_err(g_d, gd) < 1e-4
    assert core._eta_adjoint_iteration_history == [its]


def test_gpu_eta_adjoint_matches_central_differences():
    """dJ/drhs and dJ/dd of J = <g, x(rhs, d)> against central differences
    (FP64 sums of the FP32 solutions, solves run to the FP32 floor) along
    random unit directions that keep half their weight on the gradient, so
    that the difference of two FP32 solves carries signal.  Bound: 1e-3
    relative."""
    A, Sc, adj = _case()
    core = _core(A, Sc)
    core.eta_solver_rel_tol = 1e-12
    dev = "cuda"
    rhs0 = torch.tensor(adj["rhs"], device=dev)
    d0 = torch.tensor(adj["d2d"], device=dev)
    g = torch.tensor(adj["g"], device=dev)
    zero = torch.zeros_like(rhs0)

    def J(r, d):
        with torch.no_grad():
            x = core.solve_implicit_eta_cg(r, d, max_iter=400, tol=1e-14, initial_guess=zero)
        return float((x.double() * g.double()).sum())

    rhs = rhs0.clone().requires_grad_(True)
    d2d = d0.clone().requires_grad_(True)
    x = core.solve_implicit_eta_cg(rhs, d2d, max_iter=400, tol=1e-14, initial_guess=zero)
    (x * g).sum().backward()
    gen = torch.Generator(device="cpu").manual_seed(5)

    def direction(grad):
        r = torch.randn(grad.shape, generator=gen, dtype=torch.float64).to(dev)
        u = grad.double() / grad.double().norm() + r / r.norm()
        return (u / u.norm()).float()

    for _ in range(4):
        v = direction(rhs.grad)
        eps = 1e-3 * float(rhs0.abs().max())
        fd = (J(rhs0 + eps * v, d0) - J(rhs0 - eps * v, d0)) / (2 * eps)
        an = float((rhs.grad.double() * v.double()).sum())
        assert abs(fd - an) <= 1e-3 * max(abs(fd), abs(an)), (fd, an)
        w = direction(d2d.grad)
        eps = 1e-3 * float(d0.abs().max())
        fd = (J(rhs0, d0 + eps * w) - J(rhs0, d0 - eps * w)) / (2 * eps)
        an = float((d2d.grad.double() * w.double()).sum())
        assert abs(fd - an) <= 1e-3 * max(abs(fd), abs(an)), (fd, an)


def test_gpu_eta_adjoint_rejects_non_finite_cotangent():
    """A NaN cotangent is reported as FloatingPointError before any solve;
    the next backward on the same core works."""
    A, Sc, adj = _case()
    core = _core(A, Sc)
    rhs = torch.tensor(adj["rhs"], device="cuda", requires_grad=True)
    d2d = torch.tensor(adj["d2d"], device="cuda")
    x = core.solve_implicit_eta_cg(rhs, d2d, max_iter=200, tol=1e-10, initial_guess=torch.zeros_like(d2d))
    bad = torch.tensor(adj["g"], device="cuda")
    bad[3, 4] = float("nan")
    with pytest.raises(FloatingPointError):
        x.backward(bad)
    rhs.grad = None
    x = core.solve_implicit_eta_cg(rhs, d2d, max_iter=200, tol=1e-10, initial_guess=torch.zeros_like(d2d))
    x.backward(torch.tensor(adj["g"], device="cuda"))
    assert torch.isfinite(rhs.grad).all()
