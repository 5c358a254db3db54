"""The oracle against the reference core's own outputs (golden vectors made
by tests/golden/make_golden.py) and the reference tests' known answers."""
import numpy as np
import pytest

from golden_io import golden_path, load_step_golden, oracle_params, rel_err, step_field_error
from oracle import pom_oracle as O

STEP_FILES = [("step_explicit_12x10.npz", "explicit"), ("step_implicit_12x10.npz", "implicit_p0_fixed"),
              ("step_implicit_20x18.npz", "implicit_p0_fixed"), ("step_coastal_40x34.npz", "explicit"),
              # the POM08-WAD closure of the reference's case policies
              ("step_pom08_explicit_12x10.npz", "explicit"), ("step_pom08_implicit_20x18.npz", "implicit_p0_fixed"),
              # the semi-implicit core with its spatial Shapiro filters on
              ("step_implicit_shapiro_20x18.npz", "implicit_p0_fixed")]
PROGNOSTIC = ("u", "v", "t", "s", "el", "q2", "q2l", "km", "kh", "w", "rho", "ua", "va", "elf", "etf")


@pytest.mark.parametrize("fname,core", STEP_FILES)
def test_oracle_matches_reference_steps(fname, core):
    A, Sc, OUT = load_step_golden(fname)
    S = {k: v.copy() for k, v in A.items()}
    P = oracle_params(Sc, A, core)
    done = 0
    for n in sorted(OUT):
        hist = O.run(S, P, n - done, core)
        done = n
        # one step: 1e-5 relative on every stored field (measured ~4e-7);
        # three steps: 1e-4 (baroclinic gradient amplifies rounding)
        for f, ref in OUT[n].items():
            if f.startswith("scalar") or f == "cg_iters":
                continue
            err, bound = step_field_error(S[f], ref, f, n, fname)
            assert err < bound, (fname, n, f, err)
        if "cg_iters" in OUT[n]:
            assert hist == [int(v) for v in OUT[n]["cg_iters"]]
        assert abs(P.time - float(OUT[n]["scalar_time"])) < 1e-9


@pytest.mark.parametrize("tag", ["f64", "f32"])
@pytest.mark.parametrize("nbc", [1, 2, 3, 4])
def test_oracle_proft_matches_reference_fixture(tag, nbc):
    z = np.load(golden_path("proft_strict_fixture.npz"))
    g = lambda n: z[f"{tag}__{n}"]  # noqa: E731
    out, dh = O.proft(g("f"), g("wfsurf"), g("fsurf"), nbc, g("h"), g("etf"), 1200.0, g("dz"), g("dzz"),
                      g("swrad"), 2, g("kh"), 1e-6, g("z"))
    ref = z[f"{tag}__nbc{nbc}__f"]
    # nbc 2/4 evaluate exp(), whose last bits differ between numpy and torch
    tol = (1e-10 if nbc in (2, 4) else 1e-13) if tag == "f64" else 2e-6
    assert rel_err(out, ref) < tol
    assert np.array_equal(dh, z[f"{tag}__nbc{nbc}__dh"])
    # the bottom ghost level is passed through untouched
    assert np.array_equal(out[..., -1], g("f")[..., -1])


def test_oracle_proft_uniform_column_known_answer():
    """tests/test_strict_vertical.py:114-122: a column of 7 with no surface
    flux stays 7; nbc 3/4 pin the surface value."""
    z = np.load(golden_path("proft_strict_fixture.npz"))
    g = lambda n: z[f"f64__{n}"]  # noqa: E731
    f = np.full_like(g("f"), 7.0)
    out, _ = O.proft(f, np.zeros_like(g("wfsurf")), g("fsurf"), 1, g("h"), g("etf"), 1200.0, g("dz"), g("dzz"),
                     g("swrad"), 2, g("kh"), 1e-6, g("z"))
    np.testing.assert_allclose(out, f, rtol=1e-15, atol=1e-15)
    for nbc in (3, 4):
        out, _ = O.proft(f, np.zeros_like(g("wfsurf")), g("fsurf"), nbc, g("h"), g("etf"), 1200.0, g("dz"),
                         g("dzz"), g("swrad"), 2, g("kh"), 1e-6, g("z"))
        assert np.array_equal(out[..., 0], g("fsurf"))


def test_barotropic_endpoint_transport_identity():
    """tests/test_fixed_core_runtime.py:41-50 known answer, in the oracle's
    endpoint-transport form 0.25*(u*dsum + u*dsum) with dsum = 2d."""
    v = np.array([0.2, -0.3], np.float32)
    d = np.array([10.0, 20.0], np.float32)
    got = 0.25 * (v * (2 * d) + v * (2 * d))
    np.testing.assert_allclose(got, v * d)


def _adjoint_case():
    z = np.load(golden_path("eta_adjoint_20x18.npz"))
    A = {k[4:]: z[k] for k in z.files if k.startswith("in__")}
    Sc = {k[8:]: (z[k].item() if z[k].dtype.kind in "biuf" else str(z[k])) for k in z.files if k.startswith("scalar__")}
    adj = {k[5:]: z[k] for k in z.files if k.startswith("adj__")}
    P = oracle_params(Sc, A, "implicit_p0_fixed")
    C = O.implicit_coefficients(A, P)
    SC = O.spectral_cache(A, P, C) if P.eta_solver_preconditioner == "spectral" else None
    return A, P, C, SC, adj


def test_oracle_eta_solve_and_adjoint_match_reference_autograd():
    """Forward solve and backward (dJ/drhs, dJ/dd) of the free-surface
    solve against the reference's _ImplicitEtaSolveFunction run under
    torch autograd (core.py:24-59, 231-252, 645-675)."""
    A, P, C, SC, adj = _adjoint_case()
    tol = float(adj["tol"])
    x, its = O.pcg_solve(adj["rhs"], adj["d2d"], adj["x0"], A, P, C, SC, int(P.eta_solver_max_iter), tol,
                         float(P.eta_solver_rel_tol), P.eta_solver_preconditioner)
    assert its == int(adj["fwd_its"][0])
    assert rel_err(x, adj["x"]) < 1e-5
    lam, grad_d, _ = O.eta_adjoint(adj["g"], adj["x"], adj["d2d"], A, P, C, SC, int(P.eta_solver_max_iter), tol,
                                   float(P.eta_solver_rel_tol), P.eta_solver_preconditioner)
    assert rel_err(lam, adj["grad_rhs"]) < 1e-5, rel_err(lam, adj["grad_rhs"])
    assert rel_err(grad_d, adj["grad_d"]) < 1e-4, rel_err(grad_d, adj["grad_d"])


def test_oracle_eta_adjoint_matches_central_differences_fp64():
    """The adjoint against central finite differences of J = <g, x(rhs, d)>
    in FP64 along random unit directions (eps 1e-3 relative), with the
    solve converged far below the difference step."""
    A, P, C, SC, adj = _adjoint_case()
    A = {k: (v.astype(np.float64) if v.dtype == np.float32 else v) for k, v in A.items()}
    C = O.implicit_coefficients(A, P)
    SC = O.spectral_cache(A, P, C) if SC is not None else None
    rhs, d2d, g = (adj[k].astype(np.float64) for k in ("rhs", "d2d", "g"))
    tol, rel = 1e-13, 1e-13

    def solve(r, d):
        return O.pcg_solve(r, d, np.zeros_like(r), A, P, C, SC, 400, tol, rel, P.eta_solver_preconditioner)[0]

    x = solve(rhs, d2d)
    lam, grad_d, _ = O.eta_adjoint(g, x, d2d, A, P, C, SC, 400, tol, rel, P.eta_solver_preconditioner)
    rng = np.random.default_rng(3)
    inner = np.zeros_like(rhs, dtype=bool)
    inner[1:-1, 1:-1] = True
    for _ in range(4):
        v = rng.standard_normal(rhs.shape) * inner
        v /= np.linalg.norm(v)
        eps = 1e-3 * np.abs(rhs).max()
        fd = (np.sum(g * solve(rhs + eps * v, d2d)) - np.sum(g * solve(rhs - eps * v, d2d))) / (2 * eps)
        assert abs(fd - np.sum(lam * v)) <= 1e-6 * max(abs(fd), 1e-12) + 1e-12
        w = rng.standard_normal(rhs.shape)
        w /= np.linalg.norm(w)
        eps = 1e-3 * np.abs(d2d).max()
        fd = (np.sum(g * solve(rhs, d2d + eps * w)) - np.sum(g * solve(rhs, d2d - eps * w))) / (2 * eps)
        assert abs(fd - np.sum(grad_d * w)) <= 1e-3 * max(abs(fd), 1e-12) + 1e-12
