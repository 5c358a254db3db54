"""Periodic x on the semi-implicit core (the benchmark seamount as a channel
periodic in x with walls in y), on the CPU.

The reference has no periodic boundary, so parity is unpinned: the oracle's
periodic step (``pom_oracle.step_implicit`` with ``periodic_x``: a halo copy
of two columns after every phase of the CUDA step, the η-solve's operator
wrapped in x) is pinned instead by properties that only a periodic model
has, and the device bodies are checked against it:

* translation equivariance: shifting the initial state (geometry included)
  by m of the unique columns shifts the result by m, with the same PCG
  iterations -- a halo that left any operator seeing a wall would break it;
* the halo columns are copies of their unique columns after every step;
* the FP64 volume sum(art fsm et) over the unique columns is conserved;
* the phase bodies of the CUDA library, compiled for the host
  (tests/emul), match the oracle.
"""
import numpy as np
import pytest

from golden_io import oracle_params, rel_err
from oracle import pom_oracle as O

CORE = "implicit_p0_fixed"
FIELDS = ("u", "v", "t", "s", "el", "q2", "q2l", "km", "kh", "w", "rho", "ua", "va", "elb", "uab", "vab", "utf",
          "vtf", "egb", "et")


def _channel(im, jm):
    from neuralpom_b200 import cases
    A, Sc = cases.seamount(im, jm, periodic_x=True)
    Sc = dict(Sc, im=im, jm=jm, kb=A["u"].shape[2])
    return A, Sc


def _planes(A, im, jm):
    return [k for k, a in A.items() if np.ndim(a) >= 2 and np.shape(a)[:2] == (im, jm)]


def _roll(A, m, im, jm):
    """The state moved by m unique columns (2..im-3), halos refilled."""
    from neuralpom_b200.cases import wrap_x
    B = {k: np.array(v, copy=True) for k, v in A.items()}
    for k in _planes(A, im, jm):
        B[k][2:im - 2] = np.roll(np.asarray(A[k])[2:im - 2], m, axis=0)
        wrap_x(B[k])
    return B


def _run(A, Sc, steps, fp64=False):
    S = {k: (v.astype(np.float64) if fp64 and v.dtype == np.float32 else np.array(v, copy=True))
         for k, v in A.items()}
    its = O.run(S, oracle_params(Sc, A, CORE), steps, CORE)
    return S, [int(v) for v in its]


def test_periodic_seamount_geometry():
    im, jm = 24, 20
    A, Sc = _channel(im, jm)
    assert Sc["periodic_x"] and Sc.get("eta_solver_preconditioner", "spectral") == "spectral"
    # walls only in y: the whole x range is wet between the j walls
    assert np.all(A["fsm"][:, 1:jm - 1] == 1.0) and np.all(A["fsm"][:, [0, jm - 1]] == 0.0)
    for k in _planes(A, im, jm):
        a = A[k]
        assert np.array_equal(a[0], a[im - 4]) and np.array_equal(a[1], a[im - 3]), k
        assert np.array_equal(a[im - 2], a[2]) and np.array_equal(a[im - 1], a[3]), k


@pytest.mark.parametrize("precond", ["jacobi", "spectral"])
def test_oracle_periodic_step_is_translation_equivariant(precond):
    im, jm, m, steps = 24, 20, 7, 4
    A, Sc = _channel(im, jm)
    Sc.update(eta_solver_preconditioner=precond, eta_solver_max_iter=1000)
    S1, it1 = _run(A, Sc, steps)
    S2, it2 = _run(_roll(A, m, im, jm), Sc, steps)
    R = _roll(S1, m, im, jm)
    if precond == "jacobi":
        # bitwise in practice: every unique column sees the same values in
        # the same order (the solve's diagonal scaling is pointwise); the
        # FP64 dot products are summed in another order
        assert it1 == it2
        for f in FIELDS:
            assert rel_err(S2[f], R[f]) <= 1e-6, (f, rel_err(S2[f], R[f]))
    else:
        # the Hartley transform of the preconditioner is equivariant only
        # up to its rounding; the solve converges to 1e-10 either way
        assert max(abs(a - b) for a, b in zip(it1, it2)) <= 1
        for f in ("u", "v", "t", "s", "el", "ua", "va", "w"):
            assert rel_err(S2[f], R[f]) <= 1e-4, (f, rel_err(S2[f], R[f]))


def test_oracle_hartley_preconditioner():
    """The periodic preconditioner's x transform: symmetric, H H = n I, and
    it diagonalises the periodic second difference with 4 sin^2(pi k/n)."""
    n = 12
    H = O.hartley_matrix(n)
    assert np.allclose(H, H.T) and np.allclose(H @ H, n * np.eye(n))
    L = 2.0 * np.eye(n) - np.roll(np.eye(n), 1, axis=1) - np.roll(np.eye(n), -1, axis=1)
    lam = 4.0 * np.sin(np.pi * np.arange(n) / n) ** 2
    assert np.allclose(H @ L @ H / n, np.diag(lam), atol=1e-10)


def test_oracle_walls_in_x_are_not_translation_equivariant():
    """The same check on the closed basin fails: it sees the walls."""
    from neuralpom_b200 import cases
    im, jm, m = 24, 20, 7
    A, Sc = cases.seamount(im, jm)
    Sc = dict(Sc, im=im, jm=jm, kb=16)
    S1, _ = _run(A, Sc, 2)
    S2, _ = _run(_roll(A, m, im, jm), Sc, 2)
    assert rel_err(S2["ua"], _roll(S1, m, im, jm)["ua"]) > 1e-3


def test_oracle_periodic_halo_columns_are_copies():
    im, jm = 24, 20
    A, Sc = _channel(im, jm)
    S, _ = _run(A, Sc, 3)
    for k in _planes(S, im, jm):
        if k in O._NOT_PLANES:
            continue
        a = S[k]
        assert np.array_equal(a[0], a[im - 4]) and np.array_equal(a[1], a[im - 3]), k
        assert np.array_equal(a[im - 2], a[2]) and np.array_equal(a[im - 1], a[3]), k


def test_oracle_periodic_volume_is_conserved_fp64():
    im, jm = 24, 20
    A, Sc = _channel(im, jm)
    U = slice(2, im - 2)

    def volume_anomaly(S):
        w = S["art"][U] * S["fsm"][U]
        return float((w * S["et"][U]).sum()), float((w * np.abs(S["et"][U])).sum())

    v0, _ = volume_anomaly({k: np.asarray(v, np.float64) for k, v in A.items()})
    S, _ = _run(A, Sc, 4, fp64=True)
    v, scale = volume_anomaly(S)
    assert scale > 0.0
    # the elevation moves by decimetres; its volume integral only by the
    # solver's residual
    assert abs(v - v0) <= 1e-9 * scale, (v, v0, scale)


def test_periodic_parameters():
    from neuralpom_b200 import state, _abi
    im, jm = 24, 20
    A, Sc = _channel(im, jm)
    p = state.make_params(Sc, im, jm, 16, CORE)
    assert p.periodic_x == 1 and p.eta_precond == _abi.PRECOND_SPECTRAL
    # Hartley over the im-4 unique columns times DST-I over jm-2 rows
    assert p.inverse_scale == 2.0 * (im - 4) * (jm - 1)
    sx, sy, ie = state.spectral_setup(A["dx"], A["dy"], A["h"], Sc["dti"], Sc["grav"], Sc["alpha"], periodic_x=True)
    assert sx.shape == (im - 4, im - 4) and ie.shape == (im - 4, jm - 2)
    assert np.allclose(sx, O.hartley_matrix(im - 4), atol=1e-5)
    for bad in (dict(nadv=2), dict(obc_form="seamount")):
        with pytest.raises(ValueError):
            state.make_params(dict(Sc, **bad), im, jm, 16, CORE)
    with pytest.raises(ValueError, match="periodic x"):
        state.make_params(dict(Sc, periodic_x=True), im, jm, 16, "explicit")
    assert state.make_params(dict(Sc, periodic_x=False), im, jm, 16, CORE).periodic_x == 0


def _has_nvcc():
    import shutil
    return shutil.which("nvcc") is not None


@pytest.mark.skipif(not _has_nvcc(), reason="nvcc needed to build the phase emulator")
def test_emulated_periodic_step_matches_oracle():
    emul = pytest.importorskip("emul_harness")
    im, jm, steps = 24, 20, 3
    A, Sc = _channel(im, jm)
    E = emul.EmulCore(A, Sc, CORE)
    its_e = [int(v) for v in E.steps(steps)]
    S, its_o = _run(A, Sc, steps)
    assert its_e == its_o
    # the bar of the other emulated steps after three steps (1e-4; w
    # without its bottom level, whose exact value is zero)
    for f in FIELDS:
        err = rel_err(E.F[f][..., :-1] if f == "w" else E.F[f], S[f][..., :-1] if f == "w" else S[f])
        assert err < 1e-4, (f, err)
