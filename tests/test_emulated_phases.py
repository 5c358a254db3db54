"""The device phase bodies, run on the CPU by tests/emul, against the
reference golden vectors and the oracle (index logic of every kernel)."""
import numpy as np
import pytest

from golden_io import load_step_golden, oracle_params, rel_err, step_field_error
from oracle import pom_oracle as O

emul = pytest.importorskip("emul_harness")


def _has_nvcc():
    import shutil
    return shutil.which("nvcc") is not None


pytestmark = pytest.mark.skipif(not _has_nvcc(), reason="nvcc needed to build the phase emulator")

STEP_FILES = [("step_explicit_12x10.npz", "explicit"), ("step_implicit_12x10.npz", "implicit_p0_fixed"),
              ("step_implicit_20x18.npz", "implicit_p0_fixed"),
              # the reference's seamount case policy (boundary and POM08-WAD closure)
              ("step_seamount_explicit_24x18.npz", "explicit"),
              # the reference's coastal tide policy (its boundary, step copies and closure)
              ("step_coastal_policy_24x18.npz", "explicit"),
              # the reference's Jiaozhou Bay tide policy (its boundary, the coastal step copies, closure)
              ("step_jzb_policy_24x18.npz", "explicit"),
              # both tide policies on the semi-implicit core (their own area-weighted CG)
              ("step_coastal_policy_implicit_24x18.npz", "implicit_p0_fixed"),
              ("step_jzb_policy_implicit_24x18.npz", "implicit_p0_fixed"),
              # the seamount policy on the semi-implicit core (Picard / Robin solve; a float64 golden)
              ("step_seamount_implicit_24x18.npz", "implicit_p0_fixed"),
              ("step_implicit_shapiro_20x18.npz", "implicit_p0_fixed")]


@pytest.mark.parametrize("fname,core", STEP_FILES)
def test_emulated_step_matches_reference(fname, core):
    A, Sc, OUT = load_step_golden(fname)
    E = emul.EmulCore(A, Sc, core)
    done = 0
    for n in sorted(OUT):
        its = E.steps(n - done)
        done = n
        for f, ref in OUT[n].items():
            if f.startswith("scalar") or f == "cg_iters":
                continue
            err, bound = step_field_error(E.F[f], ref, f, n, fname)
            assert err < bound, (fname, n, f, err)
        if "cg_iters" in OUT[n]:
            assert [int(v) for v in its] == [int(v) for v in OUT[n]["cg_iters"]]
        if "scalar_cg_iterations" in OUT[n]:
            # the tide policies' solve count of the last step
            assert int(its[-1]) == int(OUT[n]["scalar_cg_iterations"])


def _case(name):
    from neuralpom_b200 import cases
    if name == "seamount":
        return cases.seamount(24, 20), "implicit_p0_fixed"
    if name == "noise_basin":
        return cases.noise_basin(20, 18), "explicit"
    return cases.double_gyre(16, 14, "explicit"), "explicit"


@pytest.mark.parametrize("name", ["seamount", "noise_basin", "double_gyre"])
def test_emulated_step_matches_oracle_on_cases(name):
    (A, Sc), core = _case(name)
    Sc = dict(Sc)
    im, jm, kb = A["u"].shape
    Sc.update(im=im, jm=jm, kb=kb)
    E = emul.EmulCore(A, Sc, core)
    S = {k: v.copy() for k, v in A.items()}
    P = oracle_params(Sc, A, core)
    # first step from rest (internal mode skipped) and one full step
    for _ in range(2):
        E.steps(1)
        O.run(S, P, 1, core)
    for f in ("u", "v", "t", "s", "el", "q2", "km", "kh", "w", "rho", "ua", "va"):
        assert rel_err(E.F[f], S[f]) < 2e-4, (name, f, rel_err(E.F[f], S[f]))


@pytest.mark.parametrize("fname,core", [("step_mpdata_12x10.npz", "explicit"),
                                        ("step_mpdata_implicit_12x10.npz", "implicit_p0_fixed")])
def test_emulated_mpdata_step_matches_reference(fname, core):
    """MPDATA tracer advection (nadv = 2: ADVT2 + SMOL_ADIF,
    explicit/tracers.py:571-888, on the semi-implicit core through its
    numerics policy), the device bodies run on the CPU, against the
    reference's own steps (1e-5 after one step, 1e-4 after three)."""
    A, Sc, OUT = load_step_golden(fname)
    assert int(Sc["nadv"]) == 2
    E = emul.EmulCore(A, Sc, core)
    done = 0
    for n in sorted(OUT):
        E.steps(n - done)
        done = n
        tol = 1e-5 if n == 1 else 1e-4
        for f, ref in OUT[n].items():
            if f.startswith("scalar") or f == "cg_iters":
                continue
            assert rel_err(E.F[f], ref) < tol, (n, f, rel_err(E.F[f], ref))
    # and the centred scheme on the same inputs is far from it
    E1 = emul.EmulCore(A, dict(Sc, nadv=1), core)
    E1.steps(1)
    assert rel_err(E1.F["t"], OUT[1]["t"]) > 3e-5      # 7e-5: one step of different advection
