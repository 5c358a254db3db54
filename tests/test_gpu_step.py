"""Parity of the B200 step with the reference (golden vectors) and with the
oracle at the benchmark sizes, through the public drop-in API."""
import numpy as np
import pytest
import torch

from golden_io import load_step_golden, oracle_params, rel_err, step_field_error
from oracle import pom_oracle as O

pytestmark = pytest.mark.gpu

STEP_FILES = [("step_explicit_12x10.npz", "explicit"), ("step_implicit_12x10.npz", "implicit_p0_fixed"),
              ("step_implicit_20x18.npz", "implicit_p0_fixed"), ("step_coastal_40x34.npz", "explicit"),
              ("step_mpdata_12x10.npz", "explicit"), ("step_mpdata_implicit_12x10.npz", "implicit_p0_fixed"),
              # the POM08-WAD closure of the reference's case policies
              ("step_pom08_explicit_12x10.npz", "explicit"), ("step_pom08_implicit_20x18.npz", "implicit_p0_fixed"),
              # the seamount case policy (its boundary with the POM08-WAD closure)
              ("step_seamount_explicit_24x18.npz", "explicit"),
              # the coastal tide policy (tide cells, four-edge radiation, step copies, closure)
              ("step_coastal_policy_24x18.npz", "explicit"),
              # the reference's Jiaozhou Bay tide policy
              ("step_jzb_policy_24x18.npz", "explicit"),
              # both tide policies on the semi-implicit core
              ("step_coastal_policy_implicit_24x18.npz", "implicit_p0_fixed"),
              ("step_jzb_policy_implicit_24x18.npz", "implicit_p0_fixed"),
              # the seamount policy on the semi-implicit core (Picard / Robin solve; a float64 golden)
              ("step_seamount_implicit_24x18.npz", "implicit_p0_fixed"),
              # the semi-implicit core with its spatial Shapiro filters on (gamma 0.05)
              ("step_implicit_shapiro_20x18.npz", "implicit_p0_fixed")]


def _core(arrays, scalars, core):
    from neuralpom_b200 import resolve_core_class
    return resolve_core_class(core).from_state(arrays, scalars, device="cuda")


@pytest.mark.parametrize("fname,core", STEP_FILES)
def test_gpu_step_matches_reference_golden(fname, core):
    from neuralpom_b200 import B200Physics
    A, Sc, OUT = load_step_golden(fname)
    c = _core(A, Sc, core)
    phys = B200Physics(core_name=core)
    done = 0
    for n in sorted(OUT):
        c._eta_solver_iteration_history = []
        phys.advance(c, steps=n - done)
        assert c.iint == n - done
        done = n
        # 1e-5 relative after one step; 1e-4 after three (rounding growth)
        for f, ref in OUT[n].items():
            if f.startswith("scalar") or f == "cg_iters":
                continue
            err, bound = step_field_error(getattr(c, f).cpu().numpy(), ref, f, n, fname)
            assert err < bound, (fname, n, f, err)
        if "cg_iters" in OUT[n]:
            assert c._eta_solver_iteration_history == [int(v) for v in OUT[n]["cg_iters"]]
        if "scalar_cg_iterations" in OUT[n]:
            # the tide policies' own solve: the reference's count at the last step
            assert c._eta_solver_iteration_history[-1] == int(OUT[n]["scalar_cg_iterations"])
        assert abs(c.time - float(OUT[n]["scalar_time"])) < 1e-9


def _oracle_pair(case, steps, core):
    A, Sc = case
    Sc = dict(Sc)
    im, jm, kb = A["u"].shape
    Sc.update(im=im, jm=jm, kb=kb)
    c = _core(A, Sc, core)
    S = {k: v.copy() for k, v in A.items()}
    P = oracle_params(Sc, A, core)
    from neuralpom_b200 import B200Physics
    phys = B200Physics(core_name=core)
    for _ in range(steps):
        phys.advance(c, steps=1)
        O.run(S, P, 1, core)
    return c, S


def test_gpu_seamount_90x82_matches_oracle():
    """The semi-implicit benchmark basin at full size: the first step from
    rest and three full steps (PCG tolerance 1e-10, FP64 dots).  The start
    from a uniform current against closed walls is violent, so the bound is
    the oracle's own sensitivity: 10x the spread that a 1-ulp change of T
    produces over the same four steps (measured here, per field)."""
    from neuralpom_b200 import cases
    A, Sc = cases.seamount(90, 82)
    c, S = _oracle_pair((A, Sc), 4, "implicit_p0_fixed")
    A2 = dict(A)
    A2["t"] = np.nextafter(A["t"], np.float32(np.inf)).astype(np.float32)
    Sc2 = dict(Sc)
    Sc2.update(im=90, jm=82, kb=16)
    S2 = {k: v.copy() for k, v in A2.items()}
    P2 = oracle_params(Sc2, A2, "implicit_p0_fixed")
    for _ in range(4):
        O.run(S2, P2, 1, "implicit_p0_fixed")
    for f in ("u", "v", "t", "s", "el", "q2", "km", "kh", "w", "rho", "ua", "va", "elf"):
        spread = rel_err(S2[f], S[f])
        err = rel_err(getattr(c, f).cpu().numpy(), S[f])
        assert err <= max(10.0 * spread, 1e-6), (f, err, spread)


def test_gpu_explicit_basin_64x64_matches_oracle():
    from neuralpom_b200 import cases
    c, S = _oracle_pair(cases.noise_basin(64, 64), 3, "explicit")
    for f in ("u", "v", "t", "s", "el", "q2", "km", "kh", "w", "rho", "ua", "va"):
        got = getattr(c, f).cpu().numpy()
        assert rel_err(got, S[f]) < 1e-4, (f, rel_err(got, S[f]))


def _budgets(art, fsm, h, et, dz, t, s):
    vol = art.astype(np.float64) * fsm * (h + et)
    kbm1 = t.shape[2] - 1
    lay_t = [(vol * dz[k] * t[:, :, k]).sum() for k in range(kbm1)]
    lay_s = [(vol * dz[k] * s[:, :, k]).sum() for k in range(kbm1)]
    return vol.sum(), np.array(lay_t), np.array(lay_s)


def test_gpu_conservation_diagnostics_match_oracle():
    """Volume and layer T/S budgets in FP64 (the reference's volume weights,
    hybrid/sparse_coupling.py:18-20) agree with the oracle to rounding."""
    from neuralpom_b200 import cases
    c, S = _oracle_pair(cases.double_gyre(40, 36, "implicit_p0_fixed"), 3, "implicit_p0_fixed")
    g = {n: getattr(c, n).cpu().numpy() for n in ("art", "fsm", "h", "et", "dz", "t", "s")}
    bg = _budgets(g["art"], g["fsm"], g["h"], g["et"], g["dz"], g["t"], g["s"])
    bo = _budgets(S["art"], S["fsm"], S["h"], S["et"], S["dz"], S["t"], S["s"])
    assert abs(bg[0] - bo[0]) / abs(bo[0]) < 1e-9
    np.testing.assert_allclose(bg[1], bo[1], rtol=1e-7)
    np.testing.assert_allclose(bg[2], bo[2], rtol=1e-7)


def test_gpu_run_twice_is_bitwise_deterministic():
    from neuralpom_b200 import B200Physics, cases
    A, Sc = cases.seamount(40, 36)
    outs = []
    for _ in range(2):
        c = _core(A, Sc, "implicit_p0_fixed")
        B200Physics(core_name="implicit_p0_fixed").advance(c, steps=3)
        outs.append({f: getattr(c, f).cpu().numpy() for f in ("u", "v", "t", "el", "q2", "kh")})
    for f in outs[0]:
        assert np.array_equal(outs[0][f], outs[1][f]), f


def test_gpu_vmax_raises_floating_point_error():
    """A barotropic velocity beyond vmaxl is reported by the device status
    word and raised on the host, like implicit time_loop.py:685-688."""
    from neuralpom_b200 import B200Physics, cases
    A, Sc = cases.double_gyre(20, 18, "implicit_p0_fixed")
    c = _core(A, Sc, "implicit_p0_fixed")
    c.vmaxl = 1e-12
    c.time = c.time0 = 1000.0
    with pytest.raises(FloatingPointError):
        B200Physics(core_name="implicit_p0_fixed").advance(c, steps=1)
    torch.cuda.synchronize()


def test_gpu_graph_replay_is_bitwise_identical_to_direct_launches(monkeypatch):
    """Steps replayed from the cached CUDA graph equal direct launches."""
    from neuralpom_b200 import B200Physics, cases
    A, Sc = cases.seamount(40, 36)
    Sc = dict(Sc)
    Sc.update(time=1000.0, time0=1000.0)
    outs = []
    for graph in ("0", "1"):
        monkeypatch.setenv("NPOM_GRAPH", graph)
        c = _core(A, Sc, "implicit_p0_fixed")
        B200Physics(core_name="implicit_p0_fixed").advance(c, steps=3)
        outs.append({f: getattr(c, f).cpu().numpy() for f in ("u", "v", "t", "el", "q2", "kh", "w")})
    for f in outs[0]:
        assert np.array_equal(outs[0][f], outs[1][f]), f


@pytest.mark.parametrize("grid", [(40, 36), (128, 112)])
def test_gpu_cluster_and_grid_barrier_pcg_agree(monkeypatch, grid):
    """The cluster (DSMEM) PCG and the grid-barrier PCG solve the same
    system to the PCG tolerance.  At 128x112 the cluster layout reads Sy from
    global memory (its fragment table does not fit in shared memory); the
    two solvers' DSTs round differently, so their fields are not bitwise
    equal, which shows that the cluster form ran."""
    from neuralpom_b200 import B200Physics, cases
    A, Sc = cases.seamount(*grid)
    outs = []
    for mode in ("coop", "cluster"):
        monkeypatch.setenv("NPOM_PCG", mode)
        c = _core(A, Sc, "implicit_p0_fixed")
        B200Physics(core_name="implicit_p0_fixed").advance(c, steps=2)
        outs.append({f: getattr(c, f).cpu().numpy() for f in ("el", "ua", "va", "u", "t")})
    for f in outs[0]:
        assert rel_err(outs[1][f], outs[0][f]) < 1e-4, f
    assert not np.array_equal(outs[0]["el"], outs[1]["el"])


@pytest.mark.parametrize("grid", [(177, 161), (90, 82)])
def test_gpu_coop_pcg_row_pair_dsts_equal_tiles(monkeypatch, grid):
    """The grid-barrier PCG's two forms of the DST stages -- tiles (the
    one-member solve) and row pairs (the batched solve: each i-stage fused
    with its j-stage over bands of whole rows, one grid barrier instead of
    three per preconditioner) -- sum every output in FP64 in index order, so
    both give the same bits: fields and PCG iteration counts compared
    bitwise over three steps."""
    from neuralpom_b200 import B200Physics, cases
    A, Sc = cases.seamount(*grid)
    monkeypatch.setenv("NPOM_PCG", "coop")
    outs = []
    for form in ("tiles", "rows"):
        monkeypatch.setenv("NPOM_PCG_DST", form)
        c = _core(A, Sc, "implicit_p0_fixed")
        B200Physics(core_name="implicit_p0_fixed").advance(c, steps=3)
        outs.append(({f: getattr(c, f).cpu().numpy() for f in ("el", "elf", "ua", "u", "t")},
                     list(c._eta_solver_iteration_history)))
    assert outs[0][1] == outs[1][1]
    for f in outs[0][0]:
        assert np.array_equal(outs[0][0][f], outs[1][0][f]), (f, rel_err(outs[1][0][f], outs[0][0][f]))


@pytest.mark.parametrize("core", ["implicit_p0_fixed", "explicit"])
def test_gpu_lane_columns_equal_thread_columns(monkeypatch, core):
    """The 16-lane column kernels (level per lane, shuffled recurrences)
    compute bitwise the same step as the thread-per-column bodies."""
    from neuralpom_b200 import B200Physics, cases
    A, Sc = cases.double_gyre(30, 26, core)
    Sc = dict(Sc)
    Sc.update(time=1000.0, time0=1000.0)
    outs = []
    for lanes in ("0", "1"):
        monkeypatch.setenv("NPOM_LANES", lanes)
        c = _core(A, Sc, core)
        B200Physics(core_name=core).advance(c, steps=2)
        outs.append({f: getattr(c, f).cpu().numpy() for f in ("u", "v", "ub", "t", "s", "el", "q2", "q2l", "km",
                                                              "kh", "kq", "l", "w", "rho", "aam", "drhox", "wubot")})
    for f in outs[0]:
        assert np.array_equal(outs[0][f], outs[1][f]), (f, rel_err(outs[1][f], outs[0][f]))


def test_gpu_coastal_open_boundary_matches_oracle():
    """The explicit core with the open southern boundary (Flather, rfs = 1)
    on a 96x80 coastal basin, three steps against the oracle."""
    from neuralpom_b200 import cases
    A, Sc = cases.coastal_tide(96, 80)
    Sc = dict(Sc)
    Sc.update(time=0.25, time0=0.25)
    c, S = _oracle_pair((A, Sc), 3, "explicit")
    for f in ("u", "v", "t", "s", "el", "q2", "km", "kh", "rho", "ua", "va", "elf", "w"):
        err, bound = step_field_error(getattr(c, f).cpu().numpy(), S[f], f, 3, "step_coastal")
        assert err < bound, (f, err)


def test_gpu_explicit_double_gyre_48_steps_matches_oracle():
    """The explicit basin of the 64x64x16 double-gyre set-up (dx = 20 km,
    dtE = 6 s, isplit 30) from rest for the full 48 internal steps in one
    call (graph replay after the first step): T and S within 1e-5, every
    field within 10x the oracle's own spread under a 1-ulp change of T
    (floor 1e-5)."""
    from neuralpom_b200 import B200Physics, cases
    A, Sc = cases.noise_basin(64, 64)
    Sc = dict(Sc)
    Sc.update(im=64, jm=64, kb=16)
    c = _core(A, Sc, "explicit")
    B200Physics(core_name="explicit").advance(c, steps=48)
    runs = []
    for perturb in (False, True):
        A2 = dict(A)
        if perturb:
            A2["t"] = np.nextafter(A["t"], np.float32(np.inf)).astype(np.float32)
        S = {k: v.copy() for k, v in A2.items()}
        O.run(S, oracle_params(Sc, A2, "explicit"), 48, "explicit")
        runs.append(S)
    S, S2 = runs
    for f in ("t", "s", "u", "v", "el", "q2", "kh", "km", "w", "rho", "ua", "va"):
        spread = rel_err(S2[f], S[f])
        bound = 1e-5 if f in ("t", "s") else max(10.0 * spread, 1e-5)
        err = rel_err(getattr(c, f).cpu().numpy(), S[f])
        assert err <= bound, (f, err, spread)


def test_gpu_restart_continues_bitwise(tmp_path):
    """save_restart after some steps, continue; load_restart, continue the
    same steps again: bitwise the same state (the reference's bit-exact
    restart test, tests/test_fixed_core_runtime.py:91-138)."""
    from neuralpom_b200 import cases, formats, resolve_core_class
    A, Sc = cases.seamount(24, 20)
    Sc = dict(Sc)
    core = resolve_core_class("implicit_p0_fixed").from_state(A, Sc, device="cuda")
    core.time0 = float(core.time)
    core.iend = 3
    core.run_time_loop()
    formats.save_restart(tmp_path / "restart.pt", core)
    t_restart = float(core.time)

    def advance():
        core.time0 = float(core.time)
        core.iend = 4
        core.run_time_loop()
        return {n: getattr(core, n).detach().cpu().clone() for n in ("u", "v", "t", "s", "el", "elb", "q2", "km")}

    first = advance()
    formats.load_restart(tmp_path / "restart.pt", core)
    assert float(core.time) == t_restart
    second = advance()
    for n in first:
        assert torch.equal(first[n], second[n]), n


@pytest.mark.parametrize("fname", ["step_pom08_explicit_12x10.npz", "step_seamount_explicit_24x18.npz",
                                   "step_coastal_policy_24x18.npz", "step_jzb_policy_24x18.npz",
                                   "step_coastal_policy_implicit_24x18.npz", "step_seamount_implicit_24x18.npz"])
def test_gpu_case_policies_refuse_gradients(fname):
    """The case policies advance forward only, as the reference's registry
    requires (cores/case_adapters/registry.py:38-41)."""
    A, Sc, OUT = load_step_golden(fname)
    c = _core(A, Sc, "explicit")
    c.t = c.t.detach().clone().requires_grad_(True)
    c.time0, c.iend = float(Sc["time"]), 1
    with pytest.raises(RuntimeError, match="no_grad"):
        c.run_time_loop()
