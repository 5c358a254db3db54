"""Kernel-level parity on the GPU: every phase of a step against the same
phase body run on the CPU (tests/emul), PROFT against the reference's
strict-vertical fixture and the oracle, the PCG solve against the oracle."""
import ctypes

import numpy as np
import pytest
import torch

from golden_io import golden_path, load_step_golden, oracle_params, rel_err
from oracle import pom_oracle as O

pytestmark = pytest.mark.gpu


def _lib():
    from neuralpom_b200 import _abi
    return _abi.load_library()


@pytest.mark.parametrize("fname,core", [("step_implicit_20x18.npz", "implicit_p0_fixed"),
                                        ("step_explicit_12x10.npz", "explicit")])
def test_each_phase_matches_emulated_body(fname, core):
    emul = pytest.importorskip("emul_harness")
    from neuralpom_b200 import _abi, resolve_core_class
    A, Sc, _ = load_step_golden(fname)
    E = emul.EmulCore(A, Sc, core)
    c = resolve_core_class(core).from_state(A, Sc, device="cuda")
    lib = _lib()
    c._workspace()
    ws = c._ws
    for name in _abi.WS_NAMES:
        ws["bufs"][name].copy_(torch.from_numpy(E.W[name]))
    stream = torch.cuda.current_stream()
    phases = [0, 1, 2, 3] + ([4] if core != "explicit" else []) + list(range(5, 15))
    for ph in phases:
        # start both sides from the emulator's state
        for n in _abi.FIELD_NAMES:
            getattr(c, n).copy_(torch.from_numpy(E.F[n]))
        for n in _abi.WS_NAMES:
            ws["bufs"][n].copy_(torch.from_numpy(E.W[n]))
        p = c.params()
        fa = c._fields()
        E.phase(ph, 1.0)
        _abi.check(lib.npom_run_phase(ctypes.byref(p), ctypes.byref(fa), ctypes.byref(ws["struct"]), ph, 1.0,
                                      ctypes.c_void_p(stream.cuda_stream)), "phase")
        torch.cuda.synchronize()
        # bodies are identical; only the device libm (cos/exp/pow) and the
        # parallel PCG reduction order can move the last bits
        tol = 1e-5 if ph == 3 and core != "explicit" else 2e-6
        for n in _abi.FIELD_NAMES:
            got = getattr(c, n).cpu().numpy()
            assert rel_err(got, E.F[n]) < tol, (_abi.PHASES[ph], n, rel_err(got, E.F[n]))


@pytest.mark.parametrize("nbc", [1, 2, 3, 4])
def test_proft_matches_reference_fixture(nbc):
    z = np.load(golden_path("proft_strict_fixture.npz"))
    g = lambda n: torch.from_numpy(np.ascontiguousarray(z[f"f32__{n}"])).cuda()  # noqa: E731
    f = g("f")
    im, jm, kb = f.shape
    out = torch.empty_like(f)
    dh = torch.empty((im, jm), device="cuda")
    keep = [g(n) for n in ("wfsurf", "fsurf", "h", "etf", "dz", "dzz", "swrad", "kh", "z")]
    wf, fs, h, etf, dz, dzz, sw, kh, zz = keep
    st = _lib().npom_proft(im * jm, kb, f.data_ptr(), wf.data_ptr(), fs.data_ptr(), nbc, h.data_ptr(),
                           etf.data_ptr(), 1200.0, dz.data_ptr(), dzz.data_ptr(), sw.data_ptr(), 2, kh.data_ptr(),
                           1e-6, zz.data_ptr(), out.data_ptr(), dh.data_ptr(), None)
    assert st == 0
    torch.cuda.synchronize()
    ref = z[f"f32__nbc{nbc}__f"]
    assert rel_err(out.cpu().numpy(), ref) < 2e-6
    assert np.array_equal(dh.cpu().numpy(), z[f"f32__nbc{nbc}__dh"])
    assert np.array_equal(out[..., -1].cpu().numpy(), z["f32__f"][..., -1])


def test_proft_many_columns_matches_oracle():
    g = np.random.default_rng(5)
    im, jm, kb = 200, 150, 16
    f = (10 + g.random((im, jm, kb))).astype(np.float32)
    kh = (g.random((im, jm, kb)) * 1e-2).astype(np.float32)
    h = (100 + 4000 * g.random((im, jm))).astype(np.float32)
    etf = (g.standard_normal((im, jm)) * 0.1).astype(np.float32)
    wf = (g.standard_normal((im, jm)) * 1e-5).astype(np.float32)
    fs = np.zeros((im, jm), np.float32)
    sw = np.zeros((im, jm), np.float32)
    from neuralpom_b200 import cases
    zl, zz, dz, dzz = cases.sigma_levels(kb)
    ref, dh_ref = O.proft(f, wf, fs, 1, h, etf, 1200.0, dz, dzz, sw, 2, kh, 2e-5, zl)
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    tf, tkh, th, te, tw, tfs, tsw, tdz, tdzz, tz = map(T, (f, kh, h, etf, wf, fs, sw, dz, dzz, zl))
    out = torch.empty_like(tf)
    dh = torch.empty_like(th)
    st = _lib().npom_proft(im * jm, kb, tf.data_ptr(), tw.data_ptr(), tfs.data_ptr(), 1, th.data_ptr(),
                           te.data_ptr(), 1200.0, tdz.data_ptr(), tdzz.data_ptr(), tsw.data_ptr(), 2, tkh.data_ptr(),
                           2e-5, tz.data_ptr(), out.data_ptr(), dh.data_ptr(), None)
    assert st == 0
    torch.cuda.synchronize()
    assert rel_err(out.cpu().numpy(), ref) < 1e-6


def test_pcg_solve_matches_oracle():
    """npom_pcg_solve on the seamount operator with a seeded RHS against the
    oracle PCG (same spectral preconditioner, tolerance 1e-10)."""
    from neuralpom_b200 import _abi, cases, resolve_core_class
    A, Sc = cases.seamount(90, 82)
    Sc = dict(Sc)
    Sc.update(im=90, jm=82, kb=16)
    c = resolve_core_class("implicit_p0_fixed").from_state(A, Sc, device="cuda")
    rng = np.random.default_rng(3)
    rhs = (rng.standard_normal((90, 82)) * A["fsm"]).astype(np.float32)
    c._workspace()
    c._ws["bufs"]["rhs"].copy_(torch.from_numpy(rhs))
    c.elf.zero_()
    p = c.params()
    fa = c._fields()
    lib = _lib()
    _abi.check(lib.npom_pcg_solve(ctypes.byref(p), ctypes.byref(fa), ctypes.byref(c._ws["struct"]),
                                  ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)), "pcg")
    bits, its = c.read_status(1)
    got = c.elf.cpu().numpy()
    P = oracle_params(Sc, A, "implicit_p0_fixed")
    C = O.implicit_coefficients(A, P)
    SC = O.spectral_cache(A, P, C)
    x, oits = O.pcg_solve(rhs, A["d"], np.zeros_like(rhs), A, P, C, SC, 200, 1e-10, 1e-10, "spectral")
    assert rel_err(got, x) < 1e-5
    assert abs(its[0] - oits) <= 2
    assert not (bits & _abi.DEV_PCG_MAXIT)
    # the solution satisfies the operator to the requested tolerance
    res = O.elliptic_apply(got, A["d"], C)[1:-1, 1:-1] - rhs[1:-1, 1:-1]
    assert np.linalg.norm(res) / np.linalg.norm(rhs[1:-1, 1:-1]) < 1e-4


@pytest.mark.parametrize("case", ["gyre", "coastal"])
@pytest.mark.parametrize("phase,env,fields", [
    (0, "NPOM_A1", ("advx", "advy", "curv", "wusurf", "wvsurf", "wtsurf", "wssurf")),
    (10, "NPOM_B5", ("uf", "vf", "q2", "q2b", "q2l", "q2lb", "t", "tb", "s", "sb"))])
def test_flux_tiles_equal_point_kernel(monkeypatch, case, phase, env, fields):
    """The flux-once tiled kernels of large grids (A1: forcing + ADVCT; B5:
    q filter + ADVT1 of T and S) write bitwise what the point kernels
    write."""
    from neuralpom_b200 import _abi, cases, resolve_core_class
    if case == "gyre":
        A, Sc = cases.double_gyre(37, 45, "explicit")
    elif case == "coastal":
        A, Sc = cases.coastal_tide(60, 52)
    else:
        A, Sc = cases.coastal_tide(180, 160)
    Sc = dict(Sc)
    Sc.update(time=0.25, time0=0.25)
    lib = _lib()
    stream = torch.cuda.current_stream()
    outs = []
    for form in ("points", "tiles"):
        monkeypatch.setenv(env, form)
        c = resolve_core_class("explicit").from_state(A, Sc, device="cuda")
        # a developed state: two steps, then the phase alone
        c.launch_steps(2, 0.25, 1, stream)
        p, fa, ws = c.params(), c._fields(), c._workspace()
        _abi.check(lib.npom_run_phase(ctypes.byref(p), ctypes.byref(fa), ctypes.byref(ws["struct"]), phase, 1.0,
                                      ctypes.c_void_p(stream.cuda_stream)), "phase")
        torch.cuda.synchronize()
        outs.append({n: getattr(c, n).cpu().numpy() for n in fields + ("u", "el")})
    for other in outs[1:]:
        for n in outs[0]:
            assert np.array_equal(outs[0][n], other[n]), n


@pytest.mark.parametrize("case", ["gyre", "coastal", "coastal_180x160"])
def test_cluster_subcycle_equals_grid_subcycle(monkeypatch, case):
    """On small grids the explicit external subcycle runs on one thread-block
    cluster with the hardware cluster barrier; it writes bitwise what the
    grid-barrier form and the one-launch-per-phase form (no barrier at all)
    write, for the phase alone and over whole steps.  The 180x160 grid runs
    the cluster form (NPOM_SUBCYCLE=nocoop) with two cells per thread."""
    from neuralpom_b200 import _abi, cases, resolve_core_class
    if case == "gyre":
        A, Sc = cases.double_gyre(37, 45, "explicit")
    else:
        A, Sc = cases.coastal_tide(60, 52)
    Sc = dict(Sc)
    Sc.update(time=0.25, time0=0.25)
    lib = _lib()
    stream = torch.cuda.current_stream()
    names = ("el", "elb", "elf", "ua", "uab", "uaf", "va", "vab", "vaf", "egf", "utf", "vtf", "d", "etf")
    outs = []
    for form in ("grid", "cluster", "phases", "nocoop"):
        monkeypatch.setenv("NPOM_SUBCYCLE", form)
        c = resolve_core_class("explicit").from_state(A, Sc, device="cuda")
        c.launch_steps(2, 0.25, 1, stream)
        p, fa, ws = c.params(), c._fields(), c._workspace()
        _abi.check(lib.npom_run_phase(ctypes.byref(p), ctypes.byref(fa), ctypes.byref(ws["struct"]), 3, 1.0,
                                      ctypes.c_void_p(stream.cuda_stream)), "phase")
        c.launch_steps(4, 0.25, 1, stream)
        torch.cuda.synchronize()
        bits, _ = c.read_status(1)
        assert bits == 0
        outs.append({n: getattr(c, n).cpu().numpy() for n in names + ("u", "v", "t")})
    for other in outs[1:]:
        for n in outs[0]:
            assert np.array_equal(outs[0][n], other[n]), n
