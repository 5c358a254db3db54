"""Generate the golden vectors that pin the oracle to the reference core.

Run where the reference package is importable: ``NPOM_REFERENCE_SRC`` names
the ``src`` directory of its sources (or the ``baseline/_ref`` install is
used)::

    python tests/golden/make_golden.py [proft] [steps] [adjoint] [coastal] [step_adjoint] [coupling] [mpdata]
        [pom08] [seamount] [shapiro]

Writes ``tests/golden/*.npz``.  Every file records the reference's own CPU
float32 outputs on seeded inputs; nothing here is needed at test time except
the written fixtures.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import ref_harness as rh  # noqa: E402

# Fields written by one internal step that the golden files keep.
OUTPUT_FIELDS = (
    "u", "ub", "v", "vb", "w", "t", "tb", "s", "sb", "rho", "q2", "q2b", "q2l", "q2lb",
    "km", "kh", "kq", "l", "aam", "advx", "advy", "curv", "drhox", "drhoy",
    "el", "elb", "elf", "et", "etb", "etf", "d", "dt", "ua", "uab", "uaf", "va", "vab", "vaf",
    "utf", "utb", "vtf", "vtb", "egf", "egb", "adx2d", "ady2d", "drx2d", "dry2d", "aam2d",
    "advua", "advva", "fluxua", "fluxva", "wubot", "wvbot", "tps", "wusurf", "wtsurf", "wssurf",
)


def perturbed_core(name, im, jm, seed):
    """Production-configured reference core, clock at 1000 days (so the first
    step runs the internal mode, as in the reference's own tests), spun up two
    steps, then given seeded perturbations on every prognostic field."""
    import torch
    core = rh.build_reference_core(name, im, jm)
    core.time = core.time0 = 1000.0
    rh.advance(core, name, 2)
    g = torch.Generator().manual_seed(seed)

    def rn(shape):
        return torch.randn(shape, generator=g, dtype=torch.float32)

    def ru(shape):
        return torch.rand(shape, generator=g, dtype=torch.float32)

    fsm3, dum3, dvm3 = core.fsm[:, :, None], core.dum[:, :, None], core.dvm[:, :, None]
    p3 = rn(core.t.shape)
    core.t = core.t + 0.5 * p3 * fsm3
    core.tb = core.tb + 0.45 * p3 * fsm3 + 0.05 * rn(core.t.shape) * fsm3
    p3 = rn(core.s.shape)
    core.s = core.s + 0.1 * p3 * fsm3
    core.sb = core.sb + 0.1 * p3 * fsm3
    for f, m in (("u", dum3), ("ub", dum3), ("v", dvm3), ("vb", dvm3)):
        setattr(core, f, getattr(core, f) + 0.05 * rn(core.u.shape) * m)
    for f, m in (("ua", core.dum), ("uab", core.dum), ("va", core.dvm), ("vab", core.dvm)):
        setattr(core, f, getattr(core, f) + 0.02 * rn(core.ua.shape) * m)
    for f in ("el", "elb", "et", "etb"):
        setattr(core, f, getattr(core, f) + 0.05 * rn(core.el.shape) * core.fsm)
    core.elf = core.el.clone()
    core.etf = core.et.clone()
    core.d = core.h + core.el
    core.dt = core.h + core.et
    for f in ("q2", "q2b", "q2l", "q2lb"):
        cur = getattr(core, f)
        setattr(core, f, cur * (1.0 + 0.5 * ru(cur.shape)) + 1e-6 * ru(cur.shape))
    for f in ("km", "kh", "kq"):
        cur = getattr(core, f)
        setattr(core, f, cur * (1.0 + 0.3 * ru(cur.shape)))
    core.aam = core.aam * (1.0 + 0.3 * ru(core.aam.shape))
    core.wubot = core.wubot + 1e-5 * rn(core.el.shape) * core.dum
    core.wvbot = core.wvbot + 1e-5 * rn(core.el.shape) * core.dvm
    return core


def make_step_golden(name, im, jm, seed, steps=(1, 3), core=None, tag=None):
    import torch
    if core is None:
        core = perturbed_core(name, im, jm, seed)
    arrays, scalars = rh.extract_state(core)
    out = {f"in__{k}": v for k, v in arrays.items()}
    for k, v in scalars.items():
        out[f"scalar__{k}"] = np.asarray(v)
    done = 0
    for n in steps:
        if hasattr(core, "_eta_solver_iteration_history"):
            core._eta_solver_iteration_history = []
        rh.advance(core, name, n - done)
        done = n
        a, _ = rh.extract_state(core)
        for f in OUTPUT_FIELDS:
            out[f"out{n}__{f}"] = a[f]
        out[f"out{n}__scalar_time"] = np.asarray(float(core.time))
        hist = getattr(core, "_eta_solver_iteration_history", None)
        if hist:  # (a case policy's own solve keeps no history)
            out[f"out{n}__cg_iters"] = np.asarray(hist, dtype=np.int32)
    tag = tag or ("explicit" if name == "explicit" else "implicit")
    path = os.path.join(HERE, f"step_{tag}_{im}x{jm}.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path))
    _ = torch


def make_proft_golden():
    """Seeded column fixture of the reference's strict-vertical tests
    (``tests/test_strict_vertical.py:11-21``, seed 817, 3x4 columns, kb=6)
    passed through the reference ``TracersMixin.proft`` for nbc 1-4."""
    import torch
    from neuralpom.cores.implicit_p0_fixed.strict_vertical import _reference
    out = {}
    for dtype, tag in ((torch.float64, "f64"), (torch.float32, "f32")):
        g = torch.Generator().manual_seed(817)
        kb = 6

        def rnd(shape):
            return torch.rand(shape, generator=g, dtype=dtype)
        shape = (3, 4)
        inputs = [torch.linspace(0, -1, kb, dtype=dtype), 10 + rnd((*shape, kb)), rnd(shape) * 1e-5,
                  rnd(shape) + 10, 100 + rnd(shape) * 20, rnd(shape) * .1,
                  torch.full((kb,), 1 / (kb - 1), dtype=dtype), torch.full((kb,), 1 / (kb - 1), dtype=dtype),
                  rnd(shape) * 1e-4, rnd((*shape, kb)) * 1e-3]
        names = ("z", "f", "wfsurf", "fsurf", "h", "etf", "dz", "dzz", "swrad", "kh")
        for n, v in zip(names, inputs):
            out[f"{tag}__{n}"] = v.numpy()
        for nbc in (1, 2, 3, 4):
            res = _reference(inputs, (nbc, 1200., 2, 1e-6))
            out[f"{tag}__nbc{nbc}__f"] = res[0].numpy()
            out[f"{tag}__nbc{nbc}__dh"] = res[1].numpy()
    path = os.path.join(HERE, "proft_strict_fixture.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path))


def make_coastal_golden(im=40, jm=34, seed=4):
    """The explicit core with an open southern boundary (Flather, rfs = 1,
    boundary elevation 1 m) on the coastal basin of
    ``neuralpom_b200.cases.coastal_tide``, clock at 0.25 days so that the
    first step runs the internal mode."""
    sys.path.insert(0, ROOT)
    from neuralpom_b200 import cases
    A, Sc = cases.coastal_tide(im, jm, seed=seed)
    Sc = dict(Sc)
    Sc.update(time=0.25, time0=0.25)
    core = rh.build_reference_core("explicit", im, jm)
    rh.load_state(core, A, Sc)
    make_step_golden("explicit", im, jm, seed, core=core, tag="coastal")


def make_eta_adjoint_golden(im=20, jm=18, seed=21):
    """Forward and backward of the reference's free-surface solve
    (``POM2K_Core.solve_implicit_eta_cg`` under autograd, i.e.
    ``_ImplicitEtaSolveFunction``, core.py:24-59 and 231-252) on a perturbed
    production core: seeded rhs, depth and cotangent g; J = sum(g * x)."""
    import torch
    name = "implicit_p0_fixed"
    core = perturbed_core(name, im, jm, seed)
    arrays, scalars = rh.extract_state(core)
    g = torch.Generator().manual_seed(seed + 1000)
    fsm = core.fsm
    rhs = (core.elb + 0.02 * torch.randn(core.el.shape, generator=g) * fsm).detach().requires_grad_(True)
    d2d = (core.d * (1.0 + 0.05 * torch.rand(core.el.shape, generator=g))).detach().requires_grad_(True)
    x0 = (2.0 * core.el - core.elb).detach()
    cot = torch.randn(core.el.shape, generator=g) * fsm
    tol = 1.0e-10
    core._eta_solver_iteration_history = []
    x = core.solve_implicit_eta_cg(rhs, d2d, max_iter=200, tol=tol, print_cg_residual=False, initial_guess=x0)
    fwd_its = list(core._eta_solver_iteration_history)
    (x * cot).sum().backward()
    out = {f"in__{k}": v for k, v in arrays.items()}
    for k, v in scalars.items():
        out[f"scalar__{k}"] = np.asarray(v)
    out.update({"adj__rhs": rhs.detach().numpy(), "adj__d2d": d2d.detach().numpy(), "adj__x0": x0.numpy(),
                "adj__x": x.detach().numpy(), "adj__g": cot.numpy(), "adj__grad_rhs": rhs.grad.numpy(),
                "adj__grad_d": d2d.grad.numpy(), "adj__tol": np.asarray(tol),
                "adj__fwd_its": np.asarray(fwd_its, dtype=np.int32)})
    path = os.path.join(HERE, f"eta_adjoint_{im}x{jm}.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path))


# State fields of the explicit core that carry a cotangent (everything the
# step reads or writes apart from geometry, forcing and boundary arrays).
ADJ_STATE_FIELDS = (
    "u", "ub", "uf", "v", "vb", "vf", "w", "t", "tb", "s", "sb", "rho", "q2", "q2b", "q2l", "q2lb", "km", "kh",
    "kq", "l", "aam", "advx", "advy", "drhox", "drhoy", "curv", "el", "elb", "elf", "et", "etb", "etf", "d", "dt",
    "ua", "uab", "uaf", "va", "vab", "vaf", "utf", "utb", "vtf", "vtb", "egf", "egb", "adx2d", "ady2d", "drx2d",
    "dry2d", "aam2d", "advua", "advva", "fluxua", "fluxva", "wubot", "wvbot", "tps",
)
ADJ_COT_FIELDS = ("u", "ub", "v", "vb", "t", "tb", "s", "sb", "el", "elb", "ua", "uab", "va", "vab", "q2", "q2l",
                  "km", "kh", "et", "etb", "egb", "utb", "vtb", "wubot", "wvbot", "rho")


def make_step_adjoint_golden(tag, core, steps=(1, 3), seed=0, cot_fields=ADJ_COT_FIELDS, name="explicit"):
    """Reverse mode of the reference's step under torch autograd
    (``SparsePhysics.advance(..., differentiable=True)``, sparse_physics.py:
    91-149): seeded cotangents on ``cot_fields`` after ``n`` steps,
    J = sum(cot * state), and dJ/d(start state) for every state field."""
    import torch
    arrays, scalars = rh.extract_state(core)
    im, jm = arrays["u"].shape[:2]
    out = {f"in__{k}": v for k, v in arrays.items()}
    for k, v in scalars.items():
        out[f"scalar__{k}"] = np.asarray(v)
    g = torch.Generator().manual_seed(seed)
    cot = {f: torch.randn(arrays[f].shape, generator=g, dtype=torch.float32) for f in cot_fields}
    for f, v in cot.items():
        out[f"cot__{f}"] = v.numpy()
    for n in steps:
        c2 = rh.build_reference_core(name, im, jm)
        rh.load_state(c2, arrays, scalars)
        leaves = {}
        for f in ADJ_STATE_FIELDS:
            leaves[f] = getattr(c2, f).detach().clone().requires_grad_(True)
            setattr(c2, f, leaves[f])
        rh.advance(c2, name, n, differentiable=True)
        loss = sum((getattr(c2, f) * cot[f]).sum() for f in cot_fields)
        loss.backward()
        for f in ADJ_STATE_FIELDS:
            gr = leaves[f].grad
            if gr is not None and bool(torch.any(gr != 0)):
                out[f"grad{n}__{f}"] = gr.numpy()
    path = os.path.join(HERE, f"step_adjoint_{tag}_{im}x{jm}.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path))


def make_step_adjoint_goldens():
    core = perturbed_core("explicit", 12, 10, 31)
    core.time0 = float(core.time)
    make_step_adjoint_golden("explicit", core, steps=(1, 3), seed=32)
    core = perturbed_core("explicit", 12, 10, 33)
    core.time = core.time0 = 0.0
    make_step_adjoint_golden("rest", core, steps=(1, 2), seed=34)
    sys.path.insert(0, ROOT)
    from neuralpom_b200 import cases
    A, Sc = cases.coastal_tide(16, 14, seed=4)
    Sc = dict(Sc)
    Sc.update(time=0.25, time0=0.25)
    core = rh.build_reference_core("explicit", 16, 14)
    rh.load_state(core, A, Sc)
    rh.advance(core, "explicit", 3)
    core.time0 = float(core.time)
    make_step_adjoint_golden("coastal", core, steps=(1,), seed=35,
                             cot_fields=("u", "v", "t", "s", "el", "ua", "va", "q2", "km"))
    name = "implicit_p0_fixed"
    core = perturbed_core(name, 12, 10, 36)
    core.time0 = float(core.time)
    make_step_adjoint_golden("implicit", core, steps=(1, 3), seed=37, name=name)
    core = perturbed_core(name, 12, 10, 38)
    core.time = core.time0 = 0.0
    make_step_adjoint_golden("implicit_rest", core, steps=(1, 2), seed=39, name=name)


COUPLING_LEAVES = ("u", "ub", "v", "vb", "t", "tb", "s", "sb", "rho", "et", "etf", "dt")


def make_coupling_golden(im=12, jm=10, seed=41):
    """The reference's corrector coupling under torch autograd
    (hybrid/sparse_coupling.py:10-82) on a perturbed explicit core:
    apply_joint_correction with a seeded raw output large enough to engage
    the paired limiter, and pressure_velocity_error against a perturbed
    reference (t, s); seeded cotangents on every output, gradients of the
    state leaves and of raw."""
    import torch
    from neuralpom.hybrid import sparse_coupling as sc
    core = perturbed_core("explicit", im, jm, seed)
    arrays, scalars = rh.extract_state(core)
    out = {f"in__{k}": v for k, v in arrays.items()}
    for k, v in scalars.items():
        out[f"scalar__{k}"] = np.asarray(v)
    g = torch.Generator().manual_seed(seed + 1)
    raw = (2.0 * torch.randn((sc.OUTPUT_CHANNELS, im, jm), generator=g)).requires_grad_(True)
    scales = {"u": 0.05, "v": 0.05, "t": 0.2, "s": 0.05}
    leaves = {}
    for f in COUPLING_LEAVES:
        leaves[f] = getattr(core, f).detach().clone().requires_grad_(True)
        setattr(core, f, leaves[f])
    info = sc.apply_joint_correction(core, raw, scales)
    outs = {f: getattr(core, f) for f in ("u", "ub", "v", "vb", "t", "tb", "s", "sb", "rho")}
    cot = {f: torch.randn(v.shape, generator=g) for f, v in outs.items()}
    loss = sum((outs[f] * cot[f]).sum() for f in outs) + 3.0 * info["ts_limit_factor"] + 5.0 * info["t_budget"]
    loss.backward()
    out["jc__raw"] = raw.detach().numpy()
    out["jc__scales"] = np.array([scales[f] for f in sc.OUTPUT_FIELDS])
    for f, v in outs.items():
        out[f"jc_out__{f}"] = v.detach().numpy()
        out[f"jc_cot__{f}"] = cot[f].numpy()
    for k in ("ts_limit_factor", "t_budget", "s_budget"):
        out[f"jc_info__{k}"] = np.asarray(float(info[k]))
    out["jc_grad__raw"] = raw.grad.numpy()
    for f in COUPLING_LEAVES:
        if leaves[f].grad is not None:
            out[f"jc_grad__{f}"] = leaves[f].grad.numpy()
    # pressure_velocity_error on a fresh copy of the start state
    c2 = rh.build_reference_core("explicit", im, jm)
    rh.load_state(c2, arrays, scalars)
    leaves = {}
    for f in COUPLING_LEAVES:
        leaves[f] = getattr(c2, f).detach().clone().requires_grad_(True)
        setattr(c2, f, leaves[f])
    ref_t = (c2.t.detach() + 0.3 * torch.randn(c2.t.shape, generator=g) * c2.fsm[:, :, None]).requires_grad_(True)
    ref_s = (c2.s.detach() + 0.05 * torch.randn(c2.s.shape, generator=g) * c2.fsm[:, :, None]).requires_grad_(True)
    ku, kv = sc.pressure_velocity_error(c2, ref_t, ref_s)
    cu, cv = torch.randn(ku.shape, generator=g), torch.randn(kv.shape, generator=g)
    ((ku * cu).sum() + (kv * cv).sum()).backward()
    out["pv__ref_t"], out["pv__ref_s"] = ref_t.detach().numpy(), ref_s.detach().numpy()
    out["pv_out__u"], out["pv_out__v"] = ku.detach().numpy(), kv.detach().numpy()
    out["pv_cot__u"], out["pv_cot__v"] = cu.numpy(), cv.numpy()
    out["pv_grad__ref_t"], out["pv_grad__ref_s"] = ref_t.grad.numpy(), ref_s.grad.numpy()
    for f in COUPLING_LEAVES:
        if leaves[f].grad is not None:
            out[f"pv_grad__{f}"] = leaves[f].grad.numpy()
    path = os.path.join(HERE, f"coupling_{im}x{jm}.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "limit factor", float(info["ts_limit_factor"]))


def make_mpdata_golden(im=12, jm=10, seed=51):
    """Both cores with MPDATA tracer advection (nadv = 2, ADVT2 and
    SMOL_ADIF, explicit/tracers.py:571-888; the semi-implicit core reaches
    its copy through its numerics policy, implicit_p0_fixed/numerics/
    double_gyre.py:60-74) on perturbed production states, 1 and 3 steps."""
    core = perturbed_core("explicit", im, jm, seed)
    core.nadv = 2
    make_step_golden("explicit", im, jm, seed, core=core, tag="mpdata")
    name = "implicit_p0_fixed"
    core = perturbed_core(name, im, jm, seed + 5)
    core.nadv = 2
    make_step_golden(name, im, jm, seed + 5, core=core, tag="mpdata_implicit")


def make_mpdata_adjoint_golden(im=12, jm=10, seed=52, steps=(1, 3), ndirs=2, eps=1e-6, name="explicit",
                               tag="mpdata"):
    """Reverse mode of the explicit step with MPDATA tracer advection
    (nadv = 2) on a perturbed production state, 1 and 3 steps.

    The reference's autograd of ADVT2 is not the derivative of its forward:
    SMOL_ADIF reassigns slices of the mass fluxes in place after abs() and
    the square have saved them (explicit/tracers.py:607-633,648-667,
    685-706).  Without the step checkpoint torch refuses that backward;
    under SparsePhysics' non-reentrant checkpoint (sparse_physics.py:140)
    the recomputation hands the backward the overwritten tensors,
    so the u, v, etb, ... gradients it returns differ from the forward's
    derivative by a few per cent.  This file therefore also records
    directional derivatives of the reference's own forward in float64:
    for every field autograd differentiates, ``ndirs`` seeded relative
    directions d = r |x| (r standard normal: no value crosses zero, so the
    clamps of the small turbulence fields keep their branch;
    ``dir{n}__{f}__{q}``) and the central difference
    (J(x + eps d) - J(x - eps d)) / (2 eps) of J = sum(cot * state after n
    steps) (``fd{n}__{f}__{q}``)."""
    import torch
    core = perturbed_core(name, im, jm, seed)
    core.nadv = 2
    core.time0 = float(core.time)
    make_step_adjoint_golden(tag, core, steps=steps, seed=seed + 1, name=name)
    path = os.path.join(HERE, f"step_adjoint_{tag}_{im}x{jm}.npz")
    z = dict(np.load(path))
    A = {k[4:]: v for k, v in z.items() if k.startswith("in__")}
    Sc = {k[8:]: v.item() for k, v in z.items() if k.startswith("scalar__")}
    cot = {k[5:]: v for k, v in z.items() if k.startswith("cot__")}
    g = np.random.default_rng(seed + 2)

    def loss(n, f, d):
        c2 = rh.build_reference_core(name, im, jm)
        rh.load_state(c2, A, Sc)
        rh.ReferenceFloat64.promote(c2)
        with rh.ReferenceFloat64():
            if hasattr(c2, "_build_acceleration_cache"):
                c2._build_acceleration_cache()
            setattr(c2, f, getattr(c2, f) + torch.from_numpy(d))
            rh.advance(c2, name, n)
        return sum(float((getattr(c2, h).detach().double() * torch.from_numpy(cot[h]).double()).sum())
                   for h in cot)

    for n in steps:
        fields = [k.split("__")[1] for k in z if k.startswith(f"grad{n}__")]
        for f in fields:
            for q in range(ndirs):
                d = g.standard_normal(A[f].shape) * np.abs(A[f].astype(np.float64))
                z[f"dir{n}__{f}__{q}"] = d.astype(np.float32)
                d = z[f"dir{n}__{f}__{q}"].astype(np.float64)
                z[f"fd{n}__{f}__{q}"] = np.asarray((loss(n, f, eps * d) - loss(n, f, -eps * d)) / (2 * eps))
    np.savez_compressed(path, **z)
    print("wrote", path, os.path.getsize(path))


def make_seamount_golden(im=24, jm=18, seed=71, steps=(1, 3)):
    """The explicit core under the reference's seamount case policy
    (cores/case_adapters/seamount_runtime.py:6-25: the seamount boundary of
    seamount_boundary.py and the POM08-WAD closure), installed by the
    reference's own installer on an open-east/west seamount
    (``cases.open_seamount``) with seeded T and u perturbations, clock at
    0.25 day; 1 and 3 steps."""
    import torch
    sys.path.insert(0, ROOT)
    from neuralpom_b200 import cases
    from neuralpom.cores.case_adapters import seamount_runtime
    A, Sc = cases.open_seamount(im, jm)
    g = np.random.default_rng(seed)
    fsm3, dum3 = A["fsm"][:, :, None], A["dum"][:, :, None]
    for f, sd, m in (("t", 0.2, fsm3), ("u", 0.02, dum3), ("v", 0.02, A["dvm"][:, :, None])):
        p = (sd * g.standard_normal(A[f].shape) * m).astype(np.float32)
        p[:, :, -1] = 0.0
        A[f] = A[f] + p
        A[f[0] + "b"] = A[f[0] + "b"] + p
    A, Sc = cases.seamount_policy(A, Sc)
    Sc = dict(Sc, time=0.25, time0=0.25)
    core = rh.build_reference_core("explicit", im, jm)
    rh.load_state(core, {k: v for k, v in A.items() if hasattr(core, k)}, Sc)
    seamount_runtime.install(core, "explicit")
    torch.set_default_dtype(torch.float32)
    core.profq_form, core.zsh, core.obc_form = "pom08", 0.01, "seamount"
    make_step_golden("explicit", im, jm, seed, steps=steps, core=core, tag="seamount_explicit")


def make_seamount_implicit_golden(im=24, jm=18, seed=72, steps=(1, 3)):
    """The semi-implicit core under the reference's seamount case policy
    (seamount_runtime.install(core, "implicit"): its predictor, Robin CG
    with Picard iterations, corrector, body continuity and boundary, and
    the POM08-WAD closure) on ``cases.open_seamount`` with seeded T and u
    perturbations, clock at 0.25 day; 1 and 3 steps, in float64, the only
    precision whose Picard test (1e-11 m) the policy can pass."""
    import torch
    sys.path.insert(0, ROOT)
    from neuralpom_b200 import cases
    from neuralpom.cores.case_adapters import seamount_runtime
    name = "implicit_p0_fixed"
    A, Sc = cases.open_seamount(im, jm, dte=5.0, isplit=30, core=name)
    g = np.random.default_rng(seed)
    fsm3, dum3 = A["fsm"][:, :, None], A["dum"][:, :, None]
    for f, sd, m in (("t", 0.2, fsm3), ("u", 0.02, dum3), ("v", 0.02, A["dvm"][:, :, None])):
        p = (sd * g.standard_normal(A[f].shape) * m).astype(np.float32)
        p[:, :, -1] = 0.0
        A[f] = A[f] + p
        A[f[0] + "b"] = A[f[0] + "b"] + p
    A, Sc = cases.seamount_policy(A, Sc, core=name)
    Sc = dict(Sc, time=0.25, time0=0.25)
    core = rh.build_reference_core(name, im, jm)
    rh.load_state(core, {k: v for k, v in A.items() if hasattr(core, k)}, Sc)
    for k, v in list(vars(core).items()):
        if torch.is_tensor(v) and v.is_floating_point():
            setattr(core, k, v.double())
    torch.set_default_dtype(torch.float64)
    seamount_runtime.install(core, "implicit")
    core.profq_form, core.zsh, core.obc_form = "pom08", 0.01, "seamount"
    make_step_golden(name, im, jm, seed, steps=steps, core=core, tag="seamount_implicit")
    torch.set_default_dtype(torch.float32)


def make_coastal_policy_golden(im=24, jm=18, steps=(1, 3), family="explicit"):
    """The explicit (or semi-implicit) core under the reference's coastal
    tide policy, set up the way its registry does (cores/case_adapters/
    registry.py:136-146: alpha and smoth of the family, the policy's step
    copies bound as methods, coastal_boundary.install with a tide table
    file, coastal_compat.install with the POM08-WAD closure) on
    ``cases.tidal_inlet`` (kb = 16), clock at 0.25 day; one internal step
    per call with the tide substep counter reset, as the registry's
    advancement does (registry.py:38-63); 1 and 3 steps.  The registry
    would refuse a float32 state; the steps run in float32, the arithmetic
    the B200 step restates."""
    import tempfile
    import torch
    from importlib import import_module
    sys.path.insert(0, ROOT)
    from neuralpom_b200 import cases
    from neuralpom.cores.case_adapters import coastal_boundary, coastal_compat, registry
    name = "explicit" if family == "explicit" else "implicit_p0_fixed"
    A, Sc = cases.tidal_inlet(im, jm, kb=16, core=name)
    Sc = dict(Sc, time=0.25, time0=0.25)
    core = rh.build_reference_core(name, im, jm)
    rh.load_state(core, {k: v for k, v in A.items() if hasattr(core, k)}, Sc)
    core.alpha, core.smoth = (0.225, 0.1) if family == "explicit" else (0.333, 0.15)
    for module, cls in (("momentum", "MomentumMixin"), ("tracers", "TracersMixin"), ("time_loop", "TimeLoopMixin")):
        registry._bind_mixin(core, getattr(import_module(
            f"neuralpom.cores.case_adapters.kernels.coastal_{family}_{module}"), cls))
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "tide.dat")
        np.savetxt(path, np.c_[A["tide_i"] + 1, A["tide_j"] + 1, A["tide_amp"], A["tide_phase"]])
        coastal_boundary.install(core, family, path)
    coastal_compat.install(core)
    torch.set_default_dtype(torch.float32)
    core.profq_form, core.zsh, core.obc_form = "pom08", 0.01, "coastal"

    arrays, scalars = rh.extract_state(core)
    out = {f"in__{k}": v for k, v in arrays.items()}
    for k, v in scalars.items():
        out[f"scalar__{k}"] = np.asarray(v)
    done = 0
    for n in steps:
        while done < n:
            core._tide_substep = 0
            rh.advance(core, name, 1)
            done += 1
        a, _ = rh.extract_state(core)
        for f in OUTPUT_FIELDS:
            out[f"out{n}__{f}"] = a[f]
        out[f"out{n}__cbc"] = a["cbc"]
        out[f"out{n}__scalar_time"] = np.asarray(float(core.time))
        if family != "explicit":
            out[f"out{n}__scalar_cg_iterations"] = np.asarray(int(core._validation_eta_iterations))
    tag = "coastal_policy" if family == "explicit" else "coastal_policy_implicit"
    path = os.path.join(HERE, f"step_{tag}_{im}x{jm}.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path))


def make_jzb_policy_golden(im=24, jm=18, steps=(1, 3), family="explicit"):
    """The explicit (or semi-implicit) core under the reference's Jiaozhou
    Bay tide policy, set up the way its registry does (cores/case_adapters/
    registry.py:147-156: alpha and smoth of the family, the coastal step
    copies of the family bound as methods, jzb_boundary.install with a
    tide table file, jzb_compat.install with the POM08-WAD closure) on
    ``cases.bay`` (kb = 16), clock at 0.25 day (ramp 0.083 of the bay's
    3-day ramp); one internal step per call with the tide substep counter
    reset, as the registry's advancement does (registry.py:38-63); 1 and 3
    steps."""
    import tempfile
    import torch
    from importlib import import_module
    sys.path.insert(0, ROOT)
    from neuralpom_b200 import cases
    from neuralpom.cores.case_adapters import jzb_boundary, jzb_compat, registry
    name = "explicit" if family == "explicit" else "implicit_p0_fixed"
    A, Sc = cases.bay(im, jm, kb=16, core=name)
    Sc = dict(Sc, time=0.25, time0=0.25)
    core = rh.build_reference_core(name, im, jm)
    rh.load_state(core, {k: v for k, v in A.items() if hasattr(core, k) and k != "period"}, Sc)
    core.alpha, core.smoth = (0.225, 0.1) if family == "explicit" else (0.333, 0.15)
    for module, cls in (("momentum", "MomentumMixin"), ("tracers", "TracersMixin"), ("time_loop", "TimeLoopMixin")):
        registry._bind_mixin(core, getattr(import_module(
            f"neuralpom.cores.case_adapters.kernels.coastal_{family}_{module}"), cls))
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "tide.dat")
        np.savetxt(path, np.c_[A["tide_i"] + 1, A["tide_j"] + 1, A["tide_amp"], A["tide_phase"]])
        jzb_boundary.install(core, family, path)
    jzb_compat.install(core)
    torch.set_default_dtype(torch.float32)
    core.profq_form, core.zsh, core.obc_form = "pom08", 0.01, "jzb"

    arrays, scalars = rh.extract_state(core)
    out = {f"in__{k}": v for k, v in arrays.items()}
    for k, v in scalars.items():
        out[f"scalar__{k}"] = np.asarray(v)
    done = 0
    for n in steps:
        while done < n:
            core._tide_substep = 0
            rh.advance(core, name, 1)
            done += 1
        a, _ = rh.extract_state(core)
        for f in OUTPUT_FIELDS:
            out[f"out{n}__{f}"] = a[f]
        out[f"out{n}__cbc"] = a["cbc"]
        out[f"out{n}__scalar_time"] = np.asarray(float(core.time))
        if family != "explicit":
            out[f"out{n}__scalar_cg_iterations"] = np.asarray(int(core._validation_eta_iterations))
    tag = "jzb_policy" if family == "explicit" else "jzb_policy_implicit"
    path = os.path.join(HERE, f"step_{tag}_{im}x{jm}.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path))


def make_shapiro_golden(im=20, jm=18, seed=81, gamma=0.05):
    """The semi-implicit core with its spatial Shapiro filters on (barotropic
    elevation after the solve, core.py:893-916, and tracers,
    numerics/double_gyre.py:78-131; production runs them at gamma 0) on a
    perturbed production state, 1 and 3 steps."""
    name = "implicit_p0_fixed"
    core = perturbed_core(name, im, jm, seed)
    core.barotropic_shapiro = gamma
    core.tracer_shapiro = gamma
    make_step_golden(name, im, jm, seed, core=core, tag="implicit_shapiro")


def make_pom08_goldens():
    """Both cores with the POM08-WAD closure of the reference's case
    policies bound by the reference's own installer
    (cores/case_adapters/fortran_compat.py:147-161, default reference
    pressure, zsh = 0.01 m) on perturbed production states: 1 and 3 steps of
    the explicit 12x10 core, 1 and 2 of the implicit 20x18 core."""
    from neuralpom.cores.case_adapters import fortran_compat
    for name, im, jm, seed, steps in (("explicit", 12, 10, 61, (1, 3)), ("implicit_p0_fixed", 20, 18, 62, (1, 2))):
        core = perturbed_core(name, im, jm, seed)
        fortran_compat.install(core, zsh=0.01)
        core.profq_form = "pom08"
        core.zsh = 0.01
        tag = "pom08_explicit" if name == "explicit" else "pom08_implicit"
        make_step_golden(name, im, jm, seed, steps=steps, core=core, tag=tag)


def main(which=("proft", "steps", "adjoint", "coastal", "step_adjoint", "coupling", "mpdata", "pom08", "seamount",
                "shapiro", "jzb", "coastal_implicit", "seamount_implicit")):
    src = rh.default_reference_path()
    if src is None:
        raise SystemExit("reference sources not found; set NPOM_REFERENCE_SRC")
    rh.import_reference(src)
    import torch
    torch.set_num_threads(1)
    if "proft" in which:
        make_proft_golden()
    if "steps" in which:
        make_step_golden("explicit", 12, 10, seed=11)
        make_step_golden("implicit_p0_fixed", 12, 10, seed=12)
        make_step_golden("implicit_p0_fixed", 20, 18, seed=13, steps=(1,))
    if "adjoint" in which:
        make_eta_adjoint_golden()
    if "coastal" in which:
        make_coastal_golden()
    if "step_adjoint" in which:
        make_step_adjoint_goldens()
    if "coupling" in which:
        make_coupling_golden()
    if "mpdata" in which:
        make_mpdata_golden()
        make_mpdata_adjoint_golden()
        make_mpdata_adjoint_golden(seed=54, steps=(1, 2), name="implicit_p0_fixed", tag="mpdata_implicit")
    if "pom08" in which:
        make_pom08_goldens()
    if "seamount" in which:
        make_seamount_golden()
        make_coastal_policy_golden()
    if "shapiro" in which:
        make_shapiro_golden()
    if "jzb" in which:
        make_jzb_policy_golden()
    if "coastal_implicit" in which:
        make_coastal_policy_golden(family="implicit")
        make_jzb_policy_golden(family="implicit")
    if "seamount_implicit" in which:
        make_seamount_implicit_golden()


if __name__ == "__main__":
    main(tuple(sys.argv[1:]) or ("proft", "steps", "adjoint", "coastal", "step_adjoint", "coupling", "mpdata",
                                 "pom08", "seamount", "shapiro", "jzb", "coastal_implicit",
                                 "seamount_implicit"))
