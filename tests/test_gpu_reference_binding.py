"""The reference's own executor driving a B200-bound reference core.

``neuralpom_b200.reference_binding`` gives the reference's ``POM2K_Core``
classes a ``run_time_loop`` on the B200 library.  These tests import the
unmodified reference (the ``baseline/_ref`` install, or
``NPOM_REFERENCE_SRC``), build its cores with its own constructor, advance
them with its own ``SparsePhysics`` -- whose ``_configure`` rebinds the
core's class on every advance -- and check that:

* the CUDA library ran (the bound module's device-step count, and results
  bitwise equal to the B200 host core's on the same state, which the
  PyTorch step cannot produce: its dot products are float32);
* the result matches the reference's golden step;
* ``advance(differentiable=True)`` (the reference's checkpointed chunks)
  gives the B200 step adjoint's gradients.
"""
import numpy as np
import pytest
import torch

from golden_io import load_step_golden, step_field_error
from oracle import ref_harness as rh

REF = rh.default_reference_path()
pytestmark = [pytest.mark.gpu, pytest.mark.skipif(REF is None, reason="reference package not importable")]

CASES = [("step_implicit_12x10.npz", "implicit_p0_fixed"), ("step_explicit_12x10.npz", "explicit")]
COMPARED = ("u", "v", "t", "s", "el", "elf", "ua", "va", "q2", "q2l", "km", "kh", "w", "rho", "aam", "uaf")


@pytest.fixture(autouse=True)
def _reference_importable():
    rh.import_reference(REF)


def _physics_kw(core_name):
    return dict(core_name="explicit", compiled_kernels=()) if core_name == "explicit" else {}


def _bound(fname, core_name):
    rh.import_reference(REF)
    from neuralpom_b200 import reference_binding as rb
    A, Sc, OUT = load_step_golden(fname)
    core = rh.build_reference_core(core_name, int(Sc["im"]), int(Sc["jm"]), device="cuda")
    rh.load_state(core, A, Sc)
    rb.bind(core)
    return core, A, Sc, OUT


def _b200(A, Sc, core_name):
    from neuralpom_b200 import resolve_core_class
    return resolve_core_class(core_name).from_state(A, Sc, device="cuda")


@pytest.mark.parametrize("fname,core_name", CASES)
def test_reference_executor_runs_the_b200_step(fname, core_name):
    from neuralpom.hybrid.sparse_physics import SparsePhysics
    from neuralpom_b200 import B200Physics
    from neuralpom_b200 import reference_binding as rb
    core, A, Sc, OUT = _bound(fname, core_name)
    bound_cls = type(core)
    b = _b200(A, Sc, core_name)
    phys = SparsePhysics("cuda", **_physics_kw(core_name))
    done = 0
    for n in sorted(OUT):
        before = rb.steps_on_device()
        if hasattr(core, "_eta_solver_iteration_history"):
            core._eta_solver_iteration_history = []
        phys.advance(core, steps=n - done)
        B200Physics(core_name=core_name).advance(b, steps=n - done)
        # the executor rebinds core.__class__ on every advance; the bound
        # class stays, and the steps ran on the device
        assert type(core) is bound_cls
        assert rb.steps_on_device() - before == n - done
        done = n
        for f in COMPARED:
            got = getattr(core, f).detach().cpu().numpy()
            assert np.array_equal(got, getattr(b, f).cpu().numpy()), f
            if f in OUT[n]:
                err, bound = step_field_error(got, OUT[n][f], f, n, fname)
                assert err < bound, (f, n, err)
        if "cg_iters" in OUT[n]:
            assert core._eta_solver_iteration_history == [int(v) for v in OUT[n]["cg_iters"]]
        assert abs(core.time - float(OUT[n]["scalar_time"])) < 1e-9
        assert core.iint == b.iint


@pytest.mark.parametrize("fname,core_name", CASES)
def test_reference_executor_differentiable_uses_the_b200_adjoint(fname, core_name):
    """SparsePhysics.advance(differentiable=True): the reference's
    checkpointed chunks around the bound step; gradients of an MSE loss
    against the B200 host core's differentiable advance (same step adjoint;
    its scatters are atomic, so equal to rounding rather than bitwise)."""
    from neuralpom.hybrid.sparse_physics import SparsePhysics
    from neuralpom_b200 import B200Physics
    from neuralpom_b200 import reference_binding as rb
    core, A, Sc, _ = _bound(fname, core_name)
    b = _b200(A, Sc, core_name)
    leaves = {}
    for c, tag in ((core, "ref"), (b, "b200")):
        for f in ("t", "s", "u", "v"):
            x = getattr(c, f).detach().clone().requires_grad_(True)
            setattr(c, f, x)
            leaves[(tag, f)] = x
    g = torch.Generator(device="cpu").manual_seed(5)
    tgt = {f: (getattr(b, f).detach().cpu() + 0.01 * torch.randn(getattr(b, f).shape, generator=g)).cuda()
           for f in ("u", "v", "t", "s")}
    before = rb.steps_on_device()
    SparsePhysics("cuda", chunk_steps=2, **_physics_kw(core_name)).advance(core, steps=3, differentiable=True)
    assert rb.steps_on_device() - before >= 3
    B200Physics("cuda", chunk_steps=2, core_name=core_name).advance(b, steps=3, differentiable=True)
    for f in ("u", "v", "t", "s", "el", "q2", "kh"):
        assert np.array_equal(getattr(core, f).detach().cpu().numpy(), getattr(b, f).detach().cpu().numpy()), f

    def loss(c):
        return sum(((getattr(c, f) - tgt[f]) ** 2).mean() for f in ("u", "v", "t", "s"))

    loss(core).backward()
    loss(b).backward()
    for f in ("t", "s", "u", "v"):
        gr = leaves[("ref", f)].grad.cpu().numpy()
        gb = leaves[("b200", f)].grad.cpu().numpy()
        scale = max(float(np.abs(gb).max()), 1e-30)
        assert float(np.abs(gr - gb).max()) / scale < 1e-5, f

