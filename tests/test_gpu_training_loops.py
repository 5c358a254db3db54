"""The reference's own training loops on a B200-bound core.

``full_bptt`` (``src/neuralpom/v1/engine.py:148-161``) and ``post_window``
(``src/neuralpom/v1/posttrain/truncated.py:6-47``) drive a runtime object
with the contract of the reference's ``Runtime`` (``v1/runtime.py:91-125``):
``advance`` through ``SparsePhysics`` (checkpointed chunks when
differentiable), ``correct`` by ``apply_joint_correction`` of a model's raw
output, ``score`` against target fields, ``detach``.  The runtime here keeps
that contract around one production double-gyre core and a seeded target
(the reference's datasets and normalisation assets are not needed for the
physics).  Each loop runs twice -- on the reference's PyTorch core and on
the same core class bound to the B200 library
(``neuralpom_b200.reference_binding``) -- and the losses and the gradients
reaching the model's parameters are compared.
"""

import numpy as np
import pytest
import torch

from oracle import ref_harness as rh

REF = rh.default_reference_path()
pytestmark = [pytest.mark.gpu, pytest.mark.skipif(REF is None, reason="reference package not importable")]

FIELDS = ("u", "v", "t", "s")


class CoreRuntime:
    """The reference Runtime's physics contract on one core (see module
    docstring); ``interval_steps`` internal steps per interval."""

    def __init__(self, core, core_name, interval_steps, target, chunk_steps=2):
        from neuralpom.hybrid.sparse_physics import SparsePhysics
        kw = dict(core_name="explicit", compiled_kernels=()) if core_name == "explicit" else {}
        self.core = core
        self.physics = SparsePhysics("cuda", chunk_steps=chunk_steps, **kw)
        self.interval_seconds = int(round(interval_steps * float(core.dti)))
        self.steps = interval_steps
        self.target = target
        self.start = {k: v.detach().clone() for k, v in vars(core).items() if torch.is_tensor(v)}
        self.scales = {f: 1.0 for f in FIELDS}
        self.advanced = 0

    def reset(self, day):
        for k, v in self.start.items():
            setattr(self.core, k, v.clone())
        self.core.time = day + self.interval_seconds / 86400.0

    def load_cached(self, member, day):
        self.reset(day)
        return {"packed": None}

    def advance(self, differentiable=False):
        self.physics.advance(self.core, steps=self.steps, differentiable=differentiable)
        self.advanced += self.steps

    def correct(self, model, packed=None):
        from neuralpom.hybrid.sparse_coupling import apply_joint_correction
        info = apply_joint_correction(self.core, model(), self.scales)
        return {"ts_limit_factor": info["ts_limit_factor"]}

    def detach(self):
        from neuralpom.hybrid.sparse_physics import SparsePhysics
        SparsePhysics.release_completed_rollout(self.core)

    def score(self, member, day, lead, include_eta=True):
        loss = sum(((getattr(self.core, f)[:, :, :15] - self.target[f]) ** 2).mean() for f in FIELDS)
        return loss, {"mse": loss}


class RawModel(torch.nn.Module):
    """A network stand-in: raw (60, im, jm) = a[c] * F[c] with seeded F."""

    def __init__(self, im, jm, seed=3):
        super().__init__()
        g = torch.Generator().manual_seed(seed)
        self.register_buffer("feature", 1e-3 * torch.randn((60, im, jm), generator=g))
        self.a = torch.nn.Parameter(torch.linspace(0.5, 1.5, 60))

    def forward(self):
        return self.a[:, None, None] * self.feature


def _runtimes(core_name, im, jm, interval_steps):
    """(reference runtime, B200-bound runtime) on the same perturbed core."""
    rh.import_reference(REF)
    import make_golden as mg
    from neuralpom_b200 import reference_binding as rb
    base = mg.perturbed_core(core_name, im, jm, 21)
    arrays, scalars = rh.extract_state(base)
    g = np.random.default_rng(5)
    target = {f: torch.tensor(arrays[f][:, :, :15] + 1e-2 * g.standard_normal(arrays[f][:, :, :15].shape),
                              dtype=torch.float32, device="cuda") for f in FIELDS}
    out = []
    for bind in (False, True):
        core = rh.build_reference_core(core_name, im, jm, device="cuda")
        rh.load_state(core, arrays, scalars)
        if bind:
            rb.bind(core)
        out.append(CoreRuntime(core, core_name, interval_steps, target))
    return out


def _grads(loop, rt, model):
    model.zero_grad()
    loss, metrics = loop(rt, model)
    loss.backward()
    return float(loss.detach()), model.a.grad.detach().cpu().numpy().copy(), metrics


def _rel(a, b):
    return float(np.abs(np.asarray(a) - b).max() / max(float(np.abs(b).max()), 1e-30))


@pytest.fixture(autouse=True)
def _golden_path():
    import os
    import sys
    here = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    if here not in sys.path:
        sys.path.insert(0, here)
    rh.import_reference(REF)


@pytest.mark.parametrize("core_name,im,jm", [("implicit_p0_fixed", 20, 18), ("explicit", 12, 10)])
def test_full_bptt_on_a_b200_core_matches_the_reference_core(core_name, im, jm):
    """Three intervals of two steps, differentiable physics between the
    corrections: the loss and d loss / d model within rounding of the
    reference core's own autograd."""
    from neuralpom.v1.engine import full_bptt
    from neuralpom_b200 import reference_binding as rb
    ref_rt, b_rt = _runtimes(core_name, im, jm, 2)
    model = RawModel(im, jm).cuda()
    loop = lambda rt, m: full_bptt(rt, m, 0, 1000.0, 3)  # noqa: E731
    lr, gr, mr = _grads(loop, ref_rt, model)
    before = rb.steps_on_device()
    lb, gb, mb = _grads(loop, b_rt, model)
    assert rb.steps_on_device() - before >= 4          # the B200 library ran the physics
    assert type(b_rt.core).__name__.startswith("B200Bound")
    assert abs(lb - lr) <= 1e-5 * abs(lr), (lb, lr)
    # per component of d loss / d a, relative to max|g|.  Explicit core: all
    # 60 channels within 1e-4.  Semi-implicit core: the median channel
    # within 1e-5 and at most 6 channels beyond 1e-4 (measured: 5, all at
    # the bottom levels of the salinity and temperature increments, up to
    # 6.4e-3), where the two float32 forwards take different branches of the
    # near-bottom clamps -- the cells the step adjoint's own golden check
    # allows for the same reason
    err = np.abs(gb - gr) / max(float(np.abs(gr).max()), 1e-30)
    if core_name == "explicit":
        assert float(err.max()) < 1e-4, err
    else:
        assert float(np.median(err)) < 1e-5, err
        assert int(np.count_nonzero(err >= 1e-4)) <= 6, err
        assert float(err.max()) < 1e-2, err
    assert float(mb["correction/count"]) == float(mr["correction/count"]) == 3


@pytest.mark.parametrize("core_name,im,jm", [("implicit_p0_fixed", 20, 18)])
def test_post_window_hourly_on_a_b200_core_matches_the_reference_core(core_name, im, jm):
    """Hourly post-training window over one simulated day (24 corrections,
    the physics without a graph, only the final correction trained): the
    loss and the final correction's gradient against the reference core."""
    from neuralpom.v1.engine import post_window
    ref_rt, b_rt = _runtimes(core_name, im, jm, int(round(3600 / 600)))
    assert ref_rt.interval_seconds == 3600
    model = RawModel(im, jm).cuda()

    def loop(rt, m):
        rt.reset(1000.0)
        return post_window(rt, m, 0, 1000.0, window=0, rollout_days=1)
    lr, gr, _ = _grads(loop, ref_rt, model)
    lb, gb, _ = _grads(loop, b_rt, model)
    assert b_rt.advanced == ref_rt.advanced == 23 * 6
    # a day of float32 stepping in two implementations: agreement to the
    # rounding growth of 138 steps of the gyre
    assert abs(lb - lr) <= 1e-4 * abs(lr), (lb, lr)
    assert _rel(gb, gr) < 1e-3, _rel(gb, gr)
