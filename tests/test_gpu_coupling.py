"""Corrector coupling on the B200 core against the reference's autograd
(golden vectors of hybrid/sparse_coupling.py:10-82): the reference's own
coupling functions, run on a B200 core, whose dens()/baropg() methods are the
CUDA DENS/BAROPG operators with hand-written adjoints
(neuralpom_b200.coupling): apply_joint_correction with the paired limiter
engaged, and pressure_velocity_error."""
import numpy as np
import pytest
import torch

from golden_io import golden_path
from oracle import ref_harness as rh

REF = rh.default_reference_path()
pytestmark = pytest.mark.gpu


def _sparse_coupling():
    if REF is None:
        pytest.skip("reference package not importable")
    rh.import_reference(REF)
    from neuralpom.hybrid import sparse_coupling
    return sparse_coupling


LEAVES = ("u", "ub", "v", "vb", "t", "tb", "s", "sb", "rho", "et", "etf", "dt")


def _load():
    z = np.load(golden_path("coupling_12x10.npz"))
    A = {k[4:]: z[k] for k in z.files if k.startswith("in__")}
    Sc = {k[8:]: z[k].item() for k in z.files if k.startswith("scalar__")}
    return z, A, Sc


def _core(A, Sc):
    from neuralpom_b200 import resolve_core_class
    core = resolve_core_class("explicit").from_state(A, Sc, device="cuda")
    leaves = {}
    for f in LEAVES:
        leaves[f] = getattr(core, f).detach().clone().requires_grad_(True)
        setattr(core, f, leaves[f])
    return core, leaves


def _rel(a, b):
    return float(np.abs(np.asarray(a, np.float64) - b).max() / max(float(np.abs(b).max()), 1e-30))


def test_gpu_apply_joint_correction_matches_reference():
    coupling = _sparse_coupling()
    z, A, Sc = _load()
    core, leaves = _core(A, Sc)
    raw = torch.tensor(z["jc__raw"], device="cuda", requires_grad=True)
    scales = dict(zip(coupling.OUTPUT_FIELDS, (float(v) for v in z["jc__scales"])))
    info = coupling.apply_joint_correction(core, raw, scales)
    # forward: elementwise sums and per-level reductions in another order
    for f in ("u", "ub", "v", "vb", "t", "tb", "s", "sb", "rho"):
        assert _rel(getattr(core, f).detach().cpu().numpy(), z[f"jc_out__{f}"]) < 1e-6, f
    ref = float(z["jc_info__ts_limit_factor"])
    assert abs(float(info["ts_limit_factor"].detach()) - ref) <= 1e-6 * ref
    # the budgets are zero by construction: rounding residue, bounded
    # against the increment scale
    for k, f in (("t_budget", "t"), ("s_budget", "s")):
        assert abs(float(info[k].detach())) <= 1e-6 * scales[f], (k, float(info[k].detach()))
    loss = sum((getattr(core, f) * torch.tensor(z[f"jc_cot__{f}"], device="cuda")).sum()
               for f in ("u", "ub", "v", "vb", "t", "tb", "s", "sb", "rho"))
    loss = loss + 3.0 * info["ts_limit_factor"] + 5.0 * info["t_budget"]
    loss.backward()
    assert _rel(raw.grad.cpu().numpy(), z["jc_grad__raw"]) < 1e-4
    for f in LEAVES:
        key = f"jc_grad__{f}"
        if key in z.files:
            assert _rel(leaves[f].grad.cpu().numpy(), z[key]) < 1e-4, f


def test_gpu_pressure_velocity_error_matches_reference():
    coupling = _sparse_coupling()
    z, A, Sc = _load()
    core, leaves = _core(A, Sc)
    ref_t = torch.tensor(z["pv__ref_t"], device="cuda", requires_grad=True)
    ref_s = torch.tensor(z["pv__ref_s"], device="cuda", requires_grad=True)
    ku, kv = coupling.pressure_velocity_error(core, ref_t, ref_s)
    assert _rel(ku.detach().cpu().numpy(), z["pv_out__u"]) < 1e-5
    assert _rel(kv.detach().cpu().numpy(), z["pv_out__v"]) < 1e-5
    loss = (ku * torch.tensor(z["pv_cot__u"], device="cuda")).sum() + \
        (kv * torch.tensor(z["pv_cot__v"], device="cuda")).sum()
    loss.backward()
    assert _rel(ref_t.grad.cpu().numpy(), z["pv_grad__ref_t"]) < 1e-4
    assert _rel(ref_s.grad.cpu().numpy(), z["pv_grad__ref_s"]) < 1e-4
    for f in LEAVES:
        key = f"pv_grad__{f}"
        if key in z.files:
            assert _rel(leaves[f].grad.cpu().numpy(), z[key]) < 1e-4, f


def test_gpu_core_dens_baropg_methods_match_the_step():
    """core.dens() and core.baropg() (the operator override points) give
    what the step's own phases give on the same state."""
    z, A, Sc = _load()
    from neuralpom_b200 import resolve_core_class
    core = resolve_core_class("explicit").from_state(A, Sc, device="cuda")
    with torch.no_grad():
        _, _, rho = core.dens()
        _, px, py = core.baropg()
    from oracle import pom_oracle as O
    from golden_io import oracle_params
    S = {k: v.copy() for k, v in A.items()}
    im, jm, kb = A["u"].shape
    P = oracle_params(dict(Sc, im=im, jm=jm, kb=kb), A, "explicit")
    assert _rel(rho.cpu().numpy(), O.dens(S, P)) < 1e-6
    # BAROPG differences nearly equal densities, which magnifies the ulp
    # differences of the two EOS evaluations (the oracle's float32 power and
    # square root come from numpy's host-CPU-dependent SIMD paths): it is
    # checked on the same rho
    S["rho"] = rho.cpu().numpy()
    _, ox, oy = O.baropg(S, P)
    assert _rel(px.cpu().numpy(), ox) < 1e-6 and _rel(py.cpu().numpy(), oy) < 1e-6
