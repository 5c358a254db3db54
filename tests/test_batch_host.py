"""Host-side checks of the ensemble call (no GPU): member validation before
any library call."""
import types

import pytest


def _fake(kind="explicit", dev="cuda"):
    import torch
    return types.SimpleNamespace(core_name=kind, device=torch.device(dev, 0) if dev == "cuda" else torch.device(dev))


def test_batch_rejects_empty_mixed_and_oversized():
    from neuralpom_b200 import batch
    with pytest.raises(ValueError, match="empty"):
        batch._member_args([])
    with pytest.raises(ValueError, match="one core kind"):
        batch._member_args([_fake("explicit"), _fake("implicit_p0_fixed")])
    with pytest.raises(ValueError, match="at most 64"):
        batch._member_args([_fake()] * 65)
    with pytest.raises(ValueError, match="one CUDA device"):
        batch._member_args([_fake(dev="cpu")])


def test_run_batch_requires_one_clock():
    from neuralpom_b200 import batch
    a = types.SimpleNamespace(iend=3, time0=0.0)
    b = types.SimpleNamespace(iend=4, time0=0.0)
    with pytest.raises(ValueError, match="one clock"):
        batch.run_batch([a, b])


def test_host_scalar_reads_a_tensor_once_per_version():
    """The ramp period is a tensor in the reference's state; its host value
    is read once and re-read after an in-place write."""
    import torch
    from neuralpom_b200 import state
    t = torch.full((), 3.0)
    assert state.host_scalar(t) == 3.0
    assert state.host_scalar(t) == 3.0
    t.fill_(5.0)
    assert state.host_scalar(t) == 5.0
    assert state.host_scalar(2.5) == 2.5
