"""Host-side helpers of bench.py, without a GPU."""
import sys

import pytest


@pytest.fixture()
def bench(monkeypatch):
    monkeypatch.setattr(sys, "argv", ["bench.py"])
    import bench as b
    return b


def test_reference_modes_reports_the_faster_mode_and_every_figure(bench):
    calls = []

    def sample(physics_kw=None, **kw):
        calls.append((physics_kw, kw))
        if physics_kw:
            return {"value": 2.0, "unit": "u"}
        return {"value": 1.0, "unit": "u"}

    out = bench.reference_modes(sample, "implicit_p0_fixed", "cuda:0", device="cuda:0", core_name="implicit_p0_fixed")
    assert out["mode"] == "strict_vertical_compiled+triton_cg" and out["value"] == 2.0
    assert out["modes"] == {"eager": 1.0, "strict_vertical_compiled+triton_cg": 2.0}
    assert all(kw["device"] == "cuda:0" for _, kw in calls)
    # explicit core, or a CPU run: the default options only
    out = bench.reference_modes(sample, "explicit", "cuda:0", device="cuda:0")
    assert out["mode"] == "eager" and list(out["modes"]) == ["eager"]


def test_reference_modes_reports_a_failing_mode(bench):
    def sample(physics_kw=None, **kw):
        if physics_kw:
            raise RuntimeError("no triton here")
        return {"value": 1.0}

    out = bench.reference_modes(sample, "implicit_p0_fixed", "cuda:0")
    assert out["mode"] == "eager"
    assert "no triton here" in out["modes"]["strict_vertical_compiled+triton_cg"]["error"]
