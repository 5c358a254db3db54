"""Restart capture/restore, the reference-ensemble NPZ reader and state
injection (neuralpom_b200.formats; reference v1/checkpoint.py:51-95,
v1/data.py:14-126, hybrid/state.py:228-306) on CPU."""
import json

import numpy as np
import pytest
import torch

from neuralpom_b200 import ExplicitCore, ImplicitCore, formats


def _core(cls=ImplicitCore):
    core = cls(12, 10, device="cpu")
    g = torch.Generator().manual_seed(3)
    for n in ("t", "s", "u", "el", "q2"):
        setattr(core, n, torch.randn(getattr(core, n).shape, generator=g))
    core.time, core.time0, core.iint = 12.5, 12.5, 7
    return core


def test_capture_restore_round_trip(tmp_path):
    core = _core()
    state = formats.capture(core)
    assert state["complete"] and "t" in state["tensors"] and state["scalars"]["iint"] == 7
    assert "_ws" not in state["tensors"] and "_ws" not in state["scalars"]
    before = {k: v.clone() for k, v in state["tensors"].items()}
    core.t.add_(1.0)
    core.extra_attribute = 5
    core.time = 99.0
    formats.restore(core, state)
    assert not hasattr(core, "extra_attribute")
    assert core.time == 12.5 and core._ws is None
    for k, v in before.items():
        assert torch.equal(getattr(core, k), v), k
    formats.save_restart(tmp_path / "r" / "restart.pt", core)
    core.t.zero_()
    formats.load_restart(tmp_path / "r" / "restart.pt", core)
    assert torch.equal(core.t, before["t"])
    assert not list((tmp_path / "r").glob("*.tmp"))


def test_capture_rejects_unknown_state():
    core = _core(ExplicitCore)
    core.policy = object()
    with pytest.raises(TypeError):
        formats.capture(core)
    with pytest.raises(ValueError):
        formats.restore(core, {"tensors": {}, "scalars": {}})


def _write_dataset(root, grid=(12, 10), core="implicit_p0_fixed", day=5, shift=0.0):
    from neuralpom_b200.core import NUMERICS_VERSION
    root.mkdir(parents=True, exist_ok=True)
    (root / "manifest.json").write_text(json.dumps({
        "generation_core_requested": core, "generation_core_numerics_version": NUMERICS_VERSION[core],
        "implicit_spatial_shapiro_requested": "off", "downsampling": {"coarse_grid": list(grid), "algorithm": "box"}}))
    base = root / "member_0_gpu0"
    (base / "checkpoints_lowres_consistent").mkdir(parents=True, exist_ok=True)
    (base / "reference_data_lowres_consistent").mkdir(parents=True, exist_ok=True)
    (base / "provenance.json").write_text(json.dumps({
        "member": 0, "core_requested": core, "core_numerics_version": NUMERICS_VERSION[core],
        "downsampling_algorithm": "box",
        "resolved_numerics": {"spatial_shapiro_enabled": False, "barotropic_shapiro_gamma": 0.0,
                              "tracer_shapiro_gamma": 0.0, "velocity_shapiro_gamma": 0.0}}))
    g = np.random.default_rng(1)
    im, jm = grid
    st = {f: g.standard_normal((im, jm, 16)).astype(np.float32) for f in formats.INITIAL_3D_FIELDS}
    st.update({f: g.standard_normal((im, jm)).astype(np.float32) for f in formats.INITIAL_2D_FIELDS})
    st["time"] = np.float64(day + shift)
    st["iint"] = np.int64(0)
    np.savez(base / "checkpoints_lowres_consistent" / f"checkpoint_Day{day - 1:04d}.npz", **st)
    lab = {f: st[f] for f in formats.LABEL_FIELDS}
    lab["time"] = np.float64(day + 2400 / 86400.0)
    np.savez(base / "reference_data_lowres_consistent" / f"ref_Day{day:04d}_seg01.npz", **lab)
    return st


def test_dataset_reads_initial_state_and_label(tmp_path):
    st = _write_dataset(tmp_path / "ds")
    ds = formats.FixedCoreDataset(tmp_path / "ds", frequency_seconds=3600)
    assert ds.grid == (12, 10, 16)
    ics = ds.load_initial(0, 5)
    assert torch.equal(ics["t"], torch.from_numpy(st["t"])) and ics["time"].dtype == torch.float64
    lab = ds.load_target(0, 5, 2400)
    assert set(lab) == set(formats.LABEL_FIELDS) | {"time"}
    with pytest.raises(ValueError):
        ds.label_path(0, 5, 1000)          # not on the 20 min grid
    with pytest.raises(ValueError):
        ds.label_path(0, 5, 5 * 3600)      # beyond the first 4 h
    with pytest.raises(ValueError):
        ds.initial_path(8, 5)              # members 0..7


def test_dataset_rejects_mismatches(tmp_path):
    _write_dataset(tmp_path / "clock", shift=1e-5)
    with pytest.raises(ValueError, match="clock"):
        formats.FixedCoreDataset(tmp_path / "clock").load_initial(0, 5)
    _write_dataset(tmp_path / "core")
    with pytest.raises(ValueError, match="registered dynamical core"):
        formats.FixedCoreDataset(tmp_path / "core", core_name="explicit")
    _write_dataset(tmp_path / "grid")
    m = json.loads((tmp_path / "grid" / "manifest.json").read_text())
    m["downsampling"]["coarse_grid"] = [14, 10]
    (tmp_path / "grid" / "manifest.json").write_text(json.dumps(m))
    with pytest.raises(ValueError, match="shape"):
        formats.FixedCoreDataset(tmp_path / "grid").load_initial(0, 5)


def test_inject_core_state(tmp_path):
    st = _write_dataset(tmp_path / "ds")
    ics = formats.FixedCoreDataset(tmp_path / "ds").load_initial(0, 5)
    del ics["drx2d"]                      # optional fields fall back to zero
    ics["ub"] = ics.pop("u")              # and a missing previous level ...
    core = ImplicitCore(12, 10, device="cpu")
    formats.inject_core_state(core, ics)
    assert torch.equal(core.t, torch.from_numpy(st["t"]))
    assert torch.equal(core.ub, torch.from_numpy(st["u"]))
    assert torch.count_nonzero(core.drx2d) == 0
    assert core.time == 5.0 and core.time0 == 5.0 and core.iint == 0
    batch = {k: torch.stack([v, v]) if k != "time" else torch.tensor([3.0, 4.0], dtype=torch.float64)
             for k, v in ics.items()}
    formats.inject_core_state(core, batch, sample_index=1)
    assert core.time == 4.0
