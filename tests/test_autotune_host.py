"""The launch-shape autotuner's host logic, without a GPU: the coordinate
descent, the search space per core, the JSON cache and the tuning block of
npom_params."""
import json
from types import SimpleNamespace

import pytest

from neuralpom_b200 import _abi, autotune, state


def test_search_finds_the_separable_minimum_and_respects_min_gain():
    space = {"a": (0, 1, 2), "b": (0, 8, 32), "c": (0, 3)}
    cost = {"a": {0: 5.0, 1: 3.0, 2: 4.0}, "b": {0: 2.0, 8: 1.0, 32: 2.5}, "c": {0: 1.0, 3: 0.995}}
    calls = []

    def measure(t):
        calls.append(dict(t))
        return sum(cost[k][t.get(k, 0)] for k in cost)

    best, t_best, t_base = autotune.search(measure, space, min_gain=0.02)
    # c=3 is better by 0.005 of ~5.0 only: below min_gain, the rule stays
    assert best == {"a": 1, "b": 8}
    assert t_base == 8.0 and t_best == 5.0
    assert calls[0] == {} and len(calls) == 1 + 2 + 2 + 1


def test_space_per_core():
    imp = SimpleNamespace(kb=16, core_name="implicit_p0_fixed", nadv=1)
    exp = SimpleNamespace(kb=16, core_name="explicit", nadv=1)
    k12 = SimpleNamespace(kb=12, core_name="explicit", nadv=1)
    assert "pcg_form" in autotune.space_for(imp) and "subcycle_form" not in autotune.space_for(imp)
    assert "subcycle_form" in autotune.space_for(exp) and "pcg_form" not in autotune.space_for(exp)
    assert set(autotune.space_for(k12)) == {"subcycle_form"}
    assert "batch_pcg_blocks" in autotune.space_for(imp, batch=True)
    assert all(k in _abi.TUNING_FIELDS for k in autotune.BATCH_SPACE)


def test_cache_round_trip_and_bad_entries(tmp_path, monkeypatch):
    path = str(tmp_path / "sub" / "tuning.json")
    monkeypatch.setattr(autotune, "device_name", lambda dev: "NVIDIA B200")
    core = SimpleNamespace(core_name="explicit", im=64, jm=64, kb=16, nadv=1, mode=3, device="cuda:0", tuning=None)
    key = autotune.key_of(core)
    assert key == "NVIDIA B200|explicit|64x64x16|nadv1|mode3|-"
    assert autotune.apply(core, path) is None and core.tuning is None
    autotune.store(key, {"a1_form": 2, "subcycle_form": 3}, {"rule_ms_per_step": 1.0, "tuned_ms_per_step": 0.8}, path)
    assert autotune.apply(core, path) == {"a1_form": 2, "subcycle_form": 3}
    assert core.tuning == {"a1_form": 2, "subcycle_form": 3}
    data = json.load(open(path))
    data["x"] = {"tuning": {"not_a_knob": 1}}
    json.dump(data, open(path, "w"))
    assert autotune.lookup("x", path) is None
    open(path, "w").write("{broken")
    assert autotune.load(path) == {}


def test_tuning_reaches_npom_params():
    s = dict(state.default_scalars("explicit"), tuning={"a1_form": 1, "batch_pcg_blocks": 56})
    p = state.make_params(s, 64, 64, 16, "explicit")
    assert p.tuning.a1_form == 1 and p.tuning.batch_pcg_blocks == 56 and p.tuning.pcg_form == 0
    with pytest.raises(ValueError):
        state.make_params(dict(s, tuning={"warp_size": 16}), 64, 64, 16, "explicit")


def test_profq_form_reaches_npom_params():
    s = dict(state.default_scalars("explicit"), profq_form="pom08", zsh=0.02)
    p = state.make_params(s, 12, 10, 16, "explicit")
    assert p.profq_form == _abi.PROFQ_POM08 and abs(p.zsh - 0.02) < 1e-15
    p = state.make_params(dict(state.default_scalars("explicit")), 12, 10, 16, "explicit")
    assert p.profq_form == _abi.PROFQ_PRODUCTION and abs(p.zsh - 0.01) < 1e-15
    with pytest.raises(ValueError):
        state.make_params(dict(s, profq_form="pom2k"), 12, 10, 16, "explicit")


def test_boundary_policy_reaches_npom_params():
    """obc_form: native by default; the seamount, coastal and Jiaozhou Bay
    policies on either core (the semi-implicit one with its Shapiro filter
    off)."""
    s = dict(state.default_scalars("explicit"), obc_form="seamount")
    assert state.make_params(s, 24, 18, 16, "explicit").obc_form == _abi.OBC_SEAMOUNT
    assert state.make_params(dict(state.default_scalars("explicit")), 24, 18, 16, "explicit").obc_form == \
        _abi.OBC_NATIVE
    with pytest.raises(ValueError):
        state.make_params(dict(s, obc_form="orlanski"), 24, 18, 16, "explicit")
    for form, code in (("seamount", _abi.OBC_SEAMOUNT), ("coastal", _abi.OBC_COASTAL), ("jzb", _abi.OBC_JZB)):
        for core in ("explicit", "implicit_p0_fixed"):
            assert state.make_params(dict(state.default_scalars(core), obc_form=form), 24, 18, 16,
                                     core).obc_form == code
        with pytest.raises(ValueError):
            state.make_params(dict(state.default_scalars("implicit_p0_fixed"), obc_form=form,
                                   barotropic_shapiro=0.05), 24, 18, 16, "implicit_p0_fixed")
