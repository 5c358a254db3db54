"""The launch-shape autotuner on the GPU: every launch shape it tries
computes what the library's rules compute, bit for bit; the winner is no
slower than the rules, and the cache round-trips."""
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case,im,jm,core", [("noise_basin", 64, 64, "explicit"),
                                             ("seamount", 90, 82, "implicit_p0_fixed"),
                                             ("coastal_tide", 150, 120, "explicit")])
def test_autotuner_candidates_reproduce_the_rules(case, im, jm, core, tmp_path):
    from neuralpom_b200 import autotune, cases, resolve_core_class
    A, Sc = getattr(cases, case)(im, jm)
    Sc = dict(Sc, time=0.25, time0=0.25)   # the internal mode runs from the first step
    c = resolve_core_class(core).from_state(A, Sc, device="cuda")
    tuning, report = autotune.tune(c, steps=2, reps=2)
    assert report["reproduces_rules"], report
    assert report["tuned_ms_per_step"] <= report["rule_ms_per_step"]
    for cand, ms in report["tried"]:
        assert ms != float("inf"), cand
        assert autotune.same_result(c, cand, steps=2), cand
    path = str(tmp_path / "tuning.json")
    autotune.store(autotune.key_of(c), tuning, report, path)
    c.tuning = None
    assert autotune.apply(c, path) == tuning
