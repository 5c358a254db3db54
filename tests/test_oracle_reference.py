"""The oracle against the reference core run live, on seeds and grid sizes
that the committed golden vectors do not cover.  Runs only where the
reference sources can be imported (the fixtures in tests/golden pin the
oracle everywhere else)."""
import os
import sys

import numpy as np
import pytest

from golden_io import oracle_params, rel_err
from oracle import pom_oracle as O
from oracle import ref_harness as rh

REF = rh.default_reference_path()
pytestmark = pytest.mark.skipif(REF is None, reason="reference sources not importable here")

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))

FIELDS = ("u", "v", "w", "t", "s", "rho", "q2", "q2l", "km", "kh", "kq", "l", "aam", "el", "elf", "et", "etf",
          "ua", "va", "uaf", "vaf", "egf", "utf", "vtf", "wubot", "wvbot", "drhox", "advx")


@pytest.mark.parametrize("name,im,jm,seed", [("explicit", 14, 12, 5), ("implicit_p0_fixed", 16, 14, 6),
                                              ("implicit_p0_fixed", 11, 17, 7)])
def test_oracle_matches_live_reference_step(name, im, jm, seed):
    rh.import_reference(REF)
    import make_golden as mg
    core = mg.perturbed_core(name, im, jm, seed)
    arrays, scalars = rh.extract_state(core)
    S = {k: np.array(v, copy=True) for k, v in arrays.items()}
    P = oracle_params(scalars, arrays, name)
    if hasattr(core, "_eta_solver_iteration_history"):
        core._eta_solver_iteration_history = []
    rh.advance(core, name, 1)
    hist = O.run(S, P, 1, name)
    after, _ = rh.extract_state(core)
    for f in FIELDS:
        assert rel_err(S[f], after[f]) < 1e-5, (f, rel_err(S[f], after[f]))
    if name != "explicit":
        assert hist == list(core._eta_solver_iteration_history)
    assert abs(P.time - float(core.time)) < 1e-9
