"""Load golden fixtures into oracle/B200 state dictionaries (test helper)."""
from __future__ import annotations

import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden_path(name):
    return os.path.join(GOLDEN, name)


def load_step_golden(name):
    """Returns (arrays, scalars, outputs) where outputs[n][field] holds the
    reference state after n steps."""
    z = np.load(golden_path(name))
    arrays, scalars, outputs = {}, {}, {}
    for key in z.files:
        if key.startswith("in__"):
            arrays[key[4:]] = z[key]
        elif key.startswith("scalar__"):
            v = z[key]
            scalars[key[8:]] = v.item() if v.dtype.kind in "biuf" else str(v)
        elif key.startswith("out"):
            n, field = key[3:].split("__", 1)
            outputs.setdefault(int(n), {})[field] = z[key]
    return arrays, scalars, outputs


def oracle_params(scalars, arrays, core):
    """Params for the oracle from the reference scalars."""
    from oracle.pom_oracle import Params
    P = Params(**scalars)
    P.period = np.float32(arrays["period"]) if "period" in arrays else np.float32(scalars.get("period", 1.0))
    P.core = core
    if core != "explicit":
        P.eta_solver_max_iter = scalars.get("eta_solver_max_iter", 200)
        P.eta_solver_tol = scalars.get("eta_solver_tol", 1.0e-12)
        P.eta_solver_rel_tol = scalars.get("eta_solver_rel_tol", 1e-5)
        P.eta_solver_preconditioner = scalars.get("eta_solver_preconditioner", "spectral")
        for k in ("barotropic_shapiro", "tracer_shapiro", "velocity_shapiro"):
            setattr(P, k, scalars.get(k, 0.0))
    return P


def rel_err(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = max(float(np.max(np.abs(b))), 1e-30)
    return float(np.max(np.abs(a - b))) / den
