"""Long oracle runs for the full-length parity tests (test helper).

The oracle is CPU numpy; a simulated day of the 90x82x16 seamount takes
about 25 s in float32 and 50 s in float64, so the runs a test needs are
made in parallel worker processes (``spawn`` start method: the parent holds
a CUDA context, and a forked child of it would hang).
"""
from __future__ import annotations

import multiprocessing as mp

import numpy as np

# the fields compared after a long run
FIELDS = ("u", "v", "t", "s", "el", "elf", "ua", "va", "q2", "q2l", "km", "kh", "w", "rho")


def case_state(case, im, jm):
    """(arrays, scalars) of a named case of ``neuralpom_b200.cases`` with
    the grid size in the scalars."""
    from neuralpom_b200 import cases
    A, Sc = getattr(cases, case)(im, jm)
    Sc = dict(Sc)
    kb = A["u"].shape[2]
    Sc.update(im=im, jm=jm, kb=kb)
    return A, Sc


def budgets(S):
    """FP64 volume and layer T/S budgets with the reference's volume
    weights (hybrid/sparse_coupling.py:18-20): sum art*fsm*(h+et), and per
    level sum art*fsm*(h+et)*dz_k*T_k (and S)."""
    vol = S["art"].astype(np.float64) * S["fsm"] * (S["h"].astype(np.float64) + S["et"])
    kbm1 = S["t"].shape[2] - 1
    lay_t = np.array([(vol * float(S["dz"][k]) * S["t"][:, :, k]).sum() for k in range(kbm1)])
    lay_s = np.array([(vol * float(S["dz"][k]) * S["s"][:, :, k]).sum() for k in range(kbm1)])
    return float(vol.sum()), lay_t, lay_s


def oracle_run(case, im, jm, core, steps, variant):
    """Run the oracle ``steps`` internal steps from the case's initial
    state.  variant: 'fp32' (the reference's arithmetic), 'fp32_ulp' (T
    moved up by one ulp: the run's own sensitivity), 'fp64' (float64 state
    and constants: the FP64 run of the same core).  Returns (fields, PCG
    iterations per step, budgets)."""
    from golden_io import oracle_params
    from oracle import pom_oracle as O
    A, Sc = case_state(case, im, jm)
    if variant == "fp32_ulp":
        A = dict(A)
        A["t"] = np.nextafter(A["t"], np.float32(np.inf)).astype(np.float32)
    if variant == "fp64":
        S = {k: (v.astype(np.float64) if v.dtype == np.float32 else v.copy()) for k, v in A.items()}
    else:
        S = {k: v.copy() for k, v in A.items()}
    P = oracle_params(Sc, A, core)
    its = O.run(S, P, steps, core)
    out = {f: S[f] for f in FIELDS}
    for f in ("art", "fsm", "h", "et", "dz"):
        out[f] = S[f]
    return out, [int(v) for v in its], budgets(S)


def oracle_runs(jobs):
    """Run several ``oracle_run`` argument tuples in parallel (spawned
    workers); returns their results in order.  The caller's main module must
    be import-safe (pytest's is): spawned workers import it."""
    ctx = mp.get_context("spawn")
    with ctx.Pool(processes=len(jobs)) as pool:
        return pool.starmap(oracle_run, jobs)


def fd_loss(path, scalars, core, steps, index, sign, eps):
    """Float64 oracle loss after ``steps`` steps from the start state stored
    in the ``.npz`` at ``path`` (``start__*`` arrays, ``target__*`` and
    ``scale__*`` of the loss fields, ``dir{index}__*`` directions), with the
    start moved by ``sign * eps`` along direction ``index``: sum over the
    loss fields of mean((S - target)^2) / scale^2."""
    from golden_io import oracle_params
    from oracle import pom_oracle as O
    z = np.load(path)
    start = {k[7:]: z[k] for k in z.files if k.startswith("start__")}
    S = {n: v.astype(np.float64) for n, v in start.items()}
    fields = [k[8:] for k in z.files if k.startswith("target__")]
    for f in fields:
        S[f] = S[f] + sign * eps * z[f"dir{index}__{f}"]
    P = oracle_params(dict(scalars), start, core)
    O.run(S, P, steps, core)
    return sum(float(((S[f] - z[f"target__{f}"]) ** 2).mean()) / float(z[f"scale__{f}"]) ** 2 for f in fields)


def fd_losses(path, scalars, core, steps, ndirs, eps, workers=8):
    """(plus, minus) float64 losses of ``fd_loss`` for every direction, in
    parallel spawned workers."""
    jobs = [(path, scalars, core, steps, i, s, eps) for i in range(ndirs) for s in (1.0, -1.0)]
    ctx = mp.get_context("spawn")
    with ctx.Pool(processes=min(workers, len(jobs))) as pool:
        out = pool.starmap(fd_loss, jobs)
    return [(out[2 * i], out[2 * i + 1]) for i in range(ndirs)]
