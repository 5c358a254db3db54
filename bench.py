#!/usr/bin/env python
"""Throughput of the NeuralPOM physical time step on B200.

Workload: the semi-implicit free-surface core on the 90x82x16 closed basin
with a Gaussian seamount (dx = 5 km, dtI = 300 s, PCG tolerance 1e-10, FP64
dot products), synthetic seeded state.  One benchmark step = one simulated
day (288 internal steps).  Metric: simulated days per second.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

With N > 1 (torchrun) every rank advances its own ensemble member (weak
scaling, no collective on the data path); value = all members' simulated
days / the slowest rank's time.  ``--impl reference`` times the reference's
own PyTorch core on the host CPU (all cores) on the same configuration.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "simulated days/s (fwd, fwd+adjoint) at 90x82x16 vs ref torch core; % HBM peak"
UNIT = "simulated days/s"
GRID = (90, 82, 16)
DTI = 300.0

# Workloads: the headline (the semi-implicit seamount basin, one bench step =
# one simulated day) and a roofline-only one whose state (~290 MB) exceeds
# L2: the explicit core on the 354x322x16 coastal basin with its open
# southern boundary, one bench step = 6 simulated hours.
WORKLOADS = {
    "seamount": {"grid": GRID, "core": "implicit_p0_fixed", "internal": 288,
                 "desc": "semi-implicit core, closed 90x82x16 seamount basin (dx=5 km), forward"},
    "gyre": {"grid": (64, 64, 16), "core": "explicit", "internal": 480,
             "desc": "explicit core, 64x64x16 double-gyre basin (dx=20 km, dtE=6 s, isplit=30, seeded "
                     "bathymetry noise), forward; one bench step = one simulated day (480 internal steps)"},
    "batch": {"grid": None, "core": None, "internal": None,
              "desc": "64 members on mixed grids in one GPU (24 x 90x82x16, 24 x 128x112x16, 16 x 177x161x16; even "
                      "members the explicit noise basin at dtI=180 s, odd members the semi-implicit seamount at "
                      "dtI=300 s, seed = member), one simulated day of every member per bench step; the members "
                      "of each core advance as one batch, one launch per phase over all of them, the step "
                      "replayed as a CUDA graph"},
    "channel": {"grid": GRID, "core": "implicit_p0_fixed", "internal": 288,
                "desc": "semi-implicit core, 90x82x16 seamount channel periodic in x (two halo columns on each "
                        "side, unique columns 2..87, walls in y; PCG preconditioned by Hartley along x times "
                        "DST-I along y, cooperative-grid form), forward"},
    "coastal": {"grid": (354, 322, 16), "core": "explicit", "internal": 60, "horizon": 360,
                "desc": "explicit core, 354x322x16 coastal basin (dx=500 m, open south boundary with Flather "
                        "condition and M2 elevation 1 m updated every bench step), forward; one bench step = 1 "
                        "simulated hour, restarted from the initial state every 6 h"},
}

# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per launch of the
# phase's kernel at 90x82x16, read from one ncu capture of that kernel (not
# measured by this script); reported with the capture it comes from.
NCU_DRAM_BYTES = {"E_external": (570368, "ncu --set full capture of one k_pcg_cluster launch, bulk-copy form "
                                         "(90x82x16 seamount, in-step input)")}

# Distinct arrays each phase reads / writes (3-D count, 2-D count): the
# algorithmic-byte rule bytes = 4 * (sum of read numel + sum of written numel).
PHASE_IO = {
    "A1_forcing_advct": (5, 12, 3, 8),
    "A2_baropg_smag_means": (6, 5, 3, 5),
    "A3_advave_predictor": (2, 27, 1, 15),
    "E_external": (0, 18, 0, 4),
    "E_external_explicit": (0, 33, 0, 19),
    "I5_corrector_filter": (0, 22, 0, 13),
    "B1_barotropic_fix": (2, 6, 2, 0),
    "B2A_vertvl": (3, 8, 1, 0),
    "B2B_advq": (9, 11, 2, 0),
    "B3_profq": (15, 8, 6, 0),
    "B4_edges_bcond6": (2, 1, 2, 0),
    "B5_qfilter_advt1": (17, 10, 10, 0),
    "B6_proft": (3, 6, 2, 1),
    "B7_tsfilter_dens": (6, 2, 5, 0),
    "B8_advuv_profuv": (14, 17, 2, 3),
    "B9_velfilter_shift": (6, 12, 6, 7),
}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=("b200", "reference"))
    ap.add_argument("--internal-steps", type=int, default=None,
                    help="internal steps per benchmark step (default: one simulated day / 6 h, per workload)")
    ap.add_argument("--workload", default="seamount", choices=sorted(WORKLOADS))
    ap.add_argument("--ref-internal-steps", type=int, default=6, help="reference arm: internal steps per sample")
    ap.add_argument("--ref-device", default="cpu")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-fp64", action="store_true", help="skip the per-field error against a float64 reference day")
    ap.add_argument("--no-batch-tune", action="store_true", help="batch workload: the library's launch rules only")
    ap.add_argument("--no-coastal", action="store_true", help="skip the 354x322x16 coastal forward+adjoint sample")
    ap.add_argument("--no-periodic", action="store_true", help="skip the periodic-x channel sample")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--members", type=int, default=8,
                    help="ensemble members advanced concurrently on one GPU for the 'ensemble' key (1 = skip)")
    ap.add_argument("--no-ref-gpu", action="store_true", help="skip timing the reference core on this GPU")
    ap.add_argument("--no-fwd-adjoint", action="store_true", help="skip the forward+adjoint sample")
    ap.add_argument("--fa-steps", type=int, default=36,
                    help="internal steps of the headline forward+adjoint sample")
    ap.add_argument("--fa-reps", type=int, default=3, help="timed forward+adjoint samples (median)")
    ap.add_argument("--fa-only", action="store_true",
                    help="headline forward+adjoint sample only (after --warmup forward days); for profiling")
    ap.add_argument("--batch-chunk", type=int, default=24,
                    help="batch workload: turns per simulated day in which the groups (or members) enqueue "
                         "their steps")
    ap.add_argument("--batch-streams", type=int, default=2, choices=(1, 2),
                    help="batch workload: the explicit and semi-implicit batches on one stream in turns (1) or "
                         "each on its own stream (2, the default)")
    ap.add_argument("--no-batch", action="store_true",
                    help="skip the 64-member batch ('batch' key of the default workload)")
    ap.add_argument("--batch-mode", default="launch", choices=("launch", "streams"),
                    help="batch workload: 'launch' = one launch per phase over all members of a core "
                         "(npom_step_batch); 'streams' = every member its own core call on its own stream")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# helpers
# ---------------------------------------------------------------------------

def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def workload(member=0, name="seamount"):
    from neuralpom_b200 import cases
    if name == "gyre":
        im, jm, kb = WORKLOADS[name]["grid"]
        return cases.noise_basin(im, jm, kb=kb)
    if name == "coastal":
        im, jm, kb = WORKLOADS[name]["grid"]
        A, Sc = cases.coastal_tide(im, jm, kb=kb)
        Sc = dict(Sc)
        Sc.update(time=0.25, time0=0.25)   # internal mode from the first step
        return A, Sc
    if name == "channel":
        A, Sc = cases.seamount_channel(*GRID[:2], kb=GRID[2], dti=DTI)
        return A, dict(Sc)
    A, Sc = cases.seamount(*GRID[:2], kb=GRID[2], dti=DTI)
    if member:
        # ensemble members: seeded temperature perturbation (0.2 degC)
        g = np.random.default_rng(100 + member)
        p = (0.2 * g.standard_normal(A["t"].shape) * A["fsm"][:, :, None]).astype(np.float32)
        A["t"] = A["t"] + p
        A["tb"] = A["tb"] + p
    return A, dict(Sc)


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-f", self.path], stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        try:
            rows = [r.split(",") for r in open(self.path).read().strip().splitlines() if r.strip()]
            os.unlink(self.path)
        except Exception:
            return None
        if not rows:
            return None
        sm = [float(r[1]) for r in rows]
        mx = [float(r[2]) for r in rows]
        reasons = set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for r in rows:
            for name, val in zip(names, r[5:9]):
                if val.strip().lower() in ("active", "1"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(rows)}


def l2_flush(buf):
    buf.add_(1.0)


def max_over_ranks(ms, pg=None, dev=None):
    """The slowest rank's device time (ms): every rank contributes its own
    CUDA-event total; an FP64 all-reduce MAX is the only collective."""
    if pg is None:
        return float(ms)
    import torch
    t = torch.tensor([float(ms)], dtype=torch.float64, device=dev)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def aggregate_days_per_s(n_members, steps, internal_steps, dti, t_max_ms):
    """Whole-job throughput: every member's simulated days over the slowest
    rank's time (weak scaling: one member per rank)."""
    return n_members * steps * internal_steps * dti / 86400.0 / (t_max_ms / 1000.0)


# ---------------------------------------------------------------------------
# the B200 arm
# ---------------------------------------------------------------------------

SUB_CLUSTER_CELLS = 16 * 1024  # largest grid of the one-cluster explicit subcycle


def launches_of(core, nsteps, time0):
    """Kernels one npom_step_* call enqueues (see npom_kernels.cu run_steps):
    the operator coefficients once (implicit), then per internal step A1 A2
    A3 + PCG + I5 (implicit) or A1 A2 A3 + subcycle (explicit), the nine
    internal-mode kernels B1-B8 unless the step is the first from rest, and
    B9.  With NPOM_SUBCYCLE=phases (or =nocoop on grids above four cells
    per thread of one cluster) the explicit subcycle is 3 x isplit launches
    instead of one."""
    implicit = core.core_name != "explicit"
    sub = 1
    form = os.environ.get("NPOM_SUBCYCLE")
    if not implicit and (form == "phases" or (form == "nocoop" and core.im * core.jm > 4 * SUB_CLUSTER_CELLS)):
        sub = 3 * int(core.params().isplit)
    n = 1 if implicit else 0
    for s in range(nsteps):
        iint = 1 + s
        n += (5 if implicit else 3 + sub) + 1
        if (iint != 1 or time0 != 0.0) and core.mode != 2:
            n += 9
    return n


def run_b200(args):
    import torch
    from neuralpom_b200 import _abi, build, resolve_core_class

    ws_n, rank, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pg = None
    if ws_n > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
        pg = dist
    build.build()
    W = WORKLOADS[args.workload]
    if args.workload == "coastal":
        # roofline-only workload: no reference samples, no host round trip
        args.no_e2e = args.no_ref_gpu = args.no_cpu_baseline = True
    if args.workload == "channel":
        # the reference has no periodic boundary: no reference samples
        args.no_ref_gpu = args.no_cpu_baseline = True
    A, Sc = workload(member=rank, name=args.workload)
    core = resolve_core_class(W["core"]).from_state(A, Sc, device=dev)
    nin = args.internal_steps or W["internal"]
    stream = torch.cuda.current_stream(dev)
    flush = torch.zeros(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MiB > L2

    def day():
        t0 = float(core.time)
        core.launch_steps(nin, t0, 1, stream)
        core.time = core.dti * nin / 86400.0 + t0
        return t0

    # coastal workload: the boundary tide between bench steps and a restart
    # from the initial state at the 6 h horizon (the set-up's window), both
    # outside the timed region
    horizon = W.get("horizon")
    snapshot = {n: getattr(core, n).clone() for n in _abi.FIELD_NAMES} if horizon else None
    start_time = float(core.time)
    done = [0]

    def prepare():
        if not horizon:
            return
        if done[0] + nin > horizon:
            for n in _abi.FIELD_NAMES:
                getattr(core, n).copy_(snapshot[n])
            core.time = core.time0 = start_time
            done[0] = 0
        from neuralpom_b200 import cases
        core.els.fill_(cases.tide_elevation(float(core.time) - start_time))
        done[0] += nin

    for _ in range(args.warmup):
        prepare()
        day()
    bits, _ = core.read_status(nin)
    if bits & (_abi.DEV_TIMEOUT | _abi.DEV_VMAX | _abi.DEV_NONFINITE):
        raise RuntimeError(f"device status 0x{bits:x} during warm-up")
    if args.fa_only:
        # profiling mode: the workload's forward+adjoint sample alone
        if args.workload == "coastal":
            fa = coastal_fwd_adjoint(args, dev, nsteps=args.fa_steps)
        else:
            fa, _, _ = seamount_fwd_adjoint(core, args, dev, nsteps=args.fa_steps, reps=args.fa_reps)
        if rank == 0:
            print(json.dumps({"fwd_adjoint": fa}), flush=True)
        return

    launches = 0
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    if pg:
        pg.barrier()
    torch.cuda.synchronize(dev)
    with ClockSampler(local) as clk:
        for k in range(args.steps):
            l2_flush(flush)
            prepare()
            ev[k][0].record(stream)
            t0 = day()
            ev[k][1].record(stream)
            launches += launches_of(core, nin, t0)
        torch.cuda.synchronize(dev)
    if pg:
        pg.barrier()
    elapsed_ms = sum(a.elapsed_time(b) for a, b in ev)
    bits, its = core.read_status(nin)
    if bits & (_abi.DEV_TIMEOUT | _abi.DEV_VMAX | _abi.DEV_NONFINITE):
        raise RuntimeError(f"device status 0x{bits:x} in the timed region")
    t_max = max_over_ranks(elapsed_ms, pg, dev)
    value = aggregate_days_per_s(ws_n, args.steps, nin, core.dti, t_max)

    # dominant kernel, timed alone on the same stream (CUDA events)
    roofline = dominant_kernel_roofline(core, stream, dev)

    e2e = None
    if not args.no_e2e:
        e2e = end_to_end(core, A, Sc, args, stream, dev, pg, ws_n, nin)

    ens = None
    if rank == 0 and ws_n == 1 and args.workload == "seamount" and args.members > 1:
        ens = ensemble_sample(args, W, nin, dev, flush)

    ref_gpu = None
    if rank == 0 and ws_n == 1 and not args.no_ref_gpu:
        ref_gpu = reference_modes(reference_gpu_sample, W["core"], dev, A=A, Sc=Sc, device=dev,
                                  core_name=W["core"])

    # (the channel has no float64 reference run: the reference has no
    # periodic boundary; its float64 comparison is the oracle's, in the tests)
    fp64 = None
    if rank == 0 and ws_n == 1 and not args.no_fp64 and args.workload in ("seamount", "gyre"):
        fp64 = fp64_day_error(A, Sc, nin, dev, W["core"])

    cpu = None
    if rank == 0 and ws_n == 1 and not args.no_cpu_baseline:
        cpu = reference_cpu_sample(A, Sc, internal_steps=args.ref_internal_steps, warm=1, reps=2,
                                   core_name=W["core"])

    fa = fam = famb = None
    if rank == 0 and ws_n == 1 and args.workload == "coastal" and not args.no_fwd_adjoint:
        fa = coastal_fwd_adjoint(args, dev)
    if rank == 0 and ws_n == 1 and args.workload == "seamount" and not args.no_fwd_adjoint:
        fa, A_dev, t_dev = seamount_fwd_adjoint(core, args, dev, nsteps=args.fa_steps, reps=args.fa_reps)
        case = (A_dev, dict(Sc, time=t_dev, time0=t_dev))
        if not args.no_ref_gpu:
            fa["reference_gpu"] = reference_modes(reference_fwd_adjoint_sample, W["core"], dev, device=dev,
                                                  case=case, core_name=W["core"], seed=11)
        if not args.no_cpu_baseline:
            fa["reference_cpu"] = reference_fwd_adjoint_sample("cpu", internal_steps=3, case=case,
                                                               core_name=W["core"], seed=11)
        fam = None if args.fa_only else fwd_adjoint_sample(args, dev)
        famb = None if args.fa_only else fwd_adjoint_midtrain_batch(args, dev)
        if fam is not None and not args.no_ref_gpu:
            fam["reference_gpu"] = reference_fwd_adjoint_sample(dev)
        if fam is not None and not args.no_cpu_baseline:
            fam["reference_cpu"] = reference_fwd_adjoint_sample("cpu", internal_steps=3)

    per = None
    if rank == 0 and ws_n == 1 and args.workload == "seamount" and not args.no_periodic:
        per = periodic_sample(args, dev, flush)

    bat = None
    if rank == 0 and ws_n == 1 and args.workload == "seamount" and not args.no_batch and not args.fa_only:
        bat = batch_summary(args)

    # the coastal configuration's differentiation at its own size (354x322x16,
    # 6 h, checkpoint per internal step): days/s and peak device memory
    coastal = None
    if rank == 0 and ws_n == 1 and args.workload == "seamount" and not args.no_fwd_adjoint and not args.no_coastal:
        torch.cuda.empty_cache()
        coastal = coastal_fwd_adjoint(args, dev)
        torch.cuda.empty_cache()

    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws_n, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_max / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 (FP64 PCG dot products)", "data": "synthetic",
        "config": {"workload": W["desc"], "grid": list(W["grid"]), "dti_s": float(core.dti),
                   "internal_steps_per_step": nin,
                   "pcg_tol": 1e-10 if W["core"] != "explicit" else None,
                   "pcg_iterations_last_step": (its[-1] if its else None) if W["core"] != "explicit" else None,
                   "members": ws_n, "parallelism": f"ensemble x{ws_n}" if ws_n > 1 else "single member",
                   "l2": "flushed (256 MiB write) before every timed step"},
        "pcg_iterations_timed": ({"per_step_min": int(min(its)), "per_step_max": int(max(its)),
                                  "per_step_mean": float(np.mean(its)), "steps": len(its)}
                                 if (its and W["core"] != "explicit") else None),
        "fp64_error": fp64,
        "roofline": roofline, "cpu_baseline": cpu, "reference_gpu": ref_gpu, "ensemble": ens, "fwd_adjoint": fa,
        "fwd_adjoint_midtrain": fam, "fwd_adjoint_midtrain_batch": famb, "fwd_adjoint_coastal": coastal,
        "batch": bat, "periodic_x": per, "e2e": e2e,
        "gpu_launches": launches,
        "clocks": clk.summary(),
    }
    if rank == 0:
        print(json.dumps(out), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()


def periodic_sample(args, dev, flush, days=2):
    """The headline basin as a channel periodic in x (the configuration's
    boundary; the reference has none, so the headline runs closed walls):
    one day of warm-up, then ``days`` simulated days timed with CUDA events
    on the launching stream, L2 flushed before each."""
    import torch
    from neuralpom_b200 import _abi, resolve_core_class
    W = WORKLOADS["channel"]
    A, Sc = workload(name="channel")
    core = resolve_core_class(W["core"]).from_state(A, Sc, device=dev)
    stream = torch.cuda.current_stream(dev)
    nin = W["internal"]

    def day():
        t0 = float(core.time)
        core.launch_steps(nin, t0, 1, stream)
        core.time = core.dti * nin / 86400.0 + t0

    day()
    bits, _ = core.read_status(nin)
    if bits & (_abi.DEV_TIMEOUT | _abi.DEV_VMAX | _abi.DEV_NONFINITE | _abi.DEV_PCG_MAXIT):
        raise RuntimeError(f"periodic channel: device status 0x{bits:x} during warm-up")
    ms = []
    for _ in range(days):
        l2_flush(flush)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        day()
        b.record(stream)
        torch.cuda.synchronize(dev)
        ms.append(a.elapsed_time(b))
    bits, its = core.read_status(nin)
    if bits & (_abi.DEV_TIMEOUT | _abi.DEV_VMAX | _abi.DEV_NONFINITE | _abi.DEV_PCG_MAXIT):
        raise RuntimeError(f"periodic channel: device status 0x{bits:x}")
    per_day = statistics.median(ms)
    return {"workload": W["desc"], "days_per_s": 1000.0 / per_day, "ms_per_day": per_day, "days_timed": days,
            "pcg_iterations_last_call": {"mean": float(np.mean(its)), "min": int(min(its)), "max": int(max(its))}
            if its else None}


def ensemble_sample(args, W, nin, dev, flush):
    """Members of an ensemble advanced together on one GPU: each seeded
    member has its own core and its own stream, and every bench step
    launches one simulated day of every member.  The step is latency bound
    and the PCG cluster holds 8 of the SMs, so the members overlap; value =
    all members' simulated days over the device time of the steps."""
    import torch
    from neuralpom_b200 import _abi, resolve_core_class
    m = args.members
    cores, streams = [], []
    for member in range(m):
        A, Sc = workload(member=member, name=args.workload)
        cores.append(resolve_core_class(W["core"]).from_state(A, Sc, device=dev))
        streams.append(torch.cuda.Stream(dev))
    main = torch.cuda.current_stream(dev)

    def day_all():
        start = torch.cuda.Event()
        start.record(main)
        ends = []
        for c, st in zip(cores, streams):
            st.wait_event(start)
            t0 = float(c.time)
            c.launch_steps(nin, t0, 1, st)
            c.time = c.dti * nin / 86400.0 + t0
            e = torch.cuda.Event()
            e.record(st)
            ends.append(e)
        for e in ends:
            main.wait_event(e)

    for _ in range(args.warmup):
        day_all()
    torch.cuda.synchronize(dev)
    steps = max(2, args.steps // 2)
    total = 0.0
    for _ in range(steps):
        l2_flush(flush)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(main)
        day_all()
        b.record(main)
        torch.cuda.synchronize(dev)
        total += a.elapsed_time(b)
    for c in cores:
        bits, _ = c.read_status(nin)
        if bits & (_abi.DEV_TIMEOUT | _abi.DEV_VMAX | _abi.DEV_NONFINITE):
            raise RuntimeError(f"device status 0x{bits:x} in the ensemble run")
    value = aggregate_days_per_s(m, steps, nin, cores[0].dti, total)
    return {"members": m, "value": value, "unit": UNIT, "ms_per_step": total / steps, "steps": steps,
            "per_member": value / m,
            "how": f"{m} seeded members (0.2 degC temperature perturbations), one core and one CUDA stream each, "
                   "one simulated day of every member per step; device time with CUDA events around each step"}


def dominant_kernel_roofline(core, stream, dev, reps=20):
    """Time each phase of one internal step (CUDA events on the launching
    stream around that phase alone) and report the slowest one against the
    HBM roofline.  Every repetition restores the state at the start of the
    step and runs the preceding phases untimed, so each phase -- the PCG in
    particular, whose iteration count depends on its input -- sees the
    input it has inside a step."""
    import torch
    from neuralpom_b200 import _abi
    lib = _abi.load_library()
    p = core.params()
    fa = core._fields()
    ws = core._workspace()
    im, jm, kb = core.im, core.jm, core.kb
    n3, n2 = im * jm * kb, im * jm
    times = {}
    snapshot = {n: getattr(core, n).clone() for n in _abi.FIELD_NAMES}
    phases = [i for i, n in enumerate(_abi.PHASES) if n != "I5_corrector_filter" or core.core_name != "explicit"]

    def run(ph):
        _abi.check(lib.npom_run_phase(ctypes.byref(p), ctypes.byref(fa), ctypes.byref(ws["struct"]), ph, 1.0,
                                      ctypes.c_void_p(stream.cuda_stream)), "phase")

    for ph in phases:
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(reps + 2)]
        for k in range(reps + 2):
            for n in _abi.FIELD_NAMES:
                getattr(core, n).copy_(snapshot[n])
            for q in phases:
                if q == ph:
                    break
                run(q)
            ev[k][0].record(stream)
            run(ph)
            ev[k][1].record(stream)
        torch.cuda.synchronize(dev)
        times[_abi.PHASES[ph]] = sum(a.elapsed_time(b) for a, b in ev[2:]) / reps
    for n in _abi.FIELD_NAMES:
        getattr(core, n).copy_(snapshot[n])
    core.read_status(0)
    def phase_bytes(ph):
        key = "E_external_explicit" if (ph == "E_external" and core.core_name == "explicit") else ph
        r3, r2, w3, w2 = PHASE_IO[key]
        nb = 4 * ((r3 + w3) * n3 + (r2 + w2) * n2)
        if ph == "E_external" and core.core_name != "explicit":
            ni, nj = im - 2, jm - 2
            nb += 4 * (ni * ni + nj * nj + ni * nj)  # DST matrices and eigenvalues
        return nb

    name = max(times, key=times.get)
    nbytes = phase_bytes(name)
    sec = times[name] / 1000.0
    achieved = nbytes / sec / 1e9
    peak, src = measured_peaks()
    # the capture is of the closed basin's cluster solve
    closed = (im, jm, kb) == GRID and not bool(getattr(core, "periodic_x", False))
    traffic, traffic_src = NCU_DRAM_BYTES.get(name, (None, None)) if closed else (None, None)
    step_bytes = sum(phase_bytes(ph) for ph in times)
    step_ms = sum(times.values())
    notes = {
        "E_external": "the PCG / external subcycle is bound by synchronisation latency (cluster or grid "
                      "barriers per iteration or substep), not by HBM: its arrays stay on chip or in L2; "
                      "frac is reported against HBM for the record only",
    }
    bound = "sync-latency" if name == "E_external" else "hbm"
    return {"kernel": name, "bound": bound, "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_source": src, "traffic": traffic, "traffic_source": traffic_src,
            "algorithmic_bytes": nbytes,
            "note": notes.get(name),
            "launch_ms": times[name], "phase_ms": {k: round(v, 5) for k, v in times.items()},
            "phase_frac": {k: round(phase_bytes(k) / (v / 1000.0) / 1e9 / peak, 4) for k, v in times.items()},
            "step": {"algorithmic_bytes": step_bytes, "ms": step_ms,
                     "achieved": step_bytes / (step_ms / 1000.0) / 1e9,
                     "frac": step_bytes / (step_ms / 1000.0) / 1e9 / peak}}


def end_to_end(core, A, Sc, args, stream, dev, pg, ws_n, nin):
    """Same metric through the public drop-in API with the state in pinned
    host memory: every step copies the full state host->device, advances one
    simulated day, and reads the prognostic state back."""
    import torch
    from neuralpom_b200 import _abi
    names = list(_abi.FIELD_NAMES)
    host = {n: torch.from_numpy(np.ascontiguousarray(A[n] if n in A else np.zeros(
        _abi.field_shape(n, core.im, core.jm, core.kb), np.float32))).pin_memory() for n in names}
    outs = ("u", "v", "t", "s", "el", "ua", "va", "q2", "q2l", "km", "kh", "w", "rho")
    host_out = {n: torch.empty_like(host[n]).pin_memory() for n in outs}
    h2d = sum(host[n].numel() * 4 for n in names)
    d2h = sum(host_out[n].numel() * 4 for n in outs)
    steps = max(1, args.steps // 2)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if pg:
        pg.barrier()
    torch.cuda.synchronize(dev)
    a.record(stream)
    for _ in range(steps):
        for n in names:
            getattr(core, n).copy_(host[n], non_blocking=True)
        core.time = core.time0 = 1000.0
        core.launch_steps(nin, 1000.0, 1, stream)
        for n in outs:
            host_out[n].copy_(getattr(core, n), non_blocking=True)
    b.record(stream)
    torch.cuda.synchronize(dev)
    ms = a.elapsed_time(b)
    if pg:
        t = torch.tensor([ms], device=dev, dtype=torch.float64)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        ms = float(t.item())
    bits, _ = core.read_status(nin)
    if bits & (_abi.DEV_TIMEOUT | _abi.DEV_VMAX | _abi.DEV_NONFINITE):
        raise RuntimeError(f"device status 0x{bits:x} in the end-to-end region")
    days = ws_n * steps * nin * core.dti / 86400.0
    return {"value": days / (ms / 1000.0), "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
            "steps": steps}


# ---------------------------------------------------------------------------
# the reference's own implementation
# ---------------------------------------------------------------------------

# Forward+adjoint: the differentiation set-up of the Midtrain stage on the
# explicit core (90x82x16 basin, dtI = 120 s, isplit = 20), three 1 h
# intervals with an additive increment on T, S, u, v between them, loss =
# MSE of u, v, T, S against a seeded target, gradient of every state field.
FA_GRID = (90, 82, 16)
FA_INTERVALS, FA_STEPS_PER_INTERVAL = 3, 30


def midtrain_case(member=0):
    """Seeded member: the explicit noise basin at 90x82x16 with the
    dtE = 6 s, isplit = 20 clock; T/S perturbations from a Gaussian random
    field (std 0.2 degC / 0.05 psu, correlation length 5 cells) and u/v
    perturbations (std 0.05 m/s) on the wet faces; clock at 1 day."""
    from scipy.ndimage import gaussian_filter
    from neuralpom_b200 import cases
    im, jm, kb = FA_GRID
    A, Sc = cases.noise_basin(im, jm, kb=kb, dte=6.0, isplit=20, seed=member)
    Sc = dict(Sc)
    Sc.update(time=1.0, time0=1.0)
    g = np.random.default_rng(100 + member)
    shape = A["t"].shape

    def grf(std):
        n = gaussian_filter(g.standard_normal(shape), (5.0, 5.0, 0.0), mode="reflect")
        return (n / n.std() * std).astype(np.float32)
    fsm3 = A["fsm"][:, :, None]
    pt, ps = grf(0.2) * fsm3, grf(0.05) * fsm3
    pt[:, :, -1] = ps[:, :, -1] = 0.0
    A["t"] = A["t"] + pt
    A["tb"] = A["tb"] + pt
    A["s"] = A["s"] + ps
    A["sb"] = A["sb"] + ps
    for f, m in (("u", "dum"), ("v", "dvm")):
        p = (0.05 * g.standard_normal(shape) * A[m][:, :, None]).astype(np.float32)
        p[:, :, -1] = 0.0
        A[f] = A[f] + p
        A[f + "b"] = A[f + "b"] + p
    return A, Sc


def _fa_targets(A, seed, dev=None):
    g = np.random.default_rng(seed)
    out = {}
    for f, sd, m in (("t", 0.1, "fsm"), ("s", 0.02, "fsm"), ("u", 0.02, "dum"), ("v", 0.02, "dvm")):
        out[f] = (A[f] + sd * g.standard_normal(A[f].shape) * A[m][:, :, None]).astype(np.float32)
    incs = {}
    for f, sd, m in (("t", 1e-3, "fsm"), ("s", 2e-4, "fsm"), ("u", 1e-4, "dum"), ("v", 1e-4, "dvm")):
        incs[f] = (sd * g.standard_normal(A[f].shape) * A[m][:, :, None]).astype(np.float32)
    return out, incs


def fwd_adjoint_timing(core, start, tgt, correct, intervals, steps_per_interval, t0, reps, warm, dev):
    """Median CUDA-event time (ms) of forward+backward through the drop-in
    API under torch autograd: every state field a leaf, ``intervals``
    differentiable run_time_loop() calls of ``steps_per_interval`` internal
    steps with ``correct(core)`` between them, MSE(u, v, T, S) loss,
    backward()."""
    import torch
    from neuralpom_b200 import _abi
    stream = torch.cuda.current_stream(dev)
    dti = float(core.dti)

    def prepare():
        for f in _abi.FIELD_NAMES:
            setattr(core, f, start[f].clone())
        return [getattr(core, f).requires_grad_(True) for f in _abi.ADJ_STATE_FIELDS]

    def fwd_bwd():
        for k in range(intervals):
            core.time0 = t0 + k * steps_per_interval * dti / 86400.0
            core.iend = steps_per_interval
            core.run_time_loop()
            if k < intervals - 1 and correct is not None:
                correct(core)
        loss = sum(((getattr(core, f) - tgt[f]) ** 2).mean() for f in tgt)
        loss.backward()

    for _ in range(max(warm, 1)):
        prepare()
        fwd_bwd()
    torch.cuda.synchronize(dev)
    ms = []
    for _ in range(reps):
        leaves = prepare()
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fwd_bwd()
        e1.record(stream)
        torch.cuda.synchronize(dev)
        ms.append(e0.elapsed_time(e1))
        assert all(t.grad is not None for t in leaves[:12])
    with torch.no_grad():
        for f in _abi.FIELD_NAMES:
            setattr(core, f, start[f].clone())
    return statistics.median(ms)


def seamount_fwd_adjoint(core, args, dev, nsteps=36, reps=3):
    """Forward+adjoint on the headline workload: the semi-implicit core on
    the 90x82x16 seamount basin from its state after the timed region,
    ``nsteps`` internal steps (3 h), MSE(u, v, T, S) against a seeded
    target, backward to every state field (the free-surface solve
    differentiates through its CUDA adjoint)."""
    import torch
    from neuralpom_b200 import _abi
    start = {f: getattr(core, f).detach().clone() for f in _abi.FIELD_NAMES}
    A = {f: v.cpu().numpy() for f, v in start.items()}
    tgt, _ = _fa_targets(A, 11)
    tgt = {f: torch.from_numpy(v).to(dev) for f, v in tgt.items()}
    t0 = float(core.time)
    best = fwd_adjoint_timing(core, start, tgt, None, 1, nsteps, t0, reps, args.warmup, dev)
    days = nsteps * float(core.dti) / 86400.0
    core.time = t0
    return {"value": days / (best / 1000.0), "unit": UNIT, "ms_per_sample": best,
            "workload": f"the headline workload (semi-implicit core, closed {GRID[0]}x{GRID[1]}x{GRID[2]} seamount "
                        f"basin, dtI=300 s, PCG tolerance 1e-10) from its state after the timed region; {nsteps} "
                        "internal steps forward under autograd, MSE(u,v,T,S) loss, backward to every state field; "
                        "checkpoint per internal step, hand-written CUDA step adjoint with the free-surface "
                        "solve's CUDA adjoint",
            "timing": f"median of {reps} samples, CUDA events around forward+backward"}, A, t0


def coastal_fwd_adjoint(args, dev, nsteps=360):
    """The coastal differentiation workload: the explicit core on the
    354x322x16 coastal basin, ``nsteps`` internal steps (6 h at dtI = 60 s)
    forward under autograd from the set-up state (tide elevation held at its
    start value inside the window), MSE(u, v, T, S) against a seeded
    target, backward to every state field with a checkpoint per internal
    step.  Reports the peak device memory of the call."""
    import torch
    from neuralpom_b200 import _abi, resolve_core_class
    A, Sc = workload(0, "coastal")
    core = resolve_core_class("explicit").from_state(A, Sc, device=dev)
    tgt, _ = _fa_targets(A, 13)
    tgt = {f: torch.from_numpy(v).to(dev) for f, v in tgt.items()}
    start = {f: getattr(core, f).detach().clone() for f in _abi.FIELD_NAMES}
    torch.cuda.synchronize(dev)
    torch.cuda.reset_peak_memory_stats(dev)
    base = torch.cuda.memory_allocated(dev)
    best = fwd_adjoint_timing(core, start, tgt, None, 1, nsteps, float(Sc["time"]), 1, 1, dev)
    peak = torch.cuda.max_memory_allocated(dev)
    days = nsteps * float(core.dti) / 86400.0
    return {"value": days / (best / 1000.0), "unit": UNIT, "ms_per_sample": best,
            "peak_hbm_gb": peak / 1e9, "state_and_inputs_gb": base / 1e9,
            "workload": f"explicit core, 354x322x16 coastal basin (open south boundary, Flather, M2 elevation); "
                        f"{nsteps} internal steps (6 h) forward under autograd, MSE(u,v,T,S) loss, backward to "
                        "every state field; checkpoint per internal step (one flat copy of the 58 state fields)",
            "timing": "one sample after one warm-up, CUDA events around forward+backward; peak_hbm_gb = "
                      "torch.cuda.max_memory_allocated over the warm-up and the sample"}


def reference_coupling():
    """The reference's own corrector coupling module
    (hybrid/sparse_coupling.py), which runs unchanged on a B200 core: its
    EOS and pressure-gradient calls go to the core's dens()/baropg(), the
    CUDA operators with hand-written adjoints."""
    import importlib
    import types
    for path in (os.environ.get("NPOM_REFERENCE_SRC", ""), os.path.join(ROOT, "baseline", "_ref")):
        if path and os.path.isdir(os.path.join(path, "neuralpom")):
            break
    else:
        raise RuntimeError("the reference package (baseline/_ref) is needed for the corrector coupling")
    if "netCDF4" not in sys.modules:
        try:
            importlib.import_module("netCDF4")
        except ModuleNotFoundError:  # imported by the reference's cores, never used
            sys.modules["netCDF4"] = types.ModuleType("netCDF4")
    if path not in sys.path:
        sys.path.insert(0, path)
    return importlib.import_module("neuralpom.hybrid.sparse_coupling")


def fwd_adjoint_sample(args, dev, reps=3):
    """The Midtrain-shaped forward+adjoint: the explicit-core member of
    ``midtrain_case``, three differentiable 1 h intervals with the
    increment between them, MSE(u, v, T, S), backward (see
    ``fwd_adjoint_timing``)."""
    import torch
    from neuralpom_b200 import _abi, resolve_core_class
    coupling = reference_coupling()
    A, Sc = midtrain_case(0)
    core = resolve_core_class("explicit").from_state(A, Sc, device=dev)
    tgt, _ = _fa_targets(A, 7)
    tgt = {f: torch.from_numpy(v).to(dev) for f, v in tgt.items()}
    start = {f: getattr(core, f).detach().clone() for f in _abi.FIELD_NAMES}
    # the network's raw output between intervals (seeded, unit scales),
    # itself a leaf: gradients reach it as they would reach a U-Net
    g = torch.Generator(device=dev).manual_seed(17)
    raw = (1e-3 * torch.randn((coupling.OUTPUT_CHANNELS, core.im, core.jm), generator=g, device=dev)).requires_grad_()
    scales = {f: 1.0 for f in coupling.OUTPUT_FIELDS}

    def correct(c):
        coupling.apply_joint_correction(c, raw, scales)

    best = fwd_adjoint_timing(core, start, tgt, correct, FA_INTERVALS, FA_STEPS_PER_INTERVAL, float(Sc["time"]),
                              reps, args.warmup, dev)
    nint = FA_INTERVALS * FA_STEPS_PER_INTERVAL
    days = nint * float(core.dti) / 86400.0
    return {"value": days / (best / 1000.0), "unit": UNIT, "ms_per_sample": best,
            "workload": f"explicit core, {FA_GRID[0]}x{FA_GRID[1]}x{FA_GRID[2]} noise basin (dtE=6 s, isplit=20, "
                        f"dtI=120 s), T/S/u/v-perturbed member; {FA_INTERVALS} x 1 h intervals ({nint} internal "
                        "steps) with apply_joint_correction of a seeded raw (60, im, jm) output (unit scales) between "
                        "them, MSE(u,v,T,S) loss, backward to every state field and the raw output; checkpoint per "
                        "internal step, hand-written CUDA step adjoint",
            "timing": f"median of {reps} samples, CUDA events around forward+backward (L2 not flushed: the "
                      "90x82x16 state fits in L2)"}


def fwd_adjoint_midtrain_batch(args, dev, members=8, reps=3):
    """The Midtrain-shaped forward+adjoint of an ensemble: ``members``
    seeded members (``midtrain_case(m)``), each with its own core, raw
    correction output and CUDA stream.  Every member's three differentiable
    intervals are enqueued on its stream through run_time_loop with
    ``status_deferred`` (no host synchronisation between
    intervals); the loss is the sum of the members' MSE(u, v, T, S) and one
    backward() reaches every member's state leaves and raw output.  Timed
    with CUDA events on the launching stream around forward+backward; the
    device status of every member is checked after each sample."""
    import torch
    from neuralpom_b200 import _abi, resolve_core_class
    coupling = reference_coupling()
    main = torch.cuda.current_stream(dev)
    mem = []
    for m in range(members):
        A, Sc = midtrain_case(m)
        core = resolve_core_class("explicit").from_state(A, Sc, device=dev)
        core.status_deferred = True
        tgt, _ = _fa_targets(A, 7 + m)
        g = torch.Generator(device=dev).manual_seed(17 + m)
        mem.append({"core": core, "t0": float(Sc["time"]), "stream": torch.cuda.Stream(dev),
                    "tgt": {f: torch.from_numpy(v).to(dev) for f, v in tgt.items()},
                    "start": {f: getattr(core, f).detach().clone() for f in _abi.FIELD_NAMES},
                    "raw0": 1e-3 * torch.randn((coupling.OUTPUT_CHANNELS, core.im, core.jm), generator=g,
                                               device=dev)})
    scales = {f: 1.0 for f in coupling.OUTPUT_FIELDS}

    def prepare():
        for mb in mem:
            c = mb["core"]
            for f in _abi.FIELD_NAMES:
                setattr(c, f, mb["start"][f].clone())
            mb["leaves"] = [getattr(c, f).requires_grad_(True) for f in _abi.ADJ_STATE_FIELDS]
            mb["raw"] = mb["raw0"].clone().requires_grad_()

    def fwd_bwd():
        go = torch.cuda.Event()
        go.record(main)
        losses = []
        for mb in mem:
            c, st = mb["core"], mb["stream"]
            st.wait_event(go)
            with torch.cuda.stream(st):
                dti = float(c.dti)
                for k in range(FA_INTERVALS):
                    c.time0 = mb["t0"] + k * FA_STEPS_PER_INTERVAL * dti / 86400.0
                    c.iend = FA_STEPS_PER_INTERVAL
                    c.run_time_loop()
                    if k < FA_INTERVALS - 1:
                        coupling.apply_joint_correction(c, mb["raw"], scales)
                losses.append(sum(((getattr(c, f) - mb["tgt"][f]) ** 2).mean() for f in mb["tgt"]))
        for mb in mem:
            main.wait_stream(mb["stream"])
        for loss in losses:
            loss.record_stream(main)
        torch.stack(losses).sum().backward()

    for _ in range(max(args.warmup, 1)):
        prepare()
        fwd_bwd()
    torch.cuda.synchronize(dev)
    ms = []
    for _ in range(reps):
        prepare()
        torch.cuda.synchronize(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(main)
        fwd_bwd()
        e1.record(main)
        torch.cuda.synchronize(dev)
        ms.append(e0.elapsed_time(e1))
        for mb in mem:
            mb["core"].check_deferred_status()
            assert mb["raw"].grad is not None and all(t.grad is not None for t in mb["leaves"][:12])
    best = statistics.median(ms)
    nint = FA_INTERVALS * FA_STEPS_PER_INTERVAL
    days = members * nint * float(mem[0]["core"].dti) / 86400.0
    return {"value": days / (best / 1000.0), "unit": UNIT, "ms_per_sample": best, "members": members,
            "workload": f"{members} seeded members of the Midtrain-shaped case (explicit core, "
                        f"{FA_GRID[0]}x{FA_GRID[1]}x{FA_GRID[2]}, {FA_INTERVALS} x 1 h with apply_joint_correction "
                        "between intervals), each on its own core and CUDA stream; sum of the members' "
                        "MSE(u,v,T,S), one backward to every member's state and raw output",
            "timing": f"median of {reps} samples, CUDA events around forward+backward of all members"}


# The reference's registered GPU training setup for the implicit core
# (configs/examples/implicit_1h.json:7-12): compiled strict vertical kernels
# and the Triton CG operator (hybrid/sparse_physics.py:19-28).
REF_FAST_MODE = {"acceleration": "strict_vertical_compiled", "cg_backend": "triton", "compiled_kernels": ("proft",)}


def reference_modes(fn, kind, where, **kw):
    """``fn`` timed under the reference's default options (eager, torch CG)
    and, for the implicit core (``kind``) on a GPU (``where``), under its
    compiled training setup;
    the line reports the faster (the reference's best on this GPU) and
    every mode's figure."""
    modes = {"eager": {}}
    if kind != "explicit" and str(where) != "cpu":
        modes["strict_vertical_compiled+triton_cg"] = REF_FAST_MODE
    out = {}
    for name, opts in modes.items():
        try:
            out[name] = fn(physics_kw=opts, **kw)
        except Exception as exc:  # a mode the reference cannot run here is reported, not fatal
            out[name] = {"error": f"{type(exc).__name__}: {exc}"[:300]}
    ok = {k: v for k, v in out.items() if "value" in v}
    if not ok:
        return {"error": "no reference mode ran", "modes": out}
    best = max(ok, key=lambda k: ok[k]["value"])
    res = dict(ok[best])
    res["mode"] = best
    res["modes"] = {k: (v.get("value") if "value" in v else v) for k, v in out.items()}
    return res


def reference_fwd_adjoint_sample(device, internal_steps=6, case=None, core_name="explicit", seed=7, physics_kw=None):
    """The reference core under torch autograd
    (SparsePhysics.advance(differentiable=True) + backward) on the same
    state: ``internal_steps`` steps, wall clock."""
    import torch
    A, Sc = case if case is not None else midtrain_case(0)
    core, rh = reference_core(A, Sc, device, core_name)
    tgt, _ = _fa_targets(A, seed)
    from neuralpom_b200 import _abi
    names = [k for k in _abi.ADJ_STATE_FIELDS if torch.is_tensor(getattr(core, k, None))]

    def once(n):
        leaves = []
        for k in names:
            t = getattr(core, k).detach().clone().requires_grad_(True)
            setattr(core, k, t)
            leaves.append(t)
        rh.advance(core, core_name, n, differentiable=True, device=device, **(physics_kw or {}))
        loss = sum(((getattr(core, f) - torch.from_numpy(v).to(device)) ** 2).mean() for f, v in tgt.items())
        loss.backward()
        for k, v in list(vars(core).items()):
            if torch.is_tensor(v):
                setattr(core, k, v.detach())
    once(1)
    if device != "cpu":
        torch.cuda.synchronize()
    t0 = time.perf_counter()
    once(internal_steps)
    if device != "cpu":
        torch.cuda.synchronize()
    sec = time.perf_counter() - t0
    days = internal_steps * float(core.dti) / 86400.0
    return {"value": days / sec, "unit": UNIT, "device": str(device),
            "threads": (os.cpu_count() or 1) if device == "cpu" else None,
            "sample": f"{internal_steps} internal steps forward+backward of the {_basin_name(A)} (reference "
                      f"{core_name} core, torch autograd through SparsePhysics.advance(differentiable=True"
                      f"{', ' + str(physics_kw) if physics_kw else ''}), after a 1-step warm-up; wall clock)"}


def reference_core(A, Sc, device="cpu", core_name="implicit_p0_fixed"):
    """Reference core (baseline/_ref install, else the source tree) loaded
    with this benchmark's state and clock."""
    from oracle import ref_harness as rh
    path = os.path.join(ROOT, "baseline", "_ref")
    if not os.path.isdir(os.path.join(path, "neuralpom")):
        path = rh.default_reference_path()
    if path is None:
        raise RuntimeError("reference package not installed (baseline/_ref missing)")
    rh.import_reference(path)
    import torch
    from neuralpom.core_factory import resolve_core_class as ref_resolve
    from neuralpom.hybrid import build_initialized_core
    im, jm, kb = A["u"].shape
    core = build_initialized_core(ref_resolve(core_name), torch.device(device), im, jm, dte=Sc["dte"],
                                  isplit=Sc["isplit"])
    core.prtd1 = core.prtd2 = 1e9
    core.iprint = 10 ** 9
    scal = {k: v for k, v in Sc.items() if k in (
        "alpha", "smoth", "horcon", "eta_solver_rel_tol", "eta_solver_tol", "eta_solver_preconditioner",
        "barotropic_shapiro", "tracer_shapiro", "velocity_shapiro", "double_gyre_wind_stress_pa", "hmax",
        "time", "time0")}
    scal["spatial_shapiro_enabled"] = False
    rh.load_state(core, {k: v for k, v in A.items() if hasattr(core, k)}, scal)
    return core, rh


FP64_FIELDS = ("u", "v", "t", "s", "el", "ua", "va", "q2", "q2l", "km", "kh", "w", "rho")


def fp64_day_error(A, Sc, nin, dev, core_name):
    """Error of every field of the B200 step after ``nin`` internal steps
    from the workload's initial state, against the reference core's own run
    of the same steps in float64 on the same device (outside the timed
    region), and the PCG iteration counts of both runs."""
    import torch
    from neuralpom_b200 import resolve_core_class
    b = resolve_core_class(core_name).from_state(A, Sc, device=dev)
    b.time0, b.iend = float(b.time), nin
    b.run_time_loop()
    got = {f: getattr(b, f).detach().cpu().numpy().astype(np.float64) for f in FP64_FIELDS}
    its_b = list(b._eta_solver_iteration_history)
    core, rh = reference_core(A, Sc, dev, core_name)
    rh.ReferenceFloat64.promote(core)
    if hasattr(core, "_eta_solver_iteration_history"):
        core._eta_solver_iteration_history = []
    t0 = time.perf_counter()
    with rh.ReferenceFloat64():
        if hasattr(core, "_build_acceleration_cache"):
            core._build_acceleration_cache()
        rh.advance(core, core_name, nin, device=dev)
    torch.cuda.synchronize(dev)
    sec = time.perf_counter() - t0
    ref = {f: getattr(core, f).detach().cpu().numpy() for f in FP64_FIELDS}
    assert all(v.dtype == np.float64 for v in ref.values())
    err = {f: float(np.abs(got[f] - ref[f]).max() / max(float(np.abs(ref[f]).max()), 1e-30)) for f in FP64_FIELDS}
    out = {"fields": err, "metric": "max|b200 - ref64| / max|ref64| per field",
           "run": f"{nin} internal steps from the workload's initial state; the reference core in float64 "
                  f"(float32 scratch promoted) on {dev}, {sec:.1f} s, outside the timed region"}
    its_r = list(getattr(core, "_eta_solver_iteration_history", []))
    if its_b:
        out["pcg_iterations"] = {"b200_total": int(sum(its_b)), "b200_min": int(min(its_b)),
                                 "b200_max": int(max(its_b)), "b200_mean": float(np.mean(its_b)),
                                 "ref64_total": int(sum(its_r)) if its_r else None,
                                 "first_12_b200": its_b[:12], "first_12_ref64": its_r[:12]}
    return out


def _basin_name(A):
    im, jm, kb = A["u"].shape
    return f"{im}x{jm}x{kb} basin"


def reference_cpu_sample(A, Sc, internal_steps=6, warm=1, reps=2, device="cpu", core_name="implicit_p0_fixed"):
    import torch
    threads = os.cpu_count() or 1
    torch.set_num_threads(threads)
    core, rh = reference_core(A, Sc, device, core_name)
    rh.advance(core, core_name, warm, device=device)
    t0 = time.perf_counter()
    for _ in range(reps):
        rh.advance(core, core_name, internal_steps, device=device)
    if device != "cpu":
        torch.cuda.synchronize()
    sec = time.perf_counter() - t0
    days = reps * internal_steps * float(core.dti) / 86400.0
    return {"value": days / sec, "unit": UNIT, "cores": threads, "kind": "reference",
            "sample": f"{reps} x {internal_steps} internal steps of the {_basin_name(A)} "
                      f"(reference PyTorch core {core_name}, {device}, after {warm} warm-up step)"}


def reference_gpu_sample(A, Sc, device, internal_steps=12, warm=2, reps=2, core_name="implicit_p0_fixed",
                         physics_kw=None):
    """The reference PyTorch core on this GPU, on the same basin, under the
    SparsePhysics options ``physics_kw`` (default: eager mode, torch CG):
    the comparison the B200 core is built to beat on the same hardware."""
    import torch
    core, rh = reference_core(A, Sc, device, core_name)
    kw = physics_kw or {}
    rh.advance(core, core_name, warm, device=device, **kw)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(reps):
        rh.advance(core, core_name, internal_steps, device=device, **kw)
    torch.cuda.synchronize()
    sec = time.perf_counter() - t0
    days = reps * internal_steps * float(core.dti) / 86400.0
    return {"value": days / sec, "unit": UNIT, "device": str(device),
            "sample": f"{reps} x {internal_steps} internal steps of the {_basin_name(A)} (reference PyTorch core "
                      f"{core_name}, {kw or 'eager, torch CG'}, after {warm} warm-up steps; wall clock around "
                      "synchronised calls)"}


def run_reference(args):
    ws_n, rank, local = dist_env()
    if rank != 0:
        return
    A, Sc = workload(0)
    import torch
    dev = args.ref_device
    threads = os.cpu_count() or 1
    torch.set_num_threads(threads)
    core, rh = reference_core(A, Sc, dev)
    n = args.ref_internal_steps
    for _ in range(args.warmup):
        rh.advance(core, "implicit_p0_fixed", n, device=dev)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        rh.advance(core, "implicit_p0_fixed", n, device=dev)
    if dev != "cpu":
        torch.cuda.synchronize()
    sec = time.perf_counter() - t0
    days = args.steps * n * float(core.dti) / 86400.0
    value = days / sec
    out = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 0 if dev == "cpu" else 1,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * sec / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "semi-implicit core, closed 90x82x16 seamount basin (dx=5 km), forward",
                   "grid": list(GRID), "dti_s": DTI, "internal_steps_per_step": n, "device": dev},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "reference",
                         "sample": f"{args.steps} x {n} internal steps, reference PyTorch core on {dev}"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


# ---------------------------------------------------------------------------
# batch workload: 64 members on mixed grids (one GPU)
# ---------------------------------------------------------------------------
BATCH_GRIDS = ((90, 82, 24), (128, 112, 24), (177, 161, 16))


def batch_member(m, im, jm):
    """Member m of the batch: even members the explicit noise basin
    (dtE = 6 s, isplit = 30), odd members the semi-implicit seamount with a
    seeded 0.2 degC temperature perturbation; clock at 2 days (ramp
    saturated, so every step replays its graph)."""
    from neuralpom_b200 import cases
    if m % 2 == 0:
        A, Sc = cases.noise_basin(im, jm, kb=16, seed=m)
        name = "explicit"
    else:
        A, Sc = cases.seamount(im, jm, kb=16, dti=DTI)
        g = np.random.default_rng(100 + m)
        p = (0.2 * g.standard_normal(A["t"].shape) * A["fsm"][:, :, None]).astype(np.float32)
        A["t"] = A["t"] + p
        A["tb"] = A["tb"] + p
        name = "implicit_p0_fixed"
    Sc = dict(Sc)
    Sc.update(time=2.0, time0=2.0)
    return A, Sc, name


def step_algorithmic_bytes(im, jm, kb, core_name):
    """Algorithmic bytes of one internal step (PHASE_IO, 4 B per element of
    every distinct array each phase reads or writes)."""
    n3, n2 = im * jm * kb, im * jm
    phases = ["A1_forcing_advct", "A2_baropg_smag_means", "A3_advave_predictor"]
    if core_name == "explicit":
        phases += ["E_external_explicit"]
    else:
        phases += ["E_external", "I5_corrector_filter"]
    phases += ["B1_barotropic_fix", "B2A_vertvl", "B2B_advq", "B3_profq", "B4_edges_bcond6", "B5_qfilter_advt1",
               "B6_proft", "B7_tsfilter_dens", "B8_advuv_profuv", "B9_velfilter_shift"]
    total = 0
    for ph in phases:
        r3, r2, w3, w2 = PHASE_IO[ph]
        total += 4 * ((r3 + w3) * n3 + (r2 + w2) * n2)
    if core_name != "explicit":
        ni, nj = im - 2, jm - 2
        total += 4 * (ni * ni + nj * nj + ni * nj)
    return total


def run_batch(args):
    print(json.dumps(batch_measure(args)), flush=True)


def batch_summary(args):
    """The 64-member batch (one timed simulated day of every member) as a
    key of the default bench line."""
    import copy
    import torch
    a = copy.copy(args)
    a.steps, a.warmup, a.internal_steps, a.batch_mode = 1, 1, None, "launch"
    out = batch_measure(a)
    torch.cuda.empty_cache()
    ref = out["reference_gpu_loop"]
    return {"value": out["value"], "unit": out["unit"], "ms_per_step": out["ms_per_step"], "steps": 1,
            "warmup": 1, "workload": out["config"]["workload"], "gpu_launches": out["gpu_launches"],
            "hbm_frac": out["roofline"]["frac"], "reference_gpu_loop": ref["value"] if ref else None,
            "clocks": out["clocks"], "autotune": out["autotune"]}


def batch_measure(args):
    if args.batch_mode == "launch" and args.batch_streams == 2:
        if os.environ.get("NPOM_BATCH_SUBCYCLE") == "coop":
            # two batches that both launch cooperative grids share one stream
            args.batch_streams = 1
        # otherwise only the semi-implicit batch launches a cooperative grid
        # (the PCG of its largest members); the autotuner picks the cap on
        # its blocks per member, which leaves SMs to the explicit batch on
        # the other stream (npom_tuning.batch_pcg_blocks)
    if args.batch_mode == "streams":
        # members run concurrently: the explicit subcycle runs on one cluster
        # per member (up to four cells per thread), never as a cooperative
        # grid, which needs all of its blocks resident while other streams
        # hold SMs
        os.environ.setdefault("NPOM_SUBCYCLE", "nocoop")
        # one hardware queue per stream up to 32 (the default 8 makes streams
        # that share a queue wait on each other's work); before the context
        os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")
    import torch
    from neuralpom_b200 import _abi, batch, build, resolve_core_class
    ws_n, rank, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    build.build()
    members = []
    m = 0
    for im, jm, count in BATCH_GRIDS:
        for _ in range(count):
            A, Sc, name = batch_member(m, im, jm)
            core = resolve_core_class(name).from_state(A, Sc, device=dev)
            nday = int(round(86400.0 / float(core.dti)))
            members.append({"core": core, "stream": torch.cuda.Stream(dev), "nday": nday, "name": name,
                            "grid": (im, jm), "A": A, "Sc": Sc})
            m += 1
    main_stream = torch.cuda.current_stream(dev)
    flush = torch.zeros(64 * 1024 * 1024, dtype=torch.float32, device=dev)

    def launch_all(steps_of):
        # members enqueue their steps in --batch-chunk turns a day, so that
        # the hardware queues hold every member's work from the start
        start = torch.cuda.Event()
        start.record(main_stream)
        todo = []
        for mb in members:
            mb["stream"].wait_event(start)
            todo.append([mb, steps_of(mb), 0, float(mb["core"].time)])
        while any(t[2] < t[1] for t in todo):
            for t in todo:
                mb, n, done, t0 = t
                k = min(max(1, -(-n // max(1, args.batch_chunk))), n - done)
                if k > 0:
                    mb["core"].launch_steps(k, t0, 1 + done, mb["stream"])
                    t[2] += k
        for mb, n, _, t0 in todo:
            mb["core"].time = mb["core"].dti * n / 86400.0 + t0
            e = torch.cuda.Event()
            e.record(mb["stream"])
            main_stream.wait_event(e)

    groups = {}
    for mb in members:
        groups.setdefault(mb["name"], []).append(mb)

    group_streams = [torch.cuda.Stream(dev) for _ in groups] if args.batch_streams == 2 else None

    def launch_batched(steps_of):
        # each core's members advance as one batch (one launch per phase);
        # the two batches take turns on one stream (or run each on its own
        # stream), --batch-chunk turns a day
        todo = []
        if group_streams:
            go = torch.cuda.Event()
            go.record(main_stream)
        for g, mbs in enumerate(groups.values()):
            n = steps_of(mbs[0])
            st = group_streams[g] if group_streams else main_stream
            if group_streams:
                st.wait_event(go)
            todo.append([[mb["core"] for mb in mbs], n, 0, float(mbs[0]["core"].time),
                         max(1, -(-n // max(1, args.batch_chunk))), st])
        launches = 0
        while any(t[2] < t[1] for t in todo):
            for t in todo:
                cores, n, done, t0, per_turn, st = t
                k = min(per_turn, n - done)
                if k > 0:
                    launches += batch.launch_batch(cores, k, t0, 1 + done, st)
                    t[2] += k
        for cores, n, _, t0, _, st in todo:
            for c in cores:
                c.time = c.dti * n / 86400.0 + t0
            if group_streams:
                main_stream.wait_stream(st)
        return launches

    def advance(steps_of):
        if args.batch_mode == "launch":
            return launch_batched(steps_of)
        launch_all(steps_of)
        return sum(launches_of(mb["core"], steps_of(mb), 2.0) for mb in members)

    # a bench step is one simulated day of every member; --internal-steps
    # replaces the day by that many internal steps of every member (profiling)
    def steps_of(mb):
        return args.internal_steps or mb["nday"]

    for _ in range(args.warmup):
        advance(lambda mb: 4)
    torch.cuda.synchronize(dev)

    def set_tuning(tuning):
        # tuning: {(core name, knob): value}; members of one core share it
        for name, mbs in groups.items():
            t = {k: v for (g, k), v in tuning.items() if g == name and v}
            for mb in mbs:
                mb["core"].tuning = t or None

    def timed_day():
        total, n = 0.0, 0
        for _ in range(args.steps):
            l2_flush(flush)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(main_stream)
            n += advance(steps_of)
            b.record(main_stream)
            torch.cuda.synchronize(dev)
            total += a.elapsed_time(b)
        return total, n

    tune_info = None
    if args.batch_mode == "launch" and not args.no_batch_tune:
        # the autotuner over both batches together (they share the GPU):
        # one simulated hour of every member per candidate, median of 2
        from neuralpom_b200 import autotune
        space = {}
        for name, mbs in groups.items():
            for k, vals in autotune.space_for(mbs[0]["core"], batch=True).items():
                if k in ("pcg_form",) or (k == "subcycle_form" and args.batch_streams == 2):
                    continue  # cooperative grids stay with the rules on shared SMs
                space[(name, k)] = vals

        def measure(tuning):
            set_tuning(tuning)
            try:
                advance(lambda mb: max(1, mb["nday"] // 24))
                ts = []
                for _ in range(2):
                    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    a.record(main_stream)
                    advance(lambda mb: max(1, mb["nday"] // 24))
                    b.record(main_stream)
                    torch.cuda.synchronize(dev)
                    ts.append(a.elapsed_time(b))
            except Exception:
                return float("inf")
            bad = 0
            for mb in members:
                bits, _ = mb["core"].read_status(0)
                bad |= bits & (_abi.DEV_TIMEOUT | _abi.DEV_VMAX | _abi.DEV_NONFINITE)
            return float("inf") if bad else statistics.median(ts)

        log = []
        t0 = time.perf_counter()
        best, t_best, t_rule = autotune.search(measure, space, log=log)
        set_tuning({})
        rule_ms, _ = timed_day()
        set_tuning(best)
        tune_info = {"tuning": {f"{g}.{k}": v for (g, k), v in best.items()},
                     "rule_value": sum(steps_of(mb) * float(mb["core"].dti) / 86400.0 for mb in members) * args.steps
                     / (rule_ms / 1000.0),
                     "hour_ms_rule": t_rule, "hour_ms_tuned": t_best, "candidates": len(log),
                     "search_s": time.perf_counter() - t0,
                     "note": "coordinate descent over npom_tuning (A1/B5 forms and tile rows, column form, PCG "
                             "CTA count and cooperative block cap, per core batch); rule_value: the library's "
                             "rules, no cap"}
    total_ms, launches = 0.0, 0
    with ClockSampler(local) as clk:
        total_ms, launches = timed_day()
    for mb in members:
        bits, _ = mb["core"].read_status(0)
        if bits & (_abi.DEV_TIMEOUT | _abi.DEV_VMAX | _abi.DEV_NONFINITE):
            raise RuntimeError(f"device status 0x{bits:x} in the batch run")
    nmem = len(members)
    member_days = sum(steps_of(mb) * float(mb["core"].dti) / 86400.0 for mb in members) * args.steps
    value = member_days / (total_ms / 1000.0)
    nbytes = sum(steps_of(mb) * step_algorithmic_bytes(*mb["grid"], 16, mb["name"]) for mb in members) * args.steps
    peak, src = measured_peaks()
    achieved = nbytes / (total_ms / 1000.0) / 1e9
    ref = None
    if not args.no_ref_gpu:
        # the reference core looping the members: its time per internal step
        # on each (grid, core) pair on this GPU, times every member's steps
        per_step = {}
        for mb in members:
            key = (mb["grid"], mb["name"])
            if key in per_step:
                continue
            smp = reference_gpu_sample(mb["A"], mb["Sc"], dev, internal_steps=4, warm=1, reps=1,
                                       core_name=mb["name"])
            dti = float(mb["core"].dti)
            per_step[key] = (4 * dti / 86400.0) / smp["value"] / 4
        loop_sec = sum(mb["nday"] * per_step[(mb["grid"], mb["name"])] for mb in members)
        ref = {"value": nmem / loop_sec, "unit": UNIT, "device": str(dev),
               "sample": "the reference PyTorch core (eager, its default SparsePhysics options) timed over 4 "
                         "internal steps on each of the 6 (grid, core) pairs on this GPU, looped over every "
                         "member's day: sum of member steps x time per step",
               "seconds_per_step": {f"{g[0]}x{g[1]} {n}": v for (g, n), v in per_step.items()}}
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 (FP64 PCG dot products)", "data": "synthetic",
        "config": {"workload": WORKLOADS["batch"]["desc"], "members": nmem, "mode": args.batch_mode,
                   "explicit_subcycle": (os.environ.get("NPOM_BATCH_SUBCYCLE", "phases")
                                         if args.batch_mode == "launch" else os.environ.get("NPOM_SUBCYCLE")),
                   "turns_per_day": args.batch_chunk, "streams": args.batch_streams,
                   "pcg_blocks_per_member": os.environ.get("NPOM_BATCH_PCG_BLOCKS"),
                   "hw_queues": os.environ.get("CUDA_DEVICE_MAX_CONNECTIONS"),
                   "member_days_per_step": member_days / args.steps, "internal_steps": args.internal_steps,
                   "l2": "flushed (256 MiB write) before every timed step"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": src, "traffic": None, "algorithmic_bytes": nbytes,
                     "note": "whole batch: algorithmic bytes of every member's steps over the device time"},
        "reference_gpu_loop": ref, "cpu_baseline": None, "e2e": None, "gpu_launches": launches,
        "clocks": clk.summary(), "autotune": tune_info,
    }
    for mb in members:
        mb["core"] = None
    return out


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "batch":
        run_batch(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
