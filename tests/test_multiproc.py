"""Host logic of the multi-GPU bench path on CPU: two gloo ranks, each with
its own seeded ensemble member (no exchange of state), each advancing it
(here three steps through the CPU emulation of the device phases, the
stand-in for its GPU) and reporting it, and the max-over-ranks timing that
every rank agrees on."""
import os
import socket
import sys

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _emulator():
    import shutil
    return shutil.which("nvcc") is not None


def _advance(A, Sc, steps=3):
    """(checksum of T, PCG iterations) after ``steps`` steps of a member,
    through the CPU emulation of the device phases."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import emul_harness as emul
    im, jm, kb = A["u"].shape
    E = emul.EmulCore(A, dict(Sc, im=im, jm=jm, kb=kb), "implicit_p0_fixed")
    its = [int(v) for v in E.steps(steps)]
    return float(E.F["t"].astype(np.float64).sum()), its


def _rank(rank, world, port, out):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    ws_n, r, local = bench.dist_env()
    A, Sc = bench.workload(member=r)
    t_local = 10.0 + 5.0 * r                        # a per-rank device time (ms)
    t_max = bench.max_over_ranks(t_local, dist)
    value = bench.aggregate_days_per_s(ws_n, 2, 288, Sc["dti"], t_max)
    advanced = None
    if _emulator():
        reports = [None] * world
        dist.all_gather_object(reports, _advance(A, Sc))
        advanced = reports
    out[r] = (ws_n, float(A["t"].astype(np.float64).sum()), t_max, value, advanced)
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_shard_members_and_agree_on_the_slowest_time():
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        res = dict(out)
    assert res[0][0] == res[1][0] == 2
    # each rank advances its own member: seeded, different temperature fields
    assert res[0][1] != res[1][1]
    # both ranks hold the slowest rank's time and the same whole-job value
    assert res[0][2] == res[1][2] == 15.0
    assert res[0][3] == res[1][3]
    expect = 2 * 2 * 288 * 300.0 / 86400.0 / (15.0 / 1000.0)
    assert abs(res[0][3] - expect) < 1e-9 * expect
    if _emulator():
        # every rank advanced its own member and every rank holds the
        # reports of all: each equal to that member advanced alone
        sys.path.insert(0, ROOT)
        import bench
        assert res[0][4] == res[1][4]
        for r in range(2):
            A, Sc = bench.workload(member=r)
            assert tuple(res[0][4][r]) == _advance(A, Sc)
        assert res[0][4][0][0] != res[0][4][1][0]


def test_member_workloads_are_reproducible():
    sys.path.insert(0, ROOT)
    import bench
    a, _ = bench.workload(member=1)
    b, _ = bench.workload(member=1)
    c, _ = bench.workload(member=0)
    assert np.array_equal(a["t"], b["t"])
    assert not np.array_equal(a["t"], c["t"])
    assert torch.tensor(0).numel() == 1
