"""The failure path of the device's bounded waits, made to run out without
a GPU fault.

Every spin-wait of the library is bounded: the grid barrier of the
cooperative kernels gives up after 2 s, the mbarrier waits of the cluster
PCG's exchanges after 0.5 s, and either records NPOM_DEV_TIMEOUT in the
status word and returns.  ``npom_wait_selftest`` runs those same waits on a
condition nothing satisfies (a block that never arrives, bytes that never
come).  The tests check that the status reaches the host, that the host
raises the reference's error type for it (``RuntimeError``, as for a
failed chunk), through ``run_time_loop`` and through ``batch.run_batch``,
and that the context stays usable: the next step still matches the golden.
"""
import ctypes

import numpy as np
import pytest
import torch

from golden_io import load_step_golden, rel_err

pytestmark = pytest.mark.gpu


def _core(fname, core_name):
    from neuralpom_b200 import resolve_core_class
    A, Sc, OUT = load_step_golden(fname)
    return resolve_core_class(core_name).from_state(A, Sc, device="cuda"), A, Sc, OUT


def _selftest(core, which):
    from neuralpom_b200 import _abi
    lib = _abi.load_library()
    core._workspace()
    st = torch.cuda.current_stream()
    _abi.check(lib.npom_wait_selftest(which, ctypes.byref(core._ws["struct"]), ctypes.c_void_p(st.cuda_stream)),
               "wait self-test")
    torch.cuda.synchronize()


@pytest.mark.parametrize("which", [0, 1])
def test_bounded_wait_runs_out_and_the_core_raises(which):
    from neuralpom_b200 import _abi
    core, A, Sc, OUT = _core("step_implicit_12x10.npz", "implicit_p0_fixed")
    _selftest(core, which)
    bits, _ = core.read_status(0)
    assert bits & _abi.DEV_TIMEOUT, hex(bits)
    with pytest.raises(RuntimeError):
        core._raise_for(bits)
    # the status was cleared by the read and the context is usable: one
    # step from the golden start state matches the reference's
    core.time0, core.iend = float(Sc["time"]), 1
    core.run_time_loop()
    for f, ref in OUT[1].items():
        if f.startswith("scalar") or f == "cg_iters":
            continue
        assert rel_err(getattr(core, f).detach().cpu().numpy(), ref) < 1e-5, f


def test_a_member_timeout_surfaces_through_run_batch():
    """A timeout recorded in one member's status word (here by the grid
    barrier's own bounded wait) makes ``run_batch`` raise for the batch,
    as ``run_time_loop`` does for one core; the next batch step runs."""
    from neuralpom_b200 import batch
    a, A, Sc, OUT = _core("step_implicit_12x10.npz", "implicit_p0_fixed")
    b, _, _, _ = _core("step_implicit_12x10.npz", "implicit_p0_fixed")
    for c in (a, b):
        c.time0, c.iend = float(Sc["time"]), 1
        c._workspace()
    _selftest(b, 0)
    with pytest.raises(RuntimeError, match="timed out"):
        batch.run_batch([a, b])
    for c in (a, b):
        c.time0, c.iend = float(c.time), 1
    batch.run_batch([a, b])
    assert np.array_equal(a.t.cpu().numpy(), b.t.cpu().numpy())
