"""The C-ABI library loads without a GPU and exports what include/npom.h
declares, with matching layouts (no compute calls)."""
import ctypes
import os
import re

import pytest

from neuralpom_b200 import _abi, build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def lib():
    build.build()
    return _abi.load_library()


def declared_functions():
    text = open(os.path.join(ROOT, "include", "npom.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(npom_[a-z_0-9]+)\s*\(", text)))


def test_every_declared_symbol_is_exported(lib):
    names = declared_functions()
    assert "npom_step_implicit" in names and "npom_proft" in names
    for n in names:
        assert hasattr(lib, n), n


def test_layouts_match_header(lib):
    _abi.check_layout(lib)
    assert lib.npom_abi_version() == 1
    assert lib.npom_field_count() == len(_abi.FIELD_NAMES)
    assert lib.npom_params_size() == ctypes.sizeof(_abi.NpomParams)


def test_argument_errors_need_no_gpu(lib):
    # null pointers and bad sizes are rejected before any CUDA call
    assert lib.npom_proft(1, 2, None, None, None, 1, None, None, 1.0, None, None, None, 2, None, 1e-6, None, None,
                          None, None) == 1
    assert lib.npom_proft(1, 6, None, None, None, 9, None, None, 1.0, None, None, None, 2, None, 1e-6, None, None,
                          None, None) == 1
    assert lib.npom_proft(0, 6, None, None, None, 1, None, None, 1.0, None, None, None, 2, None, 1e-6, None, None,
                          None, None) == 0
    assert lib.npom_step_implicit(None, None, None, None, None) == 1
    assert lib.npom_pcg_adjoint(None, None, None, None, None, None, None, None, None) == 1
    # the ensemble call: no members, too many members, null arrays
    assert lib.npom_step_batch(0, None, None, None, None, None) == 1
    assert lib.npom_step_batch(65, None, None, None, None, None) == 1
    assert lib.npom_step_batch(2, None, None, None, None, None) == 1
    # a case policy's free-surface solve is part of its step: the standalone
    # solve refuses it before touching any pointer
    p = _abi.NpomParams()
    p.core, p.im, p.jm, p.kb, p.obc_form = _abi.CORE_IMPLICIT, 24, 20, 16, _abi.OBC_COASTAL
    fa = _abi.FieldArray()
    dummy = ctypes.c_float(0.0)
    assert lib.npom_pcg_solve_static(ctypes.byref(p), ctypes.byref(fa), ctypes.byref(dummy), None, None, None,
                                     None, None, None) == 1


def test_library_is_sm100a(lib):
    # the build targets sm_100a only
    assert "arch=compute_100a,code=sm_100a" in " ".join(build.NVCC_FLAGS)
