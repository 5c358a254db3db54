"""ctypes mirror of ``include/npom.h`` and the loader of the CUDA library.

The struct layouts and name lists here must match the header; the library
exports its own field/workspace names and struct sizes so that a mismatch is
caught at load time (``check_layout``).
"""
from __future__ import annotations

import ctypes
import os

FIELD_NAMES = (
    "h dx dy art aru arv fsm dum dvm cor cbc north_e "
    "z zz dz dzz "
    "ele elw eln els uabe uabw vabn vabs tbe sbe tbw sbw tbn sbn tbs sbs "
    "u ub uf v vb vf w t tb s sb rho rmean tclim sclim q2 q2b q2l q2lb km kh kq l aam advx advy drhox drhoy curv "
    "el elb elf et etb etf d dt ua uab uaf va vab vaf utf utb vtf vtb egf egb adx2d ady2d drx2d dry2d aam2d "
    "advua advva fluxua fluxva wubot wvbot wusurf wvsurf wtsurf wssurf vfluxf vfluxb swrad e_atmos tps tsurf ssurf"
).split()

WS_NAMES = "us vs den_u den_v d_baro rhs x r p zv ap ce cw cn cs inv_art diag sx sy inv_eigs t1 t2".split()

PHASES = ("A1_forcing_advct", "A2_baropg_smag_means", "A3_advave_predictor", "E_external",
          "I5_corrector_filter", "B1_barotropic_fix", "B2A_vertvl", "B2B_advq", "B3_profq",
          "B4_edges_bcond6", "B5_qfilter_advt1", "B6_proft", "B7_tsfilter_dens", "B8_advuv_profuv",
          "B9_velfilter_shift")

FIELDS_1D_K = ("z", "zz", "dz", "dzz")
FIELDS_EDGE_J = ("ele", "elw", "uabe", "uabw")
FIELDS_EDGE_I = ("eln", "els", "vabn", "vabs")
FIELDS_EDGE_JK = ("tbe", "sbe", "tbw", "sbw")
FIELDS_EDGE_IK = ("tbn", "sbn", "tbs", "sbs")
FIELDS_3D = tuple("u ub uf v vb vf w t tb s sb rho rmean tclim sclim q2 q2b q2l q2lb km kh kq l aam advx advy "
                  "drhox drhoy curv".split())

CORE_EXPLICIT, CORE_IMPLICIT = 0, 1
PRECOND_JACOBI, PRECOND_SPECTRAL = 0, 1
PROFQ_PRODUCTION, PROFQ_POM08 = 0, 1
OBC_NATIVE, OBC_SEAMOUNT, OBC_COASTAL, OBC_JZB = 0, 1, 2, 3
DEV_VMAX, DEV_TIMEOUT, DEV_PCG_MAXIT, DEV_NONFINITE = 0x1, 0x2, 0x4, 0x8
MAX_COOP_BLOCKS = 1024


def field_shape(name, im, jm, kb):
    if name in FIELDS_3D:
        return (im, jm, kb)
    if name in FIELDS_1D_K:
        return (kb,)
    if name in FIELDS_EDGE_J:
        return (jm,)
    if name in FIELDS_EDGE_I:
        return (im,)
    if name in FIELDS_EDGE_JK:
        return (jm, kb)
    if name in FIELDS_EDGE_IK:
        return (im, kb)
    return (im, jm)


def ws_shape(name, im, jm):
    ni, nj = im - 2, jm - 2
    if name == "sx":
        return (ni, ni)
    if name == "sy":
        return (nj, nj)
    if name in ("inv_eigs", "t1", "t2"):
        return (ni, nj)
    return (im, jm)


TUNING_FIELDS = ("a1_form", "b5_form", "tile_blocks_per_sm", "column_form", "subcycle_form", "pcg_form", "pcg_ctas",
                 "batch_pcg_blocks")


class NpomTuning(ctypes.Structure):
    """Launch shapes of the step (``npom_tuning``): all zero keeps the
    library's rules."""
    _fields_ = [(n, ctypes.c_int32) for n in TUNING_FIELDS] + [("reserved", ctypes.c_int32 * 2)]


class NpomParams(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int32) for n in (
        "device", "im", "jm", "kb", "core", "isplit", "ispadv", "nbct", "nbcs", "ntp", "mode", "nadv",
        "eta_max_iter", "eta_precond", "wind_forcing", "has_vmix", "lramp")] + [
        (n, ctypes.c_double) for n in (
            "dti", "dte", "dti2", "dte2", "ispi", "isp2i", "alpha", "smoth", "horcon", "grav", "umol", "tprni",
            "small", "kappa", "rhoref", "tbias", "sbias", "vmaxl", "hmax", "rfe", "rfw", "rfn", "rfs", "aam_min",
            "pi", "eta_tol", "eta_rel_tol", "barotropic_shapiro", "tracer_shapiro", "velocity_shapiro",
            "wind_tau0", "vmix", "period", "inverse_scale", "sw")] + [
        ("nitera", ctypes.c_int32), ("profq_form", ctypes.c_int32),
        ("obc_form", ctypes.c_int32), ("tuning", NpomTuning), ("zsh", ctypes.c_double),
        ("periodic_x", ctypes.c_int32)]


class NpomWorkspace(ctypes.Structure):
    _fields_ = [("buf", ctypes.c_void_p * len(WS_NAMES)), ("partials", ctypes.c_void_p),
                ("sync", ctypes.c_void_p), ("status", ctypes.c_void_p), ("cg_iters", ctypes.c_void_p),
                ("mp3d", ctypes.c_void_p), ("tide", ctypes.c_void_p), ("robin", ctypes.c_void_p)]


class NpomClock(ctypes.Structure):
    _fields_ = [("time0", ctypes.c_double), ("first_iint", ctypes.c_int32), ("nsteps", ctypes.c_int32)]


FieldArray = ctypes.c_void_p * len(FIELD_NAMES)


class NpomAdjointWs(ctypes.Structure):
    _fields_ = [("lam", ctypes.c_void_p * len(FIELD_NAMES)), ("save", ctypes.c_void_p),
                ("save_floats", ctypes.c_size_t), ("pcg_x", ctypes.c_void_p)]


# State fields of the explicit core that carry a cotangent through a step:
# everything the step reads or writes apart from geometry, forcing and
# open-boundary arrays (explicit/base.py:129-195).
ADJ_STATE_FIELDS = (
    "u", "ub", "uf", "v", "vb", "vf", "w", "t", "tb", "s", "sb", "rho", "q2", "q2b", "q2l", "q2lb", "km", "kh",
    "kq", "l", "aam", "advx", "advy", "drhox", "drhoy", "curv", "el", "elb", "elf", "et", "etb", "etf", "d", "dt",
    "ua", "uab", "uaf", "va", "vab", "vaf", "utf", "utb", "vtf", "vtb", "egf", "egb", "adx2d", "ady2d", "drx2d",
    "dry2d", "aam2d", "advua", "advva", "fluxua", "fluxva", "wubot", "wvbot", "tps",
)

STATUS_NAMES = {0: "NPOM_OK", 1: "NPOM_ERR_ARG", 2: "NPOM_ERR_CUDA", 3: "NPOM_ERR_DEVICE", 4: "NPOM_ERR_TOO_LARGE"}
STATIC_MAX_CELLS = 32768


def library_path():
    return os.path.join(os.path.dirname(os.path.abspath(__file__)), "_lib", "libnpom_b200.so")


_LIB = None


def load_library():
    """Load ``libnpom_b200.so`` and declare its signatures.  Raises if the
    library has not been built -- there is no other implementation."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = library_path()
    if not os.path.exists(path):
        raise RuntimeError(f"neuralpom_b200 CUDA library missing at {path}; run `python -m neuralpom_b200.build`")
    lib = ctypes.CDLL(path)
    vp, i32, dbl = ctypes.c_void_p, ctypes.c_int, ctypes.c_double
    P = ctypes.POINTER
    lib.npom_abi_version.restype = i32
    lib.npom_field_count.restype = i32
    lib.npom_field_name.restype = ctypes.c_char_p
    lib.npom_field_name.argtypes = [i32]
    lib.npom_ws_count.restype = i32
    lib.npom_ws_name.restype = ctypes.c_char_p
    lib.npom_ws_name.argtypes = [i32]
    lib.npom_params_size.restype = ctypes.c_size_t
    lib.npom_workspace_struct_size.restype = ctypes.c_size_t
    lib.npom_phase_count.restype = i32
    lib.npom_phase_name.restype = ctypes.c_char_p
    lib.npom_phase_name.argtypes = [i32]
    for name in ("npom_step_explicit", "npom_step_implicit"):
        fn = getattr(lib, name)
        fn.restype = i32
        fn.argtypes = [P(NpomParams), P(FieldArray), P(NpomWorkspace), P(NpomClock), vp]
    # members as arrays of pointers: params, field-pointer arrays, workspaces
    lib.npom_step_batch.restype = i32
    lib.npom_step_batch.argtypes = [i32, vp, vp, vp, P(NpomClock), vp]
    lib.npom_batch_launches.restype = ctypes.c_longlong
    lib.npom_batch_launches.argtypes = []
    lib.npom_run_phase.restype = i32
    lib.npom_run_phase.argtypes = [P(NpomParams), P(FieldArray), P(NpomWorkspace), i32, dbl, vp]
    lib.npom_pcg_solve.restype = i32
    lib.npom_pcg_solve.argtypes = [P(NpomParams), P(FieldArray), P(NpomWorkspace), vp]
    lib.npom_pcg_adjoint.restype = i32
    lib.npom_pcg_solve_static.restype = i32
    lib.npom_pcg_solve_static.argtypes = [P(NpomParams), P(FieldArray), vp, vp, vp, vp, vp, vp, vp]
    lib.npom_pcg_adjoint.argtypes = [P(NpomParams), P(FieldArray), P(NpomWorkspace), vp, vp, vp, vp, vp, vp]
    lib.npom_proft.restype = i32
    lib.npom_proft.argtypes = [i32, i32, vp, vp, vp, i32, vp, vp, dbl, vp, vp, vp, i32, vp, dbl, vp, vp, vp, vp]
    lib.npom_status_read.restype = i32
    lib.npom_dens.restype = i32
    lib.npom_dens.argtypes = [P(NpomParams), P(FieldArray), vp, vp, vp, vp]
    lib.npom_dens_adjoint.restype = i32
    lib.npom_dens_adjoint.argtypes = [P(NpomParams), P(FieldArray), vp, vp, vp, vp, vp, vp, vp]
    lib.npom_baropg.restype = i32
    lib.npom_baropg.argtypes = [P(NpomParams), P(FieldArray), vp, vp, dbl, vp, vp, vp, vp]
    lib.npom_baropg_adjoint.restype = i32
    lib.npom_baropg_adjoint.argtypes = [P(NpomParams), P(FieldArray), vp, vp, dbl, vp, vp, vp, vp, vp]
    lib.npom_adjoint_save_floats.restype = ctypes.c_size_t
    lib.npom_adjoint_save_floats.argtypes = [P(NpomParams)]
    for fn in (lib.npom_step_explicit_adjoint, lib.npom_step_implicit_adjoint):
        fn.restype = i32
        fn.argtypes = [P(NpomParams), P(FieldArray), P(NpomWorkspace), P(NpomClock), P(FieldArray),
                       P(NpomAdjointWs), vp]
    lib.npom_status_read.argtypes = [P(NpomWorkspace), i32, P(ctypes.c_uint), vp]
    lib.npom_wait_selftest.restype = i32
    lib.npom_wait_selftest.argtypes = [i32, P(NpomWorkspace), vp]
    check_layout(lib)
    _LIB = lib
    return lib


def check_layout(lib):
    """The library's field/workspace lists and struct sizes must match this
    module's, or every pointer would land in the wrong slot."""
    names = [lib.npom_field_name(i).decode() for i in range(lib.npom_field_count())]
    if names != list(FIELD_NAMES):
        raise RuntimeError("npom field list mismatch between include/npom.h and neuralpom_b200._abi")
    ws = [lib.npom_ws_name(i).decode() for i in range(lib.npom_ws_count())]
    if ws != list(WS_NAMES):
        raise RuntimeError("npom workspace list mismatch")
    if lib.npom_params_size() != ctypes.sizeof(NpomParams):
        raise RuntimeError("npom_params size mismatch")
    if lib.npom_workspace_struct_size() != ctypes.sizeof(NpomWorkspace):
        raise RuntimeError("npom_workspace size mismatch")
    phases = [lib.npom_phase_name(i).decode() for i in range(lib.npom_phase_count())]
    if tuple(phases) != PHASES:
        raise RuntimeError("npom phase list mismatch")


def check(status, what):
    if status != 0:
        raise RuntimeError(f"{what} failed: {STATUS_NAMES.get(status, status)}")
