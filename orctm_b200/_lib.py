"""ctypes binding of liborctm_gpu.so (the C ABI declared in include/orctm_gpu.h).

The shared library is built in-tree (orctm_b200/build.py).  There is no
fallback: if the library is missing or cannot be loaded, load() raises.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
SO = os.path.join(_HERE, "liborctm_gpu.so")
_D = C.POINTER(C.c_double)

ORCTM_OK = 0
ORCTM_E_ARG = -1
ORCTM_E_CUDA = -2
ORCTM_E_NOMEM = -3
ORCTM_E_NOT_CONVERGED = -4
ORCTM_E_GEOMETRY = -5
ORCTM_E_UNSUPPORTED = -6
ORCTM_E_NODEVICE = -7
ORCTM_E_TOO_LARGE = -8

F_UOO, F_VOE, F_WNO, F_UKO, F_VKE, F_WO, F_UOO_1, F_VOE_1, F_WNO_1, F_PNH, F_ZO, F_DVO, F_AVO, \
    F_THO, F_SAO = range(15)
SOLVER_FP64, SOLVER_FP32_REFINED = 0, 1


class Desc(C.Structure):
    _fields_ = [
        ("ie", C.c_int), ("je", C.c_int), ("ke", C.c_int),
        ("i_start", C.c_int), ("j_start", C.c_int), ("ntracers", C.c_int),
        ("ob_west", C.c_int), ("ob_east", C.c_int), ("ob_north", C.c_int), ("ob_south", C.c_int),
        ("dt", C.c_double), ("almzer", C.c_double), ("aulapts", C.c_double),
        ("aulapuv", C.c_double), ("ah00", C.c_double),
        ("dzw", _D), ("di", _D),
        ("dlxp", _D), ("dlyp", _D), ("dtdxpo", _D), ("dtdyo", _D),
        ("dlxu", _D), ("dlyu", _D), ("dtdxuo", _D),
        ("dlxv", _D), ("dlyv", _D), ("dpye", _D),
        ("ddpo", _D), ("weto", _D), ("dduo", _D), ("amsuo", _D), ("ddue", _D), ("amsue", _D),
        ("device", C.c_int),
    ]


class SolveStats(C.Structure):
    _fields_ = [("iterations", C.c_int), ("outer_iterations", C.c_int), ("converged", C.c_int),
                ("relres", C.c_double), ("relres_initial", C.c_double), ("solve_ms", C.c_double)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


OBC_MAX_TIDES = 8


class Obc(C.Structure):
    """orctm_obc: open-boundary tidal constants and sponge parameters."""
    _fields_ = [
        ("ntide", C.c_int), ("period", _D), ("sponge", C.c_int * 4), ("width", C.c_int * 4),
        ("relax_inner", C.c_double), ("relax_bound", C.c_double),
        ("amp", (_D * 3) * 4), ("pha", (_D * 3) * 4),
    ]


class GridInfo(C.Structure):
    """orctm_gridinfo: coordinates and depths of GRID_INFO.ext."""
    _fields_ = [(k, _D) for k in ("lonp", "latp", "lonu", "latu", "lonv", "latv", "depto",
                                  "deuto", "deute")]


class Barotropic(C.Structure):
    """orctm_barotropic: ITPREP's inputs and the barotropic solve's constants."""
    _fields_ = [("deuto", _D), ("deute", _D), ("minvalue", C.c_double), ("grav", C.c_double),
                ("stabn", C.c_double), ("conn", C.c_double), ("rlsa1", C.c_double),
                ("sorpar", C.c_double), ("niter", C.c_int), ("eta_forc", C.c_int)]


B_Z1O, B_B1O, B_USO, B_VSE, B_UZO, B_VZE, B_U1O, B_V1E = range(8)


class Thermo(C.Structure):
    """orctm_thermo: OCTHER's constants and surface forcing."""
    _fields_ = [("eos", C.c_int), ("rho0", C.c_double), ("drdt", C.c_double),
                ("drds", C.c_double), ("t0", C.c_double), ("s0", C.c_double),
                ("grav", C.c_double), ("relsal", C.c_double), ("reltem", C.c_double),
                ("rhoicwa", C.c_double), ("rhosnwa", C.c_double), ("wt", C.c_double),
                ("cstabeps", C.c_double), ("dv0", C.c_double), ("av0", C.c_double),
                ("cavocon", C.c_double), ("cdvocon", C.c_double),
                ("preff", _D), ("dbackv", _D), ("abackv", _D),
                ("sicomo", _D), ("sictho", _D), ("sicsno", _D), ("relsao", _D), ("reltho", _D),
                ("giriv", _D), ("fu10", _D)]


class Coriolis(C.Structure):
    """orctm_coriolis: OCMODMOM's Coriolis inputs."""
    _fields_ = [("ftwou", _D), ("ftwov", _D), ("gila", _D), ("giph", _D), ("omega", C.c_double)]


EOS_UNESCO, EOS_LINEAR = 0, 1
(C_PO, C_STABIO, C_RHOO, C_UK1O, C_VK1E, C_EMINPO, C_RIVRUN, C_KCONDEP) = range(8)
E_UNSTABLE = -9


class NoAllocArgs(C.Structure):
    """orctm_octdiff_noalloc_args: device pointers in the reference's layouts."""
    _fields_ = [("ie", C.c_int), ("je", C.c_int), ("ke", C.c_int),
                ("dt", C.c_double), ("almzer", C.c_double), ("aulapts", C.c_double),
                ("ah00", C.c_double),
                ("tracer_in", C.c_void_p), ("tracer_out", C.c_void_p), ("dvo", C.c_void_p),
                ("ddpo", C.c_void_p), ("weto", C.c_void_p), ("di", C.c_void_p),
                ("dzw", C.c_void_p), ("dlxp", C.c_void_p), ("dlyp", C.c_void_p),
                ("dlxu", C.c_void_p), ("dlyu", C.c_void_p), ("dlxv", C.c_void_p),
                ("dlyv", C.c_void_p), ("zo", C.c_void_p), ("stream", C.c_void_p)]


EXPORTS = (
    "orctm_abi_version", "orctm_status_string", "orctm_last_error", "orctm_create",
    "orctm_destroy", "orctm_field_size", "orctm_upload", "orctm_download", "orctm_ocuad",
    "orctm_ocvad", "orctm_ocwad", "orctm_ocadpo", "orctm_octdiff", "orctm_octimf",
    "orctm_ocvisc", "orctm_ocvtot_nh", "orctm_step_hotpath", "orctm_set_solver",
    "orctm_synchronize", "orctm_build_grid", "orctm_timer_start", "orctm_timer_stop",
    "orctm_set_profiling", "orctm_profile_get", "orctm_kernel_launches", "orctm_device_bytes",
    "orctm_trim_device_memory", "orctm_set_tuning", "orctm_get_tuning",
    "orctm_serve_create", "orctm_serve_submit", "orctm_serve_wait", "orctm_serve_poll",
    "orctm_serve_drain", "orctm_serve_get_stats", "orctm_serve_destroy", "orctm_batch_run",
    "orctm_estimate_device_bytes", "orctm_check_division", "orctm_ocadpo_all",
    "orctm_upload_async", "orctm_download_async", "orctm_set_step_outputs", "orctm_wait_copies",
    "orctm_write_extra", "orctm_write_extra_host", "orctm_read_extra", "orctm_read_extra_host",
    "orctm_set_obc", "orctm_obc_eta", "orctm_obc_uv", "orctm_write_gridinfo",
    "orctm_set_obc_ts", "orctm_obc_ts", "orctm_set_obc_sponge_exp", "orctm_octdiff_noalloc",
    "orctm_set_barotropic", "orctm_troneu", "orctm_ocvtro", "orctm_ocvtot",
    "orctm_download_barotropic", "orctm_ocbarp", "orctm_ocwind", "orctm_trotest",
    "orctm_set_thermo", "orctm_set_coriolis", "orctm_octher", "orctm_ocmodmom", "orctm_occlit",
    "orctm_upload_baroclinic", "orctm_download_baroclinic", "orctm_step_full",
)

PROF_KINDS = ("ocuad", "ocvad", "ocwad", "ocadpo", "octdiff", "ocvisc", "nh_rhs", "pcg_spmv",
              "pcg_col", "resid", "nh_post")

_lib = None


def load(build_if_missing: bool = True):
    """Loads the CUDA library (building it with nvcc first if it is absent)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(SO):
        if not build_if_missing:
            raise RuntimeError(f"{SO} is missing; run orctm_b200/build.py")
        from . import build as _build

        _build.build()
    lib = C.CDLL(SO)
    lib.orctm_status_string.restype = C.c_char_p
    lib.orctm_last_error.restype = C.c_char_p
    lib.orctm_last_error.argtypes = [C.c_void_p]
    lib.orctm_create.argtypes = [C.POINTER(Desc), C.POINTER(C.c_void_p)]
    for name in ("orctm_destroy", "orctm_ocuad", "orctm_ocvad", "orctm_ocwad", "orctm_octdiff",
                 "orctm_octimf", "orctm_ocvisc", "orctm_synchronize", "orctm_ocadpo_all"):
        getattr(lib, name).argtypes = [C.c_void_p]
    lib.orctm_ocadpo.argtypes = [C.c_void_p, C.c_int]
    lib.orctm_ocvtot_nh.argtypes = [C.c_void_p, C.POINTER(SolveStats)]
    lib.orctm_step_hotpath.argtypes = [C.c_void_p, C.POINTER(SolveStats)]
    lib.orctm_set_solver.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_int]
    lib.orctm_field_size.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_size_t)]
    lib.orctm_upload.argtypes = [C.c_void_p, C.c_int, _D, C.c_size_t]
    lib.orctm_download.argtypes = [C.c_void_p, C.c_int, _D, C.c_size_t]
    lib.orctm_upload_async.argtypes = [C.c_void_p, C.c_int, _D, C.c_size_t]
    lib.orctm_download_async.argtypes = [C.c_void_p, C.c_int, _D, C.c_size_t]
    lib.orctm_set_step_outputs.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int),
                                           C.POINTER(_D), C.POINTER(C.c_size_t)]
    lib.orctm_wait_copies.argtypes = [C.c_void_p]
    lib.orctm_write_extra.argtypes = [C.c_void_p, C.c_char_p, C.c_int, C.c_int, C.c_int,
                                      C.POINTER(C.c_int), C.POINTER(C.c_int)]
    lib.orctm_write_extra_host.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_int, C.c_int,
                                           C.POINTER(C.c_int), C.c_int, _D]
    lib.orctm_read_extra.argtypes = [C.c_void_p, C.c_char_p, C.c_int, C.POINTER(C.c_int),
                                     C.POINTER(C.c_int)]
    lib.orctm_read_extra_host.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_int, _D,
                                          C.POINTER(C.c_int)]
    lib.orctm_write_gridinfo.argtypes = [C.c_char_p, C.POINTER(Desc), C.POINTER(GridInfo)]
    lib.orctm_set_obc.argtypes = [C.c_void_p, C.POINTER(Obc)]
    lib.orctm_obc_eta.argtypes = [C.c_void_p, C.c_int]
    lib.orctm_obc_uv.argtypes = [C.c_void_p, C.c_int]
    lib.orctm_set_obc_ts.argtypes = [C.c_void_p, C.c_int, C.POINTER(_D)]
    lib.orctm_obc_ts.argtypes = [C.c_void_p]
    lib.orctm_set_obc_sponge_exp.argtypes = [C.c_void_p, C.c_double]
    lib.orctm_timer_start.argtypes = [C.c_void_p]
    lib.orctm_timer_stop.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
    lib.orctm_set_profiling.argtypes = [C.c_void_p, C.c_int]
    lib.orctm_profile_get.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_longlong),
                                      C.POINTER(C.c_double)]
    lib.orctm_kernel_launches.restype = C.c_ulonglong
    lib.orctm_kernel_launches.argtypes = []
    lib.orctm_device_bytes.argtypes = [C.c_void_p, C.POINTER(C.c_ulonglong)]
    lib.orctm_trim_device_memory.argtypes = [C.c_int]
    lib.orctm_set_tuning.argtypes = [C.c_void_p, C.c_int, C.c_int]
    lib.orctm_check_division.argtypes = [C.c_int, _D, _D, _D, C.c_size_t]
    lib.orctm_get_tuning.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    lib.orctm_octdiff_noalloc.argtypes = [C.POINTER(NoAllocArgs)]
    lib.orctm_set_barotropic.argtypes = [C.c_void_p, C.POINTER(Barotropic)]
    lib.orctm_troneu.argtypes = [C.c_void_p, _D, _D, _D, _D]
    lib.orctm_ocvtro.argtypes = [C.c_void_p]
    lib.orctm_ocvtot.argtypes = [C.c_void_p]
    lib.orctm_download_barotropic.argtypes = [C.c_void_p, C.c_int, _D, C.c_size_t]
    lib.orctm_ocbarp.argtypes = [C.c_void_p]
    lib.orctm_trotest.argtypes = [C.c_void_p, C.c_int, C.c_int, _D]
    lib.orctm_ocwind.argtypes = [C.c_void_p, _D, _D, _D, _D, _D, _D]
    lib.orctm_set_thermo.argtypes = [C.c_void_p, C.POINTER(Thermo)]
    lib.orctm_set_coriolis.argtypes = [C.c_void_p, C.POINTER(Coriolis)]
    lib.orctm_octher.argtypes = [C.c_void_p]
    lib.orctm_ocmodmom.argtypes = [C.c_void_p]
    lib.orctm_occlit.argtypes = [C.c_void_p, _D]
    lib.orctm_upload_baroclinic.argtypes = [C.c_void_p, C.c_int, _D, C.c_size_t]
    lib.orctm_download_baroclinic.argtypes = [C.c_void_p, C.c_int, _D, C.c_size_t]
    lib.orctm_step_full.argtypes = [C.c_void_p, C.c_int, C.POINTER(SolveStats), _D]
    _lib = lib
    return lib


class OrctmError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"ORCTM status {status}: {msg}")
        self.status = status


def check(status: int, handle=None, allow=()):
    if status == ORCTM_OK or status in allow:
        return status
    lib = load()
    detail = lib.orctm_last_error(handle).decode()
    raise OrctmError(status, f"{lib.orctm_status_string(status).decode()} {detail}".strip())
