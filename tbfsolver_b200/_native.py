"""ctypes binding of ``libtbfp.so`` (the C ABI declared in ``include/tbfp.h``).

The shared library is built in-tree (``tbfsolver_b200/lib/libtbfp.so``) by
``tbfsolver_b200.build``.  There is no fallback: if the library is missing or
fails to load, every entry point raises ``TbfpError``.
"""
from __future__ import annotations

import ctypes as C
import os

LIB_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib")
LIB_PATH = os.path.join(LIB_DIR, "libtbfp.so")

# status codes (tbfp.h)
TBFP_OK = 0
TBFP_ENOTCONVERGED = 1
TBFP_EINVAL = -1
TBFP_ENULL = -2
TBFP_ECUDA = -3
TBFP_ENOMEM = -4
TBFP_EUNSUPPORTED = -5
TBFP_ENODEVICE = -6
TBFP_ENONFINITE = -7
TBFP_ESINGULAR = -8
TBFP_ETIMEOUT = -9
TBFP_ENS_AUTO = 0
TBFP_ENS_GRAPH = 1
TBFP_ENS_PERSISTENT = 2

TBFP_FP64 = 0
TBFP_MIXED = 1
TBFP_FLAG_ASYNC = 1
TBFP_FLAG_TIMING = 2
TBFP_FLAG_RESIDUAL = 4
STAGES = ("recip", "rhs_fftx", "fftz_fwd", "tridiag", "fftz_inv", "fftx_inv", "correct", "div")


class TbfpError(RuntimeError):
    """A hard error (< 0) returned by the library, or a missing library."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"tbfp error {code}: {msg}")
        self.code = code


class TbfpDesc(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("hd_psi", C.c_int), ("hd_u", C.c_int), ("hd_rho", C.c_int), ("hd_st", C.c_int),
        ("dx_fft", C.c_double), ("dz_fft", C.c_double),
        ("dxf", C.POINTER(C.c_double)), ("dxc", C.POINTER(C.c_double)),
        ("dyf", C.POINTER(C.c_double)), ("dyc", C.POINTER(C.c_double)),
        ("dzf", C.POINTER(C.c_double)), ("dzc", C.POINTER(C.c_double)),
        ("s_Vg", C.c_double),
        ("precision", C.c_int), ("tol", C.c_double), ("max_iter", C.c_int),
        ("device", C.c_int), ("stream", C.c_void_p), ("flags", C.c_uint),
    ]


class TbfpMgParams(C.Structure):
    _fields_ = [("n_levels", C.c_int), ("n_pre", C.c_int), ("n_post", C.c_int), ("tol_mg", C.c_double),
                ("max_iter_mg", C.c_int), ("tol_pcg", C.c_double), ("max_iter_pcg", C.c_int)]


class TbfpVofDesc(C.Structure):
    _fields_ = [("xc", C.c_void_p), ("yc", C.c_void_p), ("zc", C.c_void_p), ("xf", C.c_void_p), ("yf", C.c_void_p),
                ("zf", C.c_void_p), ("rhol", C.c_double), ("rhog", C.c_double), ("mul", C.c_double),
                ("mug", C.c_double)]


class TbfpMomentumDesc(C.Structure):
    _fields_ = [("scheme", C.c_int), ("gch", C.c_double), ("g", C.c_double)] + [
        (n, C.c_void_p) for n in ("dxf", "dxc", "dyf", "dyc", "dzf", "dzc", "yc", "yf")] + [
        ("ubot", C.c_double * 3), ("utop", C.c_double * 3)]


class TbfpMemberIO(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in ("ux_in", "uy_in", "uz_in", "ux_out", "uy_out", "uz_out", "rho", "psi_n",
                                           "psi_nm1", "psi")]


class TbfpStats(C.Structure):
    _fields_ = [
        ("iterations", C.c_int),
        ("rel_residual", C.c_double),
        ("max_div", C.c_double),
        ("cont_err", C.c_double),
        ("ms_device", C.c_double),
        ("ms_stage", C.c_double * 8),
    ]


_P = C.c_void_p  # every array argument is passed as a raw address
_PP = C.c_void_p  # const double *const * (address of a 3-pointer array) or NULL
_D = C.c_double
_H = C.c_void_p

# name -> (restype, argtypes); the set of exported symbols is checked against
# include/tbfp.h by the test suite.
PROTOTYPES = {
    "tbfp_abi_version": (C.c_int, []),
    "tbfp_strerror": (C.c_char_p, [C.c_int]),
    "tbfp_last_error": (C.c_char_p, [_H]),
    "tbfp_create": (C.c_int, [C.POINTER(TbfpDesc), C.POINTER(_H)]),
    "tbfp_destroy": (C.c_int, [_H]),
    "tbfp_device_bytes": (C.c_size_t, [_H]),
    "tbfp_get_stats": (C.c_int, [_H, C.POINTER(TbfpStats)]),
    "tbfp_slab_create": (C.c_int, [C.POINTER(TbfpDesc), C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    "tbfp_slab_forward_x": (C.c_int, [_H, _P, _P]),
    "tbfp_slab_spectral": (C.c_int, [_H, _P]),
    "tbfp_slab_inverse_x": (C.c_int, [_H, _P, _P]),
    "tbfp_slab_unpack_kx": (C.c_int, [_H, C.c_int, C.POINTER(C.c_int), _P, _P]),
    "tbfp_slab_pack_z": (C.c_int, [_H, C.c_int, C.POINTER(C.c_int), _P, _P]),
    "tbfp_ensemble_create": (C.c_int, [C.c_int, C.POINTER(TbfpDesc), C.c_int, C.POINTER(C.c_void_p)]),
    "tbfp_ensemble_destroy": (C.c_int, [_H]),
    "tbfp_ensemble_size": (C.c_int, [_H]),
    "tbfp_ensemble_set_mode": (C.c_int, [_H, C.c_int, C.c_int]),
    "tbfp_ensemble_get_mode": (C.c_int, [_H, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_float)]),
    "tbfp_ensemble_set_wait_limit": (C.c_int, [_H, C.c_longlong]),
    "tbfp_set_wait_limit": (C.c_int, [_H, C.c_longlong]),
    "tbfp_ensemble_projection_dev": (C.c_int, [_H, C.POINTER(TbfpMemberIO), C.c_double, C.c_double, C.c_double,
                                               C.POINTER(TbfpStats)]),
    "tbfp_pcg_setup": (C.c_int, [_H, C.POINTER(TbfpMgParams)]),
    "tbfp_vof_setup": (C.c_int, [_H, C.POINTER(TbfpVofDesc)]),
    "tbfp_momentum_setup": (C.c_int, [_H, C.POINTER(TbfpMomentumDesc)]),
    "tbfp_momentum_fluxes": (C.c_int, [_H, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]),
    "tbfp_momentum_predictor": (C.c_int, [_H] + [C.c_void_p] * 7 + [C.c_double] * 6),
    "tbfp_momentum_predictor_dev": (C.c_int, [_H] + [C.c_void_p] * 7 + [C.c_double] * 6),
    "tbfp_momentum_predictor_out_dev": (C.c_int, [_H] + [C.c_void_p] * 10 + [C.c_double] * 6),
    "tbfp_material_props_pass_dev": (C.c_int, [_H, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "tbfp_update_boundaries_v": (C.c_int, [_H, C.c_void_p, C.c_void_p, C.c_void_p]),
    "tbfp_rho_face_sum": (C.c_int, [_H, C.c_void_p, C.POINTER(C.c_double)]),
    "tbfp_rho_face_sum_dev": (C.c_int, [_H, C.c_void_p, C.POINTER(C.c_double)]),
    "tbfp_flow_rate": (C.c_int, [_H, C.c_void_p, C.POINTER(C.c_double)]),
    "tbfp_flow_rate_dev": (C.c_int, [_H, C.c_void_p, C.POINTER(C.c_double)]),
    "tbfp_add_ux": (C.c_int, [_H, C.c_void_p, C.c_double]),
    "tbfp_add_ux_dev": (C.c_int, [_H, C.c_void_p, C.c_double]),
    "tbfp_update_boundaries_v_dev": (C.c_int, [_H, C.c_void_p, C.c_void_p, C.c_void_p]),
    "tbfp_material_props": (C.c_int, [_H, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "tbfp_material_props_dev": (C.c_int, [_H, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
    "tbfp_pcg_solve": (C.c_int, [_H, _P, _P, _P, C.POINTER(TbfpStats)]),
    "tbfp_pcg_solve_dev": (C.c_int, [_H, _P, _P, _P, C.POINTER(TbfpStats)]),
    "tbfp_projection_mg": (C.c_int, [_H, _P, _P, _P, _P, C.c_double, C.c_double, _P, C.POINTER(TbfpStats)]),
    "tbfp_projection_mg_dev": (C.c_int, [_H, _P, _P, _P, _P, _P, _P, _P, C.c_double, C.c_double, _P,
                                         C.POINTER(TbfpStats)]),
    "tbfp_solve_fps": (C.c_int, [_H, _P, _P]),
    "tbfp_solve_fps_dev": (C.c_int, [_H, _P, _P]),
    "tbfp_rhs_split": (C.c_int, [_H, _P, _P, _P, _P, _P, _P, _PP, _PP, _D, _D, _D, _P]),
    "tbfp_rhs_split_dev": (C.c_int, [_H, _P, _P, _P, _P, _P, _P, _PP, _PP, _D, _D, _D, _P]),
    "tbfp_correct": (C.c_int, [_H, _P, _P, _P, _P, _P, _P, _P, _PP, _PP, _D, _D, _D]),
    "tbfp_correct_dev": (C.c_int, [_H, _P, _P, _P, _P, _P, _P, _P, _PP, _PP, _D, _D, _D]),
    "tbfp_continuity_error": (C.c_int, [_H, _P, _P, _P, _D, C.POINTER(_D), C.POINTER(_D)]),
    "tbfp_continuity_error_dev": (C.c_int, [_H, _P, _P, _P, _D, C.POINTER(_D), C.POINTER(_D)]),
    "tbfp_projection": (C.c_int, [_H, _P, _P, _P, _P, _P, _P, _PP, _PP, _D, _D, _D, _P, C.POINTER(TbfpStats)]),
    "tbfp_projection_dev": (C.c_int, [_H, _P, _P, _P, _P, _P, _P, _P, _P, _P, _PP, _PP, _D, _D, _D, _P,
                                      C.POINTER(TbfpStats)]),
    "tbfp_solve_fps_noalloc": (C.c_int, [C.POINTER(TbfpDesc), _P, _P]),
    "tbfp_surface_tension": (C.c_int, [_H, _P, C.c_double, _P, _P, _P, _P]),
    "tbfp_surface_tension_dev": (C.c_int, [_H, _P, C.c_double, _P, _P, _P, _P]),
}

_lib = None


def load(path: str | None = None):
    """Load (once) and return the library with its prototypes set."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise TbfpError(TBFP_ENODEVICE, f"{p} not found: build it with `python -m tbfsolver_b200.build`")
    try:
        lib = C.CDLL(p)
    except OSError as e:  # pragma: no cover - depends on the environment
        raise TbfpError(TBFP_ENODEVICE, f"cannot load {p}: {e}") from e
    for name, (res, args) in PROTOTYPES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def check(rc: int, handle=None) -> int:
    """Raise TbfpError for hard errors; return soft status codes (>= 0)."""
    if rc < 0:
        lib = load()
        detail = lib.tbfp_last_error(handle)
        detail = detail.decode() if detail else ""
        raise TbfpError(rc, f"{lib.tbfp_strerror(rc).decode()}: {detail}")
    return rc
