"""ctypes binding of libagd_b200.so (the C ABI declared in include/agd_b200.h).

The library is the product: there is no fallback.  Loading fails with an
ImportError-like RuntimeError if the shared object is missing or was built for
another ABI version.
"""
import ctypes
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libagd_b200.so")

AGD_STATUS_OK = 0
AGD_STATUS_INVALID = 1
AGD_STATUS_NOT_CONVERGED = 2
AGD_STATUS_CUDA = 4
AGD_STATUS_WATCHDOG = 8
AGD_STATUS_WORKSPACE = 16
AGD_STATUS_UNSUPPORTED = 32

AGD_MODEL_ISOTROPIC = 0
AGD_MODEL_RIEMANN = 1
AGD_MODEL_DIAGONAL = 2
AGD_MODEL_RANDER = 3
AGD_FLAG_ACTIVATE_ALL = 1
AGD_FLAG_SOLVER_AGSI = 2
AGD_FLAG_SOLVER_GLOBAL = 4

_c_int3 = ctypes.c_int * 3
_c_float3 = ctypes.c_float * 3


class AgdInstance(ctypes.Structure):
    _fields_ = [
        ("model", ctypes.c_int), ("ndim", ctypes.c_int), ("shape", _c_int3), ("shape_i", _c_int3),
        ("niter_i", ctypes.c_int), ("fim_front_width", ctypes.c_int), ("nitermax_o", ctypes.c_int),
        ("flags", ctypes.c_int), ("atol", ctypes.c_float), ("rtol", ctypes.c_float),
        ("iso_weights", _c_float3), ("multip_step", ctypes.c_float), ("multip_max", ctypes.c_float),
        ("values", ctypes.c_void_p), ("valuesq", ctypes.c_void_p), ("values_next", ctypes.c_void_p),
        ("valuesq_next", ctypes.c_void_p), ("geom", ctypes.c_void_p),
        ("rhs", ctypes.c_void_p), ("seedbits", ctypes.c_void_p), ("trigger", ctypes.c_void_p),
        ("factor_radius2", ctypes.c_float), ("factor_origin", _c_float3), ("factor_metric", ctypes.c_float * 6),
        ("order2_threshold", ctypes.c_float), ("wall_dist", ctypes.c_void_p), ("release", ctypes.c_void_p),
    ]


class AgdStats(ctypes.Structure):
    _fields_ = [("niter_o", ctypes.c_int32), ("status", ctypes.c_int32), ("tile_visits", ctypes.c_int64)]


class AgdLaunch(ctypes.Structure):
    _fields_ = [("ctas", ctypes.c_int), ("warps_per_cta", ctypes.c_int), ("timeout_ns", ctypes.c_int64)]


class AgdBatchPrep(ctypes.Structure):
    _fields_ = [
        ("model", ctypes.c_int), ("ndim", ctypes.c_int), ("shape", _c_int3), ("shape_i", _c_int3),
        ("n", ctypes.c_int), ("is_dual", ctypes.c_int), ("grid_scales", ctypes.c_double * 3),
        ("metric", ctypes.c_void_p), ("cost", ctypes.c_void_p), ("seed_index", ctypes.c_void_p),
        ("seed_values", ctypes.c_void_p), ("nseeds", ctypes.c_int), ("geom", ctypes.c_void_p),
        ("rhs", ctypes.c_void_p), ("values", ctypes.c_void_p), ("seedbits", ctypes.c_void_p),
        ("bad_seed", ctypes.c_void_p), ("walls", ctypes.c_void_p), ("walls_shared", ctypes.c_int),
        ("trigger", ctypes.c_void_p),
    ]


class AgdConvSrc(ctypes.Structure):
    _fields_ = [("data", ctypes.c_void_p), ("channels", ctypes.c_int), ("up", ctypes.c_int)]


class AgdConv(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int), ("H", ctypes.c_int), ("W", ctypes.c_int), ("src", AgdConvSrc * 2),
                ("cout", ctypes.c_int)]


class AgdWsTerm(ctypes.Structure):
    _fields_ = [("data", ctypes.c_void_p), ("mode", ctypes.c_int), ("channels", ctypes.c_int),
                ("offset", ctypes.c_int)]


# Every exported symbol, with its ctypes signature.
_P = ctypes.c_void_p
_I = ctypes.c_int
SIGNATURES = {
    "agd_plan_create": (_I, [_P, _I, _P]),
    "agd_plan_destroy": (None, [_P]),
    "agd_plan_workspace_bytes": (ctypes.c_size_t, [_P]),
    "agd_plan_upload": (_I, [_P, _P, ctypes.c_size_t, _P]),
    "agd_plan_run": (_I, [_P, _P, ctypes.c_size_t, _P, _P, _P]),
    "agd_eikonal_workspace_bytes": (ctypes.c_size_t, [_P, _I]),
    "agd_eikonal_solve": (_I, [_P, _I, _P, ctypes.c_size_t, _P, _P, _P]),
    "agd_eikonal_solve_fixed_scratch": (_I, [_P, _I, _P, _P, _P]),
    "agd_prep_geom": (_I, [_I, _P, _P, _P, _I, _I, _P, _P, _P]),
    "agd_prep_geom_diagonal": (_I, [_I, _P, _P, _P, _I, _I, _P, _P, _P]),
    "agd_prep_geom_rander": (_I, [_I, _P, _P, _P, _I, _I, _P, _P, _P]),
    "agd_block_expand": (_I, [_I, _P, _P, _I, _P, _I, ctypes.c_float, _P, _P]),
    "agd_block_squeeze": (_I, [_I, _P, _P, _I, _P, _P, _P]),
    "agd_prep_seeds": (_I, [_I, _P, _P, _P, _P, _I, _P, _P, _P, _P]),
    "agd_prep_batch": (_I, [_P, _P]),
    "agd_prep_walls": (_I, [_I, _P, _P, _P, _I, _P, _P, _P, _P, _P]),
    "agd_prep_walls_batch": (_I, [_I, _P, _P, _I, _P, _I, _P, _P, _P]),
    "agd_selling": (_I, [_I, _P, _I, _P, _P, _P]),
    "agd_voronoi_decomposition": (_I, [_I, _P, ctypes.c_longlong, _P, _P, _I, _P]),
    "agd_flow": (_I, [_P, _P, _P, _P, _P, _P]),
    "agd_eucl_map": (_I, [_I, _P, _P, _I, _I, _P, _P, _P]),
    "agd_geodesics": (_I, [_P, _P, _P, _P, _P, _I, ctypes.c_float, ctypes.c_float, _I, _I, _I, _I, _I, _P, _I,
                           _P, _P, _P]),
    "agd_reverse_workspace_bytes": (ctypes.c_size_t, [_P]),
    "agd_reverse": (_I, [_P, _P, _P, _P, _P, _P, ctypes.c_float, ctypes.c_float, _P, ctypes.c_size_t, _P, _P,
                         _P]),
    "agd_forward": (_I, [_P, _P, _P, _P, _P, _P, ctypes.c_float, ctypes.c_float, _P, ctypes.c_size_t, _P, _P,
                         _P]),
    # the learned warm start (include/agd_warmstart.h)
    "agd_conv_kpad": (_I, [_I]),
    "agd_conv3x3_forward": (_I, [_P, _P, _P, _I, _P, _P, _P, _P]),
    "agd_conv3x3_weight_grad": (_I, [_P, _P, _P, _P, _P]),
    "agd_conv_weight_flip": (_I, [_I, _I, _P, _P, _P]),
    "agd_ws_features": (_I, [_P, _P, _I, _I, _I, _I, ctypes.c_float, _P, _P, _P]),
    "agd_ws_target": (_I, [_P, _I, _I, _I, _P, _P, _P]),
    "agd_ws_avgpool": (_I, [_P, _I, _I, _I, _I, _P, _P]),
    "agd_ws_upsample": (_I, [_P, _I, _I, _I, _I, _P, _P]),
    "agd_ws_route": (_I, [_I, _I, _I, _I, _P, AgdWsTerm, AgdWsTerm, _P, _P]),
    "agd_ws_bias_grad": (_I, [_P, ctypes.c_longlong, _I, _P, _P]),
    "agd_ws_head_forward": (_I, [_P, ctypes.c_longlong, _P, _P, _P, _P]),
    "agd_ws_head_loss_backward": (_I, [_P, ctypes.c_longlong, _P, _P, _P, ctypes.c_longlong, _P, _P, _P, _P, _P]),
    "agd_ws_adam": (_I, [_P, _P, _P, _P, ctypes.c_longlong, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                         ctypes.c_float, _I, _P, _P]),
    "agd_ws_release": (_I, [_P, _I, _I, _I, ctypes.c_float, _I, _P, _P]),
    "agd_ws_warm_values": (_I, [_P, _I, _I, _I, ctypes.c_float, _P, _P]),
    "agd_last_error": (ctypes.c_char_p, []),
    "agd_version": (_I, []),
}

_lock = threading.Lock()
_lib = None


class AgdError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"agd_b200 error {status}: {msg}")
        self.status = status


def lib():
    """The loaded library (built on first use if absent and nvcc is available)."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                try:
                    from . import build as _build
                    _build.build()
                except Exception as exc:  # noqa: BLE001
                    raise RuntimeError(f"libagd_b200.so is missing and could not be built: {exc}") from exc
            L = ctypes.CDLL(LIB_PATH)
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(L, name)
                fn.restype = res
                fn.argtypes = args
            if L.agd_version() != 4:
                raise RuntimeError("libagd_b200.so has an unexpected ABI version")
            _lib = L
    return _lib


def check(status, what=""):
    if status != AGD_STATUS_OK:
        msg = lib().agd_last_error().decode(errors="replace")
        raise AgdError(status, f"{what}: {msg}" if what else msg)
    return status


def ptr(t):
    """Device pointer of a torch tensor (None -> NULL)."""
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def stream_ptr(stream=None):
    import torch
    s = torch.cuda.current_stream() if stream is None else stream
    return ctypes.c_void_p(s.cuda_stream)
