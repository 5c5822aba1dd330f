"""ctypes binding of libpf5d.so, the sm_100a CUDA step library (include/pf5d.h).

There is no CPU fallback: importing a GPU entry point without the built
library or without a CUDA device raises immediately.  Build the library with
``python -c "import __graft_entry__ as g; g.build()"`` (or ``make -C
phasefield5d_b200/csrc``).
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libpf5d.so")

PF5D_OK = 0
PF5D_ERR_ARG = 1
PF5D_ERR_DIM = 2
PF5D_ERR_CUDA = 3
PF5D_ERR_CUFFT = 4
PF5D_ERR_NN_DISTANCE = 5
PF5D_ERR_OOB = 6
PF5D_ERR_CAPACITY = 7

FLAG_NONFINITE = 0x01
FLAG_OOB_HARD = 0x02
FLAG_OOB_SOFT = 0x04
FLAG_NN_FAR = 0x08
FLAG_NN_TRUNCATED = 0x10
FLAG_NN_USED = 0x20
FLAG_HALTED = 0x40
FLAG_NN_NONFINITE = 0x80

STAGE_RATE, STAGE_UPDATE, STAGE_FFT_FWD, STAGE_BMUL, STAGE_FFT_INV = 0, 1, 2, 3, 4
PRECISION_FP64, PRECISION_FP32C = 0, 1

_vp = ctypes.c_void_p
_i32 = ctypes.c_int32
_i64 = ctypes.c_int64
_f64 = ctypes.c_double
_i64p = ctypes.POINTER(ctypes.c_int64)
_f64p = ctypes.POINTER(ctypes.c_double)


class StepperDesc(ctypes.Structure):
    """pf5d_stepper_desc (include/pf5d.h)."""
    _fields_ = [
        ("dim", _i32), ("shape", _i64 * 3), ("dx", _f64), ("kappa", _f64 * 4),
        ("x0", _f64 * 4), ("elastic", _i32), ("lvec", _f64 * 4), ("bk", _f64p),
        ("grid", _vp), ("table_n", _i32), ("nprops", _i32), ("node_stride", _i32),
        ("resolution", _f64), ("node_coord", _vp), ("max_nn_dist", _f64),
        ("ctld", _f64), ("t_cfl", _f64), ("lower_limit", _f64), ("upper_limit", _f64),
        ("max_change_factor", _f64), ("adaptive", _i32), ("dt0", _f64),
        ("oob_interval", _i32), ("precision", _i32), ("grid32", _vp), ("node_stride32", _i32),
        ("mu0", _f64 * 4),
    ]


class BatchSolve(ctypes.Structure):
    """pf5d_batch_solve (include/pf5d.h)."""
    _fields_ = [
        ("dim", _i32), ("shape", _i64 * 2), ("dx", _f64), ("kappa", _f64 * 4), ("x0", _f64 * 4),
        ("elastic", _i32), ("lvec", _f64 * 4), ("bk", _f64p), ("table", _i32),
        ("max_nn_dist", _f64), ("ctld", _f64), ("t_cfl", _f64), ("lower_limit", _f64),
        ("upper_limit", _f64), ("max_change_factor", _f64), ("adaptive", _i32), ("dt0", _f64),
        ("oob_interval", _i32), ("X", _vp), ("hi", _vp), ("lo", _vp), ("time0", _f64),
        ("step0", _i64),
    ]


class StepState(ctypes.Structure):
    """pf5d_step_state (include/pf5d.h)."""
    _fields_ = [("dt", _f64), ("time", _f64), ("xdotmax", _f64), ("step", _i64),
                ("flags", ctypes.c_uint32), ("halted", ctypes.c_uint32)]


class SaveDiag(ctypes.Structure):
    """pf5d_save_diag (include/pf5d.h)."""
    _fields_ = [("net", _f64 * 4), ("max_change", _f64 * 4), ("total_flux", _f64 * 4),
                ("mass", _f64 * 4), ("comp_min", _f64 * 4), ("comp_max", _f64 * 4),
                ("comp_fe_min", _f64), ("comp_var", _f64 * 4), ("f_grad", _f64),
                ("xdotmax", _f64), ("dt", _f64), ("time", _f64), ("step", _i64),
                ("halted", _i32), ("pad", _i32)]


_SIGS = {
    "pf5d_last_error": (ctypes.c_char_p, []),
    "pf5d_version": (_i32, []),
    "pf5d_interp4d": (_i32, [_vp, _i64, _vp, _i32, _i32, _i32, _f64, _vp, _f64, _vp, _i64, _vp,
                             _vp, _vp]),
    "pf5d_laplacian": (_i32, [_i32, _i64p, _i32, _vp, _f64, _vp, _vp]),
    "pf5d_kappa_subtract": (_i32, [_vp, _i64, _vp, _f64p, _i64, _i32, _vp]),
    "pf5d_divergence_from_mu": (_i32, [_i32, _i64p, _i32, _vp, _vp, _i64, _vp, _i64, _f64, _vp,
                                       _vp]),
    "pf5d_gradients_pm": (_i32, [_i32, _i64p, _i32, _vp, _i64, _f64, _vp, _vp, _vp]),
    "pf5d_fluxes_pm": (_i32, [_i32, _i64p, _i32, _vp, _vp, _i64, _vp, _vp, _vp, _vp, _vp]),
    "pf5d_elastic_create": (_i32, [_i32, _i64p, _f64p, _f64p, _f64p, ctypes.POINTER(_vp)]),
    "pf5d_elastic_apply": (_i32, [_vp, _vp, _i64, _vp, _vp]),
    "pf5d_elastic_destroy": (_i32, [_vp]),
    "pf5d_abs_max": (_i32, [_vp, _i64, _vp, _vp]),
    "pf5d_abs_max_noalloc": (_i32, [_vp, _i64, _vp, _vp]),
    "pf5d_clamp_simplex": (_i32, [_vp, _i64, _i32, _vp]),
    "pf5d_update": (_i32, [_vp, _vp, _i64, _f64, _vp]),
    "pf5d_oob_stats": (_i32, [_vp, _i64, _i32, _f64p, _vp]),
    "pf5d_adaptive_dt": (_f64, [_f64, _f64, _f64, _f64, _f64, _f64, _f64]),
    "pf5d_stepper_create": (_i32, [ctypes.POINTER(StepperDesc), _vp, _vp, ctypes.POINTER(_vp)]),
    "pf5d_stepper_advance": (_i32, [_vp, _i64, _vp]),
    "pf5d_stepper_state": (_i32, [_vp, ctypes.POINTER(StepState), _vp]),
    "pf5d_stepper_rate": (_vp, [_vp]),
    "pf5d_stepper_field": (_i32, [_vp, _vp, _vp]),
    "pf5d_stepper_mass": (_i32, [_vp, _f64p, _vp]),
    "pf5d_stepper_launch_stage": (_i32, [_vp, _i32, _vp]),
    "pf5d_stepper_autotune": (_i32, [_vp, ctypes.POINTER(_i32), ctypes.POINTER(ctypes.c_float),
                                     _vp]),
    "pf5d_stepper_set_variant": (_i32, [_vp, _i32]),
    "pf5d_stepper_variant_count": (_i32, [_vp]),
    "pf5d_stepper_launches_per_step": (_i32, [_vp]),
    "pf5d_stepper_rate_kernels": (ctypes.c_char_p, [_vp]),
    "pf5d_stepper_step_save": (_i32, [_vp, ctypes.POINTER(SaveDiag), _vp]),
    "pf5d_batch_variant_count": (_i32, []),
    "pf5d_stepper_reset": (_i32, [_vp, _f64, _f64, _vp]),
    "pf5d_stepper_destroy": (_i32, [_vp]),
    "pf5d_batch_create": (_i32, [ctypes.POINTER(BatchSolve), _i32, ctypes.POINTER(_vp), _i32,
                                 _i32, _f64, _vp, _vp, ctypes.POINTER(_vp)]),
    "pf5d_batch_advance": (_i32, [_vp, _i64, _vp]),
    "pf5d_batch_states": (_i32, [_vp, ctypes.POINTER(StepState), _vp]),
    "pf5d_batch_field": (_i32, [_vp, _i32, _vp, _vp]),
    "pf5d_batch_export": (_i32, [_vp, _i32, _vp, _vp, _vp]),
    "pf5d_batch_autotune": (_i32, [_vp, ctypes.POINTER(_i32), ctypes.POINTER(ctypes.c_float),
                                   _vp]),
    "pf5d_batch_set_variant": (_i32, [_vp, _i32]),
    "pf5d_batch_destroy": (_i32, [_vp]),
}

_lib = None


def exported_symbols():
    """Names the C ABI header declares (and the library must export)."""
    return list(_SIGS)


def load(require_cuda=True):
    """Load libpf5d.so; raises if it is missing or (by default) CUDA is absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"CUDA library {LIB_PATH} is not built; run "
                           "`python -c \"import __graft_entry__ as g; g.build()\"`")
    if require_cuda:
        import torch
        if not torch.cuda.is_available():
            raise RuntimeError("phasefield5d_b200 needs a CUDA device; there is no CPU fallback")
        torch.cuda.init()
    L = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in _SIGS.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def last_error():
    return (load(require_cuda=False).pf5d_last_error() or b"").decode()


def check(status, what=""):
    """Map a pf5d_status to the reference's exception types."""
    if status == PF5D_OK:
        return
    msg = f"{what}: {last_error()}" if what else last_error()
    if status == PF5D_ERR_ARG:
        raise ValueError(msg)
    if status == PF5D_ERR_DIM:
        raise ValueError(msg)
    if status == PF5D_ERR_NN_DISTANCE:
        raise RuntimeError(NN_FAR_MSG)
    raise RuntimeError(f"pf5d error {status}: {msg}")


NN_NONFINITE_MSG = "'x' must be finite, check for nan or inf values"
NN_FAR_MSG = "Some compositions are outside the CALPHAD domain (KD-tree)."


def nn_flags(flags):
    """Decode the nearest-row fallback bits of a device status word."""
    return {"nn_used": bool(flags & FLAG_NN_USED), "nn_far": bool(flags & FLAG_NN_FAR),
            "nn_nonfinite": bool(flags & FLAG_NN_NONFINITE),
            "nn_no_row": bool(flags & FLAG_NN_TRUNCATED)}


def raise_nn_errors(flags, check_far=True):
    """Raise where the reference's fallback raises: ValueError for a
    non-finite composition (cKDTree.query), RuntimeError for a row farther
    than max_nn_dist (interpolation.py:207-208) or a table without rows."""
    if flags & FLAG_NN_NONFINITE:
        raise ValueError(NN_NONFINITE_MSG)
    if check_far and flags & FLAG_NN_FAR:
        raise RuntimeError(NN_FAR_MSG)
    if flags & FLAG_NN_TRUNCATED:
        raise RuntimeError("nearest-row fallback: the table has no rows")


def stream_handle(stream=None):
    """cudaStream_t of ``stream`` (default: torch's current stream) as void*."""
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else ctypes.c_void_p(0)


def shape_arg(shape):
    arr = (ctypes.c_int64 * 3)(*(list(shape) + [1] * (3 - len(shape))))
    return ctypes.cast(arr, _i64p), arr


def f64_array(vals):
    vals = [float(v) for v in vals]
    arr = (ctypes.c_double * len(vals))(*vals)
    return ctypes.cast(arr, _f64p), arr
