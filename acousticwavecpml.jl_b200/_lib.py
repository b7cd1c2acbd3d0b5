"""ctypes binding of libawcpml.so (the C ABI in include/awcpml.h).

The library is built in-tree (``lib/libawcpml.so``, see build.py). There is no
fallback: if the shared object is missing or fails to load, every entry point
of this package raises.
"""
import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libawcpml.so")

AWC_OK = 0
AWC_ERR_INVALID = -1
AWC_ERR_OOM = -2
AWC_ERR_CUDA = -3
AWC_ERR_TIMEOUT = -4
AWC_ERR_NODEVICE = -5
AWC_F32 = 1
AWC_F64 = 2

_ERRNAMES = {
    AWC_ERR_INVALID: "invalid argument",
    AWC_ERR_OOM: "out of device memory",
    AWC_ERR_CUDA: "CUDA error",
    AWC_ERR_TIMEOUT: "device wait timed out",
    AWC_ERR_NODEVICE: "no usable device",
}


class Problem(ctypes.Structure):
    """`awc_problem` of include/awcpml.h."""

    _fields_ = [
        ("ndim", ctypes.c_int32),
        ("precision", ctypes.c_int32),
        ("nx", ctypes.c_int64),
        ("ny", ctypes.c_int64),
        ("nz", ctypes.c_int64),
        ("halo", ctypes.c_int32),
        ("freetop", ctypes.c_int32),
        ("dx", ctypes.c_double),
        ("dy", ctypes.c_double),
        ("dz", ctypes.c_double),
        ("dt", ctypes.c_double),
        ("nt", ctypes.c_int64),
        ("nsrc", ctypes.c_int64),
        ("nrec", ctypes.c_int64),
    ]


class Shot(ctypes.Structure):
    """`awc_shot` of include/awcpml.h."""

    _fields_ = [
        ("model", ctypes.c_int32),
        ("nsrc", ctypes.c_int32),
        ("nrec", ctypes.c_int32),
        ("coeffs", ctypes.c_void_p),
        ("possrcs", ctypes.c_void_p),
        ("dt2srctf", ctypes.c_void_p),
        ("posrecs", ctypes.c_void_p),
    ]


class AwcError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{_ERRNAMES.get(code, 'error')} ({code}): {msg}")
        self.code = code


class AwcInvalidArgument(AwcError, ValueError):
    pass


_dp = ctypes.POINTER(ctypes.c_double)
_i64p = ctypes.POINTER(ctypes.c_int64)
_vp = ctypes.c_void_p
_PP = ctypes.POINTER(Problem)

# name -> (restype, argtypes); every function declared in include/awcpml.h
SIGNATURES = {
    "awc_coeffs_len": (ctypes.c_int64, [_PP]),
    "awc_cpml_coeffs": (ctypes.c_int, [ctypes.c_int32, ctypes.c_double, ctypes.c_double,
                                       ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                       ctypes.c_int32, _dp, _dp, _dp, _dp]),
    "awc_problem_coeffs": (ctypes.c_int, [_PP, ctypes.c_double, ctypes.c_double,
                                          ctypes.c_double, _dp]),
    "awc_ricker": (ctypes.c_int, [ctypes.c_int64, _dp, ctypes.c_double, ctypes.c_double, _dp]),
    "awc_create": (ctypes.c_int, [ctypes.POINTER(_vp), ctypes.c_int32]),
    "awc_destroy": (None, [_vp]),
    "awc_last_error": (ctypes.c_char_p, [_vp]),
    "awc_last_run_ms": (ctypes.c_float, [_vp]),
    "awc_ctx_stream": (ctypes.c_void_p, [_vp]),
    "awc_ctx_set_autotune": (ctypes.c_int, [_vp, ctypes.c_int64]),
    "awc_forward": (ctypes.c_int, [_vp, _PP, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "awc_plan_create": (ctypes.c_int, [_vp, _PP, _vp, _vp, _vp, _vp, _vp, ctypes.POINTER(_vp)]),
    "awc_plan_destroy": (None, [_vp]),
    "awc_plan_reset": (ctypes.c_int, [_vp]),
    "awc_plan_run": (ctypes.c_int, [_vp, ctypes.c_int64, ctypes.c_int32,
                                    ctypes.POINTER(ctypes.c_float)]),
    "awc_plan_step": (ctypes.c_int64, [_vp]),
    "awc_plan_traces": (ctypes.c_int, [_vp, _vp]),
    "awc_plan_field": (ctypes.c_int, [_vp, _vp]),
    "awc_plan_launches_per_step": (ctypes.c_int32, [_vp]),
    "awc_plan_set_launch": (ctypes.c_int, [_vp, ctypes.c_int32, ctypes.c_int32,
                                           ctypes.c_int32]),
    "awc_plan_get_launch": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_int32),
                                           ctypes.POINTER(ctypes.c_int32),
                                           ctypes.POINTER(ctypes.c_int32)]),
    "awc_plan_autotune": (ctypes.c_int, [_vp, ctypes.c_int64, ctypes.POINTER(ctypes.c_float)]),
    "awc_plan_set_blocking": (ctypes.c_int, [_vp, ctypes.c_int32, ctypes.c_int32,
                                             ctypes.c_int32]),
    "awc_plan_get_blocking": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_int32),
                                             ctypes.POINTER(ctypes.c_int32),
                                             ctypes.POINTER(ctypes.c_int32)]),
    "awc_plan_launch_count": (ctypes.c_int64, [_vp, ctypes.c_int64]),
    "awc_forward_decomposed": (ctypes.c_int, [ctypes.POINTER(_vp), ctypes.c_int32, _PP, _vp, _vp,
                                              _vp, _vp, _vp, _vp, _vp]),
    "awc_plan_run_snapshots": (ctypes.c_int, [_vp, ctypes.c_int64, ctypes.c_int64, _vp,
                                              ctypes.c_int64, ctypes.POINTER(ctypes.c_int64)]),
    "awc_plan_set_wait": (ctypes.c_int, [_vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32]),
    "awc_misfit_gradient": (ctypes.c_int, [_vp, _PP, _vp, _vp, _vp, _vp, _vp, _vp, ctypes.c_int32,
                                           _vp, _vp, _vp]),
    "awc_misfit_gradient_shots": (ctypes.c_int, [_vp, _PP, ctypes.c_int32, _vp, _vp, _vp, _vp,
                                                 _vp, _vp, ctypes.c_int32, _vp, _vp]),
    "awc_adjoint_sources": (ctypes.c_int, [_vp, _PP, _vp, _vp, _vp, _vp, _vp, _vp]),
    "awc_learned_weights_len": (ctypes.c_int, [ctypes.c_int32]),
    "awc_forward_learned": (ctypes.c_int, [_vp, _PP, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "awc_forward2d_f32_static": (ctypes.c_int, [_PP, _vp, _vp, _vp, _vp, _vp, _vp, _vp]),
    "awc_batch_create": (ctypes.c_int, [_vp, ctypes.c_int32, _PP, _vp, ctypes.c_int32, _vp,
                                        ctypes.POINTER(_vp)]),
    "awc_batch_destroy": (None, [_vp]),
    "awc_batch_reset": (ctypes.c_int, [_vp]),
    "awc_batch_run": (ctypes.c_int, [_vp, ctypes.c_int64, ctypes.c_int32,
                                     ctypes.POINTER(ctypes.c_float)]),
    "awc_batch_step": (ctypes.c_int64, [_vp]),
    "awc_batch_traces": (ctypes.c_int, [_vp, ctypes.c_int32, _vp]),
    "awc_batch_field": (ctypes.c_int, [_vp, ctypes.c_int32, _vp]),
    "awc_batch_set_launch": (ctypes.c_int, [_vp, ctypes.c_int32, ctypes.c_int32]),
    "awc_batch_get_launch": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_int32),
                                            ctypes.POINTER(ctypes.c_int32)]),
    "awc_batch_autotune": (ctypes.c_int, [_vp, ctypes.c_int64, ctypes.POINTER(ctypes.c_float)]),
    "awc_forward_batch": (ctypes.c_int, [_vp, ctypes.c_int32, _PP, _vp, ctypes.c_int32, _vp,
                                         _vp]),
}

_LIB = None


def lib():
    """Loads the in-tree shared library (raises if it is missing)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python -c 'import __graft_entry__ as g; "
                "g.build()'` (nvcc, sm_100a). There is no CPU fallback.")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = L
    return _LIB


def check(rc, ctx=None):
    """Raises AwcError/AwcInvalidArgument for a non-zero status."""
    if rc != AWC_OK:
        msg = lib().awc_last_error(ctx)
        msg = msg.decode() if msg else ""
        cls = AwcInvalidArgument if rc == AWC_ERR_INVALID else AwcError
        raise cls(rc, msg)
    return rc
