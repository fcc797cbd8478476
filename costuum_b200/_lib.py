"""ctypes binding of libtmx.so (the CUDA library built from costuum_b200/csrc).

There is no CPU fallback: if the library is missing or no CUDA device is
usable, the calls below raise.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtmx.so")

_D = ctypes.POINTER(ctypes.c_double)
_I32 = ctypes.POINTER(ctypes.c_int32)
_I64 = ctypes.POINTER(ctypes.c_int64)
_VP = ctypes.c_void_p


class TmxSchedule(ctypes.Structure):
    _fields_ = [("min_order", ctypes.c_int32),
                ("max_order", ctypes.c_int32),
                ("gauss_legendre_factor", ctypes.c_int32),
                ("bessel_start", ctypes.c_int32),
                ("tolerance", ctypes.c_double)]


# name -> (restype, argtypes): every entry point declared in include/tmx.h
SIGNATURES = {
    "tmx_create": (ctypes.c_int, [ctypes.POINTER(_VP), ctypes.c_int]),
    "tmx_destroy": (None, [_VP]),
    "tmx_last_error": (ctypes.c_char_p, [_VP]),
    "tmx_tmatrix_size": (ctypes.c_int64, [ctypes.c_int32]),
    "tmx_tmatrix_batch": (ctypes.c_int, [_VP, ctypes.c_int64, _D, _D, _D, _D,
                                         _D, ctypes.POINTER(TmxSchedule)]),
    "tmx_batch_upload": (ctypes.c_int, [_VP, ctypes.c_int64, _D, _D, _D, _D,
                                        _D, ctypes.POINTER(TmxSchedule)]),
    "tmx_batch_compute": (ctypes.c_int, [_VP]),
    "tmx_tmatrix_batch_fixed": (ctypes.c_int, [_VP, ctypes.c_int64, _D, _D, _D,
                                               _D, _D, _I32, _I32]),
    "tmx_tmatrix_batch_calculator": (ctypes.c_int, [_VP, ctypes.c_int64, _D, _D, _D,
                                                    _D, _D, ctypes.c_int32,
                                                    ctypes.c_double, ctypes.c_int32,
                                                    ctypes.c_int32]),
    "tmx_batch_orientation_average": (ctypes.c_int, [_VP, _D, ctypes.c_int32,
                                                     ctypes.c_int32, _I32]),
    "tmx_batch_scattering_matrix": (ctypes.c_int, [_VP, ctypes.c_int64, _I64, _D, _D,
                                                   _D, _D, _D, _D, _D, _D]),
    "tmx_batch_extinction_matrix": (ctypes.c_int, [_VP, ctypes.c_int64, _I64, _D, _D,
                                                   _D, _D, _D]),
    "tmx_batch_absorption_cross_sections": (ctypes.c_int, [_VP, ctypes.c_int64,
                                                           ctypes.c_int32, _D,
                                                           ctypes.c_int32, _D]),
    "tmx_batch_average_absorption_cross_section": (ctypes.c_int, [_VP, ctypes.c_int64,
                                                                  ctypes.c_int32, _D]),
    "tmx_batch_results": (ctypes.c_int, [_VP, _I32, _I32, _I32, _D]),
    "tmx_batch_observables": (ctypes.c_int, [_VP, ctypes.c_int32, _D, _D,
                                             ctypes.c_int32, _D]),
    "tmx_batch_gradients": (ctypes.c_int, [_VP, ctypes.c_int32, _D, _D,
                                           ctypes.c_int32, _D, _D]),
    "tmx_batch_tmatrix": (ctypes.c_int, [_VP, ctypes.c_int64, _D]),
    "tmx_batch_tmatrix_total": (ctypes.c_int, [_VP, _I64]),
    "tmx_batch_tmatrices": (ctypes.c_int, [_VP, _D, _I64]),
    "tmx_set_tmatrix_sink": (ctypes.c_int, [_VP, _D, ctypes.c_int64]),
    "tmx_probe_fp64": (ctypes.c_int, [_VP, ctypes.c_int, _D]),
    "tmx_kernel_launches": (ctypes.c_int64, [_VP]),
    "tmx_timer_start": (ctypes.c_int, [_VP]),
    "tmx_timer_stop": (ctypes.c_int, [_VP, _D]),
    "tmx_profile_enable": (ctypes.c_int, [_VP, ctypes.c_int]),
    "tmx_profile_read": (ctypes.c_int, [_VP, ctypes.c_int, _D,
                                        ctypes.POINTER(ctypes.c_int64), _D]),
    "tmx_profile_bytes": (ctypes.c_int, [_VP, ctypes.c_int, _D]),
    "tmx_profile_timeline": (ctypes.c_int, [_VP, ctypes.c_int64, _D, _I64]),
    "tmx_batch_host_times": (ctypes.c_int, [_VP, _D]),
    "tmx_set_batch_mode": (ctypes.c_int, [_VP, ctypes.c_int]),
    "tmx_get_batch_mode": (ctypes.c_int, [_VP, _I32]),
    "tmx_last_batch_mode": (ctypes.c_int, [_VP, _I32]),
    "tmx_batch_flops_survey": (ctypes.c_double, [_VP]),
    "tmx_host_alloc": (ctypes.c_void_p, [ctypes.c_size_t]),
    "tmx_host_free": (None, [ctypes.c_void_p]),
    "tmx_get_dispatch": (ctypes.c_int, [_VP, _I32]),
    "tmx_set_dispatch": (ctypes.c_int, [_VP, _I32]),
    "tmx_autotune": (ctypes.c_int, [_VP, ctypes.c_int64, _D, _D, _D, _D, _D,
                                    _I32, _I32, ctypes.c_int, _D]),
    "tmx_orientation_coefficients": (ctypes.c_int, [ctypes.c_int, ctypes.c_double,
                                                     ctypes.c_int, _VP, _VP, _D]),
    "tmx_shape_distribution": (ctypes.c_int, [ctypes.c_int, ctypes.c_int,
                                              ctypes.c_double, ctypes.c_double,
                                              _D, _D, _D]),
    "tmx_rv_over_rs": (ctypes.c_double, [ctypes.c_double]),
    "tmx_get_table": (ctypes.c_int, [_VP, ctypes.c_int32, ctypes.c_int32, _D,
                                     ctypes.c_int32, _D, ctypes.c_int32, _D,
                                     ctypes.c_int32, _D, _D, _D, _D, _I32,
                                     ctypes.c_int32, _D, ctypes.c_int32,
                                     ctypes.c_int32, ctypes.c_int32,
                                     ctypes.POINTER(TmxSchedule), _D, _D, _I32]),
    "tmx_tmatrix_fixed_noalloc": (ctypes.c_int, [ctypes.c_double] * 5
                                  + [ctypes.c_int32, ctypes.c_int32, _VP, _VP, _VP]),
}

_lib = None


def load():
    """Load libtmx.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            "libtmx.so not found at %s: build it with "
            "`python -m costuum_b200.build` (nvcc, sm_100a)" % LIB_PATH)
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def ptr(a):
    return a.ctypes.data_as(_D)


def iptr(a):
    return a.ctypes.data_as(_I32)


def lptr(a):
    return a.ctypes.data_as(_I64)


# p(beta) callback of a custom orientation distribution
ORIENT_FN = ctypes.CFUNCTYPE(ctypes.c_double, ctypes.c_double, ctypes.c_void_p)


class TmxError(RuntimeError):
    pass


def check(ctx, rc, what):
    if rc != 0:
        msg = load().tmx_last_error(ctx) if ctx else b""
        raise TmxError("%s failed (%d): %s" % (what, rc,
                                               (msg or b"").decode(errors="replace")))
