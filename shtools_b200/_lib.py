"""ctypes binding of libshtcuda (include/shtcuda.h).

The library is loaded from the package tree (shtools_b200/lib/libshtcuda.so).
There is no fallback: if the library is missing, or no CUDA device is
visible, every transform raises.  PyTorch supplies device memory and the
current CUDA stream; the arithmetic happens in the library's kernels.
"""
import ctypes
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(_HERE, "lib", "libshtcuda.so")

_P = ctypes.c_void_p
_LL = ctypes.c_longlong
_I = ctypes.c_int
_D = ctypes.c_double
_SZ = ctypes.c_size_t
_DP = ctypes.POINTER(ctypes.c_double)
_IP = ctypes.POINTER(ctypes.c_int)

_lock = threading.Lock()
_lib = None

# exported C-ABI symbols, in the order of include/shtcuda.h
EXPORTS = (
    "shtc_version", "shtc_status_string", "shtc_plan_create_dh",
    "shtc_plan_create_glq", "shtc_plan_destroy", "shtc_plan_info",
    "shtc_plan_set_tuning", "shtc_timing_enable", "shtc_timing_collect",
    "shtc_plan_set_precision", "shtc_mixed_status", "shtc_mixed_wait_selftest",
    "shtc_plan_legendre_table",
    "shtc_synthesis_noalloc",
    "shtc_workspace_bytes", "shtc_synthesis", "shtc_analysis",
    "shtc_synthesis_adjoint", "shtc_analysis_adjoint", "shtc_synthesis_ex",
    "shtc_analysis_ex", "shtc_synthesis_adjoint_ex", "shtc_analysis_adjoint_ex",
    "shtc_batch_create", "shtc_batch_destroy", "shtc_batch_layout",
    "shtc_batch_workspace_bytes", "shtc_batch_synthesis", "shtc_batch_analysis",
    "shtc_preglq",
    "shtc_dhaj", "MakeGridDH", "SHExpandDH", "MakeGridGLQ", "SHExpandGLQ",
    "SHGLQ", "PreGLQ", "DHaj", "GLQGridCoord", "shtc_plan_create_dhc", "shtc_plan_create_glqc",
    "shtc_synthesis_c", "shtc_analysis_c", "MakeGridDHC", "SHExpandDHC",
    "MakeGridGLQC", "SHExpandGLQC", "shtc_gradient_workspace_bytes",
    "shtc_gradient_dh", "MakeGradientDH", "shtc_gravity_workspace_bytes",
    "shtc_gravity_dh", "shtc_multiply_workspace_bytes", "shtc_multiply",
    "MakeGravGridDH", "NormalGravity", "SHMultiply",
)


class SHTCudaError(RuntimeError):
    """A libshtcuda call returned a non-zero status (reference exit codes 1-5
    plus GPU-side codes 6-9)."""

    def __init__(self, status, what=""):
        self.status = int(status)
        msg = status_string(status)
        super().__init__("%s%s (status %d)" % (what + ": " if what else "", msg,
                                               self.status))


def _bind(L):
    L.shtc_version.restype = _I
    L.shtc_status_string.restype = ctypes.c_char_p
    L.shtc_status_string.argtypes = [_I]
    L.shtc_plan_create_dh.argtypes = [ctypes.POINTER(_P), _I, _I, _I, _I, _I, _I, _P]
    L.shtc_plan_create_glq.argtypes = [ctypes.POINTER(_P), _I, _DP, _DP, _I, _I, _I,
                                       _I, _P]
    L.shtc_plan_destroy.argtypes = [_P]
    L.shtc_plan_info.argtypes = [_P, ctypes.POINTER(_LL), _I]
    L.shtc_plan_set_tuning.argtypes = [_P, _I, _I, _I]
    L.shtc_plan_set_precision.argtypes = [_P, _I]
    L.shtc_mixed_status.argtypes = [ctypes.POINTER(_I), _P]
    L.shtc_mixed_wait_selftest.argtypes = [_P]
    L.shtc_plan_legendre_table.argtypes = [_P, _I, ctypes.POINTER(ctypes.c_ulonglong)]
    L.shtc_workspace_bytes.restype = _SZ
    L.shtc_workspace_bytes.argtypes = [_P, _I]
    coef = [_P, _LL, _LL, _LL, _LL, _I]
    grid = [_P, _LL, _LL, _LL]
    tail = [_I, _P, _SZ, _P]
    L.shtc_synthesis.argtypes = [_P] + coef + grid + tail
    L.shtc_analysis.argtypes = [_P] + grid + coef + tail
    L.shtc_synthesis_adjoint.argtypes = [_P] + grid + coef + tail
    L.shtc_analysis_adjoint.argtypes = [_P] + coef + grid + tail
    coefx = [_P, _I, _LL, _LL, _LL, _LL, _I]
    gridx = [_P, _I, _LL, _LL, _LL]
    L.shtc_synthesis_ex.argtypes = [_P] + coefx + gridx + tail
    L.shtc_analysis_ex.argtypes = [_P] + gridx + coefx + tail
    L.shtc_synthesis_adjoint_ex.argtypes = [_P] + gridx + coefx + tail
    L.shtc_analysis_adjoint_ex.argtypes = [_P] + coefx + gridx + tail
    L.shtc_plan_create_dhc.argtypes = [ctypes.POINTER(_P), _I, _I, _I, _I, _I, _I, _P]
    L.shtc_plan_create_glqc.argtypes = [ctypes.POINTER(_P), _I, _DP, _DP, _I, _I, _I,
                                        _I, _P]
    L.shtc_synthesis_c.argtypes = [_P] + coef + grid + tail
    L.shtc_analysis_c.argtypes = [_P] + grid + coef + tail
    L.shtc_gradient_workspace_bytes.restype = _SZ
    L.shtc_gradient_workspace_bytes.argtypes = [_P, _I]
    L.shtc_gradient_dh.argtypes = [_P] + coef + [_P, _P, _LL, _LL, _LL, _D] + tail
    L.shtc_gravity_workspace_bytes.restype = _SZ
    L.shtc_gravity_workspace_bytes.argtypes = [_P, _I]
    L.shtc_gravity_dh.argtypes = ([_P] + coef + [_D, _D, _D, _D, _I, _D, _I, _D,
                                                 _P, _P, _P, _P, _P, _LL, _LL, _LL] + tail)
    L.shtc_multiply_workspace_bytes.restype = _SZ
    L.shtc_multiply_workspace_bytes.argtypes = [_P, _I]
    L.shtc_multiply.argtypes = ([_P, _P, _LL, _LL, _LL, _LL, _I, _P, _LL, _LL, _LL, _LL, _I]
                                + coef + tail)
    L.shtc_preglq.argtypes = [_D, _D, _I, _P, _P, _P]
    L.shtc_dhaj.argtypes = [_I, _P, _I, _P]
    L.MakeGridDH.argtypes = [_DP, _I, _I, _IP, _DP, _I, _I, _IP, _IP, _IP, _IP, _IP,
                             _IP]
    L.SHExpandDH.argtypes = [_DP, _I, _I, _I, _DP, _I, _IP, _IP, _IP, _IP, _IP, _IP]
    L.MakeGridGLQ.argtypes = [_DP, _I, _I, _DP, _I, _I, _DP, _DP, _IP, _IP, _IP, _IP,
                              _IP]
    L.SHExpandGLQ.argtypes = [_DP, _I, _I, _DP, _DP, _DP, _DP, _IP, _IP, _IP, _IP]
    L.SHGLQ.argtypes = [_I, _DP, _DP, _DP, _IP, _IP, _IP, _IP]
    L.PreGLQ.argtypes = [_D, _D, _I, _DP, _DP, _IP]
    L.DHaj.argtypes = [_I, _DP, _I, _IP, _IP]
    # complex arrays as untyped pointers to interleaved (re, im) doubles
    L.MakeGridDHC.argtypes = [_P, _I, _I, _IP, _P, _I, _I, _IP, _IP, _IP, _IP, _IP, _IP]
    L.SHExpandDHC.argtypes = [_P, _I, _I, _I, _P, _I, _IP, _IP, _IP, _IP, _IP, _IP]
    L.MakeGridGLQC.argtypes = [_P, _I, _I, _P, _I, _I, _DP, _DP, _IP, _IP, _IP, _IP, _IP]
    L.SHExpandGLQC.argtypes = [_P, _I, _I, _P, _DP, _DP, _DP, _IP, _IP, _IP, _IP]
    L.MakeGradientDH.argtypes = [_DP, _I, _I, _DP, _DP, _I, _I, _IP, _IP, _IP, _IP, _DP,
                                 _IP]
    L.SHMultiply.argtypes = [_DP, _I, _DP, _I, _I, _DP, _I, _I, _IP, _IP, _IP, _IP]
    L.MakeGravGridDH.argtypes = [_DP, _I, _I, _D, _D, _D, _D, _DP, _I, _I, _DP, _DP, _DP,
                                 _IP, _IP, _IP, _DP, _IP, _DP, _IP, _IP]
    L.NormalGravity.argtypes = [_D, _D, _D, _D, _D]
    L.NormalGravity.restype = _D
    for name in ("SHMultiply", "MakeGridDH", "SHExpandDH", "MakeGridGLQ", "SHExpandGLQ", "SHGLQ",
                 "PreGLQ", "DHaj", "MakeGridDHC", "SHExpandDHC", "MakeGridGLQC",
                 "SHExpandGLQC", "MakeGradientDH", "MakeGravGridDH"):
        getattr(L, name).restype = None
    return L


def load(path=None):
    """Load (once) and return the ctypes handle of libshtcuda."""
    global _lib
    with _lock:
        if _lib is None:
            p = path or LIBPATH
            if not os.path.exists(p):
                raise RuntimeError(
                    "libshtcuda is not built (%s missing): run "
                    "`python -m shtools_b200.build`" % p)
            _lib = _bind(ctypes.CDLL(p))
        return _lib


def status_string(status):
    try:
        return load().shtc_status_string(int(status)).decode()
    except Exception:  # library missing: generic text
        return "status %d" % status


def check(status, what=""):
    if status != 0:
        raise SHTCudaError(status, what)
