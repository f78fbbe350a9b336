"""The 'cuda' backend of pyshtools.

A module with the function signatures of the reference's non-Fortran backend
(pyshtools/backends/ducc0_wrapper.py:454, 659, 837, 1003): numpy arrays in,
numpy arrays out, the arithmetic on the GPU.  After ``register()``,
``pyshtools.backends.select_preferred_backend('cuda')`` makes
``SHCoeffs.expand()`` and ``SHGrid.expand()`` run here unchanged
(pyshtools/shclasses/shcoeffs.py:4343-4377, shgrid.py:2105, 3011).

The real and complex DH and GLQ transforms run on the GPU.  The other
names that the backend injectors rebind (pyshtools/expand/__init__.py:91-111,
pyshtools/rotate/__init__.py:18-21) are taken from the reference's own
'shtools' backend when pyshtools is importable, so that switching backends
never removes a function; without pyshtools they raise NotImplementedError.
"""
import sys

import numpy as np

from . import hostio
from . import transforms as _t

__all__ = ["MakeGridDH", "SHExpandDH", "MakeGridGLQ", "SHExpandGLQ", "SHGLQ",
           "GLQGridCoord",
           "MakeGridDHC", "SHExpandDHC", "MakeGridGLQC", "SHExpandGLQC",
           "MakeGradientDH", "MakeGravGridDH", "NormalGravity", "SHRotateRealCoef",
           "available", "register", "set_nthreads", "set_precision", "get_precision"]

# Legendre arithmetic of the four real transforms (no counterpart in the
# reference, whose backends are FP64): "fp64" (the default), or a mixed
# precision of shtools_b200.transforms.PRECISIONS, e.g. "int8x7-table" for
# the INT8 tensor-core sums from each plan's P_lm digit table
_precision = "fp64"


def available():
    """True when libshtcuda loads and a CUDA device is visible."""
    try:
        import torch
        from . import _lib
        _lib.load()
        return torch.cuda.is_available()
    except Exception:
        return False


def set_nthreads(ntnew):
    """Accepted for interface compatibility with the ducc backend; the GPU
    backend has no host thread pool."""
    return None


def set_precision(precision="fp64"):
    """Select the Legendre arithmetic of MakeGridDH, SHExpandDH, MakeGridGLQ
    and SHExpandGLQ for later calls ("fp64", "int8x7", "int8x7-table", ...;
    ValueError otherwise).  The mixed forms apply to norms 1, 2 and 4."""
    global _precision
    _t._precision_code(precision)
    _precision = precision


def get_precision():
    """The Legendre arithmetic selected by set_precision."""
    return _precision


def _np(t):
    """The result as a new numpy array (through pinned staging buffers)."""
    return hostio.to_host(t)


def _dev(a, dtype=np.float64):
    """The numpy input on the current CUDA device (through pinned staging)."""
    return hostio.to_device(np.asarray(a, dtype=dtype))


def _dev_cilm(cilm):
    """A real cilm on the current CUDA device: only its entries m <= l, the
    ones the synthesis reads, cross the staging buffers (entries m > l are
    zero on the device)."""
    return hostio.to_device_lower(np.asarray(cilm, dtype=np.float64))


def MakeGridDH(cilm, lmax=None, norm=1, sampling=1, csphase=1, lmax_calc=None,
               extend=False):
    """griddh = MakeGridDH(cilm, [lmax, norm, sampling, csphase, lmax_calc,
    extend]) -- see src/MakeGridDH.f95:1 and ducc0_wrapper.py:454."""
    return _np(_t.MakeGridDH(_dev_cilm(cilm), lmax=lmax,
                             norm=norm, sampling=sampling, csphase=csphase,
                             lmax_calc=lmax_calc, extend=extend, precision=_precision))


def SHExpandDH(griddh, norm=1, sampling=1, csphase=1, lmax_calc=None):
    """cilm = SHExpandDH(griddh, [norm, sampling, csphase, lmax_calc]) -- see
    src/SHExpandDH.f95:1 and ducc0_wrapper.py:659."""
    return _np(_t.SHExpandDH(_dev(griddh), norm=norm,
                             sampling=sampling, csphase=csphase,
                             lmax_calc=lmax_calc, precision=_precision))


def MakeGridGLQ(cilm, zero=None, lmax=None, norm=1, csphase=1, lmax_calc=None,
                extend=False):
    """gridglq = MakeGridGLQ(cilm, [zero, lmax, norm, csphase, lmax_calc,
    extend]) -- see src/MakeGridGLQ.f95:1 and ducc0_wrapper.py:837.  With
    zero=None the nodes come from the GPU PreGLQ."""
    return _np(_t.MakeGridGLQ(_dev_cilm(cilm), zero=zero,
                              lmax=lmax, norm=norm, csphase=csphase,
                              lmax_calc=lmax_calc, extend=extend, precision=_precision))


def SHExpandGLQ(gridglq, w=None, zero=None, norm=1, csphase=1, lmax_calc=None):
    """cilm = SHExpandGLQ(gridglq, [w, zero, norm, csphase, lmax_calc]) -- see
    src/SHExpandGLQ.f95:1 and ducc0_wrapper.py:1003."""
    return _np(_t.SHExpandGLQ(_dev(gridglq), w=w,
                              zero=zero, norm=norm, csphase=csphase,
                              lmax_calc=lmax_calc, precision=_precision))


def SHGLQ(lmax):
    """zero, w = SHGLQ(lmax) -- Gauss-Legendre nodes and weights from the GPU
    PreGLQ (src/SHGLQ.f95:188)."""
    return _t.SHGLQ(lmax)


def GLQGridCoord(lmax, extend=0):
    """latglq, longlq = GLQGridCoord(lmax, [extend]) -- latitudes (degrees)
    of the GPU PreGLQ nodes and longitudes of a GLQ grid
    (src/GLQGridCoord.f95:112-118, pyshtools.pyf:424-438)."""
    lmax = int(lmax)
    if lmax < 0:
        raise ValueError("lmax must be >= 0, got %d" % lmax)
    if extend not in (0, 1, False, True):
        raise ValueError("extend must be 0 or 1, got %r" % (extend,))
    zero = np.asarray(SHGLQ(lmax)[0], dtype=np.float64)
    nlong = 2 * lmax + 1
    latglq = np.arcsin(zero) * 180.0 / np.pi
    longlq = 360.0 * np.arange(nlong + int(extend), dtype=np.float64) / nlong
    return latglq, longlq


def _fallback(name):
    """The reference 'shtools' backend's function of this name."""
    try:
        from pyshtools.backends import shtools as _ref_shtools
        return getattr(_ref_shtools, name)
    except Exception:
        return None


def _passthrough(name):
    def fn(*args, **kwargs):
        f = _fallback(name)
        if f is None:
            raise NotImplementedError(
                "%s is not part of the GPU transforms (DH/GLQ only) and "
                "the reference 'shtools' backend is not importable" % name)
        return f(*args, **kwargs)
    fn.__name__ = name
    fn.__doc__ = ("Delegates to the reference 'shtools' backend: the GPU "
                  "backend implements the DH and GLQ transforms only.")
    return fn


def MakeGridDHC(cilm, lmax=None, norm=1, sampling=1, csphase=1, lmax_calc=None,
                extend=False):
    """griddh = MakeGridDHC(cilm, [lmax, norm, sampling, csphase, lmax_calc,
    extend]) -- see src/MakeGridDHC.f95:1 and ducc0_wrapper.py:552."""
    return _np(_t.MakeGridDHC(_dev(cilm, np.complex128), lmax=lmax,
                              norm=norm, sampling=sampling, csphase=csphase,
                              lmax_calc=lmax_calc, extend=extend))


def SHExpandDHC(griddh, norm=1, sampling=1, csphase=1, lmax_calc=None):
    """cilm = SHExpandDHC(griddh, [norm, sampling, csphase, lmax_calc]) -- see
    src/SHExpandDHC.f95:1 and ducc0_wrapper.py:745."""
    return _np(_t.SHExpandDHC(_dev(griddh, np.complex128), norm=norm,
                              sampling=sampling, csphase=csphase, lmax_calc=lmax_calc))


def MakeGridGLQC(cilm, zero=None, lmax=None, norm=1, csphase=1, lmax_calc=None,
                 extend=False):
    """gridglq = MakeGridGLQC(cilm, [zero, lmax, norm, csphase, lmax_calc,
    extend]) -- see src/MakeGridGLQC.f95:1 and ducc0_wrapper.py:917."""
    return _np(_t.MakeGridGLQC(_dev(cilm, np.complex128), zero=zero,
                               lmax=lmax, norm=norm, csphase=csphase,
                               lmax_calc=lmax_calc, extend=extend))


def SHExpandGLQC(gridglq, w=None, zero=None, norm=1, csphase=1, lmax_calc=None):
    """cilm = SHExpandGLQC(gridglq, [w, zero, norm, csphase, lmax_calc]) -- see
    src/SHExpandGLQC.f95:1."""
    return _np(_t.SHExpandGLQC(_dev(gridglq, np.complex128), w=w,
                               zero=zero, norm=norm, csphase=csphase,
                               lmax_calc=lmax_calc))


def MakeGradientDH(cilm, lmax=None, sampling=1, lmax_calc=None, extend=False,
                   radius=None):
    """theta, phi = MakeGradientDH(cilm, [lmax, sampling, lmax_calc, extend,
    radius]) -- see src/MakeGradientDH.f95:1 and ducc0_wrapper.py:1164."""
    th, ph = _t.MakeGradientDH(_dev(cilm), lmax=lmax,
                               sampling=sampling, lmax_calc=lmax_calc, extend=extend,
                               radius=radius)
    return _np(th), _np(ph)


def MakeGravGridDH(cilm, gm, r0, lmax=None, a=None, f=0.0, sampling=2, lmax_calc=None,
                   omega=0.0, normal_gravity=1, normal_gravity_gm=None, extend=0):
    """rad, theta, phi, total, pot = MakeGravGridDH(cilm, gm, r0, [lmax, a, f,
    sampling, lmax_calc, omega, normal_gravity, normal_gravity_gm, extend])
    -- the signature of pyshtools.gravmag.MakeGravGridDH
    (src/pyshtools.pyf:1440-1477, src/MakeGravGridDH.f95:1).  As through f2py,
    None for an optional argument takes its default (omega 0.0, f 0.0,
    sampling 2, normal_gravity 1, extend 0), as SHGravCoeffs.expand() relies
    on (pyshtools/shclasses/shgravcoeffs.py:2574)."""
    g = _t.MakeGravGridDH(_dev(cilm), gm, r0, lmax=lmax, a=a,
                          f=0.0 if f is None else f,
                          sampling=2 if sampling is None else sampling,
                          lmax_calc=lmax_calc, omega=0.0 if omega is None else omega,
                          normal_gravity=1 if normal_gravity is None else normal_gravity,
                          normal_gravity_gm=normal_gravity_gm,
                          extend=0 if extend is None else extend)
    return tuple(_np(x) for x in g)


def NormalGravity(geocentric_lat, gm, omega, a, b):
    """value = NormalGravity(geocentric_lat, gm, omega, a, b) -- see
    src/NormalGravity.f95:1."""
    return _t.NormalGravity(geocentric_lat, gm, omega, a, b)


SHRotateRealCoef = _passthrough("SHRotateRealCoef")


def register(registry=None):
    """Add this module as backend 'cuda' to the pyshtools backend registry
    (pyshtools/backends/backends.py:27).  ``registry`` may be given
    explicitly (a module with ``_available_backends``); otherwise
    pyshtools.backends.backends is used.  pyshtools/backends/__init__.py:29
    deletes the name ``backends`` from its package, so the module is taken
    from sys.modules.  Returns the registry module."""
    if registry is None:
        import pyshtools  # noqa: F401
        registry = sys.modules["pyshtools.backends.backends"]
    registry._available_backends["cuda"] = sys.modules[__name__]
    return registry
