"""ctypes front end of the CPU oracle (oracle/sht_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, by the smoke check in
__graft_entry__.py and by the CPU-baseline leg of bench.py.  The product
package (shtools_b200) never imports it.

The function signatures mirror the f2py signatures of the reference Python
API (src/pyshtools.pyf:235-376) and the argument resolution of
pyshtools/backends/ducc0_wrapper.py:268-281, so that parity tests read like
calls into pyshtools itself.  Arrays are numpy float64, C order.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIBPATH = os.path.join(_HERE, "lib", "liboracle.so")
_lib = None

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.c_int


class OracleError(RuntimeError):
    """Non-zero exit status of an oracle routine (reference codes 1-5)."""


def build(force=False):
    """Compile the oracle library with its Makefile (gcc, no GPU needed)."""
    if force or not os.path.exists(_LIBPATH) or (
            os.path.getmtime(_LIBPATH)
            < os.path.getmtime(os.path.join(_HERE, "sht_oracle.c"))):
        subprocess.check_call(["make", "-s", "-C", _HERE, "lib/liboracle.so"])
    return _LIBPATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIBPATH)
        L.orc_makegrid_dh.argtypes = [_D, _D, _I, _I, _I, _I, _I, _I, _I]
        L.orc_makegrid_dh_window.argtypes = [_D, _D, _I, _I, _I, _I, _I, _I,
                                             _I, _I, _I]
        L.orc_shexpand_dh.argtypes = [_D, _I, _D, _I, _I, _I, _I, _I, _I]
        L.orc_shexpand_dh_window.argtypes = [_D, _I, _D, _I, _I, _I, _I, _I,
                                             _I, _I, _I]
        L.orc_makegrid_glq.argtypes = [_D, _D, _I, _I, _D, _I, _I, _I, _I]
        L.orc_makegrid_glq_window.argtypes = [_D, _D, _I, _I, _D, _I, _I, _I,
                                              _I, _I, _I]
        L.orc_shexpand_glq.argtypes = [_D, _I, _I, _D, _I, _D, _D, _I, _I, _I]
        L.orc_shexpand_glq_window.argtypes = [_D, _I, _I, _D, _I, _D, _D, _I,
                                              _I, _I, _I, _I]
        L.orc_preglq.argtypes = [ctypes.c_double, ctypes.c_double, _I, _D, _D]
        L.orc_preglq_iter.argtypes = [ctypes.c_double, ctypes.c_double, _I,
                                      _D, _D, _I]
        L.orc_dhaj.argtypes = [_I, _D, _I]
        L.orc_makegradient_dh.argtypes = [_D, _D, _D, _I, _I, _I, _I, _I, ctypes.c_double]
        L.orc_shmultiply.argtypes = [_D, _I, _D, _I, _I, _D, _I, _I, _I, _I]
        _F = ctypes.c_double
        L.orc_makegravgrid_dh.argtypes = [_D, _D, _D, _D, _D, _D, _I, _I, _F, _F, _F, _F,
                                          _I, _I, _I, _F, _I, _F, _I]
        L.orc_normal_gravity.argtypes = [_F, _F, _F, _F, _F]
        L.orc_normal_gravity.restype = _F
        L.orc_makegrid_dhc.argtypes = [_D, _D, _I, _I, _I, _I, _I, _I, _I]
        L.orc_shexpand_dhc.argtypes = [_D, _I, _D, _I, _I, _I, _I, _I, _I]
        L.orc_makegrid_glqc.argtypes = [_D, _D, _I, _I, _D, _I, _I, _I, _I]
        L.orc_shexpand_glqc.argtypes = [_D, _I, _I, _D, _I, _D, _D, _I, _I, _I]
        L.orc_rec_tables.argtypes = [_I, _I, _D, _D]
        L.orc_fft_c2c.argtypes = [_I, _D, _D, _I]
        L.orc_fft_r2c.argtypes = [_I, _D, _D, _D]
        L.orc_fft_c2r.argtypes = [_I, _D, _D, _D]
        L.orc_makegrid_dh_adjoint.argtypes = [_D, _I, _D, _I, _I, _I, _I, _I, _I]
        L.orc_makegrid_glq_adjoint.argtypes = [_D, _I, _D, _I, _D, _I, _I, _I, _I]
        L.orc_shexpand_dh_adjoint.argtypes = [_D, _D, _I, _I, _I, _I, _I, _I]
        L.orc_shexpand_glq_adjoint.argtypes = [_D, _D, _I, _I, _D, _D, _I, _I, _I]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(_D)


def _check(status):
    if status != 0:
        raise OracleError("oracle exit status %d" % status)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


# --------------------------------------------------------------------------
# Quadrature (PreGLQ.f95, DHaj.f95, SHGLQ.f95:188)
# --------------------------------------------------------------------------
def preglq(x1, x2, n, itermax=1000):
    zero = np.zeros(n)
    w = np.zeros(n)
    _check(lib().orc_preglq_iter(float(x1), float(x2), int(n), _p(zero), _p(w),
                                 int(itermax)))
    return zero, w


def shglq(lmax):
    """Gauss-Legendre nodes (descending) and weights for bandwidth lmax."""
    return preglq(-1.0, 1.0, lmax + 1)


def dhaj(n, extend=0):
    aj = np.zeros(n + extend)
    _check(lib().orc_dhaj(int(n), _p(aj), int(extend)))
    return aj


def rec_tables(lc, norm):
    ff1 = np.zeros((lc + 1, lc + 1))
    ff2 = np.zeros((lc + 1, lc + 1))
    _check(lib().orc_rec_tables(int(lc), int(norm), _p(ff1), _p(ff2)))
    return ff1, ff2


# --------------------------------------------------------------------------
# FFT (stand-in for FFTW's r2c / c2r, FFTW3.f95:212-271)
# --------------------------------------------------------------------------
def fft_c2c(x, sign=-1):
    x = np.asarray(x, dtype=np.complex128)
    re = np.ascontiguousarray(x.real)
    im = np.ascontiguousarray(x.imag)
    _check(lib().orc_fft_c2c(len(x), _p(re), _p(im), int(sign)))
    return re + 1j * im


def fft_r2c(x):
    x = _f64(x)
    n = len(x)
    re = np.zeros(n // 2 + 1)
    im = np.zeros(n // 2 + 1)
    _check(lib().orc_fft_r2c(n, _p(x), _p(re), _p(im)))
    return re + 1j * im


def fft_c2r(X, n):
    X = np.asarray(X, dtype=np.complex128)
    re = _f64(X.real)
    im = _f64(X.imag)
    out = np.zeros(n)
    _check(lib().orc_fft_c2r(int(n), _p(re), _p(im), _p(out)))
    return out


# --------------------------------------------------------------------------
# Transforms
# --------------------------------------------------------------------------
def _lmaxes(cilm, lmax, lmax_calc):
    if lmax is None:
        lmax = cilm.shape[1] - 1
    if lmax_calc is None:
        lmax_calc = lmax
    return int(lmax), int(lmax_calc)


def makegrid_dh(cilm, lmax=None, norm=1, sampling=1, csphase=1,
                lmax_calc=None, extend=0, pair_window=None):
    """MakeGridDH (MakeGridDH.f95:1).  Returns (n+extend, sampling*n+extend)."""
    cilm = _f64(cilm)
    lmax, lmax_calc = _lmaxes(cilm, lmax, lmax_calc)
    n = 2 * lmax + 2
    grid = np.zeros((n + int(extend), sampling * n + int(extend)))
    if pair_window is None:
        st = lib().orc_makegrid_dh(_p(grid), _p(cilm), cilm.shape[1], lmax,
                                   int(norm), int(sampling), int(csphase),
                                   lmax_calc, int(extend))
    else:
        st = lib().orc_makegrid_dh_window(_p(grid), _p(cilm), cilm.shape[1],
                                          lmax, int(norm), int(sampling),
                                          int(csphase), lmax_calc, int(extend),
                                          int(pair_window[0]),
                                          int(pair_window[1]))
    _check(st)
    return grid


def shexpand_dh(grid, norm=1, sampling=1, csphase=1, lmax_calc=None,
                pair_window=None):
    """SHExpandDH (SHExpandDH.f95:1).  Returns (2, lmax_calc+1, lmax_calc+1)."""
    grid = _f64(grid)
    n = grid.shape[0]
    if lmax_calc is None:
        lmax_calc = n // 2 - 1
    cilm = np.zeros((2, lmax_calc + 1, lmax_calc + 1))
    if pair_window is None:
        st = lib().orc_shexpand_dh(_p(cilm), lmax_calc + 1, _p(grid), n,
                                   grid.shape[1], int(norm), int(sampling),
                                   int(csphase), int(lmax_calc))
    else:
        st = lib().orc_shexpand_dh_window(_p(cilm), lmax_calc + 1, _p(grid), n,
                                          grid.shape[1], int(norm),
                                          int(sampling), int(csphase),
                                          int(lmax_calc), int(pair_window[0]),
                                          int(pair_window[1]))
    _check(st)
    return cilm


def makegrid_glq(cilm, zero=None, lmax=None, norm=1, csphase=1,
                 lmax_calc=None, extend=0, pair_window=None):
    """MakeGridGLQ (MakeGridGLQ.f95:1).  Returns (lmax+1, 2*lmax+1+extend)."""
    cilm = _f64(cilm)
    lmax, lmax_calc = _lmaxes(cilm, lmax, lmax_calc)
    if zero is None:
        zero, _ = shglq(lmax)
    zero = _f64(zero)
    grid = np.zeros((lmax + 1, 2 * lmax + 1 + int(extend)))
    if pair_window is None:
        st = lib().orc_makegrid_glq(_p(grid), _p(cilm), cilm.shape[1], lmax,
                                    _p(zero), int(norm), int(csphase),
                                    lmax_calc, int(extend))
    else:
        st = lib().orc_makegrid_glq_window(_p(grid), _p(cilm), cilm.shape[1],
                                           lmax, _p(zero), int(norm),
                                           int(csphase), lmax_calc,
                                           int(extend), int(pair_window[0]),
                                           int(pair_window[1]))
    _check(st)
    return grid


def shexpand_glq(grid, w=None, zero=None, norm=1, csphase=1, lmax_calc=None,
                 pair_window=None):
    """SHExpandGLQ (SHExpandGLQ.f95:1).  Returns (2, lmax_calc+1, lmax_calc+1)."""
    grid = _f64(grid)
    lmax = grid.shape[0] - 1
    if zero is None or w is None:
        zero, w = shglq(lmax)
    zero = _f64(zero)
    w = _f64(w)
    if lmax_calc is None:
        lmax_calc = lmax
    cilm = np.zeros((2, lmax_calc + 1, lmax_calc + 1))
    if pair_window is None:
        st = lib().orc_shexpand_glq(_p(cilm), lmax_calc + 1, lmax, _p(grid),
                                    grid.shape[1], _p(w), _p(zero), int(norm),
                                    int(csphase), int(lmax_calc))
    else:
        st = lib().orc_shexpand_glq_window(_p(cilm), lmax_calc + 1, lmax,
                                           _p(grid), grid.shape[1], _p(w),
                                           _p(zero), int(norm), int(csphase),
                                           int(lmax_calc), int(pair_window[0]),
                                           int(pair_window[1]))
    _check(st)
    return cilm


def makegrid_dh_adjoint(grid, lmax, norm=1, sampling=1, csphase=1,
                        lmax_calc=None, extend=0):
    """Transpose of makegrid_dh (MakeGridDH.f95:504-639) applied to a grid
    cotangent of the synthesis output shape.  Returns (2, lmax+1, lmax+1)."""
    grid = _f64(grid)
    lmax = int(lmax)
    lmax_calc = lmax if lmax_calc is None else int(lmax_calc)
    n = 2 * lmax + 2
    assert grid.shape == (n + int(extend), sampling * n + int(extend))
    cilm = np.zeros((2, lmax + 1, lmax + 1))
    _check(lib().orc_makegrid_dh_adjoint(_p(cilm), lmax + 1, _p(grid), lmax,
                                         int(norm), int(sampling), int(csphase),
                                         lmax_calc, int(extend)))
    return cilm


def makegrid_glq_adjoint(grid, lmax, zero=None, norm=1, csphase=1,
                         lmax_calc=None, extend=0):
    """Transpose of makegrid_glq (MakeGridGLQ.f95:547-665).  Returns
    (2, lmax+1, lmax+1)."""
    grid = _f64(grid)
    lmax = int(lmax)
    lmax_calc = lmax if lmax_calc is None else int(lmax_calc)
    if zero is None:
        zero, _ = shglq(lmax)
    zero = _f64(zero)
    assert grid.shape == (lmax + 1, 2 * lmax + 1 + int(extend))
    cilm = np.zeros((2, lmax + 1, lmax + 1))
    _check(lib().orc_makegrid_glq_adjoint(_p(cilm), lmax + 1, _p(grid), lmax,
                                          _p(zero), int(norm), int(csphase),
                                          lmax_calc, int(extend)))
    return cilm


def shexpand_dh_adjoint(cilm, n, norm=1, sampling=1, csphase=1, lmax_calc=None):
    """Transpose of shexpand_dh (SHExpandDH.f95:463-702) applied to a
    coefficient cotangent.  Returns the (n, sampling*n) grid cotangent."""
    cilm = _f64(cilm)
    n = int(n)
    lmax_calc = n // 2 - 1 if lmax_calc is None else int(lmax_calc)
    grid = np.zeros((n, sampling * n))
    _check(lib().orc_shexpand_dh_adjoint(_p(grid), _p(cilm), cilm.shape[1], n,
                                         int(norm), int(sampling), int(csphase),
                                         lmax_calc))
    return grid


def shexpand_glq_adjoint(cilm, lmax, w=None, zero=None, norm=1, csphase=1,
                         lmax_calc=None):
    """Transpose of shexpand_glq (SHExpandGLQ.f95:445-649).  Returns the
    (lmax+1, 2*lmax+1) grid cotangent."""
    cilm = _f64(cilm)
    lmax = int(lmax)
    lmax_calc = lmax if lmax_calc is None else int(lmax_calc)
    if zero is None or w is None:
        zero, w = shglq(lmax)
    grid = np.zeros((lmax + 1, 2 * lmax + 1))
    _check(lib().orc_shexpand_glq_adjoint(_p(grid), _p(cilm), cilm.shape[1], lmax,
                                          _p(_f64(w)), _p(_f64(zero)), int(norm),
                                          int(csphase), lmax_calc))
    return grid


def power_law_cilm(lmax, seed, beta=2.0):
    """Seeded Gaussian coefficients with degree power S(l) = (l+1)^-beta.

    Each coefficient has std sqrt(S(l)/(2l+1)); m > l and the m = 0 sine
    terms are zero.  Same recipe as the TimingAccuracy examples
    (examples/python/TimingAccuracy/TimingAccuracyDH.py:16-74) with a
    numpy Generator in place of the global seed.
    """
    rng = np.random.default_rng(seed)
    c = rng.standard_normal((2, lmax + 1, lmax + 1))
    l = np.arange(lmax + 1)
    c *= np.sqrt((l + 1.0) ** (-beta) / (2 * l + 1.0))[None, :, None]
    mask = l[None, :, None] >= l[None, None, :]
    c = np.where(mask, c, 0.0)
    c[1, :, 0] = 0.0
    return c


# --------------------------------------------------------------------------
# Complex transforms (complex128 arrays; cilm[0] the order +m, cilm[1] -m)
# --------------------------------------------------------------------------
def _c128(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.complex128))


def makegrid_dhc(cilm, lmax=None, norm=1, sampling=1, csphase=1, lmax_calc=None,
                 extend=0):
    """MakeGridDHC (MakeGridDHC.f95:1).  Returns complex (n+extend, sampling*n+extend)."""
    cilm = _c128(cilm)
    lmax, lmax_calc = _lmaxes(cilm, lmax, lmax_calc)
    n = 2 * lmax + 2
    grid = np.zeros((n + int(extend), sampling * n + int(extend)), dtype=np.complex128)
    _check(lib().orc_makegrid_dhc(_p(grid), _p(cilm), cilm.shape[1], lmax, int(norm),
                                  int(sampling), int(csphase), lmax_calc, int(extend)))
    return grid


def shexpand_dhc(grid, norm=1, sampling=1, csphase=1, lmax_calc=None):
    """SHExpandDHC (SHExpandDHC.f95:1).  Returns complex (2, lmax_calc+1, lmax_calc+1)."""
    grid = _c128(grid)
    n = grid.shape[0]
    if lmax_calc is None:
        lmax_calc = n // 2 - 1
    cilm = np.zeros((2, lmax_calc + 1, lmax_calc + 1), dtype=np.complex128)
    _check(lib().orc_shexpand_dhc(_p(cilm), lmax_calc + 1, _p(grid), n, grid.shape[1],
                                  int(norm), int(sampling), int(csphase), int(lmax_calc)))
    return cilm


def makegrid_glqc(cilm, zero=None, lmax=None, norm=1, csphase=1, lmax_calc=None,
                  extend=0):
    """MakeGridGLQC (MakeGridGLQC.f95:1).  Returns complex (lmax+1, 2*lmax+1+extend)."""
    cilm = _c128(cilm)
    lmax, lmax_calc = _lmaxes(cilm, lmax, lmax_calc)
    if zero is None:
        zero, _ = shglq(lmax)
    zero = _f64(zero)
    grid = np.zeros((lmax + 1, 2 * lmax + 1 + int(extend)), dtype=np.complex128)
    _check(lib().orc_makegrid_glqc(_p(grid), _p(cilm), cilm.shape[1], lmax, _p(zero),
                                   int(norm), int(csphase), lmax_calc, int(extend)))
    return grid


def shexpand_glqc(grid, w=None, zero=None, norm=1, csphase=1, lmax_calc=None):
    """SHExpandGLQC (SHExpandGLQC.f95:1).  Returns complex (2, lmax_calc+1, lmax_calc+1)."""
    grid = _c128(grid)
    lmax = grid.shape[0] - 1
    if zero is None or w is None:
        zero, w = shglq(lmax)
    zero = _f64(zero)
    w = _f64(w)
    if lmax_calc is None:
        lmax_calc = lmax
    cilm = np.zeros((2, lmax_calc + 1, lmax_calc + 1), dtype=np.complex128)
    _check(lib().orc_shexpand_glqc(_p(cilm), lmax_calc + 1, lmax, _p(grid), grid.shape[1],
                                   _p(w), _p(zero), int(norm), int(csphase),
                                   int(lmax_calc)))
    return cilm


def power_law_cilm_complex(L, seed, beta=2.0):
    """Seeded complex coefficients (2, L+1, L+1) with per-degree power
    S(l) = (l+1)^-beta; cilm[1, :, 0] (order -0) is zero."""
    rng = np.random.default_rng(seed)
    c = rng.standard_normal((2, L + 1, L + 1)) + 1j * rng.standard_normal((2, L + 1, L + 1))
    l = np.arange(L + 1)
    c *= np.sqrt((l + 1.0) ** -beta / (2 * (2 * l + 1.0)))[None, :, None]
    c = np.where(l[:, None] >= l[None, :], c, 0.0)
    c[1, :, 0] = 0.0
    return c


def makegradient_dh(cilm, lmax=None, sampling=1, lmax_calc=None, extend=0, radius=1.0):
    """MakeGradientDH (MakeGradientDH.f95:1).  Returns (theta, phi) grids."""
    cilm = _f64(cilm)
    lmax, lmax_calc = _lmaxes(cilm, lmax, lmax_calc)
    n = 2 * lmax + 2
    shape = (n + int(extend), sampling * n + int(extend))
    th = np.zeros(shape)
    ph = np.zeros(shape)
    _check(lib().orc_makegradient_dh(_p(th), _p(ph), _p(cilm), cilm.shape[1], lmax,
                                     int(sampling), lmax_calc, int(extend), float(radius)))
    return th, ph


def normal_gravity(geocentric_lat, gm, omega, a, b):
    """NormalGravity (NormalGravity.f95:1): latitude in degrees."""
    return lib().orc_normal_gravity(float(geocentric_lat), float(gm), float(omega),
                                    float(a), float(b))


def makegravgrid_dh(cilm, gm, r0, lmax=None, a=None, f=0.0, sampling=2, lmax_calc=None,
                    omega=None, normal_gravity=0, normal_gravity_gm=None, extend=0,
                    pot=True):
    """MakeGravGridDH (MakeGravGridDH.f95:1).  omega=None is the Fortran's
    absent OMEGA (no rotation terms).  Returns (rad, theta, phi, total, pot),
    pot None when not requested."""
    cilm = _f64(cilm)
    lmax, lmax_calc = _lmaxes(cilm, lmax, lmax_calc)
    n = 2 * lmax + 2
    shape = (n + int(extend), sampling * n + int(extend))
    g = [np.zeros(shape) for _ in range(5 if pot else 4)]
    a = r0 if a is None else a
    ngm = gm if normal_gravity_gm is None else normal_gravity_gm
    _check(lib().orc_makegravgrid_dh(_p(g[0]), _p(g[1]), _p(g[2]), _p(g[3]),
                                     _p(g[4]) if pot else None, _p(cilm), cilm.shape[1],
                                     lmax, float(gm), float(r0), float(a), float(f),
                                     int(sampling), lmax_calc, int(omega is not None),
                                     0.0 if omega is None else float(omega),
                                     int(normal_gravity), float(ngm), int(extend)))
    return (g[0], g[1], g[2], g[3], g[4] if pot else None)


def shmultiply(cilm1, cilm2, lmax1=None, lmax2=None, norm=1, csphase=1):
    """SHMultiply (SHMultiply.f95:1).  Returns (2, lmax1+lmax2+1, lmax1+lmax2+1)."""
    c1 = _f64(cilm1)
    c2 = _f64(cilm2)
    lmax1 = c1.shape[1] - 1 if lmax1 is None else int(lmax1)
    lmax2 = c2.shape[1] - 1 if lmax2 is None else int(lmax2)
    lo = lmax1 + lmax2
    out = np.zeros((2, lo + 1, lo + 1))
    _check(lib().orc_shmultiply(_p(out), lo + 1, _p(c1), c1.shape[1], lmax1, _p(c2),
                                c2.shape[1], lmax2, int(norm), int(csphase)))
    return out
