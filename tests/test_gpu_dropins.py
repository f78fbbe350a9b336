"""The hot-path C drop-ins of libshtcuda, called through the C ABI exactly as
a C or Fortran caller of include/shtools.h would (src/cWrapper.f95:209-374):
Fortran column-major arrays, NULL or set optional arguments, the n / lmax
out-parameters, leading dimensions larger than needed, and the exit
statuses 1 (dimensions), 2 (bounds) and 5 (GLQ nodes missing).  Results are
compared with the oracle at the parity tolerances.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GRID_TOL = 1e-12
DEG_TOL = 1e-11

D = ctypes.POINTER(ctypes.c_double)
I = ctypes.POINTER(ctypes.c_int)


def perdeg(a, b):
    num = np.sqrt(((np.asarray(a) - b) ** 2).sum(axis=(0, 2)))
    den = np.sqrt((np.asarray(b) ** 2).sum(axis=(0, 2)))
    den[den == 0] = 1.0
    return num / den


def grid_rel(a, b):
    return np.abs(np.asarray(a) - b).max() / np.abs(b).max()


def dp(a):
    return None if a is None else a.ctypes.data_as(D)


def ip(v):
    return None if v is None else ctypes.byref(ctypes.c_int(v))


@pytest.fixture(scope="module")
def lib(cuda):
    from shtools_b200 import _lib
    return _lib.load()


def _cilm_padded(oracle, L, cdim, seed):
    """(2, cdim, cdim) Fortran-ordered cilm whose degrees beyond L hold
    noise: the drop-ins must use only l <= lmax_comp."""
    c = oracle.power_law_cilm(L, seed)
    full = np.random.default_rng(seed + 1).standard_normal((2, cdim, cdim))
    full[:, :L + 1, :L + 1] = c
    return np.asfortranarray(full), c


@pytest.mark.parametrize("opts", [
    dict(),                                                    # every optional NULL
    dict(norm=2, sampling=2, csphase=-1, lmax_calc=17, extend=1),
    dict(norm=4, sampling=1, csphase=1, lmax_calc=None, extend=1),
])
def test_makegrid_shexpand_dh_dropins(lib, oracle, opts):
    L, cdim = 23, 27
    cf, c = _cilm_padded(oracle, L, cdim, 71)
    samp = opts.get("sampling", 1)
    ext = opts.get("extend", 0)
    n = 2 * L + 2
    d0, d1 = n + ext + 3, samp * n + ext + 2            # larger leading dimensions
    grid = np.full((d0, d1), 7.0, order="F")
    st, nn = ctypes.c_int(-1), ctypes.c_int(0)
    lib.MakeGridDH(dp(grid), d0, d1, ctypes.byref(nn), dp(cf), cdim, L,
                   ip(opts.get("norm")), ip(opts.get("sampling")), ip(opts.get("csphase")),
                   ip(opts.get("lmax_calc")), ip(opts.get("extend")), ctypes.byref(st))
    assert st.value == 0 and nn.value == n
    kw = dict(norm=opts.get("norm", 1), sampling=samp, csphase=opts.get("csphase", 1),
              lmax_calc=opts.get("lmax_calc"), extend=ext)
    ref = oracle.makegrid_dh(c, **kw)
    got = grid[:n + ext, :samp * n + ext]
    assert grid_rel(got, ref) <= GRID_TOL
    assert (grid[n + ext:, :] == 7.0).all() and (grid[:, samp * n + ext:] == 7.0).all()

    # analysis of the oracle's grid (without the extend row/column)
    g = np.asfortranarray(ref[:n, :samp * n])
    lc = opts.get("lmax_calc") or L
    out = np.full((2, cdim, cdim), 3.0, order="F")
    lm = ctypes.c_int(-1)
    lib.SHExpandDH(dp(g), n, samp * n, n, dp(out), cdim, ctypes.byref(lm),
                   ip(opts.get("norm")), ip(opts.get("sampling")), ip(opts.get("csphase")),
                   ip(opts.get("lmax_calc")), ctypes.byref(st))
    assert st.value == 0 and lm.value == L
    bref = oracle.shexpand_dh(ref[:n, :samp * n], norm=kw["norm"], sampling=samp,
                              csphase=kw["csphase"], lmax_calc=opts.get("lmax_calc"))
    assert perdeg(out[:, :lc + 1, :lc + 1], bref).max() <= DEG_TOL
    # the reference zeroes the whole cilm (SHExpandDH.f95:283)
    assert (out[:, lc + 1:, :] == 0).all() and (out[:, :, lc + 1:] == 0).all()


@pytest.mark.parametrize("opts", [
    dict(),
    dict(norm=2, csphase=-1, lmax_calc=15, extend=1),
])
def test_makegrid_shexpand_glq_dropins(lib, oracle, opts):
    L, cdim = 22, 25
    cf, c = _cilm_padded(oracle, L, cdim, 81)
    z, w = oracle.shglq(L)
    ext = opts.get("extend", 0)
    d0, d1 = L + 1 + 2, 2 * L + 1 + ext + 1
    grid = np.full((d0, d1), 7.0, order="F")
    st = ctypes.c_int(-1)
    lib.MakeGridGLQ(dp(grid), d0, d1, dp(cf), cdim, L, None, dp(z),
                    ip(opts.get("norm")), ip(opts.get("csphase")), ip(opts.get("lmax_calc")),
                    ip(opts.get("extend")), ctypes.byref(st))
    assert st.value == 0
    kw = dict(norm=opts.get("norm", 1), csphase=opts.get("csphase", 1),
              lmax_calc=opts.get("lmax_calc"))
    ref = oracle.makegrid_glq(c, zero=z, extend=ext, **kw)
    assert grid_rel(grid[:L + 1, :2 * L + 1 + ext], ref) <= GRID_TOL
    assert (grid[L + 1:, :] == 7.0).all()

    g = np.asfortranarray(ref[:, :2 * L + 1])
    lc = opts.get("lmax_calc") or L
    out = np.full((2, cdim, cdim), 3.0, order="F")
    lib.SHExpandGLQ(dp(out), cdim, L, dp(g), dp(w), None, dp(z),
                    ip(opts.get("norm")), ip(opts.get("csphase")), ip(opts.get("lmax_calc")),
                    ctypes.byref(st))
    assert st.value == 0
    bref = oracle.shexpand_glq(ref[:, :2 * L + 1], w=w, zero=z, **kw)
    assert perdeg(out[:, :lc + 1, :lc + 1], bref).max() <= DEG_TOL
    assert (out[:, lc + 1:, :] == 0).all()


def test_quadrature_dropins(lib, oracle):
    st = ctypes.c_int(-1)
    for L in (0, 9, 64):
        z = np.zeros(L + 1)
        w = np.zeros(L + 1)
        lib.SHGLQ(L, dp(z), dp(w), None, None, None, None, ctypes.byref(st))
        assert st.value == 0
        zr, wr = oracle.shglq(L)
        assert np.abs(z - zr).max() <= 1e-15 and np.abs(w - wr).max() <= 1e-15
        lib.PreGLQ(ctypes.c_double(-1.0), ctypes.c_double(1.0), L + 1, dp(z), dp(w),
                   ctypes.byref(st))
        assert st.value == 0 and np.abs(z - zr).max() <= 1e-15
        # GLQGridCoord (GLQGridCoord.f95:112-118)
        for ext in (None, 1):
            e = ext or 0
            lat = np.zeros(L + 1)
            lon = np.zeros(2 * L + 1 + e)
            nlat, nlong = ctypes.c_int(0), ctypes.c_int(0)
            lib.GLQGridCoord(dp(lat), L + 1, dp(lon), 2 * L + 1 + e, L, ctypes.byref(nlat),
                             ctypes.byref(nlong), ip(ext), ctypes.byref(st))
            assert st.value == 0 and nlat.value == L + 1 and nlong.value == 2 * L + 1
            assert np.abs(lat - np.degrees(np.arcsin(zr))).max() <= 1e-12
            assert np.allclose(lon, 360.0 * np.arange(2 * L + 1 + e) / (2 * L + 1),
                               rtol=0, atol=1e-12)
    # the PreGLQ interval [x1, x2] maps the nodes affinely
    z = np.zeros(9)
    w = np.zeros(9)
    lib.PreGLQ(ctypes.c_double(0.5), ctypes.c_double(2.0), 9, dp(z), dp(w), ctypes.byref(st))
    zr, wr = oracle.preglq(0.5, 2.0, 9)
    assert st.value == 0 and np.abs(z - zr).max() <= 1e-15 and np.abs(w - wr).max() <= 1e-15
    for n, ext in ((8, None), (40, 1)):
        e = ext or 0
        aj = np.zeros(n + e)
        lib.DHaj(n, dp(aj), n + e, ip(ext), ctypes.byref(st))
        assert st.value == 0
        ar = oracle.dhaj(n)
        assert np.abs(aj[:n] - ar).max() <= 1e-14 * np.abs(ar).max()
        if e:
            assert aj[n] == 0.0


def test_dropin_exit_statuses(lib, oracle):
    L = 7
    cf, _ = _cilm_padded(oracle, L, L + 1, 5)
    n = 2 * L + 2
    st, nn = ctypes.c_int(-1), ctypes.c_int(0)
    grid = np.zeros((n + 1, 2 * n + 1), order="F")
    # 1: grid too small
    lib.MakeGridDH(dp(grid), n - 1, 2 * n, ctypes.byref(nn), dp(cf), L + 1, L, None, ip(2),
                   None, None, None, ctypes.byref(st))
    assert st.value == 1 and nn.value == n
    # 2: bad sampling, extend, norm, csphase, lmax_calc > lmax
    for args in ((None, 3, None, None, None), (None, 1, None, None, 2), (5, 1, None, None, None),
                 (None, 1, 0, None, None), (None, 1, None, L + 1, None)):
        nrm, samp, cs, lc, ext = args
        lib.MakeGridDH(dp(grid), n + 1, 2 * n + 1, ctypes.byref(nn), dp(cf), L + 1, L,
                       ip(nrm), ip(samp), ip(cs), ip(lc), ip(ext), ctypes.byref(st))
        assert st.value == 2, args
    # SHExpandDH: odd n -> 2; cilm too small -> 1
    out = np.zeros((2, L + 1, L + 1), order="F")
    lm = ctypes.c_int(0)
    lib.SHExpandDH(dp(grid), n + 1, 2 * n + 1, n + 1, dp(out), L + 1, ctypes.byref(lm),
                   None, None, None, None, ctypes.byref(st))
    assert st.value == 2
    lib.SHExpandDH(dp(grid), n + 1, 2 * n + 1, n, dp(out), L, ctypes.byref(lm), None, None,
                   None, None, ctypes.byref(st))
    assert st.value == 1 and lm.value == L
    # GLQ: nodes missing -> 5, plx given -> 2, grid too small -> 1
    g = np.zeros((L + 1, 2 * L + 2), order="F")
    z, w = oracle.shglq(L)
    lib.MakeGridGLQ(dp(g), L + 1, 2 * L + 1, dp(cf), L + 1, L, None, None, None, None, None,
                    None, ctypes.byref(st))
    assert st.value == 5
    lib.MakeGridGLQ(dp(g), L + 1, 2 * L + 1, dp(cf), L + 1, L, dp(g), dp(z), None, None, None,
                    None, ctypes.byref(st))
    assert st.value == 2
    lib.MakeGridGLQ(dp(g), L, 2 * L + 1, dp(cf), L + 1, L, None, dp(z), None, None, None,
                    None, ctypes.byref(st))
    assert st.value == 1
    lib.SHExpandGLQ(dp(out), L + 1, L, dp(g), dp(w), None, None, None, None, None,
                    ctypes.byref(st))
    assert st.value == 5
    lib.SHExpandGLQ(dp(out), L, L, dp(g), dp(w), None, dp(z), None, None, None,
                    ctypes.byref(st))
    assert st.value == 1
    lib.SHGLQ(L, dp(z), dp(w), dp(g), None, None, None, ctypes.byref(st))
    assert st.value == 2
    lat = np.zeros(L + 1)
    lon = np.zeros(2 * L + 1)
    lib.GLQGridCoord(dp(lat), L, dp(lon), 2 * L + 1, L, None, None, None, ctypes.byref(st))
    assert st.value == 1
    lib.GLQGridCoord(dp(lat), L + 1, dp(lon), 2 * L + 1, L, None, None, ip(2),
                     ctypes.byref(st))
    assert st.value == 2
    lib.DHaj(7, dp(lat), 8, None, ctypes.byref(st))
    assert st.value == 2
    lib.DHaj(8, dp(lat), 8, ip(1), ctypes.byref(st))
    assert st.value == 1
