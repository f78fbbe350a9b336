"""GPU parity of MakeGradientDH (src/MakeGradientDH.f95) against the oracle:
theta and phi grids within the grid tolerance of the transforms (max-abs
relative <= 1e-12), for both samplings, extend, lmax_calc and radius, on
batches, and through the C drop-in with Fortran column-major arrays."""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

GRID_TOL = 1e-12


def rel(a, b):
    return np.abs(np.asarray(a) - b).max() / np.abs(b).max()


@pytest.mark.parametrize("sampling", [1, 2])
@pytest.mark.parametrize("extend", [0, 1])
@pytest.mark.parametrize("L", [16, 95])
def test_gradient_matches_oracle(cuda, oracle, sampling, extend, L):
    c = oracle.power_law_cilm(L, 90)
    for lc, radius in ((L, None), (L // 2, 6371.0)):
        t, p = cuda.MakeGradientDH(c, sampling=sampling, lmax_calc=lc, extend=extend,
                                   radius=radius)
        tr, pr = oracle.makegradient_dh(c, sampling=sampling, lmax_calc=lc, extend=extend,
                                        radius=1.0 if radius is None else radius)
        assert t.shape == tr.shape and p.shape == pr.shape
        assert rel(t.cpu().numpy(), tr) <= GRID_TOL
        assert rel(p.cpu().numpy(), pr) <= GRID_TOL


def test_gradient_batch_and_large(cuda, oracle):
    L = 300
    cs = np.stack([oracle.power_law_cilm(L, 91 + i) for i in range(3)])
    t, p = cuda.MakeGradientDH(torch.from_numpy(cs).cuda(), sampling=2)
    tr, pr = oracle.makegradient_dh(cs[1], sampling=2)
    assert rel(t[1].cpu().numpy(), tr) <= GRID_TOL
    assert rel(p[1].cpu().numpy(), pr) <= GRID_TOL
    t0, _ = cuda.MakeGradientDH(cs[0], sampling=2)
    assert torch.equal(t0, t[0])


def test_gradient_dropin(cuda, oracle):
    from shtools_b200 import _lib
    lib = _lib.load()
    L = 24
    c = oracle.power_law_cilm(L, 95)
    cf = np.asfortranarray(c)
    n = 2 * L + 2
    th = np.zeros((n + 1, 2 * n + 1), order="F")
    ph = np.zeros((n + 1, 2 * n + 1), order="F")
    D = ctypes.POINTER(ctypes.c_double)
    st, nn = ctypes.c_int(-1), ctypes.c_int(0)
    samp, ext = ctypes.c_int(2), ctypes.c_int(1)
    r = ctypes.c_double(2.0)
    lib.MakeGradientDH(cf.ctypes.data_as(D), L + 1, L, th.ctypes.data_as(D),
                       ph.ctypes.data_as(D), n + 1, 2 * n + 1, ctypes.byref(nn),
                       ctypes.byref(samp), None, ctypes.byref(ext), ctypes.byref(r),
                       ctypes.byref(st))
    assert st.value == 0 and nn.value == n
    tr, pr = oracle.makegradient_dh(c, sampling=2, extend=1, radius=2.0)
    assert rel(th, tr) <= GRID_TOL
    assert rel(ph, pr) <= GRID_TOL


def test_gradient_errors(cuda):
    with pytest.raises(ValueError):
        cuda.MakeGradientDH(np.zeros((2, 5, 5)), sampling=3)
    with pytest.raises(ValueError):
        cuda.MakeGradientDH(np.zeros((2, 5, 5)), radius=0.0)
