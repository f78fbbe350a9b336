"""GPU parity of the complex transforms (MakeGridDHC, SHExpandDHC,
MakeGridGLQC, SHExpandGLQC) against the oracle on identical inputs.

Tolerances as the real transforms: grids max-abs relative <= 1e-12,
coefficients per degree <= 1e-11 (norm 3 relative to the grid magnitude);
also round trips, a real field through the complex path, the C drop-ins
(Fortran column-major host arrays) and error handling.
"""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

GRID_TOL = 1e-12
DEG_TOL = 1e-11


def perdeg(a, b):
    num = np.sqrt((np.abs(a - b) ** 2).sum(axis=(0, 2)))
    den = np.sqrt((np.abs(b) ** 2).sum(axis=(0, 2)))
    den[den == 0] = 1.0
    return num / den


def grid_rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


def coef_check(gpu, ref, norm, grid):
    if norm == 3:
        scale = np.abs(grid).max()
        assert np.abs(gpu - ref).max() / scale < 1e-15 * max(1.0, ref.shape[-1] ** 2)
    else:
        e = perdeg(gpu, ref)
        assert e.max() <= DEG_TOL, (e.max(), e.argmax())


@pytest.mark.parametrize("norm", [1, 2, 3, 4])
@pytest.mark.parametrize("csphase", [1, -1])
@pytest.mark.parametrize("sampling", [1, 2])
@pytest.mark.parametrize("extend", [0, 1])
def test_dhc_matches_oracle(cuda, oracle, norm, csphase, sampling, extend):
    L = 15 if norm == 3 else 40
    c = oracle.power_law_cilm_complex(L, 31)
    for lc in (L, L // 2):
        g = cuda.MakeGridDHC(c, norm=norm, sampling=sampling, csphase=csphase,
                             extend=extend, lmax_calc=lc).cpu().numpy()
        gref = oracle.makegrid_dhc(c, norm=norm, sampling=sampling, csphase=csphase,
                                   extend=extend, lmax_calc=lc)
        assert g.shape == gref.shape
        assert grid_rel(g, gref) <= (GRID_TOL if norm != 3 else 1e-11)
        gin = gref[:2 * L + 2, :sampling * (2 * L + 2)]
        b = cuda.SHExpandDHC(gin, norm=norm, sampling=sampling, csphase=csphase,
                             lmax_calc=lc).cpu().numpy()
        bref = oracle.shexpand_dhc(gin, norm=norm, sampling=sampling, csphase=csphase,
                                   lmax_calc=lc)
        coef_check(b, bref, norm, gin)


@pytest.mark.parametrize("norm", [1, 2, 3, 4])
@pytest.mark.parametrize("csphase", [1, -1])
@pytest.mark.parametrize("extend", [0, 1])
@pytest.mark.parametrize("L", [14, 41])
def test_glqc_matches_oracle(cuda, oracle, norm, csphase, extend, L):
    if norm == 3 and L > 15:
        pytest.skip("norm 3 is unstable beyond degree ~15 in the reference")
    c = oracle.power_law_cilm_complex(L, 32)
    z, w = oracle.shglq(L)
    g = cuda.MakeGridGLQC(c, zero=z, norm=norm, csphase=csphase,
                          extend=extend).cpu().numpy()
    gref = oracle.makegrid_glqc(c, zero=z, norm=norm, csphase=csphase, extend=extend)
    assert grid_rel(g, gref) <= (GRID_TOL if norm != 3 else 1e-11)
    gin = gref[:, :2 * L + 1]
    b = cuda.SHExpandGLQC(gin, w=w, zero=z, norm=norm, csphase=csphase).cpu().numpy()
    bref = oracle.shexpand_glqc(gin, w=w, zero=z, norm=norm, csphase=csphase)
    coef_check(b, bref, norm, gin)


def test_complex_batched_and_roundtrip(cuda, oracle):
    L = 300
    cs = np.stack([oracle.power_law_cilm_complex(L, 40 + i) for i in range(3)])
    ct = torch.from_numpy(cs).cuda()
    g = cuda.MakeGridDHC(ct, sampling=2)
    b = cuda.SHExpandDHC(g, sampling=2)
    for i in range(3):
        gi = cuda.MakeGridDHC(ct[i], sampling=2)
        assert torch.equal(g[i], gi)
        assert perdeg(b[i].cpu().numpy(), cs[i]).max() < 1e-10
    zg = cuda.MakeGridGLQC(ct)
    bg = cuda.SHExpandGLQC(zg)
    assert perdeg(bg[1].cpu().numpy(), cs[1]).max() < 1e-10


def test_real_field_through_complex_path(cuda, oracle):
    L = 60
    cr = oracle.power_law_cilm(L, 50)
    g = cuda.MakeGridDH(cr, sampling=2).cpu().numpy()
    cc = cuda.SHExpandDHC(g.astype(np.complex128), sampling=2).cpu().numpy()
    for m in range(1, L + 1):
        expect = (cr[0, m:, m] - 1j * cr[1, m:, m]) / np.sqrt(2.0)
        assert np.abs(cc[0, m:, m] - expect).max() < 1e-12
    back = cuda.MakeGridDHC(cc, sampling=2).cpu().numpy()
    assert np.abs(back.imag).max() < 1e-12
    assert np.abs(back.real - g).max() < 1e-12


def test_complex_dropins_fortran_layout(cuda, oracle):
    from shtools_b200 import _lib
    lib = _lib.load()
    L = 20
    c = oracle.power_law_cilm_complex(L, 60)
    cf = np.asfortranarray(c)
    n = 2 * L + 2
    grid = np.zeros((n, 2 * n), dtype=np.complex128, order="F")
    st = ctypes.c_int(-1)
    nn = ctypes.c_int(0)
    samp = ctypes.c_int(2)
    P = ctypes.c_void_p
    lib.MakeGridDHC(P(grid.ctypes.data), n, 2 * n, ctypes.byref(nn), P(cf.ctypes.data),
                    L + 1, L, None, ctypes.byref(samp), None, None, None, ctypes.byref(st))
    assert st.value == 0 and nn.value == n
    gref = oracle.makegrid_dhc(c, sampling=2)
    assert grid_rel(grid, gref) <= GRID_TOL
    back = np.zeros((2, L + 1, L + 1), dtype=np.complex128, order="F")
    lm = ctypes.c_int(0)
    lib.SHExpandDHC(P(grid.ctypes.data), n, 2 * n, n, P(back.ctypes.data), L + 1,
                    ctypes.byref(lm), None, ctypes.byref(samp), None, None,
                    ctypes.byref(st))
    assert st.value == 0 and lm.value == L
    assert perdeg(back, c).max() < 1e-11
    z, w = oracle.shglq(L)
    gq = np.zeros((L + 1, 2 * L + 1), dtype=np.complex128, order="F")
    D = ctypes.POINTER(ctypes.c_double)
    lib.MakeGridGLQC(P(gq.ctypes.data), L + 1, 2 * L + 1, P(cf.ctypes.data), L + 1, L,
                     None, z.ctypes.data_as(D), None, None, None, None, ctypes.byref(st))
    assert st.value == 0
    assert grid_rel(gq, oracle.makegrid_glqc(c, zero=z)) <= GRID_TOL
    bq = np.zeros((2, L + 1, L + 1), dtype=np.complex128, order="F")
    lib.SHExpandGLQC(P(bq.ctypes.data), L + 1, L, P(gq.ctypes.data), w.ctypes.data_as(D),
                     None, z.ctypes.data_as(D), None, None, None, ctypes.byref(st))
    assert st.value == 0
    assert perdeg(bq, c).max() < 1e-11


def test_complex_errors(cuda):
    with pytest.raises(ValueError):
        cuda.MakeGridDHC(np.zeros((2, 4, 4), complex), sampling=3)
    with pytest.raises(ValueError):
        cuda.SHExpandDHC(np.zeros((7, 7), complex))
    # a real entry point refuses a complex plan and vice versa
    from shtools_b200 import transforms as T
    pc = T.get_plan(T.GRID_DH, 8, 8, 1, 1, 1, 0, cplx=True)
    pr = T.get_plan(T.GRID_DH, 8, 8, 1, 1, 1, 0)
    c = torch.zeros((1, 2, 9, 9), dtype=torch.float64, device="cuda")
    with pytest.raises(Exception):
        pc.synthesis(c)
    with pytest.raises(Exception):
        pr.synthesis_c(c.to(torch.complex128))


@pytest.mark.parametrize("kind", ["dh", "glq"])
def test_complex_long_rings_match_oracle(cuda, oracle, kind):
    """Rings of 1024 points or more take the FFT passes that read the bins or
    the ring in the first pass and write the ring or the bins from the last:
    DH lmax 260, sampling 2 (1044 points) and GLQ lmax 520 (1041 points),
    with the extend column, against the oracle."""
    if kind == "dh":
        L = 260
        c = oracle.power_law_cilm_complex(L, 33)
        g = cuda.MakeGridDHC(c, sampling=2, extend=1).cpu().numpy()
        gref = oracle.makegrid_dhc(c, sampling=2, extend=1)
        gin = gref[:2 * L + 2, :2 * (2 * L + 2)]
        b = cuda.SHExpandDHC(gin, sampling=2).cpu().numpy()
        bref = oracle.shexpand_dhc(gin, sampling=2)
    else:
        L = 520
        c = oracle.power_law_cilm_complex(L, 34)
        z, w = oracle.shglq(L)
        g = cuda.MakeGridGLQC(c, zero=z, extend=1).cpu().numpy()
        gref = oracle.makegrid_glqc(c, zero=z, extend=1)
        gin = gref[:, :2 * L + 1]
        b = cuda.SHExpandGLQC(gin, w=w, zero=z).cpu().numpy()
        bref = oracle.shexpand_glqc(gin, w=w, zero=z)
    assert g.shape == gref.shape
    assert grid_rel(g, gref) <= GRID_TOL
    coef_check(b, bref, 1, gin)
