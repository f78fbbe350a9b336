"""CPU tests of the oracle (oracle/sht_oracle.c).

The reference has no stored outputs for this path and cannot be built here
(no Fortran compiler, no FFTW), so the oracle is pinned against independent
known answers:
  * FFTs against numpy.fft (FFTW's sign and scaling conventions);
  * grids against direct sums of scipy's spherical Legendre functions;
  * PreGLQ against numpy's Gauss-Legendre nodes and weights;
  * DHaj against the exactness of the Driscoll-Healy quadrature;
  * band-limited round trips (the reference's own benchmark criterion,
    examples/python/TimingAccuracy/TimingAccuracyDH.py:60-72);
and against the committed golden fixtures as a regression pin.
"""
import math
import os

import numpy as np
import pytest
import scipy.special as sp

HERE = os.path.dirname(os.path.abspath(__file__))


def plm_known(L, theta, norm, csphase):
    """P_lm(cos theta) for all l, m <= L from scipy (independent of the oracle)."""
    th = np.atleast_1d(theta)
    P = np.zeros((L + 1, L + 1, len(th)))
    for l in range(L + 1):
        for m in range(l + 1):
            # scipy's spherical Legendre functions are orthonormal and carry
            # the Condon-Shortley phase
            v = sp.sph_legendre_p(l, m, th) * (-1) ** m * np.sqrt(
                4 * np.pi * (2 - (m == 0)))
            if norm == 2:
                v = v / np.sqrt(2 * l + 1)
            elif norm == 4:
                v = v / np.sqrt(4 * np.pi)
            elif norm == 3:
                v = v / np.sqrt((2 - (m == 0)) * (2 * l + 1) * math.factorial(l - m)
                                / math.factorial(l + m))
            if csphase == -1:
                v = v * (-1) ** m
            P[l, m] = v
    return P


def grid_known(cilm, theta, phi, norm, csphase, lc):
    P = plm_known(lc, theta, norm, csphase)
    g = np.zeros((len(theta), len(phi)))
    for l in range(lc + 1):
        for m in range(l + 1):
            g += np.outer(P[l, m], cilm[0, l, m] * np.cos(m * phi)
                          + cilm[1, l, m] * np.sin(m * phi))
    return g


@pytest.mark.parametrize("n", [1, 2, 3, 5, 7, 8, 12, 13, 63, 97, 127, 256, 1023,
                               1440, 2880, 4095])
def test_fft_matches_numpy(oracle, n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    ref = np.fft.fft(x)
    scale = max(1.0, np.abs(ref).max())
    assert np.abs(oracle.fft_c2c(x, -1) - ref).max() / scale < 1e-14
    assert np.abs(oracle.fft_c2c(x, 1) - np.fft.ifft(x) * n).max() / scale < 1e-14
    xr = x.real
    R = np.fft.rfft(xr)
    assert np.abs(oracle.fft_r2c(xr) - R).max() / max(1, np.abs(R).max()) < 1e-14
    back = oracle.fft_c2r(R, n)
    assert np.abs(back - xr * n).max() / max(1, np.abs(xr * n).max()) < 1e-14


@pytest.mark.parametrize("norm", [1, 2, 3, 4])
@pytest.mark.parametrize("csphase", [1, -1])
@pytest.mark.parametrize("sampling", [1, 2])
@pytest.mark.parametrize("extend", [0, 1])
def test_makegrid_dh_known_answer(oracle, norm, csphase, sampling, extend):
    L = 12
    c = oracle.power_law_cilm(L, 11)
    for lc in (L, 7):
        g = oracle.makegrid_dh(c, norm=norm, sampling=sampling, csphase=csphase,
                               extend=extend, lmax_calc=lc)
        n = 2 * L + 2
        th = np.pi * np.arange(n + extend) / n
        ph = 2 * np.pi * np.arange(sampling * n + extend) / (sampling * n)
        gd = grid_known(c, th, ph, norm, csphase, lc)
        assert g.shape == gd.shape
        assert np.abs(g - gd).max() / np.abs(gd).max() < 1e-13


@pytest.mark.parametrize("norm", [1, 2, 3, 4])
@pytest.mark.parametrize("csphase", [1, -1])
@pytest.mark.parametrize("extend", [0, 1])
def test_makegrid_glq_known_answer(oracle, norm, csphase, extend):
    for L in (11, 12):   # even L has an equator ring
        c = oracle.power_law_cilm(L, 12)
        z, w = oracle.shglq(L)
        for lc in (L, 5):
            g = oracle.makegrid_glq(c, zero=z, norm=norm, csphase=csphase,
                                    extend=extend, lmax_calc=lc)
            ph = 2 * np.pi * np.arange(2 * L + 1 + extend) / (2 * L + 1)
            gd = grid_known(c, np.arccos(z), ph, norm, csphase, lc)
            assert np.abs(g - gd).max() / np.abs(gd).max() < 1e-13


@pytest.mark.parametrize("norm", [1, 2, 4])
@pytest.mark.parametrize("csphase", [1, -1])
def test_roundtrip_bandlimited(oracle, norm, csphase):
    """Analysis of a band-limited synthesis returns the input (quadrature
    exactness), to the accuracy of the reference algorithm at small L."""
    L = 40
    c = oracle.power_law_cilm(L, 13)
    for samp in (1, 2):
        g = oracle.makegrid_dh(c, norm=norm, sampling=samp, csphase=csphase)
        back = oracle.shexpand_dh(g, norm=norm, sampling=samp, csphase=csphase)
        assert np.abs(back - c).max() < 1e-13
    z, w = oracle.shglq(L)
    g = oracle.makegrid_glq(c, zero=z, norm=norm, csphase=csphase)
    back = oracle.shexpand_glq(g, w=w, zero=z, norm=norm, csphase=csphase)
    assert np.abs(back - c).max() < 1e-13


def test_roundtrip_norm3_small(oracle):
    # norm 3 (unnormalised) is only stable to about degree 15 (MakeGridDH.f95:15-18)
    L = 8
    c = oracle.power_law_cilm(L, 14)
    g = oracle.makegrid_dh(c, norm=3)
    back = oracle.shexpand_dh(g, norm=3)
    assert np.abs(back - c).max() / np.abs(c).max() < 1e-9


@pytest.mark.parametrize("n", [1, 2, 3, 4, 17, 50, 64, 513])
def test_preglq_matches_leggauss(oracle, n):
    z, w = oracle.preglq(-1.0, 1.0, n)
    x, wx = np.polynomial.legendre.leggauss(n)
    assert np.abs(z - x[::-1]).max() < 2e-15
    # PreGLQ evaluates P'_n at the last-but-one Newton iterate (PreGLQ.f95:121-146),
    # so the weights nearest the poles carry a relative error ~ n^2 * 1e-15
    assert (np.abs(w - wx[::-1]) / wx[::-1]).max() < 1e-8
    assert np.abs(w - wx[::-1]).max() < 1e-13
    assert np.all(np.diff(z) < 0)


def test_preglq_interval(oracle):
    z, w = oracle.preglq(0.0, 2.0, 9)
    x, wx = np.polynomial.legendre.leggauss(9)
    assert np.abs(z - (1 + x[::-1])).max() < 2e-15
    assert np.abs(w - wx[::-1]).max() < 1e-14


def test_preglq_nonconvergence_status(oracle):
    # host-side fault injection: a zero iteration cap makes PreGLQ return 5
    with pytest.raises(oracle.OracleError, match="5"):
        oracle.preglq(-1.0, 1.0, 20, itermax=0)


@pytest.mark.parametrize("n", [4, 16, 64, 130])
def test_dhaj_quadrature_exact(oracle, n):
    """sum_j a_j P_l(cos theta_j) = sqrt(2) delta_l0 for l < n/2: the DH
    quadrature integrates band-limited functions exactly (a_j carries the
    factor sqrt(8)/n of DHaj.f95:99, i.e. 1/sqrt(2) of the integral 2)."""
    aj = oracle.dhaj(n)
    th = np.pi * np.arange(n) / n
    vals = [np.dot(aj, sp.eval_legendre(l, np.cos(th))) for l in range(n // 2)]
    assert abs(vals[0] - np.sqrt(2)) < 1e-13
    assert max(abs(v) for v in vals[1:]) < 1e-13
    assert aj[0] == 0.0
    ext = oracle.dhaj(n, extend=1)
    assert ext.shape == (n + 1,) and ext[-1] == 0.0
    assert np.array_equal(ext[:n], aj)


def test_dhaj_odd_n_rejected(oracle):
    with pytest.raises(oracle.OracleError):
        oracle.dhaj(7)


def test_error_codes(oracle):
    c = oracle.power_law_cilm(4, 1)
    with pytest.raises(oracle.OracleError, match="2"):
        oracle.makegrid_dh(c, sampling=3)
    with pytest.raises(oracle.OracleError, match="2"):
        oracle.makegrid_dh(c, norm=5)
    with pytest.raises(oracle.OracleError, match="2"):
        oracle.makegrid_dh(c, csphase=0)
    with pytest.raises(oracle.OracleError, match="2"):
        oracle.makegrid_dh(c, lmax_calc=9)


def test_lmax_zero(oracle):
    c = np.zeros((2, 1, 1))
    c[0, 0, 0] = 3.0
    g = oracle.makegrid_dh(c)
    assert g.shape == (2, 2) and np.all(g == 3.0)
    g = oracle.makegrid_glq(c, zero=np.zeros(1))
    assert g.shape == (1, 1) and np.all(g == 3.0)


def test_recursion_table_quirk(oracle):
    """ff1(l, l-1) is built with the Fortran DO variable left at l-1
    (MakeGridDH.f95:341): sqrt(2l+1) up to the rounding of that expression."""
    ff1, ff2 = oracle.rec_tables(30, 1)
    for l in range(2, 31):
        assert abs(ff1[l, l - 1] - math.sqrt(2 * l + 1)) < 1e-14 * math.sqrt(2 * l + 1)
        assert ff2[l, l - 1] == 0.0


def test_golden_fixtures_reproduce(oracle):
    """The oracle still reproduces the committed golden fixtures bit for bit."""
    data = np.load(os.path.join(HERE, "golden", "transforms_small.npz"))
    keys = sorted({k.split("__")[0] for k in data.files})
    assert len(keys) > 100
    for key in keys[::7]:
        kind, L, norm, cs, samp, ext, lc = key.split("_")
        L, norm, cs, samp, ext, lc = (int(L[1:]), int(norm[1:]), int(cs[1:]),
                                      int(samp[1:]), int(ext[1:]), int(lc[2:]))
        c = data[key + "__cilm"]
        if kind == "dh":
            g = oracle.makegrid_dh(c, norm=norm, sampling=samp, csphase=cs,
                                   lmax_calc=lc, extend=ext)
        else:
            g = oracle.makegrid_glq(c, zero=data[key + "__zero"], norm=norm,
                                    csphase=cs, lmax_calc=lc, extend=ext)
        assert np.array_equal(g, data[key + "__grid"]), key
