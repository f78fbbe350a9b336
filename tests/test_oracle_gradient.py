"""CPU tests of the oracle's MakeGradientDH (oracle/sht_oracle.c), pinned
against the analytic gradient of the field built from scipy's spherical
Legendre functions and their theta derivatives:
    theta = (1/r) dF/dtheta,  phi = 1/(r sin theta) dF/dphi,
with both components zero on the pole rows (MakeGradientDH.f95:510-514)."""
import numpy as np
import pytest
import scipy.special as sp


def gradient_known(cilm, theta, phi, lc, r):
    th = np.atleast_1d(theta)
    gt = np.zeros((len(th), len(phi)))
    gp = np.zeros((len(th), len(phi)))
    st = np.sin(th)
    for l in range(lc + 1):
        for m in range(l + 1):
            v, dv = sp.sph_legendre_p(l, m, th, diff_n=1)
            k = (-1) ** m * np.sqrt(4 * np.pi * (2 - (m == 0)))
            P, dP = v * k, dv * k
            a = cilm[0, l, m] * np.cos(m * phi) + cilm[1, l, m] * np.sin(m * phi)
            da = m * (-cilm[0, l, m] * np.sin(m * phi) + cilm[1, l, m] * np.cos(m * phi))
            gt += np.outer(dP, a) / r
            with np.errstate(divide="ignore", invalid="ignore"):
                gp += np.outer(np.where(st > 0, P / st, 0.0), da) / r
    return gt, gp


@pytest.mark.parametrize("sampling", [1, 2])
@pytest.mark.parametrize("extend", [0, 1])
@pytest.mark.parametrize("radius", [1.0, 6371.0])
def test_makegradient_dh_known_answer(oracle, sampling, extend, radius):
    L = 14
    c = oracle.power_law_cilm(L, 81)
    for lc in (L, 8):
        t, p = oracle.makegradient_dh(c, sampling=sampling, lmax_calc=lc, extend=extend,
                                      radius=radius)
        n = 2 * L + 2
        th = np.pi * np.arange(n + extend) / n
        ph = 2 * np.pi * np.arange(sampling * n + extend) / (sampling * n)
        gt, gp = gradient_known(c, th, ph, lc, radius)
        gt[0] = gp[0] = 0.0                      # poles: defined as zero
        if extend:
            gt[n] = gp[n] = 0.0
        scale_t, scale_p = np.abs(gt).max(), np.abs(gp).max()
        assert np.abs(t - gt).max() / scale_t < 1e-12
        assert np.abs(p - gp).max() / scale_p < 1e-12
