"""CPU tests of the oracle's MakeGravGridDH and NormalGravity
(oracle/sht_oracle.c), pinned against independent known answers:

  * the gravity vector and potential of V = GM/r sum_l (r0/r)^l C_lm Y_lm
    built from scipy's spherical Legendre functions and their theta
    derivatives, evaluated on each ring at the ellipsoid radius
    r = a b / sqrt((b cos lat)^2 + (a sin lat)^2), b = a (1 - f):
        rad = dV/dr, theta = (1/r) dV/dtheta, phi = 1/(r sin theta) dV/dphi,
    theta and phi zero on the pole rows (MakeGravGridDH.f95:809-812);
  * the centrifugal terms r sin^2(theta) w^2, sin cos r w^2 and
    (r sin(theta) w)^2 / 2 (MakeGravGridDH.f95:987-1013);
  * the WGS84 normal gravity at the equator and the poles (the published
    constants 9.7803253359 and 9.8321849378 m/s^2) and the closed forms of
    the spherical branches of NormalGravity.f95.
"""
import numpy as np
import pytest
import scipy.special as sp

WGS84 = dict(gm=3986004.418e8, a=6378137.0, f=1.0 / 298.257223563, omega=7292115e-11)


def ellipsoid_radius(a, f, theta):
    b = a * (1.0 - f)
    lat = np.pi / 2 - theta
    return a * b / np.sqrt((b * np.cos(lat)) ** 2 + (a * np.sin(lat)) ** 2)


def grav_known(cilm, th, ph, lc, gm, r0, rex):
    nt, npp = len(th), len(ph)
    rad, gt, gp, pot = (np.zeros((nt, npp)) for _ in range(4))
    st = np.sin(th)
    for l in range(lc + 1):
        q = (r0 / rex) ** l
        for m in range(l + 1):
            v, dv = sp.sph_legendre_p(l, m, th, diff_n=1)
            k = (-1) ** m * np.sqrt(4 * np.pi * (2 - (m == 0)))
            P, dP = v * k, dv * k
            a = cilm[0, l, m] * np.cos(m * ph) + cilm[1, l, m] * np.sin(m * ph)
            da = m * (-cilm[0, l, m] * np.sin(m * ph) + cilm[1, l, m] * np.cos(m * ph))
            rad += np.outer(-(l + 1) * gm / rex ** 2 * q * P, a)
            pot += np.outer(gm / rex * q * P, a)
            gt += np.outer(gm / rex ** 2 * q * dP, a)
            with np.errstate(divide="ignore", invalid="ignore"):
                gp += np.outer(np.where(st > 0, gm / rex ** 2 * q * P / st, 0.0), da)
    return rad, gt, gp, pot


@pytest.mark.parametrize("sampling", [1, 2])
@pytest.mark.parametrize("extend", [0, 1])
@pytest.mark.parametrize("shape", ["sphere", "ellipsoid"])
def test_makegravgrid_dh_known_answer(oracle, sampling, extend, shape):
    L = 13
    c = oracle.power_law_cilm(L, 91)
    c[0, 0, 0] = 1.0
    gm, r0 = 4.2828372e13, 3396000.0
    a, f = (r0, 0.0) if shape == "sphere" else (3395428.0, 0.00589)
    n = 2 * L + 2
    th = np.pi * np.arange(n + extend) / n
    ph = 2 * np.pi * np.arange(sampling * n + extend) / (sampling * n)
    rex = ellipsoid_radius(a, f, th)
    for lc in (L, 6):
        rad, t, p, tot, pot = oracle.makegravgrid_dh(c, gm, r0, a=a, f=f, sampling=sampling,
                                                     lmax_calc=lc, extend=extend)
        kr, kt, kp, ku = grav_known(c, th, ph, lc, gm, r0, rex)
        kt[0] = kp[0] = 0.0
        if extend:
            kt[n] = kp[n] = 0.0
        for got, ref in ((rad, kr), (t, kt), (p, kp), (pot, ku)):
            assert got.shape == ref.shape
            assert np.abs(got - ref).max() / np.abs(ref).max() < 1e-12
        ktot = np.sqrt(kr ** 2 + kt ** 2 + kp ** 2)
        assert np.abs(tot - ktot).max() / ktot.max() < 1e-12
        if extend:
            for g in (rad, t, p, tot, pot):
                assert np.array_equal(g[:, -1], g[:, 0])


def test_makegravgrid_dh_rotation_and_normal_gravity(oracle):
    L = 10
    c = oracle.power_law_cilm(L, 92) * 1e-3
    c[0, 0, 0] = 1.0
    w = WGS84
    r0 = w["a"]
    n = 2 * L + 2
    th = np.pi * np.arange(n + 1) / n
    rex = ellipsoid_radius(w["a"], w["f"], th)
    base = oracle.makegravgrid_dh(c, w["gm"], r0, a=w["a"], f=w["f"], extend=1)
    rot = oracle.makegravgrid_dh(c, w["gm"], r0, a=w["a"], f=w["f"], extend=1,
                                 omega=w["omega"])
    st, ct = np.sin(th)[:, None], np.cos(th)[:, None]
    om = w["omega"]
    scale = np.abs(base[0]).max()
    assert np.abs(rot[0] - base[0] - rex[:, None] * (st * om) ** 2).max() < 1e-13 * scale
    assert np.abs(rot[1] - base[1] - st * ct * rex[:, None] * om ** 2).max() < 1e-13 * scale
    assert np.array_equal(rot[2], base[2])
    assert np.abs(rot[4] - base[4] - 0.5 * (rex[:, None] * st * om) ** 2).max() \
        < 1e-13 * np.abs(base[4]).max()
    # gravity disturbance: |g| minus the normal gravity of the row's latitude
    dist = oracle.makegravgrid_dh(c, w["gm"], r0, a=w["a"], f=w["f"], extend=1,
                                  omega=om, normal_gravity=1)
    b = w["a"] * (1 - w["f"])
    lat = (np.pi / 2 - th) * 180 / np.pi
    ng = np.array([oracle.normal_gravity(x, w["gm"], om, w["a"], b) for x in lat])
    mag = np.sqrt(rot[0] ** 2 + rot[1] ** 2 + rot[2] ** 2)
    assert np.abs(dist[3] - (mag - ng[:, None])).max() < 1e-12 * mag.max()
    # a different GM for the normal field
    d2 = oracle.makegravgrid_dh(c, w["gm"], r0, a=w["a"], f=w["f"], extend=1, omega=om,
                                normal_gravity=1, normal_gravity_gm=w["gm"] * 1.001)
    ng2 = np.array([oracle.normal_gravity(x, w["gm"] * 1.001, om, w["a"], b) for x in lat])
    assert np.abs(d2[3] - (mag - ng2[:, None])).max() < 1e-12 * mag.max()


def test_normal_gravity_wgs84(oracle):
    w = WGS84
    b = w["a"] * (1 - w["f"])
    ge = oracle.normal_gravity(0.0, w["gm"], w["omega"], w["a"], b)
    gp = oracle.normal_gravity(90.0, w["gm"], w["omega"], w["a"], b)
    gs = oracle.normal_gravity(-90.0, w["gm"], w["omega"], w["a"], b)
    assert abs(ge - 9.7803253359) < 2e-10
    assert abs(gp - 9.8321849378) < 2e-10
    assert abs(gs - gp) < 1e-12
    # the sphere: GM/a^2 without rotation; with rotation GM/a^2 - a w^2 at the
    # equator and GM/a^2 at the poles
    assert oracle.normal_gravity(30.0, w["gm"], 0.0, w["a"], w["a"]) == \
        pytest.approx(w["gm"] / w["a"] ** 2, rel=1e-15)
    assert oracle.normal_gravity(0.0, w["gm"], w["omega"], w["a"], w["a"]) == \
        pytest.approx(w["gm"] / w["a"] ** 2 - w["a"] * w["omega"] ** 2, rel=1e-14)
    assert oracle.normal_gravity(90.0, w["gm"], w["omega"], w["a"], w["a"]) == \
        pytest.approx(w["gm"] / w["a"] ** 2, rel=1e-14)


def test_makegravgrid_dh_status(oracle):
    c = oracle.power_law_cilm(8, 93)
    with pytest.raises(oracle.OracleError, match="status 5"):
        oracle.makegravgrid_dh(c, 1.0, 1.0, normal_gravity=1)
    with pytest.raises(oracle.OracleError, match="status 2"):
        oracle.makegravgrid_dh(c, 1.0, 1.0, sampling=3)
    with pytest.raises(oracle.OracleError, match="status 2"):
        oracle.makegravgrid_dh(c, 1.0, 1.0, lmax=8, lmax_calc=9)
    # degree 0 only: rad = -GM/r^2, pot = GM/r, no horizontal components
    c0 = np.zeros((2, 1, 1))
    c0[0, 0, 0] = 1.0
    rad, t, p, tot, pot = oracle.makegravgrid_dh(c0, 2.0, 1.0, lmax=4, sampling=1)
    assert np.allclose(rad, -2.0, rtol=0, atol=1e-15)
    assert np.allclose(pot, 2.0, rtol=0, atol=1e-15)
    assert np.abs(t).max() == 0.0 and np.abs(p).max() == 0.0
    assert rad.shape == (10, 10)
