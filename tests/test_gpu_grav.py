"""GPU parity of MakeGravGridDH (src/MakeGravGridDH.f95) and NormalGravity
against the oracle: rad, theta, phi and pot within the grid tolerance of the
transforms (max-abs relative <= 1e-12 of each grid), total (|g| minus the
normal gravity) within 1e-12 of the magnitude of g, for both samplings,
extend, lmax_calc, the sphere and the flattened ellipsoid, with and without
rotation and normal gravity, on batches, at lmax 719, and through the C
drop-in with Fortran column-major arrays."""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

GRID_TOL = 1e-12
MARS = dict(gm=4.2828372e13, r0=3396000.0, a=3395428.0, f=0.00589, omega=7.088218e-5)


def rel(a, b, scale=None):
    b = np.asarray(b)
    s = np.abs(b).max() if scale is None else scale
    return np.abs(np.asarray(a) - b).max() / s


def check(gpu, ref):
    rad, t, p, tot, pot = [np.asarray(x.cpu().numpy() if torch.is_tensor(x) else x)
                           for x in gpu]
    rr, tr, pr, totr, potr = ref
    assert rad.shape == rr.shape
    assert rel(rad, rr) <= GRID_TOL
    assert rel(t, tr) <= GRID_TOL
    assert rel(p, pr) <= GRID_TOL
    assert rel(pot, potr) <= GRID_TOL
    assert rel(tot, totr, np.abs(rr).max()) <= GRID_TOL


CASES = {
    "sphere": dict(a=MARS["r0"], f=0.0, omega=None, normal_gravity=0),
    "ellipsoid": dict(a=MARS["a"], f=MARS["f"], omega=None, normal_gravity=0),
    "rotating": dict(a=MARS["a"], f=MARS["f"], omega=MARS["omega"], normal_gravity=0),
    "disturbance": dict(a=MARS["a"], f=MARS["f"], omega=MARS["omega"], normal_gravity=1),
}


@pytest.mark.parametrize("sampling", [1, 2])
@pytest.mark.parametrize("extend", [0, 1])
@pytest.mark.parametrize("case", sorted(CASES))
def test_grav_matches_oracle(cuda, oracle, sampling, extend, case):
    L = 40
    c = oracle.power_law_cilm(L, 110) * 1e-3
    c[0, 0, 0] = 1.0
    kw = CASES[case]
    for lc in (L, 17):
        g = cuda.MakeGravGridDH(c, MARS["gm"], MARS["r0"], sampling=sampling, lmax_calc=lc,
                                extend=extend, **kw)
        ref = oracle.makegravgrid_dh(c, MARS["gm"], MARS["r0"], sampling=sampling,
                                     lmax_calc=lc, extend=extend, **kw)
        check(g, ref)


def test_grav_lmax719_and_batch(cuda, oracle):
    """Config-3 size (lmax 719, sampling 2), three fields in one call: each
    equals its own oracle run and the single-field call bit for bit."""
    L = 719
    cs = np.stack([oracle.power_law_cilm(L, 111 + i) * 1e-3 for i in range(3)])
    cs[:, 0, 0, 0] = 1.0
    kw = dict(a=MARS["a"], f=MARS["f"], omega=MARS["omega"], normal_gravity=1)
    g = cuda.MakeGravGridDH(torch.from_numpy(cs).cuda(), MARS["gm"], MARS["r0"], **kw)
    ref = oracle.makegravgrid_dh(cs[1], MARS["gm"], MARS["r0"], **kw)
    check([x[1] for x in g], ref)
    g0 = cuda.MakeGravGridDH(cs[0], MARS["gm"], MARS["r0"], **kw)
    for a, b in zip(g0, g):
        assert torch.equal(a, b[0])


@pytest.mark.parametrize("F", [2, 4, 8])
def test_grav_grouped_fields(cuda, oracle, F):
    """2, 4 and 8 fields: their 6, 12 and 24 sums share recursions in groups
    of 2, 4 and 8 (across fields); each field equals its single-field call
    and the oracle."""
    L = 95
    cs = np.stack([oracle.power_law_cilm(L, 120 + i) * 1e-3 for i in range(F)])
    cs[:, 0, 0, 0] = 1.0
    kw = dict(a=MARS["a"], f=MARS["f"], omega=MARS["omega"], normal_gravity=1)
    g = cuda.MakeGravGridDH(torch.from_numpy(cs).cuda(), MARS["gm"], MARS["r0"], **kw)
    for i in (0, F - 1):
        gi = cuda.MakeGravGridDH(cs[i], MARS["gm"], MARS["r0"], **kw)
        for a, b in zip(gi, g):
            assert rel(b[i].cpu().numpy(), a.cpu().numpy()) <= 1e-14
    check([x[F - 1] for x in g], oracle.makegravgrid_dh(cs[F - 1], MARS["gm"], MARS["r0"], **kw))


def test_grav_default_arguments(cuda, oracle):
    """pyshtools defaults: a = r0, f = 0, sampling 2, omega 0, normal gravity
    removed with GM."""
    c = oracle.power_law_cilm(20, 112) * 1e-3
    c[0, 0, 0] = 1.0
    g = cuda.MakeGravGridDH(c, MARS["gm"], MARS["r0"])
    ref = oracle.makegravgrid_dh(c, MARS["gm"], MARS["r0"], sampling=2, omega=0.0,
                                 normal_gravity=1)
    check(g, ref)
    from shtools_b200 import backend
    gb = backend.MakeGravGridDH(c, MARS["gm"], MARS["r0"], normal_gravity_gm=MARS["gm"] * 1.01,
                                f=MARS["f"], omega=MARS["omega"])
    refb = oracle.makegravgrid_dh(c, MARS["gm"], MARS["r0"], f=MARS["f"], omega=MARS["omega"],
                                  normal_gravity=1, normal_gravity_gm=MARS["gm"] * 1.01)
    check(gb, refb)
    # f2py semantics of the backend: None takes the default (omega 0.0)
    gn = backend.MakeGravGridDH(c, MARS["gm"], MARS["r0"], omega=None, normal_gravity=0,
                                f=None, sampling=None)
    refn = oracle.makegravgrid_dh(c, MARS["gm"], MARS["r0"], sampling=2, omega=0.0)
    check(gn, refn)


def test_normal_gravity_matches_oracle(cuda, oracle):
    w = dict(gm=3986004.418e8, a=6378137.0, omega=7292115e-11)
    b = w["a"] * (1 - 1 / 298.257223563)
    for lat in (-90.0, -37.5, 0.0, 12.25, 45.0, 89.0, 90.0):
        for bb, om in ((b, w["omega"]), (w["a"], w["omega"]), (w["a"], 0.0)):
            got = cuda.NormalGravity(lat, w["gm"], om, w["a"], bb)
            ref = oracle.normal_gravity(lat, w["gm"], om, w["a"], bb)
            assert abs(got - ref) <= 1e-14 * ref


def test_grav_dropin(cuda, oracle):
    from shtools_b200 import _lib
    lib = _lib.load()
    L = 24
    c = oracle.power_law_cilm(L, 113) * 1e-3
    c[0, 0, 0] = 1.0
    cf = np.asfortranarray(c)
    n = 2 * L + 2
    grids = [np.zeros((n + 1, 2 * n + 1), order="F") for _ in range(5)]
    D = ctypes.POINTER(ctypes.c_double)
    st, nn = ctypes.c_int(-1), ctypes.c_int(0)
    samp, ext, ng = ctypes.c_int(2), ctypes.c_int(1), ctypes.c_int(1)
    om = ctypes.c_double(MARS["omega"])
    lib.MakeGravGridDH(cf.ctypes.data_as(D), L + 1, L, MARS["gm"], MARS["r0"], MARS["a"],
                       MARS["f"], grids[0].ctypes.data_as(D), 2 * n + 1, n + 1,
                       grids[1].ctypes.data_as(D), grids[2].ctypes.data_as(D),
                       grids[3].ctypes.data_as(D), ctypes.byref(nn), ctypes.byref(samp), None,
                       ctypes.byref(om), ctypes.byref(ng), grids[4].ctypes.data_as(D),
                       ctypes.byref(ext), ctypes.byref(st))
    assert st.value == 0 and nn.value == n
    ref = oracle.makegravgrid_dh(c, MARS["gm"], MARS["r0"], a=MARS["a"], f=MARS["f"],
                                 sampling=2, extend=1, omega=MARS["omega"], normal_gravity=1)
    check(grids, ref)
    # normal gravity without omega: the reference's exit status 5
    lib.MakeGravGridDH(cf.ctypes.data_as(D), L + 1, L, MARS["gm"], MARS["r0"], MARS["a"],
                       MARS["f"], grids[0].ctypes.data_as(D), 2 * n + 1, n + 1,
                       grids[1].ctypes.data_as(D), grids[2].ctypes.data_as(D),
                       grids[3].ctypes.data_as(D), ctypes.byref(nn), ctypes.byref(samp), None,
                       None, ctypes.byref(ng), None, ctypes.byref(ext), ctypes.byref(st))
    assert st.value == 5
    # without pot
    st.value = -1
    g4 = [np.zeros((n, n), order="F") for _ in range(4)]
    one = ctypes.c_int(1)
    lib.MakeGravGridDH(cf.ctypes.data_as(D), L + 1, L, MARS["gm"], MARS["r0"], MARS["a"],
                       MARS["f"], g4[0].ctypes.data_as(D), n, n, g4[1].ctypes.data_as(D),
                       g4[2].ctypes.data_as(D), g4[3].ctypes.data_as(D), ctypes.byref(nn),
                       ctypes.byref(one), None, None, None, None, None, ctypes.byref(st))
    assert st.value == 0
    ref = oracle.makegravgrid_dh(c, MARS["gm"], MARS["r0"], a=MARS["a"], f=MARS["f"],
                                 sampling=1, pot=False)
    for got, r in zip(g4[:3], ref[:3]):
        assert rel(got, r) <= GRID_TOL


def test_grav_errors(cuda):
    c = np.zeros((2, 5, 5))
    with pytest.raises(ValueError):
        cuda.MakeGravGridDH(c, 1.0, 1.0, sampling=3)
    with pytest.raises(ValueError):
        cuda.MakeGravGridDH(c, 1.0, 1.0, omega=None, normal_gravity=1)
    with pytest.raises(ValueError):
        cuda.MakeGravGridDH(c, 1.0, 1.0, normal_gravity=2)
