"""GPU parity of transforms whose longitude FFT does not fit in shared memory.

The FFT kernels ping-pong between two buffers of 16 B per point; beyond
7264 points (227 KB of shared memory per CTA) the buffers move to a global
scratch in the caller's workspace, one pair per persistent CTA.  Cases:
  * GLQ lmax 2046: nlon 4093 is prime, Bluestein length 8192 (odd n: two
    rings per complex FFT);
  * DH lmax 1900, sampling 2: nlon 7604, half length 3802 = 2 * 1901,
    Bluestein length 7680 (even n: one ring per half-length FFT);
  * DHC lmax 1819, sampling 2: complex FFT of length 7280 = 2^4*5*7*13
    (mixed radix, no Bluestein);
  * SHMultiply of two lmax-1023 fields (GLQ grid of lmax 2046).
Every grid row and every order is checked against the oracle with a small
lmax_calc (the FFT still runs at full length); the full lmax_calc is checked
on windows of ring pairs and through round trips and adjoint identities.
Tolerances: grids max-abs relative <= 1e-12, coefficients per degree <=
1e-11, round trips per degree <= 1e-9.
"""
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


def test_workspace_carries_fft_scratch(cuda):
    """The long plans report a workspace that holds the FFT scratch (at
    least one CTA's two buffers of the working length) on top of the
    coefficient and Fourier-sum regions."""
    from shtools_b200.transforms import GRID_GLQ, get_plan
    p_short = get_plan(GRID_GLQ, 2047, 2047, 1, 1)   # 4095 = 3^2*5*7*13, fits
    p_long = get_plan(GRID_GLQ, 2046, 2046, 1, 1)    # Bluestein 8192
    grow = p_long.workspace(1)[1] - p_short.workspace(1)[1]
    assert grow >= 2 * 8192 * 16


def test_glq2046_all_rings_low_calc(cuda, oracle):
    L, lc = 2046, 80
    z, w = oracle.shglq(L)
    c = oracle.power_law_cilm(L, 7001)
    g = cuda.MakeGridGLQ(torch.from_numpy(c).cuda(), zero=z, lmax_calc=lc).cpu().numpy()
    gref = oracle.makegrid_glq(c, zero=z, lmax_calc=lc)
    assert g.shape == gref.shape
    assert grid_rel(g, gref) <= GRID_TOL
    rng = np.random.default_rng(7002)
    grid = rng.standard_normal(gref.shape)
    b = cuda.SHExpandGLQ(torch.from_numpy(grid).cuda(), w=w, zero=z,
                         lmax_calc=lc).cpu().numpy()
    bref = oracle.shexpand_glq(grid, w=w, zero=z, lmax_calc=lc)
    e = perdeg(b, bref)
    assert e.max() <= DEG_TOL, (e.max(), e.argmax())


def test_glq2046_float32_grid(cuda, oracle):
    """float32 grids through the global-scratch FFT: within float32
    rounding of the float64 result."""
    L, lc = 2046, 80
    z, _ = oracle.shglq(L)
    c = torch.from_numpy(oracle.power_law_cilm(L, 7003)).cuda()
    g64 = cuda.MakeGridGLQ(c, zero=z, lmax_calc=lc)
    g32 = cuda.MakeGridGLQ(c, zero=z, lmax_calc=lc, dtype=torch.float32)
    assert g32.dtype == torch.float32
    assert ((g32.double() - g64).abs().max() / g64.abs().max()).item() < 1e-6


def test_glq2046_windows_full_calc(cuda, oracle):
    L = 2046
    z, w = oracle.shglq(L)
    nlat = L + 1
    c = oracle.power_law_cilm(L, 7004)
    g = cuda.MakeGridGLQ(torch.from_numpy(c).cuda(), zero=z).cpu().numpy()
    rng = np.random.default_rng(7005)
    grid = np.zeros_like(g)
    pairs = [(0, 2), (500, 502), (1022, 1024)]
    ref = 0.0
    for (lo, hi) in pairs:
        gr = oracle.makegrid_glq(c, zero=z, pair_window=(lo, hi))
        rows = sorted(set(r for p in range(lo, hi) for r in (p, nlat - 1 - p)))
        assert grid_rel(g[rows], gr[rows]) <= GRID_TOL, (lo, hi)
        for r in rows:
            grid[r] = rng.standard_normal(g.shape[1])
    ref = sum(oracle.shexpand_glq(grid, w=w, zero=z, pair_window=pw) for pw in pairs)
    b = cuda.SHExpandGLQ(torch.from_numpy(grid).cuda(), w=w, zero=z).cpu().numpy()
    e = perdeg(b, ref)
    assert e.max() <= DEG_TOL, (e.max(), e.argmax())


def test_glq2046_roundtrip_and_adjoint(cuda, oracle):
    L = 2046
    c = torch.from_numpy(oracle.power_law_cilm(L, 7006)).cuda()
    g = cuda.MakeGridGLQ(c)
    b = cuda.SHExpandGLQ(g)
    e = perdeg(b.cpu().numpy(), c.cpu().numpy())
    assert e.max() < 1e-9
    # <S c, y> = <c, S^T y> through autograd (adjoint FFTs use the scratch too)
    lc = 200
    cl = c[:, :lc + 1, :lc + 1].clone().requires_grad_(True)
    y = torch.randn(g.shape, dtype=torch.float64, device="cuda",
                    generator=torch.Generator("cuda").manual_seed(7007))
    gs = cuda.MakeGridGLQ(cl, lmax=L)
    (gs * y).sum().backward()
    lhs = (gs.detach() * y).sum().item()
    rhs = (cl.detach() * cl.grad).sum().item()
    assert abs(lhs - rhs) <= 1e-11 * abs(lhs)


def test_dh1900_s2_bluestein_even(cuda, oracle):
    L, lc = 1900, 80
    c = oracle.power_law_cilm(L, 7010)
    g = cuda.MakeGridDH(torch.from_numpy(c).cuda(), sampling=2, lmax_calc=lc).cpu().numpy()
    gref = oracle.makegrid_dh(c, sampling=2, lmax_calc=lc)
    assert g.shape == gref.shape == (2 * L + 2, 4 * L + 4)
    assert grid_rel(g, gref) <= GRID_TOL
    rng = np.random.default_rng(7011)
    grid = rng.standard_normal(gref.shape)
    b = cuda.SHExpandDH(torch.from_numpy(grid).cuda(), sampling=2,
                        lmax_calc=lc).cpu().numpy()
    bref = oracle.shexpand_dh(grid, sampling=2, lmax_calc=lc)
    e = perdeg(b, bref)
    assert e.max() <= DEG_TOL, (e.max(), e.argmax())
    # full lmax_calc: rings next to the pole and at the equator
    gf = cuda.MakeGridDH(torch.from_numpy(c).cuda(), sampling=2).cpu().numpy()
    nlat = 2 * L + 2
    for (lo, hi) in [(0, 2), (L, L + 2)]:
        gr = oracle.makegrid_dh(c, sampling=2, pair_window=(lo, hi))
        rows = sorted(set(r for p in range(lo, hi) for r in (p, nlat - p) if r < nlat))
        assert grid_rel(gf[rows], gr[rows]) <= GRID_TOL, (lo, hi)
    bf = cuda.SHExpandDH(torch.from_numpy(gf).cuda(), sampling=2).cpu().numpy()
    assert perdeg(bf, c).max() < 1e-9


def test_dhc1819_s2_long_c2c(cuda, oracle):
    L, lc = 1819, 60
    c = oracle.power_law_cilm_complex(L, 7020)
    ct = torch.from_numpy(c).cuda()
    g = cuda.MakeGridDHC(ct, sampling=2, lmax_calc=lc).cpu().numpy()
    gref = oracle.makegrid_dhc(c, sampling=2, lmax_calc=lc)
    assert g.shape == gref.shape == (2 * L + 2, 4 * L + 4)
    assert grid_rel(g, gref) <= GRID_TOL
    rng = np.random.default_rng(7021)
    grid = rng.standard_normal(gref.shape) + 1j * rng.standard_normal(gref.shape)
    b = cuda.SHExpandDHC(torch.from_numpy(grid).cuda(), sampling=2,
                         lmax_calc=lc).cpu().numpy()
    bref = oracle.shexpand_dhc(grid, sampling=2, lmax_calc=lc)
    e = perdeg(b, bref)
    assert e.max() <= DEG_TOL, (e.max(), e.argmax())
    gf = cuda.MakeGridDHC(ct, sampling=2)
    bf = cuda.SHExpandDHC(gf, sampling=2).cpu().numpy()
    assert perdeg(bf, c).max() < 1e-9


def test_multiply_lmax2046_identity(cuda, oracle):
    """SHMultiply on the lmax-2046 GLQ grid: a product with the constant
    field 1 (c2[0,0,0] = 1) returns the other factor; the product of two
    fields is symmetric in its factors."""
    L1 = L2 = 1023
    c1 = torch.from_numpy(oracle.power_law_cilm(L1, 7030)).cuda()
    one = torch.zeros_like(c1)
    one[0, 0, 0] = 1.0
    p = cuda.SHMultiply(c1, one)
    assert p.shape == (2, L1 + L2 + 1, L1 + L2 + 1)
    pn = p.cpu().numpy()
    e = perdeg(pn[:, :L1 + 1, :L1 + 1], c1.cpu().numpy())
    assert e.max() < 1e-11, e.max()
    assert np.abs(pn[:, L1 + 1:, :]).max() < 1e-12 * np.abs(pn).max()
    c2 = torch.from_numpy(oracle.power_law_cilm(L2, 7031)).cuda()
    a = cuda.SHMultiply(c1, c2).cpu().numpy()
    b = cuda.SHMultiply(c2, c1).cpu().numpy()
    assert np.abs(a - b).max() <= 1e-13 * np.abs(a).max()


def test_batch_rejects_long_fft(cuda):
    """Batched launches keep every ring in shared memory: a plan that needs
    the global scratch is refused at batch creation."""
    from shtools_b200 import _lib
    from shtools_b200.batch import Batch
    with pytest.raises(_lib.SHTCudaError):
        Batch.glq([2046])


def test_long_rings_column_major_grids(cuda, oracle):
    """Rings of 1024 points or more (DH lmax 511, sampling 2: 2048 points,
    one ring per item; GLQ lmax 520: 1041 points, two rings per item) go
    through the direct first / last FFT passes; with column-major grids
    (column stride other than 1) they give the same values as row-major
    grids."""
    from shtools_b200 import transforms as T
    for kind, L in (("dh", 511), ("glq", 520)):
        c = torch.from_numpy(oracle.power_law_cilm(L, 70)[None]).cuda()
        if kind == "dh":
            plan = T.get_plan(T.GRID_DH, L, L, 1, 1, 2, 0)
        else:
            z, w = oracle.shglq(L)
            plan = T.get_plan(T.GRID_GLQ, L, L, 1, 1, 1, 0, zero=z, w=w)
        g = plan.synthesis(c)
        gcm = torch.empty((g.shape[0], g.shape[2], g.shape[1]), dtype=g.dtype,
                          device=g.device).transpose(1, 2)
        assert gcm.stride(2) != 1
        plan.synthesis(c, out=gcm)
        assert torch.equal(gcm, g)
        assert torch.equal(plan.analysis(gcm), plan.analysis(g))


# Even rings of more than 4096 complex points with radices <= 10 run the
# 1024-thread register-capped FFT build with both buffers in shared memory:
# DH lmax 2399, sampling 2, nlon 9600, half length 4800 = 2^6 * 3 * 5^2
# (passes 3, 5, 5, 8, 8); DH lmax 2799, sampling 2, nlon 11200, half length
# 5600 = 2^5 * 5^2 * 7 (radix-10 passes: 10, 10, 7, 8).
@pytest.mark.parametrize("L,extend", [(2399, False), (2399, True), (2799, False)])
def test_dh2399_long_even_fft_all_rings_low_calc(cuda, oracle, L, extend):
    lc = 48
    c = oracle.power_law_cilm(L, 7101)
    ext = 1 if extend else 0
    g = cuda.MakeGridDH(torch.from_numpy(np.stack([c, 2 * c])).cuda(), sampling=2,
                        lmax_calc=lc, extend=extend).cpu().numpy()
    gref = oracle.makegrid_dh(c, sampling=2, lmax_calc=lc, extend=ext)
    assert g.shape[1:] == gref.shape
    assert grid_rel(g[0], gref) <= GRID_TOL
    assert grid_rel(g[1], 2 * gref) <= GRID_TOL
    rng = np.random.default_rng(7102)
    grid = rng.standard_normal((2,) + gref.shape[:1] + (gref.shape[1],))
    n = 2 * L + 2
    b = cuda.SHExpandDH(torch.from_numpy(grid[:, :n, :2 * n]).cuda(), sampling=2,
                        lmax_calc=lc).cpu().numpy()
    for f in range(2):
        bref = oracle.shexpand_dh(np.ascontiguousarray(grid[f, :n, :2 * n]), sampling=2,
                                  lmax_calc=lc)
        e = perdeg(b[f], bref)
        assert e.max() <= DEG_TOL, (f, e.max(), e.argmax())


@pytest.mark.parametrize("L", [2399, 2799])
def test_dh2399_long_even_fft_float32_and_adjoint(cuda, oracle, L):
    """float32 grids through the long even-ring FFTs stay within float32
    rounding of float64; the synthesis adjoint (r2c of the cotangent with
    unit weights) satisfies <S c, y> = <c, S^T y>."""
    lc = 48
    c = torch.from_numpy(oracle.power_law_cilm(L, 7103)).cuda()
    g64 = cuda.MakeGridDH(c, sampling=2, lmax_calc=lc)
    g32 = cuda.MakeGridDH(c, sampling=2, lmax_calc=lc, dtype=torch.float32)
    assert ((g32.double() - g64).abs().max() / g64.abs().max()).item() < 1e-6
    b32 = cuda.SHExpandDH(g32, sampling=2, lmax_calc=lc)
    b64 = cuda.SHExpandDH(g32.double(), sampling=2, lmax_calc=lc)
    assert ((b32.double() - b64).abs().max() / b64.abs().max()).item() < 1e-6
    cc = c.clone().requires_grad_(True)
    g = cuda.MakeGridDH(cc, sampling=2, lmax_calc=lc)
    y = torch.randn_like(g)
    (g * y).sum().backward()
    lhs = (g.detach() * y).sum().item()
    rhs = (cc.grad * c).sum().item()
    assert abs(lhs - rhs) <= 1e-10 * max(1.0, abs(lhs)), (lhs, rhs)
