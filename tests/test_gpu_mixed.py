"""The INT8 tensor-core synthesis (tcgen05 kind::i8 with an error-free split
of P_lm and the coefficients into balanced byte digits: precision "int8x7",
7 digits and 8 product weights; "int8x6", 6 digits and 7 weights) against
the FP64 GPU path, which the parity tests pin to the oracle.

Tolerances of the mixed forms (their errors are stated, not FP64's):
  * per degree: the FP64 analysis of the mixed grid against the FP64
    analysis of the FP64 grid, ||dc_l|| / ||c_l||: int8x7 <= 1e-9 (the bound
    for the non-FP64 forms), int8x6 <= 1e-6 (its measured level at lmax
    2799 is printed);
  * grid: max |grid_mixed - grid_fp64| / max |grid_fp64| <= 1e-9 (a sanity
    bound; the measured values are printed).
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

GRID_TOL = 1e-9
DEG_TOL = {"int8x7": 1e-9, "int8x6": 1e-6}


def perdeg(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    num = np.sqrt(((a - b) ** 2).sum(axis=(-3, -1)))
    den = np.sqrt((b ** 2).sum(axis=(-3, -1)))
    den[den == 0] = 1.0
    return num / den


def fields(oracle, L, nf, seed, beta=2.0):
    return np.stack([oracle.power_law_cilm(L, seed + i, beta=beta) for i in range(nf)])


@pytest.mark.parametrize("prec", ["int8x7", "int8x6"])
@pytest.mark.parametrize("kind,L,nf,opts", [
    ("dh", 63, 1, dict(sampling=2)),                                  # N = 8 columns
    ("dh", 127, 6, dict(norm=2, csphase=-1, lmax_calc=100)),          # N = 16
    ("glq", 150, 8, dict(norm=4, extend=True)),                       # N = 16
    ("dh", 200, 16, dict(sampling=2, extend=True)),                   # N = 32
    ("glq", 255, 20, dict(norm=1, csphase=-1)),                       # 16 + 4 fields
    ("dh", 64, 3, dict(norm=2, lmax_calc=40)),                        # ragged last tiles
])
def test_mixed_synthesis_against_fp64(cuda, oracle, kind, L, nf, opts, prec):
    c = torch.from_numpy(fields(oracle, L, nf, 300 + L)).cuda()
    if kind == "dh":
        g64 = cuda.MakeGridDH(c, **opts)
        gmx = cuda.MakeGridDH(c, precision=prec, **opts)
    else:
        g64 = cuda.MakeGridGLQ(c, **opts)
        gmx = cuda.MakeGridGLQ(c, precision=prec, **opts)
    assert cuda.mixed_status() == 0
    err = ((gmx - g64).abs().amax() / g64.abs().amax()).item()
    # per degree, through the FP64 analysis of both grids
    lc = opts.get("lmax_calc", L)
    ext = 1 if opts.get("extend") else 0
    if kind == "dh":
        samp = opts.get("sampling", 1)
        n = 2 * L + 2
        kw = dict(norm=opts.get("norm", 1), csphase=opts.get("csphase", 1), sampling=samp)
        a64 = cuda.SHExpandDH(g64[..., :n, :samp * n], **kw)
        amx = cuda.SHExpandDH(gmx[..., :n, :samp * n], **kw)
    else:
        kw = dict(norm=opts.get("norm", 1), csphase=opts.get("csphase", 1))
        a64 = cuda.SHExpandGLQ(g64[..., :2 * L + 1], **kw)
        amx = cuda.SHExpandGLQ(gmx[..., :2 * L + 1], **kw)
    e = perdeg(amx[..., :lc + 1, :lc + 1].cpu().numpy(),
               a64[..., :lc + 1, :lc + 1].cpu().numpy())
    print("%s %s L %d x%d: grid %.3e, per degree max %.3e" % (prec, kind, L, nf, err, e.max()))
    assert e.max() <= DEG_TOL[prec], (e.max(), np.unravel_index(e.argmax(), e.shape))
    assert err <= GRID_TOL, err


def test_mixed_synthesis_repeatable_and_plan_precision(cuda, oracle):
    """Two calls give the same bits (the INT32 sums are exact); the plan of
    precision int8x6 is separate from the FP64 plan; norm 3 is refused."""
    L = 95
    c = torch.from_numpy(fields(oracle, L, 4, 77)).cuda()
    a = cuda.MakeGridDH(c, sampling=2, precision="int8x7")
    b = cuda.MakeGridDH(c, sampling=2, precision="int8x7")
    assert torch.equal(a, b)
    g = cuda.MakeGridDH(c, sampling=2)
    assert not torch.equal(a, g)
    with pytest.raises(Exception):
        cuda.MakeGridDH(c, norm=3, precision="int8x7")
    with pytest.raises(ValueError):
        cuda.MakeGridDH(c, precision="fp16")
    assert cuda.mixed_status() == 0


def test_mixed_synthesis_lmax2799_16_fields(cuda, oracle):
    """The configuration of the precision target: 16 DH fields at lmax 2799,
    sampling 2 (5600 x 11200), S(l) = (l+1)^-3; per-degree error of the mixed
    syntheses against the FP64 synthesis, all analysed in FP64."""
    L, nf = 2799, 16
    c = torch.from_numpy(fields(oracle, L, nf, 5000, beta=3.0)).cuda()
    a64 = cuda.SHExpandDH(cuda.MakeGridDH(c, sampling=2), sampling=2).cpu().numpy()
    for prec in ("int8x7", "int8x6"):
        g64 = cuda.MakeGridDH(c, sampling=2)
        gmx = cuda.MakeGridDH(c, sampling=2, precision=prec)
        assert cuda.mixed_status() == 0
        err = ((gmx - g64).abs().amax() / g64.abs().amax()).item()
        del g64
        amx = cuda.SHExpandDH(gmx, sampling=2).cpu().numpy()
        del gmx
        e = perdeg(amx, a64)
        print("%s lmax 2799 x16 mixed synthesis: grid %.3e, per degree max %.3e"
              % (prec, err, e.max()))
        assert e.max() <= DEG_TOL[prec], (prec, e.max())
        assert err <= GRID_TOL, (prec, err)


@pytest.mark.parametrize("prec", ["int8x7", "int8x6"])
@pytest.mark.parametrize("kind,L,nf,opts", [
    ("dh", 63, 1, dict(sampling=2)),                                  # N = 16, one field
    ("dh", 127, 6, dict(norm=2, csphase=-1, lmax_calc=100)),          # N = 16
    ("glq", 150, 9, dict(norm=4, extend=True)),                       # N = 32, 9 of 16
    ("dh", 200, 16, dict(sampling=2, extend=True)),                   # N = 32
    ("glq", 255, 20, dict(norm=1, csphase=-1)),                       # 16 + 4 fields
    ("dh", 64, 3, dict(norm=2, lmax_calc=40)),                        # ragged last tiles
    ("dh", 383, 17, dict(sampling=2)),                                # 3 pair tiles, 2 groups
])
def test_table_synthesis_bit_identical(cuda, oracle, kind, L, nf, opts, prec):
    """The table-driven synthesis (the P_lm digits computed once and streamed
    from device memory) gives the same bits as the recursion-driven one:
    same digits, same kept byte products, exact INT32 sums.  The table skips
    leading all-zero degree tiles, so it is smaller than the full size."""
    from shtools_b200 import transforms as T
    c = torch.from_numpy(fields(oracle, L, nf, 500 + L)).cuda()
    f = cuda.MakeGridDH if kind == "dh" else cuda.MakeGridGLQ
    g_rec = f(c, precision=prec, **opts)
    g_tab = f(c, precision=prec + "-table", **opts)
    assert cuda.mixed_status() == 0
    assert torch.equal(g_tab, g_rec), (g_tab - g_rec).abs().max().item()
    # a second call streams the same table
    assert torch.equal(f(c, precision=prec + "-table", **opts), g_rec)
    plans = [p for k, p in T._plans.items() if k[-1] == prec + "-table" and k[1] == L]
    assert plans and plans[-1].table_bytes > 0
    p = plans[-1]
    lc = p.lc
    npad = -(-p.info["npair"] // 128) * 128
    full = npad * sum(64 * ((lc - m + 64) // 64) for m in range(lc + 1)) \
        * (7 if prec == "int8x7" else 6)
    assert p.table_bytes <= full
    print("%s %s L %d: table %.1f MB of %.1f MB" % (prec, kind, L, p.table_bytes / 2**20,
                                                   full / 2**20))


def test_table_freed_on_precision_switch(cuda, oracle):
    """Switching a plan with a table to the other mixed precision frees the
    table; the syntheses then take the recursion path and stay correct."""
    from shtools_b200 import transforms as T
    L = 95
    p = T.Plan(T.GRID_DH, L, sampling=2)
    p.set_precision(2)
    nb = p.legendre_table(True)
    assert nb > 0 and p.legendre_table(True) == nb          # built once
    c = torch.from_numpy(fields(oracle, L, 4, 91)).cuda()
    g7 = p.synthesis(c)
    p.set_precision(1)
    assert p.table_bytes == 0
    g6 = p.synthesis(c)
    assert cuda.mixed_status() == 0
    ref = cuda.MakeGridDH(c, sampling=2, precision="int8x6")
    assert torch.equal(g6, ref)
    assert (g7 - g6).abs().max().item() <= 1e-9 * g7.abs().max().item()
    p.set_precision(0)
    with pytest.raises(RuntimeError):
        p.legendre_table(True)
