"""The INT8 tensor-core Legendre sums (tcgen05 kind::i8 with an error-free
split of P_lm and the coefficients or ring sums into balanced byte digits:
precision "int8x7", 7 digits and 8 product weights; "int8x6", 6 digits and
7 weights) against the FP64 GPU path, which the parity tests pin to the
oracle: the syntheses (from the recursion or from the plan's P_lm digit
table) and the table-driven analyses and adjoints.

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
def test_table_synthesis_against_recursion(cuda, oracle, kind, L, nf, opts, prec):
    """The table-driven synthesis (the P_lm digits computed once with the
    FP64 kernels' one-step recursion and streamed from device memory) against
    the recursion-driven tensor-core synthesis (same fixed point, same kept
    byte products, a two-step recursion) and the FP64 synthesis; two calls
    give the same bits.  The table skips leading all-zero 256-degree tiles,
    so it is no larger than the padded full size."""
    from shtools_b200 import transforms as T
    c = torch.from_numpy(fields(oracle, L, nf, 500 + L)).cuda()
    f = cuda.MakeGridDH if kind == "dh" else cuda.MakeGridGLQ
    g_rec = f(c, precision=prec, **opts)
    g_tab = f(c, precision=prec + "-table", **opts)
    g64 = f(c, **opts)
    assert cuda.mixed_status() == 0
    scale = g64.abs().amax().item()
    e_rec = (g_tab - g_rec).abs().amax().item() / scale
    e_64 = (g_tab - g64).abs().amax().item() / scale
    assert e_rec <= GRID_TOL and e_64 <= GRID_TOL, (e_rec, e_64)
    # a second call streams the same table
    assert torch.equal(f(c, precision=prec + "-table", **opts), g_tab)
    plans = [p for k, p in T._plans.items() if k[-1] == prec + "-table" and k[1] == L]
    assert plans and plans[-1].table_bytes > 0
    p = plans[-1]
    lc = p.lc
    npad = -(-p.info["npair"] // 128) * 128
    # every order's degrees padded to whole 256-degree super-tiles
    full = npad * sum(256 * ((lc - m + 256) // 256) for m in range(lc + 1)) \
        * (7 if prec == "int8x7" else 6)
    assert p.table_bytes <= full
    print("%s %s L %d: table %.1f MB of %.1f MB; grid vs recursion path %.2e, vs FP64 %.2e"
          % (prec, kind, L, p.table_bytes / 2**20, full / 2**20, e_rec, e_64))


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


ANAL_CASES = [
    ("dh", 63, 1, dict(sampling=2)),                                  # N = 16, one field
    ("dh", 127, 6, dict(norm=2, csphase=-1, lmax_calc=100)),          # N = 16
    ("glq", 150, 9, dict(norm=4)),                                    # N = 32, 9 of 16
    ("dh", 200, 16, dict(sampling=2)),                                # N = 32
    ("glq", 255, 20, dict(norm=1, csphase=-1)),                       # 16 + 4 fields
    ("dh", 64, 3, dict(norm=2, lmax_calc=40)),                        # ragged last tiles
    ("dh", 383, 17, dict(sampling=2)),                                # 2 super-tiles, 2 groups
    ("glq", 600, 2, dict()),                                          # 3 super-tiles, N = 16
]


def _grids(cuda, kind, L, c, opts):
    """FP64 grids of the coefficients and the analysis keywords of the case."""
    kw = dict(norm=opts.get("norm", 1), csphase=opts.get("csphase", 1))
    if "lmax_calc" in opts:
        kw["lmax_calc"] = opts["lmax_calc"]
    if kind == "dh":
        samp = opts.get("sampling", 1)
        kw["sampling"] = samp
        g = cuda.MakeGridDH(c, norm=kw["norm"], csphase=kw["csphase"], sampling=samp)
        return g, kw, cuda.SHExpandDH
    g = cuda.MakeGridGLQ(c, norm=kw["norm"], csphase=kw["csphase"])
    return g, kw, cuda.SHExpandGLQ


@pytest.mark.parametrize("prec", ["int8x7", "int8x6"])
@pytest.mark.parametrize("kind,L,nf,opts", ANAL_CASES)
def test_table_analysis_against_fp64(cuda, oracle, kind, L, nf, opts, prec):
    """The tensor-core analysis (the plan's P_lm digit table as the MN-major
    A operand, the ring sums as balanced digits) against the FP64 analysis
    of the same grid, per degree; two calls give the same bits."""
    c = torch.from_numpy(fields(oracle, L, nf, 700 + L)).cuda()
    g, kw, expand = _grids(cuda, kind, L, c, opts)
    a64 = expand(g, **kw)
    amx = expand(g, precision=prec + "-table", **kw)
    assert cuda.mixed_status() == 0
    assert amx.shape == a64.shape
    assert torch.equal(expand(g, precision=prec + "-table", **kw), amx)
    e = perdeg(amx.cpu().numpy(), a64.cpu().numpy())
    print("%s %s L %d x%d: tensor analysis per degree max %.3e" % (prec, kind, L, nf, e.max()))
    assert e.max() <= DEG_TOL[prec], (e.max(), np.unravel_index(e.argmax(), e.shape))
    # the sin coefficients of m = 0 are exactly zero, as in the FP64 path
    assert torch.all(amx[..., 1, :, 0] == 0)


def test_table_analysis_round_trip(cuda, oracle):
    """Mixed synthesis then mixed analysis returns the coefficients (DH
    sampling 2, lmax 300, 12 fields, S(l) = (l+1)^-3)."""
    L = 300
    c = torch.from_numpy(fields(oracle, L, 12, 3100, beta=3.0)).cuda()
    g = cuda.MakeGridDH(c, sampling=2, precision="int8x7-table")
    back = cuda.SHExpandDH(g, sampling=2, precision="int8x7-table")
    ref = cuda.SHExpandDH(cuda.MakeGridDH(c, sampling=2), sampling=2)
    assert cuda.mixed_status() == 0
    e = perdeg(back.cpu().numpy(), c.cpu().numpy())
    e64 = perdeg(ref.cpu().numpy(), c.cpu().numpy())
    print("round trip per degree: int8x7-table %.3e, fp64 %.3e" % (e.max(), e64.max()))
    assert e.max() <= 1e-9


@pytest.mark.parametrize("prec", ["int8x7", "int8x6"])
def test_table_adjoints_against_fp64(cuda, oracle, prec):
    """The adjoints of a mixed plan with its table (autograd backward): the
    synthesis adjoint runs the tensor-core analysis sums with unit weights,
    the analysis adjoint the tensor-core synthesis; both against the FP64
    adjoints, per degree (coefficient gradient) and per grid (grid
    gradient)."""
    L, nf = 191, 5
    c = torch.from_numpy(fields(oracle, L, nf, 41)).cuda()
    y = torch.randn(nf, 2 * L + 2, 2 * (2 * L + 2), dtype=torch.float64, device="cuda")
    grads = {}
    for p in ("fp64", prec + "-table"):
        cc = c.clone().requires_grad_(True)
        g = cuda.MakeGridDH(cc, sampling=2, precision=p)
        (g * y).sum().backward()
        gg = g.detach().clone().requires_grad_(True)
        a = cuda.SHExpandDH(gg, sampling=2, precision=p)
        (a * c).sum().backward()
        grads[p] = (cc.grad.clone(), gg.grad.clone())
    assert cuda.mixed_status() == 0
    gc64, gg64 = grads["fp64"]
    gcm, ggm = grads[prec + "-table"]
    e = perdeg(gcm.cpu().numpy(), gc64.cpu().numpy())
    eg = ((ggm - gg64).abs().amax() / gg64.abs().amax()).item()
    print("%s adjoints: synthesis adjoint per degree %.3e, analysis adjoint grid %.3e"
          % (prec, e.max(), eg))
    assert e.max() <= DEG_TOL[prec]
    assert eg <= GRID_TOL


def test_table_analysis_lmax2799_16_fields(cuda, oracle):
    """The configuration of the precision target: 16 DH fields at lmax 2799,
    sampling 2 (5600 x 11200), S(l) = (l+1)^-3; per-degree error of the
    tensor-core analysis (int8x7 and int8x6 from the plan's table) against
    the FP64 analysis of the same FP64 grid.  Each table is freed before the
    next one is built (56 GB for int8x7)."""
    from shtools_b200 import transforms as T
    L, nf = 2799, 16
    c = torch.from_numpy(fields(oracle, L, nf, 5000, beta=3.0)).cuda()
    g = cuda.MakeGridDH(c, sampling=2)
    del c
    a64 = cuda.SHExpandDH(g, sampling=2).cpu().numpy()
    for prec in ("int8x7", "int8x6"):
        amx = cuda.SHExpandDH(g, sampling=2, precision=prec + "-table")
        assert cuda.mixed_status() == 0
        e = perdeg(amx.cpu().numpy(), a64)
        del amx
        print("%s-table lmax 2799 x16 tensor analysis: per degree max %.3e (degree %d)"
              % (prec, e.max(), int(np.unravel_index(e.argmax(), e.shape)[-1])))
        for k, p in list(T._plans.items()):
            if k[-1] == prec + "-table" and k[1] == L:
                p.legendre_table(False)
                del T._plans[k]
        assert e.max() <= DEG_TOL[prec], (prec, e.max())


def test_bounded_wait_records_timeout_and_context_survives(cuda, oracle):
    """A tensor-core wait that never completes (an mbarrier nothing arrives
    on, shtc_mixed_wait_selftest) gives up, records SHTC_ETIMEOUT, and the
    next status read returns it once; the context stays usable: a mixed
    transform afterwards is correct and reports status 0."""
    import time
    from shtools_b200 import _lib
    from shtools_b200.transforms import _stream_ptr
    lib = _lib.load()
    assert cuda.mixed_status() == 0
    t0 = time.perf_counter()
    _lib.check(lib.shtc_mixed_wait_selftest(_stream_ptr(torch.device("cuda", 0))),
               "shtc_mixed_wait_selftest")
    waited = time.perf_counter() - t0
    assert cuda.mixed_status() == 10          # SHTC_ETIMEOUT
    assert cuda.mixed_status() == 0           # read and cleared
    c = torch.from_numpy(fields(oracle, 63, 2, 901)).cuda()
    g = cuda.MakeGridDH(c, sampling=2, precision="int8x7")
    g64 = cuda.MakeGridDH(c, sampling=2)
    assert cuda.mixed_status() == 0
    assert ((g - g64).abs().max() / g64.abs().max()).item() <= GRID_TOL
    print("bounded wait gave up after %.2f s" % waited)


def test_backend_precision_switch(cuda, oracle):
    """shtools_b200.backend.set_precision('int8x7-table') routes the numpy
    backend calls (the calls pyshtools' classes make) through the
    tensor-core path: the DH2 round trip of one field stays within the
    mixed tolerances of the FP64 backend; 'fp64' restores the FP64 path
    exactly."""
    from shtools_b200 import backend as B
    L = 95
    c = fields(oracle, L, 1, 333)[0]
    g64 = B.MakeGridDH(c, sampling=2)
    b64 = B.SHExpandDH(g64, sampling=2)
    try:
        B.set_precision("int8x7-table")
        gmx = B.MakeGridDH(c, sampling=2)
        bmx = B.SHExpandDH(gmx, sampling=2)
    finally:
        B.set_precision("fp64")
    assert cuda.mixed_status() == 0
    assert np.abs(gmx - g64).max() / np.abs(g64).max() <= GRID_TOL
    assert perdeg(bmx, b64).max() <= DEG_TOL["int8x7"]
    assert not np.array_equal(gmx, g64)
    assert np.array_equal(B.MakeGridDH(c, sampling=2), g64)
