"""GPU tests of the multi-field analysis on the FP64 tensor path
(csrc/legendre_mma.cu), which the library takes for 8 or more fields on
grids of at least 256 ring pairs: every field of a batch equals its
single-field analysis (the scalar kernel) to 1e-13 per degree and the
oracle to the 1e-11 gate; field counts that leave a partial field group (12,
20), GLQ and DH grids, the complex transforms and the adjoints (autograd) go
through the same kernel.  The multi-field synthesis (scalar, 8 fields per
recursion) is checked the same way beside it."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def perdeg(a, b):
    num = np.sqrt((np.abs(a - b) ** 2).sum(axis=(0, 2)))
    den = np.sqrt((np.abs(b) ** 2).sum(axis=(0, 2)))
    den[den == 0] = 1.0
    return num / den


@pytest.mark.parametrize("F", [8, 12, 16, 20])
@pytest.mark.parametrize("kind", ["dh", "glq"])
def test_multifield_analysis_matches_single(cuda, oracle, F, kind):
    L = 300 if kind == "dh" else 511
    rng = np.random.default_rng(500 + F)
    if kind == "dh":
        grids = rng.standard_normal((F, 2 * L + 2, 2 * (2 * L + 2)))
        an = lambda g: cuda.SHExpandDH(g, sampling=2)
    else:
        z, w = oracle.shglq(L)
        grids = rng.standard_normal((F, L + 1, 2 * L + 1))
        an = lambda g: cuda.SHExpandGLQ(g, w=w, zero=z)
    gt = torch.from_numpy(grids).cuda()
    batch = an(gt).cpu().numpy()
    for i in (0, F // 2, F - 1):
        single = an(gt[i]).cpu().numpy()
        assert perdeg(batch[i], single).max() <= 1e-13
    ref = oracle.shexpand_dh(grids[F - 1], sampling=2) if kind == "dh" else \
        oracle.shexpand_glq(grids[F - 1], w=w, zero=z)
    assert perdeg(batch[F - 1], ref).max() <= 1e-11


@pytest.mark.parametrize("F", [8, 12, 16, 20])
@pytest.mark.parametrize("kind", ["dh", "glq"])
def test_multifield_synthesis_matches_single(cuda, oracle, F, kind):
    L = 300 if kind == "dh" else 511
    cs = np.stack([oracle.power_law_cilm(L, 600 + i) for i in range(F)])
    ct = torch.from_numpy(cs).cuda()
    if kind == "dh":
        sy = lambda c: cuda.MakeGridDH(c, sampling=2, extend=True)
    else:
        z, _ = oracle.shglq(L)
        sy = lambda c: cuda.MakeGridGLQ(c, zero=z, extend=True)
    batch = sy(ct).cpu().numpy()
    for i in (0, F // 2, F - 1):
        single = sy(ct[i]).cpu().numpy()
        assert np.abs(batch[i] - single).max() <= 1e-13 * np.abs(single).max()
    # full grid against the oracle for one field (lmax 300) or ring-pair windows
    if kind == "dh":
        ref = oracle.makegrid_dh(cs[F - 1], sampling=2, extend=1)
    else:
        ref = oracle.makegrid_glq(cs[F - 1], zero=z, extend=1)
    assert np.abs(batch[F - 1] - ref).max() <= 1e-12 * np.abs(ref).max()


def test_multifield_complex_and_roundtrip(cuda, oracle):
    """4 complex fields are 8 internal fields: the tensor path; a round trip
    of 16 real fields returns the coefficients."""
    L = 300
    cs = np.stack([oracle.power_law_cilm_complex(L, 510 + i) for i in range(4)])
    g = cuda.MakeGridDHC(torch.from_numpy(cs).cuda(), sampling=2)
    b = cuda.SHExpandDHC(g, sampling=2).cpu().numpy()
    for i in range(4):
        assert perdeg(b[i], cs[i]).max() < 1e-10
    single = cuda.SHExpandDHC(g[2], sampling=2).cpu().numpy()
    assert perdeg(b[2], single).max() <= 1e-13
    c = np.stack([oracle.power_law_cilm(L, 520 + i) for i in range(16)])
    ct = torch.from_numpy(c).cuda()
    back = cuda.SHExpandDH(cuda.MakeGridDH(ct, sampling=2), sampling=2).cpu().numpy()
    for i in (0, 15):
        assert perdeg(back[i], c[i]).max() < 1e-10


def test_multifield_adjoint_identity(cuda):
    """<S x, y> = <x, S^T y> with 8 fields: the backward of the synthesis
    runs the analysis kernel on the cotangent; <A g, c> = <g, A^T c> runs the
    synthesis kernel in the backward of the analysis."""
    L = 300
    g = torch.Generator(device="cuda").manual_seed(530)
    x = torch.randn((8, 2, L + 1, L + 1), dtype=torch.float64, device="cuda", generator=g)
    x = torch.tril(x)            # m <= l
    x[:, 1, :, 0] = 0.0
    xr = x.clone().requires_grad_(True)
    gs = cuda.MakeGridDH(xr, sampling=2)
    y = torch.randn(gs.shape, dtype=torch.float64, device="cuda", generator=g)
    (gs * y).sum().backward()
    lhs = (gs.detach() * y).sum().item()
    rhs = (x * xr.grad).sum().item()
    assert abs(lhs - rhs) <= 1e-11 * abs(lhs)
    gg = torch.randn((8, 2 * L + 2, 2 * (2 * L + 2)), dtype=torch.float64, device="cuda",
                     generator=g).requires_grad_(True)
    cb = cuda.SHExpandDH(gg, sampling=2)
    cc = torch.randn(cb.shape, dtype=torch.float64, device="cuda", generator=g)
    (cb * cc).sum().backward()
    lhs = (cb.detach() * cc).sum().item()
    rhs = (gg.detach() * gg.grad).sum().item()
    assert abs(lhs - rhs) <= 1e-11 * abs(lhs)
