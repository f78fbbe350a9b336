"""Autograd of the GPU transforms: the backward passes are the hand-written
adjoint kernels (weighted transpose transforms that recompute P_lm).

Checks: the dot-product identity <A x, y> = <x, A^T y> for all four
transforms, central finite differences of a weighted L2 misfit on random
coefficients, torch.autograd.gradcheck at small lmax, and a short
gradient-descent recovery (the differentiable-DH workload at reduced size).
"""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _rand_cilm(L, seed, batch=()):
    g = torch.Generator(device="cpu").manual_seed(seed)
    c = torch.randn(tuple(batch) + (2, L + 1, L + 1), generator=g, dtype=torch.float64)
    l = torch.arange(L + 1)
    mask = (l[:, None] >= l[None, :]).to(torch.float64)
    c = c * mask
    c[..., 1, :, 0] = 0.0
    return c.cuda()


@pytest.mark.parametrize("kind", ["dh1", "dh2", "dh2e", "glq", "glqe"])
@pytest.mark.parametrize("norm", [1, 2, 4])
def test_dot_product_identity(cuda, kind, norm):
    L = 23
    x = _rand_cilm(L, 1, (2,))
    ext = kind.endswith("e")
    if kind.startswith("dh"):
        samp = 2 if "2" in kind else 1
        synth = lambda c: cuda.MakeGridDH(c, sampling=samp, norm=norm, extend=ext)
        anal = lambda g: cuda.SHExpandDH(g, sampling=samp, norm=norm)
    else:
        synth = lambda c: cuda.MakeGridGLQ(c, norm=norm, extend=ext)
        anal = lambda g: cuda.SHExpandGLQ(g, norm=norm)
    # synthesis: <S x, y> = <x, S^T y>
    xr = x.clone().requires_grad_(True)
    g = synth(xr)
    y = torch.randn_like(g)
    (g * y).sum().backward()
    lhs = (g.detach() * y).sum().item()
    rhs = (xr.grad * x).sum().item()
    assert abs(lhs - rhs) <= 1e-12 * max(1.0, abs(lhs))
    # analysis: <A y, c> = <y, A^T c>
    nlat = g.shape[-2]
    nlon = g.shape[-1] - (1 if ext else 0)
    if kind.startswith("dh"):
        nlat = nlat - (1 if ext else 0)
    yy = torch.randn(2, nlat, nlon, dtype=torch.float64, device="cuda",
                     requires_grad=True)
    cc = anal(yy)
    w = torch.randn_like(cc)
    (cc * w).sum().backward()
    lhs = (cc.detach() * w).sum().item()
    rhs = (yy.grad * yy.detach()).sum().item()
    assert abs(lhs - rhs) <= 1e-12 * max(1.0, abs(lhs))


def test_gradcheck_small(cuda):
    L = 5
    c = _rand_cilm(L, 3).requires_grad_(True)
    assert torch.autograd.gradcheck(lambda t: cuda.MakeGridDH(t, sampling=2), (c,),
                                    eps=1e-6, atol=1e-8)
    g = torch.randn(12, 24, dtype=torch.float64, device="cuda", requires_grad=True)
    assert torch.autograd.gradcheck(lambda t: cuda.SHExpandDH(t, sampling=2), (g,),
                                    eps=1e-6, atol=1e-8)
    g2 = torch.randn(6, 11, dtype=torch.float64, device="cuda", requires_grad=True)
    assert torch.autograd.gradcheck(lambda t: cuda.SHExpandGLQ(t), (g2,),
                                    eps=1e-6, atol=1e-8)


def test_finite_differences_weighted_misfit(cuda):
    """Loss = sum_i w(theta_i) (MakeGridDH(c) - d)^2 on a DH grid; the
    adjoint gradient matches central differences on 64 random coefficients."""
    L = 63
    c = _rand_cilm(L, 5)
    d = cuda.MakeGridDH(_rand_cilm(L, 6), sampling=2)
    n = 2 * L + 2
    wt = torch.sin(torch.pi * torch.arange(n, dtype=torch.float64, device="cuda") / n)
    wt = wt[:, None]

    def loss(t):
        g = cuda.MakeGridDH(t, sampling=2)
        return (wt * (g - d) ** 2).sum()

    cr = c.clone().requires_grad_(True)
    loss(cr).backward()
    grad = cr.grad
    rng = np.random.default_rng(7)
    # the loss is exactly quadratic in c, so central differences carry no
    # truncation error; a large step keeps the rounding error of the loss small
    h = 0.05
    for _ in range(64):
        l = int(rng.integers(0, L + 1))
        m = int(rng.integers(0, l + 1))
        k = int(rng.integers(0, 2)) if m > 0 else 0
        e = torch.zeros_like(c)
        e[k, l, m] = h
        fd = (loss(c + e) - loss(c - e)).item() / (2 * h)
        assert abs(fd - grad[k, l, m].item()) <= 1e-8 * max(1.0, abs(fd))


def test_gradient_descent_recovers_coefficients(cuda):
    """50 steps of gradient descent on the weighted misfit recover the
    coefficients of the data grid (batch of 2 fields).  The step is 1/lambda
    with lambda the largest Hessian eigenvalue from power iteration through
    the adjoint (Hessian-vector products are synthesis + adjoint)."""
    L = 31
    target = _rand_cilm(L, 8, (2,))
    d = cuda.MakeGridDH(target, sampling=2)
    n = 2 * L + 2
    wt = torch.sin(torch.pi * (torch.arange(n, dtype=torch.float64, device="cuda")
                               + 0.5) / n)[:, None]

    def loss_fn(c):
        return (wt * (cuda.MakeGridDH(c, sampling=2) - d) ** 2).sum()

    def hvp(v):
        v = v.detach().requires_grad_(True)
        (wt * cuda.MakeGridDH(v, sampling=2) ** 2).sum().backward()
        return v.grad          # = 2 S^T W S v, the Hessian applied to v

    v = _rand_cilm(L, 9, (2,))
    lam = 0.0
    for _ in range(20):
        hv = hvp(v)
        lam = hv.norm().item() / v.norm().item()
        v = hv / hv.norm()
    c = torch.zeros_like(target)
    first = loss_fn(c).item()
    for _ in range(50):
        cr = c.clone().requires_grad_(True)
        lv = loss_fn(cr)
        lv.backward()
        c = c - cr.grad / lam
    final = loss_fn(c).item()
    assert final < 1e-6 * first
    assert (c - target).abs().max().item() < 1e-3 * target.abs().max().item()


def _perdeg(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    num = np.sqrt(((a - b) ** 2).sum(axis=(0, 2)))
    den = np.sqrt((b ** 2).sum(axis=(0, 2)))
    den[den == 0] = 1.0
    return num / den


@pytest.mark.parametrize("kind", ["dh2", "dh2e", "glq"])
def test_backward_matches_oracle_adjoint(cuda, oracle, kind):
    """Autograd at the lmax 719 sampling-2 configuration against the oracle's
    FP64 transposes of MakeGridDH / SHExpandDH (MakeGridDH.f95:504-639,
    SHExpandDH.f95:463-702) and their GLQ counterparts: the coefficient
    cotangent per degree <= 1e-11, the grid cotangent <= 1e-11 of its
    largest entry.  Two fields per call."""
    L = 719
    ext = kind.endswith("e")
    rng = np.random.default_rng(719)
    cs = [oracle.power_law_cilm(L, 7190 + k) for k in range(2)]
    c = torch.from_numpy(np.stack(cs)).cuda().requires_grad_(True)
    if kind.startswith("dh"):
        g = cuda.MakeGridDH(c, sampling=2, extend=ext)
    else:
        z, w = oracle.shglq(L)
        g = cuda.MakeGridGLQ(c, extend=ext)
    y = rng.standard_normal(tuple(g.shape))
    g.backward(torch.from_numpy(y).cuda())
    gc = c.grad.cpu().numpy()
    for k in range(2):
        if kind.startswith("dh"):
            ref = oracle.makegrid_dh_adjoint(y[k], L, sampling=2, extend=int(ext))
        else:
            ref = oracle.makegrid_glq_adjoint(y[k], L, zero=z, extend=int(ext))
        assert _perdeg(gc[k], ref).max() <= 1e-11, (kind, k)
    # analysis: the grid cotangent of a coefficient cotangent
    n = 2 * L + 2
    shape = (2, n, 2 * n) if kind.startswith("dh") else (2, L + 1, 2 * L + 1)
    gg = torch.from_numpy(rng.standard_normal(shape)).cuda().requires_grad_(True)
    if kind.startswith("dh"):
        cc = cuda.SHExpandDH(gg, sampling=2)
    else:
        cc = cuda.SHExpandGLQ(gg)
    cbar = np.stack([oracle.power_law_cilm(L, 7290 + k) for k in range(2)])
    cc.backward(torch.from_numpy(cbar).cuda())
    gy = gg.grad.cpu().numpy()
    for k in range(2):
        if kind.startswith("dh"):
            ref = oracle.shexpand_dh_adjoint(cbar[k], n, sampling=2)
        else:
            ref = oracle.shexpand_glq_adjoint(cbar[k], L, w=w, zero=z)
        assert np.abs(gy[k] - ref).max() <= 1e-11 * np.abs(ref).max(), (kind, k)
