"""Differentiable DH at the size of the reference-sized gradient workload:
8 fields, lmax 719, sampling 2 (1440 x 2880), float64 and float32.

Loss = sum_i w(theta_i) * (MakeGridDH(c) - d)^2, d synthesised from other
seeded power-law coefficients plus N(0, 0.01 rms) noise.  Checks the adjoint
gradient against central differences on 64 random coefficients, the float32
gradient against the float64 one, and 50 steps of gradient descent."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

L, NF = 719, 8


def _fields(oracle, seed0):
    return np.stack([oracle.power_law_cilm(L, seed0 + i) for i in range(NF)])


@pytest.fixture(scope="module")
def problem(oracle):
    import shtools_b200 as sht
    c_true = torch.from_numpy(_fields(oracle, 3000)).cuda()
    d = sht.MakeGridDH(torch.from_numpy(_fields(oracle, 3500)).cuda(), sampling=2)
    rng = np.random.default_rng(3500)
    rms = d.pow(2).mean().sqrt().item()
    d = d + torch.from_numpy(rng.standard_normal(tuple(d.shape)) * 0.01 * rms).cuda()
    n = 2 * L + 2
    wt = torch.sin(torch.pi * (torch.arange(n, dtype=torch.float64, device="cuda") + 0.5)
                   / n)[:, None]
    return c_true, d, wt


def _loss(sht, c, d, wt):
    g = sht.MakeGridDH(c, sampling=2)
    return (wt.to(g.dtype) * (g - d.to(g.dtype)) ** 2).sum()


def test_gradient_vs_central_differences(cuda, problem):
    c_true, d, wt = problem
    c = c_true.clone().requires_grad_(True)
    _loss(cuda, c, d, wt).backward()
    grad = c.grad
    rng = np.random.default_rng(7)
    h = 0.05                      # the loss is exactly quadratic in c
    base = c_true.clone()
    for _ in range(64):
        f = int(rng.integers(0, NF))
        l = int(rng.integers(0, L + 1))
        m = int(rng.integers(0, l + 1))
        k = int(rng.integers(0, 2)) if m > 0 else 0
        e = torch.zeros_like(base)
        e[f, k, l, m] = h
        fd = (_loss(cuda, base + e, d, wt) - _loss(cuda, base - e, d, wt)).item() / (2 * h)
        g = grad[f, k, l, m].item()
        assert abs(fd - g) <= 1e-7 * max(1.0, abs(fd)) + 1e-9 * grad.abs().max().item()


def test_float32_gradient_vs_float64(cuda, problem):
    c_true, d, wt = problem
    c0 = c_true * 0.9
    c64 = c0.clone().requires_grad_(True)
    _loss(cuda, c64, d, wt).backward()
    c32 = c0.float().requires_grad_(True)
    _loss(cuda, c32, d, wt).backward()
    rel = ((c32.grad.double() - c64.grad).norm() / c64.grad.norm()).item()
    assert rel < 1e-4


def test_fifty_steps_of_gradient_descent(cuda, problem):
    c_true, d, wt = problem

    def hvp(v):
        v = v.detach().requires_grad_(True)
        (wt * cuda.MakeGridDH(v, sampling=2) ** 2).sum().backward()
        return v.grad

    v = torch.randn_like(c_true)
    lam = 0.0
    for _ in range(15):
        hv = hvp(v)
        lam = hv.norm().item() / v.norm().item()
        v = hv / hv.norm()
    lam *= 1.05
    c = torch.zeros_like(c_true)
    losses = []
    for _ in range(50):
        cr = c.clone().requires_grad_(True)
        lv = _loss(cuda, cr, d, wt)
        lv.backward()
        losses.append(lv.item())
        c = c - cr.grad / lam
    assert losses[-1] < 1e-3 * losses[0]
