"""GPU tests of float32 arrays (configs with float32 grids / coefficients):
the kernels compute in FP64 and convert on load and store, so a float32
input gives the FP64 result of its (already rounded) values, and a float32
output is the rounded FP64 result."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def test_float32_grid_from_float64_coefficients(cuda, oracle):
    L = 95
    c = oracle.power_law_cilm(L, 31)
    ct = torch.from_numpy(c).cuda()
    g64 = cuda.MakeGridDH(ct, sampling=2)
    g32 = cuda.MakeGridDH(ct, sampling=2, dtype=torch.float32)
    assert g32.dtype == torch.float32
    assert torch.equal(g32, g64.to(torch.float32))       # rounded FP64 result


def test_float32_grid_analysis_equals_fp64_of_rounded_input(cuda, oracle):
    L = 95
    c = oracle.power_law_cilm(L, 32)
    g = cuda.MakeGridDH(torch.from_numpy(c).cuda(), sampling=2, dtype=torch.float32)
    b32in = cuda.SHExpandDH(g, sampling=2, dtype=torch.float64)
    assert b32in.dtype == torch.float64
    ref = oracle.shexpand_dh(g.double().cpu().numpy(), sampling=2)
    e = np.abs(b32in.cpu().numpy() - ref).max() / np.abs(ref).max()
    assert e < 1e-13


def test_float32_everywhere_and_autograd(cuda, oracle):
    L = 47
    c = torch.from_numpy(oracle.power_law_cilm(L, 33)).cuda().float().requires_grad_(True)
    for fn, an in ((lambda x: cuda.MakeGridGLQ(x), lambda g: cuda.SHExpandGLQ(g)),
                   (lambda x: cuda.MakeGridDH(x, sampling=1), lambda g: cuda.SHExpandDH(g))):
        g = fn(c)
        assert g.dtype == torch.float32
        b = an(g)
        assert b.dtype == torch.float32
        rel = ((b.detach().double() - c.detach().double()).norm() / c.detach().double().norm()).item()
        assert rel < 1e-5
        y = torch.randn_like(g)
        (g * y).sum().backward()
        assert c.grad.dtype == torch.float32
        lhs = (g.detach().double() * y.double()).sum().item()
        rhs = (c.grad.double() * c.detach().double()).sum().item()
        assert abs(lhs - rhs) <= 1e-4 * max(1.0, abs(lhs))
        c.grad = None
