"""GPU parity of SHMultiply (src/SHMultiply.f95) against the oracle, for
every norm and csphase, batched, and through the C drop-in with Fortran
column-major arrays.

Tolerance: max |c_gpu - c_oracle| <= 1e-12 max |c_oracle| (the grid gate of
the transforms, applied to the coefficients), and 1e-11 per degree up to
min(lmax1, lmax2).  Beyond that the product's spectrum is built by
cancellation between much larger terms (at lmax1 = lmax2 = 64 the top
degrees are ~1e-6 of the largest), so a per-degree relative error there
measures that conditioning: rounding noise of 1e-16 of the grid is 1e-10 of
those coefficients in the reference's arithmetic as in ours."""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def perdeg(a, b):
    num = np.sqrt(((a - b) ** 2).sum(axis=(0, 2)))
    den = np.sqrt((b ** 2).sum(axis=(0, 2)))
    den[den == 0] = 1.0
    return num / den


def check(out, ref, lmin):
    assert np.abs(out - ref).max() <= 1e-12 * np.abs(ref).max()
    assert perdeg(out, ref)[:lmin + 1].max() <= 1e-11


@pytest.mark.parametrize("norm", [1, 2, 4])
@pytest.mark.parametrize("csphase", [1, -1])
@pytest.mark.parametrize("L1,L2", [(20, 11), (64, 64), (3, 100)])
def test_multiply_matches_oracle(cuda, oracle, norm, csphase, L1, L2):
    c1 = oracle.power_law_cilm(L1, 110)
    c2 = oracle.power_law_cilm(L2, 111)
    out = cuda.SHMultiply(c1, c2, norm=norm, csphase=csphase).cpu().numpy()
    ref = oracle.shmultiply(c1, c2, norm=norm, csphase=csphase)
    assert out.shape == ref.shape
    check(out, ref, min(L1, L2))


def test_multiply_norm3_small(cuda, oracle):
    c1 = oracle.power_law_cilm(5, 112)
    c2 = oracle.power_law_cilm(6, 113)
    out = cuda.SHMultiply(c1, c2, norm=3).cpu().numpy()
    ref = oracle.shmultiply(c1, c2, norm=3)
    assert np.abs(out - ref).max() / np.abs(ref).max() < 1e-12


def test_multiply_batched_and_larger_arrays(cuda, oracle):
    L = 40
    c1 = np.stack([oracle.power_law_cilm(L, 120 + i) for i in range(3)])
    c2 = np.stack([oracle.power_law_cilm(L, 130 + i) for i in range(3)])
    out = cuda.SHMultiply(torch.from_numpy(c1).cuda(), torch.from_numpy(c2).cuda())
    for i in range(3):
        ref = oracle.shmultiply(c1[i], c2[i])
        check(out[i].cpu().numpy(), ref, L)
    # arrays larger than lmax1/lmax2: only degrees <= lmax are used
    big = np.zeros((2, 60, 60))
    big[:, :L + 1, :L + 1] = c1[0]
    big[:, 50, 3] = 7.0
    o2 = cuda.SHMultiply(big, c2[0], lmax1=L).cpu().numpy()
    check(o2, oracle.shmultiply(c1[0], c2[0]), L)


def test_multiply_dropin(cuda, oracle):
    from shtools_b200 import _lib
    lib = _lib.load()
    L1, L2 = 12, 9
    c1 = np.asfortranarray(oracle.power_law_cilm(L1, 140))
    c2 = np.asfortranarray(oracle.power_law_cilm(L2, 141))
    out = np.zeros((2, L1 + L2 + 1, L1 + L2 + 1), order="F")
    D = ctypes.POINTER(ctypes.c_double)
    st = ctypes.c_int(-1)
    lib.SHMultiply(out.ctypes.data_as(D), L1 + L2 + 1, c1.ctypes.data_as(D), L1 + 1, L1,
                   c2.ctypes.data_as(D), L2 + 1, L2, None, None, None, ctypes.byref(st))
    assert st.value == 0
    ref = oracle.shmultiply(np.ascontiguousarray(c1), np.ascontiguousarray(c2))
    check(out, ref, L2)
