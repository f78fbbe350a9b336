"""CPU tests of the oracle's SHMultiply (oracle/sht_oracle.c): the expansion
of the product of two band-limited fields is exact at degree lmax1+lmax2, so
its grid equals the pointwise product of the two fields' grids (evaluated
independently with scipy), and multiplying by the constant field 1 returns
the other field."""
import numpy as np
import pytest

from test_oracle import grid_known


@pytest.mark.parametrize("norm", [1, 2, 4])
@pytest.mark.parametrize("csphase", [1, -1])
def test_shmultiply_product_of_grids(oracle, norm, csphase):
    L1, L2 = 9, 6
    c1 = oracle.power_law_cilm(L1, 101)
    c2 = oracle.power_law_cilm(L2, 102)
    out = oracle.shmultiply(c1, c2, norm=norm, csphase=csphase)
    assert out.shape == (2, L1 + L2 + 1, L1 + L2 + 1)
    th = np.linspace(0.1, 3.0, 17)
    ph = np.linspace(0.0, 6.0, 23)
    g = grid_known(out, th, ph, norm, csphase, L1 + L2)
    g1 = grid_known(c1, th, ph, norm, csphase, L1)
    g2 = grid_known(c2, th, ph, norm, csphase, L2)
    assert np.abs(g - g1 * g2).max() / np.abs(g1 * g2).max() < 1e-12


def test_shmultiply_by_one(oracle):
    L = 12
    c = oracle.power_law_cilm(L, 103)
    one = np.zeros((2, 1, 1))
    one[0, 0, 0] = 1.0
    out = oracle.shmultiply(c, one)
    assert np.abs(out - c).max() < 1e-13
