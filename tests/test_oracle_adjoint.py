"""The oracle's transposes of the four real transforms (the FP64 adjoints the
GPU autograd backward passes are checked against): the dot-product identity
<S c, y> = <c, S^T y> against the oracle's own forward transforms for DH
(sampling 1 and 2, with and without the extend row and column) and GLQ, every
normalisation and both Condon-Shortley phases, and lmax_calc < lmax."""
import numpy as np
import pytest


def _masked(rng, L):
    c = rng.standard_normal((2, L + 1, L + 1))
    l = np.arange(L + 1)
    c *= (l[:, None] >= l[None, :])
    c[1, :, 0] = 0.0
    return c


def _dot_err(a, x, b, y):
    """|<a, x> - <b, y>| relative to the Cauchy-Schwarz scale of both sides."""
    lhs = float((a * x).sum())
    rhs = float((b * y).sum())
    scale = np.linalg.norm(a) * np.linalg.norm(x) + np.linalg.norm(b) * np.linalg.norm(y)
    return abs(lhs - rhs) / scale


@pytest.mark.parametrize("norm", [1, 2, 3, 4])
@pytest.mark.parametrize("csphase", [1, -1])
@pytest.mark.parametrize("sampling,extend", [(1, 0), (1, 1), (2, 0), (2, 1)])
def test_dh_adjoints_dot_identity(oracle, norm, csphase, sampling, extend):
    rng = np.random.default_rng(10 * norm + sampling + 100 * extend + (csphase > 0))
    L = 17
    c = _masked(rng, L)
    g = oracle.makegrid_dh(c, norm=norm, sampling=sampling, csphase=csphase,
                           extend=extend)
    y = rng.standard_normal(g.shape)
    a = oracle.makegrid_dh_adjoint(y, L, norm=norm, sampling=sampling,
                                   csphase=csphase, extend=extend)
    assert _dot_err(g, y, a, c) <= 1e-14
    # the transpose touches only the coefficients the synthesis reads
    assert np.all(a[1, :, 0] == 0.0)
    assert np.all(np.triu(a[0], 1) == 0.0) and np.all(np.triu(a[1], 1) == 0.0)
    n = 2 * L + 2
    gg = rng.standard_normal((n, sampling * n))
    cc = _masked(rng, L)
    an = oracle.shexpand_dh(gg, norm=norm, sampling=sampling, csphase=csphase)
    ad = oracle.shexpand_dh_adjoint(cc, n, norm=norm, sampling=sampling,
                                    csphase=csphase)
    assert ad.shape == gg.shape
    assert _dot_err(an, cc, ad, gg) <= 1e-14


@pytest.mark.parametrize("norm", [1, 2, 3, 4])
@pytest.mark.parametrize("csphase", [1, -1])
@pytest.mark.parametrize("extend", [0, 1])
def test_glq_adjoints_dot_identity(oracle, norm, csphase, extend):
    rng = np.random.default_rng(7 + norm + 10 * extend + (csphase > 0))
    L = 16
    z, w = oracle.shglq(L)
    c = _masked(rng, L)
    g = oracle.makegrid_glq(c, zero=z, norm=norm, csphase=csphase, extend=extend)
    y = rng.standard_normal(g.shape)
    a = oracle.makegrid_glq_adjoint(y, L, zero=z, norm=norm, csphase=csphase,
                                    extend=extend)
    assert _dot_err(g, y, a, c) <= 1e-14
    gq = rng.standard_normal((L + 1, 2 * L + 1))
    cc = _masked(rng, L)
    an = oracle.shexpand_glq(gq, w=w, zero=z, norm=norm, csphase=csphase)
    ad = oracle.shexpand_glq_adjoint(cc, L, w=w, zero=z, norm=norm, csphase=csphase)
    assert _dot_err(an, cc, ad, gq) <= 1e-14


def test_adjoints_lmax_calc(oracle):
    """Truncated transforms: the transposes honour lmax_calc."""
    rng = np.random.default_rng(3)
    L, Lc = 20, 11
    c = _masked(rng, L)
    g = oracle.makegrid_dh(c, sampling=2, lmax_calc=Lc)
    y = rng.standard_normal(g.shape)
    a = oracle.makegrid_dh_adjoint(y, L, sampling=2, lmax_calc=Lc)
    assert np.all(a[:, Lc + 1:, :] == 0.0)
    assert _dot_err(g, y, a, c) <= 1e-14
    n = 2 * L + 2
    gg = rng.standard_normal((n, 2 * n))
    cc = _masked(rng, Lc)
    an = oracle.shexpand_dh(gg, sampling=2, lmax_calc=Lc)
    ad = oracle.shexpand_dh_adjoint(cc, n, sampling=2, lmax_calc=Lc)
    assert _dot_err(an, cc, ad, gg) <= 1e-14
    z, w = oracle.shglq(L)
    gq = oracle.makegrid_glq(c, zero=z, lmax_calc=Lc)
    yq = rng.standard_normal(gq.shape)
    aq = oracle.makegrid_glq_adjoint(yq, L, zero=z, lmax_calc=Lc)
    assert _dot_err(gq, yq, aq, c) <= 1e-14


def test_adjoint_small_is_explicit_transpose(oracle):
    """At lmax 3 the transpose equals the explicit matrix transpose of the
    synthesis built column by column."""
    L = 3
    n = 2 * L + 2
    idx = [(i, l, m) for i in range(2) for l in range(L + 1) for m in range(l + 1)
           if not (i == 1 and m == 0)]
    cols = []
    for (i, l, m) in idx:
        e = np.zeros((2, L + 1, L + 1))
        e[i, l, m] = 1.0
        cols.append(oracle.makegrid_dh(e, sampling=2, extend=1).ravel())
    S = np.stack(cols, axis=1)
    y = np.random.default_rng(5).standard_normal((n + 1, 2 * n + 1))
    a = oracle.makegrid_dh_adjoint(y, L, sampling=2, extend=1)
    ref = S.T @ y.ravel()
    got = np.array([a[i, l, m] for (i, l, m) in idx])
    assert np.abs(got - ref).max() <= 1e-13 * np.abs(ref).max()
