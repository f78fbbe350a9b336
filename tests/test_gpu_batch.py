"""GPU tests of the batched transforms of many fields on several grids
(GLQ fields of uneven lmax, the persistent-launch path): every field agrees
with its single-plan transform and with the oracle, and a CUDA-graph replay
reproduces the eager result."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _power_law(oracle, L, seed):
    return oracle.power_law_cilm(L, seed)


def _rel(a, b):
    a = a.detach().cpu().numpy() if isinstance(a, torch.Tensor) else np.asarray(a)
    b = b.detach().cpu().numpy() if isinstance(b, torch.Tensor) else np.asarray(b)
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def test_batch_glq_uneven_matches_single(cuda, oracle):
    from shtools_b200.batch import Batch
    lmaxes = [7, 15, 15, 16, 31, 31, 31, 40, 63, 64, 63, 2, 1, 0, 127, 100]
    b = Batch.glq(lmaxes)
    cilms = [_power_law(oracle, L, 500 + i) for i, L in enumerate(lmaxes)]
    flat = b.pack_cilm(cilms)
    grids = b.synthesis(flat)
    back = b.analysis(grids)
    torch.cuda.synchronize()
    for i, L in enumerate(lmaxes):
        ref = cuda.MakeGridGLQ(torch.from_numpy(cilms[i]).cuda())
        g = b.grid_view(grids, i)
        assert g.shape == ref.shape
        assert _rel(g, ref) <= 1e-13, (i, L)
        refb = cuda.SHExpandGLQ(ref)
        assert _rel(b.cilm_view(back, i), refb) <= 1e-13, (i, L)
    # one field against the oracle
    i = lmaxes.index(63)
    z, w = oracle.shglq(63)
    go = oracle.makegrid_glq(cilms[i], zero=z)
    assert _rel(b.grid_view(grids, i), go) <= 1e-12


def test_batch_graph_replay(cuda, oracle):
    from shtools_b200.batch import Batch
    rng = np.random.default_rng(4)
    lmaxes = [int(x) for x in rng.integers(31, 96, 40)]
    b = Batch.glq(lmaxes)
    flat = b.pack_cilm([_power_law(oracle, L, 900 + i) for i, L in enumerate(lmaxes)])
    eager = b.synthesis(flat)
    g, sin, sout = b.graph("synthesis")
    sin.copy_(flat)
    g.replay()
    torch.cuda.synchronize()
    assert torch.equal(sout, eager)
    ga, ain, aout = b.graph("analysis")
    ain.copy_(eager)
    ga.replay()
    torch.cuda.synchronize()
    assert torch.equal(aout, b.analysis(eager))
    # replays with new inputs track the inputs
    sin.mul_(2.0)
    g.replay()
    torch.cuda.synchronize()
    assert torch.allclose(sout, 2.0 * eager, rtol=0, atol=1e-13 * eager.abs().max().item())


def _glq_perdeg(a, b):
    num = np.sqrt(((np.asarray(a) - b) ** 2).sum(axis=(0, 2)))
    den = np.sqrt((np.asarray(b) ** 2).sum(axis=(0, 2)))
    den[den == 0] = 1.0
    return num / den


def test_config4_uneven_glq_at_size(cuda, oracle):
    """The batched uneven GLQ configuration at its size: 256 fields with lmax
    drawn from [31, 511] (seeded) plus chosen lmax whose longitude lengths
    2 lmax + 1 take Bluestein's algorithm (prime factors above 13: 73, 511 =
    7 * 73, 1023 = 3 * 11 * 31) and the radix-11/13 passes (121, 169, 1001 =
    7 * 11 * 13).  Every field against its single-plan transform (synthesis
    grid and analysis coefficients), and 16 fields spread over the range
    against the oracle's full GLQ transforms (SHExpandGLQ.f95:445-649,
    MakeGridGLQ.f95:547-665): grid <= 1e-12, per degree <= 1e-11."""
    from shtools_b200.batch import Batch
    rng = np.random.default_rng(4000)
    chosen = [36, 255, 511, 60, 84, 500, 31]
    lmaxes = [int(x) for x in rng.integers(31, 512, 256 - len(chosen))] + chosen
    b = Batch.glq(lmaxes)
    cilms = [_power_law(oracle, L, 4100 + i) for i, L in enumerate(lmaxes)]
    grids = b.synthesis(b.pack_cilm(cilms))
    back = b.analysis(grids)
    torch.cuda.synchronize()
    for i, L in enumerate(lmaxes):
        ref = cuda.MakeGridGLQ(torch.from_numpy(cilms[i]).cuda())
        assert _rel(b.grid_view(grids, i), ref) <= 1e-13, (i, L)
        refb = cuda.SHExpandGLQ(ref)
        assert _rel(b.cilm_view(back, i), refb) <= 1e-13, (i, L)
    # 16 fields against the oracle: the chosen ones and 9 more spread over the range
    order = np.argsort(lmaxes[:-len(chosen)])
    spread = [int(order[k]) for k in np.linspace(0, len(order) - 1, 9).astype(int)]
    picks = spread + list(range(len(lmaxes) - len(chosen), len(lmaxes)))
    assert len(picks) == 16
    # the batch analysis runs on the oracle's grids of the picked fields
    g_in = grids.clone()
    ref_grids = {}
    for i in picks:
        L = lmaxes[i]
        z, w = oracle.shglq(L)
        go = oracle.makegrid_glq(cilms[i], zero=z)
        assert _rel(b.grid_view(grids, i), go) <= 1e-12, (i, L)
        b.grid_view(g_in, i).copy_(torch.from_numpy(go))
        ref_grids[i] = (go, z, w)
    back2 = b.analysis(g_in)
    torch.cuda.synchronize()
    for i in picks:
        go, z, w = ref_grids[i]
        bo = oracle.shexpand_glq(go, w=w, zero=z)
        e = _glq_perdeg(b.cilm_view(back2, i).cpu().numpy(), bo)
        assert e.max() <= 1e-11, (i, lmaxes[i], e.max())
