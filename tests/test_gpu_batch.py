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
