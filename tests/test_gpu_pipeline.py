"""Host-buffer pipeline (shtools_b200.pipeline): overlapped copies give the
same results as the device transforms run one at a time."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def test_pipelined_matches_direct(cuda, oracle):
    from shtools_b200.pipeline import pipelined
    L = 127
    cs = [torch.from_numpy(oracle.power_law_cilm(L, 40 + i)).pin_memory() for i in range(5)]
    grids = [cuda.MakeGridGLQ(c.cuda()).cpu().pin_memory() for c in cs]
    outs = [(torch.empty_like(grids[0]).pin_memory(), torch.empty_like(cs[0]).pin_memory())
            for _ in range(5)]
    fn = lambda c, g: (cuda.MakeGridGLQ(c), cuda.SHExpandGLQ(g))
    pipelined(fn, list(zip(cs, grids[::-1])), outs, depth=2)
    torch.cuda.synchronize()
    for i in range(5):
        assert torch.equal(outs[i][0], grids[i])
        ref = cuda.SHExpandGLQ(grids[4 - i].cuda()).cpu()
        assert torch.equal(outs[i][1], ref)


def test_pipelined_reused_outputs_and_errors(cuda, oracle):
    from shtools_b200.pipeline import pipelined
    c = torch.from_numpy(oracle.power_law_cilm(31, 7)).pin_memory()
    out = (torch.empty(32, 63, dtype=torch.float64).pin_memory(),)
    pipelined(lambda x: cuda.MakeGridGLQ(x), [(c,)] * 4, [out] * 4, depth=3)
    torch.cuda.synchronize()
    assert torch.equal(out[0], cuda.MakeGridGLQ(c.cuda()).cpu())
    with pytest.raises(ValueError):
        pipelined(lambda x: x, [(c,)], [], depth=2)
    with pytest.raises(ValueError):
        pipelined([lambda x: x] * 2, [(c,)], [(c,)], depth=2)


def test_pipelined_alternating_step_kinds(cuda, oracle):
    """Synthesis and analysis as separate steps of one pipeline (inputs of
    two shapes, each with its own rotation of device buffers): the same
    results as the transforms run one at a time."""
    from shtools_b200.pipeline import pipelined
    L = 95
    cs = [torch.from_numpy(oracle.power_law_cilm(L, 60 + i)).pin_memory() for i in range(3)]
    grids = [cuda.MakeGridGLQ(c.cuda()).cpu().pin_memory() for c in cs]
    ins, outs = [], []
    for i in range(3):
        ins += [(cs[i],), (grids[2 - i],)]
        outs += [(torch.empty_like(grids[0]).pin_memory(),),
                 (torch.empty_like(cs[0]).pin_memory(),)]
    fns = [lambda t: cuda.MakeGridGLQ(t), lambda t: cuda.SHExpandGLQ(t)] * 3
    pipelined(fns, ins, outs, depth=2)
    torch.cuda.synchronize()
    for i in range(3):
        assert torch.equal(outs[2 * i][0], grids[i])
        assert torch.equal(outs[2 * i + 1][0], cuda.SHExpandGLQ(grids[2 - i].cuda()).cpu())
