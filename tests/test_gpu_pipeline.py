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


def test_hostio_staged_copies(cuda):
    """numpy <-> device copies through the pinned staging buffers
    (shtools_b200.hostio), at sizes below, at and above the chunk size, are
    exact, and a device result read back right after being computed is the
    computed one."""
    from shtools_b200 import hostio
    rng = np.random.default_rng(7)
    for n in (10, hostio.SMALL_BYTES // 8 + 3, hostio.CHUNK_BYTES // 8,
              5 * hostio.CHUNK_BYTES // 8 + 17):
        a = rng.standard_normal(n)
        t = hostio.to_device(a)
        assert t.is_cuda and torch.equal(t.cpu(), torch.from_numpy(a))
        t2 = t * 3.0
        b = hostio.to_host(t2)
        assert np.array_equal(b, a * 3.0)
    g = hostio.to_device(rng.standard_normal((3, 700, 1401)))
    assert g.shape == (3, 700, 1401) and g.is_contiguous()
    assert np.array_equal(hostio.to_host(g[1]), g[1].cpu().numpy())


def test_hostio_lower_triangle_upload(cuda, oracle):
    """to_device_lower (the backend's cilm upload for the synthesis) gives
    the array with its entries m > l zeroed, through the staged path (one
    and several staging buffers, 3-D and 4-D) and the direct ones (small,
    pinned); the backend's MakeGridDH / MakeGridGLQ results equal those of
    the torch API on the same coefficients."""
    from shtools_b200 import backend as B
    from shtools_b200 import hostio
    rng = np.random.default_rng(21)
    for shape in ((2, 12, 12), (2, 700, 700), (2, 2048, 2048), (3, 2, 1100, 1100)):
        a = rng.standard_normal(shape)
        t = hostio.to_device_lower(a)
        assert t.is_cuda and t.shape == shape
        assert torch.equal(t.cpu(), torch.tril(torch.from_numpy(a)))
    a = rng.standard_normal((2, 900, 900))
    pinned = torch.from_numpy(a).pin_memory()
    t = hostio.to_device_lower(pinned.numpy())
    assert torch.equal(t.cpu(), torch.tril(torch.from_numpy(a)))
    c = oracle.power_law_cilm(300, 2101)
    c_up = c + np.triu(rng.standard_normal(c.shape), 1)   # entries m > l are ignored
    g = B.MakeGridDH(c_up, sampling=2)
    assert np.array_equal(g, cuda.MakeGridDH(torch.from_numpy(c).cuda(), sampling=2).cpu().numpy())
    z, _ = oracle.shglq(300)
    g = B.MakeGridGLQ(c_up, zero=z)
    assert np.array_equal(g, cuda.MakeGridGLQ(torch.from_numpy(c).cuda(), zero=z).cpu().numpy())


def test_hostio_pinned_results_and_staged_large(cuda, monkeypatch):
    """Results come back in pinned memory viewed by numpy; such a result
    passed back in is uploaded directly and stays exact; results above
    PINNED_MAX take the staged path (forced here with a small limit)."""
    from shtools_b200 import hostio
    rng = np.random.default_rng(8)
    a = rng.standard_normal(3 * hostio.CHUNK_BYTES // 8 + 5)
    t = hostio.to_device(a)
    b = hostio.to_host(t * 2.0)
    assert torch.from_numpy(b).is_pinned()
    assert np.array_equal(b, a * 2.0)
    t2 = hostio.to_device(b)
    t2 = t2 + 1.0                           # work queued after the direct upload
    assert np.array_equal(hostio.to_host(t2), a * 2.0 + 1.0)
    # the buffer of a dead result is reused by the next result of its size
    ptr = b.ctypes.data
    del b, t2
    import gc
    gc.collect()
    b2 = hostio.to_host(t * 4.0)
    assert b2.ctypes.data == ptr and np.array_equal(b2, a * 4.0)
    del b2
    monkeypatch.setattr(hostio, "PINNED_MAX", 0)
    c = hostio.to_host(t * 5.0)
    assert not torch.from_numpy(c).is_pinned()
    assert np.array_equal(c, a * 5.0)
