"""CPU tests of the host-side logic: argument resolution and errors (raised
before any GPU work), the pyshtools backend registration, the benchmark's
workload arithmetic and its multi-rank timing reduction (gloo, 2 ranks)."""
import os
import sys
import types

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_resolve_synth_follows_fortran():
    from shtools_b200.transforms import _resolve_synth
    assert _resolve_synth((2, 11, 11), None, None) == (10, 10)
    assert _resolve_synth((2, 11, 11), 20, None) == (20, 10)      # zero padding
    assert _resolve_synth((2, 11, 11), 20, 15) == (20, 10)
    assert _resolve_synth((2, 11, 11), None, 4) == (10, 4)
    assert _resolve_synth((5, 2, 11, 11), 6, None) == (6, 6)       # batch
    with pytest.raises(ValueError):
        _resolve_synth((2, 11, 11), 10, 11)
    with pytest.raises(ValueError):
        _resolve_synth((2, 11, 10), None, None)
    with pytest.raises(ValueError):
        _resolve_synth((1, 11, 11), None, None)


def test_resolve_analysis():
    from shtools_b200.transforms import _resolve_anal_dh, _resolve_anal_glq
    assert _resolve_anal_dh((512, 1024), 2, None) == (255, 255)
    assert _resolve_anal_dh((512, 512), 1, 100) == (255, 100)
    assert _resolve_anal_dh((3, 512, 1030), 2, None) == (255, 255)  # extra columns ignored
    with pytest.raises(ValueError):
        _resolve_anal_dh((511, 1022), 2, None)
    with pytest.raises(ValueError):
        _resolve_anal_dh((512, 1000), 2, None)
    with pytest.raises(ValueError):
        _resolve_anal_dh((512, 1024), 3, None)
    with pytest.raises(ValueError):
        _resolve_anal_dh((512, 1024), 2, 256)
    assert _resolve_anal_glq((2048, 4095), None) == (2047, 2047)
    with pytest.raises(ValueError):
        _resolve_anal_glq((2048, 4094), None)


def test_errors_raised_before_device_use():
    import shtools_b200 as sht
    c = np.zeros((2, 5, 5))
    for kw in (dict(norm=0), dict(csphase=2), dict(sampling=3), dict(lmax_calc=7)):
        with pytest.raises(ValueError):
            sht.MakeGridDH(c, **kw)
    with pytest.raises(ValueError):
        sht.MakeGridGLQ(c, norm=5)
    with pytest.raises(ValueError):
        sht.SHExpandDH(np.zeros((7, 7)))
    with pytest.raises(ValueError):
        sht.SHExpandGLQ(np.zeros((4, 6)))


def test_backend_module_surface():
    from shtools_b200 import backend
    # the names the pyshtools injectors rebind (expand/__init__.py:91-111,
    # rotate/__init__.py:18-21) all exist
    for name in ("SHExpandGLQ", "SHExpandGLQC", "SHExpandDH", "SHExpandDHC",
                 "MakeGridGLQ", "MakeGridGLQC", "MakeGridDH", "MakeGridDHC",
                 "MakeGradientDH", "SHRotateRealCoef"):
        assert callable(getattr(backend, name))
    # names outside the GPU transforms delegate to the reference backend,
    # which is not importable here
    with pytest.raises(NotImplementedError):
        backend.SHRotateRealCoef(np.zeros((2, 3, 3)), np.zeros(3), np.zeros((4, 4, 4)))


def test_backend_register_into_registry():
    from shtools_b200 import backend
    reg = types.SimpleNamespace(_available_backends={"shtools": object()})
    out = backend.register(reg)
    assert out is reg
    assert reg._available_backends["cuda"] is backend


def test_workload_flops():
    sys.path.insert(0, ROOT)
    import bench
    w = bench.WORKLOADS["glq2047"]
    # 8 flops per ring pair and (l, m): 1024 pairs, 2048*2049/2 (l, m)
    assert bench.flops_per_transform(w) == 8.0 * 1024 * (2048 * 2049 // 2)
    w5 = bench.WORKLOADS["dh2799x16"]
    assert bench.flops_per_transform(w5) == 8.0 * 2800 * (2800 * 2801 // 2)


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    sys.path.insert(0, ROOT)
    import bench
    v = bench.max_over_ranks(10.0 + rank)
    out.put((rank, v))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_gloo_two_ranks():
    """The replicas of a multi-GPU bench run report the slowest rank's time;
    exercised with two gloo ranks on the CPU."""
    import multiprocessing as mp
    import socket
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = dict(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res == {0: 11.0, 1: 11.0}
    import bench
    assert bench.max_over_ranks(3.5) == 3.5      # no process group: identity


def test_hostio_threaded_copy_exact():
    """The host side of the pinned staging (shtools_b200.hostio): the copy
    split over threads reproduces the source for sizes below, at and above
    one thread's share, including ragged tails."""
    import numpy as np
    from shtools_b200 import hostio
    rng = np.random.default_rng(11)
    for n in (0, 1, hostio.SLICE_BYTES - 1, hostio.SLICE_BYTES,
              3 * hostio.SLICE_BYTES + 5, 17 * hostio.SLICE_BYTES + 12345):
        src = rng.integers(0, 256, n, dtype=np.uint8)
        dst = np.zeros(n, dtype=np.uint8)
        hostio._copy(dst, src)
        assert np.array_equal(dst, src)


def test_backend_precision_selection():
    """The backend's Legendre arithmetic switch accepts the library's
    precisions only and defaults to FP64 (no GPU needed)."""
    from shtools_b200 import backend as B
    assert B.get_precision() == "fp64"
    try:
        B.set_precision("int8x7-table")
        assert B.get_precision() == "int8x7-table"
        with pytest.raises(ValueError):
            B.set_precision("fp16")
        assert B.get_precision() == "int8x7-table"
    finally:
        B.set_precision("fp64")
    assert B.get_precision() == "fp64"


def test_hostio_pool_returns_buffers_when_views_die():
    """A result buffer goes back to the pinned pool only once the returned
    array and every view of it are gone (plain host tensors stand in for
    pinned ones here)."""
    import gc
    import weakref
    import torch
    from shtools_b200 import hostio as H
    before = H._free_bytes
    buf = torch.empty(96, dtype=torch.uint8)
    arr = buf.view(torch.float64).numpy()
    weakref.finalize(arr, H._give, buf)
    view = arr[3:5]
    del arr
    gc.collect()
    assert H._free_bytes == before
    del view
    gc.collect()
    assert H._free_bytes == before + 96
    assert H._take(96) is buf and H._free_bytes == before


def test_hostio_lower_band_copy():
    """The staged copy of a coefficient array moves each row's entries
    m <= l, for any split of the rows into staging blocks (the band logic of
    shtools_b200.hostio._copy_lower, run on host arrays)."""
    import numpy as np
    from shtools_b200 import hostio as H
    rng = np.random.default_rng(11)
    for n in (1, 5, 37, 64, 300):
        for lead in ((2,), (3, 2)):
            src = rng.standard_normal(lead + (n, n)).reshape(-1, n)
            rows = src.shape[0]
            deg = np.arange(rows) % n
            lower = np.arange(n)[None, :] <= deg[:, None]
            for per in (1, 7, n, rows):
                out = np.full_like(src, np.nan)
                for r0 in range(0, rows, per):
                    nr = min(per, rows - r0)
                    H._copy_lower(out[r0:r0 + nr], src[r0:r0 + nr], r0, n)
                assert np.array_equal(out[lower], src[lower]), (n, lead, per)
