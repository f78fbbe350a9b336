"""GPU test of shtc_synthesis_noalloc, the synthesis entry point that
allocates nothing (its workspace is a fixed array inside libshtcuda).  It is
meant for callers that must not allocate device memory inside their own
calls, such as programs whose GPU memory belongs to a pool or budget manager.

Called through the C ABI and compared with shtc_synthesis, the existing
entry point, on two calls in a row (different plans and inputs), within the
grid tolerance of the parity tests; a transform too large for the fixed
array is rejected.  The file name makes pytest collect it last.
"""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

GRID_TOL = 1e-12          # same grid tolerance as tests/test_gpu_parity.py
SHTC_EWORK = 9

_P = ctypes.c_void_p
_LL = ctypes.c_longlong
_I = ctypes.c_int


def _bind(lib):
    f = lib.shtc_synthesis_noalloc
    f.restype = _I
    f.argtypes = [_P, _P, _LL, _LL, _LL, _LL, _I, _P, _LL, _LL, _LL, _I, _P]
    return f


def _power_law(L, seed, nfield):
    rng = np.random.default_rng(seed)
    c = rng.standard_normal((nfield, 2, L + 1, L + 1))
    l = np.arange(L + 1)
    c *= np.sqrt((l + 1.0) ** -2 / (2 * l + 1.0))[None, None, :, None]
    c = np.where(l[:, None] >= l[None, :], c, 0.0)
    c[:, 1, :, 0] = 0.0
    return torch.from_numpy(c).cuda()


def _call(fn, plan, c, out):
    st = torch.cuda.current_stream().cuda_stream
    return fn(plan.handle, _P(c.data_ptr()), c.stride(0), c.stride(1),
              c.stride(2), c.stride(3), c.shape[2], _P(out.data_ptr()),
              out.stride(0), out.stride(1), out.stride(2), c.shape[0], _P(st))


def test_noalloc_synthesis_matches_synthesis_twice(cuda):
    from shtools_b200 import _lib
    fn = _bind(_lib.load())
    small = (cuda.get_plan(cuda.GRID_GLQ, 63, 63, 1, 1, 1, 0), _power_law(63, 1, 1))
    # the small plan again after the larger one has filled more of the array:
    # no stale bytes of an earlier call may be read
    cases = [
        small,
        (cuda.get_plan(cuda.GRID_DH, 200, 200, 4, -1, 2, 1), _power_law(200, 2, 2)),
        small,
    ]
    for plan, c in cases:
        ref = plan.synthesis(c)                      # existing entry point
        out = torch.full_like(ref, float("nan"))
        rc = _call(fn, plan, c, out)
        assert rc == 0, _lib.status_string(rc)
        torch.cuda.synchronize()
        err = (out - ref).abs().max().item() / ref.abs().max().item()
        assert err <= GRID_TOL, err


def test_noalloc_rejects_transforms_beyond_the_array(cuda):
    from shtools_b200 import _lib
    lib = _lib.load()
    fn = _bind(lib)
    plan = cuda.get_plan(cuda.GRID_DH, 1023, 1023, 1, 1, 1, 0)
    assert lib.shtc_workspace_bytes(plan.handle, 1) > (16 << 20)
    c = _power_law(1023, 3, 1)
    out = torch.zeros((1, plan.info["nlat_out"], plan.info["nlon_out"]),
                      dtype=torch.float64, device="cuda")
    assert _call(fn, plan, c, out) == SHTC_EWORK
    torch.cuda.synchronize()
    assert out.abs().max().item() == 0.0         # nothing was launched
