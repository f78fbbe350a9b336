"""Torch front end of the CUDA transforms: plans, device tensors, batches and
autograd.

Functions take and return CUDA tensors (float64).  A leading batch of fields
is allowed: cilm of shape (..., 2, D, D), grids of shape (..., nlat, nlon).
Argument names, defaults and lmax / lmax_calc resolution follow the
reference's Python API (src/pyshtools.pyf:235-376 and the Fortran routines):

    MakeGridDH (cilm, lmax, norm, sampling, csphase, lmax_calc, extend)
    SHExpandDH (grid, norm, sampling, csphase, lmax_calc)
    MakeGridGLQ(cilm, zero, lmax, norm, csphase, lmax_calc, extend)
    SHExpandGLQ(grid, w, zero, norm, csphase, lmax_calc)

All four are differentiable: the backward pass runs the hand-written
adjoint kernels (the weighted transpose transforms, which recompute the
Legendre functions).
"""
import ctypes
import threading

import numpy as np
import torch

from . import _lib

GRID_DH = 1
GRID_GLQ = 2


def _stream_ptr(device):
    return ctypes_void(torch.cuda.current_stream(device).cuda_stream)


class _NoSwitch:
    def __enter__(self):
        return self

    def __exit__(self, *exc):
        return False


_NO_SWITCH = _NoSwitch()


def _on_device(device):
    """torch.cuda.device(device), or nothing when it is already current."""
    if device.index == torch.cuda.current_device():
        return _NO_SWITCH
    return torch.cuda.device(device)


def ctypes_void(x):
    import ctypes
    return ctypes.c_void_p(int(x))


class Plan:
    """Device tables for one grid and option set (wraps shtc_plan).

    Creation synchronises the current stream; transforms do not.
    """

    def __init__(self, kind, lmax, lmax_calc=None, norm=1, csphase=1,
                 sampling=1, extend=0, zero=None, w=None, device=None, cplx=False):
        import ctypes
        self.lib = _lib.load()
        if device is None:
            device = torch.device("cuda", torch.cuda.current_device())
        device = torch.device(device)
        if device.index is None:
            device = torch.device("cuda", torch.cuda.current_device())
        self.device = device
        self.precision = 0
        self.table_bytes = 0
        lc = -1 if lmax_calc is None else int(lmax_calc)
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            st = _stream_ptr(self.device)
            self.cplx = bool(cplx)
            if kind == GRID_DH:
                fn = self.lib.shtc_plan_create_dhc if cplx else self.lib.shtc_plan_create_dh
                rc = fn(ctypes.byref(h), int(lmax), int(sampling), lc, int(norm),
                        int(csphase), int(extend), st)
            else:
                zp = wp = None
                if zero is not None:
                    self._zero = np.ascontiguousarray(zero, dtype=np.float64)
                    zp = self._zero.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
                if w is not None:
                    self._w = np.ascontiguousarray(w, dtype=np.float64)
                    wp = self._w.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
                fn = self.lib.shtc_plan_create_glqc if cplx else \
                    self.lib.shtc_plan_create_glq
                rc = fn(ctypes.byref(h), int(lmax), zp, wp, lc, int(norm), int(csphase),
                        int(extend), st)
        _lib.check(rc, "plan creation")
        self.handle = h
        info = (ctypes.c_longlong * 16)()
        _lib.check(self.lib.shtc_plan_info(h, info, 16))
        keys = ("kind", "lmax", "lmax_comp", "norm", "csphase", "sampling",
                "extend", "nlat", "nlon", "nlat_out", "nlon_out", "npair", "nlm",
                "device_bytes", "bluestein", "fft_mode")
        self.info = {k: int(v) for k, v in zip(keys, info)}

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                self.lib.shtc_plan_destroy(h)
            except Exception:
                pass
            self.handle = None

    @property
    def lc(self):
        return self.info["lmax_comp"]

    def set_precision(self, code):
        """shtc_plan_set_precision: 0 FP64, 1 INT8 tensor-core synthesis."""
        with _on_device(self.device):
            _lib.check(self.lib.shtc_plan_set_precision(self.handle, int(code)),
                       "shtc_plan_set_precision")
        if int(code) != self.precision:
            self.table_bytes = 0          # the library freed a table of other digits
        self.precision = int(code)
        self.__dict__.pop("_wsb", None)

    def legendre_table(self, enable=True):
        """shtc_plan_legendre_table: build (or free) the plan's table of P_lm
        digits for its mixed precision; the syntheses then stream it from
        device memory instead of running the recursion, and the analyses
        (and the synthesis adjoints) run on the tensor cores from it.
        Returns its size in bytes."""
        nb = ctypes.c_ulonglong(0)
        with _on_device(self.device):
            _lib.check(self.lib.shtc_plan_legendre_table(self.handle, int(bool(enable)),
                                                         ctypes.byref(nb)),
                       "shtc_plan_legendre_table")
        self.table_bytes = int(nb.value)
        self.__dict__.pop("_wsb", None)
        return self.table_bytes

    def workspace_bytes(self, nfield):
        """shtc_workspace_bytes for nfield fields, cached per plan and tile
        shape (the analysis tiles, and so the size, follow the shape that
        shtools_b200.autotune.set_shape records in self.shape)."""
        cache = self.__dict__.setdefault("_wsb", {})
        key = (nfield, getattr(self, "shape", None))
        nb = cache.get(key)
        if nb is None:
            nb = cache[key] = int(self.lib.shtc_workspace_bytes(self.handle, int(nfield)))
        return nb

    def workspace(self, nfield):
        nb = self.workspace_bytes(nfield)
        return torch.empty(nb, dtype=torch.uint8, device=self.device), nb

    # -- raw transforms on (F, 2, D, D) / (F, rows, cols) tensors -------------
    # float64 or float32 arrays; the kernels compute in FP64 either way
    def _run(self, fn, src, dst, nfield, src_is_coef):
        ws, nb = self.workspace(nfield)
        with _on_device(self.device):
            st = _stream_ptr(self.device)
            c, g = (src, dst) if src_is_coef else (dst, src)
            cargs = (ctypes_void(c.data_ptr()), _DTYPE[c.dtype], c.stride(0),
                     c.stride(1), c.stride(2), c.stride(3), c.shape[2])
            gargs = (ctypes_void(g.data_ptr()), _DTYPE[g.dtype], g.stride(0),
                     g.stride(1), g.stride(2))
            args = (cargs + gargs) if src_is_coef else (gargs + cargs)
            rc = fn(self.handle, *args, int(nfield), ctypes_void(ws.data_ptr()),
                    nb, st)
        _lib.check(rc, fn.__name__)

    def synthesis(self, cilm, out=None, dtype=None):
        F = cilm.shape[0]
        if out is None:
            out = torch.empty((F, self.info["nlat_out"], self.info["nlon_out"]),
                              dtype=dtype or cilm.dtype, device=self.device)
        self._run(self.lib.shtc_synthesis_ex, cilm, out, F, True)
        return out

    def analysis(self, grid, cdim=None, out=None, dtype=None):
        F = grid.shape[0]
        cdim = self.lc + 1 if cdim is None else cdim
        if out is None:
            out = torch.empty((F, 2, cdim, cdim), dtype=dtype or grid.dtype,
                              device=self.device)
        self._run(self.lib.shtc_analysis_ex, grid, out, F, False)
        return out

    # -- complex transforms (complex plans; complex128 tensors) ---------------
    def _run_c(self, fn, src, dst, nfield, src_is_coef):
        ws, nb = self.workspace(nfield)
        with _on_device(self.device):
            st = _stream_ptr(self.device)
            c, g = (src, dst) if src_is_coef else (dst, src)
            cargs = (ctypes_void(c.data_ptr()), c.stride(0), c.stride(1), c.stride(2),
                     c.stride(3), c.shape[2])
            gargs = (ctypes_void(g.data_ptr()), g.stride(0), g.stride(1), g.stride(2))
            args = (cargs + gargs) if src_is_coef else (gargs + cargs)
            rc = fn(self.handle, *args, int(nfield), ctypes_void(ws.data_ptr()), nb, st)
        _lib.check(rc, fn.__name__)

    def synthesis_c(self, cilm, out=None):
        F = cilm.shape[0]
        if out is None:
            out = torch.empty((F, self.info["nlat_out"], self.info["nlon_out"]),
                              dtype=torch.complex128, device=self.device)
        self._run_c(self.lib.shtc_synthesis_c, cilm, out, F, True)
        return out

    def analysis_c(self, grid, cdim=None, out=None):
        F = grid.shape[0]
        cdim = self.lc + 1 if cdim is None else cdim
        if out is None:
            out = torch.empty((F, 2, cdim, cdim), dtype=torch.complex128, device=self.device)
        self._run_c(self.lib.shtc_analysis_c, grid, out, F, False)
        return out

    def synthesis_adjoint(self, grid, cdim, dtype=None):
        F = grid.shape[0]
        out = torch.empty((F, 2, cdim, cdim), dtype=dtype or grid.dtype,
                          device=self.device)
        self._run(self.lib.shtc_synthesis_adjoint_ex, grid, out, F, False)
        return out

    def analysis_adjoint(self, cilm, dtype=None):
        F = cilm.shape[0]
        out = torch.empty((F, self.info["nlat"], self.info["nlon"]),
                          dtype=dtype or cilm.dtype, device=self.device)
        self._run(self.lib.shtc_analysis_adjoint_ex, cilm, out, F, True)
        return out


_DTYPE = {torch.float64: 0, torch.float32: 1}


_cache_lock = threading.Lock()
_plans = {}


# "-table": the synthesis streams a precomputed table of the P_lm digits
# (Plan.legendre_table) instead of running the recursion, and the analysis
# runs on the tensor cores from the same table
PRECISIONS = {"fp64": 0, "int8x6": 1, "int8x7": 2, "int8x6-table": 1, "int8x7-table": 2}


def _precision_code(precision):
    try:
        return PRECISIONS[precision]
    except KeyError:
        raise ValueError("precision must be one of %s; got %r"
                         % (sorted(PRECISIONS), precision)) from None


def get_plan(kind, lmax, lmax_calc, norm, csphase, sampling=1, extend=0,
             zero=None, w=None, device=None, tune=None, cplx=False, precision="fp64"):
    """Cached Plan for the option set (thread-safe).  New plans are
    autotuned when ``tune`` is true or the environment sets SHTC_AUTOTUNE=1
    (shtools_b200.autotune).  precision "int8x6" ("int8x7") runs the plan's
    syntheses on the INT8 tensor cores with an error-free 6-byte (7-byte)
    split (norms 1, 2, 4); "int8x6-table" / "int8x7-table" in addition build
    the plan's P_lm digit table once (Plan.legendre_table)."""
    import os
    dev = torch.device("cuda", torch.cuda.current_device()) if device is None \
        else torch.device(device)
    if dev.index is None:
        dev = torch.device("cuda", torch.cuda.current_device())
    zkey = None if zero is None else np.asarray(zero, dtype=np.float64).tobytes()
    wkey = None if w is None else np.asarray(w, dtype=np.float64).tobytes()
    prec = _precision_code(precision)
    key = (kind, int(lmax), int(lmax_calc), int(norm), int(csphase),
           int(sampling), int(extend), dev.index, zkey, wkey, bool(cplx), precision)
    with _cache_lock:
        p = _plans.get(key)
        if p is None:
            p = Plan(kind, lmax, lmax_calc, norm, csphase, sampling, extend,
                     zero, w, dev, cplx=cplx)
            if prec:
                p.set_precision(prec)
                if precision.endswith("-table"):
                    p.legendre_table(True)
            _plans[key] = p
            if tune or (tune is None and os.environ.get("SHTC_AUTOTUNE") == "1"):
                from . import autotune
                autotune.tune_plan(p)
        return p


def mixed_status(device=None):
    """Error word of the tensor-core kernels on the device: 0, or
    SHTC_ETIMEOUT (10) when a bounded in-kernel wait ran out since the last
    call (the outputs of that transform are then invalid); clears it."""
    import ctypes
    lib = _lib.load()
    dev = torch.device("cuda", torch.cuda.current_device()) if device is None \
        else torch.device(device)
    st = ctypes.c_int(0)
    with _on_device(dev):
        _lib.check(lib.shtc_mixed_status(ctypes.byref(st), _stream_ptr(dev)),
                   "shtc_mixed_status")
    return st.value


def clear_plan_cache():
    with _cache_lock:
        _plans.clear()


# ---------------------------------------------------------------------------
# argument resolution (Fortran semantics, MakeGridDH.f95:109-251)
# ---------------------------------------------------------------------------
def _check_common(norm, csphase):
    if norm not in (1, 2, 3, 4):
        raise ValueError("norm must be 1 (geodesy), 2 (Schmidt), 3 "
                         "(unnormalized) or 4 (orthonormalized); got %r" % (norm,))
    if csphase not in (1, -1):
        raise ValueError("csphase must be 1 or -1; got %r" % (csphase,))


def _resolve_synth(shape, lmax, lmax_calc):
    """lmax and lmax_comp of a synthesis from the cilm shape, as the
    reference: lmax defaults to the cilm degree, lmax_calc to lmax, and
    lmax_comp = min(lmax, cilm degree, lmax_calc) (MakeGridDH.f95:230-251,
    src/pyshtools.pyf:266-268)."""
    if len(shape) < 3 or shape[-3] < 2 or shape[-1] != shape[-2]:
        raise ValueError("cilm must be dimensioned as (..., 2, lmax+1, lmax+1); "
                         "got %s" % (tuple(shape),))
    D = int(shape[-1])
    lmax = D - 1 if lmax is None else int(lmax)
    if lmax < 0:
        raise ValueError("lmax must be >= 0")
    if lmax_calc is None:
        lmax_calc = lmax
    if lmax_calc > lmax:
        raise ValueError("lmax_calc (%d) must be less than or equal to lmax (%d)"
                         % (lmax_calc, lmax))
    lc = min(lmax, D - 1, int(lmax_calc))
    return lmax, lc


def _resolve_anal_dh(shape, sampling, lmax_calc):
    """lmax = n/2-1 and lmax_comp of SHExpandDH (SHExpandDH.f95:118-235)."""
    if sampling not in (1, 2):
        raise ValueError("sampling must be 1 (n by n) or 2 (n by 2n); got %r"
                         % (sampling,))
    if len(shape) < 2:
        raise ValueError("griddh must be two-dimensional; got %s" % (tuple(shape),))
    n = int(shape[-2])
    if n % 2 != 0 or n < 2:
        raise ValueError("The number of samples in latitude, n, must be even; "
                         "got %d" % n)
    if shape[-1] < sampling * n:
        raise ValueError("griddh must be dimensioned as (n, %s); got %s"
                         % ("n" if sampling == 1 else "2n", tuple(shape)))
    lmax = n // 2 - 1
    lc = lmax if lmax_calc is None else int(lmax_calc)
    if lc > lmax:
        raise ValueError("lmax_calc (%d) must be less than or equal to lmax (%d)"
                         % (lc, lmax))
    return lmax, lc


def _resolve_anal_glq(shape, lmax_calc):
    """lmax = nlat-1 and lmax_comp of SHExpandGLQ (SHExpandGLQ.f95:98-160)."""
    if len(shape) < 2:
        raise ValueError("gridglq must be two-dimensional; got %s" % (tuple(shape),))
    lmax = int(shape[-2]) - 1
    if shape[-1] < 2 * lmax + 1:
        raise ValueError("gridglq must be dimensioned as (lmax+1, 2*lmax+1); "
                         "got %s" % (tuple(shape),))
    lc = lmax if lmax_calc is None else int(lmax_calc)
    if lc > lmax:
        raise ValueError("lmax_calc (%d) must be less than or equal to lmax (%d)"
                         % (lc, lmax))
    return lmax, lc


def _flat(t, tail):
    lead = t.shape[:t.dim() - tail]
    return t.reshape((-1,) + tuple(t.shape[t.dim() - tail:])), lead


def _as_cuda(t, what):
    """CUDA tensor of dtype float64 or float32 (other dtypes -> float64)."""
    if isinstance(t, np.ndarray):
        t = torch.from_numpy(t)
    if not isinstance(t, torch.Tensor):
        t = torch.as_tensor(t)
    if not t.is_cuda:
        t = t.to("cuda")
    if t.dtype not in _DTYPE:
        t = t.to(torch.float64)
    return t


def _out_dtype(dtype):
    if dtype is None:
        return None
    dtype = torch.float64 if dtype in (np.float64, "float64") else \
        torch.float32 if dtype in (np.float32, "float32") else dtype
    if dtype not in _DTYPE:
        raise ValueError("dtype must be float64 or float32; got %r" % (dtype,))
    return dtype


# ---------------------------------------------------------------------------
# autograd functions
# ---------------------------------------------------------------------------
def _needs_grad(t):
    return torch.is_grad_enabled() and t.requires_grad


def _synthesis(cilm, plan, dtype):
    """Forward synthesis; through the autograd Function only when cilm
    requires a gradient (the Function's bookkeeping costs microseconds per
    call, which small transforms feel)."""
    if _needs_grad(cilm):
        return _Synthesis.apply(cilm, plan, dtype)
    c, lead = _flat(cilm[..., :2, :, :], 3)
    g = plan.synthesis(c, dtype=dtype)
    return g.reshape(tuple(lead) + tuple(g.shape[1:]))


def _analysis(grid, plan, cdim, dtype):
    """Forward analysis; through the autograd Function only when grid
    requires a gradient."""
    if _needs_grad(grid):
        return _Analysis.apply(grid, plan, cdim, dtype)
    nlat, nlon = plan.info["nlat"], plan.info["nlon"]
    g, lead = _flat(grid, 2)
    c = plan.analysis(g[:, :nlat, :nlon], cdim, dtype=dtype)
    return c.reshape(tuple(lead) + tuple(c.shape[1:]))


class _Synthesis(torch.autograd.Function):
    @staticmethod
    def forward(ctx, cilm, plan, dtype):
        c, lead = _flat(cilm[..., :2, :, :], 3)
        g = plan.synthesis(c, dtype=dtype)
        ctx.plan = plan
        ctx.cdim = cilm.shape[-1]
        ctx.lead = lead
        ctx.cshape = cilm.shape
        ctx.cdtype = cilm.dtype
        return g.reshape(tuple(lead) + tuple(g.shape[1:]))

    @staticmethod
    def backward(ctx, gout):
        plan = ctx.plan
        g, _ = _flat(gout.contiguous(), 2)
        gc = plan.synthesis_adjoint(g, ctx.cdim, dtype=ctx.cdtype)
        gc = gc.reshape(tuple(ctx.lead) + tuple(gc.shape[1:]))
        if ctx.cshape[-3] > 2:
            pad = torch.zeros(ctx.cshape, dtype=gc.dtype, device=gc.device)
            pad[..., :2, :, :] = gc
            gc = pad
        return gc, None, None


class _Analysis(torch.autograd.Function):
    @staticmethod
    def forward(ctx, grid, plan, cdim, dtype):
        nlat, nlon = plan.info["nlat"], plan.info["nlon"]
        g, lead = _flat(grid, 2)
        c = plan.analysis(g[:, :nlat, :nlon], cdim, dtype=dtype)
        ctx.plan = plan
        ctx.lead = lead
        ctx.gshape = grid.shape
        ctx.gdtype = grid.dtype
        return c.reshape(tuple(lead) + tuple(c.shape[1:]))

    @staticmethod
    def backward(ctx, gc):
        plan = ctx.plan
        c, _ = _flat(gc.contiguous(), 3)
        g = plan.analysis_adjoint(c, dtype=ctx.gdtype)
        g = g.reshape(tuple(ctx.lead) + tuple(g.shape[1:]))
        if tuple(g.shape) != tuple(ctx.gshape):
            full = torch.zeros(ctx.gshape, dtype=g.dtype, device=g.device)
            full[..., :g.shape[-2], :g.shape[-1]] = g
            g = full
        return g, None, None, None


# ---------------------------------------------------------------------------
# public API
# ---------------------------------------------------------------------------
def MakeGridDH(cilm, lmax=None, norm=1, sampling=1, csphase=1, lmax_calc=None,
               extend=False, dtype=None, precision="fp64"):
    """Driscoll-Healy synthesis on the GPU (src/MakeGridDH.f95:1).

    cilm: (..., 2, D, D) float64 or float32.  Returns (..., n+extend,
    sampling*n+extend) with n = 2*lmax+2; row 0 is 90 N, column 0 is 0 E.
    dtype: element type of the grid (default: that of cilm); the arithmetic
    is FP64 either way.  precision "int8x6": the Legendre sums on the INT8
    tensor cores with an error-free 6-byte split (norms 1, 2, 4).
    """
    _check_common(norm, csphase)
    if sampling not in (1, 2):
        raise ValueError("sampling must be 1 (n by n) or 2 (n by 2n); got %r"
                         % (sampling,))
    lmax, lc = _resolve_synth(np.shape(cilm), lmax, lmax_calc)
    dtype = _out_dtype(dtype)
    cilm = _as_cuda(cilm, "cilm")
    plan = get_plan(GRID_DH, lmax, lc, norm, csphase, sampling, int(bool(extend)),
                    device=cilm.device, precision=precision)
    return _synthesis(cilm, plan, dtype)


def SHExpandDH(griddh, norm=1, sampling=1, csphase=1, lmax_calc=None,
               dtype=None, precision="fp64"):
    """Driscoll-Healy analysis on the GPU (src/SHExpandDH.f95:1).

    griddh: (..., n, >= sampling*n) float64 or float32 with n even.  Returns
    (..., 2, lmax_calc+1, lmax_calc+1) of ``dtype`` (default: the grid's).
    precision "int8x7-table" ("int8x6-table"): the Legendre sums on the INT8
    tensor cores from the plan's P_lm digit table (norms 1, 2, 4); the
    analysis of "int8x7" / "int8x6" plans without a table stays FP64.
    """
    _check_common(norm, csphase)
    lmax, lc = _resolve_anal_dh(np.shape(griddh), sampling, lmax_calc)
    dtype = _out_dtype(dtype)
    grid = _as_cuda(griddh, "griddh")
    plan = get_plan(GRID_DH, lmax, lc, norm, csphase, sampling, 0,
                    device=grid.device, precision=precision)
    return _analysis(grid, plan, lc + 1, dtype)


def MakeGridGLQ(cilm, zero=None, lmax=None, norm=1, csphase=1, lmax_calc=None,
                extend=False, dtype=None, precision="fp64"):
    """Gauss-Legendre synthesis on the GPU (src/MakeGridGLQ.f95:1).

    zero: the lmax+1 Gauss-Legendre nodes (e.g. from SHGLQ); None computes
    them with the GPU PreGLQ.  Returns (..., lmax+1, 2*lmax+1+extend).
    precision: as for MakeGridDH.
    """
    _check_common(norm, csphase)
    lmax, lc = _resolve_synth(np.shape(cilm), lmax, lmax_calc)
    dtype = _out_dtype(dtype)
    z = None if zero is None else _host64(zero, lmax + 1, "zero")
    cilm = _as_cuda(cilm, "cilm")
    plan = get_plan(GRID_GLQ, lmax, lc, norm, csphase, 1, int(bool(extend)),
                    zero=z, device=cilm.device, precision=precision)
    return _synthesis(cilm, plan, dtype)


def SHExpandGLQ(gridglq, w=None, zero=None, norm=1, csphase=1,
                lmax_calc=None, dtype=None, precision="fp64"):
    """Gauss-Legendre analysis on the GPU (src/SHExpandGLQ.f95:1).

    gridglq: (..., lmax+1, >= 2*lmax+1).  w, zero: weights and nodes from
    SHGLQ; None computes them with the GPU PreGLQ.  precision: as for
    SHExpandDH.
    """
    _check_common(norm, csphase)
    lmax, lc = _resolve_anal_glq(np.shape(gridglq), lmax_calc)
    dtype = _out_dtype(dtype)
    nlat = lmax + 1
    z = None if zero is None else _host64(zero, nlat, "zero")
    wh = None if w is None else _host64(w, nlat, "w")
    grid = _as_cuda(gridglq, "gridglq")
    if (z is None) != (wh is None):
        # one given: complete the pair from the GPU PreGLQ
        zz, ww = SHGLQ(lmax, device=grid.device)
        z = zz if z is None else z
        wh = ww if wh is None else wh
    plan = get_plan(GRID_GLQ, lmax, lc, norm, csphase, 1, 0, zero=z, w=wh,
                    device=grid.device, precision=precision)
    return _analysis(grid, plan, lc + 1, dtype)


# ---------------------------------------------------------------------------
# complex transforms (not differentiable)
# ---------------------------------------------------------------------------
def _as_cuda_c(t):
    if isinstance(t, np.ndarray):
        t = torch.from_numpy(np.asarray(t, dtype=np.complex128))
    if not isinstance(t, torch.Tensor):
        t = torch.as_tensor(np.asarray(t, dtype=np.complex128))
    if not t.is_cuda:
        t = t.to("cuda")
    if t.dtype != torch.complex128:
        t = t.to(torch.complex128)
    return t


def _synth_c(cilm, plan):
    c, lead = _flat(cilm[..., :2, :, :], 3)
    g = plan.synthesis_c(c)
    return g.reshape(tuple(lead) + tuple(g.shape[1:]))


def _anal_c(grid, plan, cdim):
    g, lead = _flat(grid, 2)
    c = plan.analysis_c(g[:, :plan.info["nlat"], :plan.info["nlon"]], cdim)
    return c.reshape(tuple(lead) + tuple(c.shape[1:]))


def MakeGridDHC(cilm, lmax=None, norm=1, sampling=1, csphase=1, lmax_calc=None,
                extend=False):
    """Complex Driscoll-Healy synthesis on the GPU (src/MakeGridDHC.f95:1).

    cilm: (..., 2, D, D) complex; cilm[..., 0, l, m] multiplies Y_lm and
    cilm[..., 1, l, m] multiplies Y_l,-m (Y*_lm = (-1)^m Y_l,-m).  Returns the
    complex grid (..., n+extend, sampling*n+extend).
    """
    _check_common(norm, csphase)
    if sampling not in (1, 2):
        raise ValueError("sampling must be 1 (n by n) or 2 (n by 2n); got %r"
                         % (sampling,))
    lmax, lc = _resolve_synth(np.shape(cilm), lmax, lmax_calc)
    cilm = _as_cuda_c(cilm)
    plan = get_plan(GRID_DH, lmax, lc, norm, csphase, sampling, int(bool(extend)),
                    device=cilm.device, cplx=True)
    return _synth_c(cilm, plan)


def SHExpandDHC(griddh, norm=1, sampling=1, csphase=1, lmax_calc=None):
    """Complex Driscoll-Healy analysis on the GPU (src/SHExpandDHC.f95:1).
    Returns (..., 2, lmax_calc+1, lmax_calc+1) complex128."""
    _check_common(norm, csphase)
    lmax, lc = _resolve_anal_dh(np.shape(griddh), sampling, lmax_calc)
    grid = _as_cuda_c(griddh)
    plan = get_plan(GRID_DH, lmax, lc, norm, csphase, sampling, 0, device=grid.device,
                    cplx=True)
    return _anal_c(grid, plan, lc + 1)


def MakeGridGLQC(cilm, zero=None, lmax=None, norm=1, csphase=1, lmax_calc=None,
                 extend=False):
    """Complex Gauss-Legendre synthesis on the GPU (src/MakeGridGLQC.f95:1).
    Returns (..., lmax+1, 2*lmax+1+extend) complex128."""
    _check_common(norm, csphase)
    lmax, lc = _resolve_synth(np.shape(cilm), lmax, lmax_calc)
    z = None if zero is None else _host64(zero, lmax + 1, "zero")
    cilm = _as_cuda_c(cilm)
    plan = get_plan(GRID_GLQ, lmax, lc, norm, csphase, 1, int(bool(extend)), zero=z,
                    device=cilm.device, cplx=True)
    return _synth_c(cilm, plan)


def SHExpandGLQC(gridglq, w=None, zero=None, norm=1, csphase=1, lmax_calc=None):
    """Complex Gauss-Legendre analysis on the GPU (src/SHExpandGLQC.f95:1).
    Returns (..., 2, lmax_calc+1, lmax_calc+1) complex128."""
    _check_common(norm, csphase)
    lmax, lc = _resolve_anal_glq(np.shape(gridglq), lmax_calc)
    nlat = lmax + 1
    z = None if zero is None else _host64(zero, nlat, "zero")
    wh = None if w is None else _host64(w, nlat, "w")
    grid = _as_cuda_c(gridglq)
    if (z is None) != (wh is None):
        zz, ww = SHGLQ(lmax, device=grid.device)
        z = zz if z is None else z
        wh = ww if wh is None else wh
    plan = get_plan(GRID_GLQ, lmax, lc, norm, csphase, 1, 0, zero=z, w=wh,
                    device=grid.device, cplx=True)
    return _anal_c(grid, plan, lc + 1)


def MakeGradientDH(cilm, lmax=None, sampling=1, lmax_calc=None, extend=False,
                   radius=None):
    """Horizontal gradient of a real field on a Driscoll-Healy grid, on the
    GPU (src/MakeGradientDH.f95:1): returns (theta, phi) with
    theta = (1/r) dF/dtheta and phi = 1/(r sin theta) dF/dphi, zero on the
    pole rows.  cilm: (..., 2, D, D), 4-pi normalised without the
    Condon-Shortley phase (the reference's only convention).  Not
    differentiable."""
    if sampling not in (1, 2):
        raise ValueError("sampling must be 1 (n by n) or 2 (n by 2n); got %r"
                         % (sampling,))
    lmax, lc = _resolve_synth(np.shape(cilm), lmax, lmax_calc)
    r = 1.0 if radius is None else float(radius)
    if r == 0.0 or r != r:
        raise ValueError("radius must be a nonzero number; got %r" % (radius,))
    c = _as_cuda(cilm, "cilm").to(torch.float64)
    plan = get_plan(GRID_DH, lmax, lc, 1, 1, sampling, int(bool(extend)), device=c.device)
    cf, lead = _flat(c[..., :2, :, :], 3)
    F = cf.shape[0]
    shape = (F, plan.info["nlat_out"], plan.info["nlon_out"])
    th = torch.empty(shape, dtype=torch.float64, device=c.device)
    ph = torch.empty(shape, dtype=torch.float64, device=c.device)
    lib = plan.lib
    nb = int(lib.shtc_gradient_workspace_bytes(plan.handle, F))
    ws = torch.empty(max(nb, 8), dtype=torch.uint8, device=c.device)
    with _on_device(c.device):
        rc = lib.shtc_gradient_dh(plan.handle, ctypes_void(cf.data_ptr()), cf.stride(0),
                                  cf.stride(1), cf.stride(2), cf.stride(3), cf.shape[2],
                                  ctypes_void(th.data_ptr()), ctypes_void(ph.data_ptr()),
                                  th.stride(0), th.stride(1), th.stride(2), r, F,
                                  ctypes_void(ws.data_ptr()), nb, _stream_ptr(c.device))
    _lib.check(rc, "shtc_gradient_dh")
    out = tuple(lead) + shape[1:]
    return th.reshape(out), ph.reshape(out)


def MakeGravGridDH(cilm, gm, r0, lmax=None, a=None, f=0.0, sampling=2, lmax_calc=None,
                   omega=0.0, normal_gravity=1, normal_gravity_gm=None, extend=False):
    """Gravity on a flattened ellipsoid, on the GPU (src/MakeGravGridDH.f95:1,
    defaults of src/pyshtools.pyf:1440-1477): returns (rad, theta, phi,
    total, pot) DH grids of the gravity vector of V = GM/r sum_l (r0/r)^l
    C_lm Y_lm on the ellipsoid of semi-major axis a (default r0) and
    flattening f (rad positive up; theta and phi zero on the poles), its
    magnitude (minus the normal gravity when normal_gravity is 1, the
    gravity disturbance) and the potential.  omega: rotation rate, adding
    the centrifugal terms (None: the Fortran's absent OMEGA).  cilm:
    (..., 2, D, D), 4-pi normalised without the Condon-Shortley phase.  Not
    differentiable."""
    if sampling not in (1, 2):
        raise ValueError("sampling must be 1 (n by n) or 2 (n by 2n); got %r"
                         % (sampling,))
    if normal_gravity not in (0, 1):
        raise ValueError("normal_gravity must be 0 or 1; got %r" % (normal_gravity,))
    if normal_gravity == 1 and omega is None:
        raise ValueError("omega must be specified when removing the normal gravity")
    lmax, lc = _resolve_synth(np.shape(cilm), lmax, lmax_calc)
    a = float(r0) if a is None else float(a)
    ngm = float(gm) if normal_gravity_gm is None else float(normal_gravity_gm)
    c = _as_cuda(cilm, "cilm").to(torch.float64)
    plan = get_plan(GRID_DH, lmax, lc, 1, 1, sampling, int(bool(extend)), device=c.device)
    cf, lead = _flat(c[..., :2, :, :], 3)
    F = cf.shape[0]
    shape = (F, plan.info["nlat_out"], plan.info["nlon_out"])
    out = torch.empty((5,) + shape, dtype=torch.float64, device=c.device)
    g = [out[k] for k in range(5)]
    lib = plan.lib
    nb = int(lib.shtc_gravity_workspace_bytes(plan.handle, F))
    ws = torch.empty(max(nb, 8), dtype=torch.uint8, device=c.device)
    with _on_device(c.device):
        rc = lib.shtc_gravity_dh(plan.handle, ctypes_void(cf.data_ptr()), cf.stride(0),
                                 cf.stride(1), cf.stride(2), cf.stride(3), cf.shape[2],
                                 float(gm), float(r0), a, float(f), int(omega is not None),
                                 0.0 if omega is None else float(omega), int(normal_gravity),
                                 ngm, *[ctypes_void(t.data_ptr()) for t in g],
                                 g[0].stride(0), g[0].stride(1), g[0].stride(2), F,
                                 ctypes_void(ws.data_ptr()), nb, _stream_ptr(c.device))
    _lib.check(rc, "shtc_gravity_dh")
    shp = tuple(lead) + shape[1:]
    return tuple(t.reshape(shp) for t in g)


def NormalGravity(geocentric_lat, gm, omega, a, b):
    """Normal gravity of a rotating ellipsoid at a geocentric latitude in
    degrees (src/NormalGravity.f95:1), through the C ABI's host
    implementation."""
    return float(_lib.load().NormalGravity(float(geocentric_lat), float(gm), float(omega),
                                           float(a), float(b)))


def SHMultiply(cilm1, cilm2, lmax1=None, lmax2=None, precomp=None, norm=1, csphase=1):
    """Spherical-harmonic expansion of the product of two fields, on the GPU
    (src/SHMultiply.f95:1): both fields are synthesised on the Gauss-Legendre
    grid of degree lmax1 + lmax2, multiplied pointwise, and expanded to that
    degree.  cilm1, cilm2: (..., 2, D, D) with equal leading shapes.  Returns
    (..., 2, lmax1+lmax2+1, lmax1+lmax2+1).  precomp is accepted and ignored
    (it selects the reference's precomputed Legendre tables).  Not
    differentiable."""
    _check_common(norm, csphase)
    c1 = _as_cuda(cilm1, "cilm1").to(torch.float64)
    c2 = _as_cuda(cilm2, "cilm2").to(torch.float64)
    for c in (c1, c2):
        if c.dim() < 3 or c.shape[-3] < 2 or c.shape[-1] != c.shape[-2]:
            raise ValueError("cilm must be dimensioned as (..., 2, lmax+1, lmax+1); got %s"
                             % (tuple(c.shape),))
    L1 = c1.shape[-1] - 1 if lmax1 is None else int(lmax1)
    L2 = c2.shape[-1] - 1 if lmax2 is None else int(lmax2)
    if L1 < 0 or L2 < 0 or L1 > c1.shape[-1] - 1 or L2 > c2.shape[-1] - 1:
        raise ValueError("lmax1/lmax2 must lie within the dimensions of cilm1/cilm2")
    if c1.shape[:-3] != c2.shape[:-3]:
        raise ValueError("cilm1 and cilm2 must have the same leading dimensions")
    lo = L1 + L2
    plan = get_plan(GRID_GLQ, lo, lo, norm, csphase, 1, 0, device=c1.device)
    f1, lead = _flat(c1[..., :2, :, :], 3)
    f2, _ = _flat(c2[..., :2, :, :], 3)
    F = f1.shape[0]
    out = torch.zeros((F, 2, lo + 1, lo + 1), dtype=torch.float64, device=c1.device)
    lib = plan.lib
    nb = int(lib.shtc_multiply_workspace_bytes(plan.handle, F))
    ws = torch.empty(max(nb, 8), dtype=torch.uint8, device=c1.device)
    with _on_device(c1.device):
        rc = lib.shtc_multiply(plan.handle, ctypes_void(f1.data_ptr()), f1.stride(0),
                               f1.stride(1), f1.stride(2), f1.stride(3), L1,
                               ctypes_void(f2.data_ptr()), f2.stride(0), f2.stride(1),
                               f2.stride(2), f2.stride(3), L2, ctypes_void(out.data_ptr()),
                               out.stride(0), out.stride(1), out.stride(2), out.stride(3),
                               lo + 1, F, ctypes_void(ws.data_ptr()), nb,
                               _stream_ptr(c1.device))
    _lib.check(rc, "shtc_multiply")
    return out.reshape(tuple(lead) + tuple(out.shape[1:]))


def _host64(a, n, what):
    if isinstance(a, torch.Tensor):
        a = a.detach().cpu().numpy()
    a = np.ascontiguousarray(np.asarray(a, dtype=np.float64).ravel())
    if a.size < n:
        raise ValueError("%s must be dimensioned as (%d); got %d" % (what, n, a.size))
    return a[:n]


# ---------------------------------------------------------------------------
# quadrature (GPU)
# ---------------------------------------------------------------------------
def PreGLQ(x1, x2, n, device=None):
    """Gauss-Legendre nodes (descending) and weights on [x1, x2], computed on
    the GPU (src/PreGLQ.f95:1).  Returns two float64 CUDA tensors."""
    lib = _lib.load()
    dev = torch.device("cuda", torch.cuda.current_device()) if device is None \
        else torch.device(device)
    zero = torch.empty(int(n), dtype=torch.float64, device=dev)
    w = torch.empty(int(n), dtype=torch.float64, device=dev)
    with _on_device(dev):
        rc = lib.shtc_preglq(float(x1), float(x2), int(n),
                             ctypes_void(zero.data_ptr()),
                             ctypes_void(w.data_ptr()), _stream_ptr(dev))
    _lib.check(rc, "PreGLQ")
    return zero, w


def SHGLQ(lmax, device=None):
    """Nodes and weights of the lmax+1 point Gauss-Legendre quadrature
    (src/SHGLQ.f95:188), as host numpy arrays computed on the GPU."""
    z, w = PreGLQ(-1.0, 1.0, int(lmax) + 1, device)
    return z.cpu().numpy(), w.cpu().numpy()


def DHaj(n, extend=0, device=None):
    """Driscoll-Healy weights a_j (src/DHaj.f95:1) computed on the GPU."""
    lib = _lib.load()
    dev = torch.device("cuda", torch.cuda.current_device()) if device is None \
        else torch.device(device)
    aj = torch.empty(int(n) + int(extend), dtype=torch.float64, device=dev)
    with _on_device(dev):
        rc = lib.shtc_dhaj(int(n), ctypes_void(aj.data_ptr()), int(extend),
                           _stream_ptr(dev))
    _lib.check(rc, "DHaj")
    return aj
