"""Batched transforms of many fields on several grids (shtc_batch_*).

The typical use is thousands of Gauss-Legendre fields of uneven lmax, each
expanded on its own GLQ grid: fields with the same grid share a plan (and
the Legendre recursion); one batched transform is one pack launch, one
persistent Legendre launch over cost-sorted work items and one launch for
all longitude FFTs, so it can be captured in a CUDA graph and replayed.

    b = Batch.glq(lmaxes)                   # one entry per field
    flat = b.pack_cilm(cilm_list)           # caller order -> batch layout
    grids = b.synthesis(flat)               # MakeGridGLQ of every field
    back = b.analysis(grids)                # SHExpandGLQ of every field
    g = b.graph("synthesis")                # CUDA graph over static buffers
"""
import ctypes

import numpy as np
import torch

from . import _lib
from .transforms import GRID_DH, GRID_GLQ, Plan, _stream_ptr, ctypes_void


def _bind(L):
    if getattr(L, "_batch_bound", False):
        return L
    P, LL, I, SZ = ctypes.c_void_p, ctypes.c_longlong, ctypes.c_int, ctypes.c_size_t
    L.shtc_batch_create.argtypes = [ctypes.POINTER(P), I, ctypes.POINTER(P),
                                    ctypes.POINTER(I), P]
    L.shtc_batch_destroy.argtypes = [P]
    L.shtc_batch_layout.argtypes = [P, ctypes.POINTER(LL), ctypes.POINTER(LL)]
    L.shtc_batch_workspace_bytes.restype = SZ
    L.shtc_batch_workspace_bytes.argtypes = [P]
    L.shtc_batch_synthesis.argtypes = [P, P, P, P, SZ, P]
    L.shtc_batch_analysis.argtypes = [P, P, P, P, SZ, P]
    L._batch_bound = True
    return L


class Batch:
    """A batch of fields over a list of plans: ``groups`` is a list of
    (Plan, number of fields) pairs; plans need extend = 0."""

    def __init__(self, groups, device=None):
        self.lib = _bind(_lib.load())
        self.plans = [p for p, _ in groups]
        self.counts = [int(n) for _, n in groups]
        self.device = self.plans[0].device if device is None else torch.device(device)
        n = len(groups)
        arr = (ctypes.c_void_p * n)(*[p.handle.value for p in self.plans])
        cnt = (ctypes.c_int * n)(*self.counts)
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            rc = self.lib.shtc_batch_create(ctypes.byref(h), n, arr, cnt,
                                            _stream_ptr(self.device))
        _lib.check(rc, "shtc_batch_create")
        self.handle = h
        co = (ctypes.c_longlong * (n + 1))()
        go = (ctypes.c_longlong * (n + 1))()
        _lib.check(self.lib.shtc_batch_layout(h, co, go))
        self.cilm_off = np.array(co[:], dtype=np.int64)
        self.grid_off = np.array(go[:], dtype=np.int64)
        nb = int(self.lib.shtc_batch_workspace_bytes(h))
        self.work = torch.empty(max(nb, 8), dtype=torch.uint8, device=self.device)
        self.work_bytes = nb
        # caller field order -> (group, slot); filled by the constructors
        self.field_slots = [(g, s) for g, c in enumerate(self.counts) for s in range(c)]

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                self.lib.shtc_batch_destroy(h)
            except Exception:
                pass
            self.handle = None

    # -- construction --------------------------------------------------------
    @classmethod
    def glq(cls, lmaxes, norm=1, csphase=1, device=None, zeros=None):
        """Batch of GLQ fields of the given lmax (one per field), each on the
        GLQ grid of its own lmax (nodes from the GPU PreGLQ unless ``zeros``
        maps lmax -> nodes)."""
        lmaxes = [int(x) for x in lmaxes]
        dev = torch.device("cuda", torch.cuda.current_device()) if device is None \
            else torch.device(device)
        uniq = sorted(set(lmaxes))
        plans = []
        for L in uniq:
            z = None if zeros is None else zeros.get(L)
            plans.append(Plan(GRID_GLQ, L, L, norm, csphase, 1, 0, zero=z, device=dev))
        index = {L: i for i, L in enumerate(uniq)}
        counts = [0] * len(uniq)
        slots = []
        for L in lmaxes:
            g = index[L]
            slots.append((g, counts[g]))
            counts[g] += 1
        keep = [i for i, c in enumerate(counts) if c > 0]
        b = cls([(plans[i], counts[i]) for i in keep], dev)
        remap = {old: new for new, old in enumerate(keep)}
        b.field_slots = [(remap[g], s) for g, s in slots]
        b.lmaxes = lmaxes
        return b

    # -- layout helpers --------------------------------------------------------
    def _cshape(self, g):
        D = self.plans[g].lc + 1
        return (2, D, D)

    def _gshape(self, g):
        i = self.plans[g].info
        return (i["nlat"], i["nlon"])

    def cilm_view(self, flat, field):
        g, s = self.field_slots[field]
        sh = self._cshape(g)
        n = int(np.prod(sh))
        o = int(self.cilm_off[g]) + s * n
        return flat[o:o + n].view(sh)

    def grid_view(self, flat, field):
        g, s = self.field_slots[field]
        sh = self._gshape(g)
        n = int(np.prod(sh))
        o = int(self.grid_off[g]) + s * n
        return flat[o:o + n].view(sh)

    def empty_cilm(self):
        return torch.zeros(int(self.cilm_off[-1]), dtype=torch.float64, device=self.device)

    def empty_grid(self):
        return torch.zeros(int(self.grid_off[-1]), dtype=torch.float64, device=self.device)

    def pack_cilm(self, cilms):
        """Per-field coefficient arrays (2, >=lc+1, >=lc+1) in caller order ->
        one flat device tensor in batch layout."""
        flat = self.empty_cilm()
        for i, c in enumerate(cilms):
            v = self.cilm_view(flat, i)
            D = v.shape[-1]
            t = torch.as_tensor(np.asarray(c) if not isinstance(c, torch.Tensor) else c,
                                dtype=torch.float64)
            v.copy_(t[:2, :D, :D].to(self.device))
        return flat

    # -- transforms -----------------------------------------------------------
    def synthesis(self, cilm_flat, out=None):
        out = self.empty_grid() if out is None else out
        with torch.cuda.device(self.device):
            rc = self.lib.shtc_batch_synthesis(
                self.handle, ctypes_void(cilm_flat.data_ptr()),
                ctypes_void(out.data_ptr()), ctypes_void(self.work.data_ptr()),
                self.work_bytes, _stream_ptr(self.device))
        _lib.check(rc, "shtc_batch_synthesis")
        return out

    def analysis(self, grid_flat, out=None):
        out = self.empty_cilm() if out is None else out
        with torch.cuda.device(self.device):
            rc = self.lib.shtc_batch_analysis(
                self.handle, ctypes_void(grid_flat.data_ptr()),
                ctypes_void(out.data_ptr()), ctypes_void(self.work.data_ptr()),
                self.work_bytes, _stream_ptr(self.device))
        _lib.check(rc, "shtc_batch_analysis")
        return out

    def graph(self, which="synthesis", static_in=None):
        """Capture one batched transform in a CUDA graph over static buffers.
        Returns (graph, static_in, static_out): copy inputs into static_in,
        call graph.replay(), read static_out."""
        if static_in is None:
            static_in = self.empty_cilm() if which == "synthesis" else self.empty_grid()
        static_out = self.empty_grid() if which == "synthesis" else self.empty_cilm()
        fn = self.synthesis if which == "synthesis" else self.analysis
        s = torch.cuda.Stream(self.device)
        s.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(s):
            fn(static_in, static_out)          # warm-up outside the capture
        torch.cuda.current_stream(self.device).wait_stream(s)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            fn(static_in, static_out)
        return g, static_in, static_out
