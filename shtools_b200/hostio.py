"""Host <-> device copies of numpy arrays through pinned staging buffers.

The pyshtools backend takes numpy arrays (pageable host memory) and returns
new numpy arrays.  A plain ``torch.from_numpy(a).to("cuda")`` or
``t.cpu().numpy()`` copies pageable memory, which the driver stages itself
at a few GB/s.  Here the array moves in chunks through two reusable pinned
buffers per device: the host copy of one chunk (numpy into the pinned
buffer, or out of it) overlaps the PCIe transfer of the previous chunk on a
dedicated copy stream, and each host copy is split over a small pool of
threads (numpy releases the GIL while it copies), since one core copies
well below what PCIe carries.  Small arrays take the plain path.

Results of up to PINNED_MAX bytes come back without staging: they are
copied straight into a pinned host buffer that the returned numpy array
views.  The buffers come from a pool of this module, by byte size: a buffer
returns to the pool when the array viewing it (and every view of that
array) has been garbage-collected, so a loop of calls reuses the same few
buffers instead of pinning new memory (cudaHostAlloc of tens of MB takes
tens of ms).  The pool keeps at most POOL_MAX bytes of free buffers.
Inputs that already live in pinned memory (for instance such a result,
passed back in) are uploaded directly.  Real coefficient arrays for the
synthesis (to_device_lower) move only their entries m <= l.

Thread safety: one lock per device guards its staging buffers; calls from
several threads are serialised on them.
"""
import os
import threading
import weakref
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import torch

CHUNK_BYTES = 16 << 20         # bytes per staging buffer
SMALL_BYTES = 1 << 20          # arrays below this size are copied directly
SLICE_BYTES = 2 << 20          # smallest share of a host copy given to one thread
PINNED_MAX = 4 << 30           # results up to this size come back in pinned memory
POOL_MAX = 8 << 30             # free pinned result buffers kept for reuse

_lock = threading.Lock()
_state = {}                    # device index -> (lock, stream, [buffers], [events])
_pool = None
_free = {}                     # byte size -> [pinned uint8 tensors] not viewed by any array
_free_bytes = 0


def _take(nbytes):
    """A pinned uint8 host tensor of nbytes, from the pool or new."""
    global _free_bytes
    with _lock:
        lst = _free.get(nbytes)
        if lst:
            _free_bytes -= nbytes
            return lst.pop()
    return torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)


def _give(buf):
    """Return a buffer whose array has died to the pool (or drop it)."""
    global _free_bytes
    n = buf.numel()
    with _lock:
        if _free_bytes + n <= POOL_MAX:
            _free.setdefault(n, []).append(buf)
            _free_bytes += n


def _threads():
    return max(1, min(8, (os.cpu_count() or 1) // 2))


def _copy(dst, src):
    """dst[:] = src for flat uint8 arrays, split over the copy threads."""
    global _pool
    n = src.size
    parts = min(_threads(), max(1, n // SLICE_BYTES))
    if parts == 1:
        np.copyto(dst, src)
        return
    with _lock:
        if _pool is None:
            _pool = ThreadPoolExecutor(_threads(), thread_name_prefix="shtc-hostio")
        pool = _pool
    step = -(-n // parts)
    futs = [pool.submit(np.copyto, dst[o:o + step], src[o:o + step])
            for o in range(0, n, step)]
    for f in futs:
        f.result()


def _get(dev):
    with _lock:
        s = _state.get(dev.index)
        if s is None:
            bufs = [torch.empty(CHUNK_BYTES, dtype=torch.uint8, pin_memory=True)
                    for _ in range(2)]
            s = (threading.Lock(), torch.cuda.Stream(dev), bufs,
                 [torch.cuda.Event(), torch.cuda.Event()])
            _state[dev.index] = s
        return s


def to_device(a, device=None):
    """A CUDA tensor holding the numpy array ``a`` (C-contiguous copy), ready
    for work queued on the device's current stream."""
    dev = torch.device("cuda", torch.cuda.current_device()) if device is None \
        else torch.device(device)
    if dev.index is None:
        dev = torch.device("cuda", torch.cuda.current_device())
    a = np.ascontiguousarray(a)
    if a.nbytes < SMALL_BYTES:
        return torch.from_numpy(a).to(dev)
    ta = torch.from_numpy(a)
    if ta.is_pinned():
        # one DMA on the current stream, complete on return: the caller may
        # reuse or free the host array at once
        t = ta.to(dev, non_blocking=True)
        torch.cuda.current_stream(dev).synchronize()
        return t
    dst = torch.empty(a.shape, dtype=ta.dtype, device=dev)
    src = a.reshape(-1).view(np.uint8)
    dflat = dst.view(-1).view(torch.uint8)
    lock, cs, bufs, evs = _get(dev)
    cur = torch.cuda.current_stream(dev)
    with lock:
        cs.wait_stream(cur)                 # dst was allocated on the current stream
        n = src.size
        for k, off in enumerate(range(0, n, CHUNK_BYTES)):
            b = k & 1
            ln = min(CHUNK_BYTES, n - off)
            evs[b].synchronize()            # earlier transfers have read buffer b
            _copy(bufs[b].numpy()[:ln], src[off:off + ln])
            with torch.cuda.stream(cs):
                dflat[off:off + ln].copy_(bufs[b][:ln], non_blocking=True)
                evs[b].record(cs)
        cur.wait_stream(cs)
        dst.record_stream(cs)
    return dst


def _copy_lower(dst, src, r0, n):
    """dst[i, :l+1] = src[i, :l+1] for the 2-D row blocks of a coefficient
    array, l = (r0 + i) mod n the degree of row i: the rows' valid prefixes
    only, in bands of rows (each band copies the widest prefix it holds),
    split over the copy threads."""
    global _pool
    nrow = src.shape[0]
    band = max(1, n // 32)
    jobs = []
    i = 0
    while i < nrow:
        l = (r0 + i) % n
        j = min(nrow, i + band, i + (n - l))   # a band ends at a degree wrap
        cols = (r0 + j - 1) % n + 1            # widest prefix of the band
        jobs.append((i, j, cols))
        i = j
    with _lock:
        if _pool is None:
            _pool = ThreadPoolExecutor(_threads(), thread_name_prefix="shtc-hostio")
        pool = _pool
    futs = [pool.submit(np.copyto, dst[a:b, :c], src[a:b, :c]) for a, b, c in jobs]
    for f in futs:
        f.result()


def to_device_lower(a, device=None):
    """to_device for real coefficient arrays [..., n, n] of which the
    transforms read only the entries m <= l (the last index at most the one
    before it): the host copies move only those (about half the bytes of a
    square array); in the device copy the entries m > l are zero.  Other
    shapes take to_device."""
    dev = torch.device("cuda", torch.cuda.current_device()) if device is None \
        else torch.device(device)
    if dev.index is None:
        dev = torch.device("cuda", torch.cuda.current_device())
    a = np.ascontiguousarray(a)
    n = a.shape[-1] if a.ndim >= 2 else 0
    rowb = n * a.itemsize
    if (a.ndim < 2 or a.shape[-2] != n or a.nbytes < SMALL_BYTES or rowb > CHUNK_BYTES
            or torch.from_numpy(a).is_pinned()):
        t = to_device(a, dev)
        return t.tril_() if a.ndim >= 2 and a.shape[-2] == a.shape[-1] else t
    ta = torch.from_numpy(a)
    dst = torch.empty(a.shape, dtype=ta.dtype, device=dev)
    src = a.reshape(-1, n)
    rows = src.shape[0]
    per = CHUNK_BYTES // rowb               # whole rows per staging buffer
    dflat = dst.view(-1).view(torch.uint8)
    lock, cs, bufs, evs = _get(dev)
    cur = torch.cuda.current_stream(dev)
    with lock:
        cs.wait_stream(cur)
        for k, r0 in enumerate(range(0, rows, per)):
            b = k & 1
            nr = min(per, rows - r0)
            evs[b].synchronize()
            stage = bufs[b].numpy()[:nr * rowb].view(a.dtype).reshape(nr, n)
            _copy_lower(stage, src[r0:r0 + nr], r0, n)
            with torch.cuda.stream(cs):
                dflat[r0 * rowb:(r0 + nr) * rowb].copy_(bufs[b][:nr * rowb],
                                                        non_blocking=True)
                evs[b].record(cs)
        cur.wait_stream(cs)
        dst.record_stream(cs)
    # the staged rows' entries m > l hold whatever the buffers held before
    return dst.tril_()


def to_host(t):
    """A new numpy array with the contents of the CUDA tensor ``t`` (after the
    work queued on the device's current stream)."""
    t = t.detach()
    if not t.is_cuda or t.numel() * t.element_size() < SMALL_BYTES:
        return t.cpu().numpy()
    t = t.contiguous()
    dev = t.device
    nbytes = t.numel() * t.element_size()
    if nbytes <= PINNED_MAX:
        buf = _take(nbytes)
        h = buf.view(t.dtype).view(tuple(t.shape))
        h.copy_(t, non_blocking=True)
        torch.cuda.current_stream(dev).synchronize()
        out = h.numpy()
        weakref.finalize(out, _give, buf)
        return out
    out = np.empty(tuple(t.shape), dtype=t.new_empty(0).cpu().numpy().dtype)
    dst = out.reshape(-1).view(np.uint8)
    sflat = t.view(-1).view(torch.uint8)
    lock, cs, bufs, evs = _get(dev)
    cur = torch.cuda.current_stream(dev)
    n = dst.size
    offs = list(range(0, n, CHUNK_BYTES))
    with lock:
        cs.wait_stream(cur)                 # the producer of t ran on the current stream
        pend = []                           # (buffer, offset, length) transferred, not read
        for k, off in enumerate(offs):
            b = k & 1
            ln = min(CHUNK_BYTES, n - off)
            if k >= 2:
                pb, poff, pln = pend.pop(0)
                evs[pb].synchronize()
                _copy(dst[poff:poff + pln], bufs[pb].numpy()[:pln])
            with torch.cuda.stream(cs):
                bufs[b][:ln].copy_(sflat[off:off + ln], non_blocking=True)
                evs[b].record(cs)
            pend.append((b, off, ln))
        for pb, poff, pln in pend:
            evs[pb].synchronize()
            _copy(dst[poff:poff + pln], bufs[pb].numpy()[:pln])
        t.record_stream(cs)
    return out
