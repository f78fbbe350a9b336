"""Transforms of host-resident data with the PCIe copies overlapped.

A caller holding fields in (pinned) host memory pays one host->device copy
of the inputs and one device->host copy of the results per transform.  Run
one after another, the copies and the transform serialise.  ``pipelined``
runs a sequence of such steps on three streams instead: uploads on one, the
transform on the caller's current stream, downloads on a third, with
``depth`` sets of device input buffers in rotation, so that the upload of
step i+1 and the download of step i-1 overlap the transform of step i (PCIe
is full duplex).  Steps may differ in the shapes of their inputs: splitting
a synthesis + analysis pair into two steps lets the synthesis start once the
coefficients are on the device, while the grid is still being uploaded.

    from shtools_b200 import MakeGridGLQ, SHExpandGLQ
    from shtools_b200.pipeline import pipelined
    steps = [(cilm_pinned, grid_pinned)] * 10
    outs = [(grid_out[i % 2], cilm_out[i % 2]) for i in range(10)]
    pipelined(lambda c, g: (MakeGridGLQ(c), SHExpandGLQ(g)), steps, outs)
    torch.cuda.synchronize()
"""
import torch


def pipelined(fn, host_inputs, host_outputs, device=None, depth=2):
    """For each step i: copy the tensors of ``host_inputs[i]`` (a tuple of
    pinned host tensors) to the device, run ``outs = fn(*device_inputs)``
    (a tuple of device tensors; ``fn`` may also be a sequence with one
    callable per step), and copy ``outs`` into the pinned host tensors of
    ``host_outputs[i]``.  Returns once every copy is queued; the
    host outputs are valid after ``torch.cuda.synchronize()``.  A host
    output tensor reused by a later step is overwritten in step order.
    Device input buffers are kept per input signature (the shapes and
    dtypes of a step's inputs), ``depth`` sets of each, so steps of
    different kinds may alternate."""
    if len(host_inputs) != len(host_outputs):
        raise ValueError("host_inputs and host_outputs differ in length")
    fns = [fn] * len(host_inputs) if callable(fn) else list(fn)
    if len(fns) != len(host_inputs):
        raise ValueError("one function per step is needed")
    if depth < 1:
        raise ValueError("depth must be >= 1")
    dev = torch.device("cuda", torch.cuda.current_device()) if device is None \
        else torch.device(device)
    if not host_inputs:
        return
    comp = torch.cuda.current_stream(dev)
    s_in = torch.cuda.Stream(dev)
    s_out = torch.cuda.Stream(dev)
    sig = lambda hin: tuple((tuple(t.shape), t.dtype) for t in hin)
    # signature -> [buffer sets, "set consumed" events (None before the first
    # use), steps so far]; every buffer is allocated on the caller's stream
    # before any step is queued, and a first use waits for the work queued
    # there before this call only
    pools = {}
    for hin in host_inputs:
        if sig(hin) not in pools:
            pools[sig(hin)] = [
                [tuple(torch.empty(t.shape, dtype=t.dtype, device=dev) for t in hin)
                 for _ in range(depth)], [None] * depth, 0]
    start = torch.cuda.Event()
    start.record(comp)
    for i, (hin, hout) in enumerate(zip(host_inputs, host_outputs)):
        pool = pools[sig(hin)]
        bufs, free, n = pool
        k = n % depth
        pool[2] = n + 1
        loaded = torch.cuda.Event()
        with torch.cuda.stream(s_in):
            s_in.wait_event(start if free[k] is None else free[k])
            for d, h in zip(bufs[k], hin):
                d.copy_(h, non_blocking=True)
            loaded.record(s_in)
        comp.wait_event(loaded)
        outs = fns[i](*bufs[k])
        if isinstance(outs, torch.Tensor):
            outs = (outs,)
        free[k] = torch.cuda.Event()
        free[k].record(comp)
        done = torch.cuda.Event()
        done.record(comp)
        with torch.cuda.stream(s_out):
            s_out.wait_event(done)
            for h, d in zip(hout, outs):
                d.record_stream(s_out)
                h.copy_(d, non_blocking=True)
    # the caller's stream sees every download, and the buffers stay alive
    # until the last use
    end = torch.cuda.Event()
    end.record(s_out)
    comp.wait_event(end)
    for bufs, _, _ in pools.values():
        for b in bufs:
            for d in b:
                d.record_stream(s_in)
