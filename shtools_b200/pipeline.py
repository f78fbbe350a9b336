"""Transforms of host-resident data with the PCIe copies overlapped.

A caller holding fields in (pinned) host memory pays one host->device copy
of the inputs and one device->host copy of the results per transform.  Run
one after another, the copies and the transform serialise.  ``pipelined``
runs a sequence of such steps on three streams instead: uploads on one, the
transform on the caller's current stream, downloads on a third, with
``depth`` sets of device input buffers in rotation, so that the upload of
step i+1 and the download of step i-1 overlap the transform of step i (PCIe
is full duplex).

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
    (a tuple of device tensors), and copy ``outs`` into the pinned host
    tensors of ``host_outputs[i]``.  Returns once every copy is queued; the
    host outputs are valid after ``torch.cuda.synchronize()``.  A host
    output tensor reused by a later step is overwritten in step order."""
    if len(host_inputs) != len(host_outputs):
        raise ValueError("host_inputs and host_outputs differ in length")
    if depth < 1:
        raise ValueError("depth must be >= 1")
    dev = torch.device("cuda", torch.cuda.current_device()) if device is None \
        else torch.device(device)
    if not host_inputs:
        return
    comp = torch.cuda.current_stream(dev)
    s_in = torch.cuda.Stream(dev)
    s_out = torch.cuda.Stream(dev)
    first = host_inputs[0]
    bufs = [tuple(torch.empty(t.shape, dtype=t.dtype, device=dev) for t in first)
            for _ in range(depth)]
    free = [torch.cuda.Event() for _ in range(depth)]   # buffer k consumed
    for e in free:
        e.record(comp)
    for i, (hin, hout) in enumerate(zip(host_inputs, host_outputs)):
        k = i % depth
        loaded = torch.cuda.Event()
        with torch.cuda.stream(s_in):
            s_in.wait_event(free[k])
            for d, h in zip(bufs[k], hin):
                if d.shape != h.shape or d.dtype != h.dtype:
                    raise ValueError("every step's inputs must match the first step's")
                d.copy_(h, non_blocking=True)
            loaded.record(s_in)
        comp.wait_event(loaded)
        outs = fn(*bufs[k])
        if isinstance(outs, torch.Tensor):
            outs = (outs,)
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
    for b in bufs:
        for d in b:
            d.record_stream(s_in)
