"""Optional per-kernel-class timing with CUDA events (used by bench.py).

When enabled, every device call wrapped in region(name, ...) records a pair of
CUDA events on the current stream and the algorithmic work it was given
(flops, bytes, int8 ops); summary() synchronises once and returns per-class
event time and work, from which the roofline fractions are computed.  Disabled
(the default), region() costs one dictionary lookup.
"""

import contextlib

import torch

_state = {"on": False, "records": []}


def enable():
    _state["on"] = True
    _state["records"] = []


def disable():
    _state["on"] = False


@contextlib.contextmanager
def region(name, **work):
    if not _state["on"]:
        yield
        return
    s = torch.cuda.Event(enable_timing=True)
    e = torch.cuda.Event(enable_timing=True)
    s.record()
    try:
        yield
    finally:
        e.record()
        _state["records"].append((name, s, e, work))


def summary():
    """{name: {"launches": n, "ms": total event time, work keys summed}}."""
    torch.cuda.synchronize()
    out = {}
    for name, s, e, work in _state["records"]:
        d = out.setdefault(name, {"launches": 0, "ms": 0.0})
        d["launches"] += 1
        d["ms"] += s.elapsed_time(e)
        for k, v in work.items():
            d[k] = d.get(k, 0.0) + v
    return out
