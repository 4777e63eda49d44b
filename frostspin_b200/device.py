"""Device plumbing: the CUDA device, the current stream, table uploads and scratch.

PyTorch only provides memory, streams and host<->device copies here; every
computation on symmetric-tensor data goes through the C ABI in ``_native``.
"""

import os

# Sector buffers range from tens of KB to ~11 GB (chi = 256 SU(2) CTMRG) and are
# allocated and freed every move; with the caching allocator's fixed segments
# that pattern fragments until a large request fails with most of the reserved
# memory unused.  Growable segments are the default here unless the process
# configured the allocator itself; the setting only takes effect when this
# module is imported before torch's first CUDA allocation.
os.environ.setdefault("PYTORCH_CUDA_ALLOC_CONF", "expandable_segments:True")

import numpy as np  # noqa: E402
import torch  # noqa: E402

from . import _native  # noqa: E402

_scratch = {}
_available = []


def device():
    """The CUDA device tensors live on.  Raises when CUDA is unavailable: there is
    no CPU fallback for any symmetric-tensor operation."""
    if not _available:
        if not torch.cuda.is_available():
            msg = "frostspin_b200 needs a CUDA device (B200, sm_100a); none is available"
            raise RuntimeError(msg)
        _available.append(True)
    return torch.device("cuda", torch.cuda.current_device())


def stream():
    """cudaStream_t of torch's current stream, as an integer handle."""
    return torch.cuda.current_stream().cuda_stream


def ptr(t):
    return t.data_ptr() if t is not None and t.numel() > 0 else None


def upload(arr):
    """Copy a numpy array (any dtype, structured included) into a new uint8 device
    buffer.  The bytes go through pinned host memory (torch's caching host
    allocator keeps that block alive until the copy has run), so the copy is
    asynchronous and the host does not wait for the stream."""
    a = np.ascontiguousarray(arr)
    raw = torch.from_numpy(a.view(np.uint8).reshape(-1))
    if raw.numel() == 0:
        return torch.empty(0, dtype=torch.uint8, device=device())
    return raw.pin_memory().to(device(), non_blocking=True)


def upload_f64(arr):
    a = np.ascontiguousarray(arr, dtype=np.float64)
    return torch.from_numpy(a).pin_memory().to(device(), non_blocking=True)


def scratch_partials():
    """Per-device scratch for two-pass reductions (fs_reduce_partials() doubles)."""
    dev = device()
    key = ("partials", dev.index)
    buf = _scratch.get(key)
    if buf is None:
        buf = torch.empty(_native.reduce_partials(), dtype=torch.float64, device=dev)
        _scratch[key] = buf
    return buf


def empty_f64(n):
    return torch.empty(int(n), dtype=torch.float64, device=device())


def zeros_f64(n):
    return torch.zeros(int(n), dtype=torch.float64, device=device())
