"""Block re-layout on the device: pack blocks C-order at new offsets, reading
through the transposed-storage flag.  Uses the permute kernel with one
two-leg elementary block per irrep block."""

import numpy as np

from .. import _native
from .. import device as dev
from .abelian_plan import _make_tasks, _pack_ebs


def relayout_blocks(data, offsets, shapes, trans, new_offsets, total):
    nb = len(offsets)
    out = dev.empty_f64(total)
    if nb == 0 or total == 0:
        return out
    shapes = np.asarray(shapes, dtype=np.int64).reshape(-1, 2)
    m = shapes[:, 0]
    n = shapes[:, 1]
    dims = np.stack([m, n], axis=1)
    if trans:
        ostride = np.stack([np.ones_like(m), m], axis=1)
    else:
        ostride = np.stack([n, np.ones_like(n)], axis=1)
    nstride = np.stack([n, np.ones_like(n)], axis=1)
    present = np.ones(nb, dtype=bool)
    ebs, vol = _pack_ebs(dims, ostride, nstride, np.asarray(offsets, dtype=np.int64),
                         np.asarray(new_offsets, dtype=np.int64), present)
    tasks = _make_tasks(ebs)
    d_ebs = dev.upload(ebs)
    d_tasks = dev.upload(tasks)
    _native.call(
        "fs_abelian_permute",
        dev.ptr(data),
        data.numel(),
        dev.ptr(out),
        out.numel(),
        d_ebs.data_ptr(),
        ebs.size,
        d_tasks.data_ptr(),
        tasks.size,
        None,
        dev.stream(),
    )
    return out
