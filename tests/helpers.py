"""Shared test helpers: load reference fixtures into oracle tensors and device
tensors, and compare them."""

import os

import numpy as np

from oracle import frostspin_oracle as fo

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load(name):
    return np.load(os.path.join(GOLDEN, name + ".npz"), allow_pickle=False)


def oracle_from_dic(data, prefix):
    """Reference get_data_dic format -> oracle tensor."""
    nrr = int(data[prefix + "_n_row_reps"])
    ncr = int(data[prefix + "_n_col_reps"])
    rr = [data[f"{prefix}_row_rep_{i}"] for i in range(nrr)]
    cr = [data[f"{prefix}_col_rep_{i}"] for i in range(ncr)]
    irr = data[prefix + "_block_irreps"]
    blocks = [data[f"{prefix}_block_{i}"] for i in range(irr.size)]
    return fo.OTensor(rr, cr, blocks, irr, data[prefix + "_signature"])


def diag_from_dic(data, prefix):
    irr = data[prefix + "_block_irreps"]
    blocks = [data[f"{prefix}_diagonal_block_{i}"] for i in range(irr.shape[0])]
    return blocks, irr


def assert_same_structure(a, b):
    """Block structure equality: reps, signature, irreps, shapes (bit-exact)."""
    assert len(a.row_reps) == len(b.row_reps)
    assert len(a.col_reps) == len(b.col_reps)
    for r1, r2 in zip(a.row_reps, b.row_reps, strict=True):
        assert np.array_equal(np.asarray(r1), np.asarray(r2))
    for r1, r2 in zip(a.col_reps, b.col_reps, strict=True):
        assert np.array_equal(np.asarray(r1), np.asarray(r2))
    assert np.array_equal(np.asarray(a.signature), np.asarray(b.signature))
    assert np.array_equal(np.asarray(a.block_irreps), np.asarray(b.block_irreps))


def blocks_of(t):
    """Host numpy blocks of an oracle or device tensor."""
    if hasattr(t, "host_blocks"):
        return t.host_blocks()
    return [np.asarray(b) for b in t.blocks]


def assert_blocks_equal(a, b):
    ba, bb = blocks_of(a), blocks_of(b)
    assert len(ba) == len(bb)
    for x, y in zip(ba, bb, strict=True):
        assert x.shape == y.shape
        assert np.array_equal(x, y)


def assert_blocks_close(a, b, rtol):
    ba, bb = blocks_of(a), blocks_of(b)
    assert len(ba) == len(bb)
    scale = max([np.abs(x).max() for x in bb if x.size] + [1e-300])
    for x, y in zip(ba, bb, strict=True):
        assert x.shape == y.shape
        assert np.abs(x - y).max() <= rtol * scale
