"""Pin the SU(2) CPU oracle against outputs of the reference implementation
(tests/golden/su2.npz, tests/golden/simple_update_su2.npz)."""

import numpy as np
import pytest

from oracle import ctmrg_oracle as co
from oracle import su2_oracle as so
from tests.helpers import load

TOL = 1e-13


def from_dic(d, prefix):
    nrr = int(d[prefix + "_n_row_reps"])
    ncr = int(d[prefix + "_n_col_reps"])
    rr = [d[f"{prefix}_row_rep_{i}"] for i in range(nrr)]
    cr = [d[f"{prefix}_col_rep_{i}"] for i in range(ncr)]
    irr = d[prefix + "_block_irreps"]
    return so.OTensor(rr, cr, [d[f"{prefix}_block_{i}"] for i in range(irr.size)], irr,
                      d[prefix + "_signature"])


def check(t, d, prefix):
    ref = from_dic(d, prefix)
    assert np.array_equal(t.block_irreps, ref.block_irreps), prefix
    for a, b in zip(t.row_reps + t.col_reps, ref.row_reps + ref.col_reps, strict=True):
        assert np.array_equal(a, b)
    assert np.array_equal(t.signature, ref.signature)
    scale = max([np.abs(b).max() for b in ref.blocks] + [1e-300])
    for a, b in zip(t.blocks, ref.blocks, strict=True):
        assert a.shape == b.shape, prefix
        assert np.abs(a - b).max() <= TOL * scale, prefix


@pytest.mark.parametrize("base", ["sds", "sdsb", "ext", "miss", "r5", "r6"])
def test_su2_oracle_permute(base):
    d = load("su2")
    t = from_dic(d, base)
    i = 0
    while f"{base}_perm{i}_axes" in d:
        pre = f"{base}_perm{i}"
        axes = tuple(int(a) for a in d[pre + "_axes"])
        nrr = int(d[pre + "_nrr"])
        check(so.permute(t, axes[:nrr], axes[nrr:]), d, pre)
        i += 1
    assert i >= 2


def test_su2_oracle_dense_and_linear_algebra():
    d = load("su2")
    for base in ("sds", "sdsb", "ext", "r5"):
        t = from_dic(d, base)
        dense = d[base + "_dense"]
        assert np.abs(so.toarray(t) - dense).max() <= TOL * max(np.abs(dense).max(), 1)
        check(so.from_array(dense, t.row_reps, t.col_reps, t.signature), d, base)
    t = from_dic(d, "r5")
    check(so.transpose(t), d, "r5_transpose")
    check(so.dagger(t), d, "r5_dagger")
    assert abs(so.norm(t) - float(d["r5_norm"])) <= 1e-13 * float(d["r5_norm"])
    m = so.matmul(t, so.dagger(t))
    check(m, d, "r5_matmul")
    assert abs(so.trace(m) - float(d["r5_matmul_trace"])) <= 1e-12 * abs(float(d["r5_matmul_trace"]))


def test_su2_oracle_ctmrg_matches_reference_run():
    """SU(2) SequentialCTMRG of the oracle from the reference's simple-update
    tensors: chi after every iteration and the final rdms."""
    d = load("simple_update_su2")
    A = from_dic(d, "A0")
    B = from_dic(d, "A1")
    ctm = co.SequentialCTMRG(A, B, 20, cutoff=1e-10, degen_ratio=0.9999)
    for _ in range(3):
        ctm.iterate()
    for x, y in ctm.coords:
        r12 = co.ctm_rdm1x2(ctm, x, y)
        r21 = co.ctm_rdm2x1(ctm, x, y)
        assert np.abs(r12 - d[f"rdm1x2_{x}{y}"]).max() < 1e-8
        assert np.abs(r21 - d[f"rdm2x1_{x}{y}"]).max() < 1e-8
