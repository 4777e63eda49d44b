"""Pin the O(2) CPU oracle against outputs of the reference implementation
(tests/golden/o2.npz, inputs of the reference's tests/test_o2_tensor.py plus a
mixed-signature tensor): block structure bit-exact, values to 1e-13 of the
largest entry."""

import numpy as np
import pytest

from oracle import frostspin_oracle as uo
from oracle import o2_oracle as oo
from tests.helpers import load

TOL = 1e-13
NAMES = ["base", "noodd", "noeven", "nozero", "onlyzero", "doublets", "oddfix", "evenfix", "sig"]


def from_dic(d, prefix, mod=oo):
    nrr = int(d[prefix + "_n_row_reps"])
    ncr = int(d[prefix + "_n_col_reps"])
    rr = [d[f"{prefix}_row_rep_{i}"] for i in range(nrr)]
    cr = [d[f"{prefix}_col_rep_{i}"] for i in range(ncr)]
    irr = d[prefix + "_block_irreps"]
    return mod.OTensor(rr, cr, [d[f"{prefix}_block_{i}"] for i in range(irr.size)], irr,
                       d[prefix + "_signature"])


def check(t, d, prefix, mod=oo):
    ref = from_dic(d, prefix, mod)
    assert np.array_equal(t.block_irreps, ref.block_irreps), prefix
    for a, b in zip(t.row_reps + t.col_reps, ref.row_reps + ref.col_reps, strict=True):
        assert np.array_equal(a, b), prefix
    assert np.array_equal(t.signature, ref.signature), prefix
    scale = max([np.abs(b).max() for b in ref.blocks if b.size] + [1e-300])
    for a, b in zip(t.blocks, ref.blocks, strict=True):
        assert a.shape == b.shape, prefix
        assert np.abs(a - b).max(initial=0.0) <= TOL * scale, prefix


def perms(d, name):
    i = 0
    while f"{name}_perm{i}_axes" in d:
        pre = f"{name}_perm{i}"
        axes = tuple(int(a) for a in d[pre + "_axes"])
        nrr = int(d[pre + "_nrr"])
        yield pre, axes[:nrr], axes[nrr:]
        i += 1


@pytest.mark.parametrize("name", NAMES)
def test_o2_oracle_casts_and_dense(name):
    d = load("o2")
    t = from_dic(d, name)
    check(oo.to_u1(t), d, name + "_u1", uo)
    dense = d[name + "_dense"]
    assert np.abs(oo.toarray(t) - dense).max() <= TOL * max(np.abs(dense).max(), 1)
    back = oo.from_array(dense, t.row_reps, t.col_reps, t.signature)
    if back.block_irreps.size == t.block_irreps.size:
        check(back, d, name)
    else:  # blocks the fixture left out come back explicitly, as zeros
        kept = np.isin(back.block_irreps, t.block_irreps)
        assert all(np.abs(b).max() <= 1e-15 for b, k in zip(back.blocks, kept, strict=True)
                   if not k)
    assert np.abs(oo.toarray(back) - dense).max() <= TOL * max(np.abs(dense).max(), 1)


@pytest.mark.parametrize("name", NAMES)
def test_o2_oracle_permute_and_transpose(name):
    d = load("o2")
    t = from_dic(d, name)
    n = 0
    for pre, ra, ca in perms(d, name):
        p = oo.permute(t, ra, ca)
        check(p, d, pre)
        check(oo.to_u1(p), d, pre + "_u1", uo)
        n += 1
    assert n >= 2
    check(oo.transpose(t), d, name + "_transpose")


def test_o2_oracle_group_data_and_linear_algebra():
    d = load("o2")
    t = from_dic(d, "base")
    assert np.array_equal(oo.singlet(), [[1], [0]])
    r = np.array([[1, 1, 1, 1], [-1, 0, 1, 2]])
    assert np.array_equal(oo.rep_to_u1(r), [0, 0, 1, -1, 2, -2])
    perm, sign = oo.reflection_perm_sign(r)
    assert np.array_equal(perm, [0, 1, 3, 2, 5, 4])
    assert np.array_equal(sign, [-1, 1, 1, -1, 1, 1])
    assert np.array_equal(oo.rep_to_u1(np.array([[1, 2, 1, 2], [-1, 0, 1, 2]])),
                          [0, 0, 0, 1, -1, 2, 2, -2, -2])
    assert abs(oo.norm(t) - float(d["base_norm"])) <= 1e-14
    check(oo.dagger(t), d, "base_dagger")
    check(oo.matmul(t, oo.dagger(t)), d, "base_matmul")
    # combine agrees with the block structure the reference stored
    irr, shapes = oo.get_block_sizes(t.row_reps, t.col_reps, t.signature)
    assert np.array_equal(irr, t.block_irreps)
    assert np.array_equal(shapes, [b.shape for b in t.blocks])


@pytest.mark.parametrize("name", ["su2cast_int", "su2cast_half", "su2cast_mixed"])
def test_o2_oracle_su2_cast(name):
    from oracle import su2_oracle as so

    d = load("o2")
    ts = from_dic(d, name + "_su2", so)
    got = oo.from_su2_dense(so.toarray(ts), ts.row_reps, ts.col_reps, ts.signature)
    check(got, d, name)
