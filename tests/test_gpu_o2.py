"""O(2) tensors on the device against the reference (tests/golden/o2.npz).

Block structure (irreps, shapes, representations, signatures) must be
bit-identical; values agree to 1e-14 of the largest entry.  Cases follow the
reference's tests/test_o2_tensor.py: U(1) casts both ways, dense conversions,
permutes and transposes, for a generic tensor, tensors with the 0odd, 0even or
both blocks removed, only doublets, only odd or only even fixed points in the
columns, plus a mixed-signature tensor.
"""

import numpy as np
import pytest

from tests.helpers import load

pytestmark = pytest.mark.gpu

TOL = 1e-14
NAMES = ["base", "noodd", "noeven", "nozero", "onlyzero", "doublets", "oddfix", "evenfix", "sig"]


def o2_from(d, prefix):
    from frostspin_b200 import O2SymmetricTensor

    return O2SymmetricTensor.load_from_dic(d, prefix=prefix)


def check_against(t, d, prefix, tol=TOL):
    irr = d[prefix + "_block_irreps"]
    assert np.array_equal(np.asarray(t.block_irreps, dtype=np.int64), irr.astype(np.int64)), prefix
    for i, r in enumerate(t.row_reps):
        assert np.array_equal(r, d[f"{prefix}_row_rep_{i}"]), prefix
    for i, r in enumerate(t.col_reps):
        assert np.array_equal(r, d[f"{prefix}_col_rep_{i}"]), prefix
    assert np.array_equal(t.signature, d[prefix + "_signature"]), prefix
    ref = [d[f"{prefix}_block_{i}"] for i in range(irr.size)]
    scale = max([np.abs(b).max() for b in ref if b.size] + [1e-300])
    for g, b in zip(t.host_blocks(), ref, strict=True):
        assert g.shape == b.shape, prefix
        assert np.abs(g - b).max(initial=0.0) <= tol * scale, prefix


def perms(d, name):
    i = 0
    while f"{name}_perm{i}_axes" in d:
        pre = f"{name}_perm{i}"
        axes = tuple(int(a) for a in d[pre + "_axes"])
        nrr = int(d[pre + "_nrr"])
        yield pre, axes[:nrr], axes[nrr:]
        i += 1


@pytest.mark.parametrize("name", NAMES)
def test_o2_casts_and_dense(name):
    from frostspin_b200 import O2SymmetricTensor, U1SymmetricTensor

    d = load("o2")
    t = o2_from(d, name)
    tu1 = t.toU1()
    check_against(tu1, d, name + "_u1")
    dense = d[name + "_dense"]
    assert np.abs(t.toarray() - dense).max() <= TOL * max(np.abs(dense).max(), 1)
    back = O2SymmetricTensor.from_array(dense, t.row_reps, t.col_reps, t.signature)
    assert (back - t).norm() <= 1e-14
    ref_u1 = U1SymmetricTensor.load_from_dic(d, prefix=name + "_u1")
    again = O2SymmetricTensor.from_U1(ref_u1, t.row_reps, t.col_reps)
    assert (again - t).norm() <= 1e-14


@pytest.mark.parametrize("name", NAMES)
def test_o2_permute_and_transpose_match_reference(name):
    d = load("o2")
    t = o2_from(d, name)
    n = 0
    for pre, ra, ca in perms(d, name):
        p = t.permute(ra, ca)
        check_against(p, d, pre)
        check_against(p.toU1(), d, pre + "_u1")
        dense = d[pre + "_dense"]
        assert np.abs(p.toarray() - dense).max() <= TOL * max(np.abs(dense).max(), 1)
        n += 1
    assert n >= 2
    tt = t.transpose()
    check_against(tt, d, name + "_transpose")
    dense = d[name + "_transpose_dense"]
    assert np.abs(tt.toarray() - dense).max() <= TOL * max(np.abs(dense).max(), 1)


def test_o2_permute_of_transposed_storage():
    """dagger() flips the storage order; the casts read through it."""
    d = load("o2")
    t = o2_from(d, "sig")
    tt = t.dagger().dagger()
    for pre, ra, ca in perms(d, "sig"):
        check_against(tt.permute(ra, ca), d, pre)
    dense = d["sig_dense"]
    nrr = t.n_row_reps
    ref = dense.transpose(tuple(range(nrr, t.ndim)) + tuple(range(nrr)))
    assert np.abs(t.dagger().toarray() - ref).max() <= TOL * np.abs(ref).max()


def test_o2_linear_algebra_matches_reference():
    d = load("o2")
    t = o2_from(d, "base")
    assert abs(t.norm() - float(d["base_norm"])) <= 1e-14
    check_against(t.dagger(), d, "base_dagger")
    check_against(t @ t.dagger(), d, "base_matmul", tol=1e-13)
    # permute round trip: (2, 1, 4 | 0, 3) is undone by (3, 1, 0 | 4, 2)
    p = t.permute((2, 1, 4), (0, 3))
    assert (p.permute((3, 1, 0), (4, 2)) - t).norm() <= 1e-14


def test_o2_native_kernels_launched():
    """The O(2) permute runs through the C-ABI: a cast, the abelian permute and
    the cast back are counted by the native layer."""
    from frostspin_b200 import _native

    d = load("o2")
    t = o2_from(d, "base")
    before = dict(_native.CALL_COUNTS)
    t.permute((2, 1, 4), (0, 3))
    after = _native.CALL_COUNTS
    assert after.get("fs_o2_recombine", 0) - before.get("fs_o2_recombine", 0) == 2
    assert after.get("fs_abelian_permute", 0) - before.get("fs_abelian_permute", 0) == 1


@pytest.mark.parametrize("name", ["su2cast_int", "su2cast_half", "su2cast_mixed"])
def test_su2_to_o2_cast_matches_reference(name):
    """SU2SymmetricTensor.toO2 (su2_symmetric_tensor.py:249-318)."""
    from frostspin_b200 import SU2SymmetricTensor

    d = load("o2")
    ts = SU2SymmetricTensor.load_from_dic(d, prefix=name + "_su2")
    to2 = ts.cast("O2")
    check_against(to2, d, name, tol=1e-13)
    assert abs(to2.norm() - ts.norm()) <= 1e-13 * ts.norm()
