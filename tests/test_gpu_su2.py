"""SU(2) tensors on the device against the reference (tests/golden/su2.npz).

Block structure (irreps, shapes, representations, signatures) must be
bit-identical; values agree to 1e-13 relative to the largest entry (the
recoupling GEMMs sum in a different order than the reference's numba loops).
Cases follow the reference's tests/test_su2_tensor.py (known answers, permute
round trips, external degeneracies, missing blocks, casts) plus random
tensors with several irreps per leg.
"""

import numpy as np
import pytest

from tests.helpers import load

pytestmark = pytest.mark.gpu

TOL = 1e-13


def su2_from(d, prefix):
    from frostspin_b200 import SU2SymmetricTensor

    return SU2SymmetricTensor.load_from_dic(d, prefix=prefix)


def ref_blocks(d, prefix):
    irr = d[prefix + "_block_irreps"]
    return irr, [d[f"{prefix}_block_{i}"] for i in range(irr.size)]


def check_against(t, d, prefix, tol=TOL):
    irr, blocks = ref_blocks(d, prefix)
    assert np.array_equal(t.block_irreps, irr), prefix
    nrr = int(d[prefix + "_n_row_reps"])
    assert t.n_row_reps == nrr
    for i, r in enumerate(t.row_reps):
        assert np.array_equal(r, d[f"{prefix}_row_rep_{i}"])
    for i, r in enumerate(t.col_reps):
        assert np.array_equal(r, d[f"{prefix}_col_rep_{i}"])
    assert np.array_equal(t.signature, d[prefix + "_signature"])
    got = t.host_blocks()
    scale = max([np.abs(b).max() for b in blocks] + [1e-300])
    for g, b in zip(got, blocks, strict=True):
        assert g.shape == b.shape, prefix
        assert np.abs(g - b).max() <= tol * scale, prefix


def permute_cases(d, base):
    i = 0
    while f"{base}_perm{i}_axes" in d:
        pre = f"{base}_perm{i}"
        axes = tuple(int(a) for a in d[pre + "_axes"])
        nrr = int(d[pre + "_nrr"])
        yield pre, axes[:nrr], axes[nrr:]
        i += 1


@pytest.mark.parametrize("fused", [False, True])
@pytest.mark.parametrize("base", ["sds", "sdsb", "ext", "miss", "r5", "r6"])
def test_su2_permute_matches_reference(base, fused):
    """Every permute case of the reference's tensors, through the three
    launches and through the fused kernel."""
    from frostspin_b200.symmetric_tensor import lie_group_symmetric_tensor as lg

    d = load("su2")
    t = su2_from(d, base)
    n = 0
    was = lg.fused_permute_enabled()
    lg.set_fused_permute(fused)
    try:
        for pre, ra, ca in permute_cases(d, base):
            p = t.permute(ra, ca)
            check_against(p, d, pre)
            if pre + "_dense" in d:
                dense = d[pre + "_dense"]
                assert np.abs(p.toarray() - dense).max() <= TOL * max(np.abs(dense).max(), 1)
            n += 1
    finally:
        lg.set_fused_permute(was)
    assert n >= 2


@pytest.mark.parametrize("base", ["r5", "r6"])
def test_su2_permute_of_transposed_storage(base):
    """dagger() flips the storage order; the permute reads through it."""
    d = load("su2")
    t = su2_from(d, base)
    tt = t.dagger().dagger()  # same tensor, blocks read through two flips
    for pre, ra, ca in permute_cases(d, base):
        check_against(tt.permute(ra, ca), d, pre)
    # a genuinely F-order input: permute the dagger and compare with the
    # dagger of the reference tensor's dense form
    dg = t.dagger()
    nd = dg.ndim
    axes = tuple(range(1, nd)) + (0,)
    p = dg.permute(axes[:2], axes[2:])
    dense = np.asarray(d[base + "_dense"]) if base + "_dense" in d else t.toarray()
    nrr = t.n_row_reps
    ref = dense.transpose(tuple(range(nrr, t.ndim)) + tuple(range(nrr))).transpose(axes)
    assert np.abs(p.toarray() - ref).max() <= TOL * max(np.abs(ref).max(), 1)


def test_su2_known_answers():
    """tests/test_su2_tensor.py:117-140 of the reference."""
    from frostspin_b200 import SU2SymmetricTensor

    d = load("su2")
    sds = d["sds_dense"]
    r = np.array([[1], [2]])
    st = SU2SymmetricTensor.from_array(sds, (r, r), (r, r))
    assert st.nblocks == 2
    assert np.array_equal(st.block_irreps, [1, 3])
    b = st.host_blocks()
    assert abs(b[0][0, 0] + 0.75) < 1e-14
    assert abs(b[1][0, 0] - 0.25) < 1e-14
    assert abs(np.linalg.norm(sds) - st.norm()) < 1e-14
    assert np.abs(st.toarray() - sds).max() < 1e-14
    assert np.abs(st.dual().toarray() - sds).max() < 1e-14
    assert abs(st.trace()) < 1e-14
    # permute round trips
    stp = st.permute((0, 1, 2), (3,))
    stp2 = SU2SymmetricTensor.from_array(sds, (r, r, r), (r,), signature=[0, 0, 1, 1])
    assert (stp - stp2).norm() < 1e-14
    assert (st - stp.permute((0, 1), (2, 3))).norm() < 1e-14
    stp = st.permute((3, 0, 2), (1,))
    stp2 = SU2SymmetricTensor.from_array(sds.transpose(3, 0, 2, 1), (r, r, r), (r,),
                                         signature=[1, 0, 1, 0])
    assert (stp - stp2).norm() < 1e-14
    assert (st - stp.permute((1, 3), (2, 0))).norm() < 1e-14
    # scalar operations
    assert np.abs((st / 2).toarray() - sds / 2).max() < 1e-14
    assert np.abs((2 * st).toarray() - 2 * sds).max() < 1e-14


@pytest.mark.parametrize("base", ["sds", "sdsb", "ext", "r5"])
def test_su2_dense_conversions(base):
    from frostspin_b200 import SU2SymmetricTensor

    d = load("su2")
    t = su2_from(d, base)
    dense = d[base + "_dense"]
    assert np.abs(t.toarray() - dense).max() <= TOL * max(np.abs(dense).max(), 1)
    back = SU2SymmetricTensor.from_array(dense, t.row_reps, t.col_reps, t.signature)
    check_against(back, d, base)


def test_su2_missing_blocks_round_trip():
    """tests/test_su2_tensor.py:200-212 of the reference."""
    from frostspin_b200 import SU2SymmetricTensor

    d = load("su2")
    t = su2_from(d, "miss")
    tp = t.permute((3, 2, 1), (0, 5, 4))
    tp2 = tp.permute((3, 2, 1), (0, 5, 4))
    # the permutation is an involution: two applications give t back
    assert (tp2 - t).norm() <= 1e-13 * t.norm()
    td = t.toarray()
    t2 = SU2SymmetricTensor.from_array(td, t.row_reps, t.col_reps, t.signature)
    assert (t - t2).norm() <= 1e-13 * t.norm()


def test_su2_linear_algebra_matches_reference():
    d = load("su2")
    t = su2_from(d, "r5")
    check_against(t.transpose(), d, "r5_transpose")
    check_against(t.dagger(), d, "r5_dagger")
    assert abs(t.norm() - float(d["r5_norm"])) <= 1e-13 * float(d["r5_norm"])
    m = t @ t.dagger()
    check_against(m, d, "r5_matmul")
    assert abs(m.trace() - float(d["r5_matmul_trace"])) <= 1e-12 * abs(float(d["r5_matmul_trace"]))
    _, s, _ = m.truncated_svd(7)
    irr = d["r5_tsvd_s_block_irreps"]
    assert np.array_equal(s.block_irreps, irr)
    for i, blk in enumerate(s.diagonal_blocks):
        ref = d[f"r5_tsvd_s_diagonal_block_{i}"]
        np.testing.assert_allclose(blk.detach().cpu().numpy(), ref, rtol=1e-12, atol=1e-14)


def test_su2_cast_to_u1():
    d = load("su2")
    t = su2_from(d, "r5")
    u = t.toU1()
    assert np.abs(u.toarray() - d["r5_dense"]).max() <= TOL * np.abs(d["r5_dense"]).max()
    assert abs(u.norm() - t.norm()) <= 1e-13 * t.norm()


@pytest.mark.parametrize("fused", [True, False])
def test_su2_native_kernels_launched(fused):
    """The SU(2) permute runs through the C-ABI: with the fused kernel (the
    default) one launch takes the simple blocks with small recoupling
    matrices; without it, gather, recoupling GEMM and scatter launches.  Both
    give the reference's blocks."""
    from frostspin_b200 import _native
    from frostspin_b200.symmetric_tensor import lie_group_symmetric_tensor as lg

    d = load("su2")
    t = su2_from(d, "r5")
    was = lg.fused_permute_enabled()
    lg.set_fused_permute(fused)
    try:
        before = dict(_native.CALL_COUNTS)
        p = t.permute((3, 0, 2), (1, 4))
        after = dict(_native.CALL_COUNTS)
        lg.set_fused_permute(not fused)
        q = t.permute((3, 0, 2), (1, 4))
    finally:
        lg.set_fused_permute(was)

    def delta(*names):
        return sum(after.get(k, 0) - before.get(k, 0) for k in names)

    gemms = delta("fs_grouped_dgemm", "fs_grouped_dgemm_uniform", "fs_grouped_dgemm_thin")
    if fused:
        assert delta("fs_su2_permute_fused") == 1
        # blocks beyond the fused kernel's limits, if any, take the other path
        assert delta("fs_abelian_permute") in (0, 2)
    else:
        assert delta("fs_su2_permute_fused") == 0
        assert delta("fs_abelian_permute") == 2
        assert 1 <= gemms <= 2  # thin groups and tiled groups, one launch each
    for a, b in zip(p.host_blocks(), q.host_blocks(), strict=True):
        assert np.abs(a - b).max() <= TOL * max(1.0, np.abs(b).max())
