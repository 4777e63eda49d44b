"""Host logic of the O(2) data plane, on the CPU.

The O(2) casts and permute are fs_o2_recombine maps around the abelian permute.
Here their host tables are applied by numpy emulations of the kernels' index
arithmetic (same products, same order) and compared with outputs of the
reference implementation (tests/golden/o2.npz): block structure bit-exact,
values to 1e-14 of the largest entry.
"""

import numpy as np
import pytest
import torch

from frostspin_b200 import _native
from frostspin_b200.symmetric_tensor import O2SymmetricTensor, U1SymmetricTensor
from frostspin_b200.symmetric_tensor import o2_symmetric_tensor as o2m
from frostspin_b200.symmetric_tensor.abelian_plan import emulate_permute
from tests.helpers import load

TOL = 1e-14
NAMES = ["base", "noodd", "noeven", "nozero", "onlyzero", "doublets", "oddfix", "evenfix", "sig"]


def emulate_recombine(plan, src):
    out = np.full(plan.out_len, np.nan)
    for rec in plan.blocks:
        nr, nc, nt = int(rec["nrows"]), int(rec["ncols"]), int(rec["nterms"])
        assert 1 <= nt <= _native.FS_O2_MAXTERMS
        acc = np.zeros((nr, nc))
        for t in range(nt):
            tm = rec["terms"][t]
            ri = plan.index[tm["ridx_off"] : tm["ridx_off"] + nr]
            ci = plan.index[tm["cidx_off"] : tm["cidx_off"] + nc]
            rc = plan.coef[tm["rcoef_off"] : tm["rcoef_off"] + nr]
            cc = plan.coef[tm["ccoef_off"] : tm["ccoef_off"] + nc]
            pos = tm["src_off"] + ri[:, None] * tm["rs"] + ci[None, :] * tm["cs"]
            assert (pos >= 0).all() and (pos < src.size).all()
            acc = acc + (rc[:, None] * src[pos]) * cc[None, :]
        out[rec["out_off"] : rec["out_off"] + nr * nc] = acc.ravel()
    assert not np.isnan(out).any()
    return out


def host_tensor(cls, d, prefix, trans=False):
    """Fixture -> tensor object on a CPU torch buffer (plans only)."""
    nrr = int(d[prefix + "_n_row_reps"])
    ncr = int(d[prefix + "_n_col_reps"])
    rr = [d[f"{prefix}_row_rep_{i}"] for i in range(nrr)]
    cr = [d[f"{prefix}_col_rep_{i}"] for i in range(ncr)]
    irr = d[prefix + "_block_irreps"]
    blocks = [d[f"{prefix}_block_{i}"] for i in range(irr.size)]
    flat = [(b.T if trans else b).ravel() for b in blocks]
    shapes = np.array([b.shape for b in blocks], dtype=np.int64).reshape(-1, 2)
    offsets = np.zeros(len(blocks), dtype=np.int64)
    if len(blocks) > 1:
        offsets[1:] = np.cumsum(shapes[:-1, 0] * shapes[:-1, 1])
    data = torch.from_numpy(np.concatenate(flat) if flat else np.zeros(0))
    return cls._from_storage(rr, cr, data, offsets, shapes, irr, d[prefix + "_signature"],
                             trans)


def blocks_of(flat, offsets, shapes, trans=False):
    out = []
    for o, (m, n) in zip(offsets, shapes, strict=True):
        b = flat[o : o + m * n]
        out.append(b.reshape(n, m).T if trans else b.reshape(m, n))
    return out


def check(irreps, blocks, d, prefix):
    ref_irr = d[prefix + "_block_irreps"]
    assert np.array_equal(np.asarray(irreps, dtype=np.int64), ref_irr.astype(np.int64)), prefix
    ref = [d[f"{prefix}_block_{i}"] for i in range(ref_irr.size)]
    scale = max([np.abs(b).max() for b in ref if b.size] + [1e-300])
    for g, b in zip(blocks, ref, strict=True):
        assert g.shape == b.shape, prefix
        assert np.abs(g - b).max(initial=0.0) <= TOL * scale, prefix


def perms(d, name):
    i = 0
    while f"{name}_perm{i}_axes" in d:
        pre = f"{name}_perm{i}"
        axes = tuple(int(a) for a in d[pre + "_axes"])
        yield pre, axes, int(d[pre + "_nrr"])
        i += 1


@pytest.mark.parametrize("trans", [False, True])
@pytest.mark.parametrize("name", NAMES)
def test_o2_to_u1_tables_match_reference(name, trans):
    d = load("o2")
    t = host_tensor(O2SymmetricTensor, d, name, trans=trans)
    plan = o2m._to_u1_plan(t)
    out = emulate_recombine(plan, t.data.numpy())
    check(plan.irreps, blocks_of(out, plan.offsets, plan.shapes), d, name + "_u1")


@pytest.mark.parametrize("name", NAMES)
def test_o2_from_u1_tables_match_reference(name):
    d = load("o2")
    tu1 = host_tensor(U1SymmetricTensor, d, name + "_u1")
    t = host_tensor(O2SymmetricTensor, d, name)
    plan = o2m._from_u1_plan(tu1, t.row_reps, t.col_reps)
    out = emulate_recombine(plan, tu1.data.numpy())
    got = blocks_of(out, plan.offsets, plan.shapes)
    if len(plan.irreps) == t.nblocks:
        check(plan.irreps, got, d, name)
    else:  # blocks the fixture left out come back as explicit zeros
        ref_irr = list(d[name + "_block_irreps"])
        for q, b in zip(plan.irreps, got, strict=True):
            if q in ref_irr:
                ref = d[f"{name}_block_{ref_irr.index(q)}"]
                assert np.abs(b - ref).max() <= TOL * max(np.abs(ref).max(), 1e-300)
            else:
                assert np.abs(b).max() == 0.0


@pytest.mark.parametrize("trans", [False, True])
@pytest.mark.parametrize("name", NAMES)
def test_o2_permute_pipeline_matches_reference(name, trans):
    """cast (fs_o2_recombine) -> abelian permute (fs_abelian_permute) -> cast
    back, all three applied by emulation of the device kernels."""
    d = load("o2")
    t = host_tensor(O2SymmetricTensor, d, name, trans=trans)
    p_to = o2m._to_u1_plan(t)
    u1_flat = emulate_recombine(p_to, t.data.numpy())
    tu1 = U1SymmetricTensor._from_storage(
        [o2m.rep_to_u1(r) for r in t.row_reps], [o2m.rep_to_u1(r) for r in t.col_reps],
        torch.from_numpy(u1_flat), p_to.offsets, p_to.shapes,
        np.asarray(p_to.irreps, dtype=np.int8), t.signature)
    reps = t.row_reps + t.col_reps
    n = 0
    for pre, axes, nrr in perms(d, name):
        aplan = tu1._permute_plan(axes, nrr)
        pflat = emulate_permute(aplan, u1_flat)
        sig = t.signature[list(axes)]
        pu1 = U1SymmetricTensor._from_storage(
            [tu1.row_reps[a] if a < tu1.n_row_reps else tu1.col_reps[a - tu1.n_row_reps]
             for a in axes[:nrr]],
            [tu1.row_reps[a] if a < tu1.n_row_reps else tu1.col_reps[a - tu1.n_row_reps]
             for a in axes[nrr:]],
            torch.from_numpy(pflat), aplan.offsets, aplan.block_shapes, aplan.block_irreps, sig)
        back = o2m._from_u1_plan(pu1, [reps[a] for a in axes[:nrr]], [reps[a] for a in axes[nrr:]])
        out = emulate_recombine(back, pflat)
        check(back.irreps, blocks_of(out, back.offsets, back.shapes), d, pre)
        n += 1
    assert n >= 2


@pytest.mark.parametrize("trans", [False, True])
@pytest.mark.parametrize("name", NAMES)
def test_o2_transpose_tables_match_reference(name, trans):
    d = load("o2")
    t = host_tensor(O2SymmetricTensor, d, name, trans=trans)
    plan = o2m._transpose_plan(t)
    out = emulate_recombine(plan, t.data.numpy())
    # written in C order of the current shape, read back transposed
    check(plan.irreps, blocks_of(out, plan.offsets, plan.shapes[:, ::-1], trans=True), d,
          name + "_transpose")


def test_o2_structure_functions():
    d = load("o2")
    t = host_tensor(O2SymmetricTensor, d, "base")
    irr, shapes = O2SymmetricTensor.get_block_sizes(t.row_reps, t.col_reps, t.signature)
    assert np.array_equal(irr, t.block_irreps)
    assert np.array_equal(shapes, t.block_shapes)
    assert O2SymmetricTensor.symmetry() == "O2"
    assert np.array_equal(O2SymmetricTensor.singlet(), [[1], [0]])
    assert O2SymmetricTensor.irrep_dimension(-1) == 1
    assert O2SymmetricTensor.irrep_dimension(0) == 1
    assert O2SymmetricTensor.irrep_dimension(3) == 2
    r = np.array([[1, 2, 1, 2], [-1, 0, 1, 2]])
    assert np.array_equal(o2m.rep_to_u1(r), [0, 0, 0, 1, -1, 2, 2, -2, -2])
    assert O2SymmetricTensor.representation_dimension(r) == 9


def test_su2_to_o2_leg_maps_match_oracle():
    """Per-leg order, signs and O(2) representation of the SU(2) -> O(2) cast
    (su2_symmetric_tensor.py:272-304) against the oracle's loop restatement."""
    from oracle import o2_oracle as oo
    from frostspin_b200.symmetric_tensor.su2_symmetric_tensor import _o2_leg

    rng = np.random.default_rng(4)
    for _ in range(200):
        k = int(rng.integers(1, 5))
        irr = np.sort(rng.choice(np.arange(1, 12), k, replace=False))
        rep = np.array([rng.integers(1, 4, k), irr])
        r1, o1, s1 = _o2_leg(rep)
        r2, o2, s2 = oo.su2_leg_to_o2(rep)
        assert np.array_equal(r1, r2) and np.array_equal(o1, o2) and np.array_equal(s1, s2)


def _random_o2_rep(rng):
    irreps = [q for q in (-1, 0) if rng.random() < 0.6]
    irreps += sorted(rng.choice(np.arange(1, 4), int(rng.integers(1, 3)), replace=False).tolist())
    return np.array([rng.integers(1, 3, len(irreps)), irreps])


@pytest.mark.parametrize("seed", range(12))
def test_o2_permute_pipeline_random_against_oracle(seed):
    """Random O(2) tensors (with or without 0odd / 0even on each leg, any
    signature, plain or transposed storage), random permutations: the
    emulated device pipeline equals the oracle's permute, itself pinned to the
    reference's outputs."""
    from oracle import o2_oracle as oo

    rng = np.random.default_rng(100 + seed)
    ndim = int(rng.integers(3, 6))
    nrr = int(rng.integers(1, ndim))
    reps = [_random_o2_rep(rng) for _ in range(ndim)]
    sig = rng.random(ndim) < 0.5
    ot = oo.random(reps[:nrr], reps[nrr:], sig, rng=rng)
    if ot.block_irreps.size == 0:
        return
    trans = bool(seed % 2)
    flat = np.concatenate([(b.T if trans else b).ravel() for b in ot.blocks])
    shapes = np.array([b.shape for b in ot.blocks], dtype=np.int64)
    offsets = np.concatenate(([0], np.cumsum(shapes[:, 0] * shapes[:, 1])[:-1]))
    t = O2SymmetricTensor._from_storage(reps[:nrr], reps[nrr:], torch.from_numpy(flat), offsets,
                                        shapes, ot.block_irreps, sig, trans)
    p_to = o2m._to_u1_plan(t)
    u1_flat = emulate_recombine(p_to, flat)
    tu1 = U1SymmetricTensor._from_storage(
        [o2m.rep_to_u1(r) for r in reps[:nrr]], [o2m.rep_to_u1(r) for r in reps[nrr:]],
        torch.from_numpy(u1_flat), p_to.offsets, p_to.shapes,
        np.asarray(p_to.irreps, dtype=np.int8), sig)
    for _ in range(3):
        axes = tuple(int(a) for a in rng.permutation(ndim))
        new_nrr = int(rng.integers(1, ndim))
        aplan = tu1._permute_plan(axes, new_nrr)
        pflat = emulate_permute(aplan, u1_flat)
        u1reps = tu1.row_reps + tu1.col_reps
        pu1 = U1SymmetricTensor._from_storage(
            [u1reps[a] for a in axes[:new_nrr]], [u1reps[a] for a in axes[new_nrr:]],
            torch.from_numpy(pflat), aplan.offsets, aplan.block_shapes, aplan.block_irreps,
            sig[list(axes)])
        back = o2m._from_u1_plan(pu1, [reps[a] for a in axes[:new_nrr]],
                                 [reps[a] for a in axes[new_nrr:]])
        got = blocks_of(emulate_recombine(back, pflat), back.offsets, back.shapes)
        ref = oo.permute(ot, axes[:new_nrr], axes[new_nrr:])
        assert np.array_equal(np.asarray(back.irreps), ref.block_irreps)
        for g, b in zip(got, ref.blocks, strict=True):
            assert g.shape == b.shape
            assert np.abs(g - b).max(initial=0.0) <= 1e-14 * max(1.0, np.abs(b).max())
    # the transpose map too
    tp = o2m._transpose_plan(t)
    got = blocks_of(emulate_recombine(tp, flat), tp.offsets, tp.shapes[:, ::-1], trans=True)
    ref = oo.transpose(ot)
    for g, b in zip(got, ref.blocks, strict=True):
        assert np.abs(g - b).max(initial=0.0) <= 1e-14 * max(1.0, np.abs(b).max())
