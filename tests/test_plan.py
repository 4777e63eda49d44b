"""Host logic of the abelian permute: the elementary-block tables, applied by a
numpy emulation of the kernel's index arithmetic, reproduce the oracle (and so
the reference) bit for bit, including transposed storage, missing blocks and
unsorted Z2 representations."""

import numpy as np
import pytest

from frostspin_b200.symmetric_tensor.abelian_plan import (
    build_abelian_permute_plan,
    emulate_permute,
)
from oracle import frostspin_oracle as fo
from tests.helpers import load, oracle_from_dic


def pack(t, *, trans=False, rng=None):
    """Oracle tensor -> (buffer, offsets, shapes) with optional F-order storage
    and shuffled block offsets."""
    order = np.arange(len(t.blocks))
    if rng is not None:
        rng.shuffle(order)
    offsets = np.zeros(len(t.blocks), dtype=np.int64)
    parts = []
    pos = 0
    for i in order:
        b = t.blocks[i]
        flat = (b.T if trans else b).ravel()
        offsets[i] = pos
        parts.append(flat)
        pos += flat.size
    buf = np.concatenate(parts) if parts else np.zeros(0)
    shapes = np.array([b.shape for b in t.blocks], dtype=np.int64).reshape(-1, 2)
    return buf, offsets, shapes


def run_plan(t, axes, nrr, *, trans=False, rng=None):
    buf, offs, shapes = pack(t, trans=trans, rng=rng)
    plan = build_abelian_permute_plan(
        list(t.row_reps + t.col_reps), t.signature, t.nrr, t.block_irreps, offs,
        shapes, trans, buf.size, axes, nrr,
    )
    out = emulate_permute(plan, buf)
    assert not np.isnan(out).any()
    blocks = [
        out[o : o + m * n].reshape(m, n)
        for o, (m, n) in zip(plan.offsets, plan.block_shapes, strict=True)
    ]
    return plan, blocks


def check_against_oracle(t, axes, nrr, **kw):
    plan, blocks = run_plan(t, axes, nrr, **kw)
    ref = fo.permute(t, axes[:nrr], axes[nrr:])
    assert np.array_equal(plan.block_irreps, ref.block_irreps)
    assert len(blocks) == len(ref.blocks)
    for b, r in zip(blocks, ref.blocks, strict=True):
        assert b.shape == r.shape
        assert np.array_equal(b, r)


@pytest.mark.parametrize("name", ["u1_reference_test", "z2_rank6"])
@pytest.mark.parametrize("trans", [False, True])
def test_plan_matches_reference_golden(name, trans):
    d = load(name)
    t = oracle_from_dic(d, "in")
    rng = np.random.default_rng(3)
    i = 0
    while f"perm{i}_axes" in d:
        axes = tuple(int(a) for a in d[f"perm{i}_axes"])
        nrr = int(d[f"perm{i}_nrr"])
        ref = oracle_from_dic(d, f"perm{i}")
        plan, blocks = run_plan(t, axes, nrr, trans=trans, rng=rng)
        assert np.array_equal(plan.block_irreps, ref.block_irreps)
        for b, r in zip(blocks, ref.blocks, strict=True):
            assert np.array_equal(b, r)
        i += 1


def test_plan_microbench_small():
    d = load("u1_microbench_small")
    t1 = oracle_from_dic(d, "t1")
    ref = oracle_from_dic(d, "perm")
    plan, blocks = run_plan(t1, (0, 2, 1, 3), 2)
    assert np.array_equal(plan.block_irreps, ref.block_irreps)
    for b, r in zip(blocks, ref.blocks, strict=True):
        assert np.array_equal(b, r)
    # the U(1) microbench merges legs so that EBs stay few and large
    assert plan.ebs.size < 1000


def random_reps(rng, nlegs, z2):
    reps = []
    for _ in range(nlegs):
        n = int(rng.integers(1, 6))
        if z2:
            r = rng.choice(np.array([-128, 0], dtype=np.int8), size=n)
        else:
            r = rng.integers(-3, 4, size=n).astype(np.int8)
        reps.append(r)
    return reps


@pytest.mark.parametrize("seed", range(12))
def test_plan_random_tensors(seed):
    rng = np.random.default_rng(100 + seed)
    ndim = int(rng.integers(2, 7))
    nrr = int(rng.integers(1, ndim))
    z2 = seed % 2 == 0
    for _ in range(20):
        reps = random_reps(rng, ndim, z2)
        sig = rng.integers(0, 2, size=ndim).astype(bool)
        irr, shapes = fo.get_block_sizes(reps[:nrr], reps[nrr:], sig)
        if irr.size:
            break
    else:
        pytest.skip("no allowed block")
    blocks = [rng.standard_normal(tuple(s)) for s in shapes]
    # drop a block to exercise absent sources (zero fill)
    if len(blocks) > 1 and seed % 3 == 0:
        blocks.pop(0)
        irr = irr[1:]
    t = fo.OTensor(reps[:nrr], reps[nrr:], blocks, irr, sig)
    for _ in range(4):
        axes = tuple(int(a) for a in rng.permutation(ndim))
        new_nrr = int(rng.integers(1, ndim))
        check_against_oracle(t, axes, new_nrr, trans=bool(seed % 4 == 1), rng=rng)


def test_task_tables_cover_every_row_once():
    from frostspin_b200.symmetric_tensor.abelian_plan import MAX_TASK_ROWS, _make_tasks

    d = load("u1_microbench_small")
    t1 = oracle_from_dic(d, "t1")
    plan, _ = run_plan(t1, (0, 2, 1, 3), 2)
    r = plan.ebs["ndim"].astype(np.int64)
    inner = plan.ebs["dims"][np.arange(plan.ebs.size), r - 1].astype(np.int64)
    rows = plan.ebs["volume"].astype(np.int64) // inner
    for chunk in (1, 7, 64, 8192, 10**7):
        tasks = _make_tasks(plan.ebs, chunk)
        covered = np.zeros(plan.ebs.size, dtype=np.int64)
        for t in tasks:
            assert t["start"] == covered[t["eb"]]
            assert 1 <= t["count"] <= MAX_TASK_ROWS
            covered[t["eb"]] += t["count"]
        assert np.array_equal(covered, rows)


def test_tile_runs_order_and_layout():
    """The FsTileRun table of a DMMA launch (linalg._tile_runs): problems in the
    given order with their tile counts as consecutive runs, wide problems
    (more tile columns than rows) column-major, empty problems taking no
    tiles; expanding it as fs_expand_tiles does enumerates every tile once."""
    from frostspin_b200 import linalg

    ncol = np.array([3, 4, 1, 2, 2, 5, 1], dtype=np.int64)
    nrow = np.array([2, 0, 1, 6, 0, 1, 0], dtype=np.int64)
    ntile = ncol * nrow
    order = np.array([3, 1, 0, 6, 2, 5, 4])
    runs, total = linalg._tile_runs(ntile, ncol, order, nrow)
    assert total == int(ntile.sum())
    assert list(runs["problem"]) == list(order)
    assert list(runs["start"]) == list(np.cumsum(ntile[order]) - ntile[order])
    assert list(runs["col_major"]) == [int(ncol[p] > nrow[p]) for p in order]
    tiles = []
    for t in range(total):
        r = runs[np.searchsorted(runs["start"], t, side="right") - 1]
        k = t - int(r["start"])
        if r["col_major"]:
            tiles.append((int(r["problem"]), k % int(r["nrow"]), k // int(r["nrow"])))
        else:
            tiles.append((int(r["problem"]), k // int(r["ncol"]), k % int(r["ncol"])))
    assert sorted(tiles) == sorted((p, i, j) for p in range(7) for i in range(nrow[p])
                                   for j in range(ncol[p]))
