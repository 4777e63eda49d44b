"""Host logic of the SU(2) data plane, on the CPU.

The permute and the dense conversions of an SU(2) tensor are one gather ->
grouped GEMM -> scatter map (tables built on the host, applied on the device).
Here the tables are applied by a numpy emulation of the kernels' index
arithmetic and compared with outputs of the reference implementation
(tests/golden/su2.npz): block structure bit-exact, values to 1e-13.
The Clebsch-Gordan coefficients themselves are pinned against an independent
closed-form evaluation.
"""

import numpy as np
import pytest
import torch

from frostspin_b200.symmetric_tensor import lie_group_symmetric_tensor as lg
from frostspin_b200.symmetric_tensor import su2_cg, su2_fused_plan
from frostspin_b200.symmetric_tensor.abelian_plan import emulate_permute
from frostspin_b200.symmetric_tensor.su2_symmetric_tensor import (
    SU2SymmetricTensor,
    compute_fusion_tensor,
)
from tests.helpers import load

TOL = 1e-13


class _Tables:
    def __init__(self, ebs, size):
        self.ebs = ebs
        self.size = size


def emulate_map(m, src):
    x = emulate_permute(_Tables(m.gather[0], m.x_size), src)
    assert not np.isnan(x).any()
    y_off = np.zeros(m.M.size, dtype=np.int64)
    y_off[1:] = np.cumsum((m.M * m.N)[:-1])
    y = np.empty(int((m.M * m.N).sum()))
    for g in range(m.M.size):
        M, N, K = int(m.M[g]), int(m.N[g]), int(m.K[g])
        U = m.u_host[m.u_off[g] : m.u_off[g] + M * K].reshape(M, K)
        X = x[m.x_off[g] : m.x_off[g] + K * N].reshape(K, N)
        y[y_off[g] : y_off[g] + M * N] = (U @ X).ravel()
    out = emulate_permute(_Tables(m.scatter[0], m.out_size), y)
    if getattr(m, "fused", None) is not None:
        # the simple blocks the fused kernel takes, applied as it indexes them
        su2_fused_plan.check(m.fused[0], m.fused[1], src.size, m.out_size, m.u_host.size)
        su2_fused_plan.emulate(*m.fused, m.u_host, src, out)
    if m.zero_out:
        out = np.nan_to_num(out, nan=0.0)
    assert not np.isnan(out).any()
    return out


def host_tensor(d, prefix, trans=False):
    """Reference fixture -> SU2 tensor object whose buffer is a CPU torch tensor
    (enough for building plans; never handed to a kernel)."""
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
    return SU2SymmetricTensor._from_storage(rr, cr, data, offsets, shapes, irr,
                                            d[prefix + "_signature"], trans)


def ref_blocks(d, prefix):
    irr = d[prefix + "_block_irreps"]
    return irr, [d[f"{prefix}_block_{i}"] for i in range(irr.size)]


def permute_cases(d):
    names = sorted({k.split("perm")[0] for k in d.files if "perm" in k and k.endswith("_axes")})
    for base in names:
        i = 0
        while f"{base}perm{i}_axes" in d:
            yield base.rstrip("_"), i
            i += 1


@pytest.fixture(params=["fused", "three_launch"])
def fused_mode(request):
    """Permute maps built with the fused kernel for the thin simple blocks
    (the default) and without it."""
    was = lg.fused_permute_enabled()
    lg.set_fused_permute(request.param == "fused")
    yield request.param
    lg.set_fused_permute(was)


@pytest.mark.parametrize("trans", [False, True])
def test_su2_permute_tables_match_reference(trans, fused_mode):
    d = load("su2")
    n = 0
    n_fused = 0
    for base, i in permute_cases(d):
        t = host_tensor(d, base, trans=trans)
        pre = f"{base}_perm{i}"
        axes = tuple(int(a) for a in d[pre + "_axes"])
        nrr = int(d[pre + "_nrr"])
        m = t._permute_map(axes, nrr)
        n_fused += m.fused is not None
        out = emulate_map(m, t.data.numpy())
        irr, blocks = ref_blocks(d, pre)
        assert np.array_equal(m.out_irreps, irr), pre
        assert len(blocks) == m.out_shapes.shape[0]
        scale = max(np.abs(b).max() for b in blocks)
        for o, (r, c), b in zip(m.out_offsets, m.out_shapes, blocks, strict=True):
            assert (r, c) == b.shape, pre
            got = out[o : o + r * c].reshape(r, c)
            assert np.abs(got - b).max() <= TOL * scale, pre
        n += 1
    assert n >= 15
    assert (n_fused > 0) == (fused_mode == "fused")


def test_su2_dense_conversions_match_reference():
    d = load("su2")
    for base in ("sds", "sdsb", "ext", "r5"):
        t = host_tensor(d, base)
        dense = d[base + "_dense"]
        # blocks -> dense
        got = emulate_map(t._to_dense_map(), t.data.numpy())
        assert np.abs(got - dense.ravel()).max() <= TOL * max(np.abs(dense).max(), 1)
        # dense -> blocks
        m = SU2SymmetricTensor._from_dense_map(t.row_reps, t.col_reps, t.signature)
        out = emulate_map(m, dense.ravel())
        irr, blocks = ref_blocks(d, base)
        assert np.array_equal(m.out_irreps, irr)
        for o, (r, c), b in zip(m.out_offsets, m.out_shapes, blocks, strict=True):
            assert np.abs(out[o : o + r * c].reshape(r, c) - b).max() <= TOL * max(
                np.abs(b).max(), 1
            )


def test_su2_known_answer_blocks():
    """tests/test_su2_tensor.py:117-123 of the reference: S.S of two spins 1/2 has
    blocks -3/4 (singlet) and 1/4 (triplet)."""
    d = load("su2")
    irr, blocks = ref_blocks(d, "sds")
    assert np.array_equal(irr, [1, 3])
    assert abs(blocks[0][0, 0] + 0.75) < 1e-14
    assert abs(blocks[1][0, 0] - 0.25) < 1e-14


def test_su2_structure_functions():
    r = np.array([[1, 2], [1, 3]])
    assert np.array_equal(SU2SymmetricTensor.combine_representations((r, r), None),
                          [[5, 8, 4], [1, 3, 5]])
    irr, shapes = SU2SymmetricTensor.get_block_sizes(
        (r, r), (r,), np.array([False, False, True])
    )
    assert np.array_equal(irr, [1, 3])
    assert np.array_equal(shapes, [[5, 1], [8, 2]])
    rep, proj = compute_fusion_tensor(np.array([[1], [2]]), np.array([[1], [2]]), False, False)
    assert np.array_equal(rep, [[1, 1], [1, 3]])
    # the fusion tensor is an isometry: P^T P = 1
    p = proj.reshape(4, 4)
    assert np.abs(p.T @ p - np.eye(4)).max() < 1e-15


def test_cg_coefficients_against_closed_form():
    for d1 in range(1, 6):
        for d2 in range(1, 6):
            for d3 in range(abs(d1 - d2) + 1, d1 + d2, 2):
                a = su2_cg.cg_tensor(d1, d2, d3)
                b = su2_cg.cg_tensor_racah(d1, d2, d3)
                assert np.abs(a - b).max() <= 2.3e-16


def test_packaged_cg_table_equals_sympy_evaluation():
    """The packaged table holds sympy's float64 values bit for bit (sampled,
    the largest tensors included), and covers every dimension up to 18."""
    rng = np.random.default_rng(2)
    packed = su2_cg._packed_table()["index"]
    assert (18, 18, 35 - 18) in packed and (17, 5, 13) in packed
    triples = sorted(packed)
    picks = [triples[i] for i in rng.choice(len(triples), 12, replace=False)]
    picks += [(18, 17, 18), (9, 9, 17), (17, 5, 13), (1, 1, 1)]
    for d1, d2, d3 in picks:
        a = su2_cg.cg_tensor(d1, d2, d3)
        b = su2_cg.cg_tensor_sympy(d1, d2, d3)
        assert np.array_equal(a, b), (d1, d2, d3)


@pytest.mark.parametrize("seed", range(10))
def test_su2_permute_tables_random_against_oracle(seed):
    """Random SU(2) tensors (several irreps and degeneracies per leg, any
    signature, plain or transposed storage) and random permutations: the
    gather -> recoupling GEMM -> scatter tables, applied by emulation, equal
    the oracle's permute, itself pinned to the reference's outputs."""
    from oracle import su2_oracle as so

    rng = np.random.default_rng(200 + seed)
    ndim = int(rng.integers(3, 6))
    nrr = int(rng.integers(1, ndim))
    reps = []
    for _ in range(ndim):
        k = int(rng.integers(1, 3))
        irr = np.sort(rng.choice(np.arange(1, 5), k, replace=False))
        reps.append(np.array([rng.integers(1, 3, k), irr]))
    sig = rng.random(ndim) < 0.5
    ot = so.random(reps[:nrr], reps[nrr:], sig, rng=rng)
    if len(ot.blocks) == 0:
        return
    trans = bool(seed % 2)
    flat = np.concatenate([(b.T if trans else b).ravel() for b in ot.blocks])
    shapes = np.array([b.shape for b in ot.blocks], dtype=np.int64)
    offsets = np.concatenate(([0], np.cumsum(shapes[:, 0] * shapes[:, 1])[:-1]))
    t = SU2SymmetricTensor._from_storage(reps[:nrr], reps[nrr:], torch.from_numpy(flat),
                                         offsets, shapes, ot.block_irreps, sig, trans)
    for _ in range(2):
        axes = tuple(int(a) for a in rng.permutation(ndim))
        new_nrr = int(rng.integers(1, ndim))
        m = t._permute_map(axes, new_nrr)
        out = emulate_map(m, flat)
        ref = so.permute(ot, axes[:new_nrr], axes[new_nrr:])
        assert np.array_equal(m.out_irreps, ref.block_irreps)
        scale = max([np.abs(b).max() for b in ref.blocks] + [1e-300])
        for o, (r, c), b in zip(m.out_offsets, m.out_shapes, ref.blocks, strict=True):
            assert (r, c) == b.shape
            assert np.abs(out[o : o + r * c].reshape(r, c) - b).max() <= TOL * scale


@pytest.mark.parametrize("dims", [(), (7,), (3, 5), (2, 9000), (5, 10, 3), (4, 1, 6, 2), (300, 40)])
def test_fused_tasks_cover_columns_within_row_limit(dims):
    """make_tasks: every column of a group in exactly one task, no task spans
    more than TASK_ROWS values of the outer legs, and a row longer than
    TASK_COLUMNS is cut inside the row (the kernel skips and flags a task
    that spans more rows)."""
    from frostspin_b200._native import SU2_GROUP_DTYPE
    from frostspin_b200.symmetric_tensor import su2_fused_plan as sp

    g = np.zeros(1, dtype=SU2_GROUP_DTYPE)
    g["ndim"] = len(dims)
    g["dims"] = 1
    g["dims"][0, : len(dims)] = dims
    n = int(np.prod(dims)) if dims else 1
    g["ncols"] = n
    t = sp.make_tasks(g)
    L = dims[-1] if dims else 1
    cols = np.concatenate([np.arange(s, s + c) for s, c in zip(t["start"], t["count"], strict=True)])
    assert np.array_equal(np.sort(cols), np.arange(n))
    for s, c in zip(t["start"].astype(np.int64), t["count"].astype(np.int64), strict=True):
        assert c >= 1
        assert (s + c - 1) // L - s // L + 1 <= sp.TASK_ROWS
        assert c <= max(sp.TASK_COLUMNS, L * sp.TASK_ROWS)
