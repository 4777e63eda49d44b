"""FP64 grouped GEMM kernels (DMMA tiles and the thin bandwidth kernel) against
a numpy float64 reference: every transpose combination, ragged edges, K = 0,
beta != 0 and thin recoupling shapes, all problems of a table in one launch."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SHAPES = [  # (M, N, K)
    (1, 1, 1), (7, 5, 3), (64, 64, 16), (65, 63, 17), (130, 257, 129), (3, 1000, 2),
    (32, 4097, 32), (4, 20000, 4), (33, 300, 31), (200, 3, 500), (16, 16, 0), (1, 517, 29),
]


def run_table(problems, trans_a, trans_b, beta):
    import torch

    from frostspin_b200 import _native, linalg

    rng = np.random.default_rng(17)
    arr = np.zeros(len(problems), dtype=_native.GEMM_PROBLEM_DTYPE)
    keep, refs, outs = [], [], []
    for i, (M, N, K) in enumerate(problems):
        A = rng.standard_normal((M, K))
        B = rng.standard_normal((K, N))
        C0 = rng.standard_normal((M, N))
        dA = torch.from_numpy(np.ascontiguousarray(A.T if trans_a else A)).cuda()
        dB = torch.from_numpy(np.ascontiguousarray(B.T if trans_b else B)).cuda()
        dC = torch.from_numpy(C0.copy()).cuda()
        keep += [dA, dB]
        outs.append(dC)
        refs.append((A @ B * 1.5 + beta * C0,
                     np.abs(A).sum(axis=1)[:, None] * np.abs(B).max(initial=0.0)))
        arr[i] = (dA.data_ptr(), dB.data_ptr(), dC.data_ptr(), M if trans_a else K,
                  K if trans_b else N, N, M, N, K, int(trans_a), int(trans_b), 0, 1.5, beta)
    linalg.grouped_dgemm_table(arr)
    torch.cuda.synchronize()
    for (ref, scale), dC in zip(refs, outs, strict=True):
        got = dC.cpu().numpy()
        assert np.all(np.abs(got - ref) <= 1e-14 * (scale + 1.0) * 4 + 1e-15)


@pytest.mark.parametrize("trans_a", [False, True])
@pytest.mark.parametrize("trans_b", [False, True])
def test_grouped_dgemm_all_layouts(trans_a, trans_b):
    run_table(SHAPES, trans_a, trans_b, 0.0)


def test_grouped_dgemm_beta_accumulates():
    run_table(SHAPES, False, False, 0.75)
    run_table(SHAPES[:6], True, False, -2.0)


def _delta(before, name):
    from frostspin_b200 import _native

    return _native.CALL_COUNTS.get(name, 0) - before.get(name, 0)


def test_thin_and_tile_kernels_both_launch():
    from frostspin_b200 import _native

    before = dict(_native.CALL_COUNTS)
    run_table([(4, 5000, 4), (100, 100, 100)], False, False, 0.0)
    assert _delta(before, "fs_grouped_dgemm_thin") == 1
    # one transpose combination in the table: the streaming DMMA kernel
    assert _delta(before, "fs_grouped_dgemm_uniform") == 1
    assert _delta(before, "fs_grouped_dgemm") == 0


SHORT_K = [  # (M, N, K): wide short-K sectors, ragged in every dimension
    (64, 64, 16), (65, 63, 17), (130, 257, 129), (33, 300, 31), (263, 5000, 82),
    (98, 3000, 19), (217, 4100, 58), (40, 70, 0), (7, 9, 3), (200, 3, 256),
]


@pytest.mark.parametrize("trans_a", [False, True])
@pytest.mark.parametrize("trans_b", [False, True])
def test_streaming_kernel_short_k(trans_a, trans_b):
    """Launches with one transpose combination and K <= 256 run the streaming
    kernel (cp.async ring across tiles, padded fragments skipped)."""
    from frostspin_b200 import _native

    before = dict(_native.CALL_COUNTS)
    run_table(SHORT_K, trans_a, trans_b, 0.0)
    run_table(SHORT_K, trans_a, trans_b, -0.5)
    assert _delta(before, "fs_grouped_dgemm_uniform") == 2
    assert _delta(before, "fs_grouped_dgemm") == 0


def test_long_k_uses_per_tile_kernel():
    from frostspin_b200 import _native

    before = dict(_native.CALL_COUNTS)
    run_table([(100, 100, 300), (64, 64, 64)], False, False, 0.0)
    assert _delta(before, "fs_grouped_dgemm") == 1
    assert _delta(before, "fs_grouped_dgemm_uniform") == 0


def test_mixed_transposes_in_one_launch():
    """Problems with different transpose flags share one launch of the
    per-tile kernel (the streaming kernel needs uniform flags)."""
    import torch

    from frostspin_b200 import _native, linalg

    rng = np.random.default_rng(5)
    shapes = [(65, 63, 17), (130, 257, 129), (200, 3, 500), (16, 16, 0), (64, 64, 64)]
    arr = np.zeros(len(shapes), dtype=_native.GEMM_PROBLEM_DTYPE)
    keep, refs, outs = [], [], []
    for i, (M, N, K) in enumerate(shapes):
        ta, tb = i % 2 == 1, i % 3 == 1
        A = rng.standard_normal((M, K))
        B = rng.standard_normal((K, N))
        dA = torch.from_numpy(np.ascontiguousarray(A.T if ta else A)).cuda()
        dB = torch.from_numpy(np.ascontiguousarray(B.T if tb else B)).cuda()
        dC = torch.zeros(M, N, dtype=torch.float64, device="cuda")
        keep += [dA, dB]
        outs.append(dC)
        refs.append((A @ B, np.abs(A).sum(axis=1)[:, None] * np.abs(B).max(initial=0.0)))
        arr[i] = (dA.data_ptr(), dB.data_ptr(), dC.data_ptr(), M if ta else K, K if tb else N,
                  N, M, N, K, int(ta), int(tb), 0, 1.0, 0.0)
    before = dict(_native.CALL_COUNTS)
    linalg.grouped_dgemm_table(arr)
    torch.cuda.synchronize()
    assert _delta(before, "fs_grouped_dgemm") == 1
    assert _delta(before, "fs_grouped_dgemm_uniform") == 0
    for (ref, scale), dC in zip(refs, outs, strict=True):
        got = dC.cpu().numpy()
        assert np.all(np.abs(got - ref) <= 1e-14 * (scale + 1.0) * 4 + 1e-15)


@pytest.mark.parametrize("trans_a", [False, True])
@pytest.mark.parametrize("trans_b", [False, True])
def test_split_k_for_launches_with_few_tiles(trans_a, trans_b):
    """Few output tiles with long K: the host cuts K into chunks, partial
    products go to a workspace and are summed in order (deterministic); the
    result matches float64 numpy and is reproducible bit for bit."""
    import torch

    from frostspin_b200 import _native

    shapes = [(40, 50, 20000), (5, 300, 9000), (64, 64, 4096), (3, 2, 2048)]
    before = _native.CALL_COUNTS.get("fs_splitk_reduce", 0)
    run_table(shapes, trans_a, trans_b, 0.0)
    run_table(shapes, trans_a, trans_b, 0.5)
    assert _native.CALL_COUNTS.get("fs_splitk_reduce", 0) >= before + 2

    from frostspin_b200 import linalg

    rng = np.random.default_rng(3)
    M, N, K = 40, 70, 12000
    A = torch.from_numpy(rng.standard_normal((M, K))).cuda()
    B = torch.from_numpy(rng.standard_normal((K, N))).cuda()
    outs = []
    for _ in range(2):
        C = torch.empty(M, N, dtype=torch.float64, device="cuda")
        arr = np.zeros(1, dtype=_native.GEMM_PROBLEM_DTYPE)
        arr[0] = (A.data_ptr(), B.data_ptr(), C.data_ptr(), K, N, N, M, N, K, 0, 0, 0, 1.0, 0.0)
        linalg.grouped_dgemm_table(arr)
        torch.cuda.synchronize()
        outs.append(C.cpu().numpy())
    assert np.array_equal(outs[0], outs[1])


def test_device_tile_table_matches_host_enumeration():
    """fs_expand_tiles writes the tile list: every problem's tiles row-major,
    or column-major for wide problems, problems in the given order, empty
    problems skipped."""
    import torch

    from frostspin_b200 import _native, linalg

    ncol = np.array([3, 4, 1, 2, 2, 5, 1], dtype=np.int64)
    nrow = np.array([2, 0, 1, 6, 0, 1, 0], dtype=np.int64)
    ntile = ncol * nrow
    order = np.array([3, 1, 0, 6, 2, 5, 4])
    runs, total = linalg._tile_runs(ntile, ncol, order, nrow)
    d_tiles = linalg._device_tiles(runs, total)
    torch.cuda.synchronize()
    got = d_tiles.cpu().numpy()[: total * _native.GEMM_TILE_DTYPE.itemsize].view(
        _native.GEMM_TILE_DTYPE)
    # wide problems (more tile columns than rows) column-major, the rest row-major
    want = [(p, k % nrow[p], k // nrow[p]) if ncol[p] > nrow[p] else (p, k // ncol[p], k % ncol[p])
            for p in order for k in range(ntile[p])]
    assert total == len(want)
    assert [tuple(int(x) for x in (t["problem"], t["tm"], t["tn"])) for t in got] == want
