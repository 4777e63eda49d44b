"""The allocation-free grouped Ozaki GEMM (fs_ozaki_gemm_noalloc).

Some callers of this library cannot allocate device memory -- a host
application whose own pool already reserved the GPU, or a C / Fortran driver
with no device allocator -- so this entry point keeps its digit slices and
launch tables in a fixed device array inside the library.  These tests call it
through the C ABI with a host array of problem descriptors and check that two
calls in a row reproduce the workspace-based entry points (fs_ozaki_split +
fs_ozaki_gemm) exactly, and that oversized requests are refused before any GPU
work.  This file is collected last so that a failure here never hides another
test's result.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SLICES = 6


def make_problems(rng):
    shapes = [(130, 260, 129), (7, 300, 517), (256, 256, 256), (1, 1, 1), (64, 40, 1000)]
    return [
        (rng.standard_normal((m, k)), rng.standard_normal((k, n)), bool(i % 2), bool(i % 3 == 1))
        for i, (m, n, k) in enumerate(shapes)
    ]


def device_operands(problems):
    import torch

    dev = []
    for A, B, ta, tb in problems:
        dA = torch.from_numpy(np.ascontiguousarray(A.T if ta else A)).cuda()
        dB = torch.from_numpy(np.ascontiguousarray(B.T if tb else B)).cuda()
        dev.append((dA, dB))
    return dev


def problem_table(problems, dev, outs):
    from frostspin_b200 import _native

    arr = np.zeros(len(problems), dtype=_native.GEMM_PROBLEM_DTYPE)
    for i, ((A, B, ta, tb), (dA, dB), C) in enumerate(zip(problems, dev, outs, strict=True)):
        M, K = A.shape
        N = B.shape[1]
        arr[i] = (dA.data_ptr(), dB.data_ptr(), C.data_ptr(), M if ta else K, K if tb else N, N,
                  M, N, K, int(ta), int(tb), 0, 1.0, 0.0)
    return arr


def run_noalloc(problems, dev):
    import torch

    from frostspin_b200 import _native

    outs = [torch.full((A.shape[0], B.shape[1]), np.nan, dtype=torch.float64, device="cuda")
            for A, B, _, _ in problems]
    arr = problem_table(problems, dev, outs)
    stream = torch.cuda.current_stream().cuda_stream
    st = _native.lib().fs_ozaki_gemm_noalloc(arr.ctypes.data, arr.size, SLICES, stream)
    assert st == 0, _native.lib().fs_status_string(st)
    assert noalloc_status(stream) == 0
    torch.cuda.synchronize()
    return [c.cpu().numpy() for c in outs]


def noalloc_status(stream):
    import ctypes

    from frostspin_b200 import _native

    status = ctypes.c_int32(99)
    assert _native.lib().fs_ozaki_noalloc_status(stream, ctypes.byref(status)) == 0
    return status.value


def run_workspace(problems, dev):
    import torch

    from frostspin_b200 import linalg

    outs = [torch.full((A.shape[0], B.shape[1]), np.nan, dtype=torch.float64, device="cuda")
            for A, B, _, _ in problems]
    arr = problem_table(problems, dev, outs)
    linalg.ozaki_gemm(arr, SLICES)
    torch.cuda.synchronize()
    linalg.check_ozaki_flags()
    return [c.cpu().numpy() for c in outs]


def test_noalloc_matches_workspace_entry_points_twice():
    rng = np.random.default_rng(123)
    for _ in range(2):  # second call reuses the same scratch with new data
        problems = make_problems(rng)
        dev = device_operands(problems)
        got = run_noalloc(problems, dev)
        ref = run_workspace(problems, dev)
        for (A, B, _, _), g, r in zip(problems, got, ref, strict=True):
            assert not np.isnan(g).any()
            assert np.array_equal(g, r)
            # and the product itself is FP64-class
            err = np.abs(g - A @ B).max() / (np.abs(A).max() * np.abs(B).max() * A.shape[1])
            assert err < 2.0 * SLICES * 2.0 ** (-7 * SLICES)


def test_noalloc_rejects_requests_beyond_its_scratch():
    import torch

    from frostspin_b200 import _native

    buf = torch.zeros(16, dtype=torch.float64, device="cuda")
    arr = np.zeros(1, dtype=_native.GEMM_PROBLEM_DTYPE)
    # 4096^3 with 8 slices needs 8 * 32 * 32 * 16 KiB per operand, far above 48 MiB;
    # the request is refused on the host before any GPU work touches the buffers
    arr[0] = (buf.data_ptr(), buf.data_ptr(), buf.data_ptr(), 4096, 4096, 4096,
              4096, 4096, 4096, 0, 0, 0, 1.0, 0.0)
    st = _native.lib().fs_ozaki_gemm_noalloc(arr.ctypes.data, 1, 8, None)
    assert st == -7  # FS_ERR_TOO_LARGE
    assert _native.lib().fs_ozaki_gemm_noalloc(arr.ctypes.data, 1, 0, None) == -1


def test_noalloc_reports_a_wait_that_ran_out():
    """With the wait bound cut to one cycle the kernel's first wait runs out:
    the kernel drains its copies and returns early, and the status query (not
    the call's return value, which only covers the launch) reports
    FS_ERR_TIMEOUT.  With the default bound restored the next call is exact."""
    import torch

    from frostspin_b200 import _native

    rng = np.random.default_rng(7)
    problems = make_problems(rng)[:3]
    dev = device_operands(problems)
    outs = [torch.zeros((A.shape[0], B.shape[1]), dtype=torch.float64, device="cuda")
            for A, B, _, _ in problems]
    arr = problem_table(problems, dev, outs)
    stream = torch.cuda.current_stream().cuda_stream
    lib = _native.lib()
    old = lib.fs_set_spin_limit(1)
    try:
        assert lib.fs_ozaki_gemm_noalloc(arr.ctypes.data, arr.size, SLICES, stream) == 0
        assert noalloc_status(stream) == -4  # FS_ERR_TIMEOUT
    finally:
        lib.fs_set_spin_limit(old)
    got = run_noalloc(problems, dev)
    ref = run_workspace(problems, dev)
    for g, r in zip(got, ref, strict=True):
        assert np.array_equal(g, r)


def test_noalloc_refuses_stream_capture():
    """The staged host tables do not outlive a call, so a call on a stream that
    is being captured is refused before anything is enqueued."""
    import torch

    from frostspin_b200 import _native

    rng = np.random.default_rng(8)
    problems = make_problems(rng)[:1]
    dev = device_operands(problems)
    outs = [torch.zeros((A.shape[0], B.shape[1]), dtype=torch.float64, device="cuda")
            for A, B, _, _ in problems]
    arr = problem_table(problems, dev, outs)
    g = torch.cuda.CUDAGraph()
    s = torch.cuda.Stream()
    torch.cuda.synchronize()
    with torch.cuda.stream(s):
        g.capture_begin()
        try:
            st = _native.lib().fs_ozaki_gemm_noalloc(arr.ctypes.data, arr.size, SLICES,
                                                     s.cuda_stream)
            outs[0].add_(0.0)  # keep the captured graph non-empty
        finally:
            g.capture_end()
    assert st == -5  # FS_ERR_UNSUPPORTED
