"""The bounded device waits of the tcgen05 kernels end in FS_ERR_TIMEOUT.

The reference has no device code; the failure-detection plan for this library
is that every spin on an mbarrier carries an iteration bound, after which the
kernel raises an error flag, drains the copies and MMAs it has in flight,
frees its tensor memory and returns, leaving the context usable.  Here the
bound is cut to one clock cycle (fs_set_spin_limit), so the first wait on a
copy that has not landed yet runs out; the host reads the flag and raises, and
the next GEMM with the default bound restored is exact.  Nothing here faults
or hangs the GPU: the drains keep their default bound."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _problem(M, N, K, seed):
    import torch

    rng = np.random.default_rng(seed)
    A = rng.standard_normal((M, K))
    B = rng.standard_normal((K, N))
    dA = torch.from_numpy(A).cuda().reshape(-1)
    dB = torch.from_numpy(B).cuda().reshape(-1)
    dC = torch.zeros(M * N, dtype=torch.float64, device="cuda")
    spec = [{"A": dA, "a_off": 0, "a_trans": False, "B": dB, "b_off": 0, "b_trans": False,
             "C": dC, "c_off": 0, "M": M, "N": N, "K": K}]
    return A, B, dC, spec


def test_single_cta_kernel_reports_timeout_and_recovers():
    import torch

    from frostspin_b200 import _native, linalg

    lib = _native.lib()
    A, B, dC, spec = _problem(100, 300, 700, 1)
    old = lib.fs_set_spin_limit(1)
    try:
        with (linalg.gemm_precision_mode("ozaki6"), linalg.ozaki_dispatch_mode("all"),
              linalg.ozaki_pair_mode(False)):
            linalg.grouped_gemm(spec)
        torch.cuda.synchronize()
        with pytest.raises(_native.NativeError, match="status -4"):
            linalg.check_ozaki_flags()
    finally:
        lib.fs_set_spin_limit(old)
    assert lib.fs_set_spin_limit(0) == old  # 0 restores the default
    with (linalg.gemm_precision_mode("ozaki6"), linalg.ozaki_dispatch_mode("all"),
          linalg.ozaki_pair_mode(False)):
        linalg.grouped_gemm(spec)
    torch.cuda.synchronize()
    linalg.check_ozaki_flags()
    C = dC.cpu().numpy().reshape(100, 300)
    err = np.abs(C - A @ B).max() / (np.abs(A).max() * np.abs(B).max() * 700)
    assert err < 2 * 6 * 2.0 ** (-42)
