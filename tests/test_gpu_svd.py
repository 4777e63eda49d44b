"""Truncated SVD of the CTMRG projectors (svd_tools.truncated_svd_block and the
lock-step form truncated_svd_blocks) against cuSOLVER's dense SVD, on blocks
with the fast-decaying spectra of CTMRG corner products (the reference runs
ARPACK there, svd_tools.py:154-197, to the same values)."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _block(rng, nr, nc, decay):
    import torch

    r = min(nr, nc)
    u, _ = np.linalg.qr(rng.standard_normal((nr, r)))
    v, _ = np.linalg.qr(rng.standard_normal((nc, r)))
    s = np.exp(-decay * np.arange(r))
    return torch.from_numpy((u * s) @ v.T).cuda(), s


def test_randomized_blocks_match_dense_svd():
    from frostspin_b200.misc_tools.svd_tools import truncated_svd_block, truncated_svd_blocks

    rng = np.random.default_rng(4)
    specs = [(900, 700, 0.35, 30), (400, 1200, 0.2, 20), (60, 50, 0.3, 12), (1500, 1500, 0.15, 60),
             (300, 300, 0.5, 200)]
    blocks, ks, fulls, svals = [], [], [], []
    for nr, nc, decay, k in specs:
        m, s = _block(rng, nr, nc, decay)
        blocks.append(m)
        ks.append(k)
        fulls.append(min(nr, nc) < 100)
        svals.append(s)
    us, ss, vs = truncated_svd_blocks(blocks, ks, fulls)
    for i, m in enumerate(blocks):
        k = ks[i]
        s_ref = svals[i][: ss[i].numel()]
        got = ss[i].cpu().numpy()
        # leading values to near machine precision relative to the largest
        assert np.abs(got[:k] - s_ref[:k]).max() < 1e-12 * s_ref[0], i
        # U s Vh reproduces the rank-k part of the block
        approx = (us[i][:, :k] * ss[i][:k]) @ vs[i][:k]
        assert float((approx - m).abs().max()) < 2.0 * s_ref[min(k, s_ref.size - 1)] + 1e-12, i
        # the lock-step form equals the per-block form
        u1, s1, v1 = truncated_svd_block(m, k, full=fulls[i])
        assert np.abs(s1.cpu().numpy()[:k] - got[:k]).max() < 1e-13 * s_ref[0], i
