"""tcgen05 Ozaki GEMM: bit-exact against a numpy emulation of the same digit
split and the same FP64 recombination order, and within its error bound of the
plain FP64 GEMM (relative to max|A| max|B| K)."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def emulate(A, B, S, alpha=1.0):
    """Ozaki-scheme product with the kernel's arithmetic (beta = 0)."""
    def split(X):
        m = np.abs(X).max(axis=1) if X.shape[1] else np.zeros(X.shape[0])
        e = np.frexp(m)[1].astype(np.int64)
        e[m == 0] = 0
        x = np.ldexp(X, -e[:, None])
        digits = []
        for _ in range(S):
            t = x * 128.0
            d = np.trunc(t)
            x = t - d
            digits.append(d.astype(np.int64))
        return e, digits

    ea, As = split(A)
    eb, Bs = split(B.T)
    C = None
    for d in range(S - 1, -1, -1):
        P = sum(As[s] @ Bs[d - s].T for s in range(d + 1))
        val = alpha * np.ldexp(P.astype(np.float64), ea[:, None] + eb[None, :] - 7 * (d + 2))
        C = val if C is None else C + val
    return C


def run_grouped(problems, mode):
    import torch

    from frostspin_b200 import linalg

    outs = []
    specs = []
    for A, B, ta, tb in problems:
        dA = torch.from_numpy(np.ascontiguousarray(A.T if ta else A)).cuda()
        dB = torch.from_numpy(np.ascontiguousarray(B.T if tb else B)).cuda()
        C = torch.full((A.shape[0], B.shape[1]), np.nan, dtype=torch.float64, device="cuda")
        outs.append(C)
        specs.append({"A": dA.reshape(-1), "a_off": 0, "a_trans": ta,
                      "B": dB.reshape(-1), "b_off": 0, "b_trans": tb,
                      "C": C.reshape(-1), "c_off": 0,
                      "M": A.shape[0], "N": B.shape[1], "K": A.shape[1],
                      "_keep": (dA, dB)})
    with linalg.gemm_precision_mode(mode), linalg.ozaki_dispatch_mode("all"):
        linalg.grouped_gemm(specs)
    torch.cuda.synchronize()
    linalg.check_ozaki_flags()
    return [c.cpu().numpy() for c in outs]


def random_problems(rng):
    shapes = [(1, 1, 1), (5, 7, 3), (128, 256, 128), (130, 260, 129), (300, 40, 517),
              (64, 600, 250), (257, 513, 64), (33, 17, 1000)]
    probs = []
    for i, (m, n, k) in enumerate(shapes):
        A = rng.standard_normal((m, k)) * np.exp(rng.normal(0, 3, size=(m, 1)))
        B = rng.standard_normal((k, n)) * np.exp(rng.normal(0, 3, size=(1, n)))
        probs.append((A, B, bool(i % 2), bool(i % 3 == 1)))
    return probs


@pytest.mark.parametrize("S", [3, 5, 7])
def test_ozaki_bit_exact_vs_emulation(S):
    rng = np.random.default_rng(S)
    probs = random_problems(rng)
    got = run_grouped(probs, f"ozaki{S}")
    for (A, B, _, _), C in zip(probs, got, strict=True):
        ref = emulate(A, B, S)
        assert np.array_equal(C, ref), np.abs(C - ref).max()


@pytest.mark.parametrize("S", [4, 6, 7])
def test_ozaki_accuracy_vs_fp64(S):
    rng = np.random.default_rng(10 + S)
    probs = random_problems(rng)
    got = run_grouped(probs, f"ozaki{S}")
    ref = run_grouped(probs, "fp64")
    for (A, B, _, _), C, R in zip(probs, got, ref, strict=True):
        scale = (np.abs(A).max(axis=1)[:, None] * np.abs(B).max(axis=0)[None, :]) * A.shape[1]
        err = np.abs(C - R) / scale
        # dropped digits beyond S of each operand and dropped diagonals d >= S
        assert err.max() < 2.0 * S * 2.0 ** (-7 * S), (S, err.max())


@pytest.mark.parametrize("S", [4, 7])
def test_ozaki_pair_kernel_bit_exact(S):
    """Problems above 128 rows run on CTA pairs (tcgen05 cta_group::2); the
    result is bit-identical to the single-CTA kernel and to the emulation,
    including odd row-tile counts (padded) and ragged edges."""
    from frostspin_b200 import _native, linalg

    rng = np.random.default_rng(50 + S)
    shapes = [(129, 300, 200), (384, 256, 128), (600, 700, 300), (257, 5, 1000), (1024, 512, 640)]
    probs = []
    for i, (m, n, k) in enumerate(shapes):
        A = rng.standard_normal((m, k)) * np.exp(rng.normal(0, 2, size=(m, 1)))
        B = rng.standard_normal((k, n))
        probs.append((A, B, bool(i % 2), bool(i % 3 == 1)))
    before = _native.CALL_COUNTS.get("fs_ozaki_gemm_pair", 0)
    with linalg.ozaki_pair_mode(True):
        pair = run_grouped(probs, f"ozaki{S}")
    assert _native.CALL_COUNTS.get("fs_ozaki_gemm_pair", 0) > before
    with linalg.ozaki_pair_mode(False):
        single = run_grouped(probs, f"ozaki{S}")
    for (A, B, _, _), cp, cs in zip(probs, pair, single, strict=True):
        assert np.array_equal(cp, cs)
        assert np.array_equal(cp, emulate(A, B, S))
