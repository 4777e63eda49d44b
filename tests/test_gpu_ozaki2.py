"""tcgen05 Ozaki II (CRT) GEMM: bit-exact against the numpy restatement of the
same arithmetic (tests/ozaki2_reference.py), and within its error bound of the
exact product."""

import math

import numpy as np
import pytest

from tests import ozaki2_reference as ref
from tests.test_gpu_ozaki import run_grouped

pytestmark = pytest.mark.gpu


def problems(rng, shapes, spread=3.0):
    out = []
    for i, (m, n, k) in enumerate(shapes):
        A = rng.standard_normal((m, k)) * np.exp(rng.normal(0, spread, size=(m, 1)))
        B = rng.standard_normal((k, n)) * np.exp(rng.normal(0, spread, size=(1, n)))
        out.append((A, B, bool(i % 2), bool(i % 3 == 1)))
    return out


SHAPES = [(1, 1, 1), (5, 7, 3), (256, 256, 128), (130, 260, 129), (300, 40, 517),
          (64, 600, 250), (257, 513, 64), (33, 17, 3000), (512, 300, 1024)]


@pytest.mark.parametrize("n", [8, 11, 13, 14])
def test_ozaki2_bit_exact_vs_reference(n):
    rng = np.random.default_rng(100 + n)
    probs = problems(rng, SHAPES)
    got = run_grouped(probs, f"ozaki2_{n}")
    for (A, B, _, _), C in zip(probs, got, strict=True):
        want = ref.emulate(A, B, n)
        assert np.array_equal(C, want), (A.shape, B.shape, np.abs(C - want).max())


def test_ozaki2_zero_rows_columns_and_long_k():
    """All-zero rows and columns (exponent 0, zero residues), a K long enough
    to lower the operand bits, and a single column."""
    rng = np.random.default_rng(7)
    A = rng.standard_normal((300, 20000))
    A[5] = 0.0
    B = rng.standard_normal((20000, 260))
    B[:, 17] = 0.0
    A2 = rng.standard_normal((260, 700))
    B2 = rng.standard_normal((700, 1))
    probs = [(A, B, False, False), (A2, B2, True, False)]
    got = run_grouped(probs, "ozaki2_14")
    for (a, b, _, _), C in zip(probs, got, strict=True):
        assert np.array_equal(C, ref.emulate(a, b, 14))
    assert not got[0][5].any() and not got[0][:, 17].any()


@pytest.mark.parametrize("n", [12, 14])
def test_ozaki2_accuracy_vs_exact(n):
    rng = np.random.default_rng(200 + n)
    probs = problems(rng, SHAPES[2:])
    got = run_grouped(probs, f"ozaki2_{n}")
    for (A, B, _, _), C in zip(probs, got, strict=True):
        # sampled entries against a correctly summed FP64 product: only the
        # rounding of A and B to a and b bits remains (plus the final rounding)
        bound = ref.rounding_error_bound(A, B, n)
        for f in rng.integers(0, C.size, size=64):
            i, j = divmod(int(f), C.shape[1])
            terms = A[i] * B[:, j]
            exact = math.fsum(terms)
            tol = bound[i, j] + 2.3e-16 * (np.abs(terms).sum() + abs(exact))
            assert abs(C[i, j] - exact) <= tol, (i, j, C[i, j], exact, tol)
