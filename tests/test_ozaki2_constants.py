"""The library's Ozaki II constants (CRT weights on the two binary grids, the
moduli, operand bits) against an exact computation with Python integers, and
the exactness conditions the kernels rely on.  No GPU needed."""

import math

import numpy as np
import pytest

from frostspin_b200 import _native, linalg
from tests import ozaki2_reference as ref

NS = range(_native.FS_OZAKI2_MIN_MODULI, _native.FS_OZAKI2_MAX_MODULI + 1)


@pytest.mark.parametrize("n", NS)
def test_constants_match_exact_integers(n):
    got = _native.ozaki2_constants(n)
    c = ref.crt_constants(n)
    assert list(got["moduli"]) == list(ref.MODULI[:n])
    assert np.array_equal(got["w1"], c["w1"])
    assert np.array_equal(got["w2"], c["w2"])
    assert got["P"][0] == c["P1"] and got["P"][1] == c["P2"]
    assert np.array_equal(got["frac"], c["frac"])
    assert list(got["grids"]) == [c["e1"], c["e2"]]


@pytest.mark.parametrize("n", NS)
def test_exact_evaluation_bounds(n):
    """Every product r W and partial sum of the two grid levels stays on its
    grid below 2^53 ulps, and the dropped level is far below the rounding of
    the operands."""
    c = ref.crt_constants(n)
    P = c["P"]
    assert np.all(np.abs(c["w1"]) / 2.0 ** c["e1"] < 2.0 ** 45)
    assert 256 * n * P < 2 ** (53 + c["e1"])
    assert 256 * n * 2 ** c["e1"] <= 2 ** (53 + c["e2"])
    for K in (1, 100, 2048, _native.FS_OZAKI2_MAX_K):
        a, b = ref.operand_bits(n, K)
        assert K * 2 ** (a + b) <= P // 4
        assert 2 ** (c["e2"] + 12) < 2 ** (min(a, b) - 1) * K  # dropped part << rounding
        assert a <= 50 and b <= 50   # |A'| <= 2^50 keeps the one-FMA quotient exact


@pytest.mark.parametrize("n", [8, 12, 14])
def test_operand_bits_match_library(n):
    for K in (1, 2, 3, 127, 128, 129, 2048, 5000, 131071):
        assert _native.ozaki2_bits(n, K) == ref.operand_bits(n, K) == linalg.ozaki2_bits(n, K)


def test_pairwise_coprime():
    for i, p in enumerate(ref.MODULI):
        for q in ref.MODULI[:i]:
            assert math.gcd(p, q) == 1


def test_emulation_is_exact_crt():
    """The numpy emulation recovers the exact integer product of the scaled
    operands (checked against Python integers on a small case)."""
    rng = np.random.default_rng(3)
    A = rng.standard_normal((5, 37))
    B = rng.standard_normal((37, 4))
    n = 13
    Ai, Bi, ea, eb, a, b = ref.scaled_integers(A, B, n)
    C = ref.emulate(A, B, n)
    for i in range(5):
        for j in range(4):
            X = sum(int(x) * int(y) for x, y in zip(Ai[i], Bi[j], strict=True))
            want = float(X) * 2.0 ** (int(ea[i]) + int(eb[j]) - a - b)
            assert abs(C[i, j] - want) <= 2 ** -50 * abs(want)
    assert np.abs(C - A @ B).max() < 1e-12


def test_residue_shortcuts_are_exact():
    """The device shortcuts, restated in exact arithmetic: adding 1.5 * 2^52
    leaves A' mod 2^32 in the low word, and q = rint(A' * fl(1/p) + 1.5 * 2^52)
    (one FMA) is the nearest integer to A'/p for |A'| <= 2^50, so the low byte
    of A' - q p is the symmetric residue; likewise for int32 accumulators."""
    import struct
    from fractions import Fraction

    magic = 6755399441055744.0

    def lo32(x):
        v = struct.unpack("<q", struct.pack("<d", x))[0] & 0xFFFFFFFF
        return v - (1 << 32) if v >= 1 << 31 else v

    def fma(a, b, c):
        return float(Fraction(a) * Fraction(b) + Fraction(c))

    def byte(v):
        v &= 0xFF
        return v - 256 if v >= 128 else v

    rng = np.random.default_rng(11)
    vals = [int(v) for v in rng.integers(-(2**50), 2**50, size=300)]
    for p in ref.MODULI[1:]:
        for n0 in rng.integers(0, 2**40, size=20):
            for off in ((p - 1) // 2, (p + 1) // 2):
                vals += [int(p * n0 + off), -int(p * n0 + off)]
    vals += [2**50, -(2**50), 0, 1, -1]
    for v in vals:
        t = float(v) + magic
        lo, ad = lo32(t), t - magic
        assert ad == v
        assert byte(lo) == ref.sym_residue(np.int64(v), 256) or byte(lo) == -128
        for p in ref.MODULI[1:]:
            q = lo32(fma(ad, 1.0 / p, magic))
            assert byte(lo - q * p) == ref.sym_residue(np.int64(v), p)
    accs = [int(v) for v in rng.integers(-(2**31) + 1, 2**31 - 1, size=300)]
    for acc in accs:
        for p in ref.MODULI[1:]:
            q = lo32(fma(float(acc), 1.0 / p, magic))
            assert byte(acc - q * p) == ref.sym_residue(np.int64(acc), p)
