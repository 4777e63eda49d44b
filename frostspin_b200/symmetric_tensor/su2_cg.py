"""SU(2) Clebsch-Gordan coefficients, computed on demand.

Irreps are labelled by their dimension d = 2 s + 1 and the basis of an irrep is
ordered by decreasing S_z (index i <-> m = s - i), the layout of the reference's
CG tables (frostspin/groups/su2_clebsch_gordan.py:8-32):
p[i1, i2, i3] = <s1 m1; s2 m2 | s3 m3> (Condon-Shortley phases).

cg_tensor evaluates every coefficient with sympy's exact CG routine and casts it
to float64, the same published routine and conversion the reference used to
write its table, so the values are identical to the reference's (a correctly
rounded evaluation differs from them by one ulp on about a third of the tensors).
Tensors with every dimension <= 18 come from su2_cg_table.npz, the same sympy
values written once by make_su2_cg_table.py, which saves the sympy import and
evaluation (seconds) on first use; larger ones are evaluated on demand.
cg_coefficient is an independent evaluation by Racah's closed formula
(G. Racah, Phys. Rev. 62, 438 (1942)) in exact rational arithmetic, used to
cross-check.  There is no size limit: tensors are generated when first needed
and cached.
"""

import decimal
import os
from fractions import Fraction
from functools import lru_cache
from math import factorial

import numpy as np

_CTX = decimal.Context(prec=60)

TABLE_FILE = "su2_cg_table.npz"
_PACKED = {}

# coefficients loaded from a table file, (d1, d2, d3) -> (flat indices, values);
# tensors missing from it are computed
_TABLE = {}


def _sqrt_fraction(x):
    """Correctly rounded float64 square root of a non-negative Fraction."""
    if x == 0:
        return 0.0
    q = _CTX.divide(decimal.Decimal(x.numerator), decimal.Decimal(x.denominator))
    return float(_CTX.sqrt(q))


def cg_coefficient(d1, i1, d2, i2, d3, i3):
    """<s1 m1; s2 m2 | s3 m3> with d = 2s + 1 and m = s - i, as a float."""
    # doubled quantities, so that half-integer spins are integers
    j1, j2, j3 = d1 - 1, d2 - 1, d3 - 1
    m1, m2, m3 = j1 - 2 * i1, j2 - 2 * i2, j3 - 2 * i3
    if m1 + m2 != m3:
        return 0.0
    if not (abs(j1 - j2) <= j3 <= j1 + j2) or (j1 + j2 + j3) % 2:
        return 0.0
    f = factorial
    a = (j1 + j2 - j3) // 2
    b = (j1 - j2 + j3) // 2
    c = (-j1 + j2 + j3) // 2
    tri = Fraction((j3 + 1) * f(a) * f(b) * f(c), f((j1 + j2 + j3) // 2 + 1))
    fac = Fraction(
        f((j3 + m3) // 2) * f((j3 - m3) // 2) * f((j1 - m1) // 2) * f((j1 + m1) // 2)
        * f((j2 - m2) // 2) * f((j2 + m2) // 2)
    )
    s = Fraction(0)
    kmin = max(0, (j2 - j3 - m1) // 2, (j1 - j3 + m2) // 2)
    kmax = min(a, (j1 - m1) // 2, (j2 + m2) // 2)
    for k in range(kmin, kmax + 1):
        den = (f(k) * f(a - k) * f((j1 - m1) // 2 - k) * f((j2 + m2) // 2 - k)
               * f((j3 - j2 + m1) // 2 + k) * f((j3 - j1 - m2) // 2 + k))
        s += Fraction((-1) ** k, den)
    if s == 0:
        return 0.0
    sq = _sqrt_fraction(tri * fac * s * s)
    return sq if s > 0 else -sq


def nonzero_entries(d1, d2, d3):
    """(i1, i2, i3) index arrays of the structurally allowed entries (m1 + m2 =
    m3), in C order of (i1, i2)."""
    j1, j2, j3 = d1 - 1, d2 - 1, d3 - 1
    i1, i2 = np.meshgrid(np.arange(d1), np.arange(d2), indexing="ij")
    m3 = (j1 - 2 * i1) + (j2 - 2 * i2)
    ok = (np.abs(m3) <= j3) & ((j3 - m3) % 2 == 0)
    return i1[ok], i2[ok], (j3 - m3[ok]) // 2


def _nonzero_entries(d1, d2, d3):
    yield from zip(*(x.tolist() for x in nonzero_entries(d1, d2, d3)), strict=True)


def _packed_table():
    """Packaged coefficients: (d1, d2, d3) -> values in nonzero_entries order."""
    if not _PACKED:
        path = os.path.join(os.path.dirname(os.path.abspath(__file__)), TABLE_FILE)
        index = {}
        if os.path.exists(path):
            with np.load(path) as f:
                values = f["values"]
                offsets = f["offsets"]
                for k, t in enumerate(f["triples"].tolist()):
                    index[tuple(t)] = (int(offsets[k]), int(offsets[k + 1]))
            _PACKED["values"] = values
        _PACKED["index"] = index
    return _PACKED


def set_table(table):
    """Use the given sparse coefficients ((d1, d2, d3) -> (flat C-order indices,
    values)) instead of computing them."""
    _TABLE.clear()
    _TABLE.update(table)
    cg_tensor.cache_clear()


@lru_cache(maxsize=None)
def cg_tensor(d1, d2, d3):
    """Read-only array p[i1, i2, i3] of shape (d1, d2, d3)."""
    if (d1, d2, d3) in _TABLE:
        inds, vals = _TABLE[d1, d2, d3]
        p = np.zeros(d1 * d2 * d3)
        p[np.asarray(inds, dtype=np.int64)] = vals
        p = p.reshape(d1, d2, d3)
        p.setflags(write=False)
        return p
    packed = _packed_table()
    span = packed["index"].get((d1, d2, d3))
    if span is not None:
        p = np.zeros((d1, d2, d3))
        p[nonzero_entries(d1, d2, d3)] = packed["values"][span[0] : span[1]]
        p.setflags(write=False)
        return p
    return cg_tensor_sympy(d1, d2, d3)


def cg_tensor_sympy(d1, d2, d3):
    """p[i1, i2, i3] from sympy's exact CG routine, cast to float64."""
    import sympy as sp
    from sympy.physics.quantum.cg import CG

    p = np.zeros((d1, d2, d3))
    s1, s2, s3 = (sp.Rational(d - 1, 2) for d in (d1, d2, d3))
    for i1, i2, i3 in _nonzero_entries(d1, d2, d3):
        p[i1, i2, i3] = float(CG(s1, s1 - i1, s2, s2 - i2, s3, s3 - i3).doit())
    p.setflags(write=False)
    return p


def cg_tensor_racah(d1, d2, d3):
    """Same tensor from Racah's formula, correctly rounded (cross-check)."""
    p = np.zeros((d1, d2, d3))
    for i1, i2, i3 in _nonzero_entries(d1, d2, d3):
        p[i1, i2, i3] = cg_coefficient(d1, i1, d2, i2, d3, i3)
    return p
