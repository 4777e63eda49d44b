#!/usr/bin/env python
"""Write su2_cg_table.npz, the packaged SU(2) Clebsch-Gordan table.

Every coefficient <s1 m1; s2 m2 | s3 m3> with irrep dimensions d1, d2, d3 <=
DMAX is evaluated by sympy's exact CG routine and cast to float64, exactly as
su2_cg.cg_tensor does on demand; the file only saves that work (and the sympy
import) on first use.  Layout: ``triples`` (n, 3) sorted (d1, d2, d3),
``offsets`` (n + 1,) into ``values``, which holds each tensor's coefficients
in the structural order of su2_cg.nonzero_entries.

    python -m frostspin_b200.symmetric_tensor.make_su2_cg_table
"""

import os

import numpy as np

from . import su2_cg

DMAX = 18


def allowed_triples(dmax):
    for d1 in range(1, dmax + 1):
        for d2 in range(1, dmax + 1):
            for d3 in range(abs(d1 - d2) + 1, min(d1 + d2, dmax + 1), 2):
                yield d1, d2, d3


def main():
    triples, offsets, values = [], [0], []
    for d1, d2, d3 in allowed_triples(DMAX):
        p = su2_cg.cg_tensor_sympy(d1, d2, d3)
        i1, i2, i3 = su2_cg.nonzero_entries(d1, d2, d3)
        triples.append((d1, d2, d3))
        values.append(p[i1, i2, i3])
        offsets.append(offsets[-1] + i1.size)
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), su2_cg.TABLE_FILE)
    np.savez_compressed(path, dmax=np.array(DMAX), triples=np.array(triples, dtype=np.int16),
                        offsets=np.array(offsets, dtype=np.int64),
                        values=np.concatenate(values))
    print("wrote", path, os.path.getsize(path), "bytes,", len(triples), "tensors")


if __name__ == "__main__":
    main()
