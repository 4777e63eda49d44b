"""Double-layer SequentialCTMRG on the device against the reference's own run
(fixture: the random U(1) AB/BA network of the reference's tests/test_ctmrg.py).

Before any truncation the reduced density matrices are deterministic products
and must agree to 1e-12.  After iterations only gauge-invariant quantities are
compared (rdms, PEPS norm), since singular vectors are defined up to sign, as
in the reference's tests/test_symmetrized_ctm.py:65-66; both sides take the
dense SVD path at this chi, so they agree to 1e-9."""

import numpy as np
import pytest

from tests.helpers import load

pytestmark = pytest.mark.gpu


def test_sequential_ctmrg_matches_reference():
    from frostspin_b200 import U1SymmetricTensor
    from frostspin_b200.ctmrg import SequentialCTMRG

    d = load("ctmrg_u1_random")
    A = U1SymmetricTensor.load_from_dic(d, prefix="A")
    B = U1SymmetricTensor.load_from_dic(d, prefix="B")
    ctm = SequentialCTMRG.from_elementary_tensors("AB\nBA", (A, B), 20)
    for it in range(4):
        if it:
            ctm.iterate()
        tol = 1e-12 if it == 0 else 1e-9
        for x, y in ctm.site_coords:
            for kind, fn in (("rdm1x2", ctm.compute_rdm1x2), ("rdm2x1", ctm.compute_rdm2x1)):
                got = fn(x, y).toarray()
                ref = d[f"it{it}_{kind}_{x}{y}"]
                assert np.abs(got - ref).max() < tol * max(1.0, np.abs(ref).max()), (it, kind)
        assert ctm.chi_values == list(d[f"it{it}_chi"])
        logz = ctm.compute_PEPS_norm_log()
        assert abs(logz - float(d[f"it{it}_logZ"])) < tol * 10
