"""The mixed-precision arithmetic end to end against the reference's own runs.

Every sector GEMM of the CTMRG and simple-update drivers runs on the tcgen05
int8 path (ozaki_dispatch_mode("all"), so even the small sectors of these test
sizes take it), at the precisions the benchmark uses.  The checks are the same
gauge-invariant quantities, with the same tolerances, as the plain FP64 parity
tests: truncation decisions (chi per iteration, bond representations) must be
bit-identical, reduced density matrices agree to 1e-9 and the energy per bond
to 1e-9 relative (the benchmark's stated energy tolerance for the mixed form).
"""

import numpy as np
import pytest

from tests.helpers import load

pytestmark = pytest.mark.gpu

SDS = np.array([[0.25, 0, 0, 0], [0, -0.25, 0.5, 0], [0, 0.5, -0.25, 0],
                [0, 0, 0, 0.25]]).reshape(2, 2, 2, 2)

# ozaki2_11 is the benchmark's default, the fewest moduli that pass both
# tests (10 moduli give a simple-update logZ 3e-11 from the reference's)
MIXED = ["ozaki7", "ozaki2_11", "ozaki2_12", "ozaki2_13", "ozaki2_14"]


@pytest.mark.parametrize("precision", MIXED)
def test_su2_ctmrg_d24_mixed_matches_reference(precision):
    """SequentialCTMRG (sequential_ctmrg.py:24-32) from the reference's D=24
    SU(2) simple-update tensors at beta = 2 (Dmax 28), chi = 24, 2 iterations,
    against the reference's run."""
    from frostspin_b200 import SU2SymmetricTensor, linalg
    from frostspin_b200.ctmrg import SequentialCTMRG

    d = load("su2_d24_beta2")
    ref = load("ctmrg_su2_d24")
    tensors = [SU2SymmetricTensor.load_from_dic(d, prefix=p) for p in ("A0", "A1")]
    with linalg.gemm_precision_mode(precision), linalg.ozaki_dispatch_mode("all"):
        ctm = SequentialCTMRG.from_elementary_tensors("AB\nBA", tensors, 24, cutoff=1e-10,
                                                      degen_ratio=0.9999)
        for it in range(2):
            ctm.iterate()
            assert np.array_equal(ctm.chi_values, ref[f"it{it}_chi"]), it
        es = []
        for x, y in ctm.site_coords:
            r12 = ctm.compute_rdm1x2(x, y).toarray()
            r21 = ctm.compute_rdm2x1(x, y).toarray()
            assert np.abs(r12 - ref[f"rdm1x2_{x}{y}"]).max() < 1e-9
            assert np.abs(r21 - ref[f"rdm2x1_{x}{y}"]).max() < 1e-9
            es += [np.einsum("ijkl,klij->", r12, SDS), np.einsum("ijkl,klij->", r21, SDS)]
    linalg.check_ozaki_flags()
    e_ref = float(ref["energy"])
    assert abs(np.mean(es) - e_ref) < 1e-9 * abs(e_ref)


@pytest.mark.parametrize("precision", MIXED)
def test_u1_simple_update_then_ctmrg_mixed_matches_reference(precision):
    """The U(1) chain (simple_update.py:599-790 then SequentialCTMRG): D = 6,
    tau = 0.01 to beta = 0.4, chi = 16, 3 iterations, every GEMM of both
    drivers on the int8 path; weights, logZ, bond representations, rdms and
    the PEPS norm against the reference's run."""
    from frostspin_b200 import U1SymmetricTensor, linalg
    from frostspin_b200.ctmrg import SequentialCTMRG
    from frostspin_b200.simple_update import SimpleUpdate

    d = load("simple_update_u1")
    h = U1SymmetricTensor.load_from_dic(d, prefix="h")
    with linalg.gemm_precision_mode(precision), linalg.ozaki_dispatch_mode("all"):
        su = SimpleUpdate.square_lattice_first_neighbor(h, int(d["D"]), float(d["tau"]),
                                                        rcutoff=1e-10, degen_ratio=0.9999)
        for k in range(2):
            su.evolve(0.2)
            assert abs(su.beta - float(d[f"b{k}_beta"])) < 1e-12
            assert abs(su.logZ - float(d[f"b{k}_logZ"])) < 1e-11
            for i, w in enumerate(su.get_weights()):
                np.testing.assert_allclose(w, d[f"b{k}_w{i}"], rtol=1e-9, atol=1e-13)
            for i, r in enumerate(su.get_bond_representations()):
                assert np.array_equal(r, d[f"b{k}_rep{i}"])
        ctm = SequentialCTMRG.from_elementary_tensors("AB\nBA", su.get_tensors(), 16,
                                                      cutoff=1e-10, degen_ratio=0.9999)
        for _ in range(3):
            ctm.iterate()
        for x, y in ctm.site_coords:
            for kind, fn in (("rdm1x2", ctm.compute_rdm1x2), ("rdm2x1", ctm.compute_rdm2x1)):
                got = fn(x, y).toarray()
                assert np.abs(got - d[f"{kind}_{x}{y}"]).max() < 1e-8
        logz = ctm.compute_PEPS_norm_log()
    linalg.check_ozaki_flags()
    assert abs(logz - float(d["logZ_ctm"])) < 1e-8
