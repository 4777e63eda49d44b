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


@pytest.mark.parametrize("tag", ["su2", "u1"])
def test_transfer_spectrum_and_corr_length_match_reference(tag):
    """abstract_ctmrg.py:519-579 / observables.py:4-154 on the device against the
    reference's values after 3 CTMRG iterations at chi=20: the 4 leading
    transfer eigenvalues (as a multiset; conjugate pairs may come in either
    order) and the correlation lengths, horizontal and vertical."""
    from frostspin_b200 import SU2SymmetricTensor, U1SymmetricTensor
    from frostspin_b200.ctmrg import SequentialCTMRG

    ref = load("corr_length")
    if tag == "su2":
        d = load("simple_update_su2")
        tensors = [SU2SymmetricTensor.load_from_dic(d, prefix=p) for p in ("A0", "A1")]
    else:
        d = load("ctmrg_u1_random")
        tensors = [U1SymmetricTensor.load_from_dic(d, prefix=p) for p in ("A", "B")]
    ctm = SequentialCTMRG.from_elementary_tensors("AB\nBA", tensors, 20, cutoff=1e-10,
                                                  degen_ratio=0.9999)
    for _ in range(3):
        ctm.iterate()
    assert np.array_equal(ctm.chi_values, ref[f"{tag}_chi"])
    for k in range(2):
        for kind, fn in (("h", ctm.compute_transfer_spectrum_h),
                         ("v", ctm.compute_transfer_spectrum_v)):
            got = np.asarray(fn(k, 4))
            exp = np.asarray(ref[f"{tag}_spec_{kind}{k}"])
            key = lambda z: (round(float(np.abs(z)), 9), round(float(np.imag(z)), 9))  # noqa: E731
            for a, b in zip(sorted(got, key=key), sorted(exp, key=key), strict=True):
                assert abs(a - b) < 1e-8, (kind, k, got, exp)
        xh = ctm.compute_corr_length_h(k)
        xv = ctm.compute_corr_length_v(k)
        assert abs(xh - float(ref[f"{tag}_xi_h{k}"])) < 1e-7 * float(ref[f"{tag}_xi_h{k}"])
        assert abs(xv - float(ref[f"{tag}_xi_v{k}"])) < 1e-7 * float(ref[f"{tag}_xi_v{k}"])


@pytest.mark.parametrize("fused", [False, True])
def test_su2_ctmrg_from_reference_d24_tensors(fused):
    """SU(2) SequentialCTMRG on the benchmark's site tensors (the reference's
    own D=24 simple update at beta=2, Dmax=28) at chi=24: chi after each
    iteration (bit-identical truncation), rdms and energy against the
    reference's run; with the SU(2) permutes through the three launches and
    through the fused kernel."""
    from frostspin_b200 import SU2SymmetricTensor
    from frostspin_b200.ctmrg import SequentialCTMRG
    from frostspin_b200.symmetric_tensor import lie_group_symmetric_tensor as lg

    d = load("su2_d24_beta2")
    ref = load("ctmrg_su2_d24")
    tensors = [SU2SymmetricTensor.load_from_dic(d, prefix=p) for p in ("A0", "A1")]
    was = lg.fused_permute_enabled()
    lg.set_fused_permute(fused)
    try:
        ctm = SequentialCTMRG.from_elementary_tensors("AB\nBA", tensors, 24, cutoff=1e-10,
                                                      degen_ratio=0.9999)
        for it in range(2):
            ctm.iterate()
            assert np.array_equal(ctm.chi_values, ref[f"it{it}_chi"])
        sds = np.array([[0.25, 0, 0, 0], [0, -0.25, 0.5, 0], [0, 0.5, -0.25, 0],
                        [0, 0, 0, 0.25]]).reshape(2, 2, 2, 2)
        es = []
        for x, y in ctm.site_coords:
            r12 = ctm.compute_rdm1x2(x, y).toarray()
            r21 = ctm.compute_rdm2x1(x, y).toarray()
            assert np.abs(r12 - ref[f"rdm1x2_{x}{y}"]).max() < 1e-9
            assert np.abs(r21 - ref[f"rdm2x1_{x}{y}"]).max() < 1e-9
            es += [np.einsum("ijkl,klij->", r12, sds), np.einsum("ijkl,klij->", r21, sds)]
    finally:
        lg.set_fused_permute(was)
    assert abs(np.mean(es) - float(ref["energy"])) < 1e-10


@pytest.mark.parametrize("tag", ["u1", "su2"])
def test_simultaneous_ctmrg_matches_reference(tag):
    """SimultaneousCTMRG (simultaneous_ctmrg.py:14-132) against the reference's
    run on the same tensors: chi values, rdms and the PEPS norm after each of 3
    iterations at chi = 20."""
    from frostspin_b200 import SU2SymmetricTensor, U1SymmetricTensor
    from frostspin_b200.ctmrg import SimultaneousCTMRG

    ref = load("simultaneous_ctmrg")
    if tag == "su2":
        d = load("simple_update_su2")
        tensors = [SU2SymmetricTensor.load_from_dic(d, prefix=p) for p in ("A0", "A1")]
    else:
        d = load("ctmrg_u1_random")
        tensors = [U1SymmetricTensor.load_from_dic(d, prefix=p) for p in ("A", "B")]
    ctm = SimultaneousCTMRG.from_elementary_tensors("AB\nBA", tensors, 20, cutoff=1e-10,
                                                    degen_ratio=0.9999)
    assert "SimultaneousCTMRG" in repr(ctm)
    for it in range(3):
        ctm.iterate()
        assert ctm.chi_values == list(ref[f"{tag}_it{it}_chi"]), it
        for x, y in ctm.site_coords:
            for kind, fn in (("rdm1x2", ctm.compute_rdm1x2), ("rdm2x1", ctm.compute_rdm2x1)):
                r = ref[f"{tag}_it{it}_{kind}_{x}{y}"]
                got = fn(x, y).toarray()
                assert np.abs(got - r).max() < 1e-8 * max(1.0, np.abs(r).max()), (it, kind)
        assert abs(ctm.compute_PEPS_norm_log() - float(ref[f"{tag}_it{it}_logZ"])) < 1e-8


def test_second_neighbor_rdms_match_reference():
    """compute_rdm1x1_cell and compute_rdm_2nd_neighbor_cell
    (abstract_ctmrg.py:438-518, rdm.py:190-269) after 3 SequentialCTMRG
    iterations at chi = 20 on the SU(2) simple-update tensors."""
    from frostspin_b200 import SU2SymmetricTensor
    from frostspin_b200.ctmrg import SequentialCTMRG

    ref = load("ctmrg_variants")
    d = load("simple_update_su2")
    tensors = [SU2SymmetricTensor.load_from_dic(d, prefix=p) for p in ("A0", "A1")]
    ctm = SequentialCTMRG.from_elementary_tensors("AB\nBA", tensors, 20, cutoff=1e-10,
                                                  degen_ratio=0.9999)
    for _ in range(3):
        ctm.iterate()
    for i, r in enumerate(ctm.compute_rdm1x1_cell()):
        assert np.abs(r.toarray() - ref[f"seq_rdm1x1_{i}"]).max() < 1e-8
    dr, ur = ctm.compute_rdm_2nd_neighbor_cell()
    for i, (a, b) in enumerate(zip(dr, ur, strict=True)):
        assert np.abs(a.toarray() - ref[f"seq_rdm_dr_{i}"]).max() < 1e-8
        assert np.abs(b.toarray() - ref[f"seq_rdm_ur_{i}"]).max() < 1e-8


def test_symmetrized_ctmrg_matches_reference():
    """SymmetrizedCTMRG (symmetrized_ctmrg.py:19-274) on the input of the
    reference's tests/test_symmetrized_ctm.py (B = rotated dagger of A,
    chi = 50): PEPS norm before and after each of 3 iterations, chi values,
    nearest- and second-neighbour rdms."""
    from frostspin_b200 import SU2SymmetricTensor
    from frostspin_b200.ctmrg import SymmetrizedCTMRG

    ref = load("ctmrg_variants")
    A = SU2SymmetricTensor.load_from_dic(ref, prefix="symA")
    B = A.dagger().permute((4, 5), (2, 3, 0, 1))
    ctm = SymmetrizedCTMRG.from_elementary_tensors("AB\nBA", [A, B], 50)
    assert "SymmetrizedCTMRG" in repr(ctm)
    assert abs(ctm.compute_PEPS_norm_log() - float(ref["sym_it-1_logZ"])) < 1e-10
    for it in range(3):
        ctm.iterate()
        assert ctm.chi_values == list(ref[f"sym_it{it}_chi"]), it
        for x, y in ctm.site_coords:
            for kind, fn in (("rdm1x2", ctm.compute_rdm1x2), ("rdm2x1", ctm.compute_rdm2x1)):
                r = ref[f"sym_it{it}_{kind}_{x}{y}"]
                assert np.abs(fn(x, y).toarray() - r).max() < 1e-8, (it, kind)
        assert abs(ctm.compute_PEPS_norm_log() - float(ref[f"sym_it{it}_logZ"])) < 1e-8
    (dr, _), (ur, _) = ctm.compute_rdm_2nd_neighbor_cell()
    assert np.abs(dr.toarray() - ref["sym_rdm_dr"]).max() < 1e-8
    assert np.abs(ur.toarray() - ref["sym_rdm_ur"]).max() < 1e-8
