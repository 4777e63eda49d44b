"""Simple update on the device against the reference's own run (U(1)
Heisenberg, D=6, tau=0.01): bond weights, logZ and bond representations after
beta = 0.2 and 0.4, then SequentialCTMRG observables on the resulting tensors.
Weights and logZ are gauge invariant; tensors are compared through the
reduced density matrices of the CTMRG environment."""

import numpy as np
import pytest

from tests.helpers import load

pytestmark = pytest.mark.gpu


def test_simple_update_then_ctmrg_matches_reference():
    from frostspin_b200 import U1SymmetricTensor
    from frostspin_b200.ctmrg import SequentialCTMRG
    from frostspin_b200.simple_update import SimpleUpdate

    d = load("simple_update_u1")
    h = U1SymmetricTensor.load_from_dic(d, prefix="h")
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
    assert abs(ctm.compute_PEPS_norm_log() - float(d["logZ_ctm"])) < 1e-8


def test_su2_simple_update_then_ctmrg_matches_reference():
    """The same chain with SU(2) symmetry (D=8 states, chi=20): weights, logZ and
    bond representations after beta = 0.2 and 0.4, the CTMRG chi after each
    iteration (bit-identical truncation decisions), then the rdms."""
    from frostspin_b200 import SU2SymmetricTensor
    from frostspin_b200.ctmrg import SequentialCTMRG
    from frostspin_b200.simple_update import SimpleUpdate

    d = load("simple_update_su2")
    h = SU2SymmetricTensor.load_from_dic(d, prefix="h")
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
    ctm = SequentialCTMRG.from_elementary_tensors("AB\nBA", su.get_tensors(), 20,
                                                  cutoff=1e-10, degen_ratio=0.9999)
    for it in range(3):
        ctm.iterate()
        assert np.array_equal(ctm.chi_values, d[f"it{it}_chi"])
    for x, y in ctm.site_coords:
        for kind, fn in (("rdm1x2", ctm.compute_rdm1x2), ("rdm2x1", ctm.compute_rdm2x1)):
            got = fn(x, y).toarray()
            assert np.abs(got - d[f"{kind}_{x}{y}"]).max() < 1e-8
    assert abs(ctm.compute_PEPS_norm_log() - float(d["logZ_ctm"])) < 1e-8


def test_su2_simple_update_d24_matches_reference():
    """The benchmark's simple update (SU(2), D=24 target, tau=0.01) evolved to
    beta=2 on the device against the reference's own run: Dmax, bond
    representations (bit-exact truncation decisions over 200 Trotter steps),
    weights and logZ."""
    from frostspin_b200 import SU2SymmetricTensor
    from frostspin_b200.simple_update import SimpleUpdate

    d = load("su2_d24_beta2")
    r = np.array([[1], [2]])
    sds = np.array([[0.25, 0, 0, 0], [0, -0.25, 0.5, 0], [0, 0.5, -0.25, 0],
                    [0, 0, 0, 0.25]]).reshape(2, 2, 2, 2)
    h = SU2SymmetricTensor.from_array(sds, (r, r), (r, r))
    su = SimpleUpdate.square_lattice_first_neighbor(h, 24, 0.01, rcutoff=1e-10,
                                                    degen_ratio=0.9999)
    su.evolve(2.0)
    assert abs(su.beta - float(d["beta"])) < 1e-12
    assert su.Dmax == int(d["Dmax"])
    for i, rep in enumerate(su.get_bond_representations()):
        assert np.array_equal(rep, d[f"rep{i}"])
    for i, w in enumerate(su.get_weights()):
        np.testing.assert_allclose(w, d[f"w{i}"], rtol=1e-8, atol=1e-12)
    assert abs(su.logZ - float(d["logZ"])) < 1e-10


@pytest.mark.parametrize("model", ["J1-J2", "checkerboard", "Shastry-Sutherland"])
def test_second_neighbor_models_match_reference(model):
    """square_lattice_second_neighbor (simple_update.py:366-407) with the U(1)
    Heisenberg gates (J2 = 0.5, D = 4): beta, logZ, bond representations and
    weights after each of two evolve steps equal the reference's run.  The
    second-neighbour gates go through update_through_proxy
    (simple_update.py:700-790)."""
    from frostspin_b200 import U1SymmetricTensor
    from frostspin_b200.simple_update import SimpleUpdate

    d = load("simple_update_j1j2")
    h1 = U1SymmetricTensor.load_from_dic(d, prefix="h1")
    su = SimpleUpdate.square_lattice_second_neighbor(h1, 0.5 * h1, 4, 0.01, model=model,
                                                     rcutoff=1e-10, degen_ratio=0.9999)
    for k in range(2):
        su.evolve(0.04)
        assert abs(su.beta - float(d[f"{model}_b{k}_beta"])) < 1e-12
        assert abs(su.logZ - float(d[f"{model}_b{k}_logZ"])) < 1e-10
        for i, r in enumerate(su.get_bond_representations()):
            assert np.array_equal(r, d[f"{model}_b{k}_rep{i}"]), (k, i)
        for i, w in enumerate(su.get_weights()):
            assert np.abs(w - d[f"{model}_b{k}_w{i}"]).max() < 1e-8, (k, i)


def test_symmetrized_simple_update_matches_reference():
    """SymmetrizedSimpleUpdate (symmetrized_simple_update.py:10-271) on the input
    of the reference's tests/test_symmetrized_ctm.py (D = 7), tau = 0.01, two
    evolve steps: beta, logZ, bond representations and weights equal the
    reference's run; the tensors of the cell are A and its rotated dagger."""
    from frostspin_b200 import SU2SymmetricTensor
    from frostspin_b200.simple_update import SymmetrizedSimpleUpdate

    d = load("symmetrized_simple_update")
    h = SU2SymmetricTensor.load_from_dic(d, prefix="h")
    su = SymmetrizedSimpleUpdate.from_infinite_temperature(7, 0.01, [h])
    assert su.n_bonds == 4 and su.beta == 0.0
    for k in range(2):
        su.evolve(0.1)
        assert abs(su.beta - float(d[f"b{k}_beta"])) < 1e-12
        assert abs(su.logZ - float(d[f"b{k}_logZ"])) < 1e-10
        for i, r in enumerate(su.get_bond_representations()):
            assert np.array_equal(r, d[f"b{k}_rep{i}"]), (k, i)
        for i, w in enumerate(su.get_weights()):
            assert np.abs(w - d[f"b{k}_w{i}"]).max() < 1e-8, (k, i)
    A, B = su.get_tensors()
    assert (B - A.dagger().permute((4, 5), (2, 3, 0, 1))).norm() < 1e-14
