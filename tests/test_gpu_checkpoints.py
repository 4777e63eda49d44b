"""Checkpoint interchange with the reference (ctm_environment.py:240-276,
abstract_ctmrg.py:169-216, abstract_simple_update.py:149-187,
simple_update.py:538-597).

The fixtures ckpt_ctmrg_u1.npz and ckpt_su_u1.npz are files the reference's
own save_to_file wrote (tests/golden/make_golden.py, case_checkpoints); the
device drivers load them, continue, and must reproduce what the reference
computed after reloading the same files (ckpt_expect.npz).  In the other
direction, a checkpoint the device writes has the reference's keys, and every
array in it equals the one the reference wrote for the same state.  Finally a
run interrupted by save / load continues exactly like an uninterrupted one
(SimpleUpdate and SymmetrizedSimpleUpdate)."""

import os

import numpy as np
import pytest

from tests.helpers import GOLDEN, load

pytestmark = pytest.mark.gpu


def test_reference_ctmrg_checkpoint_loads_and_continues(tmp_path):
    from frostspin_b200.ctmrg import SequentialCTMRG

    ref_file = os.path.join(GOLDEN, "ckpt_ctmrg_u1.npz")
    exp = load("ckpt_expect")
    ctm = SequentialCTMRG.load_from_file(ref_file)
    # written back unchanged: the reference's keys and arrays, exactly
    mine = tmp_path / "ctm.npz"
    ctm.save_to_file(mine)
    with np.load(ref_file) as a, np.load(mine) as b:
        assert set(a.files) == set(b.files)
        for k in a.files:
            assert np.array_equal(np.asarray(a[k]), np.asarray(b[k])), k
    ctm.iterate()
    assert list(ctm.chi_values) == list(exp["ctm_chi"])
    for x, y in ctm.site_coords:
        for kind, fn in (("rdm1x2", ctm.compute_rdm1x2), ("rdm2x1", ctm.compute_rdm2x1)):
            assert np.abs(fn(x, y).toarray() - exp[f"ctm_{kind}_{x}{y}"]).max() < 1e-9
    assert abs(ctm.compute_PEPS_norm_log() - float(exp["ctm_logZ"])) < 1e-9


def test_reference_simple_update_checkpoint_loads_and_continues(tmp_path):
    from frostspin_b200.simple_update import SimpleUpdate

    ref_file = os.path.join(GOLDEN, "ckpt_su_u1.npz")
    exp = load("ckpt_expect")
    su = SimpleUpdate.load_from_file(ref_file)
    mine = tmp_path / "su.npz"
    su.save_to_file(mine)
    with np.load(ref_file) as a, np.load(mine) as b:
        assert set(a.files) == set(b.files)
        for k in a.files:
            assert np.array_equal(np.asarray(a[k]), np.asarray(b[k])), k
    su.evolve(0.2)
    assert abs(su.beta - float(exp["su_beta"])) < 1e-12
    assert abs(su.logZ - float(exp["su_logZ"])) < 1e-11
    for i, w in enumerate(su.get_weights()):
        np.testing.assert_allclose(w, exp[f"su_w{i}"], rtol=1e-9, atol=1e-13)
    for i, r in enumerate(su.get_bond_representations()):
        assert np.array_equal(r, exp[f"su_rep{i}"])


@pytest.mark.parametrize("kind", ["plain", "symmetrized"])
def test_interrupted_simple_update_continues_identically(tmp_path, kind):
    from frostspin_b200 import SU2SymmetricTensor
    from frostspin_b200.simple_update import SimpleUpdate, SymmetrizedSimpleUpdate

    if kind == "plain":
        d = load("simple_update_su2")
        h = SU2SymmetricTensor.load_from_dic(d, prefix="h")

        def make():
            return SimpleUpdate.square_lattice_first_neighbor(h, 8, 0.01, rcutoff=1e-10,
                                                              degen_ratio=0.9999)
        cls = SimpleUpdate
    else:
        d = load("symmetrized_simple_update")
        h = SU2SymmetricTensor.load_from_dic(d, prefix="h")

        def make():
            return SymmetrizedSimpleUpdate.from_infinite_temperature(7, 0.01, [h])
        cls = SymmetrizedSimpleUpdate
    a = make()
    a.evolve(0.1)
    a.evolve(0.1)
    b = make()
    b.evolve(0.1)
    f = tmp_path / "su.npz"
    b.save_to_file(f)
    c = cls.load_from_file(f)
    c.evolve(0.1)
    assert abs(c.beta - a.beta) < 1e-14
    assert abs(c.logZ - a.logZ) < 1e-12
    for wa, wc in zip(a.get_weights(), c.get_weights(), strict=True):
        np.testing.assert_allclose(wc, wa, rtol=1e-12, atol=1e-15)
    for ra, rc in zip(a.get_bond_representations(), c.get_bond_representations(), strict=True):
        assert np.array_equal(ra, rc)
    for ta, tc in zip(a.get_tensors(), c.get_tensors(), strict=True):
        assert (ta - tc).norm() < 1e-12 * ta.norm()
