"""Many independent C4v CTMRG runs advanced in lock step (iterate_c4v_many):
every step launches the sector GEMMs of all runs together and the permutes of
all runs together (fs_abelian_permute_multi), and the results equal those of
the runs iterated one by one, including the reference's own run."""

import numpy as np
import pytest

from tests.helpers import diag_from_dic, load

pytestmark = pytest.mark.gpu


def _runs(specs):
    from frostspin_b200.ctmrg import ising_initial_environment, ising_site_tensors

    out = []
    for i, (beta, chi) in enumerate(specs):
        a, a2, a0d, mopd = ising_site_tensors(beta)
        s, T = ising_initial_environment(chi, np.random.default_rng(100 + i))
        out.append([s, T, a, a2, chi, a0d, mopd])
    return out


def test_lock_step_runs_equal_single_runs():
    from frostspin_b200 import _native
    from frostspin_b200.ctmrg import energy_per_bond, iterate_c4v, iterate_c4v_many

    specs = [(0.35, 8), (0.44, 16), (0.55, 12), (0.41, 16), (0.30, 8)]
    batch = _runs(specs)
    single = _runs(specs)
    for it in range(6):
        before = dict(_native.CALL_COUNTS)
        res = iterate_c4v_many([r[:5] for r in batch])
        after = dict(_native.CALL_COUNTS)
        for r, (s, T) in zip(batch, res, strict=True):
            r[0], r[1] = s, T
        for r in single:
            r[0], r[1] = iterate_c4v(r[0], r[1], r[2], r[3], r[4])
        # six permute steps and four GEMM steps, one launch each for all runs
        assert after.get("fs_abelian_permute_multi", 0) - before.get(
            "fs_abelian_permute_multi", 0) == 6
        assert after.get("fs_abelian_permute", 0) == before.get("fs_abelian_permute", 0)
    for rb, rs in zip(batch, single, strict=True):
        assert np.array_equal(rb[0].block_irreps, rs[0].block_irreps)
        for x, y in zip(rb[0].host_blocks(), rs[0].host_blocks(), strict=True):
            np.testing.assert_allclose(x, y, rtol=1e-10, atol=1e-13)
        eb = energy_per_bond(rb[0], rb[1], rb[5], rb[6])
        es = energy_per_bond(rs[0], rs[1], rs[5], rs[6])
        assert abs(eb - es) < 1e-10


def test_lock_step_run_matches_reference():
    """The reference's chi = 8 run (examples/ising_classical_ctmrg.py) inside a
    batch with other runs: corner spectra and energies after each stored
    iteration."""
    from frostspin_b200 import DiagonalTensor
    from frostspin_b200.ctmrg import energy_per_bond, ising_site_tensors, iterate_c4v_many
    from tests.test_gpu_tensor import dev_from_dic

    d = load("ising_chi8")
    beta = float(d["beta"])
    a, a2, a0d, mopd = ising_site_tensors(beta)
    runs = [[DiagonalTensor.load_from_dic(d, prefix="s0"), dev_from_dic(d, "T0"), a, a2, 8]]
    runs += [r[:5] for r in _runs([(0.5, 16), (0.33, 12)])]
    for it in range(1, 11):
        res = iterate_c4v_many(runs)
        for r, (s, T) in zip(runs, res, strict=True):
            r[0], r[1] = s, T
        if f"s{it}_block_irreps" in d:
            ref_blocks, ref_irr = diag_from_dic(d, f"s{it}")
            assert np.array_equal(runs[0][0].block_irreps, ref_irr)
            for x, y in zip(runs[0][0].host_blocks(), ref_blocks, strict=True):
                np.testing.assert_allclose(x, y, rtol=1e-9, atol=1e-13)
            e = energy_per_bond(runs[0][0], runs[0][1], a0d, mopd)
            assert abs(e - float(d[f"energy{it}"])) < 1e-9
