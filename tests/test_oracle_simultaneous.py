"""Pin the oracle's SimultaneousCTMRG against the reference's own runs
(tests/golden/simultaneous_ctmrg.npz): the random U(1) AB/BA network and the
SU(2) simple-update tensors, chi = 20, 3 iterations.  Singular vectors are
defined up to a gauge, so gauge-invariant quantities are compared: reduced
density matrices after every iteration."""

import numpy as np
import pytest

from oracle import ctmrg_oracle as co
from oracle import frostspin_oracle as fo
from oracle import su2_oracle as so
from tests.helpers import load


def site_tensors(tag):
    if tag == "u1":
        d, names, mod = load("ctmrg_u1_random"), ("A", "B"), fo
    else:
        d, names, mod = load("simple_update_su2"), ("A0", "A1"), so
    out = []
    for p in names:
        nrr = int(d[p + "_n_row_reps"])
        ncr = int(d[p + "_n_col_reps"])
        irr = d[p + "_block_irreps"]
        out.append(mod.OTensor([d[f"{p}_row_rep_{i}"] for i in range(nrr)],
                               [d[f"{p}_col_rep_{i}"] for i in range(ncr)],
                               [d[f"{p}_block_{i}"] for i in range(irr.size)], irr,
                               d[p + "_signature"]))
    return out


@pytest.mark.parametrize("tag", ["u1", "su2"])
def test_simultaneous_ctmrg_oracle_matches_reference_run(tag):
    ref = load("simultaneous_ctmrg")
    A, B = site_tensors(tag)
    ctm = co.SimultaneousCTMRG(A, B, 20, cutoff=1e-10, degen_ratio=0.9999)
    for it in range(3):
        ctm.iterate()
        chi = sorted({s for C in ctm.t["C1"] + ctm.t["C3"] for s in C.shape})
        assert chi == list(ref[f"{tag}_it{it}_chi"]), it
        for x, y in ctm.coords:
            for kind, fn in (("rdm1x2", co.ctm_rdm1x2), ("rdm2x1", co.ctm_rdm2x1)):
                r = ref[f"{tag}_it{it}_{kind}_{x}{y}"]
                assert np.abs(fn(ctm, x, y) - r).max() < 1e-8 * max(1.0, np.abs(r).max())


def test_symmetrized_reference_run_equals_simultaneous_oracle():
    """With B the rotated dagger of A the symmetrized and simultaneous
    algorithms build the same environment: the oracle's SimultaneousCTMRG on
    the input of the reference's tests/test_symmetrized_ctm.py reproduces the
    reference's SymmetrizedCTMRG chi values and rdms (tests/golden/
    ctmrg_variants.npz), which pins that fixture independently."""
    ref = load("ctmrg_variants")
    p = "symA"
    nrr = int(ref[p + "_n_row_reps"])
    ncr = int(ref[p + "_n_col_reps"])
    irr = ref[p + "_block_irreps"]
    A = so.OTensor([ref[f"{p}_row_rep_{i}"] for i in range(nrr)],
                   [ref[f"{p}_col_rep_{i}"] for i in range(ncr)],
                   [ref[f"{p}_block_{i}"] for i in range(irr.size)], irr, ref[p + "_signature"])
    B = so.permute(so.dagger(A), (4, 5), (2, 3, 0, 1))
    ctm = co.SimultaneousCTMRG(A, B, 50, cutoff=1e-11, degen_ratio=0.9999)
    for it in range(3):
        ctm.iterate()
        chi = sorted({s for C in ctm.t["C1"] + ctm.t["C3"] for s in C.shape})
        assert chi == list(ref[f"sym_it{it}_chi"]), it
        for x, y in ctm.coords:
            for kind, fn in (("rdm1x2", co.ctm_rdm1x2), ("rdm2x1", co.ctm_rdm2x1)):
                r = ref[f"sym_it{it}_{kind}_{x}{y}"]
                assert np.abs(fn(ctm, x, y) - r).max() < 1e-12
