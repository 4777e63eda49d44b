"""Pin the CPU simple-update oracle (oracle/simple_update_oracle.py) against
runs of the reference implementation: tests/golden/simple_update_u1.npz (U(1),
D=6, two evolve(0.2)), simple_update_su2.npz (SU(2), D=8, two evolve(0.2)) and
su2_d24_beta2.npz (SU(2), D=24, evolve(2.0), the benchmark's model)."""

import numpy as np
import pytest

from oracle import frostspin_oracle as fo
from oracle import simple_update_oracle as suo
from oracle import su2_oracle as so
from tests.helpers import load

SDS = np.array([[0.25, 0, 0, 0], [0, -0.25, 0.5, 0], [0, 0.5, -0.25, 0],
                [0, 0, 0, 0.25]]).reshape(2, 2, 2, 2)


def _h(d, m):
    nrr, ncr = int(d["h_n_row_reps"]), int(d["h_n_col_reps"])
    irr = d["h_block_irreps"]
    return m.OTensor([d[f"h_row_rep_{i}"] for i in range(nrr)],
                     [d[f"h_col_rep_{i}"] for i in range(ncr)],
                     [d[f"h_block_{i}"] for i in range(irr.size)], irr, d["h_signature"])


def _check_state(su, d, pre, *, logz_tol, w_tol):
    assert abs(su.beta - float(d[pre + "beta"])) < 1e-12
    assert abs(su.logZ - float(d[pre + "logZ"])) < logz_tol
    for i in range(4):
        rep = su.bond_representation(i)
        assert np.array_equal(rep, d[f"{pre}rep{i}"]), i
        w = su.sorted_weights(i)
        ref = np.sort(np.asarray(d[f"{pre}w{i}"]))[::-1]
        assert w.shape == ref.shape, i
        assert np.abs(w - ref).max() < w_tol, i


@pytest.mark.parametrize("name,module", [("simple_update_u1", fo), ("simple_update_su2", so)])
def test_simple_update_oracle_matches_reference_runs(name, module):
    d = load(name)
    su = suo.SimpleUpdate(_h(d, module), int(d["D"]), float(d["tau"]), rcutoff=1e-10,
                          degen_ratio=0.9999)
    for k in range(2):
        su.evolve(0.2)
        _check_state(su, d, f"b{k}_", logz_tol=1e-12, w_tol=1e-13)


def test_su2_simple_update_oracle_d24_to_beta2():
    """The benchmark's simple update (SU(2), D=24 target, tau=0.01) evolved to
    beta=2 in one call, as the reference's run that wrote the fixture."""
    d = load("su2_d24_beta2")
    r = np.array([[1], [2]])
    h = so.from_array(SDS, (r, r), (r, r))
    su = suo.SimpleUpdate(h, 24, 0.01, rcutoff=1e-10, degen_ratio=0.9999)
    su.evolve(2.0)
    assert abs(su.beta - float(d["beta"])) < 1e-12
    assert abs(su.logZ - float(d["logZ"])) < 1e-12
    for i in range(4):
        assert np.array_equal(su.bond_representation(i), d[f"rep{i}"]), i
        ref = np.sort(np.asarray(d[f"w{i}"]))[::-1]
        assert np.abs(su.sorted_weights(i) - ref).max() < 1e-12, i
    assert max(int(su.bond_representation(i)[0] @ su.bond_representation(i)[1])
               for i in range(4)) == int(d["Dmax"])
