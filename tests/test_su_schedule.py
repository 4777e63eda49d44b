"""Simple-update schedules on the CPU: the model tables and the update
sequence (legs, swaps, gates) against the reference's own get_update_data
(tests/golden/su_schedules.npz).  The schedule only multiplies Hamiltonians by
2, so scalars stand in for them."""

import json

import numpy as np
import pytest

from frostspin_b200.simple_update.simple_update import UpdateSchedule
from frostspin_b200.simple_update.su_models import TENSOR_BOND_INDICES, j1_j2_models
from tests.helpers import load

CASES = ["first", "J1-J2", "checkerboard", "Shastry-Sutherland"]


def plain(v):
    if isinstance(v, (list, tuple)):
        return [plain(x) for x in v]
    return v


@pytest.mark.parametrize("name", CASES)
def test_update_schedule_matches_reference(name):
    d = load("su_schedules")
    if name == "first":
        tbi = [[0, 1, 2, 3], [2, 3, 0, 1]]
        table = np.array([[b, b, 0, 0, 1, -1] for b in range(4)])
        hams = [1.0]
    else:
        tbi = TENSOR_BOND_INDICES
        table = j1_j2_models[name]
        hams = [1.0, 0.5]
    assert np.array_equal(table, d[f"{name}_table"])
    s = UpdateSchedule(tbi, table, hams)

    def ref(key):
        return json.loads(str(d[f"{name}_{key}"]))

    for key, mine in (("bond1", s.bond1), ("bond2", s.bond2), ("gate", s.gate),
                      ("left", s.left), ("right", s.right), ("middle", s.middle),
                      ("lperm", s.lperm), ("rperm", s.rperm), ("mperm", s.mperm),
                      ("initial_swap", s.initial_swap), ("final_swap", s.final_swap),
                      ("hamiltonians", s.hamiltonians)):
        assert plain([None if x is None else (x if isinstance(x, (tuple, list)) else
                      (float(x) if key == "hamiltonians" else int(x))) for x in mine]) \
            == ref(key), (name, key)


def test_unknown_model_rejected():
    from frostspin_b200.simple_update import SimpleUpdate

    with pytest.raises(KeyError):
        SimpleUpdate.square_lattice_second_neighbor(None, None, 4, 0.01, model="kagome")
