"""The autotuner's dispatch rule (frostspin_b200/autotune.py) on a hand-made
table: measured classes follow the measurement, unmeasured ones their nearest
measured neighbours, and classes with no neighbour the cost model.  Measuring needs a GPU; the rule does not."""

import numpy as np

from frostspin_b200 import _native, autotune, linalg


def _arr(shapes):
    arr = np.zeros(len(shapes), dtype=_native.GEMM_PROBLEM_DTYPE)
    for i, (m, n, k) in enumerate(shapes):
        arr["M"][i], arr["N"][i], arr["K"][i] = m, n, k
    return arr


def test_decide_uses_measured_classes_only():
    autotune.clear()
    arr = _arr([(3000, 3000, 3000), (100, 5000, 40), (7, 7, 7)])
    mode = "ozaki2_13"
    autotune._TABLE[(mode, autotune.shape_class(3000, 3000, 3000))] = {
        "fp64": 3e-14, "mixed": 1e-14, "shape": (3000, 3000, 3000)}
    autotune._TABLE[(mode, autotune.shape_class(100, 5000, 40))] = {
        "fp64": 1e-13, "mixed": 4e-13, "shape": (100, 5000, 40)}
    assert autotune.decide(arr, mode) == [True, False, None]
    model = np.array([False, True, True])
    autotune.set_enabled(True)
    try:
        assert list(linalg._tuned(arr, mode, model)) == [True, False, True]
    finally:
        autotune.set_enabled(False)
        autotune.clear()
    assert list(linalg._tuned(arr, mode, model)) == [False, True, True]


def test_shape_classes_are_bit_lengths():
    assert autotune.shape_class(1, 2, 3) == (1, 2, 2)
    assert autotune.shape_class(255, 256, 257) == (8, 9, 9)


def test_unmeasured_classes_take_nearest_measured_choice():
    autotune.clear()
    mode = "ozaki2_13"
    big = autotune.shape_class(3000, 3000, 3000)        # (12, 12, 12)
    thin = autotune.shape_class(100, 5000, 40)          # (7, 13, 6)
    autotune._TABLE[(mode, big)] = {"fp64": 3e-14, "mixed": 1e-14, "shape": (3000,) * 3}
    autotune._TABLE[(mode, thin)] = {"fp64": 1e-13, "mixed": 4e-13, "shape": (100, 5000, 40)}
    try:
        arr = _arr([(5000, 3000, 3000),     # (13, 12, 12): distance 1 from big
                    (100, 9000, 40),        # (7, 14, 6): distance 1 from thin
                    (5000, 5000, 5000),     # (13, 13, 13): distance 3, none near
                    (7, 7, 7)])
        assert autotune.decide(arr, mode) == [True, False, None, None]
        # equidistant neighbours that disagree: FP64
        mid = autotune.shape_class(3000, 3000, 3000)
        autotune._TABLE[(mode, (12, 12, 14))] = {"fp64": 1e-14, "mixed": 2e-14,
                                                  "shape": (3000, 3000, 9000)}
        assert autotune.decide(_arr([(3000, 3000, 5000)]), mode) == [False]
        assert mid == (12, 12, 12)
    finally:
        autotune.clear()


def test_predict_sums_measured_rates():
    autotune.clear()
    mode = "ozaki2_11"
    big = (3000, 3000, 3000)
    thin = (100, 5000, 40)
    autotune._TABLE[(mode, autotune.shape_class(*big))] = {"fp64": 3e-14, "mixed": 1e-14,
                                                           "shape": big}
    autotune._TABLE[(mode, autotune.shape_class(*thin))] = {"fp64": 1e-13, "mixed": 4e-13,
                                                            "shape": thin}
    try:
        rec = [_arr([big, thin, (7, 7, 7)])]
        got = autotune.predict(rec, mode)
        fb, ft = 2.0 * 3000**3, 2.0 * 100 * 5000 * 40
        assert abs(got["fp64"] - (3e-14 * fb + 1e-13 * ft)) < 1e-12
        assert abs(got["mixed"] - (1e-14 * fb + 4e-13 * ft)) < 1e-12
        assert abs(got["chosen"] - (1e-14 * fb + 1e-13 * ft)) < 1e-12
    finally:
        autotune.clear()
