"""The error statistics of accuracy.field_errors (used by the bench, smoke() and the parity
tests): field-scaled and pointwise relative errors, the pointwise floor, NaN bookkeeping."""
import numpy as np

from distorteddustydiscanalysistoolkits_b200 import accuracy


def test_field_errors_scaled_and_pointwise():
    ref = np.array([1.0, -2.0, 4.0, 1e-9, np.nan])
    got = np.array([1.0 + 1e-6, -2.0, 4.0 - 4e-6, 2e-9, np.nan])
    st = accuracy.field_errors([got], [ref], ["f"])["f"]
    assert st["points"] == 4 and st["nan_mismatch"] == 0
    assert np.isclose(st["max_field_scaled"], 4e-6 / 4.0)
    # the 1e-9 point is below the 1e-6 * max floor: it counts in the field-scaled error only
    assert st["rel_points"] == 3 and np.isclose(st["max_rel"], 1e-6)
    assert np.isclose(st["frac_rel_above_1e-5"], 0.0)
    loose = accuracy.field_errors([got], [ref], ["f"], floor=0.0)["f"]
    assert loose["rel_points"] == 4 and np.isclose(loose["max_rel"], 1.0)


def test_field_errors_nan_mismatch_and_worst():
    a = accuracy.field_errors([np.array([1.0, np.nan]), np.array([2.0, 3.0])],
                              [np.array([1.0, 1.0]), np.array([2.0, 3.0 + 3e-7])], ["a", "b"])
    assert a["a"]["nan_mismatch"] == 1 and a["b"]["nan_mismatch"] == 0
    # the NaN point is left out of the error and counted as a mismatch
    assert a["a"]["points"] == 1 and a["a"]["max_field_scaled"] == 0.0
    assert accuracy.worst(a, "max_field_scaled") == a["b"]["max_field_scaled"]
    assert accuracy.worst({"x": {"e": float("nan")}, "y": {"e": 1.0}}, "e") == float("inf")
