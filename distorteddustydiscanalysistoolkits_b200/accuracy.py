"""Error statistics of interpolated fields against a reference evaluation of the same fields.

Two measures per field, both over the points where neither value is NaN (a NaN in one field
and not in the other is counted as a ``nan_mismatch``):
  field-scaled   |got - ref| / max|ref|  (the error relative to the field's magnitude);
  pointwise      |got - ref| / |ref| over the points with |ref| >= floor * max|ref|
                 (the relative error of each value; the floor leaves out the neighbourhood of
                 the field's zero crossings, where a relative error has no meaning).
Used for the FP32-compensated mode against the FP64 mode or the CPU oracle.
"""
import numpy as np

POINTWISE_FLOOR = 1e-6


def field_errors(got, ref, names=None, floor=POINTWISE_FLOOR):
    """Per-field dict of max/RMS field-scaled and pointwise relative errors.  ``got`` and
    ``ref`` are sequences of equally long 1-D arrays (one per field); NaN positions must agree
    (a mismatch is reported as ``nan_mismatch``)."""
    out = {}
    names = names if names is not None else [str(i) for i in range(len(ref))]
    for name, a, r in zip(names, got, ref):
        a = np.asarray(a, np.float64)
        r = np.asarray(r, np.float64)
        ok = ~np.isnan(r) & ~np.isnan(a)
        e = {"nan_mismatch": int(np.count_nonzero(np.isnan(a) != np.isnan(r))), "points": int(ok.sum())}
        if ok.any():
            sc = float(np.max(np.abs(r[ok])))
            d = np.abs(a[ok] - r[ok])
            fs = d / sc if sc > 0 else d
            e["max_field_scaled"] = float(fs.max())
            e["rms_field_scaled"] = float(np.sqrt(np.mean(fs ** 2)))
            keep = np.abs(r[ok]) >= floor * sc
            if keep.any():
                rel = d[keep] / np.abs(r[ok][keep])
                e["max_rel"] = float(rel.max())
                e["rms_rel"] = float(np.sqrt(np.mean(rel ** 2)))
                e["frac_rel_above_1e-5"] = float(np.mean(rel > 1e-5))
            e["rel_floor"] = floor
            e["rel_points"] = int(keep.sum())
        out[name] = e
    return out


def worst(stats, key):
    """Largest value of ``key`` over the fields of a field_errors result (0 if absent; a NaN
    value counts as infinite, so it is never hidden by the order of the fields)."""
    vals = [v.get(key, 0.0) for v in stats.values()]
    return max((float("inf") if v != v else v for v in vals), default=0.0)
