"""Comparison helpers shared by the parity tests."""
import numpy as np


def assert_dense_close(gpu, ref, rtol, name, atol_abs=0.0, mask=None):
    """Dense bucket-major node fields: NaN marks inactive buckets in both.
    Values must agree within atol_abs + rtol * max|ref| over active nodes."""
    g = np.asarray(gpu, dtype=np.float64)
    r = np.asarray(ref, dtype=np.float64)
    assert g.shape == r.shape, f"{name}: shape {g.shape} vs {r.shape}"
    gn, rn = np.isnan(g), np.isnan(r)
    assert np.array_equal(gn, rn), f"{name}: active-node sets differ ({gn.sum()} vs {rn.sum()} NaN)"
    keep = ~rn if mask is None else (~rn & mask)
    if not keep.any():
        return 0.0
    scale = max(np.abs(r[keep]).max(), 1e-300)
    err = np.abs(g[keep] - r[keep]).max()
    assert err <= atol_abs + rtol * scale, (
        f"{name}: max abs err {err:.3e} > {atol_abs:.1e} + {rtol:.1e} * {scale:.3e}")
    return err / scale


def assert_close(gpu, ref, rtol, name, atol_abs=0.0):
    g = np.asarray(gpu, dtype=np.float64)
    r = np.asarray(ref, dtype=np.float64)
    assert g.shape == r.shape, f"{name}: shape {g.shape} vs {r.shape}"
    if r.size == 0:
        return 0.0
    scale = max(np.abs(r).max(), 1e-300)
    err = np.abs(g - r).max()
    assert err <= atol_abs + rtol * scale, (
        f"{name}: max abs err {err:.3e} > {atol_abs:.1e} + {rtol:.1e} * {scale:.3e}")
    return err / scale


def assert_pointwise(gpu, ref, rtol, name, floor_rel):
    """Pointwise relative agreement where the reference is not small: every
    finite entry with |ref| >= floor_rel * max|ref| must satisfy
    |gpu - ref| <= rtol * |ref|.  Complements the max-normalised checks, which
    a field with a wide dynamic range could pass while its small entries are
    wrong.  Returns the largest pointwise relative error over those entries."""
    g = np.asarray(gpu, dtype=np.float64).reshape(-1)
    r = np.asarray(ref, dtype=np.float64).reshape(-1)
    assert g.shape == r.shape, f"{name}: shape {g.shape} vs {r.shape}"
    fin = np.isfinite(r)
    assert np.array_equal(fin, np.isfinite(g)), f"{name}: finite-entry sets differ"
    if not fin.any():
        return 0.0
    a = np.abs(r[fin])
    if a.max() == 0:
        return 0.0
    keep = a >= floor_rel * a.max()
    rel = np.abs(g[fin][keep] - r[fin][keep]) / a[keep]
    worst = float(rel.max())
    k = int(np.argmax(rel))
    assert worst <= rtol, (f"{name}: pointwise relative error {worst:.3e} > {rtol:.1e} at "
                           f"|ref| = {a[keep][k]:.3e} (floor {floor_rel:.0e} x max {a.max():.3e}, "
                           f"{int(keep.sum())} entries checked)")
    return worst


# Rotated terminator objects of the four analytic types in three distance-field
# groups, for the terminator tests (scenes in the unit box, liquid below y = 0.5).
TERMINATOR_SHAPES = [
    {"type": "sphere", "inside": False, "center": (0.5, 0.3, 0.5), "param": (0.12, 0, 0, 0),
     "group": 1},
    {"type": "capsule", "inside": False, "center": (0.3, 0.2, 0.6), "axis": (0.0, 0.0, 1.0),
     "angle": 0.7, "param": (0.06, 0.15, 0, 0), "group": 1},
    {"type": "cylinder", "inside": False, "center": (0.7, 0.25, 0.3), "axis": (1.0, 0.0, 0.0),
     "angle": 0.4, "param": (0.1, 0.02, 0.08, 0), "group": 2},
    {"type": "box", "inside": True, "center": (0.5, 0.5, 0.5), "axis": (0.0, 1.0, 0.0),
     "angle": 0.3, "param": (0.45, 0.45, 0.45, 0.01), "group": 3},
]

