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
