"""The pressure solve in the pencil layout against the tile wavefront.

Both layouts run the same MIC(0)-PCG arithmetic (the order of the three
lower-neighbour terms and the products sent across patch edges can round
differently), so pressures agree to 1e-10 relative to their maximum in FP64
and iteration counts agree to one.  The scenes cover each axis as the stream
axis and boxes spanning several patches along both cut axes (patch edges and
the tagged edge words between patches)."""
import os

import numpy as np
import pytest

from libwetcloth_b200 import _capi, scenes
from libwetcloth_b200.solver import FluidScene

pytestmark = pytest.mark.gpu
DT = 1e-3


def _scene(kind):
    if kind == "dam16_y":
        return scenes.dam_break(16, 8, 0)
    if kind == "slab64_x":
        return scenes.dam_break(64, 2, 3, block_hi=(0.9, 0.3, 0.6))
    if kind == "slab48_z":
        return scenes.dam_break(48, 2, 4, block_hi=(0.5, 0.3, 0.95))
    if kind == "curl48":
        return scenes.half_box(48, 2, 5, amplitude=0.5, sigma_cells=2.0)
    if kind == "curl96":  # 6 patches along c: several cluster columns
        return scenes.half_box(96, 2, 6, amplitude=0.5, sigma_cells=3.0)
    raise ValueError(kind)


def _solve(sc, layout, precision, cluster=1):
    cc, ca = (str(cluster).split("x") + ["1"])[:2] if "x" in str(cluster) else (str(cluster), "1")
    env = {"WCG_PCG_LAYOUT": layout, "WCG_SWEEP_CLUSTER": cc, "WCG_SWEEP_CLUSTER_A": ca}
    old = {k: os.environ.get(k) for k in env}
    os.environ.update(env)
    try:
        g = FluidScene(sc, precision=precision)
    finally:
        for k, v in old.items():
            if v is None:
                del os.environ[k]
            else:
                os.environ[k] = v
    g.rebucketize_and_resample()
    g.map_particle_nodes()
    g.step_velocity(DT)
    g.project_fine(DT)
    p = g.field("pressure")
    st = g.stats()
    g.close()
    return p, st


@pytest.mark.parametrize("kind", ["dam16_y", "slab64_x", "slab48_z", "curl48"])
def test_pencil_matches_tiles_fp64(kind, wcg):
    sc = _scene(kind)
    p_pl, st_pl = _solve(sc, "pencil", _capi.WCG_FP64)
    p_t, st_t = _solve(sc, "tiles", _capi.WCG_FP64)
    assert st_pl["converged"] == 1 and st_t["converged"] == 1
    assert abs(st_pl["pcg_iters"] - st_t["pcg_iters"]) <= 1, (st_pl, st_t)
    m = ~np.isnan(p_t)
    assert np.array_equal(m, ~np.isnan(p_pl))
    scale = np.abs(p_t[m]).max()
    assert np.abs(p_pl[m] - p_t[m]).max() <= 1e-10 * scale
    assert st_pl["residual"] <= sc.params.criterion * st_pl["rhs_norm"]


@pytest.mark.parametrize("kind", ["slab64_x", "curl48"])
def test_pencil_matches_tiles_fp32_refine(kind, wcg):
    sc = _scene(kind)
    p_pl, st_pl = _solve(sc, "pencil", _capi.WCG_FP32_REFINE)
    p_t, st_t = _solve(sc, "tiles", _capi.WCG_FP32_REFINE)
    assert st_pl["converged"] == 1 and st_t["converged"] == 1
    m = ~np.isnan(p_t)
    scale = np.abs(p_t[m]).max()
    assert np.abs(p_pl[m] - p_t[m]).max() <= 1e-5 * scale
    assert st_pl["residual"] <= sc.params.criterion * st_pl["rhs_norm"]


def test_pencil_deterministic(wcg):
    sc = _scene("curl48")
    a, sa = _solve(sc, "pencil", _capi.WCG_FP32_REFINE)
    b, sb = _solve(sc, "pencil", _capi.WCG_FP32_REFINE)
    assert sa["pcg_iters"] == sb["pcg_iters"]
    m = ~np.isnan(a)
    assert np.array_equal(a[m], b[m])


@pytest.mark.parametrize("precision", [_capi.WCG_FP32_REFINE, _capi.WCG_FP64])
def test_pencil_deterministic_256_patches(precision, wcg):
    """The 256^3 half box (256 patches, more than the SMs hold at one CTA
    each): three solves of the same system give the same pressures and
    iteration counts bit for bit."""
    sc = scenes.half_box(256, 2, seed=1)
    res = []
    for _ in range(3):
        g = FluidScene(sc, precision=precision)
        g.set_correction_count(0)
        g.rebucketize_and_resample()
        g.map_particle_nodes()
        g.step_velocity(DT)
        g.project_fine(DT)
        st = g.stats()
        res.append((np.nan_to_num(g.field("pressure")), st["pcg_iters"], st["refinements"]))
        g.close()
    for p, it, rf in res[1:]:
        assert it == res[0][1] and rf == res[0][2]
        assert np.array_equal(p, res[0][0])


@pytest.mark.parametrize("cluster", [2, 4, 8, 16, "1x4", "2x4", "4x4", "1x8", "2x8"])
@pytest.mark.parametrize("kind,precision", [("curl48", _capi.WCG_FP64),
                                            ("slab64_x", _capi.WCG_FP64),
                                            ("curl96", _capi.WCG_FP64),
                                            ("curl48", _capi.WCG_FP32_REFINE)])
def test_pencil_cluster_sweeps_bit_identical(kind, precision, cluster, wcg):
    """Clusters only change how edge values travel (shared memory of the
    neighbouring CTA instead of a global round trip): c-faces with clusters
    along c ("8"), both faces with 2-D clusters ("CCxCA": CC c-patches by CA
    a-patches).  The arithmetic is the same, so pressures and iteration
    counts are bit-identical, also when the patch counts are not multiples
    of the cluster extents."""
    sc = _scene(kind)
    a, sa = _solve(sc, "pencil", precision, 1)
    b, sb = _solve(sc, "pencil", precision, cluster)
    assert sb["converged"] == 1
    assert sa["pcg_iters"] == sb["pcg_iters"] and sa["refinements"] == sb["refinements"]
    m = ~np.isnan(a)
    assert np.array_equal(m, ~np.isnan(b))
    assert np.array_equal(a[m], b[m])
