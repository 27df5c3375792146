"""Particle correction (correctLiquidParticles) and the solid projection after
advection (solidProjection) on the GPU against the oracle.

The oracle's restatements of both are pinned to the reference in
tests/test_oracle_vs_reference.py (test_solid_projection,
test_particle_correction).  Here the GPU runs the same scenes through the
C-ABI: stage by stage with an explicit particle subset, and whole steps with
the seeded subset stream both sides share.  FP64 agrees to 1e-10 relative
(velocities, affine matrices against the size of their terms) and 1e-12 on
positions; FP32 with FP64 refinement to 1e-5 and 1e-6."""
import numpy as np
import pytest

from libwetcloth_b200 import _capi, scenes
from libwetcloth_b200.solver import FluidScene
from oracle import oracle as oo

pytestmark = pytest.mark.gpu
DT = 1e-3


def _close(a, b, tol, name, scale=0.0):
    a = np.asarray(a).reshape(-1)
    b = np.asarray(b).reshape(-1)
    s = max(np.abs(b).max(), scale, 1e-300)
    err = np.abs(a - b).max() / s
    assert err <= tol, f"{name}: {err:.3e}"


def _fall(n=16, vy=-3.0):
    sc = scenes.dam_break(n, 8, 0)
    sc.v[:, 1] = vy
    return sc


def _scene(kind, strength=0.2, seed=3):
    if kind == "dam16":
        sc = scenes.dam_break(16, 8, 0)
    elif kind == "curl16":
        sc = scenes.half_box(16, 2, 7, amplitude=1.0, sigma_cells=1.5)
    elif kind == "fall":
        sc = _fall()
    else:
        raise ValueError(kind)
    sc.params.correction_strength = strength
    sc.params.correction_seed = seed
    return sc


@pytest.mark.parametrize("dt", [1e-3, 2e-2])
def test_solid_projection_step_fp64(dt, wcg):
    sc = _fall()
    o = oo.OracleScene(sc)
    n = o.step(dt, snapshot=True)
    assert o.get("projected")[0] > 0
    g = FluidScene(sc)
    g.step(dt)
    assert g.stats()["substeps"] == n
    x, v, C = g.download()
    _close(v, o.get("g2p_v"), 1e-10, "g2p_v")
    _close(x, o.get("adv_x"), 1e-12, "adv_x")
    g.close()


def test_solid_projection_separate_advect(wcg):
    """wcg_map_node_particles then wcg_advect: the advection projects too."""
    sc = _fall()
    o = oo.OracleScene(sc)
    o.step(DT, snapshot=True)
    g = FluidScene(sc)
    g.rebucketize_and_resample()
    g.map_particle_nodes()
    g.step_velocity(DT)
    g.project_fine(DT)
    g.apply_pressure_drag_fluid(DT)
    g.constrain_liquid_velocity()
    g.correct_liquid_particles(DT)  # every sub-step (projection only at strength 0)
    g.map_node_particles()
    g.advect(DT)
    _close(g.download()[0], o.get("adv_x"), 1e-12, "adv_x")
    g.close()


@pytest.mark.parametrize("kind,sel", [("dam16", 2), ("curl16", 5), ("fall", 0)])
def test_correction_stages_fp64(kind, sel, wcg):
    sc = _scene(kind)
    o = oo.OracleScene(sc)
    o.set_correction_selector(sel)
    o.step(DT, snapshot=True)
    g = FluidScene(sc)
    g.rebucketize_and_resample()
    g.map_particle_nodes()
    g.step_velocity(DT)
    g.project_fine(DT)
    g.apply_pressure_drag_fluid(DT)
    g.constrain_liquid_velocity()
    g.correct_liquid_particles(DT, sel)
    xc = g.download()[0]
    moved = np.abs(xc - sc.x).max(axis=1) > 0
    assert moved.any()
    assert np.all(np.arange(sc.x.shape[0])[moved] % sc.params.correction_step == sel)
    _close(xc, o.get("corr_x"), 1e-12, "corr_x")
    g.map_node_particles()
    x, v, C = g.download()
    ov = o.get("g2p_v")
    _close(v, ov, 1e-10, "g2p_v")
    _close(C, o.get("g2p_C"), 1e-10, "g2p_C", np.abs(ov).max() * 4.0 / sc.params.dx)
    g.advect(DT)
    _close(g.download()[0], o.get("adv_x"), 1e-12, "adv_x")
    g.close()


def test_correction_coincident_pairs(wcg):
    """Pairs closer than 1e-4 re are pushed apart by the seeded hash of their
    indices (scalarRand in the reference)."""
    sc = _scene("dam16")
    sel = 1
    idx = np.arange(sc.x.shape[0])
    first = idx[(idx % 8 == sel)][:40]
    sc.x[first + 1] = sc.x[first]
    o = oo.OracleScene(sc)
    o.set_correction_selector(sel)
    o.step(DT, snapshot=True)
    g = FluidScene(sc)
    g.rebucketize_and_resample()
    g.map_particle_nodes()
    g.step_velocity(DT)
    g.project_fine(DT)
    g.apply_pressure_drag_fluid(DT)
    g.constrain_liquid_velocity()
    g.correct_liquid_particles(DT, sel)
    xc = g.download()[0]
    assert np.all(np.abs(xc[first] - sc.x[first]).max(axis=1) > 0)
    _close(xc, o.get("corr_x"), 1e-12, "corr_x")
    g.close()


@pytest.mark.parametrize("kind", ["dam16", "curl16"])
def test_correction_seeded_steps_fp64(kind, wcg):
    """Whole steps with the correction on: both sides draw the subset of
    sub-step k from the same seeded stream (wcg_correction_selector)."""
    sc = _scene(kind, seed=7)
    o = oo.OracleScene(sc)
    g = FluidScene(sc)
    L = _capi.load()
    k = 0
    for _ in range(3):
        n = o.step(DT, snapshot=True)
        g.step(DT)
        k += n
    assert int(o.get("correction_selector")[0]) == L.wcg_correction_selector(7, k - 1, 8)
    x, v, C = g.download()
    _close(v, o.get("g2p_v"), 1e-10, "g2p_v")
    _close(x, o.get("adv_x"), 1e-12, "adv_x")
    g.close()


def test_correction_fp32(wcg):
    sc = _scene("curl16", seed=9)
    o = oo.OracleScene(sc)
    o.step(DT, snapshot=True)
    g = FluidScene(sc, precision=_capi.WCG_FP32_REFINE)
    g.step(DT)
    x, v, C = g.download()
    _close(v, o.get("g2p_v"), 1e-5, "g2p_v")
    _close(x, o.get("adv_x"), 1e-6, "adv_x")
    g.close()


def test_correction_args(wcg):
    sc = _scene("dam16")
    g = FluidScene(sc)
    g.rebucketize_and_resample()
    g.map_particle_nodes()
    with pytest.raises(_capi.WcgError) as e:
        g.correct_liquid_particles(DT, 8)
    assert e.value.code == _capi.WCG_ERR_ARG
    g.close()
