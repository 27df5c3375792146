"""GPU path against the golden fixtures of the compiled reference, plus edge
cases: empty scenes, CFL sub-stepping, solver non-convergence, invalid input,
run-to-run determinism."""
import os

import numpy as np
import pytest

from libwetcloth_b200 import _capi, scenes
from libwetcloth_b200.solver import FluidScene
from oracle import oracle as oo
from tests.golden.make_golden import NODE_FIELDS

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
DT = 1e-3


@pytest.mark.parametrize("name", ["golden_dam", "golden_curl"])
def test_golden_fixture(name, wcg):
    d = np.load(os.path.join(HERE, "golden", name + ".npz"))
    sc = scenes.Scene(scenes.SceneParams(dx=float(d["dx"][0])), d["x"], d["v"], d["mass"],
                      d["vol"], d["radius"], name=name)
    g = FluidScene(sc)
    g.rebucketize_and_resample()
    assert np.array_equal(g.ifield("array_idx"), d["array_idx"])
    assert np.array_equal(g.ifield("active"), d["active"])
    assert np.array_equal(g.ifield("stencil_base"), d["stencil_base"])
    act = np.repeat(d["active"].astype(bool), 64)
    g.map_particle_nodes()
    g.step_velocity(DT)
    g.project_fine(DT)
    assert np.array_equal(g.ifield("dof_index"), d["dof_index"])
    assert abs(g.stats()["pcg_iters"] - int(d["pcg_iters"][0])) <= 1
    got = {"pressure": g.field("pressure")}
    for k in ("mass_fluid_x", "vol_fluid_y", "liquid_phi", "solid_weight_z", "v_star_y"):
        got[k] = g.field(k)
    g.apply_pressure_drag_fluid(DT)
    g.constrain_liquid_velocity()
    for a in "xyz":
        got["u_final_" + a] = g.field("u_" + a)
    for k, v in got.items():
        ref = d["node_" + k]
        tol = 1e-9 if k in ("pressure",) or k.startswith("u_final") else 1e-10
        assert np.abs(v[act] - ref).max() <= tol * np.abs(ref).max(), k
    g.correct_liquid_particles(DT)  # every sub-step (projection only at strength 0)
    g.map_node_particles()
    g.advect(DT)
    g.step(DT)
    g.step(DT)
    x, v, C = g.download()
    for k, a in (("step3_x", x), ("step3_v", v), ("step3_C", C)):
        ref = d[k].reshape(a.shape)
        assert np.abs(a - ref).max() <= 1e-8 * np.abs(ref).max(), k
    g.close()


def test_empty_scene(wcg):
    sc = scenes.dam_break(16, 8, 0)
    e = scenes.Scene(sc.params, np.zeros((0, 3)), np.zeros((0, 3)), np.zeros(0), np.zeros(0),
                     np.zeros(0))
    g = FluidScene(e)
    assert g.step(DT) == 1
    x, v, C = g.download()
    assert x.shape == (0, 3)
    g.close()


def test_cfl_substeps_match_oracle(wcg):
    sc = scenes.dam_break(16, 8, 1, block_hi=(0.3, 0.4, 0.3))
    sc.v[:] = np.array([0.0, -250.0, 0.0])  # 3 CFL at dx=1/16 allows 187.5 m/s: two sub-steps
    o = oo.OracleScene(sc)
    g = FluidScene(sc)
    assert g.num_substeps(DT) == 2
    assert g.step(DT) == 2
    assert o.step(DT, snapshot=True) == 2
    x, v, C = g.download()
    n = sc.x.shape[0]
    ov = o.get("g2p_v").reshape(n, 3)
    assert np.abs(v - ov).max() <= 1e-9 * np.abs(ov).max()
    assert np.abs(x - o.get("adv_x").reshape(n, 3)).max() <= 1e-12
    g.close()


def test_nonconvergence_is_reported(wcg):
    sc = scenes.dam_break(16, 8, 0)
    sc.params.maxiters = 1
    g = FluidScene(sc)
    g.rebucketize_and_resample()
    g.map_particle_nodes()
    g.step_velocity(DT)
    with pytest.raises(_capi.WcgError) as ei:
        g.project_fine(DT)
    assert ei.value.code == _capi.WCG_ERR_NOT_CONVERGED
    st = g.stats()
    assert st["converged"] == 0 and st["pcg_iters"] == 1
    g.close()


def test_invalid_particles_rejected(wcg):
    sc = scenes.dam_break(16, 8, 0)
    sc.x[3, 1] = np.nan
    with pytest.raises(_capi.WcgError) as ei:
        FluidScene(sc)
    assert ei.value.code == _capi.WCG_ERR_ARG
    sc = scenes.dam_break(16, 8, 0)
    sc.mass[0] = -1.0
    with pytest.raises(_capi.WcgError):
        FluidScene(sc)


def test_calls_out_of_order_rejected(wcg):
    sc = scenes.dam_break(16, 8, 0)
    g = FluidScene(sc)
    with pytest.raises(_capi.WcgError) as ei:
        g.project_fine(DT)
    assert ei.value.code == _capi.WCG_ERR_STATE
    g.close()


@pytest.mark.parametrize("precision", [_capi.WCG_FP64, _capi.WCG_FP32_REFINE])
def test_run_to_run_determinism(precision, wcg):
    sc = scenes.half_box(32, 2, 5, amplitude=0.5, sigma_cells=2.0)
    res = []
    for _ in range(2):
        g = FluidScene(sc, precision=precision)
        g.step(DT)
        g.step(DT)
        res.append(g.download())
        g.close()
    for a, b in zip(res[0], res[1]):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("precision", [_capi.WCG_FP64, _capi.WCG_FP32_REFINE])
def test_wavefront_wait_limit_reached(precision, wcg):
    """The wavefront's bounded waits, run out on purpose: the last patch of
    the pencil layout waits for an edge-word tag no producer writes, with a
    limit of 200 polls.  The solve comes back (no hang) with WCG_ERR_DEVICE
    naming the wait limit, as the reference's PCGSolver::solve would return
    false; after the hook is cleared the same context steps again and matches
    a fresh context bit for bit."""
    sc = scenes.half_box(48, 2, 5, amplitude=0.5, sigma_cells=2.0)  # several patches
    g = FluidScene(sc, precision=precision)
    L = g.L
    _capi.check(L.wcg_set_wait_limit(g.h, 200, 1 << 30))
    g.rebucketize_and_resample()
    g.map_particle_nodes()
    g.step_velocity(1e-3)
    with pytest.raises(_capi.WcgError) as e:
        g.project_fine(1e-3)
    assert e.value.code == _capi.WCG_ERR_DEVICE
    assert "wait limit" in str(e.value)
    # back to the default limit and no stale patch: the context works
    _capi.check(L.wcg_set_wait_limit(g.h, 1 << 20, -1))
    g.upload(sc.x, sc.v, sc.C, sc.mass, sc.vol, sc.radius)
    g.step(1e-3)
    x, v, C = g.download()
    h = FluidScene(sc, precision=precision)
    h.step(1e-3)
    x2, v2, C2 = h.download()
    assert np.array_equal(x, x2) and np.array_equal(v, v2) and np.array_equal(C, C2)
    assert L.wcg_set_wait_limit(g.h, 0, -1) == _capi.WCG_ERR_ARG
    g.close()
    h.close()
