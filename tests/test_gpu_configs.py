"""The GPU path against the oracle and the compiled reference on the benchmark
plan's own configurations, at their stated sizes.

* Config 0 (64^3 dam break, 8 per cell, seed 0; 265,302 particles):
  the first FP64 step against the compiled reference with the MIC(0) solve,
  field by field (grid and sort bit-exact, transfers and grid update to
  1e-10 of each field's largest value and pointwise, pressure and everything
  after it to 1e-9); ten steps against the C oracle run live; and 100 steps
  against the oracle's committed digest (tests/golden/config0_dam64.npz).
* Config 1 (128^3 liquid sphere falling onto a 128 x 128-vertex sheet,
  dt 5e-4): the first step against the oracle -- liquid and sheet state --
  and 200 steps against the oracle's committed digest
  (tests/golden/config1_sheet128.npz).
* Config 2 (256^3 half box, 16.8M particles): a 64^3 replica of the same
  generator for three steps against the oracle run live, and the first
  full-size FP64 step against the oracle's committed digest
  (tests/golden/config2_half256.npz).

The per-step MIC(0) iteration counts match the oracle's within one."""
import os

import numpy as np
import pytest

from libwetcloth_b200 import scenes
from libwetcloth_b200.solver import FluidScene
from oracle import oracle as oo
from oracle import ref as oref
from tests.parity import assert_close, assert_dense_close, assert_pointwise
from tests.test_gpu_parity import P2G_FIELDS, PREDICT_FIELDS, pointwise_floor

pytestmark = pytest.mark.gpu

DT = 1e-3
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _stages(sc):
    """One sub-step through the stage calls, with every field the reference
    snapshots."""
    g = FluidScene(sc)
    out = {}
    g.rebucketize_and_resample()
    out["dims"], out["origin"], out["bbx"] = g.grid_info()
    for k in ["active", "array_idx", "array_sup", "stencil_base"]:
        out[k] = g.ifield(k)
    g.map_particle_nodes()
    for k in P2G_FIELDS:
        out[k] = g.field(k)
    g.step_velocity(DT)
    for k in PREDICT_FIELDS:
        out[k] = g.field(k)
    g.project_fine(DT)
    out["dof_index"] = g.ifield("dof_index")
    out["system"] = g.pressure_system()
    out["pressure"] = g.field("pressure")
    out["stats"] = g.stats()
    g.apply_pressure_drag_fluid(DT)
    for a in "xyz":
        out["valid_" + a] = g.ifield("valid_" + a)
    g.constrain_liquid_velocity()
    for a in "xyz":
        out["u_final_" + a] = g.field("u_" + a)
    g.correct_liquid_particles(DT)  # every sub-step (projection only at strength 0)
    g.map_node_particles()
    out["g2p_x"], out["g2p_v"], out["g2p_C"] = g.download()
    g.advect(DT)
    out["adv_x"], _, _ = g.download()
    g.close()
    return out


def test_config0_first_step_vs_reference(wcg):
    if not oref.available():
        pytest.skip("oracle/_ref not built")
    sc = scenes.dam_break(64, 8, 0)
    n = sc.x.shape[0]
    r = oref.RefScene(sc, mic=True)
    r.step(DT, snapshot=True)
    out = _stages(sc)
    assert np.array_equal(out["dims"], r.get("grid_dims"))
    assert np.array_equal(out["origin"], r.get("grid_origin"))
    for k in ["active", "array_idx", "array_sup", "stencil_base"]:
        assert np.array_equal(out[k], r.get(k)), k
    for k in P2G_FIELDS + PREDICT_FIELDS:
        assert_dense_close(out[k], r.get(k), 1e-10, k)
        assert_pointwise(out[k], r.get(k), 1e-10, k, pointwise_floor(k))
    assert np.array_equal(out["dof_index"], r.get("dof_index"))
    rs, col, val, rhs = out["system"]
    assert np.array_equal(rs, r.get("A_rowstart")) and np.array_equal(col, r.get("A_col"))
    assert_close(val, r.get("A_val"), 1e-10, "A values")
    assert_close(rhs, r.get("b"), 1e-10, "rhs")
    it_ref, _ = r.solver_stats()
    assert abs(out["stats"]["pcg_iters"] - it_ref) <= 1, (out["stats"]["pcg_iters"], it_ref)
    assert_dense_close(out["pressure"], r.get("pressure"), 1e-9, "pressure")
    assert_pointwise(out["pressure"], r.get("pressure"), 1e-6, "pressure", 1e-4)
    for a in "xyz":
        assert np.array_equal(out["valid_" + a], r.get("valid_" + a)), "valid_" + a
        assert_dense_close(out["u_final_" + a], r.get("u_final_" + a), 1e-9, "u_final_" + a)
    assert_close(out["g2p_v"], r.get("g2p_v").reshape(n, 3), 1e-9, "G2P velocity")
    assert_close(out["g2p_C"], r.get("g2p_C").reshape(n, 9), 1e-9, "G2P affine C")
    assert_close(out["adv_x"], r.get("adv_x").reshape(n, 3), 1e-12, "advected x")
    r.close()


def _state_close(x, v, C, ox, ov, oC, xtol, vtol, name):
    assert_close(x, ox, xtol, name + " x")
    assert_close(v, ov, vtol, name + " v")
    # C sums terms of size |v| 4/dx that cancel: measured against that size
    assert np.abs(C - oC).max() <= vtol * max(np.abs(oC).max(), np.abs(ov).max() * 4 * 64)


def test_config0_ten_steps_vs_oracle(wcg):
    sc = scenes.dam_break(64, 8, 0)
    n = sc.x.shape[0]
    o = oo.OracleScene(sc)
    g = FluidScene(sc)
    for k in range(10):
        o.step(DT, snapshot=(k == 9))
        g.step(DT)
        assert abs(g.stats()["pcg_iters"] - o.solver_stats()[0]) <= 1, k
    x, v, C = g.download()
    _state_close(x, v, C, o.get("adv_x").reshape(n, 3), o.get("g2p_v").reshape(n, 3),
                 o.get("g2p_C").reshape(n, 9), 1e-11, 1e-8, "10 steps")
    o.close()
    g.close()


def test_config0_hundred_steps_vs_oracle_digest(wcg):
    d = np.load(os.path.join(GOLDEN, "config0_dam64.npz"))
    sc = scenes.dam_break(64, 8, 0)
    assert sc.x.shape[0] == int(d["n"][0])
    idx = d["idx"]
    g = FluidScene(sc)
    iters = []
    for k in range(1, 101):
        g.step(DT)
        iters.append(g.stats()["pcg_iters"])
        if k in (10, 100):
            x, v, C = g.download()
            p = f"s{k}_"
            vtol = 1e-8 if k == 10 else 1e-6
            _state_close(x[idx], v[idx], C[idx], d[p + "x"], d[p + "v"], d[p + "C"],
                         1e-10 if k == 10 else 1e-8, vtol, f"{k} steps")
            vs = np.abs(d[p + "v_sum"]).max() + np.sqrt(d[p + "v_sq"][0])
            assert np.abs(v.sum(axis=0) - d[p + "v_sum"]).max() <= vtol * vs
            assert abs((v * v).sum() - d[p + "v_sq"][0]) <= vtol * d[p + "v_sq"][0]
            assert np.abs(x.sum(axis=0) - d[p + "x_sum"]).max() <= 1e-9 * np.abs(d[p + "x_sum"]).max()
    assert np.abs(np.array(iters) - d["iters"]).max() <= 1
    g.close()


def test_config1_first_step_vs_oracle(wcg):
    dt = 5e-4
    sc = scenes.liquid_on_sheet(128, 8, 3, sheet_spacing=0.8 / 127)
    assert sc.elasto.n == 128 * 128
    o = oo.OracleScene(sc)
    g = FluidScene(sc)
    assert g.num_substeps(dt) == o.num_substeps(dt)
    o.step(dt, snapshot=True)
    g.step(dt)
    assert abs(g.stats()["pcg_iters"] - o.solver_stats()[0]) <= 1
    ne = sc.elasto.n
    x, v, C = g.download()
    ov = o.get("g2p_v").reshape(-1, 3)[ne:]
    _state_close(x, v, C, o.get("adv_x").reshape(-1, 3)[ne:], ov,
                 o.get("g2p_C").reshape(-1, 9)[ne:], 1e-12, 1e-9, "liquid")
    x4, v4, B = g.download_elasto()
    assert_close(x4, o.get("adv_x4").reshape(-1, 4)[:ne], 1e-12, "sheet x")
    assert_close(v4, o.get("adv_ev4").reshape(-1, 4)[:ne], 1e-9, "sheet v")
    o.close()
    g.close()


def test_config1_two_hundred_steps_vs_oracle_digest(wcg):
    """Config 1 for its stated 200 steps (dt 5e-4) against the oracle's
    committed digest (tests/golden/config1_sheet128.npz): the liquid sample,
    sums and norms after 20 and 200 steps, the sheet's positions and
    velocities at a sample of its vertices and summed over all of them, and
    the MIC(0) iteration count of every step (within one)."""
    dt = 5e-4
    d = np.load(os.path.join(GOLDEN, "config1_sheet128.npz"))
    sc = scenes.liquid_on_sheet(128, 8, 3, sheet_spacing=0.8 / 127)
    ne = sc.elasto.n
    assert sc.x.shape[0] == int(d["n"][0]) and ne == int(d["ne"][0])
    idx, sidx = d["idx"], d["sheet_idx"]
    g = FluidScene(sc)
    iters = []
    for k in range(1, 201):
        g.step(dt)
        iters.append(g.stats()["pcg_iters"])
        if k in (20, 200):
            x, v, C = g.download()
            p = f"s{k}_"
            xtol, vtol = (1e-10, 1e-8) if k == 20 else (1e-8, 1e-6)
            _state_close(x[idx], v[idx], C[idx], d[p + "x"], d[p + "v"], d[p + "C"], xtol, vtol,
                         f"{k} steps")
            vs = np.abs(d[p + "v_sum"]).max() + np.sqrt(d[p + "v_sq"][0])
            assert np.abs(v.sum(axis=0) - d[p + "v_sum"]).max() <= vtol * vs
            assert abs((v * v).sum() - d[p + "v_sq"][0]) <= vtol * d[p + "v_sq"][0]
            x4, v4, _ = g.download_elasto()
            assert_close(x4[sidx], d[p + "sheet_x4"], xtol, f"sheet x, {k} steps")
            assert_close(v4[sidx], d[p + "sheet_v4"], vtol, f"sheet v, {k} steps")
            xs = np.abs(d[p + "sheet_x4_sum"]).max()
            assert np.abs(x4.sum(axis=0) - d[p + "sheet_x4_sum"]).max() <= xtol * xs
            vs = np.abs(d[p + "sheet_v4_sum"]).max() + np.sqrt(d[p + "sheet_v4_sq"][0])
            assert np.abs(v4.sum(axis=0) - d[p + "sheet_v4_sum"]).max() <= vtol * vs
    assert np.abs(np.array(iters) - d["iters"]).max() <= 1
    g.close()


def test_config2_replica_three_steps_vs_oracle(wcg):
    sc = scenes.half_box(64, 2, seed=1)
    n = sc.x.shape[0]
    o = oo.OracleScene(sc)
    g = FluidScene(sc)
    for k in range(3):
        o.step(DT, snapshot=(k == 2))
        g.step(DT)
        assert abs(g.stats()["pcg_iters"] - o.solver_stats()[0]) <= 1, k
    x, v, C = g.download()
    _state_close(x, v, C, o.get("adv_x").reshape(n, 3), o.get("g2p_v").reshape(n, 3),
                 o.get("g2p_C").reshape(n, 9), 1e-11, 1e-8, "3 steps")
    o.close()
    g.close()


def test_config2_full_size_first_step_vs_oracle_digest(wcg):
    path = os.path.join(GOLDEN, "config2_half256.npz")
    d = np.load(path)
    sc = scenes.half_box(256, 2, seed=1)
    assert sc.x.shape[0] == int(d["n"][0])
    idx = d["idx"]
    g = FluidScene(sc)
    g.step(DT)
    assert abs(g.stats()["pcg_iters"] - int(d["iters"][0])) <= 1
    x, v, C = g.download()
    g.close()
    _state_close(x[idx], v[idx], C[idx], d["s1_x"], d["s1_v"], d["s1_C"], 1e-12, 1e-9,
                 "256^3 step")
    vs = np.abs(d["s1_v_sum"]).max() + np.sqrt(d["s1_v_sq"][0])
    assert np.abs(v.sum(axis=0) - d["s1_v_sum"]).max() <= 1e-9 * vs
    assert abs((v * v).sum() - d["s1_v_sq"][0]) <= 1e-9 * d["s1_v_sq"][0]
