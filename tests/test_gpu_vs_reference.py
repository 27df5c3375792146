"""GPU FP64 path against the compiled reference Core, stage by stage.

The reference (oracle/_ref, built from the libWetCloth sources) runs one
sub-step of the fluid hot path on the same seeded scene and snapshots every
field; the GPU runs the same sub-step through the C-ABI stage calls.
Tolerances: integer/index data bit-exact; FP64 fields within 1e-10 relative
to the field's max magnitude (the solver-dependent pressures and everything
after them within 1e-9, since PCG iterates accumulate rounding differently).
"""
import numpy as np
import pytest

from oracle import ref as oref
from libwetcloth_b200 import scenes
from libwetcloth_b200.solver import FluidScene
from tests.parity import assert_close, assert_dense_close

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not oref.available(), reason="oracle/_ref not built")]

DT = 1e-3

P2G_FIELDS = ["mass_fluid_x", "mass_fluid_y", "mass_fluid_z", "vel_fluid_x",
              "vel_fluid_y", "vel_fluid_z", "vol_fluid_x", "vol_fluid_y",
              "vol_fluid_z", "sat_x", "sat_y", "sat_z", "psi_x", "psi_y", "psi_z",
              "sat_p", "psi_p", "pore_pressure_p", "liquid_phi", "solid_phi",
              "solid_weight_x", "solid_weight_y", "solid_weight_z",
              "solid_vel_x", "solid_vel_y", "solid_vel_z"]
PREDICT_FIELDS = ["v_star_x", "v_star_y", "v_star_z", "rhs_fluid_x",
                  "rhs_fluid_y", "rhs_fluid_z", "inv_C_x", "inv_C_y", "inv_C_z",
                  "psi_fs_x", "psi_fs_y", "psi_fs_z"]


def _scene(kind):
    if kind == "dam16":
        return scenes.dam_break(16, 8, 0)
    if kind == "dam32":
        return scenes.dam_break(32, 8, 3)
    if kind == "curl32":
        return scenes.half_box(32, 2, 5, amplitude=0.5, sigma_cells=2.0)
    raise ValueError(kind)


@pytest.fixture(scope="module", params=["dam16", "curl32"])
def pair(request, wcg):
    sc = _scene(request.param)
    r = oref.RefScene(sc, mic=True)
    r.step(DT, snapshot=True)
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
        out["u_proj_" + a] = g.field("u_" + a)
        out["valid_" + a] = g.ifield("valid_" + a)
    g.constrain_liquid_velocity()
    for a in "xyz":
        out["u_final_" + a] = g.field("u_" + a)
    g.map_node_particles()
    out["g2p_x"], out["g2p_v"], out["g2p_C"] = g.download()
    g.advect(DT)
    out["adv_x"], _, _ = g.download()
    yield sc, r, out
    g.close()
    r.close()


def test_grid_and_sort_bit_exact(pair):
    sc, r, out = pair
    assert np.array_equal(out["dims"], r.get("grid_dims"))
    assert np.array_equal(out["origin"], r.get("grid_origin"))
    assert np.array_equal(out["bbx"], r.get("bbx"))
    assert np.array_equal(out["active"], r.get("active")), "bucket activation differs"
    assert np.array_equal(out["array_idx"], r.get("array_idx")), "sorted keys differ"
    assert np.array_equal(out["array_sup"], r.get("array_sup")), "bucket ranges differ"
    assert np.array_equal(out["stencil_base"], r.get("stencil_base")), "stencil indices differ"


def test_p2g_fields(pair):
    sc, r, out = pair
    for k in P2G_FIELDS:
        assert_dense_close(out[k], r.get(k), 1e-10, k)


def test_predict_fields(pair):
    sc, r, out = pair
    for k in PREDICT_FIELDS:
        assert_dense_close(out[k], r.get(k), 1e-10, k)


def test_pressure_system(pair):
    sc, r, out = pair
    assert np.array_equal(out["dof_index"], r.get("dof_index")), "DOF numbering differs"
    rs, col, val, rhs = out["system"]
    assert np.array_equal(rs, r.get("A_rowstart")), "row structure differs"
    assert np.array_equal(col, r.get("A_col")), "column structure differs"
    assert_close(val, r.get("A_val"), 1e-10, "A values")
    assert_close(rhs, r.get("b"), 1e-10, "rhs")


def test_pressure_mic_pcg(pair):
    sc, r, out = pair
    it_ref, res_ref = r.solver_stats()
    st = out["stats"]
    assert abs(st["pcg_iters"] - it_ref) <= 1, (st["pcg_iters"], it_ref)
    assert st["converged"] == 1
    assert_dense_close(out["pressure"], r.get("pressure"), 1e-9, "pressure")


def test_projection_and_constraint(pair):
    sc, r, out = pair
    for a in "xyz":
        assert np.array_equal(out["valid_" + a], r.get("valid_" + a)), "valid_" + a
        assert_dense_close(out["u_proj_" + a], r.get("u_proj_" + a), 1e-9, "u_proj_" + a)
        assert_dense_close(out["u_final_" + a], r.get("u_final_" + a), 1e-9, "u_final_" + a)


def test_g2p_and_advect(pair):
    sc, r, out = pair
    n = sc.x.shape[0]
    assert_close(out["g2p_v"], r.get("g2p_v").reshape(n, 3), 1e-9, "G2P velocity")
    assert_close(out["g2p_C"], r.get("g2p_C").reshape(n, 9), 1e-9, "G2P affine C")
    assert_close(out["adv_x"], r.get("adv_x").reshape(n, 3), 1e-12, "advected x")


def test_multi_step_state(wcg):
    sc = _scene("dam16")
    r = oref.RefScene(sc, mic=True)
    g = FluidScene(sc)
    for k in range(3):
        r.step(DT, snapshot=(k == 2))
        g.step(DT)
    x, v, C = g.download()
    n = sc.x.shape[0]
    assert_close(v, r.get("g2p_v").reshape(n, 3), 1e-8, "v after 3 steps")
    assert_close(C, r.get("g2p_C").reshape(n, 9), 1e-8, "C after 3 steps")
    assert_close(x, r.get("adv_x").reshape(n, 3), 1e-11, "x after 3 steps")
    r.step(DT, snapshot=True)
    g.rebucketize_and_resample()
    assert np.array_equal(g.ifield("active"), r.get("active"))
    assert np.array_equal(g.ifield("array_idx"), r.get("array_idx"))
