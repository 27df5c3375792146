"""GPU FP64 path against the oracle, stage by stage.

Checkers: the C restatement oracle (oracle/wc_oracle.c, always built) and,
when it is built, the compiled reference Core (oracle/_ref).  Both run one
sub-step of the fluid hot path on the same seeded scene and snapshot every
field; the GPU runs the same sub-step through the C-ABI stage calls.
Tolerances: integer/index data bit-exact (sort keys, bucket ranges,
activation masks, stencil indices, DOF numbering, matrix structure, valid
masks); FP64 fields within 1e-10 relative to the field's max magnitude; the
PCG-dependent pressure and everything after it within 1e-9 (the same MIC(0)
iterates, accumulated in a different order).  Pointwise: every entry above
1e-6 of its field's largest magnitude agrees to 1e-10 of itself in the P2G and
grid-update fields (1e-4 of the largest for the velocity-like fields, ratios
of sums whose terms cancel, so that their small entries carry the rounding of
terms up to the field's largest value), and every entry above 1e-4 of the
largest to 1e-6 of itself in the pressure and the fields after it (a PCG
solution's small entries carry the rounding of the whole solve).
"""
import numpy as np
import pytest

from libwetcloth_b200 import scenes
from libwetcloth_b200.solver import FluidScene
from oracle import oracle as oo
from oracle import ref as oref
from tests.parity import assert_close, assert_dense_close, assert_pointwise

pytestmark = pytest.mark.gpu

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


def boundary_lattice():
    """Particles exactly on cell faces, edges, corners and half-cells: every
    floor/frac tie of the stencil bases (frac == 0 and frac == 0.5)."""
    dx = 1.0 / 16
    g = np.arange(4, 13) * (dx / 2)
    z, y, x = np.meshgrid(g, np.arange(0, 9) * (dx / 2), g, indexing="ij")
    pts = np.stack([x.ravel(), y.ravel(), z.ravel()], 1)
    m, vol, r = scenes.attributes(pts.shape[0], dx, 8, 1000.0)
    return scenes.Scene(scenes.SceneParams(dx=dx), pts, np.zeros_like(pts), m, vol, r,
                        name="boundary_lattice")


def crowded_cell():
    """A dam-break block plus 64 extra particles packed into one cell."""
    sc = scenes.dam_break(16, 8, 2, block_hi=(0.3, 0.3, 0.3))
    rng = np.random.default_rng(9)
    extra = (np.array([0.4, 0.05, 0.4]) + rng.random((64, 3)) * (1 / 16))
    x = np.concatenate([sc.x, extra])
    m, vol, r = scenes.attributes(x.shape[0], sc.params.dx, 8, 1000.0)
    return scenes.Scene(sc.params, x, np.zeros_like(x), m, vol, r, name="crowded")


def make(kind):
    if kind == "dam16":
        return scenes.dam_break(16, 8, 0)
    if kind == "curl32":
        return scenes.half_box(32, 2, 5, amplitude=0.5, sigma_cells=2.0)
    if kind == "boundary":
        return boundary_lattice()
    if kind == "crowded":
        return crowded_cell()
    raise ValueError(kind)


def checker(name, sc):
    if name == "oracle":
        return oo.OracleScene(sc)
    if not oref.available():
        pytest.skip("oracle/_ref not built")
    return oref.RefScene(sc, mic=True)


@pytest.fixture(scope="module",
                params=[("dam16", "oracle"), ("curl32", "oracle"), ("boundary", "oracle"),
                        ("crowded", "oracle"), ("dam16", "reference"), ("curl32", "reference")],
                ids=lambda p: f"{p[0]}-{p[1]}")
def pair(request, wcg):
    kind, chk = request.param
    sc = make(kind)
    r = checker(chk, sc)
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
    g.correct_liquid_particles(DT)  # every sub-step (projection only at strength 0)
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


def pointwise_floor(name):
    """Floor (relative to the field's largest magnitude) above which a field
    is compared pointwise: 1e-4 for velocity-like fields, 1e-6 otherwise."""
    return 1e-4 if name.startswith(("vel", "v_star", "rhs")) else 1e-6


def test_p2g_fields(pair):
    sc, r, out = pair
    for k in P2G_FIELDS:
        assert_dense_close(out[k], r.get(k), 1e-10, k)
        assert_pointwise(out[k], r.get(k), 1e-10, k, pointwise_floor(k))


def test_predict_fields(pair):
    sc, r, out = pair
    for k in PREDICT_FIELDS:
        assert_dense_close(out[k], r.get(k), 1e-10, k)
        assert_pointwise(out[k], r.get(k), 1e-10, k, pointwise_floor(k))


@pytest.mark.parametrize("prec", [0, 1])
@pytest.mark.parametrize("kind", ["dam16", "curl32", "crowded"])
def test_tiled_transfers_match_gathers(kind, prec, wcg, monkeypatch):
    """The bucket-tile transfers (P2G: warp-per-bucket scatter into halo
    tiles and a fixed-order merge; G2P: per-bucket node neighbourhood staged
    in shared memory) against the global gathers (WCG_TRANSFERS=gather).
    P2G sums the same terms in another order: fields agree to 1e-13 (FP64) /
    1e-6 (FP32) of each field's largest value.  G2P, from one common face
    velocity field, evaluates the same sums in the same order: velocities,
    affine matrices and advected positions agree to 1e-14 / 1e-6.  The tiles
    are bit-identical run to run."""
    sc = make(kind)
    res = {}
    u_common = None
    for mode in ("gather", "tiles", "tiles2"):
        monkeypatch.setenv("WCG_TRANSFERS", "gather" if mode == "gather" else "tiles")
        g = FluidScene(sc, precision=prec)
        g.rebucketize_and_resample()
        g.map_particle_nodes()
        out = {k: g.field(k) for k in P2G_FIELDS}
        if u_common is None:
            u_common = {a: out["vel_fluid_" + a] for a in "xyz"}
        for a in "xyz":
            g.upload_field("u_" + a, u_common[a])
        g.map_node_particles()
        _, out["v"], out["C"] = g.download()
        g.advect(DT)
        out["x"], _, _ = g.download()
        res[mode] = out
        g.close()
    tol_p2g, tol_g2p = (1e-13, 1e-14) if prec == 0 else (1e-6, 1e-6)
    for k in P2G_FIELDS:
        assert_dense_close(res["tiles"][k], res["gather"][k], tol_p2g, k)
    for k in ("v", "C", "x"):
        assert_close(res["tiles"][k], res["gather"][k], tol_g2p, k)
    for k in P2G_FIELDS + ["v", "C", "x"]:
        a, b = res["tiles"][k], res["tiles2"][k]
        assert np.array_equal(np.isnan(a), np.isnan(b)) and np.array_equal(
            np.nan_to_num(a), np.nan_to_num(b)), k


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
    assert st["residual"] <= sc.params.criterion * st["rhs_norm"]
    assert_dense_close(out["pressure"], r.get("pressure"), 1e-9, "pressure")
    assert_pointwise(out["pressure"], r.get("pressure"), 1e-6, "pressure", 1e-4)


def test_projection_and_constraint(pair):
    sc, r, out = pair
    for a in "xyz":
        assert np.array_equal(out["valid_" + a], r.get("valid_" + a)), "valid_" + a
        assert_dense_close(out["u_proj_" + a], r.get("u_proj_" + a), 1e-9, "u_proj_" + a)
        assert_dense_close(out["u_final_" + a], r.get("u_final_" + a), 1e-9, "u_final_" + a)
        assert_pointwise(out["u_final_" + a], r.get("u_final_" + a), 1e-6, "u_final_" + a, 1e-4)


def test_g2p_and_advect(pair):
    sc, r, out = pair
    n = sc.x.shape[0]
    assert_close(out["g2p_v"], r.get("g2p_v").reshape(n, 3), 1e-9, "G2P velocity")
    assert_close(out["g2p_C"], r.get("g2p_C").reshape(n, 9), 1e-9, "G2P affine C")
    assert_close(out["adv_x"], r.get("adv_x").reshape(n, 3), 1e-12, "advected x")
    assert_pointwise(out["g2p_v"], r.get("g2p_v").reshape(n, 3), 1e-6, "G2P velocity", 1e-4)
    assert_pointwise(out["adv_x"], r.get("adv_x").reshape(n, 3), 1e-12, "advected x", 1e-6)


@pytest.mark.parametrize("chk", ["oracle", "reference"])
def test_multi_step_state(chk, wcg):
    sc = make("dam16")
    r = checker(chk, sc)
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
