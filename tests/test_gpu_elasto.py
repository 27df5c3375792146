"""Elasto (cloth / yarn) particle transfers on the GPU against the oracle.

The oracle's elasto branches are pinned to the reference in
tests/test_oracle_vs_reference.py::test_elasto_transfers.  Here the GPU runs
the same scenes through the C-ABI: the grid build with both particle kinds
(bit-exact keys, activation, stencil bases), P2G of both phases, then G2P from
the P2G node velocities (the liquid face velocity handed back through
wcg_upload_field, as the oracle's transfer does) and advection.  FP64 agrees
to 1e-10 relative to each field's maximum, FP32 to 1e-5 (the affine matrices
C and B relative to the size of their terms, max|v| 4/dx, since their sums
cancel)."""
import numpy as np
import pytest

from libwetcloth_b200 import _capi, scenes
from libwetcloth_b200.solver import FluidScene
from oracle import oracle as oo

pytestmark = pytest.mark.gpu
DT = 1e-3
P2G = ([f"{f}_{c}" for f in ("mass_fluid", "vel_fluid", "vol_fluid", "mass", "vel", "vol",
                              "psi", "sat", "shape_factor", "orientation") for c in "xyz"] +
       ["sat_p", "psi_p", "pore_pressure_p", "liquid_phi"])


def _close(a, b, tol, name, scale=0.0):
    m = ~np.isnan(b)
    assert np.array_equal(m, ~np.isnan(a)), name
    if m.any():
        scale = max(np.abs(b[m]).max(), scale, 1e-300)
        err = np.abs(a[m] - b[m]).max() / scale
        assert err <= tol, f"{name}: {err:.3e}"


def _scene(surfel_every=0, liquid=True, n=16):
    sc = scenes.liquid_on_sheet(n, 8, 3, surfel_every=surfel_every)
    sc.params.elasto_flip_coeff = 0.9
    sc.params.elasto_flip_asym_coeff = 0.3
    sc.params.elasto_advect_coeff = 0.97
    if not liquid:
        sc.x, sc.v = sc.x[:0], sc.v[:0]
        sc.mass, sc.vol, sc.radius = sc.mass[:0], sc.vol[:0], sc.radius[:0]
    return sc


def _transfer(g):
    """grid, P2G, G2P from the P2G velocities, advection"""
    g.rebucketize_and_resample()
    g.map_particle_nodes()
    fields = {k: g.field(k) for k in P2G}
    ints = {k: g.ifield(k) for k in ("array_idx", "active", "stencil_base")}
    if g.num_particles > 0:
        for c in "xyz":
            g.upload_field("u_" + c, fields["vel_fluid_" + c])
    g.map_node_particles()
    g2p = g.download(), g.download_elasto()
    g.advect(DT)
    adv = g.download(), g.download_elasto()
    return fields, ints, g2p, adv


def _check_particles(o, ne, tag, liquid, elasto, tol, xtol, dx):
    """C and B are sums of u w (x_n - x_p) 4/h^2 that cancel: their error
    is measured against the size of those terms, max|v| 4/dx."""
    (x, v, C), (x4, v4, B) = liquid, elasto
    nl = x.shape[0]
    if nl:
        ov = o.get(tag + "v").reshape(-1, 3)[ne:]
        _close(x, o.get(tag + "x").reshape(-1, 3)[ne:], xtol, tag + "x")
        _close(v, ov, tol, tag + "v")
        _close(C, o.get(tag + "C").reshape(-1, 9)[ne:], tol, tag + "C",
               np.abs(ov).max() * 4.0 / dx)
    ev = o.get(tag + "ev4").reshape(-1, 4)[:ne]
    _close(x4, o.get(tag + "x4").reshape(-1, 4)[:ne], xtol, tag + "x4")
    _close(v4, ev, tol, tag + "ev4")
    _close(B, o.get(tag + "eB").reshape(-1, 9)[:ne], tol, tag + "eB",
           np.abs(ev[:, :3]).max() * 4.0 / dx)


@pytest.mark.parametrize("surfel_every,liquid", [(0, True), (5, True), (0, False)])
def test_elasto_transfer_fp64(surfel_every, liquid, wcg):
    sc = _scene(surfel_every, liquid)
    o = oo.OracleScene(sc)
    o.transfer(DT)
    g = FluidScene(sc)
    assert g.num_elasto == sc.elasto.n
    fields, ints, g2p, adv = _transfer(g)
    for k, v in ints.items():
        assert np.array_equal(v, o.get(k)), k
    for k in P2G:
        _close(fields[k], o.get(k), 1e-10, k)
    assert np.nanmax(fields["psi_y"]) > 0.0
    ne = sc.elasto.n
    _check_particles(o, ne, "g2p_", *g2p, 1e-10, 1e-12, sc.params.dx)
    _check_particles(o, ne, "adv_", *adv, 1e-10, 1e-12, sc.params.dx)
    g.close()


def test_elasto_transfer_fp32(wcg):
    sc = _scene(5, True, n=24)
    o = oo.OracleScene(sc)
    o.transfer(DT)
    g = FluidScene(sc, precision=_capi.WCG_FP32_REFINE)
    fields, ints, g2p, adv = _transfer(g)
    for k in ("mass_x", "vel_y", "vol_z", "psi_x", "sat_y", "shape_factor_z", "orientation_x",
              "sat_p", "psi_p", "pore_pressure_p", "vel_fluid_x"):
        _close(fields[k], o.get(k), 1e-5, k)
    _check_particles(o, sc.elasto.n, "adv_", *adv, 1e-5, 1e-6, sc.params.dx)
    g.close()


@pytest.mark.parametrize("surfel_every", [0, 5])
def test_elasto_coupled_step_fp64(surfel_every, wcg):
    """A full step with a liquid sphere straddling the sheet: the drag, the
    pore-pressure gradient, the solid volume in the pressure system and the
    solid drag on the liquid (pinned to the reference in
    test_oracle_vs_reference.py::test_elasto_coupled_step), stage by stage."""
    sc = scenes.liquid_on_sheet(16, 8, 3, center=(0.5, 0.45, 0.5), surfel_every=surfel_every)
    o = oo.OracleScene(sc)
    o.step(DT, snapshot=True)
    g = FluidScene(sc)
    g.rebucketize_and_resample()
    g.map_particle_nodes()
    g.step_velocity(DT)
    for f in ("v_star_x", "v_star_y", "v_star_z", "rhs_fluid_y", "psi_fs_y"):
        _close(g.field(f), o.get(f), 1e-10, f)
    g.project_fine(DT)
    _close(g.field("pressure"), o.get("pressure"), 1e-10, "pressure")
    g.apply_pressure_drag_fluid(DT)
    g.constrain_liquid_velocity()
    g.correct_liquid_particles(DT)  # every sub-step (projection only at strength 0)
    g.map_node_particles()
    g.advect(DT)
    ne = sc.elasto.n
    x, v, C = g.download()
    _close(v, o.get("g2p_v").reshape(-1, 3)[ne:], 1e-10, "g2p_v")
    _close(x, o.get("adv_x").reshape(-1, 3)[ne:], 1e-12, "adv_x")
    x4, v4, B = g.download_elasto()
    _close(x4, o.get("adv_x4").reshape(-1, 4)[:ne], 1e-12, "adv_x4")
    _close(B, o.get("adv_eB").reshape(-1, 9)[:ne], 1e-10, "adv_eB", np.abs(v4).max() * 64)
    g.close()


def test_elasto_coupled_steps_fp32_and_cfl(wcg):
    sc = scenes.liquid_on_sheet(24, 8, 3, center=(0.5, 0.45, 0.5))
    o = oo.OracleScene(sc)
    g = FluidScene(sc, precision=_capi.WCG_FP32_REFINE)
    for dt in (1e-3, 2e-2, 0.2):
        assert g.num_substeps(dt) == o.num_substeps(dt), dt
    o.step(DT, snapshot=True)
    g.step(DT)
    assert g.stats()["converged"] == 1
    ne = sc.elasto.n
    x, v, C = g.download()
    _close(v, o.get("g2p_v").reshape(-1, 3)[ne:], 1e-5, "g2p_v")
    _close(x, o.get("adv_x").reshape(-1, 3)[ne:], 1e-6, "adv_x")
    g.close()


def test_elasto_vjp_refused(wcg):
    sc = _scene()
    g = FluidScene(sc)
    n = sc.x.shape[0]
    with pytest.raises(_capi.WcgError) as e:
        g.substep_vjp(DT, np.zeros((n, 3)), np.zeros((n, 9)), np.zeros((n, 3)))
    assert e.value.code == _capi.WCG_ERR_UNSUPPORTED
    g.close()


def test_elasto_upload_field_and_positions(tmp_path, wcg):
    """A solid-phase velocity handed in through wcg_upload_field drives the
    elasto G2P; the position file holds the elasto particles first."""
    sc = _scene()
    g = FluidScene(sc)
    g.rebucketize_and_resample()
    g.map_particle_nodes()
    vel = g.field("vel_y")
    act = ~np.isnan(vel)
    g.upload_field("vel_x", np.where(act, 0.0, np.nan))
    g.upload_field("vel_y", np.where(act, -2.0, np.nan))
    g.upload_field("vel_z", np.where(act, 0.0, np.nan))
    back = g.field("vel_y")
    assert np.all(back[act] == -2.0)
    g.map_node_particles()
    x4, v4, B = g.download_elasto()
    # a uniform field is reproduced exactly up to the weights' partition of
    # unity (weights sum to 1 over the full stencil)
    assert np.allclose(v4[:, 1], -2.0 * 0.97, rtol=1e-12)
    assert np.allclose(B, 0.0, atol=1e-9)
    path = tmp_path / "pos.bin"
    g.save_positions(path)
    import struct
    data = open(path, "rb").read()
    nb = struct.unpack_from("<i", data, 0)[0]
    pos = np.frombuffer(data, dtype="<f8", count=nb // 8, offset=4).reshape(-1, 4)
    ne = sc.elasto.n
    assert pos.shape[0] == ne + sc.x.shape[0]
    assert np.array_equal(pos[:ne], x4)
    assert np.array_equal(pos[ne:, :3], g.download()[0])
    g.load_positions(path)
    assert np.array_equal(g.download_elasto()[0], x4)
    g.close()


def test_elasto_coupled_four_steps_fp64(wcg):
    """Four whole steps with the coupling against the oracle (pinned to the
    reference over the same four steps)."""
    sc = scenes.liquid_on_sheet(16, 8, 3, center=(0.5, 0.45, 0.5), surfel_every=5)
    o = oo.OracleScene(sc)
    g = FluidScene(sc)
    for k in range(4):
        o.step(DT, snapshot=(k == 3))
        g.step(DT)
    ne = sc.elasto.n
    x, v, C = g.download()
    _close(v, o.get("g2p_v").reshape(-1, 3)[ne:], 1e-9, "g2p_v")
    _close(x, o.get("adv_x").reshape(-1, 3)[ne:], 1e-11, "adv_x")
    x4, v4, B = g.download_elasto()
    _close(x4, o.get("adv_x4").reshape(-1, 4)[:ne], 1e-11, "adv_x4")
    g.close()
