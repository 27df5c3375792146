"""Explicit liquid viscosity on the GPU against the oracle.

The oracle is pinned to the reference's viscous step in
tests/test_oracle_vs_reference.py::test_explicit_viscosity_step.  Here the GPU
runs the same scenes through the C-ABI stage by stage: liquid volume fractions
(cell centres, x/y/z edges), the viscous face velocities after two explicit
sub-steps, the rebuilt rhs, the pressure and the particle update.  FP64 fields
agree to 1e-10 relative to their maximum; the FP32 form (FP64 refinement) to
1e-5 on velocities and pressure."""
import numpy as np
import pytest

from libwetcloth_b200 import _capi, scenes
from libwetcloth_b200.solver import FluidScene
from oracle import oracle as oo

pytestmark = pytest.mark.gpu
DT = 1e-3


def _scene(kind, mu):
    if kind == "dam16":
        sc = scenes.dam_break(16, 8, 0)
    elif kind == "curl16":
        sc = scenes.half_box(16, 2, 7, amplitude=1.0, sigma_cells=1.5)
    else:
        sc = scenes.half_box(32, 2, 5, amplitude=0.5, sigma_cells=2.0)
    sc.params.viscosity = mu
    sc.params.viscosity_substeps = 2
    return sc


def _close(a, b, tol, name):
    m = ~np.isnan(b)
    assert np.array_equal(m, ~np.isnan(a)), name
    if m.any():
        scale = max(np.abs(b[m]).max(), 1e-300)
        err = np.abs(a[m] - b[m]).max() / scale
        assert err <= tol, f"{name}: {err:.3e}"


@pytest.mark.parametrize("kind,mu", [("dam16", 5.0), ("curl16", 8.9e-3), ("curl32", 1.0)])
def test_viscosity_fp64_against_oracle(kind, mu, wcg):
    sc = _scene(kind, mu)
    o = oo.OracleScene(sc)
    o.step(DT, snapshot=True)
    g = FluidScene(sc)
    g.rebucketize_and_resample()
    g.map_particle_nodes()
    for f in ("liquid_c_vf", "liquid_ex_vf", "liquid_ey_vf", "liquid_ez_vf"):
        _close(g.field(f), o.get(f), 1e-12, f)
    g.step_velocity(DT)
    for f in ("v_star_x", "v_star_y", "v_star_z", "rhs_fluid_x", "rhs_fluid_y", "rhs_fluid_z"):
        _close(g.field(f), o.get(f), 1e-10, f)
    g.project_fine(DT)
    _close(g.field("pressure"), o.get("pressure"), 1e-10, "pressure")
    g.apply_pressure_drag_fluid(DT)
    g.constrain_liquid_velocity()
    g.correct_liquid_particles(DT)  # every sub-step (projection only at strength 0)
    g.map_node_particles()
    g.advect(DT)
    x, v, C = g.download()
    n = sc.x.shape[0]
    _close(v, o.get("g2p_v").reshape(n, 3), 1e-10, "g2p_v")
    _close(x, o.get("adv_x").reshape(n, 3), 1e-12, "adv_x")
    g.close()


def test_viscosity_changes_the_flow_and_fp32(wcg):
    sc = _scene("curl32", 1.0)
    base = _scene("curl32", 0.0)
    g0 = FluidScene(base)
    g0.step(DT)
    v0 = g0.download()[1]
    g0.close()
    g = FluidScene(sc)
    g.step(DT)
    v1 = g.download()[1]
    g.close()
    assert np.abs(v1 - v0).max() > 1e-6 * np.abs(v0).max()   # the term is active
    g32 = FluidScene(sc, precision=_capi.WCG_FP32_REFINE)
    g32.step(DT)
    v32 = g32.download()[1]
    assert g32.stats()["converged"] == 1
    assert np.abs(v32 - v1).max() <= 1e-5 * np.abs(v1).max()
    g32.close()


def _implicit(kind, mu, ns, criterion):
    sc = _scene(kind, mu)
    sc.params.viscosity_substeps = ns
    sc.params.viscosity_implicit = True
    sc.params.viscosity_criterion = criterion
    sc.params.maxiters = 5000
    return sc


@pytest.mark.parametrize("kind,mu,ns", [("dam16", 0.5, 1), ("curl16", 2.0, 2), ("dam16", 50.0, 1),
                                        ("curl32", 1.0, 1)])
def test_implicit_viscosity_fp64(kind, mu, ns, wcg):
    """Implicit viscosity (stepImplicitViscosityDiagonalPCG), pinned to the
    reference through the oracle (test_oracle_vs_reference.py::
    test_implicit_viscosity).  The GPU solves the same system matrix-free with
    the diagonal as preconditioner: face volume fractions to 1e-10; on the last
    sub-step the GPU's velocities solve the oracle's assembled system to the
    criterion; the velocities agree on every face with liquid volume (where
    the system's null space vanishes) to 1e-8."""
    sc = _implicit(kind, mu, ns, 1e-13)
    o = oo.OracleScene(sc)
    o.step(DT, snapshot=True)
    g = FluidScene(sc)
    g.rebucketize_and_resample()
    g.map_particle_nodes()
    for k in ("liquid_u_vf", "liquid_v_vf", "liquid_w_vf", "liquid_c_vf", "liquid_ey_vf"):
        _close(g.field(k), o.get(k), 1e-10, k)
    g.step_velocity(DT)
    st = g.stats()
    assert st["visc_converged"] == 1 and st["visc_iters"] > 0
    vs = [g.field("v_star_" + c) for c in "xyz"]
    rs, ci, va, b = o.get("V_rowstart"), o.get("V_col"), o.get("V_val"), o.get("V_rhs")
    face = o.get("V_face")
    nn = vs[0].size
    x = np.array([vs[f // nn][f % nn] for f in face])
    import scipy.sparse as sps
    A = sps.csr_matrix((va, ci, rs), shape=(rs.size - 1, rs.size - 1))
    if ns == 1:
        assert np.abs(b - A @ x).max() <= 1e-11 * np.abs(b).max()
    errs, scale = [], 0.0
    for a, c in enumerate("xyz"):
        m = np.nan_to_num(o.get("liquid_" + "uvw"[a] + "_vf"), nan=0.0) > 0.0
        ov = o.get("v_star_" + c)
        errs.append(np.abs(vs[a][m] - ov[m]).max())
        scale = max(scale, np.abs(ov[m]).max())
    assert max(errs) <= 1e-8 * scale, errs
    g.close()


def test_implicit_viscosity_steps_and_fp32(wcg):
    """FP32 (criterion 1e-5): the velocities solve the oracle's FP64 system to
    2e-5 of its rhs (the solution itself is only as determined as the
    ill-conditioned system and the criterion allow); whole steps with the
    implicit viscosity converge in both precisions."""
    sc = _implicit("curl16", 2.0, 1, 1e-5)
    o = oo.OracleScene(sc)
    o.step(DT, snapshot=True)
    g = FluidScene(sc, precision=_capi.WCG_FP32_REFINE)
    g.rebucketize_and_resample()
    g.map_particle_nodes()
    g.step_velocity(DT)
    vs = [g.field("v_star_" + c) for c in "xyz"]
    rs, ci, va, b = o.get("V_rowstart"), o.get("V_col"), o.get("V_val"), o.get("V_rhs")
    face = o.get("V_face")
    nn = vs[0].size
    x = np.array([vs[f // nn][f % nn] for f in face])
    import scipy.sparse as sps
    A = sps.csr_matrix((va, ci, rs), shape=(rs.size - 1, rs.size - 1))
    assert np.abs(b - A @ x).max() <= 2e-5 * np.abs(b).max()
    g.close()
    for prec in (_capi.WCG_FP64, _capi.WCG_FP32_REFINE):
        g = FluidScene(_implicit("dam16", 0.5, 2, 1e-6), precision=prec)
        for _ in range(3):
            g.step(DT)
        st = g.stats()
        assert st["converged"] == 1 and st["visc_converged"] == 1 and st["visc_iters"] > 0
        x, v, C = g.download()
        assert np.all(np.isfinite(v))
        g.close()
