"""The C restatement oracle against the compiled reference Core on seeded
scenes (skipped when oracle/_ref is not built).  Runs on CPU."""
import numpy as np
import pytest

from libwetcloth_b200 import scenes
from oracle import oracle as oo
from oracle import ref as oref
from tests.parity import TERMINATOR_SHAPES

pytestmark = pytest.mark.skipif(not (oref.available() and oo.available()),
                                reason="oracle/_ref or the oracle not built")
DT = 1e-3
EXACT = ["grid_dims", "grid_origin", "bbx", "array_idx", "array_sup", "active",
         "stencil_base", "inside", "dof_index", "A_rowstart", "A_col", "valid_x",
         "valid_y", "valid_z"]
CLOSE = ["mass_fluid_x", "vel_fluid_y", "vol_fluid_z", "sat_p", "liquid_phi", "solid_phi",
         "solid_weight_x", "solid_weight_z", "v_star_y", "rhs_fluid_y", "inv_C_x",
         "psi_fs_z", "A_val", "b", "pressure", "u_proj_x", "u_final_y", "g2p_v", "g2p_C",
         "adv_x"]


def _scene(kind):
    if kind == "dam16":
        return scenes.dam_break(16, 8, 0)
    if kind == "curl16":
        return scenes.half_box(16, 2, 7, amplitude=1.0, sigma_cells=1.5)
    if kind == "dam24_tall":
        return scenes.dam_break(24, 8, 4, block_hi=(0.3, 0.9, 0.6))
    raise ValueError(kind)


@pytest.mark.parametrize("kind", ["dam16", "curl16", "dam24_tall"])
def test_first_step(kind):
    sc = _scene(kind)
    r = oref.RefScene(sc, mic=True)
    o = oo.OracleScene(sc)
    r.step(DT, snapshot=True)
    o.step(DT, snapshot=True)
    for k in EXACT:
        assert np.array_equal(r.get(k), o.get(k)), k
    assert r.solver_stats()[0] == o.solver_stats()[0]
    for k in CLOSE:
        a, b = r.get(k), o.get(k)
        m = ~np.isnan(a)
        assert np.array_equal(m, ~np.isnan(b)), k
        if m.any():
            assert np.abs(a[m] - b[m]).max() <= 1e-12 * max(np.abs(a[m]).max(), 1e-300), k


def test_five_steps_dam16():
    sc = _scene("dam16")
    r = oref.RefScene(sc, mic=True)
    o = oo.OracleScene(sc)
    for k in range(5):
        r.step(DT, snapshot=(k == 4))
        o.step(DT, snapshot=(k == 4))
    for k in ("adv_x", "g2p_v", "g2p_C"):
        a, b = r.get(k), o.get(k)
        assert np.abs(a - b).max() <= 1e-10 * np.abs(a).max(), k


def test_mic0_pcg_on_reference_matrix():
    """robertbridson::PCGSolver restated on the reference's assembled system."""
    sc = _scene("curl16")
    r = oref.RefScene(sc, mic=True)
    r.step(DT, snapshot=True)
    rs, col, val, b = r.get("A_rowstart"), r.get("A_col"), r.get("A_val"), r.get("b")
    x, ok, it, res = oo.pcg_solve(rs, col, val, b, sc.params.criterion, sc.params.maxiters)
    it_ref, _ = r.solver_stats()
    assert ok and it == it_ref
    p = r.get("pressure")
    dof = r.get("dof_index")
    pref = p[dof >= 0][np.argsort(dof[dof >= 0])]
    assert np.abs(x - pref).max() <= 1e-12 * np.abs(pref).max()
    # the residual criterion of the reference: ||b - A x||_inf <= tol ||b||_inf
    Ax = np.zeros_like(b)
    for i in range(len(b)):
        Ax[i] = np.dot(val[rs[i]:rs[i + 1]], x[col[rs[i]:rs[i + 1]]])
    assert np.abs(b - Ax).max() <= sc.params.criterion * np.abs(b).max() * 1.0001


VISC = ["liquid_c_vf", "liquid_ex_vf", "liquid_ey_vf", "liquid_ez_vf", "v_star_x",
        "v_star_y", "v_star_z", "rhs_fluid_x", "rhs_fluid_z", "pressure", "g2p_v", "adv_x"]


@pytest.mark.parametrize("kind,mu", [("dam16", 5.0), ("curl16", 8.9e-3), ("curl16", 5.0)])
def test_explicit_viscosity_step(kind, mu):
    """Explicit viscosity (estimateVolumeFractions + applyNodeViscosityExplicit,
    two sub-steps): volume fractions, the viscous face velocities and the rest
    of the step against the reference."""
    sc = _scene(kind)
    sc.params.viscosity = mu
    sc.params.viscosity_substeps = 2
    r = oref.RefScene(sc, mic=True)
    o = oo.OracleScene(sc)
    r.step(DT, snapshot=True)
    o.step(DT, snapshot=True)
    for k in VISC:
        a, b = r.get(k), o.get(k)
        m = ~np.isnan(a)
        assert np.array_equal(m, ~np.isnan(b)), k
        if m.any():
            assert np.abs(a[m] - b[m]).max() <= 1e-12 * max(np.abs(a[m]).max(), 1e-300), k
    assert (r.get("liquid_c_vf")[~np.isnan(r.get("liquid_c_vf"))] > 0).any()


ELASTO_EXACT = ["grid_dims", "grid_origin", "bbx", "array_idx", "array_sup", "active",
                "stencil_base", "inside"]
ELASTO_CLOSE = ([f"{f}_{c}" for f in ("mass_fluid", "vel_fluid", "vol_fluid", "mass", "vel",
                                      "vol", "psi", "sat", "shape_factor", "orientation")
                 for c in "xyz"] +
                ["sat_p", "psi_p", "pore_pressure_p", "liquid_phi"] +
                [t + q for t in ("g2p_", "adv_") for q in ("x", "v", "C", "x4", "ev4", "eB")])


@pytest.mark.parametrize("surfel_every,flip,asym", [(0, 0.95, 1.0), (5, 0.9, 0.3)])
def test_elasto_transfers(surfel_every, flip, asym):
    """P2G with both particle kinds (solid mass/velocity/volume, psi,
    saturation, shape factor, orientation, cell-centre psi/saturation/pore
    pressure), then G2P from the P2G velocities (the elasto B blend included)
    and advection, on a liquid sphere over a cloth sheet."""
    sc = scenes.liquid_on_sheet(16, 8, 3, surfel_every=surfel_every)
    sc.params.elasto_flip_coeff = flip
    sc.params.elasto_flip_asym_coeff = asym
    sc.params.elasto_advect_coeff = 0.97
    r = oref.RefScene(sc, mic=True)
    o = oo.OracleScene(sc)
    r.transfer(DT)
    o.transfer(DT)
    for k in ELASTO_EXACT:
        assert np.array_equal(r.get(k), o.get(k)), k
    psi = r.get("psi_x")
    assert np.nanmax(psi) > 0.0            # the sheet shows up as solid
    for k in ELASTO_CLOSE:
        a, b = r.get(k), o.get(k)
        m = ~np.isnan(a)
        assert np.array_equal(m, ~np.isnan(b)), k
        if m.any():
            assert np.abs(a[m] - b[m]).max() <= 1e-12 * max(np.abs(a[m]).max(), 1e-300), k


def test_elasto_only_scene():
    """No liquid particle: every particle is elasto and the liquid level set
    keeps its initial value (updateLiquidPhi returns early)."""
    sc = scenes.liquid_on_sheet(16, 8, 3)
    sc.x, sc.v = sc.x[:0], sc.v[:0]
    sc.mass, sc.vol, sc.radius = sc.mass[:0], sc.vol[:0], sc.radius[:0]
    r = oref.RefScene(sc, mic=True)
    o = oo.OracleScene(sc)
    r.transfer(DT)
    o.transfer(DT)
    for k in ELASTO_EXACT:
        assert np.array_equal(r.get(k), o.get(k)), k
    lp = r.get("liquid_phi")
    assert np.all(lp[~np.isnan(lp)] == 3.0 * 4 * sc.params.dx)
    for k in ("mass_x", "vel_y", "psi_z", "sat_p", "psi_p", "liquid_phi", "g2p_ev4", "g2p_eB",
              "adv_x4"):
        a, b = r.get(k), o.get(k)
        m = ~np.isnan(a)
        assert np.array_equal(m, ~np.isnan(b)), k
        assert np.abs(a[m] - b[m]).max() <= 1e-12 * max(np.abs(a[m]).max(), 1e-300), k


@pytest.mark.parametrize("surfel_every", [0, 5])
def test_elasto_coupled_step(surfel_every):
    """A full step with a liquid sphere straddling a cloth sheet: the drag of
    constructHDV, the pore-pressure gradient with the node orientation, the
    solid volume in the pressure system and applyPressureDragFluid's solid
    drag, the solid solve off (LiquidInfo::solve_solid false)."""
    sc = scenes.liquid_on_sheet(16, 8, 3, center=(0.5, 0.45, 0.5), surfel_every=surfel_every)
    r = oref.RefScene(sc, mic=True)
    o = oo.OracleScene(sc)
    assert r.step(DT, snapshot=True) == o.step(DT, snapshot=True)
    assert r.solver_stats()[0] == o.solver_stats()[0]
    for k in ("array_idx", "active", "dof_index", "A_rowstart", "A_col", "valid_x"):
        assert np.array_equal(r.get(k), o.get(k)), k
    for k in ("v_star_y", "rhs_fluid_x", "inv_C_z", "psi_fs_y", "A_val", "b", "pressure",
              "u_proj_x", "u_final_y", "g2p_v", "g2p_C", "adv_x", "g2p_ev4", "g2p_eB", "adv_x4"):
        a, b = r.get(k), o.get(k)
        m = ~np.isnan(a)
        assert np.array_equal(m, ~np.isnan(b)), k
        if m.any():
            assert np.abs(a[m] - b[m]).max() <= 1e-12 * max(np.abs(a[m]).max(), 1e-300), k
    # the coupling is active: the same liquid without the sheet steps differently
    sc2 = scenes.liquid_on_sheet(16, 8, 3, center=(0.5, 0.45, 0.5))
    sc2.elasto = None
    o2 = oo.OracleScene(sc2)
    o2.step(DT, snapshot=True)
    a, b = o.get("g2p_v")[-3 * sc.x.shape[0]:], o2.get("g2p_v")
    assert np.abs(a - b).max() > 1e-3 * np.abs(b).max()


def _fall(n=16, vy=-3.0):
    """A dam-break block thrown at the floor: many liquid particles end a
    sub-step inside the wall and are pushed back out by solidProjection."""
    sc = scenes.dam_break(n, 8, 0)
    sc.v[:, 1] = vy
    return sc


@pytest.mark.parametrize("dt", [1e-3, 2e-2])
def test_solid_projection(dt):
    """advectScene + solidProjection (TwoDScene.cpp:1776-1821) of the liquid
    particles at the end of each sub-step."""
    sc = _fall()
    r = oref.RefScene(sc, mic=True)
    o = oo.OracleScene(sc)
    n = r.step(dt, snapshot=True)
    assert o.step(dt, snapshot=True) == n
    assert o.get("projected")[0] > 0
    for k in ("g2p_v", "adv_x"):
        a, b = r.get(k), o.get(k)
        assert np.abs(a - b).max() <= 1e-12 * np.abs(a).max(), k


@pytest.mark.parametrize("kind,seed", [("dam16", 3), ("curl16", 11), ("fall", 5)])
def test_particle_correction(kind, seed):
    """correctLiquidParticles (TwoDScene.cpp:1967-2061) at the scene parser's
    defaults (strength 0.2, step 8, multiplier 2): the reference draws its
    subset with rand() after srand(seed), the oracle is handed the same subset;
    positions after the correction, G2P (weights of the uncorrected positions,
    x_n - x_p of the corrected ones) and advection agree."""
    sc = _fall() if kind == "fall" else _scene(kind)
    sc.params.correction_strength = 0.2
    sc.params.correction_seed = seed
    r = oref.RefScene(sc, mic=True)
    r.step(DT, snapshot=True)
    sel = int(r.get("correction_selector")[0])
    o = oo.OracleScene(sc)
    o.set_correction_selector(sel)
    o.step(DT, snapshot=True)
    assert int(o.get("correction_selector")[0]) == sel
    moved = np.abs(r.get("corr_x") - r.get("adv_x")).max()
    assert moved > 0
    x0 = sc.x.reshape(-1)
    dx_ref = r.get("corr_x") - x0
    assert np.abs(dx_ref).max() > 0.0
    for k in ("corr_x", "g2p_v", "g2p_C", "adv_x"):
        a, b = r.get(k), o.get(k)
        assert np.abs(a - b).max() <= 1e-12 * np.abs(a).max(), k
    # only the chosen subset moved
    idx = np.arange(sc.x.shape[0])
    still = (idx % sc.params.correction_step) != sel
    assert np.array_equal(r.get("corr_x").reshape(-1, 3)[still], sc.x[still])


@pytest.mark.parametrize("kind,mu,ns", [("dam16", 0.5, 1), ("curl16", 2.0, 2), ("dam16", 50.0, 1)])
def test_implicit_viscosity(kind, mu, ns):
    """stepImplicitViscosityDiagonalPCG (LinearizedImplicitEuler.cpp:2127) with
    constructViscosityMatrixRHS / updateViscosityRHS (Viscosity.cpp:169-1779):
    face volume fractions, the unknowns and the last sub-step's system (CSR
    structure exact, values and rhs to 1e-12; 1e-9 for the rhs of a later
    sub-step, which carries the earlier solution).  Unknowns without liquid
    volume of their own that touch liquid only across edges make the matrix
    singular, and the solution there is whatever the solver's Krylov path
    leaves, on either side; the solution is compared on the unknowns with
    their own liquid volume (the null space vanishes there; 1e-8, as the
    system is ill-conditioned next to it), and the reference's solution
    solves the oracle's system to the criterion."""
    sc = _scene(kind)
    sc.params.viscosity = mu
    sc.params.viscosity_substeps = ns
    sc.params.viscosity_implicit = True
    sc.params.viscosity_criterion = 1e-13
    sc.params.maxiters = 5000
    r = oref.RefScene(sc, mic=True)
    o = oo.OracleScene(sc)
    r.step(DT, snapshot=True)
    o.step(DT, snapshot=True)
    for k in ("V_rowstart", "V_col"):
        assert np.array_equal(r.get(k), o.get(k)), k
    for k in ("liquid_u_vf", "liquid_v_vf", "liquid_w_vf"):
        a, b = r.get(k), o.get(k)
        m = ~np.isnan(a)
        assert np.array_equal(m, ~np.isnan(b)), k
        assert np.abs(a[m] - b[m]).max() <= 1e-12, k
    va, vb = r.get("V_val"), o.get("V_val")
    assert np.abs(va - vb).max() <= 1e-12 * np.abs(va).max()
    ba, bb = r.get("V_rhs"), o.get("V_rhs")
    assert np.abs(ba - bb).max() <= (1e-12 if ns == 1 else 1e-9) * np.abs(ba).max()
    import scipy.sparse as sps
    rs, ci = o.get("V_rowstart"), o.get("V_col")
    n = rs.size - 1
    A = sps.csr_matrix((vb, ci, rs), shape=(n, n))
    xr, xo = r.get("V_soln"), o.get("V_soln")
    assert np.abs(bb - A @ xr).max() <= 1e-11 * np.abs(bb).max()
    own = o.get("V_volu") > 0.0
    assert own.sum() > 0 and (~own).sum() > 0
    assert np.abs(xr[own] - xo[own]).max() <= 1e-8 * np.abs(xr).max()
    it, res, nd = o.viscosity_stats()
    assert nd == n and it > 0
    errs, scale = [], 0.0
    for k in ("v_star_x", "v_star_y", "v_star_z"):
        f = r.get("liquid_" + "uvw"["xyz".index(k[-1])] + "_vf")
        m = np.nan_to_num(f, nan=0.0) > 0.0
        a, b = r.get(k), o.get(k)
        errs.append(np.abs(a[m] - b[m]).max())
        scale = max(scale, np.abs(a[m]).max())
    assert max(errs) <= 1e-8 * scale, errs


@pytest.mark.parametrize("kind,seed", [("dam16", 3), ("curl16", 5), ("fall", 8)])
def test_particle_merge(kind, seed):
    """updateOptiVolume + mergeLiquidParticles (TwoDScene.cpp:2484-2666) and
    removeEmptyParticles (:1713) after a step, on particles of mixed volume
    (classes S, s, o, l, L): the reference draws its subset and colour order
    with rand() after srand(seed); the oracle is handed the same draws.  Same
    particles removed, the same order after the swap-with-last removal, the
    same classes; positions, velocities, volumes, masses and radii to 1e-12."""
    sc = _fall() if kind == "fall" else _scene(kind)
    scenes.mixed_volumes(sc, seed)
    r = oref.RefScene(sc, mic=True)
    o = oo.OracleScene(sc)
    r.step(DT, snapshot=True)
    o.step(DT, snapshot=True)
    nr = r.merge(seed, 8)
    sel = int(r.get("merge_selector")[0])
    perm = r.get("merge_perm")
    assert sorted(perm[:3]) == [0, 1, 2] and sorted(perm[6:]) == [0, 1, 2]
    assert nr > 0
    assert o.merge(sel, perm) == nr
    assert np.array_equal(r.get("merge_class"), o.get("merge_class"))
    for k in ("merge_x", "merge_v", "merge_C", "merge_vol", "merge_mass", "merge_radius"):
        a, b = r.get(k), o.get(k)
        assert a.shape == b.shape, k
        assert np.abs(a - b).max() <= 1e-12 * np.abs(a).max(), k


@pytest.mark.parametrize("kind,seed", [("dam16", 3), ("curl16", 5)])
def test_particle_split(kind, seed):
    """updateOptiVolume + splitLiquidParticles (TwoDScene.cpp:2362-2480) after
    a step, on particles of mixed volume up to 40 V_fine (splits into up to 32):
    the number of children, their order (appended parent by parent), volumes,
    masses, radii, velocities, zero affine matrices and the classes match the
    reference to 1e-12, and every particle that did not split keeps its
    position.  The children's positions are not compared: the reference
    places them on its compiled sphere-pattern table rotated by
    Matrix3s::Random(), the oracle (and the GPU) on a Fibonacci lattice rotated
    by a seeded quaternion; both put them at distance |p_i| s from the
    parent's centre."""
    sc = _scene(kind)
    scenes.mixed_volumes(sc, seed, mrel=(0.3, 1.0, 2.5, 7.0, 40.0))
    r = oref.RefScene(sc, mic=True)
    o = oo.OracleScene(sc)
    r.step(DT, snapshot=True)
    o.step(DT, snapshot=True)
    added = r.split(seed)
    assert added > 0
    assert o.split(seed * 7919 + 1) == added
    for k in ("split_v", "split_C", "split_vol", "split_mass", "split_radius"):
        a, b = r.get(k), o.get(k)
        assert a.shape == b.shape, k
        assert np.abs(a - b).max() <= 1e-12 * np.abs(a).max(), k
    assert np.array_equal(r.get("split_class"), o.get("split_class"))
    n0 = sc.x.shape[0]
    before = r.get("adv_x").reshape(-1, 3)
    xr = r.get("split_x").reshape(-1, 3)
    xo = o.get("split_x").reshape(-1, 3)
    still = np.abs(xr[:n0] - before).max(axis=1) == 0
    assert still.sum() > 0 and (~still).sum() > 0
    assert np.abs(xo[:n0][still] - xr[:n0][still]).max() <= 1e-12
    # children of the oracle sit within 0.75 max(r_new, r - r_new) of their parent's centre
    assert np.all(np.abs(xo[n0:]).max() <= 2.0)


def test_elasto_coupled_four_steps():
    """Four steps of the liquid sphere straddling the sheet (drag, pore
    pressure, solid volume, the sheet carried by its transferred velocity)."""
    sc = scenes.liquid_on_sheet(16, 8, 3, center=(0.5, 0.45, 0.5), surfel_every=5)
    r = oref.RefScene(sc, mic=True)
    o = oo.OracleScene(sc)
    for k in range(4):
        assert r.step(DT, snapshot=(k == 3)) == o.step(DT, snapshot=(k == 3))
    for k in ("g2p_v", "adv_x", "adv_x4", "g2p_eB"):
        a, b = r.get(k), o.get(k)
        assert np.abs(a - b).max() <= 1e-10 * np.abs(a).max(), k


@pytest.mark.parametrize("inside", [True, False])
def test_terminate_particles(inside):
    """terminateParticles (TwoDScene.cpp:1756-1771) with a terminator box in a
    distance-field group of its own, after a step: the same particles are
    removed, the survivors take the same slots (removeEmptyParticles' swap
    with the last one) and keep their state to 1e-12; a second call removes
    nothing."""
    sc = _scene("curl16")
    lo, hi = sc.x.min(axis=0), sc.x.max(axis=0)
    p = sc.params
    p.terminator = True
    p.terminator_center = tuple(0.5 * (lo + hi))
    p.terminator_half = tuple(0.3 * (hi - lo))
    p.terminator_radius = 0.25 * p.dx
    p.terminator_inside = inside
    r = oref.RefScene(sc, mic=True)
    o = oo.OracleScene(sc)
    # the step's first stage is the terminator (WetClothCore.cpp:97)
    r.step(DT, snapshot=True)
    o.step(DT, snapshot=True)
    removed = int(r.get("terminate_removed")[0])
    assert 0 < removed < sc.x.shape[0]
    assert int(o.get("terminate_removed")[0]) == removed
    for k in ("adv_x", "adv_v", "g2p_C"):
        a, b = r.get(k), o.get(k)
        assert a.shape == b.shape, k
        assert np.abs(a - b).max() <= 1e-10 * max(np.abs(a).max(), 1.0), k
    # and a call on its own after the step: particles that moved out
    n = r.terminate()
    assert o.terminate() == n
    for k in ("term_x", "term_v", "term_C"):
        a, b = r.get(k), o.get(k)
        assert a.shape == b.shape, k
        assert np.abs(a - b).max() <= 1e-10 * max(np.abs(a).max(), 1.0), k
    assert r.terminate() == 0 and o.terminate() == 0




def test_terminate_particles_shapes():
    """terminateParticles with rotated terminator objects of all four
    analytic types in three distance-field groups (a sphere and a capsule
    removing what enters them, a cylinder, and a rotated box removing what
    leaves it): the restatement takes the reference's own rotation
    quaternions and removes the same particles, with the survivors in the
    same slots, in a step and in a call of its own after it."""
    sc = _scene("curl16")
    r = oref.RefScene(sc, mic=True)
    shapes = r.add_terminators(TERMINATOR_SHAPES)
    o = oo.OracleScene(sc)
    o.set_terminators(shapes)
    r.step(DT, snapshot=True)
    o.step(DT, snapshot=True)
    removed = int(r.get("terminate_removed")[0])
    assert 0 < removed < sc.x.shape[0] // 2
    assert int(o.get("terminate_removed")[0]) == removed
    for k in ("adv_x", "adv_v", "g2p_C"):
        a, b = r.get(k), o.get(k)
        assert a.shape == b.shape, k
        assert np.abs(a - b).max() <= 1e-10 * max(np.abs(a).max(), 1.0), k
    n = r.terminate()
    assert o.terminate() == n
    for k in ("term_x", "term_v", "term_C"):
        a, b = r.get(k), o.get(k)
        assert a.shape == b.shape, k
        assert np.abs(a - b).max() <= 1e-10 * max(np.abs(a).max(), 1.0), k


def test_zero_volume_particles_removed_every_substep():
    """terminateParticles runs in every sub-step (WetClothCore.cpp:97), so its
    removeEmptyParticles drops liquid particles without fluid volume even
    with no terminator: the same particles leave, the survivors take the same
    slots, and the step agrees to the step tolerances."""
    sc = _scene("dam16")
    sc.vol = sc.vol.copy()
    sc.vol[[3, 100, 101, len(sc.vol) - 2]] = 0.0
    r = oref.RefScene(sc, mic=True)
    o = oo.OracleScene(sc)
    r.step(DT, snapshot=True)
    o.step(DT, snapshot=True)
    assert int(r.get("terminate_removed")[0]) == 4
    assert int(o.get("terminate_removed")[0]) == 4
    for k in ("adv_x", "adv_v", "g2p_C"):
        a, b = r.get(k), o.get(k)
        assert a.shape == b.shape, k
        assert np.abs(a - b).max() <= 1e-10 * max(np.abs(a).max(), 1.0), k


@pytest.mark.parametrize("kind", ["dam16", "curl16"])
def test_harness_replay_matches_reference_stepsystem(kind):
    """The harness replays WetClothCore::stepSystem stage by stage
    (oracle/ref_harness.cpp); here it is checked against the reference's own
    stepSystem (WetClothCore.cpp:45-330) on a second copy of the scene, three
    steps.  correction_step 1 makes correctLiquidParticles' subset every
    particle, whatever rand() draws; the particle cell multiplier makes every
    particle 'optimal', so the split and merge that stepSystem runs leave the
    particles alone.  Positions, velocities and affine matrices agree to
    1e-14 of their largest value."""
    import math
    sc = _scene(kind)
    sc.params.correction_step = 1
    ppc = 8 if kind == "dam16" else 2
    sc.params.particle_cell_multiplier = (math.sqrt(3.0) * scenes.particle_radius(sc.params.dx, ppc)
                                          / sc.params.dx)
    a = oref.RefScene(sc, mic=False)
    b = oref.RefScene(sc, mic=False)
    for _ in range(3):
        a.step(DT, snapshot=True)
        b.core_step(DT)
    for k in ("adv_x", "g2p_v", "g2p_C"):
        x, y = a.get(k), b.get(k)
        assert x.shape == y.shape, k
        assert np.abs(x - y).max() <= 1e-14 * max(np.abs(x).max(), 1.0), k
    a.close()
    b.close()
