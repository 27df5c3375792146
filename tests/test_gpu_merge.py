"""Particle merge (relabelLiquidParticles, mergeLiquidParticles,
removeEmptyParticles) on the GPU against the oracle.

The oracle's restatement is pinned to the reference, with the reference's own
rand() draws, in tests/test_oracle_vs_reference.py::test_particle_merge.  Here
the GPU merges scenes of mixed particle volume after a step, with explicit
draws, and whole steps with the merge on draw from the seeded stream both
sides share.  The removed particles and the renumbering of the survivors are
exact; positions, velocities and affine matrices agree to 1e-12 relative
(FP64), and a step after the merge (which reads the merged volumes, masses and
radii) to the step tolerances."""
import numpy as np
import pytest

from libwetcloth_b200 import _capi, scenes
from libwetcloth_b200.solver import FluidScene
from oracle import oracle as oo
from oracle import ref as oref
from tests.parity import TERMINATOR_SHAPES

pytestmark = pytest.mark.gpu
DT = 1e-3


def _close(a, b, tol, name, scale=0.0):
    a = np.asarray(a).reshape(-1)
    b = np.asarray(b).reshape(-1)
    assert a.shape == b.shape, name
    s = max(np.abs(b).max(), scale, 1e-300)
    err = np.abs(a - b).max() / s
    assert err <= tol, f"{name}: {err:.3e}"


def _scene(kind, seed):
    if kind == "dam16":
        sc = scenes.dam_break(16, 8, 0)
    elif kind == "curl16":
        sc = scenes.half_box(16, 2, 7, amplitude=1.0, sigma_cells=1.5)
    else:
        sc = scenes.dam_break(16, 8, 0)
        sc.v[:, 1] = -3.0
    return scenes.mixed_volumes(sc, seed)


@pytest.mark.parametrize("kind,seed,sel", [("dam16", 3, 2), ("curl16", 5, 3), ("fall", 8, 0)])
def test_merge_after_step_fp64(kind, seed, sel, wcg):
    perm = [2, 0, 1, 1, 2, 0, 0, 2, 1]
    sc = _scene(kind, seed)
    o = oo.OracleScene(sc)
    o.step(DT, snapshot=True)
    g = FluidScene(sc)
    g.step(DT)
    n0 = g.num_particles
    nrem = g.merge_liquid_particles(sel, perm)
    assert nrem == o.merge(sel, perm)
    assert nrem > 0 and g.num_particles == n0 - nrem
    x, v, C = g.download()
    _close(x, o.get("merge_x"), 1e-12, "x")
    _close(v, o.get("merge_v"), 1e-12, "v")
    _close(C, o.get("merge_C"), 1e-12, "C")
    # the next step reads the merged volumes, masses and radii
    o.step(DT, snapshot=True)
    g.step(DT)
    x, v, C = g.download()
    _close(v, o.get("g2p_v"), 1e-10, "g2p_v")
    _close(x, o.get("adv_x"), 1e-12, "adv_x")
    g.close()


def test_merge_seeded_steps(wcg):
    """wcg_step with the merge on, both sides drawing from the same seeded
    stream (wcg_merge_draws), in FP64 and FP32."""
    sc = _scene("dam16", 11)
    sc.params.particle_merge = True
    sc.params.merge_seed = 9
    o = oo.OracleScene(sc)
    g = FluidScene(sc)
    g32 = FluidScene(sc, precision=_capi.WCG_FP32_REFINE)
    n0 = sc.x.shape[0]
    for _ in range(3):
        o.step(DT, snapshot=True)
        g.step(DT)
        g32.step(DT)
    n = int(o.get("adv_x").size // 3)
    assert n < n0
    assert g.num_particles == n and g32.num_particles == n
    x, v, C = g.download()
    _close(v, o.get("g2p_v"), 1e-10, "g2p_v")
    _close(x, o.get("adv_x"), 1e-12, "adv_x")
    x, v, C = g32.download()
    _close(v, o.get("g2p_v"), 1e-5, "g2p_v fp32")
    _close(x, o.get("adv_x"), 1e-6, "adv_x fp32")
    g.close()
    g32.close()


def test_merge_arguments(wcg):
    sc = _scene("dam16", 3)
    g = FluidScene(sc)
    with pytest.raises(_capi.WcgError) as e:
        g.merge_liquid_particles(0, [0, 1, 2] * 3)  # no grid build yet
    assert e.value.code == _capi.WCG_ERR_STATE
    g.step(DT)
    for sel, perm in ((8, [0, 1, 2] * 3), (0, [0, 0, 1] + [0, 1, 2] * 2)):
        with pytest.raises(_capi.WcgError) as e:
            g.merge_liquid_particles(sel, perm)
        assert e.value.code == _capi.WCG_ERR_ARG
    g.close()


@pytest.mark.parametrize("kind,seed", [("dam16", 3), ("curl16", 5)])
def test_split_after_step_fp64(kind, seed, wcg):
    """splitLiquidParticles (seeded pattern and rotations, the same on both
    sides): the particles added, their order, positions, velocities and
    affine matrices to 1e-12, then a step that reads their volumes, masses
    and radii."""
    sc = _scene(kind, seed)
    scenes.mixed_volumes(sc, seed, mrel=(0.3, 1.0, 2.5, 7.0, 40.0))
    key = 0x9E3779B97F4A7C15 ^ seed
    o = oo.OracleScene(sc)
    o.step(DT, snapshot=True)
    g = FluidScene(sc)
    g.step(DT)
    n0 = g.num_particles
    added = g.split_liquid_particles(key)
    assert added == o.split(key) and added > 0
    assert g.num_particles == n0 + added
    x, v, C = g.download()
    _close(x, o.get("split_x"), 1e-12, "x")
    _close(v, o.get("split_v"), 1e-12, "v")
    _close(C, o.get("split_C"), 1e-12, "C")
    o.step(DT, snapshot=True)
    g.step(DT)
    x, v, C = g.download()
    _close(v, o.get("g2p_v"), 1e-10, "g2p_v")
    _close(x, o.get("adv_x"), 1e-12, "adv_x")
    g.close()


@pytest.mark.parametrize("kind,seed", [("dam16", 3), ("curl16", 5)])
def test_split_reference_placement_fp64(kind, seed, wcg):
    """splitLiquidParticles placed as the reference places it
    (TwoDScene.cpp:2362-2480): the reference's sphere-pattern table and the
    rotations its serial build draws after srand(seed) go in through
    wcg_split_liquid_particles_with.  After one step on both sides, the
    particles added, their order, positions, velocities and affine matrices
    agree with the reference's own splitLiquidParticles, and so does the next
    step, which reads the children's volumes, masses and radii.  A rotation
    count other than the number of splitting parents is refused with the
    state unchanged."""
    if not oref.available():
        pytest.skip("oracle/_ref not built")
    sc = _scene(kind, seed)
    scenes.mixed_volumes(sc, seed, mrel=(0.3, 1.0, 2.5, 7.0, 40.0))
    r = oref.RefScene(sc, mic=True)
    r.step(DT, snapshot=True)
    g = FluidScene(sc)
    g.step(DT)
    n0 = g.num_particles
    pattern, rot = r.split_inputs(seed)
    assert pattern.shape == (1581,)
    assert g.split_parents() == rot.shape[0] > 0
    with pytest.raises(_capi.WcgError) as e:
        g.split_liquid_particles_with(pattern, rot[:-1])
    assert e.value.code == _capi.WCG_ERR_ARG and g.num_particles == n0
    added = g.split_liquid_particles_with(pattern, rot)
    assert added == r.split(seed) and added > 0
    assert g.num_particles == n0 + added
    x, v, C = g.download()
    _close(x, r.get("split_x"), 1e-12, "x")
    _close(v, r.get("split_v"), 1e-9, "v")
    _close(C, r.get("split_C"), 1e-9, "C", scale=4 * 16 * np.abs(v).max())
    r.step(DT, snapshot=True)
    g.step(DT)
    x, v, C = g.download()
    _close(v, r.get("g2p_v"), 1e-9, "g2p_v")
    _close(x, r.get("adv_x"), 1e-12, "adv_x")
    g.close()
    r.close()


def test_split_and_merge_seeded_steps(wcg):
    """wcg_step with the split and the merge on (split first, the merge on
    the re-sorted buckets), both sides drawing from the same seeded streams,
    in FP64 and FP32; the particle count grows past the first capacity."""
    sc = _scene("dam16", 13)
    scenes.mixed_volumes(sc, 13, mrel=(0.3, 0.7, 1.0, 2.5, 7.0))
    sc.params.particle_split = True
    sc.params.split_seed = 21
    sc.params.particle_merge = True
    sc.params.merge_seed = 4
    o = oo.OracleScene(sc)
    g = FluidScene(sc)
    g32 = FluidScene(sc, precision=_capi.WCG_FP32_REFINE)
    n0 = sc.x.shape[0]
    for _ in range(3):
        o.step(DT, snapshot=True)
        g.step(DT)
        g32.step(DT)
    n = int(o.get("adv_x").size // 3)
    assert n > n0
    assert g.num_particles == n and g32.num_particles == n
    x, v, C = g.download()
    _close(v, o.get("g2p_v"), 1e-10, "g2p_v")
    _close(x, o.get("adv_x"), 1e-12, "adv_x")
    x, v, C = g32.download()
    _close(v, o.get("g2p_v"), 1e-5, "g2p_v fp32")
    _close(x, o.get("adv_x"), 1e-6, "adv_x fp32")
    g.close()
    g32.close()


def _terminator_scene(inside=True):
    sc = scenes.half_box(16, 2, 7, amplitude=1.0, sigma_cells=1.5)
    lo, hi = sc.x.min(axis=0), sc.x.max(axis=0)
    p = sc.params
    p.terminator = True
    p.terminator_center = tuple(0.5 * (lo + hi))
    p.terminator_half = tuple(0.3 * (hi - lo))
    p.terminator_radius = 0.25 * p.dx
    p.terminator_inside = inside
    return sc


@pytest.mark.parametrize("inside", [True, False])
def test_terminate_call_fp64(inside, wcg):
    """terminateParticles on its own (tests/test_oracle_vs_reference.py pins
    the oracle's to the reference): the same particles removed, the survivors
    in the same order, bit-exact (the removal only moves particles)."""
    sc = _terminator_scene(inside)
    o = oo.OracleScene(sc)
    g = FluidScene(sc)
    rem = g.terminate_liquid_particles()
    assert 0 < rem < sc.x.shape[0]
    assert o.terminate() == rem
    x, v, C = g.download()
    assert np.array_equal(x.reshape(-1), o.get("term_x").reshape(-1))
    assert np.array_equal(v.reshape(-1), o.get("term_v").reshape(-1))
    assert g.terminate_liquid_particles() == 0
    g.close()


@pytest.mark.parametrize("prec", [_capi.WCG_FP64, _capi.WCG_FP32_REFINE])
def test_terminator_steps(prec, wcg):
    """Three steps, each sub-step starting with terminateParticles: FP64 agrees
    with the oracle on the removals (count and order) and the state to the
    step tolerances; FP32 on the count (its positions are rounded, so a
    particle on the box's surface may fall the other way) and, when the
    counts match, the state to 1e-5 / 1e-6."""
    sc = _terminator_scene(True)
    o = oo.OracleScene(sc)
    g = FluidScene(sc, precision=prec)
    removed = 0
    for _ in range(3):
        o.step(DT, snapshot=True)
        g.step(DT)
        removed += int(o.get("terminate_removed")[0])
    assert removed > 0
    x, v, C = g.download()
    ox = o.get("adv_x").reshape(-1, 3)
    if prec == _capi.WCG_FP64:
        _close(v, o.get("g2p_v"), 1e-10, "g2p_v")
        _close(x, ox, 1e-12, "adv_x")
    else:
        assert abs(x.shape[0] - ox.shape[0]) <= 2
        if x.shape[0] == ox.shape[0]:
            _close(v, o.get("g2p_v"), 1e-5, "g2p_v")
            _close(x, ox, 1e-6, "adv_x")
    g.close()


def _terminator_shapes():
    """Rotated terminator objects of all four analytic types (the set the
    oracle is pinned to the reference with), rotations from their axes and
    angles."""
    out = []
    for sh in TERMINATOR_SHAPES:
        ax = np.array(sh.get("axis", (0.0, 1.0, 0.0)), dtype=np.float64)
        ang = float(sh.get("angle", 0.0))
        out.append(dict(sh, rot=(np.cos(0.5 * ang), *(np.sin(0.5 * ang) * ax))))
    return out


@pytest.mark.parametrize("prec", [_capi.WCG_FP64, _capi.WCG_FP32_REFINE])
def test_terminator_shapes(prec, wcg):
    """wcg_set_terminators with a rotated sphere, capsule, cylinder and
    inside box: a call on its own removes the same particles as the oracle
    with the survivors in the same order (FP64 bit-exact; FP32 within two
    particles, whose rounded positions may fall on the other side of a
    surface), then three steps with the terminator first in each sub-step
    agree with the oracle's (FP64 step tolerances); clearing the shapes
    stops the removals."""
    sc = scenes.half_box(16, 2, 7, amplitude=1.0, sigma_cells=1.5)
    shapes = _terminator_shapes()
    o = oo.OracleScene(sc)
    o.set_terminators(shapes)
    g = FluidScene(sc, precision=prec)
    g.set_terminators(shapes)
    rem = g.terminate_liquid_particles()
    orem = o.terminate()
    assert orem > 0
    if prec == _capi.WCG_FP64:
        assert rem == orem
        x, v, _ = g.download()
        assert np.array_equal(x.reshape(-1), o.get("term_x").reshape(-1))
        assert np.array_equal(v.reshape(-1), o.get("term_v").reshape(-1))
        removed = 0
        for _ in range(3):
            o.step(DT, snapshot=True)
            g.step(DT)
            removed += int(o.get("terminate_removed")[0])
        x, v, C = g.download()
        assert x.shape[0] == o.get("adv_x").size // 3
        _close(v, o.get("g2p_v"), 1e-10, "g2p_v")
        _close(x, o.get("adv_x"), 1e-12, "adv_x")
    else:
        assert abs(rem - orem) <= 2
    g.set_terminators([])
    n = g.num_particles
    g.step(DT)
    assert g.num_particles == n
    g.close()


@pytest.mark.parametrize("split", [False, True])
def test_terminator_then_merge_steps(split, wcg):
    """The terminator removes particles first in each sub-step; the merge
    after it pairs the survivors in buckets re-sorted from their current
    positions (removeEmptyParticles re-sorts them after any removal,
    TwoDScene.cpp:1734-1743), optionally after a split.  Three FP64 steps:
    the same removals and the same state as the oracle."""
    sc = scenes.mixed_volumes(_terminator_scene(True), 17,
                              mrel=(0.3, 0.7, 1.0, 2.5, 7.0) if split else
                              (0.3, 0.7, 1.0, 1.5, 2.5))
    sc.params.particle_merge = True
    sc.params.merge_seed = 9
    if split:
        sc.params.particle_split = True
        sc.params.split_seed = 21
    o = oo.OracleScene(sc)
    g = FluidScene(sc)
    term = 0
    for _ in range(3):
        o.step(DT, snapshot=True)
        g.step(DT)
        term += int(o.get("terminate_removed")[0])
    assert term > 0
    n = int(o.get("adv_x").size // 3)
    assert g.num_particles == n
    x, v, C = g.download()
    _close(v, o.get("g2p_v"), 1e-10, "g2p_v")
    _close(x, o.get("adv_x"), 1e-12, "adv_x")
    g.close()


@pytest.mark.parametrize("prec", [_capi.WCG_FP64, _capi.WCG_FP32_REFINE])
def test_zero_volume_particles_dropped_without_terminator(prec, wcg):
    """terminateParticles runs every sub-step (WetClothCore.cpp:97) and its
    removeEmptyParticles drops liquid particles below 1e-20 of fluid volume
    even without a terminator: uploaded zero-volume particles are gone after
    the first step, in the reference's swap-with-last order."""
    sc = scenes.dam_break(16, 8, 0)
    sc.vol = sc.vol.copy()
    sc.vol[[3, 100, 101, len(sc.vol) - 2]] = 0.0
    o = oo.OracleScene(sc)
    g = FluidScene(sc, precision=prec)
    o.step(DT, snapshot=True)
    g.step(DT)
    assert int(o.get("terminate_removed")[0]) == 4
    n = int(o.get("adv_x").size // 3)
    assert n == sc.x.shape[0] - 4 and g.num_particles == n
    x, v, C = g.download()
    if prec == _capi.WCG_FP64:
        _close(v, o.get("g2p_v"), 1e-10, "g2p_v")
        _close(x, o.get("adv_x"), 1e-12, "adv_x")
    else:
        _close(v, o.get("g2p_v"), 1e-5, "g2p_v fp32")
        _close(x, o.get("adv_x"), 1e-6, "adv_x fp32")
    # the second step has nothing left to remove
    o.step(DT, snapshot=True)
    g.step(DT)
    assert g.num_particles == n
    g.close()
