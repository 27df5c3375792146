"""Independent scenes stepped together (wcg_batch_*) against each scene
stepped alone: the batch only overlaps the scenes' kernels on separate
streams from several host threads, so every particle state is bit-identical.
Scenes of uneven size, density and viscosity (the seeded generator of the
many-scenes benchmark configuration)."""
import numpy as np
import pytest

from libwetcloth_b200 import _capi, scenes
from libwetcloth_b200.solver import FluidBatch, FluidScene

pytestmark = pytest.mark.gpu
DT = 1e-3


@pytest.mark.parametrize("precision", [_capi.WCG_FP64, _capi.WCG_FP32_REFINE])
def test_batch_matches_scenes_alone(precision, wcg):
    specs = scenes.batch_scenes(7, 5, (16, 32), (2000, 20000))
    alone = []
    for sc in specs:
        g = FluidScene(sc, precision=precision)
        g.step(DT)
        g.step(DT)
        alone.append(g.download())
        g.close()
    gs = [FluidScene(sc, precision=precision) for sc in specs]
    b = FluidBatch(gs)
    b.threads = 4
    st = b.step(DT, nsteps=2)
    assert all(s == _capi.WCG_OK for s in st), st
    for g, ref in zip(gs, alone):
        for a, r in zip(g.download(), ref):
            assert np.array_equal(a, r)
    b.close()
    for g in gs:
        g.close()


def test_batch_autotune_and_per_scene_dt(wcg):
    specs = scenes.batch_scenes(5, 6, (16, 24), (2000, 8000))
    gs = [FluidScene(sc) for sc in specs]
    b = FluidBatch(gs)
    times = b.autotune(DT, candidates=(1, 2, 4))
    assert set(times) == {1, 2, 4} and b.threads in (1, 2, 4)
    assert all(t > 0 for t in times.values())
    dts = np.array([1e-3, 5e-4, 1e-3, 2e-3, 1e-3])
    b.step(dts)
    for g in gs:
        assert np.all(np.isfinite(g.download()[0]))
    b.close()
    with pytest.raises(_capi.WcgError):
        FluidBatch([])
    for g in gs:
        g.close()


def test_batch_with_particle_maintenance_matches_alone(wcg):
    """Scenes with the correction, split and merge on (each its own seeded
    streams, particle counts changing between steps) step in a batch exactly
    as they step alone."""
    specs = scenes.batch_scenes(5, 9, (16, 32), (2000, 20000))
    for k, sc in enumerate(specs):
        scenes.mixed_volumes(sc, k, mrel=(0.3, 0.7, 1.0, 2.5, 5.0))
        sc.params.correction_strength = 0.2
        sc.params.correction_seed = k
        sc.params.particle_split = True
        sc.params.split_seed = 10 + k
        sc.params.particle_merge = True
        sc.params.merge_seed = 20 + k
    alone = []
    for sc in specs:
        g = FluidScene(sc)
        for _ in range(3):
            g.step(DT)
        alone.append(g.download())
        g.close()
    gs = [FluidScene(sc) for sc in specs]
    b = FluidBatch(gs)
    b.threads = 3
    st = b.step(DT, nsteps=3)
    assert all(s == _capi.WCG_OK for s in st), st
    for g, ref, sc in zip(gs, alone, specs):
        assert g.num_particles != sc.x.shape[0]
        for a, r in zip(g.download(), ref):
            assert np.array_equal(a, r)
    b.close()
    for g in gs:
        g.close()


def test_schedule_autotune_keeps_results(wcg):
    """The per-scene schedule autotuner (sweep-cluster shape and PCG
    iterations per host check, chosen from each scene's timed steps) changes
    no result: after the tuning trials (one step per candidate) and two more
    batch steps, every scene is bit-identical to the same number of steps
    taken alone with the default schedule.  Scenes up to 96^3 so the
    clustered sweeps have patches to cluster."""
    specs = scenes.batch_scenes(5, 11, (32, 96), (20000, 400000))
    cands = [(0, 1, 8), (1, 1, 8), (2, 1, 8), (4, 1, 4), (1, 4, 16), (2, 8, 2)]
    nsteps = len(cands) + 2
    alone = []
    for sc in specs:
        g = FluidScene(sc, precision=_capi.WCG_FP32_REFINE)
        for _ in range(nsteps):
            g.step(DT)
        alone.append(g.download())
        g.close()
    gs = [FluidScene(sc, precision=_capi.WCG_FP32_REFINE) for sc in specs]
    b = FluidBatch(gs)
    b.threads = 3
    chosen, ms = b.autotune_schedules(DT, cands)
    assert ms.shape == (len(specs), len(cands)) and np.all(ms > 0)
    for g, k in zip(gs, chosen):
        assert g.schedule == cands[k]
        assert k == int(np.argmin(ms[gs.index(g)]))
    st = b.step(DT, nsteps=2)
    assert all(s == _capi.WCG_OK for s in st), st
    for g, ref in zip(gs, alone):
        for a, r in zip(g.download(), ref):
            assert np.array_equal(a, r)
    b.close()
    for g in gs:
        g.close()


def test_schedule_arguments(wcg):
    sc = scenes.batch_scenes(1, 3, (16, 16), (2000, 2000))[0]
    g = FluidScene(sc)
    assert g.schedule == (0, 1, 8)
    g.schedule = (9, 1, 32)
    assert g.schedule == (9, 1, 32)
    for bad in [(5, 1, 8), (8, 4, 8), (0, 4, 8), (4, 8, 8), (1, 2, 8), (1, 1, 0), (1, 1, 65)]:
        with pytest.raises(_capi.WcgError):
            g.schedule = bad
    assert g.schedule == (9, 1, 32)
    g.close()


@pytest.mark.parametrize("mixed,limit", [(False, None), (True, None), (False, 4)])
def test_shared_solve_matches_alone(mixed, limit, wcg):
    """The shared solve (the PCG iterations of all scenes waiting in their
    pressure solve run as one launch per kernel) changes no result: every
    scene after three batch steps is bit-identical to three steps alone.
    Scenes of uneven size; FP32 + refinement, and a batch mixing FP64 and
    FP32 scenes (two shared launch sets); some scenes on cluster schedules,
    whose sweeps outside the iterations keep them; and a patch limit under
    which the larger scene iterates alone beside the shared launches."""
    if limit is None:
        specs = scenes.batch_scenes(6, 13, (24, 72), (5000, 150000))
    else:
        # the two 16^3 dam breaks solve on a 20 x 28 x 20-cell DOF box (2 x 2
        # pencil patches) and share the launches; the 48^3 half box (3 x 4
        # patches) iterates alone
        specs = [scenes.dam_break(16, 8, 0), scenes.dam_break(16, 8, 1),
                 scenes.half_box(48, 2, 5, amplitude=0.5, sigma_cells=2.0)]
    precs = [(_capi.WCG_FP64 if (mixed and k % 2) else _capi.WCG_FP32_REFINE)
             for k in range(len(specs))]
    alone = []
    for sc, pr in zip(specs, precs):
        g = FluidScene(sc, precision=pr)
        for _ in range(3):
            g.step(DT)
        alone.append((g.download(), g.stats()["pcg_iters"]))
        g.close()
    gs = [FluidScene(sc, precision=pr) for sc, pr in zip(specs, precs)]
    for k, g in enumerate(gs):
        if k % 3 == 1:
            g.schedule = (2, 1, 4)
    b = FluidBatch(gs)
    b.threads = 4
    b.set_shared_solve(True, max_patches=limit)
    st = b.step(DT, nsteps=3)
    assert all(s == _capi.WCG_OK for s in st), st
    assert b.shared_launches > 0
    for g, (ref, it) in zip(gs, alone):
        assert g.stats()["pcg_iters"] == it
        for a, r in zip(g.download(), ref):
            assert np.array_equal(a, r)
    # off again: the scenes solve alone
    b.set_shared_solve(False)
    n0 = b.shared_launches
    st = b.step(DT)
    assert all(s == _capi.WCG_OK for s in st), st
    assert b.shared_launches == n0
    b.close()
    for g in gs:
        g.close()
