"""The reference-side binding, compiled and run: GpuWetClothCore
(oracle/binding/GpuWetClothCore.h, a WetClothCore subclass over the C-ABI)
steps a reference TwoDScene beside the reference's own
WetClothCore::stepSystem (libWetCloth/Core/WetClothCore.cpp:45-330) on a
second TwoDScene built from the same inputs.

The binding reads everything from the reference objects themselves: the
liquid particles, LiquidInfo, the gravity of the scene's SimpleGravityForce
and the solid box of its distance fields (fillGravityAndBox).  The whole
reference step runs, including terminateParticles, updateOptiVolume, the
split and merge, correctLiquidParticles and the calls that are no-ops for
liquid.  Two scene settings make the reference's rand() draws irrelevant,
so that the comparison is exact: the particle cell multiplier makes every
particle 'optimal' (the split and merge leave the particles alone), and
correction_step 1 makes every particle the correction's subset (at strength
0 it projects the particles that reach into the walls back out).  With the
reference's own solver (multigrid-PCG) the states agree to the multigrid
parity tolerances."""
import math

import numpy as np
import pytest

from libwetcloth_b200 import _capi, scenes
from oracle import ref as oref

pytestmark = pytest.mark.gpu
DT = 1e-3


def _prepare(sc, ppc):
    sc.params.particle_cell_multiplier = (math.sqrt(3.0) * scenes.particle_radius(sc.params.dx, ppc)
                                          / sc.params.dx)
    sc.params.correction_step = 1
    return sc


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("kind", ["dam16", "curl16"])
def test_binding_matches_reference_stepsystem_fp64(kind, wcg):
    if not oref.binding_available():
        pytest.skip("oracle/_ref/libwcbinding.so not built")
    if kind == "dam16":
        sc, ppc = scenes.dam_break(16, 8, 0), 8
    else:
        sc, ppc = scenes.half_box(16, 2, 7, amplitude=1.0, sigma_cells=1.5), 2
    (xr, vr, Cr), (xg, vg, Cg), sub = oref.binding_step_both(
        _prepare(sc, ppc), 3, DT, _capi.WCG_SOLVER_MG, _capi.WCG_FP64)
    assert xr.shape == xg.shape == sc.x.shape
    assert sub >= 1
    assert _rel(xg, xr) <= 1e-11, _rel(xg, xr)
    assert _rel(vg, vr) <= 1e-8, _rel(vg, vr)
    assert _rel(Cg, Cr) <= 1e-8, _rel(Cg, Cr)


def test_binding_matches_reference_stepsystem_fp32(wcg):
    """The binding with the mixed-precision form: FP32 transfers and solve
    with FP64 refinement, within the FP32 tolerances of the oracle tests."""
    if not oref.binding_available():
        pytest.skip("oracle/_ref/libwcbinding.so not built")
    sc = scenes.dam_break(16, 8, 0)
    (xr, vr, Cr), (xg, vg, Cg), _ = oref.binding_step_both(
        _prepare(sc, 8), 2, DT, _capi.WCG_SOLVER_MG, _capi.WCG_FP32_REFINE)
    assert np.abs(xg - xr).max() <= 1e-6
    assert _rel(vg, vr) <= 1e-5, _rel(vg, vr)


def test_binding_with_terminator_objects_fp64(wcg):
    """The binding reads the scene's terminator objects (a sphere cutting the
    dam block and a rotated cylinder through it) into wcg_set_terminators:
    the same particles leave in every sub-step and the states agree."""
    if not oref.binding_available():
        pytest.skip("oracle/_ref/libwcbinding.so not built")
    sc = scenes.dam_break(16, 8, 0)
    shapes = [
        {"type": "sphere", "inside": False, "center": (0.2, 0.4, 0.2), "param": (0.08, 0, 0, 0),
         "group": 1},
        {"type": "cylinder", "inside": False, "center": (0.3, 0.6, 0.1), "axis": (1.0, 0.0, 0.0),
         "angle": 0.5, "param": (0.06, 0.01, 0.2, 0), "group": 2},
    ]
    (xr, vr, Cr), (xg, vg, Cg), _ = oref.binding_step_both(
        _prepare(sc, 8), 3, DT, _capi.WCG_SOLVER_MG, _capi.WCG_FP64, terminators=shapes)
    assert xr.shape == xg.shape and xr.shape[0] < sc.x.shape[0]
    assert _rel(xg, xr) <= 1e-11, _rel(xg, xr)
    assert _rel(vg, vr) <= 1e-8, _rel(vg, vr)
    assert _rel(Cg, Cr) <= 1e-8, _rel(Cg, Cr)
