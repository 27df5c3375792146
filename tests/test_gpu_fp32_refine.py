"""FP32 transfers and PCG with FP64 reductions and iterative refinement,
against the FP64 oracle.

The FP32 form solves its own (FP32-assembled) system to the requested
relative residual, measured in FP64; the error of every result against the
FP64 oracle is then bounded by the FP32 rounding of the inputs plus the
solver tolerance.  Tolerances below: pressure 1e-5 relative to its maximum at
a 1e-8 criterion on both sides, particle velocities 1e-5, positions 1e-6
(positions are stored in FP32)."""
import numpy as np
import pytest

from libwetcloth_b200 import _capi, scenes
from libwetcloth_b200.solver import FluidScene
from oracle import oracle as oo

pytestmark = pytest.mark.gpu
DT = 1e-3


@pytest.mark.parametrize("kind", ["dam16", "curl32"])
def test_fp32_refine_against_fp64_oracle(kind, wcg):
    sc = scenes.dam_break(16, 8, 0) if kind == "dam16" else \
        scenes.half_box(32, 2, 5, amplitude=0.5, sigma_cells=2.0)
    sc.params.criterion = 1e-8
    o = oo.OracleScene(sc)
    o.step(DT, snapshot=True)
    g = FluidScene(sc, precision=_capi.WCG_FP32_REFINE)
    g.rebucketize_and_resample()
    assert np.array_equal(g.ifield("active"), o.get("active"))
    g.map_particle_nodes()
    g.step_velocity(DT)
    g.project_fine(DT)
    st = g.stats()
    assert st["converged"] == 1
    assert st["residual"] <= 1e-8 * st["rhs_norm"]     # FP64 residual of the FP32 system
    p, po = g.field("pressure"), o.get("pressure")
    m = ~np.isnan(po)
    assert np.abs(p[m] - po[m]).max() <= 1e-5 * np.abs(po[m]).max()
    g.apply_pressure_drag_fluid(DT)
    g.constrain_liquid_velocity()
    g.correct_liquid_particles(DT)  # every sub-step (projection only at strength 0)
    g.map_node_particles()
    g.advect(DT)
    x, v, C = g.download()
    n = sc.x.shape[0]
    ov = o.get("g2p_v").reshape(n, 3)
    assert np.abs(v - ov).max() <= 1e-5 * np.abs(ov).max()
    assert np.abs(x - o.get("adv_x").reshape(n, 3)).max() <= 1e-6
    g.close()


def test_fp32_refine_reaches_criterion(wcg):
    sc = scenes.half_box(32, 2, 5, amplitude=0.5, sigma_cells=2.0)
    for crit in (1e-6, 1e-8):
        sc.params.criterion = crit
        g = FluidScene(sc, precision=_capi.WCG_FP32_REFINE)
        g.step(DT)
        st = g.stats()
        assert st["converged"] == 1
        assert st["residual"] <= crit * st["rhs_norm"]
        g.close()
