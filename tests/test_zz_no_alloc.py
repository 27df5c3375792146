"""The allocation-free pressure solve, checked against wcg_project_fine.

wcg_pressure_solve_noalloc serves callers that cannot call cudaMalloc (an
application that owns all device memory, a strict pool or budget, code that
must not allocate between frames): it takes all solver scratch from a static
device array.  Here a scene runs through the normal C-ABI up to
wcg_project_fine; its assembled system (DOF mask, diagonal, couplings, rhs) is
copied into device buffers owned by the test and solved twice in a row by the
allocation-free entry point.  Both results must match the pressure
wcg_project_fine produced, within the 1e-9 relative tolerance the other
pressure tests use.  One scene's grid has exactly the 2048-bucket limit
(16 x 8 x 16 buckets), so the copies and kernels reach the last offsets of
the static array.
"""
import ctypes

import numpy as np
import pytest

from libwetcloth_b200 import _capi, scenes
from libwetcloth_b200.solver import FluidScene

pytestmark = pytest.mark.gpu

DT = 1e-3


def _assembled(sc):
    g = FluidScene(sc)
    g.rebucketize_and_resample()
    g.map_particle_nodes()
    g.step_velocity(DT)
    g.project_fine(DT)
    dims, _, _ = g.grid_info()
    dof = g.ifield("dof_index") >= 0
    fields = {k: np.nan_to_num(g.field(k), nan=0.0)
              for k in ("A_diag", "A_x", "A_y", "A_z", "b_dense", "pressure")}
    iters = g.stats()["pcg_iters"]
    crit = sc.params.criterion
    maxit = sc.params.maxiters
    g.close()
    return dims, dof, fields, iters, crit, maxit


def _scene(kind):
    if kind == "dam16":
        return scenes.dam_break(16, 8, 0)
    if kind == "curl32":
        return scenes.half_box(32, 2, 5, amplitude=0.5, sigma_cells=2.0)
    # a thin block whose grid is exactly 16 x 8 x 16 = 2048 buckets
    return scenes.dam_break(48, 2, 0, block_hi=(0.7, 0.1, 0.7))


@pytest.mark.parametrize("kind", ["dam16", "curl32", "limit2048"])
def test_noalloc_matches_project_fine(kind, wcg):
    import torch
    sc = _scene(kind)
    dims, dof, f, iters_ref, crit, maxit = _assembled(sc)
    if kind == "limit2048":
        assert int(np.prod(dims)) == 2048, dims
    dev = torch.device("cuda:0")
    d_dof = torch.from_numpy(dof.astype(np.uint8)).to(dev)
    d = {k: torch.from_numpy(np.ascontiguousarray(f[k])).to(dev)
         for k in ("A_diag", "A_x", "A_y", "A_z", "b_dense")}
    stream = torch.cuda.current_stream(dev).cuda_stream
    ref = f["pressure"][dof]
    scale = np.abs(ref).max()
    prev = None
    for call in range(2):
        out = torch.full((dof.size,), float("nan"), dtype=torch.float64, device=dev)
        iters = ctypes.c_int(-1)
        res = ctypes.c_double(-1.0)
        rc = wcg.wcg_pressure_solve_noalloc(
            int(dims[0]), int(dims[1]), int(dims[2]), d_dof.data_ptr(),
            d["A_diag"].data_ptr(), d["A_x"].data_ptr(), d["A_y"].data_ptr(),
            d["A_z"].data_ptr(), d["b_dense"].data_ptr(), out.data_ptr(), crit, maxit,
            stream, ctypes.byref(iters), ctypes.byref(res))
        assert rc == _capi.WCG_OK, wcg.wcg_last_error().decode()
        torch.cuda.synchronize(dev)
        p = out.cpu().numpy()
        assert np.all(p[~dof] == 0.0)
        err = np.abs(p[dof] - ref).max() / scale
        assert err <= 1e-9, f"call {call}: relative error {err:.3e}"
        assert abs(iters.value - iters_ref) <= 1, (iters.value, iters_ref)
        if prev is not None:
            assert np.abs(p - prev).max() <= 1e-9 * scale
        prev = p


def test_noalloc_rejects_oversized_grid(wcg):
    iters = ctypes.c_int(0)
    res = ctypes.c_double(0)
    # 16 x 16 x 16 buckets = 4096 > 2048: rejected before any device work
    rc = wcg.wcg_pressure_solve_noalloc(16, 16, 16, 1, 1, 1, 1, 1, 1, 1, 1e-6, 10,
                                        None, ctypes.byref(iters), ctypes.byref(res))
    assert rc == _capi.WCG_ERR_ARG
    assert b"limit" in wcg.wcg_last_error()
