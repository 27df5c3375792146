"""State files in the reference's formats (App/TwoDSceneSerializer.cpp).

serializePositionOnly writes an int byte count, m_x (x, y, z and the yarn
twist per particle, doubles) and an int byte count for the cloth Gauss points;
loadPosOnly reads the same.  The fluid OBJ has one "v x y z radius" line per
fluid particle at 8 significant digits.  The tests read the files with numpy
by that layout, check them against the particle state downloaded through the
C-ABI, and check the load path by a round trip."""
import struct

import numpy as np
import pytest

from libwetcloth_b200 import _capi, scenes
from libwetcloth_b200.solver import FluidScene

pytestmark = pytest.mark.gpu
DT = 1e-3


def _read_pos(path):
    with open(path, "rb") as f:
        data = f.read()
    nb = struct.unpack_from("<i", data, 0)[0]
    x4 = np.frombuffer(data, dtype="<f8", count=nb // 8, offset=4).reshape(-1, 4)
    ng = struct.unpack_from("<i", data, 4 + nb)[0]
    assert len(data) == 4 + nb + 4 + ng
    return x4, ng


@pytest.mark.parametrize("precision", [_capi.WCG_FP64, _capi.WCG_FP32_REFINE])
def test_position_file_layout_and_round_trip(tmp_path, precision, wcg):
    sc = scenes.dam_break(16, 8, 0)
    g = FluidScene(sc, precision=precision)
    g.step(DT)
    x, _, _ = g.download()
    path = tmp_path / "pos.bin"
    g.save_positions(path)
    x4, ng = _read_pos(path)
    assert ng == 0
    assert x4.shape == (sc.x.shape[0], 4)
    assert np.array_equal(x4[:, :3], x)
    assert np.all(x4[:, 3] == 0.0)
    # load a shifted copy: positions come back exactly (FP64) or rounded to FP32
    shifted = x4.copy()
    shifted[:, 1] -= 0.01
    with open(path, "wb") as f:
        f.write(struct.pack("<i", shifted.nbytes))
        f.write(shifted.astype("<f8").tobytes())
        f.write(struct.pack("<i", 0))
    g.load_positions(path)
    x2, _, _ = g.download()
    want = shifted[:, :3] if precision == _capi.WCG_FP64 else \
        shifted[:, :3].astype(np.float32).astype(np.float64)
    assert np.array_equal(x2, want)
    g.step(DT)   # the grid is rebuilt from the loaded positions
    assert g.stats()["converged"] == 1
    g.close()


def test_position_file_size_mismatch_rejected(tmp_path, wcg):
    g = FluidScene(scenes.dam_break(16, 8, 0))
    path = tmp_path / "bad.bin"
    with open(path, "wb") as f:
        f.write(struct.pack("<i", 32))
        f.write(np.zeros(4).tobytes())
        f.write(struct.pack("<i", 0))
    with pytest.raises(_capi.WcgError):
        g.load_positions(path)
    g.close()


def test_fluid_obj(tmp_path, wcg):
    sc = scenes.half_box(16, 2, 5, amplitude=0.5, sigma_cells=2.0)
    g = FluidScene(sc)
    g.step(DT)
    x, _, _ = g.download()
    path = tmp_path / "fluid.obj"
    g.write_fluid_obj(path)
    lines = open(path).read().splitlines()
    assert len(lines) == sc.x.shape[0]
    vals = np.array([[float(t) for t in ln.split()[1:]] for ln in lines])
    assert all(ln.startswith("v ") for ln in lines)
    assert np.allclose(vals[:, :3], x, rtol=1e-7, atol=1e-12)
    assert np.allclose(vals[:, 3], sc.radius, rtol=1e-7)
    g.close()


def test_async_download_overlaps_and_matches(wcg):
    """wcg_download_liquid_async: the read-back of step k, left running on the
    copy stream while the next upload and step run, equals the synchronous
    download of the same state."""
    import ctypes
    import torch
    sc = scenes.dam_break(16, 8, 0)
    g = FluidScene(sc)
    n = sc.x.shape[0]
    outs = [tuple(torch.empty(n * k, dtype=torch.float64).pin_memory() for k in (3, 3, 9))
            for _ in range(2)]
    ptr = lambda t: ctypes.cast(t.data_ptr(), ctypes.POINTER(ctypes.c_double))
    ref = []
    for k in range(4):
        g.step(1e-3)
        ref.append(g.download())
        ox, ov, oC = outs[k % 2]
        assert g.L.wcg_download_liquid_async(g.h, ptr(ox), ptr(ov), ptr(oC)) == 0
        if k % 2 == 1:
            assert g.L.wcg_synchronize(g.h) == 0
            for j in (k - 1, k):
                x, v, C = ref[j]
                bx, bv, bC = outs[j % 2]
                assert np.array_equal(bx.numpy().reshape(n, 3), x)
                assert np.array_equal(bv.numpy().reshape(n, 3), v)
                assert np.array_equal(bC.numpy().reshape(n, 9), C)
    g.close()


def test_staged_upload_matches_and_checks_input(wcg):
    """wcg_stage_liquid_async + wcg_upload_staged load the same state as
    wcg_upload_liquid, while a step is queued; bad input is caught on the
    device and the next step stops before stepping it."""
    import ctypes
    import torch
    sc = scenes.dam_break(16, 8, 0)
    n = sc.x.shape[0]
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).pin_memory()
    bufs = [pin(a) for a in (sc.x, sc.v, np.zeros((n, 9)), sc.mass, sc.vol, sc.radius)]
    ptr = lambda t: ctypes.cast(t.data_ptr(), ctypes.POINTER(ctypes.c_double))
    a = FluidScene(sc)
    a.step(1e-3)
    xa, va, Ca = a.download()
    b = FluidScene(sc)
    b.step(1e-3)  # other state first
    assert b.L.wcg_stage_liquid_async(b.h, n, *[ptr(t) for t in bufs]) == 0
    b.step(1e-3)  # runs while the copies are in flight; replaced by the staged set
    assert b.L.wcg_upload_staged(b.h) == 0
    b.set_correction_count(0)  # the correction subset a's first step took
    b.step(1e-3)
    xb, vb, Cb = b.download()
    assert np.array_equal(xa, xb) and np.array_equal(va, vb) and np.array_equal(Ca, Cb)
    bufs[1][5] = float("nan")
    assert b.L.wcg_stage_liquid_async(b.h, n, *[ptr(t) for t in bufs]) == 0
    assert b.L.wcg_upload_staged(b.h) == 0
    assert b.L.wcg_step(b.h, 1e-3, None) == _capi.WCG_ERR_DEVICE
    assert b"invalid particle input" in b.L.wcg_last_error()
    a.close()
    b.close()
