"""C-ABI checks that need no GPU: the library loads, exports every function
include/wetcloth_gpu.h declares, and reports argument errors."""
import ctypes
import os
import re

import pytest

from libwetcloth_b200 import _capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    txt = open(os.path.join(ROOT, "include", "wetcloth_gpu.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(wcg_[a-z0-9_]+)\s*\(", txt)))


def test_header_declares_entry_points():
    names = declared_functions()
    assert len(names) >= 30
    assert "wcg_step" in names and "wcg_pressure_solve_noalloc" in names


def test_library_exports_every_declared_symbol():
    L = _capi.load()
    for name in declared_functions():
        assert hasattr(L, name), f"libwcgpu.so does not export {name}"
        assert name in _capi.SIGNATURES, f"no ctypes signature for {name}"


def test_default_params():
    L = _capi.load()
    p = _capi.WcgParams()
    L.wcg_default_params(ctypes.byref(p))
    assert p.criterion == 1e-6 and p.maxiters == 1000 and p.walls == 1
    assert p.precision == _capi.WCG_FP64
    assert p.refine_inner_tol == 1e-5
    assert p.terminator == 0 and p.terminator_inside == 1
    assert list(p.terminator_half) == [0.5, 0.5, 0.5]


def test_terminator_params_checked_before_device_work():
    """A terminator box with a negative or non-finite extent is refused
    before any device is touched."""
    L = _capi.load()
    h = ctypes.c_void_p()
    p = _capi.WcgParams()
    L.wcg_default_params(ctypes.byref(p))
    p.dx = 1.0 / 16
    p.terminator = 1
    p.terminator_half[1] = -0.1
    assert L.wcg_create(ctypes.byref(p), ctypes.byref(h)) == _capi.WCG_ERR_ARG
    assert b"terminator" in L.wcg_last_error()
    p.terminator_half[1] = 0.5
    p.terminator_radius = float("nan")
    assert L.wcg_create(ctypes.byref(p), ctypes.byref(h)) == _capi.WCG_ERR_ARG
    assert L.wcg_terminate_liquid_particles(None, None) == _capi.WCG_ERR_ARG


def test_argument_errors_without_device():
    L = _capi.load()
    h = ctypes.c_void_p()
    assert L.wcg_create(None, ctypes.byref(h)) == _capi.WCG_ERR_ARG
    p = _capi.WcgParams()
    L.wcg_default_params(ctypes.byref(p))
    p.dx = -1.0
    assert L.wcg_create(ctypes.byref(p), ctypes.byref(h)) == _capi.WCG_ERR_ARG
    assert b"dx" in L.wcg_last_error()
    p.dx = 1.0 / 16
    p.precision = 7
    assert L.wcg_create(ctypes.byref(p), ctypes.byref(h)) == _capi.WCG_ERR_ARG
    # calls on a null context fail cleanly
    assert L.wcg_step(None, 1e-3, None) == _capi.WCG_ERR_ARG
    assert L.wcg_rebucketize_and_resample(None) == _capi.WCG_ERR_ARG
    assert L.wcg_num_particles(None) == -1
    # schedules and batches: null handles refused before any device work
    sched = _capi.WcgSchedule(1, 1, 8)
    assert L.wcg_set_schedule(None, ctypes.byref(sched)) == _capi.WCG_ERR_ARG
    assert L.wcg_get_schedule(None, ctypes.byref(sched)) == _capi.WCG_ERR_ARG
    assert L.wcg_batch_set_shared_solve(None, 1) == _capi.WCG_ERR_ARG
    assert L.wcg_batch_shared_launches(None) == -1
    assert L.wcg_batch_set_shared_solve_limit(None, 4) == _capi.WCG_ERR_ARG
    assert L.wcg_batch_autotune_schedules(None, None, None, 0, 1, None, None) == _capi.WCG_ERR_ARG
    b = ctypes.c_void_p()
    assert L.wcg_batch_create(0, None, ctypes.byref(b)) == _capi.WCG_ERR_ARG


def test_noalloc_size_limit_checked_before_device_work():
    L = _capi.load()
    it = ctypes.c_int(0)
    res = ctypes.c_double(0)
    rc = L.wcg_pressure_solve_noalloc(64, 64, 64, 1, 1, 1, 1, 1, 1, 1, 1e-6, 10, None,
                                      ctypes.byref(it), ctypes.byref(res))
    assert rc == _capi.WCG_ERR_ARG and b"limit" in L.wcg_last_error()
    rc = L.wcg_pressure_solve_noalloc(0, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1e-6, 10, None,
                                      ctypes.byref(it), ctypes.byref(res))
    assert rc == _capi.WCG_ERR_ARG


def test_correction_params_and_selector_stream():
    """Correction defaults and checks; the subset stream of wcg_step is the
    oracle's (host code, no device needed)."""
    L = _capi.load()
    p = _capi.WcgParams()
    L.wcg_default_params(ctypes.byref(p))
    assert p.correction_strength == 0.0 and p.correction_step == 8
    assert p.correction_multiplier == 2.0 and p.correction_seed == 0
    h = ctypes.c_void_p()
    p.correction_step = 0
    assert L.wcg_create(ctypes.byref(p), ctypes.byref(h)) == _capi.WCG_ERR_ARG
    assert b"correction" in L.wcg_last_error()
    p.correction_step = 8
    p.correction_strength = -0.1
    assert L.wcg_create(ctypes.byref(p), ctypes.byref(h)) == _capi.WCG_ERR_ARG
    assert L.wcg_correct_liquid_particles(None, 1e-3, 0) == _capi.WCG_ERR_ARG
    from oracle import oracle as oo
    if not oo.available():
        pytest.skip("oracle not built")
    O = oo.lib()
    seen = set()
    for seed in (0, 1, 7, 2**40 + 3):
        for k in range(50):
            for step in (1, 3, 8):
                s = L.wcg_correction_selector(seed, k, step)
                assert s == O.wco_correction_selector(seed, k, step)
                assert 0 <= s < step
                if step == 8:
                    seen.add(s)
    assert seen == set(range(8))


def test_merge_draw_stream():
    """The merge draws of wcg_step (host code) are the oracle's."""
    L = _capi.load()
    from oracle import oracle as oo
    if not oo.available():
        pytest.skip("oracle not built")
    O = oo.lib()
    sel_g, sel_o = ctypes.c_int(0), ctypes.c_int(0)
    pg, po = (ctypes.c_int * 9)(), (ctypes.c_int * 9)()
    seen = set()
    for seed in (0, 3, 2**33 + 1):
        for k in range(40):
            assert L.wcg_merge_draws(seed, k, 8, ctypes.byref(sel_g), pg) == 0
            O.wco_merge_draws(seed, k, 8, ctypes.byref(sel_o), po)
            assert sel_g.value == sel_o.value and list(pg) == list(po)
            for q in range(3):
                assert sorted(pg[3 * q:3 * q + 3]) == [0, 1, 2]
            seen.add(tuple(pg[:3]))
    assert len(seen) == 6


def test_split_key_stream():
    """The split keys of wcg_step (host code) are the oracle's."""
    L = _capi.load()
    from oracle import oracle as oo
    if not oo.available():
        pytest.skip("oracle not built")
    O = oo.lib()
    keys = set()
    for seed in (0, 5, 2**40 + 7):
        for k in range(30):
            a = L.wcg_split_key(seed, k)
            assert a == O.wco_split_key(seed, k)
            keys.add(a)
    assert len(keys) == 90
