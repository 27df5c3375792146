"""ctypes binding of oracle/_build/libwcoracle.so, the C restatement of the
liquid fluid-step hot path (oracle/wc_oracle.c).

TEST INFRASTRUCTURE ONLY: the checker for libwcgpu.  Same snapshot API as
oracle/ref.py (the compiled reference), so tests can compare any pair.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "libwcoracle.so")
_D = ctypes.POINTER(ctypes.c_double)
_L = ctypes.POINTER(ctypes.c_longlong)
_I = ctypes.POINTER(ctypes.c_int)
_lib = None


def available() -> bool:
    return os.path.exists(LIB)


def lib():
    global _lib
    if _lib is None:
        L = ctypes.CDLL(LIB)
        L.wco_create.restype = ctypes.c_void_p
        L.wco_create.argtypes = [ctypes.c_double, _D, ctypes.c_double, ctypes.c_double,
                                 ctypes.c_double, _D, _D, ctypes.c_double, ctypes.c_double,
                                 ctypes.c_int, ctypes.c_int, ctypes.c_int, _D, _D, _D, _D, _D, _D]
        L.wco_destroy.argtypes = [ctypes.c_void_p]
        L.wco_set_viscosity.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_int]
        L.wco_set_viscosity_implicit.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double]
        L.wco_viscosity_stats.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int),
                                          ctypes.POINTER(ctypes.c_double),
                                          ctypes.POINTER(ctypes.c_int)]
        L.wco_set_elasto.argtypes = [ctypes.c_void_p, ctypes.c_int] + [_D] * 10 + [_I, _D]
        L.wco_set_elasto_coeffs.argtypes = [ctypes.c_void_p] + [ctypes.c_double] * 3
        L.wco_transfer.argtypes = [ctypes.c_void_p, ctypes.c_double]
        L.wco_set_correction.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_int,
                                         ctypes.c_double, ctypes.c_uint64]
        L.wco_set_correction_selector.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.wco_correct_liquid.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_int]
        L.wco_merge_liquid.argtypes = [ctypes.c_void_p, ctypes.c_int, _I, _I, _I]
        L.wco_merge_liquid.restype = ctypes.c_int
        L.wco_merge_draws.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int, _I, _I]
        L.wco_set_merge.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_uint64, ctypes.c_double]
        L.wco_split_liquid.argtypes = [ctypes.c_void_p, ctypes.c_uint64]
        L.wco_split_liquid.restype = ctypes.c_int
        L.wco_split_key.argtypes = [ctypes.c_uint64, ctypes.c_uint64]
        L.wco_split_key.restype = ctypes.c_uint64
        L.wco_set_split.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_uint64]
        L.wco_terminate_liquid.argtypes = [ctypes.c_void_p]
        L.wco_terminate_liquid.restype = ctypes.c_int
        L.wco_set_terminator.argtypes = [ctypes.c_void_p, ctypes.c_int, _D, _D, ctypes.c_double,
                                         ctypes.c_int]
        L.wco_set_terminators.argtypes = [ctypes.c_void_p, ctypes.c_int,
                                          ctypes.POINTER(ctypes.c_int),
                                          ctypes.POINTER(ctypes.c_int), _D, _D, _D]
        L.wco_correction_selector.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_int]
        L.wco_correction_selector.restype = ctypes.c_int
        L.wco_step.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_int]
        L.wco_step.restype = ctypes.c_int
        L.wco_substep.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_int]
        L.wco_num_substeps.argtypes = [ctypes.c_void_p, ctypes.c_double]
        L.wco_num_substeps.restype = ctypes.c_int
        L.wco_size.argtypes = [ctypes.c_void_p, ctypes.c_char_p]
        L.wco_size.restype = ctypes.c_longlong
        L.wco_get_f.argtypes = [ctypes.c_void_p, ctypes.c_char_p, _D]
        L.wco_snap_state.argtypes = [ctypes.c_void_p, ctypes.c_char_p]
        L.wco_get_i.argtypes = [ctypes.c_void_p, ctypes.c_char_p, _L]
        L.wco_solver_stats.argtypes = [ctypes.c_void_p, _I, _D]
        L.wco_pcg_solve.restype = ctypes.c_int
        L.wco_pcg_solve.argtypes = [ctypes.c_int, _I, _I, _D, _D, _D, ctypes.c_double,
                                    ctypes.c_int, ctypes.c_double, ctypes.c_double, _D, _I]
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(_D)


def set_elasto(fn_set, fn_coeffs, h, scene, keep):
    """Pass a scene's elasto particles and elasto coefficients to a created
    scene handle (no-op for liquid-only scenes)."""
    p = scene.params
    fn_coeffs(h, getattr(p, "elasto_flip_coeff", 0.95), getattr(p, "elasto_flip_asym_coeff", 1.0),
              getattr(p, "elasto_advect_coeff", 1.0))
    e = getattr(scene, "elasto", None)
    if e is None or e.n == 0:
        return

    def arr(a):
        a = np.ascontiguousarray(a, dtype=np.float64).reshape(-1)
        keep.append(a)
        return _dp(a)

    surf = np.ascontiguousarray(e.surfel, dtype=np.int32)
    keep.append(surf)
    fn_set(h, e.n, arr(e.x4), arr(e.v4), arr(e.B), arr(e.m4), arr(e.fm4), arr(e.rest_vol),
           arr(e.rest_vf), arr(e.fluid_vol), arr(e.shape_factor), arr(e.orientation),
           surf.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), arr(e.radius))


class OracleScene:
    """The C restatement of one liquid scene (same API as oracle.ref.RefScene)."""

    def __init__(self, scene):
        L = lib()
        p = scene.params
        self._keep = []

        def arr(a):
            a = np.ascontiguousarray(a, dtype=np.float64).reshape(-1)
            self._keep.append(a)
            return _dp(a)

        C = None if scene.C is None else arr(scene.C)
        self.h = L.wco_create(p.dx, arr(p.gravity), p.liquid_density, p.flip_coeff,
                              p.liquid_boundary_friction, arr(p.box_center), arr(p.box_half),
                              p.box_radius, p.criterion, p.maxiters, 1, scene.x.shape[0],
                              arr(scene.x), arr(scene.v), C, arr(scene.mass), arr(scene.vol),
                              arr(scene.radius))
        self.L = L
        mu = getattr(p, "viscosity", 0.0)
        if mu > 0.0:
            L.wco_set_viscosity(self.h, mu, getattr(p, "viscosity_substeps", 1))
        if mu > 0.0 and getattr(p, "viscosity_implicit", False):
            L.wco_set_viscosity_implicit(self.h, 1, getattr(p, "viscosity_criterion", 1e-6))
        set_elasto(L.wco_set_elasto, L.wco_set_elasto_coeffs, self.h, scene, self._keep)
        if getattr(p, "particle_merge", False) or getattr(p, "particle_cell_multiplier", None):
            L.wco_set_merge(self.h, 1 if getattr(p, "particle_merge", False) else 0,
                            getattr(p, "merge_seed", 0),
                            getattr(p, "particle_cell_multiplier", 0.3535533906))
        if getattr(p, "particle_split", False):
            L.wco_set_split(self.h, 1, getattr(p, "split_seed", 0))
        if getattr(p, "terminator", False):
            L.wco_set_terminator(self.h, 1, arr(p.terminator_center), arr(p.terminator_half),
                                 p.terminator_radius, 1 if p.terminator_inside else 0)
        # the correction runs in every sub-step (strength 0: projection only)
        L.wco_set_correction(self.h, getattr(p, "correction_strength", 0.0),
                             getattr(p, "correction_step", 8),
                             getattr(p, "correction_multiplier", 2.0),
                             getattr(p, "correction_seed", 0))

    def close(self):
        if self.h:
            self.L.wco_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, dt, snapshot=True):
        return self.L.wco_step(self.h, dt, 1 if snapshot else 0)

    def num_substeps(self, dt):
        """CFL sub-step count of WetClothCore::stepSystem for dt."""
        return self.L.wco_num_substeps(self.h, dt)

    def transfer(self, dt):
        """Grid, P2G, then G2P from the P2G velocities and advection (no
        solve); snapshots as in a step."""
        self.L.wco_transfer(self.h, dt)

    def merge(self, selector, perm):
        """mergeLiquidParticles with the given subset and colour permutations
        (perm: 9 ints, t then s then r); returns the particles removed."""
        pm = np.ascontiguousarray(perm, dtype=np.int32).reshape(3, 3)
        rows = [np.ascontiguousarray(pm[k]) for k in range(3)]
        ip = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
        return self.L.wco_merge_liquid(self.h, int(selector), ip(rows[0]), ip(rows[1]), ip(rows[2]))

    def split(self, key):
        """splitLiquidParticles with the rotations of key; returns the
        particles added."""
        return self.L.wco_split_liquid(self.h, int(key))

    def set_terminators(self, shapes):
        """Terminator shapes (dicts: type, inside, center, rot (w, x, y, z),
        param); an empty list removes them."""
        kinds = {"box": 0, "sphere": 1, "capsule": 2, "cylinder": 3}
        n = len(shapes)
        ty = np.array([kinds[s["type"]] for s in shapes] or [0], dtype=np.int32)
        ins = np.array([1 if s.get("inside") else 0 for s in shapes] or [0], dtype=np.int32)
        c = np.array([s["center"] for s in shapes] or [[0, 0, 0]], dtype=np.float64)
        q = np.array([s.get("rot", (1, 0, 0, 0)) for s in shapes] or [[1, 0, 0, 0]],
                     dtype=np.float64)
        par = np.array([(list(s["param"]) + [0.0] * 4)[:4] for s in shapes] or [[0] * 4],
                       dtype=np.float64)
        self._keep_term = (ty, ins, c, q, par)
        ip = ctypes.POINTER(ctypes.c_int)
        self.L.wco_set_terminators(self.h, n, ty.ctypes.data_as(ip), ins.ctypes.data_as(ip),
                                   _dp(c), _dp(q), _dp(par))

    def terminate(self):
        """terminateParticles with the scene's terminator box; returns the
        particles removed."""
        return self.L.wco_terminate_liquid(self.h)

    def set_correction_selector(self, selector):
        """Particle subset (fluid index % step) of the next correction."""
        self.L.wco_set_correction_selector(self.h, int(selector))

    def snap_state(self, tag):
        """The current particle state as tag + "x", "v", "C" (for steps run
        without snapshots)."""
        self.L.wco_snap_state(self.h, tag.encode())

    def get(self, name):
        n = self.L.wco_size(self.h, name.encode())
        if n < 0:
            raise KeyError(name)
        out = np.empty(n, dtype=np.float64)
        if self.L.wco_get_f(self.h, name.encode(), _dp(out)) == 0:
            return out
        out = np.empty(n, dtype=np.int64)
        self.L.wco_get_i(self.h, name.encode(), out.ctypes.data_as(_L))
        return out

    def viscosity_stats(self):
        """(iterations, residual, unknowns) of the last implicit viscosity solve"""
        it, nd = ctypes.c_int(0), ctypes.c_int(0)
        res = ctypes.c_double(0)
        self.L.wco_viscosity_stats(self.h, ctypes.byref(it), ctypes.byref(res), ctypes.byref(nd))
        return it.value, res.value, nd.value

    def solver_stats(self):
        it = ctypes.c_int(0)
        res = ctypes.c_double(0)
        self.L.wco_solver_stats(self.h, ctypes.byref(it), ctypes.byref(res))
        return it.value, res.value


def pcg_solve(rowstart, col, val, rhs, tol, maxiters, omega=0.97, min_ratio=0.25):
    """MIC(0)-PCG of robertbridson::PCGSolver on a CSR matrix (sorted rows)."""
    L = lib()
    n = len(rhs)
    rs = np.ascontiguousarray(rowstart, dtype=np.int32)
    cl = np.ascontiguousarray(col, dtype=np.int32)
    va = np.ascontiguousarray(val, dtype=np.float64)
    b = np.ascontiguousarray(rhs, dtype=np.float64)
    x = np.zeros(n)
    res = ctypes.c_double(0)
    it = ctypes.c_int(0)
    ok = L.wco_pcg_solve(n, rs.ctypes.data_as(_I), cl.ctypes.data_as(_I), _dp(va), _dp(b), _dp(x),
                         tol, maxiters, omega, min_ratio, ctypes.byref(res), ctypes.byref(it))
    return x, bool(ok), it.value, res.value
