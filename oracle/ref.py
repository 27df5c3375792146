"""ctypes binding of oracle/_ref/libwcref*.so (the reference Core + harness).

TEST INFRASTRUCTURE ONLY (checker and timed CPU baseline).  Built by
``make -f oracle/ref.mk``; see oracle/ref_harness.cpp for what each call runs.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_D = ctypes.POINTER(ctypes.c_double)
_L = ctypes.POINTER(ctypes.c_longlong)


def lib_path(omp: bool = False) -> str:
    return os.path.join(HERE, "_ref", "libwcref_omp.so" if omp else "libwcref.so")


def available(omp: bool = False) -> bool:
    return os.path.exists(lib_path(omp))


_libs = {}


def _lib(omp: bool):
    if omp not in _libs:
        L = ctypes.CDLL(lib_path(omp))
        L.wcref_create.restype = ctypes.c_void_p
        L.wcref_create.argtypes = [ctypes.c_double, _D, ctypes.c_double,
                                   ctypes.c_double, ctypes.c_double, _D, _D,
                                   ctypes.c_double, ctypes.c_double,
                                   ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                   _D, _D, _D, _D, _D, _D]
        L.wcref_destroy.argtypes = [ctypes.c_void_p]
        L.wcref_step.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_int]
        L.wcref_step.restype = ctypes.c_int
        L.wcref_substep.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_int]
        L.wcref_num_substeps.argtypes = [ctypes.c_void_p, ctypes.c_double]
        L.wcref_size.argtypes = [ctypes.c_void_p, ctypes.c_char_p]
        L.wcref_size.restype = ctypes.c_longlong
        L.wcref_get_f.argtypes = [ctypes.c_void_p, ctypes.c_char_p, _D]
        L.wcref_get_i.argtypes = [ctypes.c_void_p, ctypes.c_char_p, _L]
        L.wcref_solver_stats.argtypes = [ctypes.c_void_p,
                                         ctypes.POINTER(ctypes.c_int), _D]
        L.wcref_timers.argtypes = [ctypes.c_void_p, _D]
        L.wcref_amg_stats.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), _D]
        L.wcref_set_viscosity.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_int]
        L.wcref_set_viscosity_implicit.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_int,
                                                   ctypes.c_double]
        _I = ctypes.POINTER(ctypes.c_int)
        L.wcref_set_elasto.argtypes = [ctypes.c_void_p, ctypes.c_int] + [_D] * 10 + [_I, _D]
        L.wcref_set_elasto_coeffs.argtypes = [ctypes.c_void_p] + [ctypes.c_double] * 3
        L.wcref_transfer.argtypes = [ctypes.c_void_p, ctypes.c_double]
        L.wcref_set_correction.argtypes = [ctypes.c_void_p, ctypes.c_double, ctypes.c_int,
                                           ctypes.c_double, ctypes.c_uint]
        L.wcref_merge.argtypes = [ctypes.c_void_p, ctypes.c_uint, ctypes.c_int]
        L.wcref_core_step.argtypes = [ctypes.c_void_p, ctypes.c_double]
        L.wcref_set_cell_multiplier.argtypes = [ctypes.c_void_p, ctypes.c_double]
        L.wcref_pcg_solve_csr.argtypes = [_L, _L, _D, ctypes.c_int, _D, _D, ctypes.c_double,
                                          ctypes.c_int, _D, ctypes.POINTER(ctypes.c_int)]
        L.wcref_pcg_solve_csr.restype = ctypes.c_int
        L.wcref_merge.restype = ctypes.c_int
        L.wcref_split.argtypes = [ctypes.c_void_p, ctypes.c_uint]
        L.wcref_split.restype = ctypes.c_int
        L.wcref_split_inputs.argtypes = [ctypes.c_void_p, ctypes.c_uint, _D, _D, ctypes.c_int]
        L.wcref_split_inputs.restype = ctypes.c_int
        L.wcref_num_particles.argtypes = [ctypes.c_void_p]
        L.wcref_num_particles.restype = ctypes.c_int
        L.wcref_set_terminator.argtypes = [ctypes.c_void_p, _D, _D, ctypes.c_double, ctypes.c_int]
        L.wcref_add_terminator.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _D, _D,
                                           ctypes.c_double, _D, ctypes.c_int, _D]
        L.wcref_terminate.argtypes = [ctypes.c_void_p]
        L.wcref_terminate.restype = ctypes.c_int
        _libs[omp] = L
    return _libs[omp]


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


class RefScene:
    """One reference TwoDScene + LinearizedImplicitEuler, liquid only."""

    def __init__(self, scene, mic: bool = True, omp: bool = False):
        self.L = _lib(omp)
        p = scene.params
        self._keep = []

        def arr(a, n=None):
            a = np.ascontiguousarray(a, dtype=np.float64)
            self._keep.append(a)
            return _dp(a)

        C = None if scene.C is None else arr(scene.C.reshape(-1))
        self.h = self.L.wcref_create(
            p.dx, arr(p.gravity), p.liquid_density, p.flip_coeff,
            p.liquid_boundary_friction, arr(p.box_center), arr(p.box_half),
            p.box_radius, p.criterion, p.maxiters, 1 if mic else 0,
            scene.x.shape[0], arr(scene.x.reshape(-1)), arr(scene.v.reshape(-1)),
            C, arr(scene.mass), arr(scene.vol), arr(scene.radius))
        mu = getattr(p, "viscosity", 0.0)
        if mu > 0.0 and getattr(p, "viscosity_implicit", False):
            self.L.wcref_set_viscosity_implicit(self.h, mu, getattr(p, "viscosity_substeps", 1),
                                                getattr(p, "viscosity_criterion", 1e-6))
        elif mu > 0.0:
            self.L.wcref_set_viscosity(self.h, mu, getattr(p, "viscosity_substeps", 1))
        set_elasto(self.L.wcref_set_elasto, self.L.wcref_set_elasto_coeffs, self.h, scene,
                   self._keep)
        if getattr(p, "terminator", False):
            self.L.wcref_set_terminator(self.h, arr(p.terminator_center), arr(p.terminator_half),
                                        p.terminator_radius, 1 if p.terminator_inside else 0)
        self.L.wcref_set_cell_multiplier(self.h, getattr(p, "particle_cell_multiplier",
                                                         0.3535533906))
        # the correction runs in every sub-step (strength 0: projection only)
        self.L.wcref_set_correction(self.h, getattr(p, "correction_strength", 0.0),
                                    getattr(p, "correction_step", 8),
                                    getattr(p, "correction_multiplier", 2.0),
                                    getattr(p, "correction_seed", 0))

    def close(self):
        if self.h:
            self.L.wcref_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, dt: float, snapshot: bool = True) -> int:
        return self.L.wcref_step(self.h, dt, 1 if snapshot else 0)

    def core_step(self, dt: float) -> None:
        """The reference's own WetClothCore::stepSystem on this scene (not the
        harness's staged replay); the particle state lands in adv_*/g2p_*."""
        self.L.wcref_core_step(self.h, dt)

    def merge(self, seed: int, step: int) -> int:
        """updateOptiVolume + mergeLiquidParticles after srand(seed); returns
        the particles removed (draws in "merge_selector", "merge_perm")."""
        return self.L.wcref_merge(self.h, seed, step)

    def add_terminators(self, shapes):
        """Terminator DistanceFieldObjects, each a dict: type ("box",
        "sphere", "capsule", "cylinder"), inside, center, axis, angle, param
        (4), group (>= 1).  Returns the shapes with the rotation quaternion
        the reference built ("rot": w, x, y, z)."""
        kinds = {"box": 0, "sphere": 1, "capsule": 2, "cylinder": 3}
        out = []
        for sh in shapes:
            rot = np.zeros(4)
            arr = lambda a: np.ascontiguousarray(a, dtype=np.float64)
            c, ax, par = arr(sh["center"]), arr(sh.get("axis", (0.0, 1.0, 0.0))), arr(sh["param"])
            self.L.wcref_add_terminator(self.h, kinds[sh["type"]], 1 if sh.get("inside") else 0,
                                        c.ctypes.data_as(_D), ax.ctypes.data_as(_D),
                                        float(sh.get("angle", 0.0)), par.ctypes.data_as(_D),
                                        int(sh.get("group", 1)), rot.ctypes.data_as(_D))
            out.append(dict(sh, rot=tuple(rot)))
        return out

    def terminate(self) -> int:
        """terminateParticles; returns the particles removed."""
        return self.L.wcref_terminate(self.h)

    def split_inputs(self, seed: int):
        """The reference's sphere-pattern table (n = 2..32, 1581 doubles) and
        the rotations its split draws after srand(seed), one row-major 3x3 per
        splitting parent (call before split(seed))."""
        pattern = np.zeros(3 * sum(range(2, 33)))
        cap = max(1, self.L.wcref_num_particles(self.h))
        rot = np.zeros(9 * cap)
        k = self.L.wcref_split_inputs(self.h, int(seed), pattern.ctypes.data_as(_D),
                                      rot.ctypes.data_as(_D), cap)
        return pattern, rot[:9 * k].reshape(k, 9)

    def split(self, seed: int) -> int:
        """updateOptiVolume + splitLiquidParticles after srand(seed);
        returns the particles added."""
        return self.L.wcref_split(self.h, seed)

    def transfer(self, dt: float) -> None:
        """Grid, P2G, then G2P from the P2G velocities and advection (no
        solve); snapshots as in a step."""
        self.L.wcref_transfer(self.h, dt)

    def get(self, name: str) -> np.ndarray:
        n = self.L.wcref_size(self.h, name.encode())
        if n < 0:
            raise KeyError(name)
        out = np.empty(n, dtype=np.float64)
        if self.L.wcref_get_f(self.h, name.encode(), _dp(out)) == 0:
            return out
        out = np.empty(n, dtype=np.int64)
        self.L.wcref_get_i(self.h, name.encode(), out.ctypes.data_as(_L))
        return out

    def solver_stats(self):
        it = ctypes.c_int(0)
        res = ctypes.c_double(0)
        self.L.wcref_solver_stats(self.h, ctypes.byref(it), ctypes.byref(res))
        return it.value, res.value

    def amg_stats(self):
        """(iterations, residual) of the reference's default multigrid-PCG
        (AMGPCGSolveSparse) on the system of the last snapshot step."""
        it = ctypes.c_int(0)
        res = ctypes.c_double(0)
        self.L.wcref_amg_stats(self.h, ctypes.byref(it), ctypes.byref(res))
        return it.value, res.value

    def timers(self) -> np.ndarray:
        out = np.zeros(12)
        self.L.wcref_timers(self.h, _dp(out))
        return out


def pcg_solve_csr(rowstart, col, val, rhs, tolerance, maxiter):
    """The reference's robertbridson::PCGSolver<double>::solve on a CSR matrix
    (MIC(0), 0.97 / 0.25).  Returns (x, residual, iterations, converged)."""
    L = _lib(False)
    rs = np.ascontiguousarray(rowstart, dtype=np.int64)
    cl = np.ascontiguousarray(col, dtype=np.int64)
    vl = np.ascontiguousarray(val, dtype=np.float64)
    b = np.ascontiguousarray(rhs, dtype=np.float64)
    n = rs.shape[0] - 1
    x = np.zeros(n, dtype=np.float64)
    res = ctypes.c_double(0.0)
    it = ctypes.c_int(0)
    ok = L.wcref_pcg_solve_csr(rs.ctypes.data_as(_L), cl.ctypes.data_as(_L),
                               vl.ctypes.data_as(_D), n, b.ctypes.data_as(_D),
                               x.ctypes.data_as(_D), float(tolerance), int(maxiter),
                               ctypes.byref(res), ctypes.byref(it))
    return x, res.value, it.value, bool(ok)


def binding_available() -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", "libwcbinding.so"))


def binding_step_both(scene, steps, dt, solver, precision, terminators=()):
    """Steps two reference scenes built from `scene`: one with the reference's
    WetClothCore::stepSystem, one with the compiled GpuWetClothCore binding
    (oracle/binding/GpuWetClothCore.h) passing the scene's criterion and
    iteration limit.  Returns ((x, v, C) reference, (x, v, C) binding,
    sub-steps of the binding's last step).  terminators: shapes added to both
    scenes as add_terminators takes them (the binding reads them from its
    scene)."""
    B = ctypes.CDLL(os.path.join(HERE, "_ref", "libwcbinding.so"))
    B.wcbind_step_both.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                   ctypes.c_double, ctypes.c_double, ctypes.c_int,
                                   ctypes.c_int, ctypes.c_int, ctypes.c_longlong, _D, _D,
                                   _L, _L, ctypes.POINTER(ctypes.c_int), ctypes.c_char_p,
                                   ctypes.c_int]
    B.wcbind_step_both.restype = ctypes.c_int
    ra = RefScene(scene, mic=False)
    rb = RefScene(scene, mic=False)
    if terminators:
        ra.add_terminators(terminators)
        rb.add_terminators(terminators)
    cap = 4 * scene.x.shape[0] + 16
    oa = np.zeros(15 * cap)
    ob = np.zeros(15 * cap)
    na, nb = ctypes.c_longlong(0), ctypes.c_longlong(0)
    sub = ctypes.c_int(0)
    err = ctypes.create_string_buffer(512)
    rc = B.wcbind_step_both(ra.h, rb.h, int(steps), float(dt), float(scene.params.criterion),
                            int(scene.params.maxiters), int(solver), int(precision), cap,
                            oa.ctypes.data_as(_D), ob.ctypes.data_as(_D), ctypes.byref(na),
                            ctypes.byref(nb), ctypes.byref(sub), err, 512)
    ra.close()
    rb.close()
    if rc != 0:
        raise RuntimeError(err.value.decode(errors="replace"))

    def split(o, n):
        return (o[:3 * n].reshape(n, 3), o[3 * n:6 * n].reshape(n, 3),
                o[6 * n:15 * n].reshape(n, 9))
    return split(oa, na.value), split(ob, nb.value), sub.value
