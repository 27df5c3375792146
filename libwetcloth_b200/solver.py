"""Python view of one GPU scene, mirroring the reference's call sequence.

``FluidScene`` wraps a ``wcg_ctx``: the methods are named after the
``TwoDScene`` / ``LinearizedImplicitEuler`` / ``WetClothCore`` calls they
replace (libWetCloth/Core/WetClothCore.cpp:115-258).  All arithmetic runs in
libwcgpu.so on the GPU.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import _capi
from ._capi import check, _dp


def make_params(p, precision=_capi.WCG_FP64, refine_inner_tol=1e-5,
                max_refinements=20, solver=_capi.WCG_SOLVER_MIC0) -> _capi.WcgParams:
    prm = _capi.WcgParams()
    _capi.load().wcg_default_params(ctypes.byref(prm))
    prm.dx = p.dx
    for a in range(3):
        prm.gravity[a] = p.gravity[a]
        prm.box_center[a] = p.box_center[a]
        prm.box_half[a] = p.box_half[a]
    prm.liquid_density = p.liquid_density
    prm.flip_coeff = p.flip_coeff
    prm.liquid_boundary_friction = p.liquid_boundary_friction
    prm.box_radius = p.box_radius
    prm.walls = 1
    prm.criterion = p.criterion
    prm.maxiters = p.maxiters
    prm.precision = precision
    prm.refine_inner_tol = refine_inner_tol
    prm.max_refinements = max_refinements
    prm.solver = solver
    prm.viscosity = getattr(p, "viscosity", 0.0)
    prm.viscosity_substeps = getattr(p, "viscosity_substeps", 1)
    prm.elasto_flip_coeff = getattr(p, "elasto_flip_coeff", 0.95)
    prm.elasto_flip_asym_coeff = getattr(p, "elasto_flip_asym_coeff", 1.0)
    prm.elasto_advect_coeff = getattr(p, "elasto_advect_coeff", 1.0)
    prm.drag_viscosity = getattr(p, "drag_viscosity", 8.9e-3)
    prm.viscosity_implicit = 1 if getattr(p, "viscosity_implicit", False) else 0
    prm.viscosity_criterion = getattr(p, "viscosity_criterion", 1e-6)
    prm.particle_merge = 1 if getattr(p, "particle_merge", False) else 0
    prm.particle_split = 1 if getattr(p, "particle_split", False) else 0
    prm.split_seed = getattr(p, "split_seed", 0)
    if getattr(p, "terminator", False):
        prm.terminator = 1
        for a in range(3):
            prm.terminator_center[a] = p.terminator_center[a]
            prm.terminator_half[a] = p.terminator_half[a]
        prm.terminator_radius = p.terminator_radius
        prm.terminator_inside = 1 if p.terminator_inside else 0
    prm.merge_seed = getattr(p, "merge_seed", 0)
    prm.particle_cell_multiplier = getattr(p, "particle_cell_multiplier", 0.3535533906)
    prm.correction_strength = getattr(p, "correction_strength", 0.0)
    prm.correction_step = getattr(p, "correction_step", 8)
    prm.correction_multiplier = getattr(p, "correction_multiplier", 2.0)
    prm.correction_seed = getattr(p, "correction_seed", 0)
    return prm


class FluidScene:
    def __init__(self, scene=None, precision=_capi.WCG_FP64, params=None, **kw):
        self.L = _capi.load()
        prm = params if params is not None else make_params(scene.params, precision, **kw)
        h = ctypes.c_void_p()
        check(self.L.wcg_create(ctypes.byref(prm), ctypes.byref(h)))
        self.h = h
        self.precision = prm.precision
        if scene is not None:
            self.upload(scene.x, scene.v, scene.C, scene.mass, scene.vol, scene.radius)
            if getattr(scene, "elasto", None) is not None:
                self.upload_elasto(scene.elasto)

    def close(self):
        if getattr(self, "h", None):
            self.L.wcg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- particles ----
    def upload(self, x, v, C, mass, vol, radius):
        arr = lambda a: None if a is None else np.ascontiguousarray(a, dtype=np.float64).reshape(-1)
        x, v, C, mass, vol, radius = map(arr, (x, v, C, mass, vol, radius))
        n = mass.shape[0]
        self._attrs = (mass, vol, radius)
        check(self.L.wcg_upload_liquid(self.h, n, _dp(x), _dp(v), _dp(C), _dp(mass),
                                       _dp(vol), _dp(radius)))

    def set_state(self, x, v, C):
        """Replace the liquid particles' positions, velocities and affine
        matrices (mass, volume and radius as last uploaded)."""
        self.upload(x, v, C, *self._attrs)

    def substep_vjp(self, dt, vbar, Cbar, xbar, with_viscosity=False):
        """Reverse mode of substep(dt) at the current (pre-step) state:
        cotangents of (v', C', x') -> of (v, C, x), and of the viscosity when
        with_viscosity.  The x-cotangent follows the transfer weights' x
        (set_adjoint_positions(False) holds the positions fixed instead)."""
        n = self.num_particles
        arr = lambda a, k: np.ascontiguousarray(a, dtype=np.float64).reshape(n * k)
        vb, Cb, xb = arr(vbar, 3), arr(Cbar, 9), arr(xbar, 3)
        v0 = np.empty(n * 3)
        C0 = np.empty(n * 9)
        x0 = np.empty(n * 3)
        mu = ctypes.c_double(0.0)
        check(self.L.wcg_substep_vjp(self.h, dt, _dp(vb), _dp(Cb), _dp(xb), _dp(v0), _dp(C0),
                                     _dp(x0), ctypes.byref(mu)))
        out = (v0.reshape(n, 3), C0.reshape(n, 9), x0.reshape(n, 3))
        return out + (mu.value,) if with_viscosity else out

    def set_adjoint_positions(self, differentiate=True):
        """Whether substep_vjp differentiates through the particle positions."""
        check(self.L.wcg_set_adjoint_positions(self.h, 1 if differentiate else 0))

    def set_viscosity(self, mu, substeps=1):
        """LiquidInfo::viscosity and its explicit sub-steps (0: off)."""
        check(self.L.wcg_set_viscosity(self.h, float(mu), int(substeps)))

    def upload_device(self, n, x, v, C, mass, vol, radius):
        """Arguments are device pointers (ints) to contiguous float64 arrays."""
        check(self.L.wcg_upload_liquid_device(self.h, n, x, v, C, mass, vol, radius))

    @property
    def num_particles(self):
        return self.L.wcg_num_particles(self.h)

    def upload_elasto(self, e):
        """Elasto particles (a scenes.ElastoSet): the reference's particles
        [0, n) ahead of the liquid ones."""
        arr = lambda a: np.ascontiguousarray(a, dtype=np.float64).reshape(-1)
        cols = [arr(a) for a in (e.x4, e.v4, e.B, e.m4, e.fm4, e.rest_vol, e.rest_vf,
                                 e.fluid_vol, e.shape_factor, e.orientation)]
        surf = np.ascontiguousarray(e.surfel, dtype=np.int32)
        check(self.L.wcg_upload_elasto(self.h, e.n, *[_dp(c) for c in cols],
                                       surf.ctypes.data_as(ctypes.POINTER(ctypes.c_int))))

    @property
    def num_elasto(self):
        return self.L.wcg_num_elasto(self.h)

    def download_elasto(self):
        """(x4, v4, B9) of the elasto particles in their original order."""
        n = self.num_elasto
        x4 = np.empty((n, 4))
        v4 = np.empty((n, 4))
        B = np.empty((n, 9))
        check(self.L.wcg_download_elasto(self.h, _dp(x4), _dp(v4), _dp(B)))
        return x4, v4, B

    def upload_field(self, name, values):
        """Set "u_x/y/z" or "vel_x/y/z" node velocities (inactive buckets
        ignored)."""
        v = np.ascontiguousarray(values, dtype=np.float64).reshape(-1)
        check(self.L.wcg_upload_field(self.h, name.encode(), _dp(v), v.shape[0]))

    def download(self):
        n = self.num_particles
        x = np.empty((n, 3))
        v = np.empty((n, 3))
        C = np.empty((n, 9))
        check(self.L.wcg_download_liquid(self.h, _dp(x), _dp(v), _dp(C)))
        return x, v, C

    # ---- state I/O (TwoDSceneSerializer formats) ----
    def save_positions(self, path):
        """serializePositionOnly's binary position file."""
        check(self.L.wcg_save_positions(self.h, os.fsencode(path)))

    def load_positions(self, path):
        """loadPosOnly: replace the positions from a position file."""
        check(self.L.wcg_load_positions(self.h, os.fsencode(path)))

    def write_fluid_obj(self, path):
        """The fluid OBJ dump: "v x y z radius" per particle."""
        check(self.L.wcg_write_fluid_obj(self.h, os.fsencode(path)))

    # ---- reference call sequence ----
    def rebucketize_and_resample(self):
        check(self.L.wcg_rebucketize_and_resample(self.h))

    def map_particle_nodes(self):
        check(self.L.wcg_map_particle_nodes(self.h))

    def step_velocity(self, dt):
        check(self.L.wcg_step_velocity(self.h, dt))

    def project_fine(self, dt):
        check(self.L.wcg_project_fine(self.h, dt))

    def apply_pressure_drag_fluid(self, dt):
        check(self.L.wcg_apply_pressure_drag_fluid(self.h, dt))

    def constrain_liquid_velocity(self):
        check(self.L.wcg_constrain_liquid_velocity(self.h))

    def split_liquid_particles(self, key):
        """relabel + splitLiquidParticles with the rotations of key; returns
        the number of particles added."""
        add = ctypes.c_longlong(0)
        check(self.L.wcg_split_liquid_particles(self.h, int(key), ctypes.byref(add)))
        return add.value

    def split_parents(self):
        """The number of particles the split would split now."""
        k = ctypes.c_longlong(0)
        check(self.L.wcg_split_parents(self.h, ctypes.byref(k)))
        return k.value

    def split_liquid_particles_with(self, pattern, rotations):
        """splitLiquidParticles placed by the reference's sphere-pattern table
        (1581 doubles: the points of n = 2..32) and one row-major rotation per
        splitting parent (original-index order); returns the number added."""
        pat = np.ascontiguousarray(pattern, dtype=np.float64).ravel()
        rot = np.ascontiguousarray(rotations, dtype=np.float64).reshape(-1, 9)
        if pat.size != 1581:
            raise ValueError("pattern must hold 1581 doubles")
        add = ctypes.c_longlong(0)
        check(self.L.wcg_split_liquid_particles_with(self.h, _dp(pat), _dp(rot), rot.shape[0],
                                                     ctypes.byref(add)))
        return add.value

    def terminate_liquid_particles(self):
        """terminateParticles with the scene's terminator box; returns the
        number of particles removed."""
        rem = ctypes.c_longlong(0)
        check(self.L.wcg_terminate_liquid_particles(self.h, ctypes.byref(rem)))
        return rem.value

    def merge_liquid_particles(self, selector, perm):
        """relabel + mergeLiquidParticles + removeEmptyParticles with the given
        subset and colour order (9 ints: z, y, x permutations); returns the
        number of particles removed."""
        pm = (ctypes.c_int * 9)(*[int(v) for v in np.asarray(perm).reshape(-1)])
        rem = ctypes.c_longlong(0)
        check(self.L.wcg_merge_liquid_particles(self.h, int(selector), pm, ctypes.byref(rem)))
        return rem.value

    @property
    def correction_count(self):
        """The call of the correction stream the next sub-step takes."""
        return int(self.L.wcg_correction_count(self.h))

    def set_terminators(self, shapes):
        """Terminator shapes: a list of dicts with keys type ("box", "sphere",
        "capsule", "cylinder"), inside (bool), center (3), rot (w, x, y, z;
        identity by default) and param (up to 4 values, as
        DistanceFieldObject's parameter).  An empty list removes them."""
        kinds = {"box": _capi.WCG_SHAPE_BOX, "sphere": _capi.WCG_SHAPE_SPHERE,
                 "capsule": _capi.WCG_SHAPE_CAPSULE, "cylinder": _capi.WCG_SHAPE_CYLINDER}
        arr = (_capi.WcgShape * max(1, len(shapes)))()
        for k, sh in enumerate(shapes):
            arr[k].type = kinds[sh["type"]]
            arr[k].inside = 1 if sh.get("inside", False) else 0
            arr[k].center[:] = [float(v) for v in sh["center"]]
            arr[k].rot[:] = [float(v) for v in sh.get("rot", (1.0, 0.0, 0.0, 0.0))]
            par = [float(v) for v in sh["param"]] + [0.0] * 4
            arr[k].param[:] = par[:4]
        check(self.L.wcg_set_terminators(self.h, len(shapes), arr))

    @property
    def schedule(self):
        """The pressure solve's launch schedule (sweep_cluster,
        sweep_cluster_a, pcg_batch); performance only, results unchanged."""
        s = _capi.WcgSchedule()
        check(self.L.wcg_get_schedule(self.h, ctypes.byref(s)))
        return (s.sweep_cluster, s.sweep_cluster_a, s.pcg_batch)

    @schedule.setter
    def schedule(self, sched):
        s = _capi.WcgSchedule(*[int(v) for v in sched])
        check(self.L.wcg_set_schedule(self.h, ctypes.byref(s)))

    def set_correction_count(self, k):
        """Call count of the correction stream (the next sub-step corrects the
        subset of call k)."""
        check(self.L.wcg_set_correction_count(self.h, int(k)))

    def correct_liquid_particles(self, dt, selector=-1):
        """correctLiquidParticles for the particles with index % step ==
        selector; -1 takes the next subset of the context's seeded stream,
        as a sub-step does (WetClothCore.cpp:242 runs it in every sub-step)."""
        check(self.L.wcg_correct_liquid_particles(self.h, dt, int(selector)))

    def map_node_particles(self):
        check(self.L.wcg_map_node_particles(self.h))

    def advect(self, dt):
        check(self.L.wcg_advect(self.h, dt))

    def substep(self, dt):
        check(self.L.wcg_substep(self.h, dt))

    def num_substeps(self, dt):
        n = ctypes.c_int(0)
        check(self.L.wcg_num_substeps(self.h, dt, ctypes.byref(n)))
        return n.value

    def step(self, dt):
        n = ctypes.c_int(0)
        check(self.L.wcg_step(self.h, dt, ctypes.byref(n)))
        return n.value

    def stats(self):
        s = _capi.WcgStats()
        check(self.L.wcg_get_stats(self.h, ctypes.byref(s)))
        return {k: getattr(s, k) for k, _ in _capi.WcgStats._fields_}

    # ---- parity downloads ----
    def grid_info(self):
        dims = (ctypes.c_int * 3)()
        org = (ctypes.c_double * 3)()
        bbx = (ctypes.c_double * 6)()
        check(self.L.wcg_grid_info(self.h, dims, org, bbx))
        return np.array(dims[:]), np.array(org[:]), np.array(bbx[:])

    def field(self, name):
        n = self.L.wcg_field_size(self.h, name.encode())
        if n < 0:
            raise KeyError(name)
        out = np.empty(n, dtype=np.float64)
        check(self.L.wcg_download_field(self.h, name.encode(), _dp(out), n))
        return out

    def ifield(self, name):
        n = self.L.wcg_field_size(self.h, name.encode())
        if n < 0:
            raise KeyError(name)
        out = np.empty(n, dtype=np.int64)
        check(self.L.wcg_download_ifield(self.h, name.encode(),
                                         out.ctypes.data_as(_capi._L), n))
        return out

    def pressure_system(self):
        ndof = ctypes.c_longlong(0)
        nnz = ctypes.c_longlong(0)
        check(self.L.wcg_export_pressure_system(self.h, ctypes.byref(ndof), ctypes.byref(nnz),
                                                None, None, None, None))
        rs = np.empty(ndof.value + 1, dtype=np.int64)
        col = np.empty(max(nnz.value, 1), dtype=np.int64)
        val = np.empty(max(nnz.value, 1), dtype=np.float64)
        rhs = np.empty(max(ndof.value, 1), dtype=np.float64)
        check(self.L.wcg_export_pressure_system(
            self.h, ctypes.byref(ndof), ctypes.byref(nnz), rs.ctypes.data_as(_capi._L),
            col.ctypes.data_as(_capi._L), _dp(val), _dp(rhs)))
        return rs, col[:nnz.value], val[:nnz.value], rhs[:ndof.value]

    # ---- instrumentation ----
    @property
    def stream_ptr(self):
        return self.L.wcg_stream(self.h)

    @property
    def launch_count(self):
        return self.L.wcg_launch_count(self.h)

    def profile_begin(self):
        check(self.L.wcg_profile_begin(self.h))

    def profile_end(self):
        n = self.L.wcg_profile_num_phases()
        ms = np.zeros(n)
        cnt = np.zeros(n, dtype=np.int64)
        check(self.L.wcg_profile_end(self.h, _dp(ms), cnt.ctypes.data_as(_capi._L), n))
        names = [self.L.wcg_profile_phase_name(i).decode() for i in range(n)]
        return {names[i]: (float(ms[i]), int(cnt[i])) for i in range(n)}



# launch schedules the batch autotuner tries by default: the sweep clusters
# chosen per solve, plain, 2 and 4 along c, and 4 or 8 PCG iterations per
# host check
DEFAULT_SCHEDULES = ((0, 1, 8), (1, 1, 8), (2, 1, 8), (4, 1, 8), (1, 1, 4), (2, 1, 4))


class FluidBatch:
    """Independent scenes stepped together (wcg_batch_*): each scene is a
    FluidScene with its own stream; a pool of host threads steps them largest
    first so their kernels overlap on the GPU."""

    def __init__(self, scenes):
        self.L = _capi.load()
        self.scenes = list(scenes)
        arr = (ctypes.c_void_p * len(self.scenes))(*[s.h.value for s in self.scenes])
        h = ctypes.c_void_p()
        check(self.L.wcg_batch_create(len(self.scenes), arr, ctypes.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.L.wcg_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, dt, nsteps=1):
        """nsteps steps of every scene; dt is a scalar or one value per
        scene.  Returns the per-scene status codes."""
        d = np.ascontiguousarray(np.broadcast_to(np.asarray(dt, dtype=np.float64),
                                                 (len(self.scenes),)))
        st = (ctypes.c_int * len(self.scenes))()
        rc = self.L.wcg_batch_step(self.h, _dp(d), nsteps, st)
        if rc not in (_capi.WCG_OK, _capi.WCG_ERR_NOT_CONVERGED):
            check(rc)
        return list(st)

    def set_shared_solve(self, on=True, max_patches=None):
        """Run the scenes' PCG iterations in shared launches over all scenes
        waiting in their solve (results unchanged); solves of more than
        max_patches pencil patches iterate alone (None: no limit)."""
        lim = 2**31 - 1 if max_patches is None else int(max_patches)
        check(self.L.wcg_batch_set_shared_solve_limit(self.h, lim))
        check(self.L.wcg_batch_set_shared_solve(self.h, 1 if on else 0))

    @property
    def shared_launches(self):
        return int(self.L.wcg_batch_shared_launches(self.h))

    @property
    def threads(self):
        return self.L.wcg_batch_threads(self.h)

    @threads.setter
    def threads(self, n):
        check(self.L.wcg_batch_set_threads(self.h, int(n)))

    def autotune(self, dt, candidates=(1, 2, 4, 8, 16)):
        """Time one batch step per candidate thread count (each advances every
        scene by one step) and keep the fastest; returns {threads: ms}."""
        d = np.ascontiguousarray(np.broadcast_to(np.asarray(dt, dtype=np.float64),
                                                 (len(self.scenes),)))
        c = (ctypes.c_int * len(candidates))(*candidates)
        ms = (ctypes.c_double * len(candidates))()
        check(self.L.wcg_batch_autotune(self.h, _dp(d), c, len(candidates), ms))
        return dict(zip(candidates, list(ms)))

    def autotune_schedules(self, dt, candidates=DEFAULT_SCHEDULES, trials=1):
        """Choose each scene's launch schedule (sweep_cluster,
        sweep_cluster_a, pcg_batch) from timed trials: every candidate is
        stepped `trials` times (each advances every scene by one step) and
        each scene keeps the one with its smallest step time.  Returns (the
        chosen candidate index per scene, the times in ms as an array
        scenes x candidates)."""
        n = len(self.scenes)
        d = np.ascontiguousarray(np.broadcast_to(np.asarray(dt, dtype=np.float64), (n,)))
        cand = (_capi.WcgSchedule * len(candidates))(
            *[_capi.WcgSchedule(*[int(v) for v in c]) for c in candidates])
        ms = np.zeros((n, len(candidates)))
        chosen = (ctypes.c_int * n)()
        check(self.L.wcg_batch_autotune_schedules(self.h, _dp(d), cand, len(candidates),
                                                  int(trials), _dp(ms), chosen))
        return list(chosen), ms
