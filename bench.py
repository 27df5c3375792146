#!/usr/bin/env python
"""Fluid-step benchmark: ms per step (bucket sort + P2G + MIC(0)-PCG pressure
projection + G2P + advection) of a 256^3 grid / ~16.8M-particle liquid scene on
one B200, FP32 transfers and PCG with FP64 reductions and iterative refinement
to a 1e-6 relative residual, beside the plain FP64 GPU step.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

One JSON line on stdout (rank 0).  Multi-GPU runs (torchrun) are independent
replicas: the path has no exchange step.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "ms/step P2G+PCG+G2P @256³/16M, FP32+refine vs FP64 GPU @1e-6 resid; HBM %"
DT = 1e-3


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=256, help="grid cells per axis")
    ap.add_argument("--ppc", type=int, default=2)
    ap.add_argument("--fp64-steps", type=int, default=None,
                    help="timed steps of the FP64 arm (default: --steps)")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-mg", action="store_true",
                    help="skip the multigrid-PCG arms (the reference's default solver)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-sample-n", type=int, default=64,
                    help="grid of the bounded CPU-baseline sample")
    ap.add_argument("--profile-steps", type=int, default=2)
    ap.add_argument("--no-batch", action="store_true",
                    help="skip the many-scenes measurement (batched vs sequential)")
    ap.add_argument("--batch-scenes", type=int, default=32)
    ap.add_argument("--batch-full", action="store_true",
                    help="the many-scenes configuration at its stated size: 256 scenes of "
                         "32..96^3 and 10k..1M particles, 50 steps, one pass per arm "
                         "(minutes; not part of the default run)")
    ap.add_argument("--no-cloth", action="store_true",
                    help="skip the liquid-on-cloth measurement (128^3 sphere on a sheet)")
    ap.add_argument("--no-config0", action="store_true",
                    help="skip the 64^3 dam-break line (100 steps)")
    ap.add_argument("--no-ref-mic", action="store_true",
                    help="reference arm: skip the MIC(0)-PCG run")
    ap.add_argument("--ref-budget-s", type=float, default=1500.0,
                    help="reference arm: wall-clock budget of the timed steps")
    ap.add_argument("--ref-child", default=None, help=argparse.SUPPRESS)
    return ap.parse_args()


# ---------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.dev = device_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-i", str(self.dev), "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = max(smax, float(f[2]))
            except ValueError:
                continue
            for k, nm in enumerate(names):
                if f[5 + k].lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


# Algorithmic bytes per phase (w = bytes per value).  Per particle: sort 4+8
# bytes of keys plus the 17-value permutation gather; P2G reads x(3) v(3) C(9)
# m V = 17 values; G2P+advect reads x(3), writes v(3) C(9) x(3) = 18 values.
# Per active cell: P2G writes 3 faces x (m, u, V) + phi + sat + psi = 12;
# grid update reads 12 and writes 8.  Per DOF: each triangular sweep 6 values,
# the factorisation 6, one PCG iteration's vector work 20 (SpMV 6, s.q 2,
# x 3, r 3, |r| 1, z.r 2, s 3).
def phase_bytes(phase, w, np_, ncell, ndof, iters, nsweeps):
    if phase == "grid_build_sort":
        return np_ * (12 + 17 * w)
    if phase == "p2g":
        return np_ * 17 * w + ncell * 12 * w
    if phase == "g2p_advect":
        return np_ * 18 * w + ncell * 3 * w
    if phase == "grid_ops":
        return ncell * 20 * w
    if phase == "mic_sweep":
        return ndof * 6 * w * nsweeps
    if phase == "mic_factor":
        return ndof * 6 * w
    if phase == "pcg_vector":
        return ndof * 20 * w * iters
    return 0


def traffic_per_launch(kernel_phase, ndof, np_):
    """DRAM bytes per launch from the committed ncu capture (profiles/),
    scaled to this workload's units; None if no capture is committed."""
    p = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if not os.path.exists(p):
        return None
    d = json.load(open(p))
    e = d.get(kernel_phase)
    if not e:
        return None
    units = ndof if e.get("unit") == "dof" else np_
    return e["bytes_per_unit"] * units


def reduce_max(x, world, device):
    """Maximum of a per-rank scalar over all ranks (the timing rule: a
    multi-GPU time is the slowest rank's)."""
    if world == 1:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


# ---------------------------------------------------------------------------
def run_ours(args, rank, world, dev):
    import numpy as np
    import torch
    from libwetcloth_b200 import scenes
    from libwetcloth_b200._capi import (WCG_FP32_REFINE, WCG_FP64, WCG_SOLVER_MG,
                                        WCG_SOLVER_MIC0)
    from libwetcloth_b200.solver import FluidScene

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    def max_over_ranks(x):
        return reduce_max(x, world, f"cuda:{dev}")

    t0 = time.time()
    sc = scenes.half_box(args.n, args.ppc, seed=1 + rank)
    gen_s = time.time() - t0
    np_ = sc.x.shape[0]

    def timed(precision, steps, warmup, sample_clocks=False, solver=WCG_SOLVER_MIC0):
        sim = FluidScene(sc, precision=precision, solver=solver)
        for _ in range(warmup):
            sim.step(DT)
        stream = torch.cuda.ExternalStream(sim.stream_ptr, device=f"cuda:{dev}")
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        barrier()
        torch.cuda.synchronize(dev)
        clk = ClockSampler(dev) if sample_clocks else None
        if clk:
            clk.start()
            time.sleep(0.3)
        l0 = sim.launch_count
        iters = []
        e0.record(stream)
        w0 = time.perf_counter()
        for _ in range(steps):
            sim.step(DT)
            st = sim.stats()
            iters.append(st["pcg_iters"])
        e1.record(stream)
        e1.synchronize()
        wall = time.perf_counter() - w0
        torch.cuda.synchronize(dev)
        clocks = clk.stop() if clk else None
        barrier()
        ms = max_over_ranks(e0.elapsed_time(e1) / steps)
        launches = sim.launch_count - l0
        info = dict(ms=ms, wall_ms=wall * 1000 / steps, launches=launches,
                    iters=iters, stats=sim.stats(), clocks=clocks)
        return sim, info

    # headline arm: FP32 transfers + FP32 PCG + FP64 refinement
    sim, main = timed(WCG_FP32_REFINE, args.steps, args.warmup, sample_clocks=True)
    st = main["stats"]
    # per-phase breakdown (separate pass; events around each phase)
    sim.profile_begin()
    for _ in range(args.profile_steps):
        sim.step(DT)
    prof = sim.profile_end()
    pst = sim.stats()
    ncell = pst["nactive_buckets"] * 64
    ndof = pst["ndof"]
    # e2e through the public C-ABI with pinned host buffers: every step
    # uploads its input state (the same seeded state each step), steps, and
    # reads its result back.  The input of step k + 1 is staged
    # (wcg_stage_liquid_async) while step k runs and the read-back of step k
    # (wcg_download_liquid_async) overlaps step k + 1; the timed region runs
    # from the first copy to wcg_synchronize after the last read-back, over
    # the same number of steps as the device-timed arm (the first upload and
    # the last read-back are not overlapped)
    e2e = None
    if not args.no_e2e:
        x, v, C = sim.download()
        pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
        hx, hv, hC = pin(x), pin(v), pin(C)
        hm, hV, hr = pin(sc.mass), pin(sc.vol), pin(sc.radius)
        outs = [tuple(torch.empty_like(t).pin_memory() for t in (hx, hv, hC)) for _ in range(2)]
        from libwetcloth_b200._capi import check
        L = sim.L
        ptr = lambda t: __import__("ctypes").cast(t.data_ptr(), __import__("ctypes").POINTER(
            __import__("ctypes").c_double))
        stream = torch.cuda.ExternalStream(sim.stream_ptr, device=f"cuda:{dev}")
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        nsub = __import__("ctypes").c_int(0)
        k_e2e = max(2, args.steps)
        e2e_iters = []
        barrier()
        torch.cuda.synchronize(dev)
        e0.record(stream)
        stage = lambda: check(L.wcg_stage_liquid_async(sim.h, np_, ptr(hx), ptr(hv), ptr(hC),
                                                       ptr(hm), ptr(hV), ptr(hr)))
        stage()
        check(L.wcg_upload_staged(sim.h))
        for k in range(k_e2e):
            if k + 1 < k_e2e:
                stage()  # the next step's input crosses PCIe while this step runs
            check(L.wcg_step(sim.h, DT, __import__("ctypes").byref(nsub)))
            e2e_iters.append(sim.stats()["pcg_iters"])  # host-side record, no wait
            ox, ov, oC = outs[k % 2]
            check(L.wcg_download_liquid_async(sim.h, ptr(ox), ptr(ov), ptr(oC)))
            if k + 1 < k_e2e:
                check(L.wcg_upload_staged(sim.h))
        check(L.wcg_synchronize(sim.h))
        e1.record(stream)
        e1.synchronize()
        e2e_ms = max_over_ranks(e0.elapsed_time(e1) / k_e2e)
        h2d = np_ * (3 + 3 + 9 + 3) * 8
        d2h = np_ * (3 + 3 + 9) * 8
        e2e = {"value": round(e2e_ms, 3), "unit": "ms/step",
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "steps": k_e2e,
               "pcg_iters_per_step": e2e_iters,
               "input": "the same seeded state uploaded every step",
               "overlap": "input of step k + 1 staged during step k; read-back of step k "
                          "during step k + 1 (separate copy streams)"}
    sim.close()
    # FP64 GPU arm at the same residual
    fp64 = None
    if not args.no_fp64:
        k64 = args.fp64_steps if args.fp64_steps is not None else args.steps
        sim64, info64 = timed(WCG_FP64, k64, args.warmup, sample_clocks=True)
        # its phases, as for the headline arm
        sim64.profile_begin()
        for _ in range(args.profile_steps):
            sim64.step(DT)
        info64["phases"] = sim64.profile_end()
        sim64.close()
        fp64 = info64
    # FP32 + refinement at the tighter criterion of the precision configuration
    tight = None
    if not args.no_fp64:
        old_crit = sc.params.criterion
        sc.params.criterion = 1e-8
        k8 = max(1, min(args.steps, 5))
        sim8, info8 = timed(WCG_FP32_REFINE, k8, args.warmup)
        sim8.close()
        sc.params.criterion = old_crit
        st8 = info8["stats"]
        tight = {"criterion": 1e-8, "ms_per_step": round(info8["ms"], 3), "steps": k8,
                 "pcg_iters_per_step": info8["iters"], "refinements": st8["refinements"],
                 "final_residual_rel": st8["residual"] / max(st8["rhs_norm"], 1e-300)}
    # the reference's default solver (multigrid-PCG) on the same workload
    mg = None
    if not args.no_mg:
        mg = {}
        for name, prec in (("fp32_refine", WCG_FP32_REFINE), ("fp64", WCG_FP64)):
            k_mg = max(1, min(args.steps, 5))
            sim_mg, info_mg = timed(prec, k_mg, args.warmup, solver=WCG_SOLVER_MG)
            sim_mg.close()
            mg[name] = {"ms_per_step": round(info_mg["ms"], 3), "steps": k_mg,
                        "pcg_iters_per_step": info_mg["iters"]}
    # roofline of the dominant phase
    peak, peak_kind = measured_peaks()
    w = 4
    iters_prof = max(pst["pcg_iters"], 1)
    dom = max(prof.items(), key=lambda kv: kv[1][0])
    dom_name, (dom_ms, dom_launch) = dom
    dom_ms_step = dom_ms / args.profile_steps
    nsweeps = max(dom_launch // args.profile_steps, 1) if dom_name == "mic_sweep" else 1
    per_launch_ms = dom_ms / max(dom_launch, 1)
    bytes_step = phase_bytes(dom_name, w, np_, ncell, ndof, iters_prof, nsweeps)
    bytes_launch = bytes_step / max(dom_launch / args.profile_steps, 1)
    achieved = bytes_launch / (per_launch_ms * 1e-3) / 1e9 if per_launch_ms > 0 else 0.0
    traffic = traffic_per_launch(dom_name, ndof, np_)
    roofline = {"bound": "hbm", "kernel": dom_name, "achieved": round(achieved, 1),
                "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4),
                "peak_kind": peak_kind, "traffic": traffic,
                "bytes_per_launch": int(bytes_launch),
                "ms_per_launch": round(per_launch_ms, 4)}
    def phases_of(pr):
        return {k: {"ms_per_step": round(v[0] / args.profile_steps, 3),
                    "launches_per_step": v[1] // args.profile_steps}
                for k, v in pr.items()}

    phases = phases_of(prof)
    # transfer-kernel HBM fractions
    transfers = {}
    for k in ("p2g", "g2p_advect"):
        ms_k = prof[k][0] / args.profile_steps
        if ms_k > 0:
            gbs = phase_bytes(k, w, np_, ncell, ndof, 1, 1) / (ms_k * 1e-3) / 1e9
            transfers[k] = {"GB/s": round(gbs, 1), "frac": round(gbs / peak, 4)}
    out = {
        "metric": METRIC,
        "value": round(main["ms"], 3),
        "unit": "ms/step",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(main["ms"], 3),
        "higher_is_better": False,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded half-filled box, curl-noise velocity)",
        "config": {
            "workload": f"half_box {args.n}^3, {args.ppc} ppc, {np_} particles, dt {DT}, "
                        "MIC(0)-PCG FP32 + FP64 refinement to 1e-6",
            "grid": args.n, "particles": np_, "active_buckets": pst["nactive_buckets"],
            "pressure_dofs": ndof, "precision": "fp32 transfers+PCG, fp64 reductions/refine",
            "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
            "l2": "inputs larger than L2 (particle state %.1f GB)" % (np_ * 80 / 1e9),
        },
        "particle_updates_per_s": round(world * np_ / (main["ms"] * 1e-3), 1),
        "pcg_iters_per_step": main["iters"],
        "refinements": st["refinements"],
        "final_residual_rel": st["residual"] / max(st["rhs_norm"], 1e-300),
        "gpu_launches": int(main["launches"]),
        "launches_per_step": round(main["launches"] / args.steps, 1),
        "phases": phases,
        "roofline": roofline,
        "transfers_hbm": transfers,
        "clocks": main["clocks"],
        "e2e": e2e,
        "scene_gen_s": round(gen_s, 1),
    }
    if fp64:
        out["fp64"] = {"ms_per_step": round(fp64["ms"], 3), "pcg_iters_per_step": fp64["iters"],
                       "speedup_fp32_refine_vs_fp64": round(fp64["ms"] / main["ms"], 3),
                       "clocks": fp64["clocks"], "phases": phases_of(fp64["phases"])}
    if tight:
        out["fp32_refine_1e-8"] = tight
    if mg:
        out["multigrid_pcg"] = dict(mg, note="same step with the reference's default "
                                              "pressure solver (AMGPCGSolveSparse restated)")
    if not args.no_config0:
        out["config0"] = run_config0(dev)
    if not args.no_batch or args.batch_full:
        out["batch"] = run_batch(args)
    if not args.no_cloth:
        out["cloth"] = run_cloth(dev)
    return out


def run_config0(dev, warmup=3, steps=97):
    """The 64^3 dam break (8 per cell, seed 0, 265,302 particles), 100 steps
    from the initial state as the reference arm's config0 runs them (3
    warm-up + 97 timed): ms per step in FP64 and FP32 + refinement with
    MIC(0)-PCG, and FP64 with the multigrid-PCG the reference uses by
    default.  Device time with CUDA events on the context's stream."""
    import torch
    from libwetcloth_b200 import scenes
    from libwetcloth_b200._capi import (WCG_FP32_REFINE, WCG_FP64, WCG_SOLVER_MG,
                                        WCG_SOLVER_MIC0)
    from libwetcloth_b200.solver import FluidScene
    sc = scenes.dam_break(64, 8, 0)
    out = {"workload": f"dam break 64^3, 8 ppc, seed 0, {sc.x.shape[0]} particles, "
                       f"100 steps ({warmup} warm-up + {steps} timed)"}
    for name, prec, solver in (("fp64_mic0", WCG_FP64, WCG_SOLVER_MIC0),
                               ("fp32_refine_mic0", WCG_FP32_REFINE, WCG_SOLVER_MIC0),
                               ("fp64_multigrid", WCG_FP64, WCG_SOLVER_MG)):
        g = FluidScene(sc, precision=prec, solver=solver)
        for _ in range(warmup):
            g.step(DT)
        stream = torch.cuda.ExternalStream(g.stream_ptr, device=f"cuda:{dev}")
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(dev)
        e0.record(stream)
        iters = 0
        for _ in range(steps):
            g.step(DT)
            iters += g.stats()["pcg_iters"]
        e1.record(stream)
        e1.synchronize()
        out[name] = {"ms_per_step": round(e0.elapsed_time(e1) / steps, 3),
                     "mean_pcg_iters": round(iters / steps, 1)}
        g.close()
    return out


def run_cloth(dev, n=128, steps=5, warmup=2, dt=5e-4):
    """The liquid-on-cloth configuration: at 128^3 a liquid sphere (r 0.15,
    8 per cell, falling at 1 m/s) onto a 128 x 128-vertex cloth sheet at
    y = 0.4 (porosity 0.5), dt 5e-4: ms per step of the liquid step with its
    coupling to the sheet (transfers of both phases, drag, pore pressure, the
    solid volume in the pressure system) in FP64 and FP32 + refinement; the
    sheet keeps its transferred velocity (the cloth solve is not part of the
    path).  Device time with CUDA events on the context's stream."""
    import torch
    from libwetcloth_b200 import scenes
    from libwetcloth_b200._capi import WCG_FP32_REFINE, WCG_FP64
    from libwetcloth_b200.solver import FluidScene
    sc = scenes.liquid_on_sheet(n, 8, 3, sheet_spacing=0.8 / 127)
    out = {"grid": n, "liquid_particles": int(sc.x.shape[0]),
           "cloth_vertices": int(sc.elasto.n), "dt": dt, "steps": steps}
    for name, prec in (("fp64", WCG_FP64), ("fp32_refine", WCG_FP32_REFINE)):
        g = FluidScene(sc, precision=prec)
        for _ in range(warmup):
            g.step(dt)
        stream = torch.cuda.ExternalStream(g.stream_ptr, device=f"cuda:{dev}")
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(dev)
        e0.record(stream)
        iters = []
        for _ in range(steps):
            g.step(dt)
            iters.append(g.stats()["pcg_iters"])
        e1.record(stream)
        e1.synchronize()
        out[name] = {"ms_per_step": round(e0.elapsed_time(e1) / steps, 3),
                     "pcg_iters_per_step": iters}
        g.close()
    # the reference Core on the same scene, one step after one warm-up
    from oracle import ref as oref
    if oref.available(omp=True):
        os.environ.setdefault("OMP_NUM_THREADS", str(os.cpu_count() or 1))
        with _quiet_stdout():
            r = oref.RefScene(sc, mic=False, omp=True)
            r.step(dt, snapshot=False)
            t0 = time.perf_counter()
            r.step(dt, snapshot=False)
            ref_ms = (time.perf_counter() - t0) * 1000
            r.close()
        out["reference_cpu"] = {"ms_per_step": round(ref_ms, 1),
                                "cores": int(os.environ["OMP_NUM_THREADS"]),
                                "note": "reference Core (OpenMP stand-in for TBB), one step"}
    return out


def run_batch(args, steps=3):
    """Many independent scenes (grid 32..64 cells, 10k..200k particles,
    seeded densities and viscosities; the many-scenes configuration scaled to
    a short run): aggregate particle-steps/s stepped one after another
    against the batch (separate streams, host thread pool), the batch with
    each scene's launch schedule chosen from timed trials, and the batch
    with the shared solve (every waiting scene's PCG iterations in one launch
    per kernel).  The thread count and the schedules are chosen first on a
    tuning copy of the scenes; every arm then starts from fresh scenes (the
    same initial state), takes one untimed step and times its passes, so all
    arms simulate the same steps.  Device-synchronised wall time around each
    whole pass (best of three; one pass each with --batch-full, which runs
    the configuration at its stated size)."""
    import torch
    from libwetcloth_b200 import scenes
    from libwetcloth_b200._capi import WCG_FP32_REFINE
    from libwetcloth_b200.solver import DEFAULT_SCHEDULES, FluidBatch, FluidScene
    full = getattr(args, "batch_full", False)
    if full:
        specs = scenes.batch_scenes(256, 4, (32, 96), (10_000, 1_000_000))
        steps = 50
    else:
        specs = scenes.batch_scenes(args.batch_scenes, 4, (32, 64), (10_000, 200_000))
    passes = 1 if full else 3
    total_p = sum(sc.x.shape[0] for sc in specs)

    def make():
        return [FluidScene(sc, precision=WCG_FP32_REFINE) for sc in specs]

    def timed_passes(step_all):
        best = float("inf")
        for _ in range(passes):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            step_all()
            torch.cuda.synchronize()
            best = min(best, time.perf_counter() - t0)
        return best

    # tuning copy: thread count, then each scene's launch schedule
    gs = make()
    b = FluidBatch(gs)
    b.step(DT)  # first-step allocations outside the trials
    tune = b.autotune(DT, candidates=(1, 2, 4, 8, 16))
    threads = b.threads
    cands = DEFAULT_SCHEDULES
    chosen, _ = b.autotune_schedules(DT, cands)
    b.close()
    for g in gs:
        g.close()
    hist = {}
    for k in chosen:
        key = "x".join(str(v) for v in cands[k])
        hist[key] = hist.get(key, 0) + 1

    # sequential: one scene after another, each its own steps
    gs = make()
    for g in gs:
        g.step(DT)

    def seq_all():
        for g in gs:
            for _ in range(steps):
                g.step(DT)

    seq_s = timed_passes(seq_all)
    for g in gs:
        g.close()

    def batch_arm(schedules, shared, max_patches=None):
        gs = make()
        if schedules:
            for g, k in zip(gs, chosen):
                g.schedule = cands[k]
        b = FluidBatch(gs)
        b.threads = threads
        if shared:
            b.set_shared_solve(True, max_patches=max_patches)
        b.step(DT)
        l0 = b.shared_launches
        t = timed_passes(lambda: b.step(DT, nsteps=steps))
        launches = (b.shared_launches - l0) // passes
        b.close()
        for g in gs:
            g.close()
        return t, launches

    bat_s, _ = batch_arm(False, False)
    sched_s, _ = batch_arm(True, False)
    shared_s, shared_launches = batch_arm(False, True)
    # the tuned schedules with the shared solve for the scenes of at most 16
    # pencil patches (the larger ones iterate alone on their own streams)
    shared16_s, _ = batch_arm(True, True, 16)
    return {"scenes": len(specs), "particles": total_p, "steps": steps,
            "precision": "fp32_refine",
            "sequential_particle_steps_per_s": round(total_p * steps / seq_s, 1),
            "batched_particle_steps_per_s": round(total_p * steps / bat_s, 1),
            "speedup": round(seq_s / bat_s, 3), "threads": threads,
            "autotune_ms": {str(k): round(v, 2) for k, v in tune.items()},
            "batched_tuned_particle_steps_per_s": round(total_p * steps / sched_s, 1),
            "speedup_tuned": round(seq_s / sched_s, 3),
            "schedules_chosen": hist,
            "schedule_key": "sweep_cluster x sweep_cluster_a x pcg_batch",
            "batched_shared_solve_particle_steps_per_s": round(total_p * steps / shared_s, 1),
            "speedup_shared_solve": round(seq_s / shared_s, 3),
            "shared_solve_launches_per_pass": shared_launches,
            "batched_tuned_shared16_particle_steps_per_s": round(total_p * steps / shared16_s, 1),
            "speedup_tuned_shared16": round(seq_s / shared16_s, 3),
            "note": f"wall time, device-synchronised, warm-up excluded, best of {passes} "
                    "pass(es) per arm, every arm from the same initial state"}


# ---------------------------------------------------------------------------
class _quiet_stdout:
    """Send file descriptor 1 to /dev/null (the reference Core prints solver
    progress with std::cout) so the JSON line stays the only stdout output."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        self.null = os.open(os.devnull, os.O_WRONLY)
        os.dup2(self.null, 1)
        return self

    def __exit__(self, *exc):
        sys.stdout.flush()
        os.dup2(self.saved, 1)
        os.close(self.saved)
        os.close(self.null)
        return False


def run_reference_cpu(args, sample_n, steps=2, warmup=1):
    """cpu_baseline of this arm: the reference Core (oracle/_ref, OpenMP
    stand-in for TBB, all host threads) on a bounded sample -- the same scene
    generator at sample_n^3 -- ms/step scaled by particle count to the full
    workload (the reference arm, --impl reference, times the full workload)."""
    from libwetcloth_b200 import scenes
    from oracle import ref as oref
    if not oref.available(omp=True):
        return None, "oracle/_ref/libwcref_omp.so not built"
    cores = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    sc = scenes.half_box(sample_n, args.ppc, seed=1)
    with _quiet_stdout():
        r = oref.RefScene(sc, mic=False, omp=True)
        for _ in range(warmup):
            r.step(DT, snapshot=False)
        t0 = time.perf_counter()
        for _ in range(steps):
            r.step(DT, snapshot=False)
        dt = (time.perf_counter() - t0) / steps
        r.close()
    n_sample = sc.x.shape[0]
    full_np = args.ppc * args.n * (args.n // 2) * args.n
    scale = full_np / n_sample
    return {"value": round(dt * 1000 * scale, 1), "unit": "ms/step",
            "cores": int(os.environ.get("OMP_NUM_THREADS", cores)), "kind": "reference",
            "sample": f"reference Core (multigrid-PCG default solver) on half_box "
                      f"{sample_n}^3/{n_sample} particles, {steps} steps after {warmup} "
                      f"warm-up, {dt*1000:.1f} ms/step x {scale:.1f} (particle ratio); "
                      f"OpenMP stand-in for TBB; the full workload is timed by "
                      f"--impl reference"}, None


def _ref_child(spec):
    """Child process of the reference arm: the reference Core on one scene,
    `warmup` untimed then up to `steps` timed WetClothCore steps, stopping
    early (and saying so) when the next step would pass the deadline.  Prints
    one JSON line; progress with the resident set size goes to stderr."""
    import resource
    from libwetcloth_b200 import scenes
    from oracle import ref as oref
    t_start = time.time()
    if spec["scene"] == "half_box":
        sc = scenes.half_box(spec["n"], spec["ppc"], seed=1)
    else:
        sc = scenes.dam_break(spec["n"], 8, 0)
    rss = lambda: resource.getrusage(resource.RUSAGE_SELF).ru_maxrss / 1e6
    print(f"scene {sc.x.shape[0]} particles, rss {rss():.1f} GB", file=sys.stderr, flush=True)
    with _quiet_stdout():
        r = oref.RefScene(sc, mic=spec["mic"], omp=True)
        print(f"created, rss {rss():.1f} GB", file=sys.stderr, flush=True)
        for k in range(spec["warmup"]):
            r.step(DT, snapshot=False)
            print(f"warm-up step {k}, rss {rss():.1f} GB", file=sys.stderr, flush=True)
        times = []
        while len(times) < spec["steps"]:
            if times and time.time() + max(times) > t_start + spec["budget_s"]:
                break
            t0 = time.perf_counter()
            r.step(DT, snapshot=False)
            times.append(time.perf_counter() - t0)
            print(f"step {len(times)}: {times[-1]:.2f} s, rss {rss():.1f} GB", file=sys.stderr,
                  flush=True)
        iters = r.amg_stats()[0] if not spec["mic"] else r.solver_stats()[0]
        r.close()
    print(json.dumps({"ms_per_step": 1000.0 * sum(times) / len(times), "steps": len(times),
                      "particles": int(sc.x.shape[0]), "rss_gb": round(rss(), 2),
                      "last_solver_iters": int(iters)}), flush=True)


def _run_ref_child(spec, timeout_s):
    """Runs _ref_child in a fresh interpreter; returns (result, None) or
    (None, why) when the child failed (out of memory, killed, timed out)."""
    cmd = [sys.executable, os.path.abspath(__file__), "--ref-child", json.dumps(spec)]
    try:
        out = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout_s, cwd=ROOT)
    except subprocess.TimeoutExpired as e:
        err = (e.stderr or b"").decode(errors="replace") if isinstance(e.stderr, bytes) else \
            (e.stderr or "")
        return None, f"timed out after {timeout_s} s; last progress: {err.strip()[-200:]}"
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    if out.returncode != 0 or not lines:
        return None, (f"reference process exited with status {out.returncode}; "
                      f"last progress: {out.stderr.strip()[-300:]}")
    return json.loads(lines[-1]), None


def run_reference_arm(args, world):
    """--impl reference: the reference's own CPU implementation of the path
    (the compiled reference Core, oracle/_ref/libwcref_omp.so, OpenMP
    stand-in for TBB, all host threads) on this arm's workload -- the
    half_box n^3 scene at ppc particles per cell, seeded as in the GPU arm --
    for the requested warm-up and timed steps, with its default solver
    (multigrid-PCG, as solveNodePressure calls it).  A MIC(0)-PCG run of the
    same scene (the GPU headline's solver) and the 64^3 dam break
    (100 steps) follow as sub-objects."""
    from oracle import ref as oref
    if not oref.available(omp=True):
        return {"impl": "reference", "unavailable": "oracle/_ref/libwcref_omp.so not built"}
    cores = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    threads = int(os.environ["OMP_NUM_THREADS"])
    spec = {"scene": "half_box", "n": args.n, "ppc": args.ppc, "mic": False,
            "warmup": args.warmup, "steps": args.steps, "budget_s": args.ref_budget_s}
    main, why = _run_ref_child(spec, args.ref_budget_s + 900)
    if main is None:
        return {"impl": "reference",
                "unavailable": f"reference Core on half_box {args.n}^3: {why}"}
    value = round(main["ms_per_step"], 1)
    workload = (f"half_box {args.n}^3, {args.ppc} ppc, {main['particles']} particles, dt {DT}, "
                "reference Core WetClothCore::stepSystem, multigrid-PCG to 1e-6")
    out = {
        "metric": METRIC, "value": value, "unit": "ms/step", "impl": "reference",
        "n_gpus": world, "steps": main["steps"], "warmup": args.warmup,
        "ms_per_step": value, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded half-filled box, "
                                                     "curl-noise velocity)",
        "config": {"workload": workload, "grid": args.n, "particles": main["particles"],
                   "threads": threads, "rss_gb": main["rss_gb"]},
        "cpu_baseline": {"value": value, "unit": "ms/step", "cores": threads,
                         "kind": "reference",
                         "sample": f"the full workload: {main['steps']} steps after "
                                   f"{args.warmup} warm-up (OpenMP stand-in for TBB)"},
        "e2e": {"value": value, "unit": "ms/step", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    if main["steps"] < args.steps:
        out["steps_requested"] = args.steps
        out["note"] = (f"stopped after {main['steps']} timed steps: the next would have "
                       f"passed the {args.ref_budget_s} s budget")
    if not args.no_ref_mic:
        spec_mic = dict(spec, mic=True, warmup=1, steps=1, budget_s=900)
        mic, why = _run_ref_child(spec_mic, 1800)
        out["mic0"] = ({"ms_per_step": round(mic["ms_per_step"], 1), "steps": mic["steps"],
                        "warmup": 1, "pcg_iters": mic["last_solver_iters"],
                        "note": "the same scene with the assembled system re-solved by the "
                                "reference's own PCGSolver<double> (MIC(0)), the GPU "
                                "headline's solver"} if mic else {"unavailable": why})
    if not args.no_config0:
        spec0 = {"scene": "dam_break", "n": 64, "ppc": 8, "mic": False, "warmup": 3,
                 "steps": 97, "budget_s": 900}
        c0, why = _run_ref_child(spec0, 1500)
        out["config0"] = ({"workload": "dam break 64^3, 8 ppc, seed 0, 265302 particles, "
                                       "100 steps (3 warm-up + 97 timed)",
                           "ms_per_step": round(c0["ms_per_step"], 2), "steps": c0["steps"],
                           "warmup": 3} if c0 else {"unavailable": why})
    return out


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.ref_child:
        _ref_child(json.loads(args.ref_child))
        return 0
    if args.impl == "reference":
        if rank != 0:
            return 0
        print(json.dumps(run_reference_arm(args, world)))
        return 0
    import torch
    if world > 1:
        torch.cuda.set_device(local)
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    else:
        torch.cuda.set_device(0)
    dev = torch.cuda.current_device()
    out = run_ours(args, rank, world, dev)
    if rank == 0 and not args.no_cpu_baseline:
        cpu, why = run_reference_cpu(args, args.cpu_sample_n)
        out["cpu_baseline"] = cpu if cpu else {"unavailable": why}
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if rank == 0:
        print(json.dumps(out))
    return 0


if __name__ == "__main__":
    sys.exit(main())
