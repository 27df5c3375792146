"""Digests of the oracle's state on two benchmark configurations whose oracle
runs are too slow for the GPU test session (minutes on one host core):

* config0_dam64.npz -- the 64^3 dam break (dx 1/64, block [0,0.4]x[0,0.8]x[0,0.4],
  8 jittered particles per cell, seed 0; 265,302 particles), FP64, dt 1e-3:
  the state after 10 and after 100 steps;
* config1_sheet128.npz -- the 128^3 liquid sphere (r 0.15 at (0.5, 0.75,
  0.5), 8 per cell, falling at 1 m/s, seed 3; 237,046 particles) onto the
  128 x 128-vertex cloth sheet at y = 0.4, FP64, dt 5e-4: the state after 20
  and after 200 steps (liquid digest as above; the sheet's positions and
  velocities at a seeded sample of its vertices, with their sums);
* config2_half256.npz -- the 256^3 half-filled box (2 per cell, curl-noise
  velocity sigma 4 cells, amplitude 0.5, seed 1; 16,777,216 particles), FP64,
  dt 1e-3: the state after the first step.

Each digest holds 2048 seeded particle indices with their positions,
velocities and affine matrices, whole-set sums and norms of x and v, and the
MIC(0)-PCG iteration count of every step.  The oracle is the C restatement
(oracle/wc_oracle.c), itself pinned to the compiled reference; it is
deterministic (serial, no FMA contraction), so the digests are reproducible
on any host with the same build.

    python tests/golden/make_config_digests.py [config0|config1|config2]
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from libwetcloth_b200 import scenes  # noqa: E402
from oracle import oracle as oo  # noqa: E402

DT = 1e-3
NSAMPLE = 2048


def sample_indices(n, seed):
    return np.sort(np.random.default_rng(seed).choice(n, NSAMPLE, replace=False))


def summary(prefix, x, v, C, idx):
    return {
        prefix + "x": x[idx], prefix + "v": v[idx], prefix + "C": C[idx],
        prefix + "x_sum": x.sum(axis=0), prefix + "v_sum": v.sum(axis=0),
        prefix + "v_sq": np.array([(v * v).sum()]), prefix + "v_absmax": np.array([np.abs(v).max()]),
    }


def config0(steps=(10, 100)):
    sc = scenes.dam_break(64, 8, 0)
    n = sc.x.shape[0]
    idx = sample_indices(n, 64)
    o = oo.OracleScene(sc)
    out = {"idx": idx, "n": np.array([n])}
    iters = []
    t0 = time.time()
    for k in range(1, max(steps) + 1):
        snap = k in steps
        o.step(DT, snapshot=snap)
        iters.append(o.solver_stats()[0])
        if snap:
            x = o.get("adv_x").reshape(-1, 3)
            v = o.get("g2p_v").reshape(-1, 3)
            C = o.get("g2p_C").reshape(-1, 9)
            out.update(summary(f"s{k}_", x, v, C, idx))
            print(f"config0 step {k}: {time.time() - t0:.0f} s", flush=True)
    out["iters"] = np.array(iters)
    o.close()
    np.savez_compressed(os.path.join(HERE, "config0_dam64.npz"), **out)


def config1(steps=(20, 200)):
    dt = 5e-4
    sc = scenes.liquid_on_sheet(128, 8, 3, sheet_spacing=0.8 / 127)
    ne = sc.elasto.n
    n = sc.x.shape[0]
    idx = sample_indices(n, 128)
    sidx = sample_indices(ne, 129)
    o = oo.OracleScene(sc)
    out = {"idx": idx, "sheet_idx": sidx, "n": np.array([n]), "ne": np.array([ne])}
    iters = []
    t0 = time.time()
    for k in range(1, max(steps) + 1):
        snap = k in steps
        o.step(dt, snapshot=snap)
        iters.append(o.solver_stats()[0])
        if snap:
            x = o.get("adv_x").reshape(-1, 3)[ne:]
            v = o.get("g2p_v").reshape(-1, 3)[ne:]
            C = o.get("g2p_C").reshape(-1, 9)[ne:]
            out.update(summary(f"s{k}_", x, v, C, idx))
            x4 = o.get("adv_x4").reshape(-1, 4)[:ne]
            v4 = o.get("adv_ev4").reshape(-1, 4)[:ne]
            out[f"s{k}_sheet_x4"] = x4[sidx]
            out[f"s{k}_sheet_v4"] = v4[sidx]
            out[f"s{k}_sheet_x4_sum"] = x4.sum(axis=0)
            out[f"s{k}_sheet_v4_sum"] = v4.sum(axis=0)
            out[f"s{k}_sheet_v4_sq"] = np.array([(v4 * v4).sum()])
            print(f"config1 step {k}: {time.time() - t0:.0f} s", flush=True)
    out["iters"] = np.array(iters)
    o.close()
    np.savez_compressed(os.path.join(HERE, "config1_sheet128.npz"), **out)


def config2():
    sc = scenes.half_box(256, 2, seed=1)
    n = sc.x.shape[0]
    idx = sample_indices(n, 256)
    o = oo.OracleScene(sc)
    t0 = time.time()
    o.step(DT, snapshot=False)  # per-stage snapshots would not fit in host memory
    print(f"config2 step: {time.time() - t0:.0f} s", flush=True)
    o.snap_state("final_")
    x = o.get("final_x").reshape(-1, 3)
    v = o.get("final_v").reshape(-1, 3)
    C = o.get("final_C").reshape(-1, 9)
    out = {"idx": idx, "n": np.array([n]), "iters": np.array([o.solver_stats()[0]])}
    out.update(summary("s1_", x, v, C, idx))
    o.close()
    np.savez_compressed(os.path.join(HERE, "config2_half256.npz"), **out)


if __name__ == "__main__":
    which = sys.argv[1:] or ["config0", "config1", "config2"]
    if "config0" in which:
        config0()
    if "config1" in which:
        config1()
    if "config2" in which:
        config2()
