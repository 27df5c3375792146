"""Host-side logic on CPU: scene generators, the bench byte model and JSON of
the reference arm, and the multi-process (replica) timing reduction over
gloo with two ranks."""
import json
import math
import os
import socket
import subprocess
import sys

import numpy as np
import pytest

from libwetcloth_b200 import scenes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_particle_volume_is_fraction_of_cell():
    for ppc in (1, 2, 8):
        r = scenes.particle_radius(1 / 64, ppc)
        vol = 4 / 3 * math.pi * r ** 3
        assert abs(vol - (1 / 64) ** 3 / ppc) < 1e-18


def test_liquid_block_counts_and_seed():
    a = scenes.liquid_block(1 / 16, (0, 0, 0), (0.25, 0.5, 0.25), 8, seed=3)
    b = scenes.liquid_block(1 / 16, (0, 0, 0), (0.25, 0.5, 0.25), 8, seed=3)
    assert np.array_equal(a, b)
    assert a.shape == (8 * 16 * 8, 3)  # one particle per (dx/2)^3 sub-cell
    assert a.min() >= 0 and a[:, 1].max() <= 0.5 + 1e-12
    c = scenes.liquid_block(1 / 16, (0, 0, 0), (0.5, 0.25, 0.5), 2, seed=1)
    assert c.shape[0] == 2 * 8 * 4 * 8


def test_curl_noise_is_nearly_divergence_free():
    n = 16
    g = (np.arange(n) + 0.5) / n
    z, y, x = np.meshgrid(g, g, g, indexing="ij")
    pts = np.stack([x.ravel(), y.ravel(), z.ravel()], 1)
    v = scenes.curl_noise_velocity(pts, n, 2.0, 0.5, seed=1)
    assert np.abs(v).max() <= 0.5 + 1e-9
    V = v.reshape(n, n, n, 3)
    h = 1.0 / n
    div = ((np.roll(V[..., 0], -1, 2) - np.roll(V[..., 0], 1, 2)) +
           (np.roll(V[..., 1], -1, 1) - np.roll(V[..., 1], 1, 1)) +
           (np.roll(V[..., 2], -1, 0) - np.roll(V[..., 2], 1, 0))) / (2 * h)
    grad_scale = np.abs(np.gradient(V[..., 0], h, axis=2)).mean()
    assert np.abs(div).mean() < 0.2 * grad_scale


def test_bench_byte_model():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.phase_bytes("p2g", 4, 100, 64, 50, 1, 1) == 100 * 17 * 4 + 64 * 12 * 4
    assert bench.phase_bytes("mic_sweep", 8, 0, 0, 10, 1, 2) == 10 * 6 * 8 * 2
    assert bench.phase_bytes("pcg_vector", 4, 0, 0, 10, 3, 1) == 10 * 20 * 4 * 3


def test_bench_reference_arm_json():
    from oracle import ref as oref
    if not oref.available(omp=True):
        pytest.skip("oracle/_ref/libwcref_omp.so not built")
    env = dict(os.environ, OMP_NUM_THREADS="2")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--steps", "2", "--warmup", "1", "--n", "16", "--no-config0"],
                         capture_output=True, text=True, env=env, timeout=300, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    line = [l for l in out.stdout.splitlines() if l.startswith("{")][-1]
    d = json.loads(line)
    assert d["impl"] == "reference" and d["unit"] == "ms/step" and d["value"] > 0
    # the arm runs the workload it names, for the steps it reports
    assert d["steps"] == 2 and d["warmup"] == 1
    assert d["config"]["grid"] == 16 and d["config"]["particles"] > 0
    assert d["cpu_baseline"]["kind"] == "reference"
    assert d["e2e"]["h2d_bytes_per_step"] == 0
    assert d["mic0"]["ms_per_step"] > 0 and d["mic0"]["pcg_iters"] > 0


def _gloo_worker(rank, world, port, q):
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    v = bench.reduce_max(float(rank + 1) * 10.0, world, "cpu")
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, v))


def test_replica_timing_reduction_gloo():
    import torch.multiprocessing as mp
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_gloo_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = [q.get(timeout=120) for _ in ps]
    for p in ps:
        p.join(timeout=60)
    assert sorted(res) == [(0, 20.0), (1, 20.0)]
