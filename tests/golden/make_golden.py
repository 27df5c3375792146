"""Generate the golden fixtures from the compiled reference Core.

Runs oracle/_ref/libwcref.so (the libWetCloth reference built from its own
sources by oracle/ref.mk, serial TBB stand-in) on two tiny seeded liquid
scenes and stores the inputs plus every hot-path field of the first step, and
the particle state after three steps, as compressed .npz files next to this
script.  Node fields keep only the nodes of active buckets (the reference
stores nothing for inactive buckets).

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from libwetcloth_b200 import scenes  # noqa: E402
from oracle import ref as oref  # noqa: E402

DT = 1e-3

INT_FIELDS = ["grid_dims", "array_idx", "array_sup", "active", "stencil_base", "inside",
              "dof_index", "A_rowstart", "A_col", "valid_x", "valid_y", "valid_z"]
FLT_FIELDS = ["grid_origin", "bbx", "A_val", "b", "g2p_v", "g2p_C", "adv_x"]
NODE_FIELDS = ["mass_fluid_x", "mass_fluid_y", "mass_fluid_z", "vel_fluid_x", "vel_fluid_y",
               "vel_fluid_z", "vol_fluid_x", "vol_fluid_y", "vol_fluid_z", "sat_x", "sat_y",
               "sat_z", "sat_p", "liquid_phi", "solid_phi", "solid_weight_x",
               "solid_weight_y", "solid_weight_z", "v_star_x", "v_star_y", "v_star_z",
               "psi_fs_x", "psi_fs_y", "psi_fs_z", "pressure", "u_final_x", "u_final_y",
               "u_final_z"]


def golden_scenes():
    """The two fixture scenes (seeded, a few hundred particles each)."""
    dx = 1.0 / 16.0
    x = scenes.liquid_block(dx, (0.0, 0.0, 0.0), (0.25, 0.5, 0.25), 8, seed=11)
    m, vol, r = scenes.attributes(x.shape[0], dx, 8, 1000.0)
    dam = scenes.Scene(scenes.SceneParams(dx=dx), x, np.zeros_like(x), m, vol, r,
                       name="golden_dam")
    x2 = scenes.liquid_block(dx, (0.3, 0.0, 0.3), (0.7, 0.3, 0.7), 2, seed=12)
    v2 = scenes.curl_noise_velocity(x2, 16, 1.5, 0.5, seed=13)
    m2, vol2, r2 = scenes.attributes(x2.shape[0], dx, 2, 1000.0)
    curl = scenes.Scene(scenes.SceneParams(dx=dx), x2, v2, m2, vol2, r2, name="golden_curl")
    return [dam, curl]


def main():
    assert oref.available(), "build oracle/_ref first (make -f oracle/ref.mk)"
    for sc in golden_scenes():
        r = oref.RefScene(sc, mic=True)
        r.step(DT, snapshot=True)
        out = {"x": sc.x, "v": sc.v, "mass": sc.mass, "vol": sc.vol, "radius": sc.radius,
               "dx": np.array([sc.params.dx])}
        it, res = r.solver_stats()
        out["pcg_iters"] = np.array([it])
        act = r.get("active").astype(bool)
        node_mask = np.repeat(act, 64)
        for k in INT_FIELDS:
            out[k] = r.get(k)
        for k in FLT_FIELDS:
            out[k] = r.get(k)
        for k in NODE_FIELDS:
            out["node_" + k] = r.get(k)[node_mask]
        r.step(DT, snapshot=False)
        r.step(DT, snapshot=True)
        out["step3_x"] = r.get("adv_x")
        out["step3_v"] = r.get("g2p_v")
        out["step3_C"] = r.get("g2p_C")
        path = os.path.join(HERE, sc.name + ".npz")
        np.savez_compressed(path, **out)
        print(path, sc.x.shape[0], "particles", os.path.getsize(path) // 1024, "KiB")
        r.close()


if __name__ == "__main__":
    main()
