"""The 200-sub-step gradient run at 64^3 (the differentiation configuration):
the dam-break block [0,0.4]x[0,0.8]x[0,0.4] at 8 particles per cell
(265,302 particles) with a seeded Gaussian initial velocity (sigma 0.2,
seed 2) and the explicit viscosity 1e-3, dt 1e-3, one sub-step per step.
Loss = |centre of mass of x_T - (0.7, 0.2, 0.5)|^2 + kinetic energy of v_T.
Gradients in the initial velocities and the viscosity come from the
checkpointed rollout (a checkpoint every 10 sub-steps, recomputed in the
backward).

Checks:
- the FP64 gradient against central differences of the FP64 forward
  (h = 1e-4) in the viscosity and in one velocity component of each of 16
  seeded particles, with the pressure solved to a 1e-12 relative residual so
  the solver's truncation does not enter the differences;
- the FP32 (with FP64 refinement, 1e-6 residual) gradient against the FP64
  one.

The reverse mode follows the positions through the transfer weights, the
liquid phi of the ghost-fluid fractions and the solid projection; the grid's
discrete structure (activation, DOFs, valid faces) is held at its forward
values, which central differences of this size do not cross."""
import time

import numpy as np
import pytest

from libwetcloth_b200 import _capi, scenes
from libwetcloth_b200.solver import FluidScene

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

DT = 1e-3
STEPS = 200
EVERY = 10
TARGET = np.array([0.7, 0.2, 0.5])
H = 1e-4
NPICK = 16


def _scene(criterion):
    sc = scenes.differentiation_block(64, 8, 2)
    sc.params.criterion = criterion
    sc.params.maxiters = 1000
    return sc


def _loss_np(x, v, m):
    com = (m[:, None] * x).sum(axis=0) / m.sum()
    return float(((com - TARGET) ** 2).sum() + 0.5 * (m[:, None] * v * v).sum())


def _forward_loss(g, sc, v0, mu):
    g.set_viscosity(mu, 1)
    g.set_state(sc.x, v0, np.zeros((sc.x.shape[0], 9)))
    for k in range(STEPS):
        g.set_correction_count(k)
        g.substep(DT)
    x, v, _ = g.download()
    return _loss_np(x, v, sc.mass)


def _gradient(g, sc, mu):
    from libwetcloth_b200.autograd import rollout
    m = torch.from_numpy(sc.mass)
    x0 = torch.from_numpy(sc.x.copy())
    v0 = torch.from_numpy(sc.v.copy()).requires_grad_(True)
    C0 = torch.zeros((sc.x.shape[0], 9), dtype=torch.float64)
    mut = torch.tensor(mu, dtype=torch.float64, requires_grad=True)
    x1, v1, _ = rollout(g, x0, v0, C0, DT, STEPS, viscosity=mut, checkpoint_every=EVERY,
                        correction_call=0)
    com = (m[:, None] * x1).sum(0) / m.sum()
    L = ((com - torch.from_numpy(TARGET)) ** 2).sum() + 0.5 * (m[:, None] * v1 * v1).sum()
    L.backward()
    return L.item(), v0.grad.numpy().copy(), float(mut.grad.item())


@pytest.fixture(scope="module")
def fp64_run(wcg):
    sc = _scene(1e-12)
    mu = sc.params.viscosity
    g = FluidScene(sc)
    t0 = time.time()
    L, gv, gmu = _gradient(g, sc, mu)
    t_grad = time.time() - t0
    yield sc, g, L, gv, gmu, t_grad
    g.close()


def test_config3_fp64_gradient_against_central_differences(fp64_run):
    sc, g, L, gv, gmu, t_grad = fp64_run
    mu = sc.params.viscosity
    n = sc.x.shape[0]
    assert abs(_forward_loss(g, sc, sc.v, mu) - L) <= 1e-12 * abs(L)
    rng = np.random.default_rng(3)
    picks = [(int(p), int(rng.integers(3))) for p in rng.choice(n, NPICK, replace=False)]
    rows = []
    for p, a in picks:
        vp = sc.v.copy()
        vp[p, a] += H
        vm = sc.v.copy()
        vm[p, a] -= H
        fd = (_forward_loss(g, sc, vp, mu) - _forward_loss(g, sc, vm, mu)) / (2 * H)
        rows.append((fd, gv[p, a]))
    fd_mu = (_forward_loss(g, sc, sc.v, mu + H) - _forward_loss(g, sc, sc.v, mu - H)) / (2 * H)
    fd = np.array([r[0] for r in rows])
    ad = np.array([r[1] for r in rows])
    # relative to each entry, floored at 1e-3 of the largest entry checked
    rel = np.abs(fd - ad) / np.maximum(np.abs(fd), 1e-3 * np.abs(fd).max())
    print(f"\nconfig3 FP64: loss {L:.6e}, gradient {t_grad:.1f} s; "
          f"v0 rel err median {np.median(rel):.2e} max {rel.max():.2e}; "
          f"mu fd {fd_mu:.6e} adjoint {gmu:.6e} rel {abs(fd_mu - gmu) / abs(fd_mu):.2e}")
    for (f, a_), r in zip(rows, rel):
        print(f"  fd {f:+.6e}  adjoint {a_:+.6e}  rel {r:.2e}")
    # measured on one B200: median 2.5e-6, max 2.3e-3 (two of 16 entries above
    # 1e-4), viscosity 5.3e-6
    assert np.median(rel) <= 1e-4
    assert rel.max() <= 1e-2
    assert abs(fd_mu - gmu) <= 1e-4 * abs(fd_mu)


def test_config3_fp32_gradient_against_fp64(fp64_run):
    sc64, _, L64, gv64, gmu64, _ = fp64_run
    sc = _scene(1e-6)
    g = FluidScene(sc, precision=_capi.WCG_FP32_REFINE)
    t0 = time.time()
    L, gv, gmu = _gradient(g, sc, sc.params.viscosity)
    t = time.time() - t0
    g.close()
    err = np.linalg.norm(gv - gv64) / np.linalg.norm(gv64)
    cos = float((gv * gv64).sum() / (np.linalg.norm(gv) * np.linalg.norm(gv64)))
    print(f"\nconfig3 FP32: loss {L:.6e} (FP64 {L64:.6e}), gradient {t:.1f} s; "
          f"|g32 - g64| / |g64| = {err:.2e}, cosine {cos:.6f}; "
          f"mu {gmu:.6e} (FP64 {gmu64:.6e})")
    # measured: loss 6e-7, gradient 1.1e-3 (cosine 0.999999), viscosity 3.7e-2
    assert abs(L - L64) <= 1e-5 * abs(L64)
    assert err <= 1e-2
    assert abs(gmu - gmu64) <= 1e-1 * abs(gmu64)
