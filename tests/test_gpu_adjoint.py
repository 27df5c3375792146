"""Reverse mode of liquid sub-steps (wcg_substep_vjp, libwetcloth_b200.autograd).

At fixed positions the sub-step is affine in the particles' velocities v and
affine matrices C, so central differences of the forward are exact up to
rounding and the solver tolerance.  In the positions it is smooth away from
the free surface and the walls (the transfer weights are C^1 quadratic
B-splines; the grid's structure and the ghost-fluid fractions only move with
particles near the surface), so the position derivative is checked on
directions carried by interior particles.  Checks, at a 1e-12 pressure
criterion:
- the adjoint identity <y, J d> = <J^T y, d> for random d and y, with J d from
  central differences of the GPU forward (FP64: 1e-9 relative; FP32 with FP64
  refinement: 1e-4);
- the same with J d from central differences of the FP64 oracle, the C
  restatement pinned to the reference (an FP64 reference gradient: 1e-6);
- torch.autograd gradients of a scalar loss against per-entry central
  differences (1e-4 relative, the tolerance the plan states);
- with the explicit viscosity on: the same identity, and the viscosity's
  cotangent against a central difference in mu;
- the position cotangent: the identity for directions in x (interior
  particles), FP64 and FP32 with refinement; wcg_set_adjoint_positions(0)
  passing x-bar through;
- rollout (checkpointed every k sub-steps, recomputed in the backward):
  gradients equal to the chain of single sub-steps."""
import numpy as np
import pytest

from libwetcloth_b200 import _capi, scenes
from libwetcloth_b200.solver import FluidScene
from oracle import oracle as oo

pytestmark = pytest.mark.gpu
DT = 1e-3


def _scene(kind):
    if kind == "dam16":
        sc = scenes.dam_break(16, 8, 0)
    else:
        sc = scenes.half_box(24, 2, 7, amplitude=1.0, sigma_cells=1.5)
    sc.params.criterion = 1e-12
    rng = np.random.default_rng(11)
    sc.C = rng.normal(0.0, 2.0, (sc.x.shape[0], 9))
    return sc


def _forward(g, x, v, C, call=0):
    """One sub-step; the particle correction (run in every sub-step) takes
    the subset of call `call` of the seeded stream, so every evaluation of
    the forward (and the reverse mode) uses the same one."""
    g.set_state(x, v, C)
    g.set_correction_count(call)
    g.substep(DT)
    x1, v1, C1 = g.download()
    return np.concatenate([v1.ravel(), C1.ravel(), x1.ravel()])


def _oracle_forward(sc, v, C):
    s2 = scenes.Scene(sc.params, sc.x.copy(), v.copy(), sc.mass, sc.vol, sc.radius, C=C.copy())
    o = oo.OracleScene(s2)
    o.L.wco_substep(o.h, DT, 1)
    n = sc.x.shape[0]
    out = np.concatenate([o.get("g2p_v"), o.get("g2p_C"), o.get("adv_x")])
    o.close()
    assert out.shape[0] == 15 * n
    return out


def _directions(n, seed):
    rng = np.random.default_rng(seed)
    dv = rng.normal(size=(n, 3))
    dC = rng.normal(size=(n, 9)) * 10.0
    y = rng.normal(size=15 * n)
    return dv, dC, y


def _vjp(g, sc, y, call=0):
    n = sc.x.shape[0]
    g.set_state(sc.x, sc.v, sc.C)
    g.set_correction_count(call)
    vb, Cb, xb = g.substep_vjp(DT, y[:3 * n].reshape(n, 3), y[3 * n:12 * n].reshape(n, 9),
                               y[12 * n:].reshape(n, 3))
    return vb, Cb


@pytest.mark.parametrize("kind", ["dam16", "curl24"])
def test_adjoint_identity_fp64(kind, wcg):
    sc = _scene(kind)
    n = sc.x.shape[0]
    g = FluidScene(sc)
    dv, dC, y = _directions(n, 3)
    h = 1e-2
    Jd = (_forward(g, sc.x, sc.v + h * dv, sc.C + h * dC) -
          _forward(g, sc.x, sc.v - h * dv, sc.C - h * dC)) / (2 * h)
    vb, Cb = _vjp(g, sc, y)
    lhs = float(y @ Jd)
    rhs = float((vb * dv).sum() + (Cb * dC).sum())
    assert abs(lhs - rhs) <= 1e-9 * max(abs(lhs), np.abs(y).sum() * 1e-12), (lhs, rhs)
    g.close()


def test_adjoint_identity_fp32_refine(wcg):
    sc = _scene("curl24")
    n = sc.x.shape[0]
    g = FluidScene(sc, precision=_capi.WCG_FP32_REFINE)
    dv, dC, y = _directions(n, 5)
    h = 1e-1
    Jd = (_forward(g, sc.x, sc.v + h * dv, sc.C + h * dC) -
          _forward(g, sc.x, sc.v - h * dv, sc.C - h * dC)) / (2 * h)
    vb, Cb = _vjp(g, sc, y)
    lhs = float(y @ Jd)
    rhs = float((vb * dv).sum() + (Cb * dC).sum())
    assert abs(lhs - rhs) <= 1e-4 * abs(lhs), (lhs, rhs)
    g.close()


def test_adjoint_against_fp64_oracle(wcg):
    """J d from the C restatement (pinned to the reference), J^T y from the
    GPU reverse mode."""
    sc = _scene("dam16")
    n = sc.x.shape[0]
    dv, dC, y = _directions(n, 9)
    h = 1e-2
    Jd = (_oracle_forward(sc, sc.v + h * dv, sc.C + h * dC) -
          _oracle_forward(sc, sc.v - h * dv, sc.C - h * dC)) / (2 * h)
    g = FluidScene(sc)
    vb, Cb = _vjp(g, sc, y)
    lhs = float(y @ Jd)
    rhs = float((vb * dv).sum() + (Cb * dC).sum())
    assert abs(lhs - rhs) <= 1e-6 * abs(lhs), (lhs, rhs)
    g.close()


def test_autograd_against_central_differences(wcg):
    torch = pytest.importorskip("torch")
    from libwetcloth_b200.autograd import substep
    sc = _scene("curl24")
    n = sc.x.shape[0]
    g = FluidScene(sc)
    rng = np.random.default_rng(2)
    wx = torch.from_numpy(rng.normal(size=(n, 3)))
    target = torch.from_numpy(rng.normal(size=(n, 3)))

    def loss_of(v, C):
        x1, v1, C1 = substep(g, torch.from_numpy(sc.x), v, C, DT, correction_call=0)
        return ((v1 - target) ** 2).sum() + (x1 * wx).sum() + 1e-3 * (C1 ** 2).sum()

    v = torch.from_numpy(sc.v.copy()).requires_grad_(True)
    C = torch.from_numpy(sc.C.copy()).requires_grad_(True)
    L = loss_of(v, C)
    L.backward()
    gv, gC = v.grad.numpy().copy(), C.grad.numpy().copy()
    h = 1e-3
    for (arr, grad, name) in ((sc.v, gv, "v"), (sc.C, gC, "C")):
        for idx in rng.choice(arr.size, 6, replace=False):
            p = arr.copy().ravel()
            p[idx] += h
            m = arr.copy().ravel()
            m[idx] -= h
            if name == "v":
                lp = loss_of(torch.from_numpy(p.reshape(arr.shape)), torch.from_numpy(sc.C)).item()
                lm = loss_of(torch.from_numpy(m.reshape(arr.shape)), torch.from_numpy(sc.C)).item()
            else:
                lp = loss_of(torch.from_numpy(sc.v), torch.from_numpy(p.reshape(arr.shape))).item()
                lm = loss_of(torch.from_numpy(sc.v), torch.from_numpy(m.reshape(arr.shape))).item()
            fd = (lp - lm) / (2 * h)
            gr = grad.ravel()[idx]
            assert abs(fd - gr) <= 1e-4 * max(abs(fd), np.abs(grad).max() * 1e-3), (name, idx, fd, gr)
    g.close()


@pytest.mark.parametrize("substeps", [1, 3])
def test_adjoint_identity_with_viscosity(substeps, wcg):
    """The explicit viscosity steps are linear in v*, so the identity holds
    with them on; the viscosity cotangent matches a central difference in mu
    (the step is a polynomial of degree `substeps` in mu)."""
    sc = _scene("curl24")
    mu = 0.5
    sc.params.viscosity = mu
    sc.params.viscosity_substeps = substeps
    n = sc.x.shape[0]
    g = FluidScene(sc)
    dv, dC, y = _directions(n, 13)
    h = 1e-2
    Jd = (_forward(g, sc.x, sc.v + h * dv, sc.C + h * dC) -
          _forward(g, sc.x, sc.v - h * dv, sc.C - h * dC)) / (2 * h)
    g.set_state(sc.x, sc.v, sc.C)
    g.set_correction_count(0)
    vb, Cb, xb, mub = g.substep_vjp(DT, y[:3 * n].reshape(n, 3), y[3 * n:12 * n].reshape(n, 9),
                                    y[12 * n:].reshape(n, 3), with_viscosity=True)
    lhs = float(y @ Jd)
    rhs = float((vb * dv).sum() + (Cb * dC).sum())
    assert abs(lhs - rhs) <= 1e-9 * abs(lhs), (lhs, rhs)
    hm = 1e-3 * mu
    g.set_viscosity(mu + hm, substeps)
    fp = _forward(g, sc.x, sc.v, sc.C)
    g.set_viscosity(mu - hm, substeps)
    fm = _forward(g, sc.x, sc.v, sc.C)
    fd = float(y @ ((fp - fm) / (2 * hm)))
    assert abs(fd - mub) <= 1e-5 * abs(fd), (fd, mub)
    g.close()


def test_autograd_viscosity_gradient(wcg):
    torch = pytest.importorskip("torch")
    from libwetcloth_b200.autograd import substep
    sc = _scene("dam16")
    sc.params.viscosity = 0.2
    g = FluidScene(sc)
    mu = torch.tensor(0.2, dtype=torch.float64, requires_grad=True)

    def loss_of(m):
        x1, v1, C1 = substep(g, torch.from_numpy(sc.x), torch.from_numpy(sc.v),
                             torch.from_numpy(sc.C), DT, viscosity=m, viscosity_substeps=2,
                             correction_call=0)
        return (v1 ** 2).sum() + (C1 ** 2).sum() * 1e-4

    L = loss_of(mu)
    L.backward()
    h = 1e-4
    fd = (loss_of(torch.tensor(0.2 + h, dtype=torch.float64)).item() -
          loss_of(torch.tensor(0.2 - h, dtype=torch.float64)).item()) / (2 * h)
    assert abs(fd - mu.grad.item()) <= 1e-4 * abs(fd), (fd, mu.grad.item())
    g.close()


@pytest.mark.parametrize("kind", ["dam16", "curl24"])
def test_adjoint_identity_with_correction(kind, wcg):
    """With correctLiquidParticles on, G2P measures x_n - x_p from the
    corrected positions and the advection starts there; the corrected
    positions depend on x alone, so the sub-step stays affine in (v, C) and
    the identity holds.  The forward differences and the reverse mode use
    the same call of the correction stream."""
    sc = _scene(kind)
    sc.params.correction_strength = 0.2
    sc.params.correction_seed = 5
    n = sc.x.shape[0]
    g = FluidScene(sc)
    dv, dC, y = _directions(n, 17)
    h = 1e-2

    def fwd(v, C):
        return _forward(g, sc.x, v, C, call=3)

    Jd = (fwd(sc.v + h * dv, sc.C + h * dC) - fwd(sc.v - h * dv, sc.C - h * dC)) / (2 * h)
    vb, Cb = _vjp(g, sc, y, call=3)
    lhs = float(y @ Jd)
    rhs = float((vb * dv).sum() + (Cb * dC).sum())
    assert abs(lhs - rhs) <= 1e-9 * abs(lhs), (lhs, rhs)
    # the correction moved particles, so the corrected path was exercised
    x_on = _forward(g, sc.x, sc.v, sc.C, call=3)[12 * n:]
    g0 = FluidScene(_scene(kind))
    x_off = _forward(g0, sc.x, sc.v, sc.C, call=3)[12 * n:]
    assert np.abs(x_on - x_off).max() > 1e-6
    g.close()
    g0.close()


def _interior(sc, margin=3.0):
    """Particles at least `margin` cells from the walls and the free surface."""
    d = margin * sc.params.dx
    x = sc.x
    top = x[:, 1].max()
    return ((x[:, 0] > d) & (x[:, 0] < 1.0 - d) & (x[:, 2] > d) & (x[:, 2] < 1.0 - d) &
            (x[:, 1] > d) & (x[:, 1] < top - d))


@pytest.mark.parametrize("precision,h,tol", [(_capi.WCG_FP64, 1e-6, 1e-6),
                                             (_capi.WCG_FP32_REFINE, 1e-4, 2e-3)])
def test_position_adjoint_identity(precision, h, tol, wcg):
    """<y, J_x d> = <J_x^T y, d> for directions d in the positions of interior
    particles: the x-cotangent through P2G's and G2P's weights and offsets.
    The advection's identity part <y_x, d> is taken out of both sides, so the
    tolerance bounds the weights' part."""
    sc = _scene("curl24")
    n = sc.x.shape[0]
    mask = _interior(sc)
    assert mask.sum() > 1000
    rng = np.random.default_rng(17)
    d = rng.normal(size=(n, 3)) * mask[:, None]
    y = rng.normal(size=15 * n)
    g = FluidScene(sc, precision=precision)
    Jd = (_forward(g, sc.x + h * d, sc.v, sc.C) - _forward(g, sc.x - h * d, sc.v, sc.C)) / (2 * h)
    g.set_state(sc.x, sc.v, sc.C)
    g.set_correction_count(0)
    _, _, xb = g.substep_vjp(DT, y[:3 * n].reshape(n, 3), y[3 * n:12 * n].reshape(n, 9),
                             y[12 * n:].reshape(n, 3))
    ident = float((y[12 * n:].reshape(n, 3) * d).sum())
    lhs = float(y @ Jd) - ident
    rhs = float((xb * d).sum()) - ident
    assert abs(lhs - rhs) <= tol * abs(lhs), (lhs, rhs, ident)
    g.close()


def test_position_adjoint_identity_free_surface(wcg):
    """The same identity for directions carried by particles within two cells
    of the free surface (away from the walls): their positions set the
    liquid phi of the surface cells, hence the ghost-fluid fractions of the
    pressure matrix and of the pressure gradient (k_adj_theta)."""
    sc = _scene("curl24")
    n = sc.x.shape[0]
    dx = sc.params.dx
    x = sc.x
    top = x[:, 1].max()
    mask = ((x[:, 0] > 3 * dx) & (x[:, 0] < 1 - 3 * dx) & (x[:, 2] > 3 * dx) &
            (x[:, 2] < 1 - 3 * dx) & (x[:, 1] > top - 2 * dx))
    assert mask.sum() > 500
    rng = np.random.default_rng(23)
    d = rng.normal(size=(n, 3)) * mask[:, None]
    y = rng.normal(size=15 * n)
    g = FluidScene(sc)
    h = 1e-7
    Jd = (_forward(g, sc.x + h * d, sc.v, sc.C) - _forward(g, sc.x - h * d, sc.v, sc.C)) / (2 * h)
    g.set_state(sc.x, sc.v, sc.C)
    g.set_correction_count(0)
    _, _, xb = g.substep_vjp(DT, y[:3 * n].reshape(n, 3), y[3 * n:12 * n].reshape(n, 9),
                             y[12 * n:].reshape(n, 3))
    ident = float((y[12 * n:].reshape(n, 3) * d).sum())
    lhs = float(y @ Jd) - ident
    rhs = float((xb * d).sum()) - ident
    assert abs(lhs - rhs) <= 1e-5 * abs(lhs), (lhs, rhs, ident)
    g.close()


def test_fixed_position_adjoint_passes_x_bar(wcg):
    sc = _scene("dam16")
    n = sc.x.shape[0]
    y = np.random.default_rng(4).normal(size=15 * n)
    g = FluidScene(sc)
    outs = []
    for diff in (False, True):
        g.set_adjoint_positions(diff)
        g.set_state(sc.x, sc.v, sc.C)
        g.set_correction_count(0)
        outs.append(g.substep_vjp(DT, y[:3 * n].reshape(n, 3), y[3 * n:12 * n].reshape(n, 9),
                                  y[12 * n:].reshape(n, 3)))
    (vb, Cb, xb), (vb2, Cb2, xb2) = outs
    assert np.array_equal(xb.ravel(), y[12 * n:])
    assert np.array_equal(vb, vb2) and np.array_equal(Cb, Cb2)
    assert not np.array_equal(xb2.ravel(), y[12 * n:])
    g.close()


def test_rollout_checkpointing_matches_substep_chain(wcg):
    """A 5-sub-step rollout with a checkpoint every 2 sub-steps gives the
    loss and the gradients of the chain of single sub-step nodes, bit for
    bit (the recomputation repeats the forward exactly)."""
    torch = pytest.importorskip("torch")
    from libwetcloth_b200.autograd import rollout, substep
    sc = _scene("curl24")
    n = sc.x.shape[0]
    rng = np.random.default_rng(8)
    wx = torch.from_numpy(rng.normal(size=(n, 3)))
    target = torch.from_numpy(rng.normal(size=(n, 3)))
    g = FluidScene(sc)
    res = []
    for mode in ("chain", "rollout"):
        x = torch.from_numpy(sc.x.copy()).requires_grad_(True)
        v = torch.from_numpy(sc.v.copy()).requires_grad_(True)
        C = torch.from_numpy(sc.C.copy()).requires_grad_(True)
        if mode == "chain":
            xs, vs, Cs = x, v, C
            for k in range(5):
                xs, vs, Cs = substep(g, xs, vs, Cs, DT, correction_call=k)
        else:
            xs, vs, Cs = rollout(g, x, v, C, DT, 5, checkpoint_every=2, correction_call=0)
        L = ((vs - target) ** 2).sum() + (xs * wx).sum() + 1e-3 * (Cs ** 2).sum()
        L.backward()
        res.append((L.item(), x.grad.numpy().copy(), v.grad.numpy().copy(),
                    C.grad.numpy().copy()))
    (l0, *g0), (l1, *g1) = res
    assert l0 == l1
    for a, b in zip(g0, g1):
        assert np.array_equal(a, b)
    g.close()
