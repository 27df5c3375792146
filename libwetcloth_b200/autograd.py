"""torch.autograd binding of the liquid sub-step (the C-ABI's wcg_substep and
wcg_substep_vjp); the arithmetic is all in libwcgpu.so.

``substep(scene, x, v, C, dt, viscosity)`` returns (x', v', C') as float64
tensors and records a node whose backward restores the checkpoint (x, v, C)
in the scene, recomputes the forward grid there and runs the reverse-mode
kernels; an optional 0-d ``viscosity`` tensor gets its gradient too.  The
gradient in x follows the positions through the transfer weights (P2G, G2P
and the advection), the liquid phi behind the ghost-fluid fractions and the
solid projection of the particle correction; the grid's discrete structure
(activation, DOFs, valid faces) is held at the checkpoint's values.  The
scene's particle state after backward is the checkpoint of the last node
differentiated.

``rollout(scene, x, v, C, dt, steps, viscosity, checkpoint_every)`` runs
``steps`` sub-steps as one node that keeps only every ``checkpoint_every``-th
state (on the host); its backward recomputes each segment of sub-steps from
its checkpoint and runs the sub-steps' reverse modes in reverse order, so the
memory held is one segment of states, not the whole trajectory.

The particle correction of a sub-step (run in every sub-step; at strength 0
it only projects its subset out of the solid) takes the subset of one call of
the scene's seeded stream: ``correction_call`` fixes that call (the default,
None, takes the scene's next call); sub-step k of a rollout takes call
``correction_call + k``, and the backward replays the same calls.
"""
from __future__ import annotations

import numpy as np
import torch


def _host(t):
    return t.detach().cpu().numpy().astype(np.float64)


class _Substep(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, v, C, mu, scene, dt, substeps, call):
        xs, vs, Cs = (_host(t) for t in (x, v, C))
        m = float(mu.detach().cpu().item()) if mu is not None else None
        if m is not None:
            scene.set_viscosity(m, substeps)
        scene.set_state(xs, vs, Cs)
        k = scene.correction_count if call is None else int(call)
        scene.set_correction_count(k)
        scene.substep(dt)
        ctx.call = k
        x1, v1, C1 = scene.download()
        ctx.scene = scene
        ctx.dt = dt
        ctx.mu = (m, substeps)
        ctx.state = (xs, vs, Cs)
        dev = v.device
        return (torch.from_numpy(x1).to(dev), torch.from_numpy(v1).to(dev),
                torch.from_numpy(C1).to(dev))

    @staticmethod
    def backward(ctx, gx1, gv1, gC1):
        n = ctx.state[0].shape[0]
        dev = gv1.device if gv1 is not None else gx1.device

        def host(g, k):
            return np.zeros((n, k)) if g is None else _host(g)

        scene = ctx.scene
        m, substeps = ctx.mu
        if m is not None:
            scene.set_viscosity(m, substeps)
        scene.set_state(*ctx.state)
        scene.set_correction_count(ctx.call)
        vb, Cb, xb, mub = scene.substep_vjp(ctx.dt, host(gv1, 3), host(gC1, 9), host(gx1, 3),
                                            with_viscosity=True)
        gmu = None if m is None else torch.tensor(mub, dtype=torch.float64, device=dev)
        return (torch.from_numpy(xb).to(dev), torch.from_numpy(vb).to(dev),
                torch.from_numpy(Cb).to(dev), gmu, None, None, None, None)


def substep(scene, x, v, C, dt: float, viscosity=None, viscosity_substeps: int = 1,
            correction_call=None):
    """One differentiable sub-step of a FluidScene (liquid).  viscosity: an
    optional 0-d tensor (LiquidInfo::viscosity) that receives a gradient;
    correction_call: the call of the seeded correction stream the sub-step
    takes (None: the scene's next)."""
    return _Substep.apply(x, v, C, viscosity, scene, dt, viscosity_substeps, correction_call)


class _Rollout(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, v, C, mu, scene, dt, steps, every, substeps, call):
        m = float(mu.detach().cpu().item()) if mu is not None else None
        if m is not None:
            scene.set_viscosity(m, substeps)
        k0 = scene.correction_count if call is None else int(call)
        state = (_host(x), _host(v), _host(C))
        ckpts = []
        scene.set_state(*state)
        for k in range(steps):
            if k % every == 0:
                ckpts.append(state if k == 0 else scene.download())
            scene.set_correction_count(k0 + k)
            scene.substep(dt)
        x1, v1, C1 = scene.download()
        ctx.scene, ctx.dt, ctx.steps, ctx.every = scene, dt, steps, every
        ctx.mu = (m, substeps)
        ctx.k0 = k0
        ctx.ckpts = ckpts
        dev = v.device
        return (torch.from_numpy(x1).to(dev), torch.from_numpy(v1).to(dev),
                torch.from_numpy(C1).to(dev))

    @staticmethod
    def backward(ctx, gx1, gv1, gC1):
        scene, dt, steps, every = ctx.scene, ctx.dt, ctx.steps, ctx.every
        m, substeps = ctx.mu
        n = ctx.ckpts[0][0].shape[0]
        dev = gv1.device if gv1 is not None else gx1.device

        def host(g, k):
            return np.zeros((n, k)) if g is None else _host(g)

        xb, vb, Cb = host(gx1, 3), host(gv1, 3), host(gC1, 9)
        mub = 0.0
        if m is not None:
            scene.set_viscosity(m, substeps)
        for seg in range(len(ctx.ckpts) - 1, -1, -1):
            k_lo = seg * every
            k_hi = min(steps, k_lo + every)
            # recompute the segment's sub-step inputs from its checkpoint
            states = [ctx.ckpts[seg]]
            scene.set_state(*states[0])
            for k in range(k_lo, k_hi - 1):
                scene.set_correction_count(ctx.k0 + k)
                scene.substep(dt)
                states.append(scene.download())
            for k in range(k_hi - 1, k_lo - 1, -1):
                scene.set_state(*states[k - k_lo])
                scene.set_correction_count(ctx.k0 + k)
                vb, Cb, xb, mk = scene.substep_vjp(dt, vb, Cb, xb, with_viscosity=True)
                mub += mk
        gmu = None if m is None else torch.tensor(mub, dtype=torch.float64, device=dev)
        return (torch.from_numpy(xb).to(dev), torch.from_numpy(vb).to(dev),
                torch.from_numpy(Cb).to(dev), gmu, None, None, None, None, None, None)


def rollout(scene, x, v, C, dt: float, steps: int, viscosity=None, viscosity_substeps: int = 1,
            checkpoint_every: int = 10, correction_call=None):
    """`steps` differentiable sub-steps of a FluidScene (liquid) as one node
    with a checkpoint every `checkpoint_every` sub-steps (recomputed in the
    backward).  Arguments as substep's; returns the final (x, v, C)."""
    if steps < 1 or checkpoint_every < 1:
        raise ValueError("steps and checkpoint_every must be positive")
    return _Rollout.apply(x, v, C, viscosity, scene, dt, int(steps), int(checkpoint_every),
                          viscosity_substeps, correction_call)
