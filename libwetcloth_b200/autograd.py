"""torch.autograd binding of one liquid sub-step (the C-ABI's wcg_substep and
wcg_substep_vjp); the arithmetic is all in libwcgpu.so.

``substep(scene, x, v, C, dt, viscosity)`` returns (x', v', C') as float64
tensors and records a node whose backward restores the checkpoint (x, v, C)
in the scene, recomputes the forward grid there and runs the reverse-mode
kernels; an optional 0-d ``viscosity`` tensor gets its gradient too.  The
positions are held fixed in the derivative: d(x')/d(x) is the identity and the
weights' dependence on x is not differentiated, so gradients through several
chained sub-steps omit that term.  The scene's particle state after backward is
the checkpoint of the last node differentiated.

The particle correction of the sub-step (run in every sub-step; at strength 0
it only projects its subset out of the solid) takes the subset of one call of
the scene's seeded stream: ``correction_call`` fixes that call (the default,
None, takes the scene's next call); the backward replays the same call.
"""
from __future__ import annotations

import numpy as np
import torch


class _Substep(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, v, C, mu, scene, dt, substeps, call):
        xs, vs, Cs = (t.detach().cpu().numpy().astype(np.float64) for t in (x, v, C))
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
            return np.zeros((n, k)) if g is None else g.detach().cpu().numpy().astype(np.float64)

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
