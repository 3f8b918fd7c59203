"""torch autograd over the render's adjoint (spk_render_vjp), for the ctypes test layer.

RenderLinear.apply(image, params, engine, delta, strength, film_seed) returns the scanned linear RGB of
`image` (H x W x 3 float32 on the CPU): the render up to the scanner's lens blur and unsharp mask, with
the grain held as fixed noise (the counts of film_seed). params (float64) are
  [print_exposure, m_filter_shift, y_filter_shift, halation weight 0..K-1, halation sigma 0..K-1],
the K halation components each one weight and one sigma (pixels) for the three channels, mixed with the
per-channel strength `strength`. The backward pass calls spk_render_vjp on the session the forward pass
opened (blurs recomputed, not stored) and returns the gradients of the image and of params.
"""

from __future__ import annotations

import numpy as np
import torch


class RenderLinear(torch.autograd.Function):
    @staticmethod
    def forward(ctx, image, params, engine, delta, strength, film_seed):
        p = params.detach().cpu().numpy().astype(np.float64)
        k = (len(p) - 3) // 2
        d = dict(delta, print_exposure=float(p[0]), m_filter_shift=float(p[1]), y_filter_shift=float(p[2]))
        s = engine.open(image.detach().cpu().numpy().astype(np.float32), d)
        try:
            if k:
                comps = [((float(wt),) * 3, (float(sg),) * 3) for wt, sg in zip(p[3:3 + k], p[3 + k:3 + 2 * k])]
                s.set_halation(comps, strength)
            y = s.render_linear(film_seed)
        except Exception:
            s.close()
            raise
        ctx.session = s
        ctx.film_seed = film_seed
        ctx.n_params = len(p)
        return torch.from_numpy(y)

    @staticmethod
    def backward(ctx, grad_y):
        s = ctx.session
        try:
            gx, gp = s.render_vjp(grad_y.detach().cpu().numpy().astype(np.float32), ctx.film_seed, ctx.n_params)
        finally:
            s.close()
        return torch.from_numpy(gx), torch.from_numpy(gp.copy()), None, None, None, None


def render_linear(image, params, engine, delta, strength=(0.03, 0.03, 0.03), film_seed=0x4ABEA221):
    return RenderLinear.apply(image, params, engine, delta, strength, film_seed)
