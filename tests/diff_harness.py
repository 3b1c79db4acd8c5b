"""torch.autograd wrapper of liblrt's renderer and path-replay adjoint, for the tests only.

render(values) -> the batch image of `jobs` with the material parameters at `values`; its backward
runs lrt_render_adjoint on the incoming image gradient over `adjoint_jobs`, the same jobs with other
samples, so that the adjoint's samples are independent of the primal's (the gradient of a nonlinear
loss then carries no correlation bias).
"""
import numpy as np
import torch


class RenderFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, values, dm, jobs, adjoint_jobs, max_depth, rr_depth):
        dm.set_values(values.detach().cpu().numpy())
        img = dm.ctx.render_batch(jobs, max_depth, rr_depth)
        ctx.dm, ctx.adjoint_jobs, ctx.max_depth, ctx.rr_depth = dm, adjoint_jobs, max_depth, rr_depth
        return torch.from_numpy(img.astype(np.float64))

    @staticmethod
    def backward(ctx, grad_img):
        g = ctx.dm.adjoint(ctx.adjoint_jobs, ctx.max_depth, ctx.rr_depth, grad_img.detach().cpu().numpy())
        return torch.from_numpy(g), None, None, None, None, None


def render(values, dm, jobs, adjoint_jobs, max_depth, rr_depth):
    return RenderFunction.apply(values, dm, jobs, adjoint_jobs, max_depth, rr_depth)
