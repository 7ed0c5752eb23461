"""PyTorch autograd wrapper of the linear-leapfrog forward model and its
hand-written discrete adjoint (swals_gpu_adjoint_linear).

    stage_series = GaugeWaveforms.apply(eta0_window, domain, U_base, window, nsteps, dt)

maps a window of the initial free surface to the stage time series at the
domain's gauges (shape (nsteps, n_gauges)); backward runs the adjoint sweep
on the GPU.  The forward and adjoint run in libswalsgpu.so; torch only
carries the tensors.
"""
from __future__ import annotations

import numpy as np
import torch


class GaugeWaveforms(torch.autograd.Function):
    @staticmethod
    def forward(ctx, eta0, domain, U_base, window, nsteps, dt):
        U = np.array(U_base, dtype=domain.dtype, copy=True)
        U[0][window] = eta0.detach().to("cpu", torch.float64).numpy()
        domain.set_U(U)
        domain.gauges_reset()
        domain.evolve_steps(int(nsteps), float(dt))
        series = domain.gauges_read()[:, :, 0]
        ctx.domain, ctx.window, ctx.nsteps, ctx.dt = domain, window, int(nsteps), float(dt)
        ctx.like = eta0
        return torch.as_tensor(np.ascontiguousarray(series), dtype=eta0.dtype, device=eta0.device)

    @staticmethod
    def backward(ctx, grad_series):
        g = grad_series.detach().to("cpu", torch.float64).numpy()
        grad = ctx.domain.adjoint_linear(ctx.nsteps, ctx.dt, gauge_adjoint=g)
        gw = torch.as_tensor(np.ascontiguousarray(grad[0][ctx.window]), dtype=ctx.like.dtype,
                             device=ctx.like.device)
        return gw, None, None, None, None, None
