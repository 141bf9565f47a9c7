"""torch.autograd.Function over the adjoint's forward / backward pair.

A thin wrapper for gradient harnesses (torch.autograd.grad, gradcheck-style
comparisons): the forward calls fdtd_set_design + fdtd_forward, the backward
calls fdtd_backward and scales dL/drho by the incoming gradient.  The
simulation object is any handle with the Sim adjoint methods (set_design,
forward, backward); it keeps the checkpoints between the two calls, so one
forward is followed by at most one backward.
"""
import numpy as np
import torch


class AbsorbedPower(torch.autograd.Function):
    """L = sum over freq_idx of the AbsTot column, as a function of the
    design-box blend rho (shape (nz, ny, nx) of the box).  The Drude
    parameter gradient of the last backward is left on the simulation
    object as `last_param_grad` (d/d omega_D, d/d gamma)."""

    @staticmethod
    def forward(ctx, rho, sim, freq_idx, checkpoint_every=200):
        r = rho.detach().to("cpu", torch.float32).numpy()
        sim.set_design(r)
        L = sim.forward(list(freq_idx), int(checkpoint_every))
        ctx.sim = sim
        ctx.rho_dtype = rho.dtype
        ctx.rho_device = rho.device
        return torch.tensor(L, dtype=torch.float64, device=rho.device)

    @staticmethod
    def backward(ctx, grad_out):
        g, gp = ctx.sim.backward()
        ctx.sim.last_param_grad = np.asarray(gp, dtype=np.float64)
        grad = torch.from_numpy(np.ascontiguousarray(g)).to(ctx.rho_device, torch.float64)
        grad = (grad * grad_out.to(torch.float64)).to(ctx.rho_dtype)
        return grad, None, None, None


def absorbed_power(rho, sim, freq_idx, checkpoint_every=200):
    """Functional form of AbsorbedPower.apply."""
    return AbsorbedPower.apply(rho, sim, freq_idx, checkpoint_every)
