"""torch.autograd.Function wrappers over the adjoint's forward / backward pairs.

Thin wrappers for gradient harnesses (torch.autograd.grad, gradcheck-style
comparisons).  The simulation object is any handle with the Sim adjoint
methods; it keeps the checkpoints between the two calls, so one forward is
followed by at most one backward.

* AbsorbedPower: rho -> sum over chosen frequencies of the absorption
  cross-section (fdtd_forward / fdtd_backward).
* ScatAbsSpectra: rho -> the whole NUM_freq x 19 ScatAbs table
  (fdtd_forward_spectra / fdtd_backward_spectra), so that any objective
  built from the spectra with torch operations gets its dL/drho from one
  reverse sweep.
"""
import numpy as np
import torch


class AbsorbedPower(torch.autograd.Function):
    """L = sum over freq_idx of the absorption cross-section sigma_abs (m^2,
    positive for an absorbing structure) as a function of the design-box
    blend rho (shape (nz, ny, nx) of the box).  The Drude parameter
    gradient of the last backward is left on the simulation object as
    `last_param_grad` (d/d omega_D, d/d gamma)."""

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


class ScatAbsSpectra(torch.autograd.Function):
    """The ScatAbs table (NUM_freq x 19, float64) as a function of rho.  The
    backward hands the incoming gradient of the table to the simulation's
    backward_spectra; the wavelength and incident-field columns (0, 16-18)
    do not depend on rho and their incoming gradient is dropped.  The
    Drude parameter gradient is left as `last_param_grad`."""

    @staticmethod
    def forward(ctx, rho, sim, checkpoint_every=200):
        r = rho.detach().to("cpu", torch.float32).numpy()
        sim.set_design(r)
        table = sim.forward_spectra(int(checkpoint_every))
        ctx.sim = sim
        ctx.rho_dtype = rho.dtype
        ctx.rho_device = rho.device
        return torch.from_numpy(np.ascontiguousarray(table)).to(rho.device, torch.float64)

    @staticmethod
    def backward(ctx, grad_out):
        G = grad_out.detach().to("cpu", torch.float64).numpy().copy()
        G[:, 0] = 0.0
        G[:, 16:] = 0.0
        g, gp = ctx.sim.backward_spectra(G)
        ctx.sim.last_param_grad = np.asarray(gp, dtype=np.float64)
        grad = torch.from_numpy(np.ascontiguousarray(g)).to(ctx.rho_device, ctx.rho_dtype)
        return grad, None, None


def scatabs_spectra(rho, sim, checkpoint_every=200):
    """Functional form of ScatAbsSpectra.apply."""
    return ScatAbsSpectra.apply(rho, sim, checkpoint_every)
