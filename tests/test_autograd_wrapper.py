"""The torch.autograd.Function over the adjoint pair (fdtd_b200.autograd),
checked on the CPU with a stand-in simulation whose objective is a known
quadratic: the wrapper must pass rho through, return L, and hand back the
simulation's gradient scaled by the incoming gradient."""
import numpy as np
import torch

from fdtd_b200.autograd import AbsorbedPower, absorbed_power


class QuadraticSim:
    """L = sum(w * rho^2) with the Sim adjoint interface."""

    def __init__(self, w):
        self.w = w
        self.calls = []

    def set_design(self, rho):
        assert rho.dtype == np.float32
        self.rho = rho.copy()
        self.calls.append("set_design")

    def forward(self, freq_idx, every):
        self.calls.append(("forward", tuple(freq_idx), every))
        return float(np.sum(self.w * self.rho.astype(np.float64) ** 2))

    def backward(self):
        self.calls.append("backward")
        return (2 * self.w * self.rho).astype(np.float32), np.array([1.5, -2.5])


def test_forward_backward_plumbing():
    rng = np.random.default_rng(0)
    w = rng.uniform(0.5, 2.0, (2, 3, 4))
    sim = QuadraticSim(w)
    rho = torch.tensor(rng.uniform(0, 1, (2, 3, 4)), dtype=torch.float32, requires_grad=True)
    L = absorbed_power(rho, sim, [0, 2], 50)
    assert L.dtype == torch.float64
    np.testing.assert_allclose(L.item(), np.sum(w * rho.detach().numpy().astype(np.float64) ** 2), rtol=1e-6)
    (3.0 * L).backward()
    np.testing.assert_allclose(rho.grad.numpy(), 3.0 * 2 * w * rho.detach().numpy(), rtol=1e-6)
    assert sim.calls == ["set_design", ("forward", (0, 2), 50), "backward"]
    np.testing.assert_array_equal(sim.last_param_grad, [1.5, -2.5])


def test_matches_torch_autograd_of_the_same_objective():
    rng = np.random.default_rng(1)
    w = rng.uniform(0.5, 2.0, (3, 2, 2))
    rho = torch.tensor(rng.uniform(0, 1, (3, 2, 2)), dtype=torch.float64, requires_grad=True)
    (g_wrap,) = torch.autograd.grad(AbsorbedPower.apply(rho, QuadraticSim(w), [1], 10), rho)
    (g_ref,) = torch.autograd.grad((torch.from_numpy(w) * rho ** 2).sum(), rho)
    np.testing.assert_allclose(g_wrap.numpy(), g_ref.numpy(), rtol=1e-6)
