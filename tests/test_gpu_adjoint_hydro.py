"""The adjoint of the hydrodynamic (nonlocal) model.

A 34^3 gold sphere with the hydrodynamic current (the "hydro" case) and a
6 x 6 x 6 design box over part of the sphere: the box's cells blend between
vacuum and the hydrodynamic metal (current and density updates scaled by
rho, coupling coefficients blended), the rest of the sphere is metal.  The
transposed hydrodynamic step (three phases and the current update,
linearised about the recorded trajectory) is checked against central
differences of the FP64 forward objective, on rho (h = 1e-3) and on gamma
(omega_D does not enter the hydrodynamic model: its gradient is zero), and
against central differences of the FP64 oracle's objective.
"""
import numpy as np
import pytest

import fdtd_b200 as F
import oracle as O
from cases import make

pytestmark = pytest.mark.gpu

BOX = [14, 20, 14, 20, 14, 20]
SEL = [2, 4, 6]
STEPS = 300
SIGMA_ABS = np.array([1.0, -1.0, 1.0, -1.0, 1.0, -1.0])
GOLD = dict(metal_custom=1, eps_inf=1.1431, omega_D=1.3202e16, gamma_D=1.0805e14,
            cp_A=(0.26698, 3.0834), cp_phi=(-1.2371, -1.0968),
            cp_Omega=(3.8711e15, 4.1684e15), cp_Gamma=(4.4642e14, 2.3555e15))
CELLS = [(0, 0, 0), (2, 3, 1), (5, 5, 5), (3, 1, 4)]


def params(mod, prec, **over):
    kw = dict(GOLD, precision=prec, Tend=STEPS - 1, design_box=BOX)
    kw.update(over)
    return make(mod, "hydro", **kw)


def rho0():
    rng = np.random.default_rng(5)
    return rng.uniform(0, 1, (BOX[5] - BOX[4], BOX[3] - BOX[2], BOX[1] - BOX[0])).astype(np.float32)


def objective(sim, rho):
    sim.set_design(rho)
    return sim.forward(SEL, 50)


@pytest.fixture(scope="module")
def fp64_grad():
    s = F.Sim(params(F, F.FDTD_FP64))
    assert s.dims.hydro == 1
    L = objective(s, rho0())
    g, gp = s.backward()
    return s, L, g, gp


def test_design_blend_forward_matches_oracle():
    """The hydrodynamic design blend itself (a new model, in the product and
    the oracle alike): fields after 200 steps within 1e-11."""
    s = F.Sim(params(F, F.FDTD_FP64))
    s.set_design(rho0())
    s.step(200)
    o = O.OracleSim(params(O, 1))
    o.set_design(rho0())
    o.step(200)
    for fam in ((0, 1, 2), (3, 4, 5)):
        ref = [o.field(c) for c in fam]
        scale = max(np.abs(x).max() for x in ref)
        for c, b in zip(fam, ref):
            assert np.abs(s.field(c) - b).max() <= 1e-11 * scale, c
    s.close()


def test_rho_gradient_matches_central_differences(fp64_grad):
    s, L, g, _ = fp64_grad
    assert L > 0
    rho, h = rho0(), 1e-3
    for c in CELLS:
        r = rho.copy(); r[c] += h; lp = objective(s, r)
        r = rho.copy(); r[c] -= h; lm = objective(s, r)
        fd = (lp - lm) / (2 * h)
        print(c, "fd", fd, "adjoint", g[c])
        assert abs(fd - g[c]) <= 1e-3 * abs(fd), (c, fd, g[c])


def test_gamma_gradient_matches_central_differences(fp64_grad):
    _, L, _, gp = fp64_grad
    v = GOLD["gamma_D"]
    vals = []
    for x in (v * (1 + 1e-4), v * (1 - 1e-4)):
        s = F.Sim(params(F, F.FDTD_FP64, gamma_D=x))
        vals.append(objective(s, rho0()))
        s.close()
    fd = (vals[0] - vals[1]) / (2e-4 * v)
    print("gamma fd", fd, "adjoint", gp[1])
    assert abs(fd - gp[1]) <= 1e-3 * abs(fd)


def test_omega_d_does_not_enter_the_hydrodynamic_model(fp64_grad):
    _, L, _, gp = fp64_grad
    s = F.Sim(params(F, F.FDTD_FP64, omega_D=GOLD["omega_D"] * 1.01))
    assert objective(s, rho0()) == L
    assert gp[0] == 0.0
    s.close()


def test_fp32_adjoint_agrees_with_fp64(fp64_grad):
    _, L64, g64, gp64 = fp64_grad
    s = F.Sim(params(F, F.FDTD_FP32))
    L = objective(s, rho0())
    g, gp = s.backward()
    assert abs(L - L64) <= 1e-4 * abs(L64)
    assert np.abs(g - g64).max() <= 1e-3 * np.abs(g64).max()
    assert abs(gp[1] - gp64[1]) <= 1e-3 * abs(gp64[1])
    s.close()


def test_cube_root_fix_gradient():
    """With FDTD_FIX_HYDRO_CBRT the cube root (N_EQ + N)^(1/3) is taken in
    FP64 and its derivative enters the transposed current update."""
    s = F.Sim(params(F, F.FDTD_FP64, fixes=F.FIX_HYDRO_CBRT))
    rho = rho0()
    objective(s, rho)
    g, _ = s.backward()
    h = 1e-3
    for c in CELLS[:2]:
        r = rho.copy(); r[c] += h; lp = objective(s, r)
        r = rho.copy(); r[c] -= h; lm = objective(s, r)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[c]) <= 1e-3 * abs(fd), (c, fd, g[c])
    s.close()


def test_general_objective(fp64_grad):
    """A weighted sum of ScatAbs columns through fdtd_backward_spectra."""
    s = fp64_grad[0]
    nf = s.dims.num_freq

    def L_of(table):
        return 1.5 * table[2, 1] - 0.7 * table[4, 3] + table[6, 13]

    G = np.zeros((nf, 19))
    G[2, 1], G[4, 3], G[6, 13] = 1.5, -0.7, 1.0
    rho = rho0()
    s.set_design(rho)
    s.forward_spectra(50)
    g, _ = s.backward_spectra(G)
    h = 1e-3
    c = CELLS[2]
    vals = []
    for d in (h, -h):
        r = rho.copy(); r[c] += d; s.set_design(r)
        vals.append(L_of(s.forward_spectra(50)))
    fd = (vals[0] - vals[1]) / (2 * h)
    assert abs(fd - g[c]) <= 1e-3 * abs(fd), (fd, g[c])


def test_rho_gradient_against_the_oracle(fp64_grad):
    _, L, g, _ = fp64_grad

    def oracle_objective(r):
        o = O.OracleSim(params(O, 1))
        o.set_design(r)
        o.step(STEPS)
        return float(np.sum(o.spectra()[SEL][:, 10:16] @ SIGMA_ABS))

    rho, h = rho0(), 1e-3
    for c in CELLS[:2]:
        r = rho.copy(); r[c] += h; lp = oracle_objective(r)
        r = rho.copy(); r[c] -= h; lm = oracle_objective(r)
        fd = (lp - lm) / (2 * h)
        print(c, "oracle fd", fd, "adjoint", g[c])
        assert abs(0.5 * (lp + lm) - L) <= 1e-8 * abs(L)
        assert abs(fd - g[c]) <= 1e-3 * abs(fd)
