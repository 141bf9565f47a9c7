"""The adjoint at the benchmark's gradient configuration.

96^3 grid (10-cell CPML), dx = 2 nm, a 32 x 32 x 16 design box at the
centre with rho ~ U[0, 1] from the benchmark's seed, FP32 fields, 4000 time
steps with checkpoints every 200, objective = the absorption cross-section
at 550, 633 and 785 nm.  The FP32 adjoint's dL/drho at 16 random design
cells and its dL/d(omega_D, gamma) are checked against central differences
(h = 1e-3, relative for the two Drude parameters) of the FP64 forward
objective, to 1e-3; dL/drho at two of those cells against central
differences of the FP64 oracle's own objective.
"""
import os
import sys

import numpy as np
import pytest

import fdtd_b200 as F
import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
import bench  # noqa: E402  (the benchmark's parameter sets)

pytestmark = pytest.mark.gpu

STEPS = 4000
EVERY = 200
H = 1e-3
TOL = 1e-3
SIGMA_ABS = np.array([1.0, -1.0, 1.0, -1.0, 1.0, -1.0])  # -s_f on ScatAbs columns 10-15


def rho0(p):
    b = list(p.design_box)
    rng = np.random.default_rng(bench.BATCH_SEED)
    return rng.uniform(0, 1, (b[5] - b[4], b[3] - b[2], b[1] - b[0])).astype(np.float32)


def cells(shape, n=16):
    rng = np.random.default_rng(11)
    out = set()
    while len(out) < n:
        out.add(tuple(int(rng.integers(0, e)) for e in shape))
    return sorted(out)


@pytest.fixture(scope="module")
def fp32_gradient():
    p = bench.adjoint_params(F, STEPS, precision=F.FDTD_FP32)
    s = F.Sim(p)
    rho = rho0(p)
    s.set_design(rho)
    L = s.forward(bench.ADJOINT_FREQS, EVERY)
    g, gp = s.backward()
    s.close()
    return p, rho, L, g, gp


@pytest.fixture(scope="module")
def fp64_sim():
    p = bench.adjoint_params(F, STEPS, precision=F.FDTD_FP64)
    s = F.Sim(p)
    yield p, s
    s.close()


def test_objective_is_positive_and_matches_fp64(fp32_gradient, fp64_sim):
    _, rho, L32, _, _ = fp32_gradient
    _, s = fp64_sim
    s.set_design(rho)
    L64 = s.forward(bench.ADJOINT_FREQS, EVERY)
    print("objective fp32", L32, "fp64", L64)
    assert L64 > 0
    assert abs(L32 - L64) <= 1e-4 * abs(L64)


def test_rho_gradient_at_16_cells(fp32_gradient, fp64_sim):
    _, rho, _, g, _ = fp32_gradient
    _, s = fp64_sim
    pts = cells(rho.shape)
    fds = []
    for c in pts:
        vals = []
        for d in (H, -H):
            r = rho.copy()
            r[c] += d
            s.set_design(r)
            vals.append(s.forward(bench.ADJOINT_FREQS, EVERY))
        fds.append((vals[0] - vals[1]) / (2 * H))
    fds = np.array(fds)
    adj = np.array([g[c] for c in pts], dtype=np.float64)
    err = np.abs(adj - fds) / np.abs(fds)
    for c, a, f, e in zip(pts, adj, fds, err):
        print(c, "adjoint %.6e fd %.6e rel %.2e" % (a, f, e))
    assert np.all(err <= TOL), err


@pytest.mark.parametrize("k,name", [(0, "omega_D"), (1, "gamma_D")])
def test_drude_parameter_gradient(fp32_gradient, k, name):
    p, rho, _, _, gp = fp32_gradient
    q = bench.adjoint_params(F, STEPS, precision=F.FDTD_FP64)
    # the metal's own parameters (gold, setup.cu:1191-1203) made explicit
    gold = dict(metal_custom=1, eps_inf=1.1431, omega_D=1.3202e16, gamma_D=1.0805e14,
                cp_A=(0.26698, 3.0834), cp_phi=(-1.2371, -1.0968),
                cp_Omega=(3.8711e15, 4.1684e15), cp_Gamma=(4.4642e14, 2.3555e15))
    q.update(**gold)
    v = gold[name]
    vals = []
    for x in (v * (1 + H), v * (1 - H)):
        setattr(q, name, x)
        s = F.Sim(q)
        s.set_design(rho)
        vals.append(s.forward(bench.ADJOINT_FREQS, EVERY))
        s.close()
    fd = (vals[0] - vals[1]) / (2 * H * v)
    print(name, "adjoint %.6e fd %.6e" % (gp[k], fd))
    assert abs(gp[k] - fd) <= TOL * abs(fd)


def test_rho_gradient_against_the_oracle(fp32_gradient):
    """Central differences of the FP64 oracle's objective (the CPU
    restatement with the same design blend; its DFT accumulates the three
    objective frequencies only) at two of the 16 cells."""
    p, rho, L, g, _ = fp32_gradient

    def oracle_objective(r):
        o = O.OracleSim(bench.adjoint_params(O, STEPS, precision=1))
        o.set_dft_freqs(bench.ADJOINT_FREQS)
        o.set_design(r)
        o.step(STEPS)
        table = o.spectra()
        return float(np.sum(table[bench.ADJOINT_FREQS][:, 10:16] @ SIGMA_ABS))

    for c in cells(rho.shape)[:2]:
        vals = []
        for d in (H, -H):
            r = rho.copy()
            r[c] += d
            vals.append(oracle_objective(r))
        fd = (vals[0] - vals[1]) / (2 * H)
        print(c, "oracle fd %.6e adjoint %.6e" % (fd, g[c]))
        assert abs(0.5 * (vals[0] + vals[1]) - L) <= 1e-4 * abs(L)
        assert abs(g[c] - fd) <= TOL * abs(fd)
