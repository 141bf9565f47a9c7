"""Reverse-time adjoint (fdtd_set_design / fdtd_forward / fdtd_backward and
the general fdtd_forward_spectra / fdtd_backward_spectra): gradients of the
absorption cross-section at three frequencies, and of weighted sums of the
ScatAbs table, with respect to the per-cell blend rho of a design box and
to the Drude omega_D and gamma, checked against central finite differences
of the forward objective."""
import numpy as np
import pytest

import fdtd_b200 as F
import oracle as O
from cases import make

pytestmark = pytest.mark.gpu

BOX = [14, 20, 14, 20, 15, 19]  # inside the absorption box of the 34^3 grid
SEL = [2, 4, 6]
GOLD = dict(metal_custom=1, eps_inf=1.1431, omega_D=1.3202e16, gamma_D=1.0805e14,
            cp_A=(0.26698, 3.0834), cp_phi=(-1.2371, -1.0968),
            cp_Omega=(3.8711e15, 4.1684e15), cp_Gamma=(4.4642e14, 2.3555e15))


# absorption cross-section from the ScatAbs face columns 10-15: the net
# inward flux, -sum_f s_f q_abs,f with s_f = -1, +1 on the -, + faces
SIGMA_ABS = np.array([1.0, -1.0, 1.0, -1.0, 1.0, -1.0])


def sigma_abs(table, sel):
    return float(np.sum(table[sel][:, 10:16] @ SIGMA_ABS))


def design_sim(prec, **over):
    return F.Sim(make(F, "vacuum", precision=prec, Tend=300, design_box=BOX, **over))


def rho0():
    rng = np.random.default_rng(1)
    return rng.uniform(0, 1, (BOX[5] - BOX[4], BOX[3] - BOX[2], BOX[1] - BOX[0])).astype(np.float32)


@pytest.fixture(scope="module")
def fp64_grad():
    s = design_sim(F.FDTD_FP64, **GOLD)
    s.set_design(rho0())
    L = s.forward(SEL, 50)
    g, gp = s.backward()
    return s, L, g, gp


def test_rho_gradient_matches_central_differences(fp64_grad):
    s, L, g, _ = fp64_grad
    rho, h = rho0(), 1e-3
    for c in [(0, 0, 0), (2, 3, 1), (3, 5, 5), (1, 2, 4)]:
        r = rho.copy(); r[c] += h; s.set_design(r); lp = s.forward(SEL, 50)
        r = rho.copy(); r[c] -= h; s.set_design(r); lm = s.forward(SEL, 50)
        fd = (lp - lm) / (2 * h)
        print(c, "fd", fd, "adjoint", g[c])
        assert abs(fd - g[c]) <= 1e-3 * abs(fd), (c, fd, g[c])


@pytest.mark.parametrize("k,name", [(0, "omega_D"), (1, "gamma_D")])
def test_drude_parameter_gradient_matches_central_differences(fp64_grad, k, name):
    _, L, _, gp = fp64_grad
    v = GOLD[name]
    h = v * 1e-4
    vals = []
    for x in (v + h, v - h):
        s = design_sim(F.FDTD_FP64, **dict(GOLD, **{name: x}))
        s.set_design(rho0())
        vals.append(s.forward(SEL, 50))
        s.close()
    fd = (vals[0] - vals[1]) / (2 * h)
    print(name, "fd", fd, "adjoint", gp[k])
    assert abs(fd - gp[k]) <= 1e-3 * abs(fd)


def test_fp32_adjoint_agrees_with_fp64(fp64_grad):
    _, L64, g64, gp64 = fp64_grad
    s = design_sim(F.FDTD_FP32, **GOLD)
    s.set_design(rho0())
    L = s.forward(SEL, 50)
    g, gp = s.backward()
    assert abs(L - L64) <= 1e-4 * abs(L64)
    assert np.abs(g - g64).max() <= 1e-3 * np.abs(g64).max()
    assert np.all(np.abs(gp - gp64) <= 1e-3 * np.abs(gp64))


@pytest.mark.parametrize("prec", [F.FDTD_FP32, F.FDTD_FP64])
def test_fused_gathers_match_coefficient_arrays(prec, monkeypatch):
    """The fused transposed sub-steps (coefficients computed on the fly away
    from the CPML slabs and the dispersive cells) and the coefficient-array
    form do the same arithmetic in the same order.  The gradients agree to
    rounding only: the objective's source adds to the corner cells shared by
    two flux faces with atomics, whose order varies from run to run."""
    out = []
    for mode in ("1", "0"):
        monkeypatch.setenv("FDTD_ADJ_FUSED", mode)
        s = design_sim(prec, **GOLD)
        s.set_design(rho0())
        L = s.forward(SEL, 50)
        g, gp = s.backward()
        out.append((L, g, gp))
        s.close()
    assert out[0][0] == out[1][0]
    tol = 1e-12 if prec == F.FDTD_FP64 else 1e-5
    g0, g1 = out[0][1], out[1][1]
    assert np.abs(g0 - g1).max() <= tol * np.abs(g1).max()
    np.testing.assert_allclose(out[0][2], out[1][2], rtol=tol)


def test_fused_gathers_plain_blocks_match_coefficient_arrays(monkeypatch):
    """On a 97 x 89 x 93 grid the fused gathers take their flag-free path
    in the blocks clear of the CPML slabs and the material box (the 34^3
    grids above have none); it must agree with the coefficient arrays too."""
    box = [40, 48, 40, 48, 44, 48]
    out = []
    for mode in ("1", "0"):
        monkeypatch.setenv("FDTD_ADJ_FUSED", mode)
        s = F.Sim(make(F, "sphere_big", precision=F.FDTD_FP64, nano_sphere=0, Tend=420,
                       design_box=box, **GOLD))
        rng = np.random.default_rng(3)
        s.set_design(rng.uniform(0, 1, (box[5] - box[4], box[3] - box[2], box[1] - box[0])).astype(np.float32))
        L = s.forward(SEL, 40)
        g, gp = s.backward()
        out.append((L, g, gp))
        s.close()
    assert out[0][0] == out[1][0]
    g0, g1 = out[0][1], out[1][1]
    assert np.abs(g1).max() > 0
    assert np.abs(g0 - g1).max() <= 1e-12 * np.abs(g1).max()
    np.testing.assert_allclose(out[0][2], out[1][2], rtol=1e-12)


def test_autograd_wrapper_matches_backward_and_differences(fp64_grad):
    """The torch.autograd.Function over fdtd_forward / fdtd_backward gives
    the adjoint's gradient and agrees with differences of its own forward."""
    import torch
    from fdtd_b200.autograd import AbsorbedPower
    _, L, g, gp = fp64_grad
    s = design_sim(F.FDTD_FP64, **GOLD)
    rho = torch.tensor(rho0(), dtype=torch.float64, requires_grad=True)
    Lt = AbsorbedPower.apply(rho, s, SEL, 50)
    assert Lt.item() == pytest.approx(L, rel=1e-12)
    Lt.backward()
    gt = rho.grad.numpy()
    assert np.abs(gt - g).max() <= 1e-12 * np.abs(g).max()
    np.testing.assert_allclose(s.last_param_grad, gp, rtol=1e-12)
    h, c = 1e-3, (2, 3, 1)
    with torch.no_grad():
        r = rho.detach().clone(); r[c] += h; lp = AbsorbedPower.apply(r, s, SEL, 50).item()
        r = rho.detach().clone(); r[c] -= h; lm = AbsorbedPower.apply(r, s, SEL, 50).item()
    fd = (lp - lm) / (2 * h)
    assert abs(fd - gt[c]) <= 1e-3 * abs(fd)
    s.close()


def test_checkpoint_interval_does_not_change_the_gradient(fp64_grad):
    _, L, g, gp = fp64_grad
    s = design_sim(F.FDTD_FP64, **GOLD)
    s.set_design(rho0())
    assert s.forward(SEL, 37) == pytest.approx(L, rel=1e-12)
    g2, gp2 = s.backward()
    np.testing.assert_allclose(g2, g, rtol=1e-5, atol=1e-6 * np.abs(g).max())
    np.testing.assert_allclose(gp2, gp, rtol=1e-10)


def test_full_metal_design_box_matches_oracle():
    """rho = 1 everywhere: the forward is the metal box itself, which the
    FP64 oracle (no adjoint) also rasterises from design_box."""
    steps = 120
    p = make(F, "vacuum", precision=F.FDTD_FP64, Tend=300, design_box=BOX)
    s = F.Sim(p)
    s.step(steps)
    o = O.OracleSim(make(O, "vacuum", precision=1, Tend=300, design_box=BOX))
    o.step(steps)
    for c in range(6):
        a, b = s.field(c), o.field(c)
        scale = max(np.abs(b).max(), 1e-300)
        assert np.abs(a - b).max() <= 1e-11 * scale, c


def test_design_errors():
    s = F.Sim(make(F, "vacuum", precision=F.FDTD_FP64))
    with pytest.raises(F.FdtdError) as e:
        s.forward(SEL, 50)
    assert e.value.status == 5
    with pytest.raises(F.FdtdError):
        F.Sim(make(F, "vacuum", precision=F.FDTD_FP64, design_box=[2, 6, 2, 6, 2, 6]))


def test_adjoint_matches_oracle_gradient(fp64_grad):
    """The FP64 oracle (the CPU restatement, with the same design blend)
    gives the reference gradient by central differences on the objective it
    computes itself; the GPU adjoint matches it, and the two forward
    objectives agree."""
    _, L, g, _ = fp64_grad

    def oracle_objective(rho):
        o = O.OracleSim(make(O, "vacuum", precision=1, Tend=300, design_box=BOX, **GOLD))
        o.set_design(rho)
        o.step(301)
        return sigma_abs(o.spectra(), SEL)

    rho, h = rho0(), 1e-3
    assert oracle_objective(rho) == pytest.approx(L, rel=1e-10)
    for c in [(0, 0, 0), (3, 5, 5)]:
        r = rho.copy(); r[c] += h; lp = oracle_objective(r)
        r = rho.copy(); r[c] -= h; lm = oracle_objective(r)
        fd = (lp - lm) / (2 * h)
        print(c, "oracle fd", fd, "adjoint", g[c])
        assert abs(fd - g[c]) <= 1e-3 * abs(fd)


def test_objective_is_the_positive_absorption_cross_section(fp64_grad):
    """fdtd_forward's objective is sigma_abs summed over the frequencies:
    -AbsTot for a geometry other than the reference's sphere, and positive
    for the absorbing design box."""
    s, L, _, _ = fp64_grad
    s.set_design(rho0())
    table = s.forward_spectra(50)
    assert sigma_abs(table, SEL) == pytest.approx(L, rel=1e-12)
    assert -float(table[SEL, 2].sum()) == pytest.approx(L, rel=1e-12)
    assert L > 0


def test_backward_spectra_of_the_same_objective_matches_backward(fp64_grad):
    s, L, g, gp = fp64_grad
    s.set_design(rho0())
    s.forward_spectra(50)
    G = np.zeros((s.dims.num_freq, 19))
    G[SEL, 10:16] = SIGMA_ABS
    g2, gp2 = s.backward_spectra(G)
    np.testing.assert_allclose(g2, g, rtol=1e-12, atol=1e-12 * np.abs(g).max())
    np.testing.assert_allclose(gp2, gp, rtol=1e-12)


def weighted_objective(table):
    """A mixed objective over the ScatAbs table: scattering, absorption and
    extinction at different frequencies and weights, and two face fluxes
    of the scattering box."""
    return (2.0 * table[1, 1] - 0.5 * table[3, 2] + 1.5 * table[5, 3] + 0.7 * table[7, 6]
            - 1.3 * table[2, 9] + table[4, 12])


def weighted_G(nf):
    G = np.zeros((nf, 19))
    G[1, 1] = 2.0
    G[3, 2] = -0.5
    G[5, 3] = 1.5
    G[7, 6] = 0.7
    G[2, 9] = -1.3
    G[4, 12] = 1.0
    return G


@pytest.mark.parametrize("name", ["vacuum", "sphere_au"])
def test_general_objective_matches_central_differences(name):
    """dL/drho and dL/d(omega_D, gamma) of a weighted sum of ScatAbs
    columns (totals and faces of both boxes) against central differences.
    sphere_au uses the reference's sphere normalisation (pi r^2) of the
    totals."""
    p = make(F, name, precision=F.FDTD_FP64, Tend=300, design_box=BOX, **GOLD)
    if name == "sphere_au":
        p.nano_sphere_radius = 4e-9
        for a, v in enumerate([13, 16, 13, 16, 13, 16]):
            p.design_box[a] = v
    s = F.Sim(p)
    b = list(p.design_box)
    rng = np.random.default_rng(7)
    rho = rng.uniform(0, 1, (b[5] - b[4], b[3] - b[2], b[1] - b[0])).astype(np.float32)
    s.set_design(rho)
    L = weighted_objective(s.forward_spectra(50))
    g, gp = s.backward_spectra(weighted_G(s.dims.num_freq))
    h = 1e-3
    for c in [(0, 0, 0), (1, 2, 1)]:
        r = rho.copy(); r[c] += h; s.set_design(r); lp = weighted_objective(s.forward_spectra(50))
        r = rho.copy(); r[c] -= h; s.set_design(r); lm = weighted_objective(s.forward_spectra(50))
        fd = (lp - lm) / (2 * h)
        print(name, c, "L", L, "fd", fd, "adjoint", g[c])
        assert abs(fd - g[c]) <= 1e-3 * abs(fd), (c, fd, g[c])
    s.close()
    for k, pname in enumerate(("omega_D", "gamma_D")):
        v = GOLD[pname]
        hv = v * 1e-4
        vals = []
        for x in (v + hv, v - hv):
            setattr(p, pname, x)
            q = F.Sim(p)
            q.set_design(rho)
            vals.append(weighted_objective(q.forward_spectra(50)))
            q.close()
        setattr(p, pname, v)
        fd = (vals[0] - vals[1]) / (2 * hv)
        print(name, pname, "fd", fd, "adjoint", gp[k])
        assert abs(fd - gp[k]) <= 1e-3 * abs(fd), (pname, fd, gp[k])


def test_backward_spectra_rejects_field_free_columns(fp64_grad):
    s = fp64_grad[0]
    s.set_design(rho0())
    s.forward_spectra(50)
    G = np.zeros((s.dims.num_freq, 19))
    G[0, 0] = 1.0
    with pytest.raises(F.FdtdError) as e:
        s.backward_spectra(G)
    assert e.value.status == 1
    with pytest.raises(F.FdtdError) as e:  # forward_spectra has no objective of its own
        s.backward()
    assert e.value.status == 5


@pytest.mark.parametrize("prec", [F.FDTD_FP32, F.FDTD_FP64])
def test_staged_gathers_match_fused_blocks(prec, monkeypatch):
    """The staged z-march gathers (32 x 8 x 16 tiles: the plain form away
    from the CPML, the grid's faces and the material box, the general form,
    driven by the cells' flags, everywhere else) do the fused gathers'
    arithmetic in the same order: the gradient with them and without them
    agrees to rounding (the objective's source adds to shared face-corner
    cells with atomics)."""
    box = [40, 48, 40, 48, 44, 48]
    out = []
    for mode in ("1", "0"):  # forced on (the grid is below the automatic threshold), off
        monkeypatch.setenv("FDTD_ADJ_STAGED", mode)
        s = F.Sim(make(F, "sphere_big", precision=prec, nano_sphere=0, Tend=420, design_box=box, **GOLD))
        rng = np.random.default_rng(3)
        s.set_design(rng.uniform(0, 1, (box[5] - box[4], box[3] - box[2], box[1] - box[0])).astype(np.float32))
        L = s.forward(SEL, 40)
        g, gp = s.backward()
        out.append((L, g, gp))
        s.close()
    assert out[0][0] == out[1][0]
    tol = 1e-12 if prec == F.FDTD_FP64 else 1e-5
    assert np.abs(out[0][1] - out[1][1]).max() <= tol * np.abs(out[1][1]).max()
    np.testing.assert_allclose(out[0][2], out[1][2], rtol=tol)


@pytest.mark.parametrize("model", ["local", "hydro"])
def test_recorded_and_recomputed_segments_agree(model, monkeypatch):
    """The forward records the dispersive cells' trajectory of as many of
    the last segments as the record budget holds; the backward recomputes
    the others from checkpoints into the rows already swept.  Every split
    gives the same rho gradient bit for bit (the recompute repeats the
    forward's arithmetic); the parameter gradients are sums over all cells
    by FP64 atomics, equal to rounding."""
    def run(budget_gb):
        if budget_gb is None:
            monkeypatch.delenv("FDTD_ADJ_RECORD_GB", raising=False)
        else:
            monkeypatch.setenv("FDTD_ADJ_RECORD_GB", str(budget_gb))
        if model == "local":
            s = design_sim(F.FDTD_FP64, **GOLD)
        else:
            s = F.Sim(make(F, "hydro", precision=F.FDTD_FP64, Tend=300, design_box=[14, 20, 14, 20, 14, 20],
                           **GOLD))
        b = s.params.design_box
        rng = np.random.default_rng(2)
        s.set_design(rng.uniform(0, 1, (b[5] - b[4], b[3] - b[2], b[1] - b[0])).astype(np.float32))
        L = s.forward(SEL, 50)
        st = s.stats()
        g, gp = s.backward()
        s.close()
        return L, g, gp, (st.adj_record_steps, st.adj_checkpoints, st.adj_record_bytes)

    # 301 steps in segments of 50: six full ones and the last step
    full = run(None)
    one = run(0)  # the last segment recorded, six recomputed
    assert full[3][:2] == (301, 0) and one[3][:2] == (1, 6)
    part = run(3.5 * full[3][2] / 7 / 2 ** 30)  # the last three segments
    assert part[3][:2] == (101, 4)
    for other in (one, part):
        assert other[0] == full[0]
        np.testing.assert_array_equal(other[1], full[1])
        np.testing.assert_allclose(other[2], full[2], rtol=1e-12)
