"""Setup tables of the product (host FP64) against the oracle: CPML
(SETUP_CPML, setup.cu:513-978), ADE (SETUP_Drude_CP, setup.cu:1282-1373),
rasteriser (MATERIAL_MATRIX, setup.cu:135-342), frequency grid and pulse.
All are integer or FP64 host arithmetic and must agree bit for bit."""
import numpy as np
import pytest

import fdtd_b200 as F
import oracle as O
from cases import CASES, make


@pytest.mark.parametrize("name", sorted(CASES))
def test_tables_bit_exact(name):
    p, q = make(F, name), make(O, name)
    s = O.OracleSim(q, dft=False)
    for w in range(30):
        np.testing.assert_array_equal(F.coefficients(p, w), s.cpml(w), err_msg=f"cpml table {w}")
    np.testing.assert_array_equal(F.coefficients(p, 100), s.ade())
    np.testing.assert_array_equal(F.coefficients(p, 101), s.freqs())
    bits, _ = s.material()
    np.testing.assert_array_equal(F.rasterise(p), bits)


def test_bh_x_far_is_zero_unless_fixed():
    # setup.cu:681 uploads bh_z_F before it is computed
    p = make(F, "sphere_au")
    assert np.all(F.coefficients(p, 6 + 6) == 0.0)
    p.fixes = F.FIX_BH_X_F
    assert np.all(F.coefficients(p, 6 + 6) > 0.0)


def test_cpml_profile_closed_form():
    p = make(F, "vacuum")
    Nc, m = p.NcpmlX, p.cpml_order
    dt = F.plan(p).dt
    smax = p.cpml_sigma_factor * (m + 1) / (376.730313462 * p.dx)
    i = np.arange(Nc + 1)
    S = ((Nc - i) / Nc) ** m * smax
    A = p.cpml_alpha_max * i / Nc
    K = 1 + (p.cpml_kappa_max - 1) * ((Nc - i) / Nc) ** m
    b = np.exp(-(S / K + A) * dt / 8.85418782e-12)
    np.testing.assert_allclose(F.coefficients(p, 6 + 0), b, rtol=1e-14)
    np.testing.assert_allclose(F.coefficients(p, 0)[: Nc + 1], K * p.dx, rtol=1e-14)


def test_drude_permittivity_closed_form():
    """The ADE recursion's eps(w) for a Drude pole reproduces
    eps_inf - wD^2/(w^2 + i g w) in the limit dt*w << 1."""
    p = make(F, "sphere_au")
    a = F.coefficients(p, 100)
    dt = a[19]
    d1, d2, d3, d4, d5 = a[3:8]
    w = 2 * np.pi * 4e14
    z = np.exp(-1j * w * dt)  # exp(-i w t) convention
    # P = (d3 z^{0} + d4 z^{-1} + d5 z^{-2}) E / (1 - d1 z^{-1} - d2 z^{-2})
    chi = (d3 + d4 / z + d5 / z**2) / (1 - d1 / z - d2 / z**2) / 8.85418782e-12
    wD, g = 1.3202e16, 1.0805e14
    exact = -wD**2 / (w**2 + 1j * g * w)
    assert abs(chi - exact) / abs(exact) < 1e-3
