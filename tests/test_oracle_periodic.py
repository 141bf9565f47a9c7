"""The oracle's periodic x/y path (the reference's Periodic_XY branches and
Reflectance_XZ) against closed-form answers: a plane wave through vacuum
is neither reflected nor attenuated, and a gold film reflects and
transmits what the Airy sums of its Drude + two-critical-point
permittivity give.  The reference switches its periodic path off
(main.cu:2398) and cannot be run on it, so these known answers pin it."""
import numpy as np
import pytest

import oracle as O
from cases import gold_film_rt, make


def run(name, **over):
    p = make(O, name, **over)
    o = O.OracleSim(p)
    o.step(p.Tend + 1)
    return p, o


def test_vacuum_transmits_everything():
    _, o = run("periodic_vacuum")
    r = o.reflectance()
    assert np.abs(r[:, 1]).max() < 1e-6      # R
    assert np.abs(r[:, 2] - 1).max() < 1e-3  # T
    np.testing.assert_allclose(r[:, 3], 1 - r[:, 1] - r[:, 2])


def test_gold_film_matches_airy():
    p, o = run("periodic_film")
    r = o.reflectance()
    d = int(p.nano_sphere_radius / p.dz) * p.dz
    R, T = gold_film_rt(r[:, 0], d)
    # 2 nm cells: the staircased film and the Yee dispersion stay within
    # 0.01 of the exact answer between 200 and 700 nm
    assert np.abs(r[:, 1] - R).max() < 0.01
    assert np.abs(r[:, 2] - T).max() < 0.01


def test_fields_are_periodic_and_uniform_in_vacuum():
    """Normal incidence on a periodic vacuum column: every xy plane is
    uniform (no lateral TFSF edges scatter)."""
    _, o = run("periodic_vacuum", Tend=400)
    for c in range(6):
        f = o.field(c)
        assert np.abs(f - f[:1, :1, :]).max() <= 1e-12 * max(np.abs(f).max(), 1e-300), c


def test_periodic_rejects_lateral_cpml_and_spectra():
    with pytest.raises(ValueError):
        O.OracleSim(make(O, "periodic_vacuum", NcpmlX=4))
    _, o = run("periodic_vacuum", Tend=50)
    with pytest.raises(RuntimeError):
        o.spectra()
    o2 = O.OracleSim(make(O, "vacuum"))
    with pytest.raises(RuntimeError):
        o2.reflectance()
