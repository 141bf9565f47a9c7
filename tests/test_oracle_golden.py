"""The oracle against the reference program's own outputs.

Fixtures under tests/golden/ were produced by running the unmodified
reference (jbaxt089/FDTD-CUDA, built by oracle/Makefile.ref) on a B200 with
the decks in ref_cases.py (make_ref_golden.sh, import_ref_golden.py).  The
reference prints 7 significant digits, so agreement is checked at 2e-6 of
each quantity's scale.  The oracle runs with the reference's float DFT
accumulators emulated (global_var.h:22)."""
import os

import numpy as np
import pytest

import oracle as O
import ref_cases as R

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
PRINT_TOL = 2e-6


@pytest.fixture(scope="module", params=sorted(R.CASES))
def case(request):
    name = request.param
    path = os.path.join(HERE, f"ref_{name}.npz")
    if not os.path.exists(path):
        pytest.skip(f"fixture {path} not generated")
    g = np.load(path)
    s = O.OracleSim(O.default_params(**R.CASES[name]), float_dft=True)
    s.step(R.CASES[name]["Tend"] + 1)
    return name, g, s


def test_centre_probe_series(case):
    name, g, s = case
    pr = s.probe()
    ey = np.concatenate([[0.0], pr[:-1, 1]])  # printed at the top of step t
    ref = g["ey_centre"]
    assert len(ref) == len(ey)
    assert np.max(np.abs(ey - ref)) <= PRINT_TOL * np.max(np.abs(ref))


def test_scatabs_columns(case):
    name, g, s = case
    sp = s.spectra()
    key = sorted((k for k in g.files if k.startswith("scatabs_")), key=lambda k: int(k.split("_")[1]))[-1]
    ref = g[key]
    assert ref.shape == sp.shape
    np.testing.assert_allclose(sp[:, 0], ref[:, 0], rtol=1e-6)
    # face fluxes: compare on the scale of the largest flux of the same box
    for cols in (range(4, 10), range(10, 16)):
        scale = max(np.max(np.abs(ref[:, c])) for c in cols)
        for c in cols:
            assert np.max(np.abs(sp[:, c] - ref[:, c])) <= 5 * PRINT_TOL * scale, (name, c)
    for c in (1, 2):  # totals (normalised by pi r^2 for the sphere)
        scale = np.max(np.abs(ref[:, c]))
        if scale > 1e-25:
            assert np.max(np.abs(sp[:, c] - ref[:, c])) <= 5 * PRINT_TOL * scale, (name, c)
    np.testing.assert_allclose(sp[:, 16:], ref[:, 16:], rtol=1e-6, atol=1e-6 * np.abs(ref[:, 16]).max())
