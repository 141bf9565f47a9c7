"""GPU parity on the benchmark's own configurations, through the C ABI.

* the small plain configuration exactly as the benchmark states it (64^3,
  kappa_max = 1, TFSF inset 8, x-polarised, 2000 steps, 101 wavelengths
  over 400-900 nm), FP32 and FP64, against the FP64 oracle;
* the headline workload (256^3 gold rod dimer with the hydrodynamic
  current, 12-cell CPML, 201 wavelengths) for the first 256 time steps,
  FP32 and FP64, against the FP64 oracle.  At 256^3 the passes run both of
  their launches (the CPML-free interior box and the CPML edge tiles) with
  the tile shapes the autotuner picks for the benchmark;
* the reference program's own outputs (tests/golden/ref_*.npz, produced
  by the unmodified reference on a B200) against this build directly.

Tolerances: FP64 within 1e-11 and FP32 within 1e-5 relative, each error
taken on the scale of its quantity (max |this - oracle| / max |oracle|):
the probe series, each spectrum column, every DFT phasor array (on the
scale of the largest E or H phasor of all faces) and the whole fields (on
the scale of the E or H family).  One exception, in FP32: the whole fields
at the end of the 2000-step run of the small configuration.  By then the
pulse has left the box and the fields are the particle's ringing, far
below the pulse whose passage set the size of the accumulated rounding;
they are bounded by 1e-4 of their own scale.
"""
import functools
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

FP64_TOL = 1e-11
FP32_TOL = 1e-5
HEADLINE_STEPS = 256


def rel(a, b, scale=None):
    if scale is None:
        scale = np.max(np.abs(b))
    return float(np.max(np.abs(a - b)) / max(scale, 1e-300))


@functools.lru_cache(maxsize=None)
def oracle_small():
    o = O.OracleSim(bench.small_params(O, 1))
    o.step(2000)
    return o


@functools.lru_cache(maxsize=None)
def oracle_headline():
    o = O.OracleSim(bench.workload_params(O, 1))
    o.step(HEADLINE_STEPS)
    return o


def compare(sim, orc, tol, spectra_cols=(1, 2, 3), field_tol=None):
    """Every error of sim against orc; asserts each is below tol (the whole
    fields below field_tol when given)."""
    out = {}
    ref = [orc.field(c) for c in range(6)]
    got = [sim.field(c) for c in range(6)]
    for fam, cs in (("E", range(3)), ("H", range(3, 6))):
        scale = max(np.max(np.abs(ref[c])) for c in cs)
        out["field_" + fam] = max(rel(got[c], ref[c], scale) for c in cs)
    pa, pb = sim.probe(), orc.probe()
    assert pa.shape == pb.shape
    out["probe"] = rel(pa, pb)
    x = {(b, f, c): sim.dft(b, f, c) for b in (0, 1) for f in range(6) for c in range(4)}
    y = {(b, f, c): orc.dft(b, f, c) for b in (0, 1) for f in range(6) for c in range(4)}
    se = max(np.max(np.abs(v)) for k, v in y.items() if k[2] < 2)
    sh = max(np.max(np.abs(v)) for k, v in y.items() if k[2] >= 2)
    out["dft"] = max(rel(x[k], y[k], se if k[2] < 2 else sh) for k in x)
    a, b = sim.spectra(), orc.spectra()
    np.testing.assert_array_equal(a[:, 0], b[:, 0])
    for c, name in zip((1, 2, 3), ("sca", "abs", "ext")):
        if c in spectra_cols:
            out[name] = rel(a[:, c], b[:, c])
    print({k: "%.2e" % v for k, v in out.items()})
    for k, v in out.items():
        bound = field_tol if (field_tol and k.startswith("field_")) else tol
        assert v < bound, (k, v, bound)
    return out


@pytest.mark.parametrize("prec", [F.FDTD_FP64, F.FDTD_FP32])
def test_small_plain_configuration(prec):
    p = bench.small_params(F, prec)
    s = F.Sim(p)
    d = s.dims
    assert (d.nx, d.ny, d.nz) == (64, 64, 64) and d.num_freq == 101
    assert (d.ntfsf_x, d.ntfsf_y, d.ntfsf_z) == (18, 18, 18)
    s.run()
    assert s.t == 2000
    if prec == F.FDTD_FP64:
        compare(s, oracle_small(), FP64_TOL)
    else:
        compare(s, oracle_small(), FP32_TOL, field_tol=1e-4)
    s.check()
    s.close()


@pytest.mark.parametrize("prec", [F.FDTD_FP64, F.FDTD_FP32])
def test_headline_workload(prec):
    """The headline's geometry, hydrodynamic cells, 201-wavelength DFT layout
    and interior/edge tile split over two 128-step graph blocks.  The
    spectra of a run stopped before the pulse has passed are not compared
    (they are not yet a physical quantity), the accumulators are."""
    p = bench.workload_params(F, prec)
    s = F.Sim(p)
    d = s.dims
    assert (d.nx, d.ny, d.nz) == (256, 256, 256) and d.num_freq == 201 and d.hydro == 1
    st = s.stats()
    assert st.h_ty > 0 and st.e_ty > 0
    s.step(HEADLINE_STEPS)
    compare(s, oracle_headline(), FP64_TOL if prec == F.FDTD_FP64 else FP32_TOL, spectra_cols=())
    s.check()
    s.close()


# ----------------------------------------------------------------------
# this build against the reference program's own outputs

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
PRINT_TOL = 2e-6  # the reference prints 7 significant digits


def golden_cases():
    sys.path.insert(0, HERE)
    import ref_cases
    return ref_cases.CASES


@pytest.mark.parametrize("prec", [F.FDTD_FP64, F.FDTD_FP32])
@pytest.mark.parametrize("name", sorted(golden_cases()))
def test_against_reference_outputs(name, prec):
    """The centre ey series the reference prints every step (main.cu:2726)
    and its ScatAbs columns (Spectral.cu:1157-1174) against this build's
    probe and spectra.  The reference accumulates its DFT in float
    (global_var.h:22) and prints 7 digits; this build accumulates in FP64.
    Bounds: the print tolerance (2e-6 of scale) for the probe, 5x it for
    the fluxes (sums of float products), plus the FP32 bound in FP32."""
    case = golden_cases()[name]
    g = np.load(os.path.join(HERE, f"ref_{name}.npz"))
    s = F.Sim(F.default_params(precision=prec, **case))
    s.run()
    extra = 0.0 if prec == F.FDTD_FP64 else FP32_TOL
    pr = s.probe()
    ey = np.concatenate([[0.0], pr[:-1, 1]])  # printed at the top of step t
    ref = g["ey_centre"]
    assert len(ref) == len(ey)
    e_probe = rel(ey, ref)
    sp = s.spectra()
    key = sorted((k for k in g.files if k.startswith("scatabs_")), key=lambda k: int(k.split("_")[1]))[-1]
    rf = g[key]
    assert rf.shape == sp.shape
    np.testing.assert_allclose(sp[:, 0], rf[:, 0], rtol=1e-6)
    errs = {"probe": e_probe}
    for tag, cols in (("sca_faces", range(4, 10)), ("abs_faces", range(10, 16))):
        scale = max(np.max(np.abs(rf[:, c])) for c in cols)
        if scale > 1e-25:
            errs[tag] = max(rel(sp[:, c], rf[:, c], scale) for c in cols)
    for c, tag in ((1, "sca"), (2, "abs")):
        scale = np.max(np.abs(rf[:, c]))
        if scale > 1e-25:
            errs[tag] = rel(sp[:, c], rf[:, c], scale)
    print(name, prec, {k: "%.2e" % v for k, v in errs.items()})
    assert errs["probe"] <= PRINT_TOL + extra, errs
    for k, v in errs.items():
        if k != "probe":
            assert v <= 5 * PRINT_TOL + extra, (k, errs)
    np.testing.assert_allclose(sp[:, 16:], rf[:, 16:], rtol=1e-6, atol=1e-6 * np.abs(rf[:, 16]).max())
    s.close()
