"""Periodic x and y (params.periodic_xy, the reference's Periodic_XY
branches): the CUDA path against the FP64 oracle's periodic mode, fields
and the reflectance / transmittance spectra (fdtd_reflectance), and the
runner's Reflectivity files.  The oracle's periodic mode is pinned by
closed-form answers (tests/test_oracle_periodic.py)."""
import os
import subprocess

import numpy as np
import pytest

import fdtd_b200 as F
import oracle as O
from cases import gold_film_rt, make

pytestmark = pytest.mark.gpu

NAMES = ["periodic_vacuum", "periodic_film", "periodic_spheres"]
FP32_TOL = 1e-5


def fields_close(s, o, tol, peak):
    """Errors on the scale of the largest field of the run so far (peak,
    updated in place): once the pulse has left through the z CPML the
    residual fields are 1e-5 of it, and rounding differences from the
    pulse's passage would read as large errors on their own scale."""
    for f, fam in enumerate(((0, 1, 2), (3, 4, 5))):
        ref = [o.field(c) for c in fam]
        peak[f] = max(peak[f], max(np.abs(x).max() for x in ref))
        assert peak[f] > 0
        for c, b in zip(fam, ref):
            err = np.abs(s.field(c) - b).max() / peak[f]
            assert err <= tol, (c, err)


@pytest.mark.parametrize("name", NAMES)
@pytest.mark.parametrize("prec", [F.FDTD_FP64, F.FDTD_FP32])
def test_fields_and_reflectance_match_oracle(name, prec):
    p = make(F, name, precision=prec)
    s = F.Sim(p)
    assert (s.dims.nx, s.dims.ny) == (p.NCELLX, p.NCELLY)
    o = O.OracleSim(make(O, name))
    peak = [0.0, 0.0]
    # the pulse crossing the TFSF plane, at the film, leaving; the end of the run
    for n in (400, 100, 200, p.Tend + 1 - 700):
        s.step(n)
        o.step(n)
        fields_close(s, o, 1e-11 if prec == F.FDTD_FP64 else FP32_TOL, peak)
    r, ro = s.reflectance(), o.reflectance()
    np.testing.assert_array_equal(r[:, 0], ro[:, 0])
    tol = 1e-9 if prec == F.FDTD_FP64 else 1e-4
    assert np.abs(r[:, 1:4] - ro[:, 1:4]).max() <= tol
    s.close()


def test_gold_film_reflectance_is_physical():
    p = make(F, "periodic_film", precision=F.FDTD_FP32)
    s = F.Sim(p)
    s.run()
    r = s.reflectance()
    R, T = gold_film_rt(r[:, 0], int(p.nano_sphere_radius / p.dz) * p.dz)
    assert np.abs(r[:, 1] - R).max() < 0.01 and np.abs(r[:, 2] - T).max() < 0.01
    s.close()


def test_periodic_refuses_box_spectra_and_batches():
    p = make(F, "periodic_vacuum", precision=F.FDTD_FP32, Tend=100)
    s = F.Sim(p)
    s.run()
    with pytest.raises(F.FdtdError):
        s.spectra()
    with pytest.raises(F.FdtdError):
        F.Batch([p, p])
    q = F.Sim(make(F, "vacuum", precision=F.FDTD_FP32, Tend=20))
    with pytest.raises(F.FdtdError):
        q.reflectance()
    s.close()
    q.close()


def test_runner_writes_reflectivity_files(tmp_path):
    p = make(F, "periodic_film", Tend=1000)
    deck = tmp_path / "Input.txt"
    F.write_input_txt(str(deck), p)
    runner = os.path.join(os.path.dirname(F.LIB_PATH), "fdtd_runner")
    r = subprocess.run([runner, str(deck), "--out", str(tmp_path), "--fp64", "--periodic-xy"],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    files = sorted(f for f in os.listdir(tmp_path) if f.startswith("ReflectivityTE."))
    assert files == sorted(f"ReflectivityTE.1.{t}.txt" for t in range(100, 1001, 100))
    assert not any(f.startswith("ScatAbs.") for f in os.listdir(tmp_path))
    q = F.load_input_txt(str(deck))
    q.precision, q.periodic_xy = F.FDTD_FP64, 1
    s = F.Sim(q)
    s.step(501)
    ref = s.reflectance()
    got = np.loadtxt(tmp_path / "ReflectivityTE.1.500.txt")
    amp = ref[1:, 4] ** 2
    want = np.c_[ref[1:, 0], ref[1:, 1], -ref[1:, 2], amp, ref[1:, 1] * amp, -ref[1:, 2] * amp]
    np.testing.assert_allclose(got, want, rtol=1e-6, atol=1e-12)
    s.close()


def test_reflectance_error_table():
    """The error of R and T against the FP64 oracle, FP64 and FP32 builds,
    max over wavelengths; written as a table to the path in
    FDTD_PARITY_REPORT_PERIODIC when set."""
    rows = []
    for name in NAMES:
        ro = None
        errs = []
        for prec in (F.FDTD_FP64, F.FDTD_FP32):
            p = make(F, name, precision=prec)
            s = F.Sim(p)
            s.run()
            r = s.reflectance()
            s.close()
            if ro is None:
                o = O.OracleSim(make(O, name))
                o.step(p.Tend + 1)
                ro = o.reflectance()
            errs += [float(np.abs(r[:, 1] - ro[:, 1]).max()), float(np.abs(r[:, 2] - ro[:, 2]).max())]
        assert max(errs[:2]) < 1e-9 and max(errs[2:]) < 1e-4, (name, errs)
        rows.append((name, errs, float(ro[:, 1].max()), float(ro[:, 2].min())))
    path = os.environ.get("FDTD_PARITY_REPORT_PERIODIC")
    if path:
        with open(path, "w") as f:
            f.write("| case | max R | min T | FP64 R | FP64 T | FP32 R | FP32 T |\n|---|---|---|---|---|---|---|\n")
            for name, e, rmax, tmin in rows:
                f.write(f"| {name} | {rmax:.3f} | {tmin:.3f} | " + " | ".join("%.1e" % x for x in e) + " |\n")
