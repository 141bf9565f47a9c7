"""GPU parity: the CUDA path (through the C ABI) against the FP64 oracle.

Tolerances: FP64 fields and spectra within 1e-11 relative (norm-wise for
fields: max |a - b| / max |b|); FP32 within the bounds stated per test.
"""
import functools
import os

import numpy as np
import pytest

import fdtd_b200 as F
import oracle as O
from cases import CASES, make

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-11
FP32_TOL = 1e-5        # probe series and spectra
FP32_FIELD_TOL = 5e-5  # whole fields, max over every cell of the grid
STEPS = 300


@functools.lru_cache(maxsize=None)
def oracle_run(name, steps, **over):
    o = O.OracleSim(make(O, name, **dict(over)))
    o.step(steps)
    return o


def oracle_fields(name, steps):
    o = oracle_run(name, steps)
    return [o.field(c) for c in range(6)], o.probe()


def rel(a, b, scale=None):
    if scale is None:
        scale = np.max(np.abs(b))
    return float(np.max(np.abs(a - b)) / max(scale, 1e-300))


def field_errors(sim_fields, ref):
    """Max error of each component on the scale of its whole E or H field
    (cross-polarised components are rounding noise on their own)."""
    se = max(np.max(np.abs(ref[c])) for c in range(3))
    sh = max(np.max(np.abs(ref[c])) for c in range(3, 6))
    return [rel(sim_fields[c], ref[c], se if c < 3 else sh) for c in range(6)]


def run_sim(name, steps, prec, **over):
    s = F.Sim(make(F, name, precision=prec, **over))
    s.step(steps)
    return s


@pytest.mark.parametrize("name", sorted(CASES))
def test_fields_fp64(name):
    ref, probe = oracle_fields(name, STEPS)
    s = run_sim(name, STEPS, F.FDTD_FP64)
    errs = field_errors([s.field(c) for c in range(6)], ref)
    print(name, "fp64 field errors", ["%.2e" % e for e in errs])
    assert max(errs) < FP64_TOL, errs
    np.testing.assert_allclose(s.probe(), probe, rtol=0, atol=FP64_TOL * max(np.abs(probe).max(), 1e-30))
    s.check()


@pytest.mark.parametrize("name", sorted(CASES))
def test_fields_fp32(name):
    ref, probe = oracle_fields(name, STEPS)
    s = run_sim(name, STEPS, F.FDTD_FP32)
    errs = field_errors([s.field(c) for c in range(6)], ref)
    perr = rel(s.probe(), probe)
    print(name, "fp32 field errors", ["%.2e" % e for e in errs], "probe %.2e" % perr)
    assert max(errs) < FP32_FIELD_TOL, errs
    assert perr < FP32_TOL, perr


def spectra_pair(name, prec):
    p = make(F, name, precision=prec)
    o = oracle_run(name, p.Tend + 1)
    s = F.Sim(p)
    s.run()
    return s, o


@pytest.mark.parametrize("name", ["sphere_au", "cube_ag", "hydro", "sphere_ref", "dimer"])
def test_spectra_fp64(name):
    s, o = spectra_pair(name, F.FDTD_FP64)
    a, b = s.spectra(), o.spectra()
    # lambda and the incident spectrum are host FP64: identical
    np.testing.assert_array_equal(a[:, 0], b[:, 0])
    np.testing.assert_allclose(a[:, 16:], b[:, 16:], rtol=1e-15)
    for col in (1, 2, 3):
        err = rel(a[:, col], b[:, col])
        assert err < FP64_TOL, (col, err)
    for cols in (range(4, 10), range(10, 16)):  # faces on their box's flux scale
        scale = max(np.max(np.abs(b[:, c])) for c in cols)
        for col in cols:
            err = rel(a[:, col], b[:, col], scale)
            assert err < FP64_TOL, (col, err)
    # DFT phasors on the scale of the largest E (or H) phasor of all faces:
    # a face inside the particle holds values far below the rounding level
    # of the fields around it
    x = {(b, f, c): s.dft(b, f, c) for b in (0, 1) for f in range(6) for c in range(4)}
    y = {(b, f, c): o.dft(b, f, c) for b in (0, 1) for f in range(6) for c in range(4)}
    se = max(np.max(np.abs(v)) for k, v in y.items() if k[2] < 2)
    sh = max(np.max(np.abs(v)) for k, v in y.items() if k[2] >= 2)
    for k in x:
        err = rel(x[k], y[k], se if k[2] < 2 else sh)
        assert err < FP64_TOL, (k, err)


@pytest.mark.parametrize("name", ["sphere_au", "hydro", "dimer"])
def test_spectra_fp32(name):
    s, o = spectra_pair(name, F.FDTD_FP32)
    a, b = s.spectra(), o.spectra()
    errs = []
    for col in (1, 2):
        scale = np.max(np.abs(b[:, col]))
        errs.append(float(np.max(np.abs(a[:, col] - b[:, col])) / scale))
    print(name, "fp32 spectra errors (sca, abs)", errs)
    assert max(errs) < FP32_TOL, errs


def test_split_calls_equal_fused_step():
    n = 40
    a = run_sim("sphere_au", n, F.FDTD_FP64)
    b = F.Sim(make(F, "sphere_au", precision=F.FDTD_FP64))
    for _ in range(n):
        b.update_h()
        b.update_line()
        b.update_e()
        b.spectral_accumulate()
    for c in range(6):
        np.testing.assert_array_equal(a.field(c), b.field(c))
    np.testing.assert_array_equal(a.dft(1, 4, 0), b.dft(1, 4, 0))


def test_graph_replay_equals_direct_launches():
    n = 300  # > one 128-step graph period
    a = run_sim("hydro", n, F.FDTD_FP32)
    b = F.Sim(make(F, "hydro", precision=F.FDTD_FP32))
    for _ in range(n):
        b.step(1)
    for c in range(6):
        np.testing.assert_array_equal(a.field(c), b.field(c))
    np.testing.assert_array_equal(a.spectra(), b.spectra())


def test_spectra_read_mid_run():
    """Reading the spectra contracts the samples that no contraction has
    taken yet (the ring's halves take 64 samples each; the stepper contracts
    a half beside the steps that fill the other); the run then continues in
    the same contraction period, so its 128-step graph replays resume.
    Only the grouping of the FP64 sums changes."""
    n = 420
    a = run_sim("sphere_au", n, F.FDTD_FP64)
    b = F.Sim(make(F, "sphere_au", precision=F.FDTD_FP64))
    # a graph period plus a partial ring, then short runs, then a long tail
    # that crosses a contraction launch with the ring half full
    for k in (132, 40, 9, 239):
        b.step(k)
        b.spectra()
    assert b.t == n
    assert b.stats().graph_launches == 2  # steps 0-127, then 256-383 after the reads
    sa, sb = a.spectra(), b.spectra()
    for col in (1, 2, 3):
        assert rel(sb[:, col], sa[:, col]) < 1e-13, col
    a.close()
    b.close()


def test_reset_restarts_identically():
    s = run_sim("sphere_au", 150, F.FDTD_FP64)
    first = s.field(1)
    s.reset()
    assert s.t == 0 and np.all(s.field(1) == 0)
    s.step(150)
    np.testing.assert_array_equal(s.field(1), first)


def test_snapshot_plane_matches_field():
    s = run_sim("sphere_au", 120, F.FDTD_FP32)
    ey = s.field(1)
    np.testing.assert_array_equal(s.plane(1, 0, 17), ey[17])
    np.testing.assert_array_equal(s.plane(1, 1, 5), ey[:, 5, :])
    np.testing.assert_array_equal(s.plane(1, 2, 20), ey[:, :, 20])


def test_watchdog_reports_nonfinite():
    s = run_sim("vacuum", 10, F.FDTD_FP32)
    hx = s.field(3)
    hx[17, 17, 17] = np.nan
    s.set_field(3, hx)
    s.step(2)
    with pytest.raises(F.FdtdError) as e:
        s.check()
    assert e.value.status == 6


def test_runner_writes_the_reference_outputs(tmp_path):
    """fdtd_runner on an Input.txt deck writes OUT.txt (t*dt and E at the
    centre at the top of every step) and ScatAbs.<Tend>.txt, matching the
    same deck run through the Python binding.  The deck holds the
    reference's Input.txt fields only, so the case uses the reference's
    other constants."""
    import subprocess
    p = make(F, "sphere_ref", precision=F.FDTD_FP64, Tend=200)
    deck = tmp_path / "Input.txt"
    F.write_input_txt(str(deck), p)
    runner = os.path.join(os.path.dirname(F.LIB_PATH), "fdtd_runner")
    r = subprocess.run([runner, str(deck), "--out", str(tmp_path), "--fp64"], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stderr
    q = F.load_input_txt(str(deck))
    q.precision = F.FDTD_FP64
    s = F.Sim(q)
    s.run()
    rows = np.loadtxt(tmp_path / "ScatAbs.200.txt")
    np.testing.assert_allclose(rows, s.spectra(), rtol=1e-6)
    out = np.loadtxt(tmp_path / "OUT.txt")
    assert out.shape == (201, 4)
    probe = s.probe()
    np.testing.assert_allclose(out[1:, 1:], probe[:200], rtol=1e-6, atol=1e-6 * np.abs(probe).max())
    np.testing.assert_array_equal(out[0, 1:], 0.0)
    np.testing.assert_allclose(out[:, 0], np.arange(201) * s.dims.dt, rtol=1e-6)
    s.close()


def test_scatabs_file_format(tmp_path):
    s = run_sim("sphere_au", 200, F.FDTD_FP64)
    path = tmp_path / "ScatAbs.200.txt"
    s.write_scatabs(str(path))
    rows = np.loadtxt(path)
    assert rows.shape == (s.dims.num_freq, 19)
    np.testing.assert_allclose(rows, s.spectra(), rtol=1e-6)


@pytest.mark.parametrize("prec", [F.FDTD_FP32, F.FDTD_FP64])
def test_pass_variants_agree(prec, monkeypatch):
    """The launch shapes the autotuner chooses between (tile height, z-chunk,
    register cap, ring depth) change data movement only: fields are
    bit-identical."""
    out = []
    for spec in ("staged:4:1:16:4", "staged:8:3:8:4", "staged:4:6:32:6"):
        monkeypatch.setenv("FDTD_PASS", spec)
        s = run_sim("sphere_big", 200, prec)
        st = s.stats()
        assert (st.h_ty, st.h_minb, st.h_kchunk, st.h_stages) == tuple(int(x) for x in spec.split(":")[1:])
        out.append([s.field(c) for c in range(6)])
    # the passes use fixed-rounding arithmetic: the shape changes nothing
    for other in out[1:]:
        for c in range(6):
            np.testing.assert_array_equal(other[c], out[0][c])


@pytest.mark.parametrize("prec", [F.FDTD_FP32, F.FDTD_FP64])
@pytest.mark.parametrize("nonlocal_", [0, 3])
def test_pass_overlap_modes_agree(prec, nonlocal_, monkeypatch):
    """The interior and CPML-edge launches of a pass write disjoint cells, and
    the 1D line and the dispersive kernels touch none of the passes' cells,
    so the two arrangements of a step give identical fields: the CPML tables
    and the line and dispersive kernels on side streams (FDTD_PDL=0), or all
    on one stream, each launch with a programmatic dependency on the one
    before (FDTD_PDL=1), with the local Drude + 2CP model and with the
    hydrodynamic model (three dependent phases).  The FP64 hydrodynamic run
    is also checked against the oracle."""
    monkeypatch.setenv("FDTD_PASS", "staged:4:6:16:4")
    steps = 300
    out = []
    for mode in ("0", "1"):
        monkeypatch.setenv("FDTD_PDL", mode)
        s = run_sim("sphere_big", steps, prec, NONLOCAL=nonlocal_)
        st = s.stats()
        assert st.h_pdl == st.e_pdl == int(mode)
        s.check()
        out.append([s.field(c) for c in range(6)])
        s.close()
    for c in range(6):
        np.testing.assert_array_equal(out[0][c], out[1][c])
    if nonlocal_ and prec == F.FDTD_FP64:
        o = oracle_run("sphere_big", steps, NONLOCAL=nonlocal_)
        errs = field_errors(out[1], [o.field(c) for c in range(6)])
        assert max(errs) < FP64_TOL, errs


@pytest.mark.parametrize("prec", [F.FDTD_FP32, F.FDTD_FP64])
def test_tensor_copy_staging_agrees(prec, monkeypatch):
    """The two ways a pass fills its shared-memory ring (per-thread cp.async
    copies, or tensor copies completing on an mbarrier) move the same
    values, zero fill outside the grid included: fields are bit-identical,
    for every tile height and ring depth."""
    for spec in ("staged:4:6:16:4", "staged:8:3:8:4", "staged:4:6:32:6"):
        monkeypatch.setenv("FDTD_PASS", spec)
        out = []
        for mode in ("0", "1"):
            monkeypatch.setenv("FDTD_TMA", mode)
            s = run_sim("sphere_big", 120, prec)
            st = s.stats()
            assert st.h_tma == st.h_etma == st.e_tma == st.e_etma == int(mode)
            s.check()
            out.append([s.field(c) for c in range(6)])
            s.close()
        for c in range(6):
            np.testing.assert_array_equal(out[0][c], out[1][c])


def test_tensor_copy_wait_timeout_is_reported(monkeypatch):
    """A tensor-copy wait gives up after one second.  With the copies never
    issued (the test switch FDTD_TMA_STALL_TEST=1) every wait of the passes
    runs out, the kernels end, and fdtd_check reports FDTD_ERR_TIMEOUT; the
    GPU context stays usable for the next simulation."""
    monkeypatch.setenv("FDTD_TMA", "1")
    monkeypatch.setenv("FDTD_TMA_STALL_TEST", "1")
    s = F.Sim(make(F, "vacuum", precision=F.FDTD_FP32))
    assert s.stats().h_tma == 1 and s.stats().e_etma == 1
    s.step(1)
    with pytest.raises(F.FdtdError) as e:
        s.check()
    assert e.value.status == 7 and "gave up" in str(e.value)
    s.close()
    monkeypatch.delenv("FDTD_TMA_STALL_TEST")
    t = run_sim("vacuum", 20, F.FDTD_FP32)
    t.check()
    assert t.stats().h_tma == 1


def test_unbuilt_pass_variant_is_rejected(monkeypatch):
    monkeypatch.setenv("FDTD_PASS", "staged:8:5:16:4")
    with pytest.raises(F.FdtdError) as e:
        F.Sim(make(F, "vacuum", precision=F.FDTD_FP32))
    assert e.value.status == 1 and "not built" in str(e.value)


def test_spectral_error_table():
    """The error of every spectrum against the FP64 oracle, FP64 and FP32
    builds: max over wavelengths of |this - oracle| / max |oracle| for the
    scattering, absorption and extinction columns.  Written as a table to
    the path in FDTD_PARITY_REPORT when set."""
    rows = []
    for name in sorted(n for n in CASES if not CASES[n].get("periodic_xy")):  # periodic: no ScatAbs
        errs = {}
        for prec, tag in ((F.FDTD_FP64, "f64"), (F.FDTD_FP32, "f32")):
            s, o = spectra_pair(name, prec)
            a, b = s.spectra(), o.spectra()
            errs[tag] = [float(np.max(np.abs(a[:, c] - b[:, c])) / np.max(np.abs(b[:, c]))) for c in (1, 2, 3)]
            s.close()
        rows.append((name, errs))
        if name != "vacuum":  # no particle: its spectra are leakage noise
            assert max(errs["f64"]) < 1e-10, (name, errs)
            assert max(errs["f32"]) < FP32_TOL, (name, errs)
    path = os.environ.get("FDTD_PARITY_REPORT")
    if path:
        with open(path, "w") as f:
            f.write("| case | FP64 sca | FP64 abs | FP64 ext | FP32 sca | FP32 abs | FP32 ext |\n")
            f.write("|---|---|---|---|---|---|---|\n")
            for name, e in rows:
                f.write(f"| {name} | " + " | ".join("%.1e" % x for x in e["f64"] + e["f32"]) + " |\n")
