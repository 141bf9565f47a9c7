"""Snapshots taken by the stepper (fdtd_snapshots_enable / _drain) and the
runner's output files: against the FP64 oracle's state at the same steps,
and against the reference program's own snapshot files
(tests/golden/ref_snap_*.npz, produced by the unmodified reference on a
B200 with the decks of ref_cases.SNAP_CASES)."""
import os
import subprocess
import sys

import numpy as np
import pytest

import fdtd_b200 as F
import oracle as O
from cases import make

pytestmark = pytest.mark.gpu

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
SKIP = dict(t_skip=40, y_skip=2, z_skip=3, Tend=299)


def expected(o, mode, p):
    """The record the reference writes after the oracle's last step."""
    nx, ny, nz = o.shape
    xc = nx // 2
    ys, zs = slice(0, ny, p.y_skip), slice(0, nz, p.z_skip)
    out = {}
    if mode in (1, 3):
        out["aux"] = o.field(1)[2, 2, zs]
        out["line"] = o.line()[0][:: p.z_skip]
    if mode == 3:
        E = [o.field(c)[xc][ys, zs] for c in range(3)]
        out["plane"] = np.sqrt(E[0] ** 2 + E[1] ** 2 + E[2] ** 2)
    if mode == 2:
        P = [o.state(0, c)[xc][ys, zs] for c in range(3)]
        out["plane"] = np.sqrt(P[0] ** 2 + P[1] ** 2 + P[2] ** 2)
        out["plane2"] = sum(o.state(1, c)[xc][ys, zs] for c in range(3)) / 3.0
    return out


@pytest.mark.parametrize("mode,name", [(3, "sphere_au"), (2, "hydro"), (1, "hydro"), (2, "sphere_au")])
def test_snapshots_match_oracle(mode, name):
    p = make(F, name, precision=F.FDTD_FP64, **SKIP)
    s = F.Sim(p)
    lay = s.enable_snapshots(mode, 16)
    s.step(p.Tend + 1)
    recs = s.drain_snapshots()
    assert [r["t"] for r in recs] == list(range(0, p.Tend + 1, p.t_skip))
    o = O.OracleSim(make(O, name, precision=1, **SKIP))
    for r in recs:
        o.step(r["t"] + 1 - o.t)
        ref = expected(o, mode, p)
        assert set(ref) == set(k for k in r if k != "t")
        # the aux line runs through the CPML corner: its values are judged
        # on the scale of the whole E field
        escale = max(np.abs(o.field(c)).max() for c in range(3))
        for k, v in ref.items():
            assert r[k].shape == v.shape, k
            scale = escale if k == "aux" else max(np.abs(v).max(), 1e-300)
            assert np.abs(r[k] - v).max() <= 1e-11 * scale, (r["t"], k)
    assert lay.record == 1 + sum(v.size for v in ref.values())
    s.close()


def test_snapshots_are_graph_replays():
    """Taken inside the 128-step graph blocks: the same records as the
    eager steps."""
    p = make(F, "sphere_au", precision=F.FDTD_FP32, t_skip=16, Tend=299)
    a = F.Sim(p)
    a.enable_snapshots(3, 32)
    a.step(256)
    ra = a.drain_snapshots()
    b = F.Sim(p)
    b.enable_snapshots(3, 32)
    for _ in range(256):
        b.step(1)
    rb = b.drain_snapshots()
    assert a.stats().graph_launches == 2 and b.stats().graph_launches == 0
    assert len(ra) == len(rb) == 16
    for x, y in zip(ra, rb):
        for k in x:
            np.testing.assert_array_equal(x[k], y[k])


def test_ring_overflow_is_refused():
    s = F.Sim(make(F, "vacuum", precision=F.FDTD_FP32, t_skip=1))
    s.enable_snapshots(1, 4)
    s.step(4)
    with pytest.raises(F.FdtdError) as e:
        s.step(1)
    assert e.value.status == 5
    assert len(s.drain_snapshots()) == 4
    s.step(3)
    assert [r["t"] for r in s.drain_snapshots()] == [4, 5, 6]


def run_runner(tmp_path, p):
    deck = tmp_path / "Input.txt"
    F.write_input_txt(str(deck), p)
    runner = os.path.join(os.path.dirname(F.LIB_PATH), "fdtd_runner")
    r = subprocess.run([runner, str(deck), "--out", str(tmp_path), "--fp64"], capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr
    return r


@pytest.mark.parametrize("mode", [2, 3])
def test_runner_writes_snapshot_files_and_spectra(tmp_path, mode):
    """fdtd_runner on a deck with Snap_in: the reference's file names and
    counter, the drained values at print precision, and ScatAbs.<t>.txt at
    every Tend/10 step."""
    # the deck carries the Input.txt fields only: the case keeps the
    # reference's other constants, and the comparison reads the deck back
    p = make(F, "sphere_ref", NONLOCAL=3, Snap_in=mode, t_skip=50, y_skip=2, z_skip=3, Tend=300)
    run_runner(tmp_path, p)
    p = F.load_input_txt(str(tmp_path / "Input.txt"))
    p.precision = F.FDTD_FP64
    s = F.Sim(p)
    s.enable_snapshots(mode, 16)
    s.step(p.Tend + 1)
    recs = s.drain_snapshots()
    count = 0
    for r in recs:
        if mode == 3:
            np.testing.assert_allclose(np.loadtxt(tmp_path / f"aux_sim.{count}.txt"), r["aux"], rtol=1e-6,
                                       atol=1e-6 * np.abs(r["aux"]).max())
            np.testing.assert_allclose(np.loadtxt(tmp_path / f"aux_sim.{count}_2.txt"), r["line"], rtol=1e-6,
                                       atol=1e-6 * np.abs(r["line"]).max())
            count += 1
        plane = np.loadtxt(tmp_path / "videofiles" / f"YZ_sim.{count}.txt", ndmin=2)
        np.testing.assert_allclose(plane, r["plane"], rtol=1e-6, atol=1e-6 * np.abs(r["plane"]).max())
        count += 1
        if mode == 2:
            nplane = np.loadtxt(tmp_path / "videofiles" / f"YZ_sim.{count}_N.txt", ndmin=2)
            np.testing.assert_allclose(nplane, r["plane2"], rtol=1e-6, atol=1e-6 * np.abs(r["plane2"]).max())
            count += 1
    dumps = sorted(int(f.split(".")[1]) for f in os.listdir(tmp_path) if f.startswith("ScatAbs."))
    assert dumps == list(range(0, 301, 30))
    s2 = F.Sim(p)
    s2.step(91)
    np.testing.assert_allclose(np.loadtxt(tmp_path / "ScatAbs.90.txt"), s2.spectra(), rtol=1e-6)
    s.close()
    s2.close()


def golden_snap_cases():
    sys.path.insert(0, HERE)
    import ref_cases
    return ref_cases.SNAP_CASES


@pytest.mark.parametrize("name", sorted(golden_snap_cases()))
@pytest.mark.parametrize("prec", [F.FDTD_FP64, F.FDTD_FP32])
def test_against_reference_snapshots(name, prec):
    """The reference's own snapshot files against this build's records, at
    the reference's print precision (7 digits; 2e-6 of each plane's or
    line's scale), plus the FP32 bound in FP32."""
    path = os.path.join(HERE, f"ref_{name}.npz")
    if not os.path.exists(path):
        pytest.skip(f"fixture {path} not generated")
    g = np.load(path)
    case = golden_snap_cases()[name]
    p = F.default_params(precision=prec, **case)
    s = F.Sim(p)
    s.enable_snapshots(p.Snap_in, 16)
    s.run()
    recs = s.drain_snapshots()
    tol = 2e-6 + (1e-5 if prec == F.FDTD_FP32 else 0.0)
    count = 0
    checked = 0
    for r in recs:
        pairs = []
        # the aux line of ey at (2, 2, z) runs through the CPML corner: judged
        # on the scale of the record's |E| plane
        plane_key = f"yz_{count + 1}" if p.Snap_in == 3 else None
        if p.Snap_in in (1, 3):
            pairs += [(f"aux_{count}", r["aux"]), (f"aux_{count}_2", r["line"])]
            count += 1
        if p.Snap_in in (2, 3):
            pairs.append((f"yz_{count}", r["plane"]))
            count += 1
        if p.Snap_in == 2:
            pairs.append((f"yz_{count}_N", r["plane2"]))
            count += 1
        for key, mine in pairs:
            ref = g[key]
            assert ref.shape == mine.shape, (key, ref.shape, mine.shape)
            scale = np.abs(ref).max()
            if plane_key and key == f"aux_{count - 2}":
                scale = max(scale, np.abs(g[plane_key]).max())
            if scale > 0:
                err = np.abs(mine - ref).max() / scale
                print(name, prec, key, "%.2e" % err)
                assert err <= tol, (key, err)
            else:
                assert np.abs(mine).max() == 0.0, key
            checked += 1
    assert checked == len([k for k in g.files if k.startswith(("yz_", "aux_"))])
    s.close()
