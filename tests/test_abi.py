"""C-ABI surface: the library loads without a GPU, exports every symbol the
public header declares, and its host-only entry points behave."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import fdtd_b200 as F
import oracle as O
from cases import CASES, make

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    text = open(os.path.join(ROOT, "include", "fdtd_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(fdtd_[a-z0-9_]+)\s*\(", text)))


def test_exports_every_declared_symbol():
    lib = F.lib()
    names = header_functions()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) <= set(F.EXPORTS) | set(names)


def test_params_layout_matches_library():
    assert F.lib().fdtd_params_size() == C.sizeof(F.Params)


def test_defaults_match_oracle():
    assert F.default_params().as_dict() == O.default_params().as_dict()


def test_input_txt_round_trip(tmp_path):
    import ref_cases
    for name, case in ref_cases.CASES.items():
        path = tmp_path / f"{name}.txt"
        path.write_text(ref_cases.deck(case))
        a = F.load_input_txt(str(path))
        b = O.load_input_txt(str(path))
        assert a.as_dict() == b.as_dict(), name
        for key, val in case.items():
            assert getattr(a, key) == pytest.approx(val), key
        out = tmp_path / f"{name}.out.txt"
        F.write_input_txt(str(out), a)
        assert F.load_input_txt(str(out)).as_dict() == a.as_dict()


def test_invalid_parameters_are_rejected_without_gpu():
    bad = make(F, "sphere_au", NUM_freq=1)
    with pytest.raises(F.FdtdError) as e:
        F.plan(bad)
    assert e.value.status == 1 and "NUM_freq" in str(e.value)
    with pytest.raises(F.FdtdError):
        F.Sim(make(F, "sphere_au", material=7))
    with pytest.raises(F.FdtdError):
        F.load_input_txt("/nonexistent/Input.txt")


def test_hydro_metal_on_boundary_rejected():
    p = make(F, "hydro", nano_sphere=0, inf_disp_slab=1, dispersive_slab=2)
    with pytest.raises(F.FdtdError) as e:
        F.plan(p)
    assert "boundary" in str(e.value)


@pytest.mark.parametrize("name", sorted(CASES))
def test_plan_matches_oracle(name):
    p = make(F, name)
    q = make(O, name)
    d = F.plan(p)
    od = O.OracleSim(q, dft=False).dims
    for f in ("nx", "ny", "nz", "ntfsf_x", "inc_length", "m0", "num_freq", "hydro"):
        assert getattr(d, f) == getattr(od, f), f
    assert list(d.abs_start) == list(od.abs_start)
    assert list(d.sca_end) == list(od.sca_end)
    assert list(d.n_metal_cells) == list(od.n_metal_cells)
    assert d.dt == od.dt and d.delay == od.delay and d.width == od.width


RUNNER = os.path.join(os.path.dirname(F.LIB_PATH), "fdtd_runner")


def test_runner_usage_and_errors_without_gpu(tmp_path):
    """fdtd_runner (the reference's program over the C ABI) is built next to
    the library; its usage and input errors need no GPU."""
    import subprocess
    assert os.access(RUNNER, os.X_OK)
    r = subprocess.run([RUNNER, "--help"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and "usage" in r.stderr
    r = subprocess.run([RUNNER, "--bogus"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 2
    r = subprocess.run([RUNNER, str(tmp_path / "missing.txt")], capture_output=True, text=True, timeout=60)
    assert r.returncode == 1 and "reading the input" in r.stderr
