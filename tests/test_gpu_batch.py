"""Batched simulations (fdtd_batch_*) against the same members run one at a
time through fdtd_step: the batch changes scheduling only, so fields,
probes and spectra agree to rounding."""
import numpy as np
import pytest

import fdtd_b200 as F
from cases import make

pytestmark = pytest.mark.gpu

MEMBERS = [("sphere_au", {}), ("vacuum", dict(NCELLX=27, NCELLY=23, NCELLZ=19)),
           ("sphere_au", dict(NCELLX=31, NCELLY=31, NCELLZ=37, nano_sphere_radius=10e-9)),
           ("cube_ag", {})]


def rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def family_errors(sa, sb):
    """Max error of E and of H, each relative to its family's peak."""
    out = []
    for fam in ((0, 1, 2), (3, 4, 5)):
        a = [sa.field(c) for c in fam]
        b = [sb.field(c) for c in fam]
        scale = max(np.abs(x).max() for x in b)
        out.append(max(float(np.abs(x - y).max()) for x, y in zip(a, b)) / scale)
    return out


@pytest.mark.parametrize("prec", [F.FDTD_FP32, F.FDTD_FP64])
def test_batch_matches_sequential(prec):
    """Bit-identical: the batched passes run the same per-cell arithmetic
    (fixed-rounding operations, so neither the tile shape nor the CPML-free
    or CPML-edge instantiation changes a result), and every other kernel of
    the step is the same body launched over all members."""
    params = [make(F, name, precision=prec, **over) for name, over in MEMBERS]
    steps = 300  # two graph periods of 128 plus an eager tail
    b = F.Batch(params)
    b.step(steps)
    for i, p in enumerate(params):
        alone = F.Sim(p)
        alone.step(steps)
        m = b.sim(i)
        assert m.t == alone.t == steps
        for c in range(6):
            np.testing.assert_array_equal(m.field(c), alone.field(c), err_msg=f"member {i} component {c}")
        np.testing.assert_array_equal(m.probe(), alone.probe())
        np.testing.assert_array_equal(b.spectra(i), alone.spectra())
        alone.close()
    kernels, graphs = b.stats()
    assert graphs == 2 and kernels > 0
    b.close()


def test_batch_launches_do_not_grow_with_members():
    one = F.Batch([make(F, "sphere_au", precision=F.FDTD_FP32)])
    four = F.Batch([make(F, "sphere_au", precision=F.FDTD_FP32) for _ in range(4)])
    one.step(5)
    four.step(5)
    assert one.stats()[0] == four.stats()[0]
    one.close()
    four.close()


def test_batch_member_spectra_read_mid_run():
    """Reading one member's spectra empties its sample ring only; the batch's
    contraction launches then find the members' rings at different fill
    levels, and each member contracts before its ring could overflow."""
    params = [make(F, "sphere_au", precision=F.FDTD_FP64) for _ in range(2)]
    b = F.Batch(params)
    b.step(150)
    b.spectra(0)
    b.step(270)
    alone = F.Sim(params[0])
    alone.step(420)
    ref = alone.spectra()
    for i in (0, 1):
        assert rel(b.spectra(i)[:, 1:4], ref[:, 1:4]) < 1e-12, i
    alone.close()
    b.close()


def test_batch_hydro_members():
    params = [make(F, "hydro", precision=F.FDTD_FP64),
              make(F, "hydro", precision=F.FDTD_FP64, NCELLX=25, nano_sphere_radius=8e-9)]
    b = F.Batch(params)
    b.step(150)
    for i, p in enumerate(params):
        alone = F.Sim(p)
        alone.step(150)
        assert max(family_errors(b.sim(i), alone)) < 1e-12
        alone.close()
    b.close()


def test_batch_rejects_mixed_members():
    with pytest.raises(F.FdtdError) as e:
        F.Batch([make(F, "sphere_au", precision=F.FDTD_FP32),
                 make(F, "sphere_au", precision=F.FDTD_FP32, Tend=500)])
    assert e.value.status == 1 and "Tend" in str(e.value)


def test_tuned_batch_is_bit_identical_and_reports_its_shapes():
    """Members of three size buckets, 2^21 cells in all: the autotuner
    picks a z-chunk per bucket and a variant per launch; the result stays
    bit-identical to the members run alone."""
    sizes = [(84, 76, 80), (60, 60, 60), (44, 44, 44)]
    params = [make(F, "sphere_big", precision=F.FDTD_FP32, NCELLX=x, NCELLY=y, NCELLZ=z) for x, y, z in sizes]
    b = F.Batch(params)
    tu = b.tuning()
    print(tu)
    assert tu["tuned"] and tu["tile"] == [32, 4]
    assert sum(q["members"] for q in tu["buckets"]) == len(params) and len(tu["buckets"]) == 3
    assert all(q["kchunk"] in (8, 16, 32) and q["ms"] > 0 for q in tu["buckets"])
    steps = 140
    b.step(steps)
    for i, p in enumerate(params):
        alone = F.Sim(p)
        alone.step(steps)
        for c in range(6):
            np.testing.assert_array_equal(b.sim(i).field(c), alone.field(c), err_msg=f"member {i} component {c}")
        alone.close()
    b.close()
