"""fdtd_snapshot_plane_static -- the plane snapshot that allocates nothing --
against the allocating fdtd_snapshot_plane, both called through the C-ABI.

The file name sorts last, so in a full run this test also runs after every
other GPU test (the scratch array lives in the library's static device
memory for the life of the process); it passes when run alone too.
"""
import ctypes as C

import numpy as np
import pytest

import fdtd_b200 as F
from cases import make

pytestmark = pytest.mark.gpu

MAX_CELLS = 1 << 20  # the scratch limit stated in include/fdtd_b200.h


def _fn(name):
    f = getattr(F.lib(), name)
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_size_t, C.c_void_p]
    return f


def _last_error():
    f = F.lib().fdtd_last_error
    f.restype = C.c_char_p
    return f().decode()


def _plane_shape(shape, axis):
    nx, ny, nz = shape
    return (ny if axis == 0 else nx, ny if axis == 2 else nz)


@pytest.mark.parametrize("prec", [F.FDTD_FP32, F.FDTD_FP64])
def test_static_plane_matches_allocating_plane(prec):
    alloc, static = _fn("fdtd_snapshot_plane"), _fn("fdtd_snapshot_plane_static")
    s = F.Sim(make(F, "sphere_au", precision=prec))
    s.step(120)
    nx, ny, nz = s.shape
    for call in range(2):  # two calls in a row, the fields moving in between
        for comp in (1, 3, 5):
            for axis, index in ((0, nx // 2), (1, 5), (2, nz - 3)):
                a = np.empty(_plane_shape(s.shape, axis))
                b = np.full_like(a, np.nan)
                assert alloc(s.h, comp, axis, index, a.ctypes.data, a.size, None) == 0
                assert static(s.h, comp, axis, index, b.ctypes.data, b.size, None) == 0, _last_error()
                # the same gather of the same values: tolerance zero
                np.testing.assert_allclose(b, a, rtol=0, atol=0)
                assert np.abs(a).max() > 0 or comp == 5
        s.step(3)
    s.close()


def test_static_plane_into_device_memory():
    import torch
    static = _fn("fdtd_snapshot_plane_static")
    s = F.Sim(make(F, "sphere_au", precision=F.FDTD_FP32))
    s.step(100)
    want = s.plane(1, 2, 17)
    got = torch.full(want.shape, float("nan"), dtype=torch.float64, device="cuda")
    st = torch.cuda.current_stream()
    assert static(s.h, 1, 2, 17, got.data_ptr(), got.numel(), st.cuda_stream) == 0, _last_error()
    np.testing.assert_array_equal(got.cpu().numpy(), want)
    s.close()


def test_static_plane_rejects_planes_beyond_the_scratch():
    static = _fn("fdtd_snapshot_plane_static")
    # 1043 x 1043 x 34 cells: the z-normal plane holds 1,087,849 > 2^20 cells
    s = F.Sim(make(F, "vacuum", NCELLX=1030, NCELLY=1030, NUM_freq=3, precision=F.FDTD_FP32))
    nx, ny, nz = s.shape
    assert nx * ny > MAX_CELLS
    s.step(2)
    big = np.empty(_plane_shape(s.shape, 2))
    status = static(s.h, 0, 2, nz // 2, big.ctypes.data, big.size, None)
    assert status == 1  # FDTD_ERR_INVALID
    assert "scratch" in _last_error()
    # a plane within the limit still works on the same simulation
    small = np.full(_plane_shape(s.shape, 0), np.nan)
    assert static(s.h, 0, 0, nx // 2, small.ctypes.data, small.size, None) == 0, _last_error()
    np.testing.assert_array_equal(small, s.plane(0, 0, nx // 2))
    s.close()
