"""ctypes wrapper of liboracle.so -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
import this module.  It is the checker (and the timed CPU baseline), never
part of the product path.
"""
import ctypes as C
import os
import subprocess
import sys

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(_HERE), "fdtd-cuda_b200"))
from fdtd_b200._abi import Dims, Params  # noqa: E402

_LIB = None


def build():
    subprocess.check_call(["make", "-s", "-C", _HERE])


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        P = C.POINTER
        L.orc_params_default.argtypes = [P(Params)]
        L.orc_load_input_txt.argtypes = [C.c_char_p, P(Params)]
        L.orc_create.argtypes = [P(Params), C.c_char_p]
        L.orc_create.restype = C.c_void_p
        L.orc_destroy.argtypes = [C.c_void_p]
        L.orc_set_design.argtypes = [C.c_void_p, C.POINTER(C.c_float), C.c_size_t]
        for f in ("orc_set_float_dft", "orc_set_dft_enabled"):
            getattr(L, f).argtypes = [C.c_void_p, C.c_int]
        L.orc_set_threads.argtypes = [C.c_int]
        L.orc_set_dft_freqs.argtypes = [C.c_void_p, C.POINTER(C.c_int), C.c_int]
        L.orc_step.argtypes = [C.c_void_p]
        L.orc_run.argtypes = [C.c_void_p, C.c_int]
        L.orc_time.argtypes = [C.c_void_p]
        L.orc_dims.argtypes = [C.c_void_p, P(Dims)]
        dp = P(C.c_double)
        L.orc_get_field.argtypes = [C.c_void_p, C.c_int, dp, C.c_size_t]
        L.orc_set_field.argtypes = [C.c_void_p, C.c_int, dp, C.c_size_t]
        L.orc_get_material.argtypes = [C.c_void_p, P(C.c_ubyte), P(C.c_int), P(C.c_int),
                                       P(C.c_int), C.c_size_t]
        L.orc_get_dft.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, dp, dp, C.c_size_t]
        L.orc_spectra.argtypes = [C.c_void_p, dp]
        L.orc_reflectance.argtypes = [C.c_void_p, dp]
        L.orc_get_freqs.argtypes = [C.c_void_p, dp, C.c_size_t]
        L.orc_get_incident.argtypes = [C.c_void_p, dp, dp, C.c_size_t]
        L.orc_get_line.argtypes = [C.c_void_p, dp, dp, C.c_size_t]
        L.orc_get_state.argtypes = [C.c_void_p, C.c_int, C.c_int, dp, C.c_size_t]
        L.orc_get_probe.argtypes = [C.c_void_p, dp, C.c_size_t]
        L.orc_get_cpml.argtypes = [C.c_void_p, C.c_int, dp, C.c_size_t]
        L.orc_get_ade.argtypes = [C.c_void_p, dp, C.c_size_t]
        _LIB = L
    return _LIB


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def default_params(**kw):
    p = Params()
    lib().orc_params_default(C.byref(p))
    p.update(**kw)
    return p


def load_input_txt(path, p=None):
    p = p or default_params()
    rc = lib().orc_load_input_txt(path.encode(), C.byref(p))
    if rc != 0:
        raise IOError(f"oracle could not read {path} ({rc})")
    return p


class OracleSim:
    def __init__(self, params, float_dft=False, dft=True, threads=0):
        err = C.create_string_buffer(256)
        if threads:
            lib().orc_set_threads(threads)
        self.h = lib().orc_create(C.byref(params), err)
        if not self.h:
            raise ValueError(err.value.decode())
        self.params = params
        lib().orc_set_float_dft(self.h, int(float_dft))
        lib().orc_set_dft_enabled(self.h, int(dft))
        d = Dims()
        lib().orc_dims(self.h, C.byref(d))
        self.dims = d
        self.shape = (d.nx, d.ny, d.nz)

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_destroy(self.h)
            self.h = None

    def set_dft_freqs(self, idx):
        """Accumulate the DFT at these frequency indices only."""
        arr = (C.c_int * len(idx))(*[int(x) for x in idx])
        assert lib().orc_set_dft_freqs(self.h, arr, len(idx)) == 0

    def step(self, n=1):
        lib().orc_run(self.h, n)

    @property
    def t(self):
        return lib().orc_time(self.h)

    def field(self, comp):
        out = np.empty(self.shape, np.float64)
        assert lib().orc_get_field(self.h, comp, _dp(out), out.size) == 0
        return out

    def set_field(self, comp, arr):
        a = np.ascontiguousarray(arr, np.float64)
        assert lib().orc_set_field(self.h, comp, _dp(a), a.size) == 0

    def material(self):
        n = int(np.prod(self.shape))
        bits = np.empty(self.shape, np.uint8)
        mx, my, mz = (np.empty(self.shape, np.int32) for _ in range(3))
        ip = C.POINTER(C.c_int)
        lib().orc_get_material(self.h, bits.ctypes.data_as(C.POINTER(C.c_ubyte)),
                               mx.ctypes.data_as(ip), my.ctypes.data_as(ip),
                               mz.ctypes.data_as(ip), n)
        return bits, (mx, my, mz)

    def dft_shape(self, box, face):
        d = self.dims
        if self.params.periodic_xy:  # the reflection (0) and transmission (1) planes
            return (d.num_freq, d.nx + 1, d.ny + 1)
        S = d.abs_start if box == 0 else d.sca_start
        E = d.abs_end if box == 0 else d.sca_end
        ax = face // 2
        a1 = 1 if ax == 0 else 0
        a2 = 1 if ax == 2 else 2
        return (d.num_freq, E[a1] - S[a1] + 1, E[a2] - S[a2] + 1)

    def dft(self, box, face, comp):
        shp = self.dft_shape(box, face)
        re = np.empty(shp, np.float64)
        im = np.empty(shp, np.float64)
        rc = lib().orc_get_dft(self.h, box, face, comp, _dp(re), _dp(im), re.size)
        if rc != 0:
            raise RuntimeError("no DFT data")
        return re + 1j * im

    def set_design(self, rho):
        """Blend per cell of params.design_box, shape (nz, ny, nx) of the box."""
        rho = np.ascontiguousarray(rho, dtype=np.float32)
        assert lib().orc_set_design(self.h, rho.ctypes.data_as(C.POINTER(C.c_float)), rho.size) == 0

    def spectra(self):
        out = np.empty((self.dims.num_freq, 19), np.float64)
        if lib().orc_spectra(self.h, _dp(out)) != 0:
            raise RuntimeError("no DFT data")
        return out

    def reflectance(self):
        """periodic_xy: (NUM_freq, 7) of lambda, R, T, 1 - R - T, |E_inc|,
        Re E_inc, Im E_inc."""
        out = np.empty((self.dims.num_freq, 7), np.float64)
        if lib().orc_reflectance(self.h, _dp(out)) != 0:
            raise RuntimeError("not a periodic simulation")
        return out

    def freqs(self):
        f = np.empty(self.dims.num_freq)
        lib().orc_get_freqs(self.h, _dp(f), f.size)
        return f

    def incident(self):
        re = np.empty(self.dims.num_freq)
        im = np.empty(self.dims.num_freq)
        lib().orc_get_incident(self.h, _dp(re), _dp(im), re.size)
        return re + 1j * im

    def line(self):
        e = np.empty(self.dims.inc_length)
        h = np.empty(self.dims.inc_length)
        lib().orc_get_line(self.h, _dp(e), _dp(h), e.size)
        return e, h

    def state(self, which, comp):
        """Dispersive state in the reference layout (see orc_get_state)."""
        out = np.empty(self.shape, np.float64)
        assert lib().orc_get_state(self.h, which, comp, _dp(out), out.size) == 0
        return out

    def probe(self):
        out = np.empty((self.t, 3))
        n = lib().orc_get_probe(self.h, _dp(out), out.size)
        return out[:n]

    def cpml(self, which):
        out = np.empty(4096)
        n = lib().orc_get_cpml(self.h, which, _dp(out), out.size)
        return out[:n].copy()

    def ade(self):
        out = np.empty(22)
        lib().orc_get_ade(self.h, _dp(out), 22)
        return out
