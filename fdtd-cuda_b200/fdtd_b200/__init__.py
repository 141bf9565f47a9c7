"""Python binding of libfdtd_b200.so -- the B200-native FDTD time step.

The binding is a thin ctypes layer over the C ABI declared in
include/fdtd_b200.h.  Nothing here computes fields: every numeric call goes
to the CUDA library, and loading fails loudly if the library is missing.
"""
import ctypes as C
import os

import numpy as np

from ._abi import (FACE_COMPONENTS, FDTD_FP32, FDTD_FP64, FDTD_KERNEL_E_PASS,
                   FDTD_KERNEL_H_PASS, FIX_BH_X_F,
                   FIX_CE_EY_XN, FIX_HYDRO_CBRT, GEOM_DISK_ARRAY, GEOM_REFERENCE, GEOM_ROD_DIMER,
                   GEOM_SPHERE, STATUS, BatchTuning, Dims, Params, SnapshotLayout, Stats)

__all__ = ["Params", "Dims", "Sim", "Batch", "FdtdError", "lib", "default_params", "load_input_txt",
           "FDTD_FP32", "FDTD_FP64", "GEOM_REFERENCE", "GEOM_ROD_DIMER", "GEOM_DISK_ARRAY",
           "GEOM_SPHERE", "FIX_BH_X_F", "FIX_CE_EY_XN", "FIX_HYDRO_CBRT", "FACE_COMPONENTS",
           "FDTD_KERNEL_H_PASS", "FDTD_KERNEL_E_PASS"]

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libfdtd_b200.so")
_LIB = None

EXPORTS = [
    "fdtd_params_default", "fdtd_params_size", "fdtd_load_input_txt", "fdtd_write_input_txt",
    "fdtd_create", "fdtd_destroy", "fdtd_get_dims", "fdtd_reset", "fdtd_last_error",
    "fdtd_update_h", "fdtd_update_line", "fdtd_update_e", "fdtd_spectral_accumulate",
    "fdtd_step", "fdtd_run", "fdtd_get_time", "fdtd_check", "fdtd_spectral_finalize",
    "fdtd_write_scatabs", "fdtd_get_dft", "fdtd_get_freqs", "fdtd_get_incident",
    "fdtd_get_field", "fdtd_set_field", "fdtd_snapshot_plane", "fdtd_get_probe",
    "fdtd_get_material", "fdtd_set_design", "fdtd_forward", "fdtd_backward",
    "fdtd_batch_create", "fdtd_batch_run", "fdtd_batch_spectra", "fdtd_batch_destroy",
    "fdtd_batch_step", "fdtd_batch_sim", "fdtd_batch_get_stats",
    "fdtd_plan", "fdtd_rasterise", "fdtd_coefficients", "fdtd_get_probe_range",
    "fdtd_set_source", "fdtd_get_stats", "fdtd_time_kernel", "fdtd_forward_spectra",
    "fdtd_backward_spectra", "fdtd_snapshots_enable", "fdtd_snapshots_drain", "fdtd_batch_get_tuning",
    "fdtd_reflectance",
]


class FdtdError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status


def lib():
    """Load libfdtd_b200.so (raises if it has not been built)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with "
                          "`python fdtd-cuda_b200/fdtd_b200/build.py` (there is no CPU fallback)")
    L = C.CDLL(LIB_PATH)
    P = C.POINTER
    vp, dp, sz = C.c_void_p, P(C.c_double), C.c_size_t
    sig = {
        "fdtd_params_default": (None, [P(Params)]),
        "fdtd_params_size": (sz, []),
        "fdtd_load_input_txt": (C.c_int, [C.c_char_p, P(Params)]),
        "fdtd_write_input_txt": (C.c_int, [C.c_char_p, P(Params)]),
        "fdtd_create": (C.c_int, [P(Params), C.c_int, P(vp)]),
        "fdtd_destroy": (C.c_int, [vp]),
        "fdtd_get_dims": (C.c_int, [vp, P(Dims)]),
        "fdtd_reset": (C.c_int, [vp]),
        "fdtd_last_error": (C.c_char_p, []),
        "fdtd_update_h": (C.c_int, [vp, vp]),
        "fdtd_update_line": (C.c_int, [vp, vp]),
        "fdtd_update_e": (C.c_int, [vp, vp]),
        "fdtd_spectral_accumulate": (C.c_int, [vp, vp]),
        "fdtd_step": (C.c_int, [vp, C.c_int, vp]),
        "fdtd_run": (C.c_int, [vp, vp]),
        "fdtd_get_time": (C.c_int, [vp, P(C.c_int)]),
        "fdtd_check": (C.c_int, [vp]),
        "fdtd_spectral_finalize": (C.c_int, [vp, dp]),
        "fdtd_reflectance": (C.c_int, [vp, dp]),
        "fdtd_write_scatabs": (C.c_int, [vp, C.c_char_p]),
        "fdtd_get_dft": (C.c_int, [vp, C.c_int, C.c_int, C.c_int, dp, dp, sz]),
        "fdtd_get_freqs": (C.c_int, [vp, dp, sz]),
        "fdtd_get_incident": (C.c_int, [vp, dp, dp, sz]),
        "fdtd_get_field": (C.c_int, [vp, C.c_int, dp, sz]),
        "fdtd_set_field": (C.c_int, [vp, C.c_int, dp, sz]),
        "fdtd_snapshot_plane": (C.c_int, [vp, C.c_int, C.c_int, C.c_int, vp, sz, vp]),
        "fdtd_get_probe": (C.c_int, [vp, dp, sz, P(C.c_int)]),
        "fdtd_get_material": (C.c_int, [vp, P(C.c_ubyte), sz]),
        "fdtd_set_design": (C.c_int, [vp, P(C.c_int), P(C.c_float), sz]),
        "fdtd_forward": (C.c_int, [vp, P(C.c_int), C.c_int, C.c_int, dp]),
        "fdtd_backward": (C.c_int, [vp, P(C.c_float), sz, dp]),
        "fdtd_forward_spectra": (C.c_int, [vp, C.c_int, dp]),
        "fdtd_backward_spectra": (C.c_int, [vp, dp, P(C.c_float), sz, dp]),
        "fdtd_batch_create": (C.c_int, [P(Params), C.c_int, C.c_int, P(vp)]),
        "fdtd_batch_run": (C.c_int, [vp, vp]),
        "fdtd_batch_spectra": (C.c_int, [vp, C.c_int, dp]),
        "fdtd_batch_destroy": (C.c_int, [vp]),
        "fdtd_batch_step": (C.c_int, [vp, C.c_int, vp]),
        "fdtd_batch_sim": (C.c_int, [vp, C.c_int, P(vp)]),
        "fdtd_batch_get_stats": (C.c_int, [vp, P(C.c_longlong), P(C.c_longlong)]),
        "fdtd_plan": (C.c_int, [P(Params), P(Dims)]),
        "fdtd_rasterise": (C.c_int, [P(Params), P(C.c_ubyte), sz]),
        "fdtd_coefficients": (C.c_int, [P(Params), C.c_int, dp, sz, P(sz)]),
        "fdtd_get_probe_range": (C.c_int, [vp, C.c_int, C.c_int, vp, vp]),
        "fdtd_set_source": (C.c_int, [vp, C.c_int, C.c_int, vp, vp]),
        "fdtd_get_stats": (C.c_int, [vp, P(Stats)]),
        "fdtd_time_kernel": (C.c_int, [vp, C.c_int, C.c_int, vp, dp]),
        "fdtd_snapshots_enable": (C.c_int, [vp, C.c_int, C.c_int, P(SnapshotLayout)]),
        "fdtd_snapshots_drain": (C.c_int, [vp, vp, C.c_int, P(C.c_int), vp]),
        "fdtd_batch_get_tuning": (C.c_int, [vp, P(BatchTuning)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    if L.fdtd_params_size() != C.sizeof(Params):
        raise ImportError("fdtd_params layout mismatch between the library and _abi.py")
    _LIB = L
    return L


def _check(status):
    if status != 0:
        raise FdtdError(status, lib().fdtd_last_error().decode(errors="replace"))


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def default_params(**kw):
    p = Params()
    lib().fdtd_params_default(C.byref(p))
    p.update(**kw)
    return p


def load_input_txt(path, p=None):
    p = p or default_params()
    _check(lib().fdtd_load_input_txt(os.fsencode(path), C.byref(p)))
    return p


def plan(p):
    """Sizes fdtd_create would derive for these parameters (host only)."""
    d = Dims()
    _check(lib().fdtd_plan(C.byref(p), C.byref(d)))
    return d


def rasterise(p):
    """Dispersive-component bits per cell, reference layout (host only)."""
    d = plan(p)
    out = np.empty((d.nx, d.ny, d.nz), np.uint8)
    _check(lib().fdtd_rasterise(C.byref(p), out.ctypes.data_as(C.POINTER(C.c_ubyte)), out.size))
    return out


def coefficients(p, which):
    """One setup table (see fdtd_coefficients in include/fdtd_b200.h)."""
    buf = np.empty(1 << 16)
    n = C.c_size_t()
    _check(lib().fdtd_coefficients(C.byref(p), which, _dp(buf), buf.size, C.byref(n)))
    return buf[: n.value].copy()


def write_input_txt(path, p):
    _check(lib().fdtd_write_input_txt(os.fsencode(path), C.byref(p)))


class Sim:
    """One simulation on one GPU (the reference's whole program state)."""

    def __init__(self, params, device=0, _handle=None, _owner=None):
        if _handle is None:
            h = C.c_void_p()
            _check(lib().fdtd_create(C.byref(params), device, C.byref(h)))
        else:
            h = _handle  # a batch member: borrowed, the batch frees it
        self.h = h
        self._owner = _owner
        self.params = params
        d = Dims()
        _check(lib().fdtd_get_dims(self.h, C.byref(d)))
        self.dims = d
        self.shape = (d.nx, d.ny, d.nz)

    def close(self):
        if getattr(self, "h", None):
            if self._owner is None:
                lib().fdtd_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # -- stepping ------------------------------------------------------
    def step(self, n=1, stream=None):
        _check(lib().fdtd_step(self.h, int(n), stream))

    def run(self, stream=None):
        _check(lib().fdtd_run(self.h, stream))

    def update_h(self, stream=None):
        _check(lib().fdtd_update_h(self.h, stream))

    def update_line(self, stream=None):
        _check(lib().fdtd_update_line(self.h, stream))

    def update_e(self, stream=None):
        _check(lib().fdtd_update_e(self.h, stream))

    def spectral_accumulate(self, stream=None):
        _check(lib().fdtd_spectral_accumulate(self.h, stream))

    def reset(self):
        _check(lib().fdtd_reset(self.h))

    def check(self):
        _check(lib().fdtd_check(self.h))

    @property
    def t(self):
        v = C.c_int()
        _check(lib().fdtd_get_time(self.h, C.byref(v)))
        return v.value

    # -- outputs -------------------------------------------------------
    def field(self, comp):
        out = np.empty(self.shape, np.float64)
        _check(lib().fdtd_get_field(self.h, comp, _dp(out), out.size))
        return out

    def set_field(self, comp, arr):
        a = np.ascontiguousarray(arr, np.float64)
        _check(lib().fdtd_set_field(self.h, comp, _dp(a), a.size))

    def plane(self, comp, axis, index):
        na = self.shape[1] if axis == 0 else self.shape[0]
        nb = self.shape[1] if axis == 2 else self.shape[2]
        out = np.empty((na, nb), np.float64)
        _check(lib().fdtd_snapshot_plane(self.h, comp, axis, index, out.ctypes.data, out.size, None))
        return out

    def probe(self):
        n = C.c_int()
        out = np.empty((self.params.Tend + 2, 3))
        _check(lib().fdtd_get_probe(self.h, _dp(out), out.size, C.byref(n)))
        return out[: n.value]

    def probe_range(self, t0, n, out_ptr, stream=None):
        """Async D2H of probe rows [t0, t0+n) into host memory at out_ptr."""
        _check(lib().fdtd_get_probe_range(self.h, t0, n, out_ptr, stream))

    def set_source(self, t0, n, src_ptr, stream=None):
        """Async H2D of soft-source samples for steps [t0, t0+n)."""
        _check(lib().fdtd_set_source(self.h, t0, n, src_ptr, stream))

    def enable_snapshots(self, mode, capacity=64):
        """Snapshots taken by the stepper every t_skip steps
        (fdtd_snapshots_enable); mode is the reference's Snap_in (0 off)."""
        lay = SnapshotLayout()
        _check(lib().fdtd_snapshots_enable(self.h, int(mode), int(capacity), C.byref(lay)))
        self.snap_layout = lay
        return lay

    def drain_snapshots(self, max_records=None):
        """The records taken since the last drain, as dicts with t and the
        parts of the mode (plane, plane2, aux, line)."""
        lay = self.snap_layout
        m = lay.capacity if max_records is None else int(max_records)
        buf = np.empty((max(m, 1), lay.record))
        n = C.c_int()
        _check(lib().fdtd_snapshots_drain(self.h, buf.ctypes.data, m, C.byref(n), None))
        lib().fdtd_check(self.h)  # synchronising call: the copy has landed
        out = []
        for r in buf[: n.value]:
            d = {"t": int(r[0])}
            shp = (lay.plane_rows, lay.plane_cols)
            if lay.off_plane >= 0:
                d["plane"] = r[lay.off_plane:lay.off_plane + shp[0] * shp[1]].reshape(shp).copy()
            if lay.off_plane2 >= 0:
                d["plane2"] = r[lay.off_plane2:lay.off_plane2 + shp[0] * shp[1]].reshape(shp).copy()
            if lay.off_aux >= 0:
                d["aux"] = r[lay.off_aux:lay.off_aux + lay.aux_len].copy()
            if lay.off_line >= 0:
                d["line"] = r[lay.off_line:lay.off_line + lay.line_len].copy()
            out.append(d)
        return out

    def stats(self):
        st = Stats()
        _check(lib().fdtd_get_stats(self.h, C.byref(st)))
        return st

    # -- adjoint ---------------------------------------------------------
    def set_design(self, rho):
        """Blend per design-box cell (params.design_box), shape (nz, ny, nx)
        of the box, values in [0, 1]."""
        b = list(self.params.design_box)
        rho = np.ascontiguousarray(rho, dtype=np.float32)
        assert rho.shape == (b[5] - b[4], b[3] - b[2], b[1] - b[0]), rho.shape
        box = (C.c_int * 6)(*b)
        _check(lib().fdtd_set_design(self.h, box, rho.ctypes.data_as(C.POINTER(C.c_float)), rho.size))

    def forward(self, freq_idx, checkpoint_every=200):
        """Runs t = 0..Tend from zero fields with checkpoints; returns the
        objective: the absorption cross-section (m^2, positive for an
        absorbing structure) summed over freq_idx."""
        idx = (C.c_int * len(freq_idx))(*[int(x) for x in freq_idx])
        out = C.c_double()
        _check(lib().fdtd_forward(self.h, idx, len(freq_idx), int(checkpoint_every), C.byref(out)))
        return out.value

    def backward(self):
        """dL/drho (box shape) and dL/d(omega_D, gamma) of the last forward."""
        b = list(self.params.design_box)
        g = np.empty((b[5] - b[4], b[3] - b[2], b[1] - b[0]), np.float32)
        gp = np.empty(2)
        _check(lib().fdtd_backward(self.h, g.ctypes.data_as(C.POINTER(C.c_float)), g.size, _dp(gp)))
        return g, gp

    def forward_spectra(self, checkpoint_every=200):
        """Runs t = 0..Tend from zero fields with checkpoints; returns the
        ScatAbs table (NUM_freq x 19) of the run."""
        out = np.empty((self.dims.num_freq, 19))
        _check(lib().fdtd_forward_spectra(self.h, int(checkpoint_every), _dp(out)))
        return out

    def backward_spectra(self, dL_dspectra):
        """dL/drho (box shape) and dL/d(omega_D, gamma) of the last forward
        for the objective whose gradient with respect to the ScatAbs table
        is dL_dspectra (NUM_freq x 19; columns 0 and 16-18 zero)."""
        G = np.ascontiguousarray(dL_dspectra, dtype=np.float64)
        assert G.shape == (self.dims.num_freq, 19), G.shape
        b = list(self.params.design_box)
        g = np.empty((b[5] - b[4], b[3] - b[2], b[1] - b[0]), np.float32)
        gp = np.empty(2)
        _check(lib().fdtd_backward_spectra(self.h, _dp(G), g.ctypes.data_as(C.POINTER(C.c_float)), g.size,
                                           _dp(gp)))
        return g, gp

    def time_kernel(self, which, reps=20, stream=None):
        """Mean device time (ms) of one launch of a single time-step kernel
        (FDTD_KERNEL_*), from CUDA events; leaves the fields changed."""
        ms = C.c_double()
        _check(lib().fdtd_time_kernel(self.h, int(which), int(reps), stream, C.byref(ms)))
        return ms.value

    def material(self):
        out = np.empty(self.shape, np.uint8)
        _check(lib().fdtd_get_material(self.h, out.ctypes.data_as(C.POINTER(C.c_ubyte)), out.size))
        return out

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
        re = np.empty(shp)
        im = np.empty(shp)
        _check(lib().fdtd_get_dft(self.h, box, face, comp, _dp(re), _dp(im), re.size))
        return re + 1j * im

    def spectra(self):
        out = np.empty((self.dims.num_freq, 19))
        _check(lib().fdtd_spectral_finalize(self.h, _dp(out)))
        return out

    def reflectance(self):
        """Periodic simulations: (NUM_freq, 7) of lambda, R, T, 1 - R - T,
        |E_inc|, Re E_inc, Im E_inc (fdtd_reflectance)."""
        out = np.empty((self.dims.num_freq, 7))
        _check(lib().fdtd_reflectance(self.h, _dp(out)))
        return out

    def write_scatabs(self, path):
        _check(lib().fdtd_write_scatabs(self.h, os.fsencode(path)))

    def freqs(self):
        f = np.empty(self.dims.num_freq)
        _check(lib().fdtd_get_freqs(self.h, _dp(f), f.size))
        return f

    def incident(self):
        re = np.empty(self.dims.num_freq)
        im = np.empty(self.dims.num_freq)
        _check(lib().fdtd_get_incident(self.h, _dp(re), _dp(im), re.size))
        return re + 1j * im


class Batch:
    """Independent simulations advanced together (fdtd_batch_*): the Yee
    passes of all members share one persistent kernel per half step."""

    def __init__(self, params_list, device=0):
        self.params = list(params_list)
        arr = (Params * len(self.params))(*self.params)
        h = C.c_void_p()
        _check(lib().fdtd_batch_create(arr, len(self.params), device, C.byref(h)))
        self.h = h
        self.n = len(self.params)

    def step(self, n=1, stream=None):
        _check(lib().fdtd_batch_step(self.h, int(n), stream))

    def run(self, stream=None):
        _check(lib().fdtd_batch_run(self.h, stream))

    def sim(self, idx):
        """Member idx as a Sim view (borrowed: valid while the batch lives)."""
        h = C.c_void_p()
        _check(lib().fdtd_batch_sim(self.h, int(idx), C.byref(h)))
        return Sim(self.params[idx], _handle=h, _owner=self)

    def spectra(self, idx):
        d = self.sim(idx).dims
        out = np.empty((d.num_freq, 19))
        _check(lib().fdtd_batch_spectra(self.h, int(idx), _dp(out)))
        return out

    def stats(self):
        k, g = C.c_longlong(), C.c_longlong()
        _check(lib().fdtd_batch_get_stats(self.h, C.byref(k), C.byref(g)))
        return k.value, g.value

    def tuning(self):
        """The launch shapes the batch's autotuner chose (fdtd_batch_get_tuning)."""
        t = BatchTuning()
        _check(lib().fdtd_batch_get_tuning(self.h, C.byref(t)))
        nb = t.nbuckets
        return {"tuned": bool(t.tuned), "tile": [t.tile_x, t.tile_y],
                "buckets": [{"edges": [t.edge_lo[q], t.edge_hi[q] if t.edge_hi[q] < 2 ** 31 - 1 else None],
                             "members": t.members[q], "kchunk": t.kchunk[q],
                             "ms": round(float(t.bucket_ms[q]), 4)} for q in range(nb)],
                "minb": {"h": list(t.minb[0]), "e": list(t.minb[1])},
                "stages": {"h": list(t.stages[0]), "e": list(t.stages[1])}}

    def close(self):
        if getattr(self, "h", None):
            lib().fdtd_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
