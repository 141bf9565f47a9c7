"""ctypes mirror of the plain-C structs in include/fdtd_b200.h.

The field order here must match the header exactly; tests check the struct
size against the library's own ``fdtd_params_size()``.
"""
import ctypes as C

_PARAM_FIELDS = [
    # Input.txt, in file order (setup.cu:17-58)
    ("Tend", C.c_int), ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double),
    ("num_trials", C.c_int), ("min_trials", C.c_int), ("max_trials", C.c_int),
    ("TE_TM", C.c_int),
    ("NCELLX", C.c_int), ("NCELLY", C.c_int), ("NCELLZ", C.c_int),
    ("NcpmlX", C.c_int), ("NcpmlY", C.c_int), ("NcpmlZ", C.c_int),
    ("inf_disp_slab", C.c_int), ("nano_sphere", C.c_int),
    ("nano_sphere_radius", C.c_double), ("material", C.c_int),
    ("first_medium", C.c_int), ("inc_plane", C.c_int), ("dispersive_slab", C.c_int),
    ("NUM_freq", C.c_int), ("WL_or_freq", C.c_int), ("NUM_freq_inc", C.c_int),
    ("Tend_inc", C.c_int), ("Snap_in", C.c_int), ("Freq_start", C.c_int),
    ("Test_offset", C.c_int), ("Spect_loc", C.c_int), ("BandWidth", C.c_double),
    ("NONLOCAL", C.c_int), ("Diverge_Gradient", C.c_int),
    ("t_skip", C.c_int), ("x_skip", C.c_int), ("y_skip", C.c_int), ("z_skip", C.c_int),
    ("Nonlocalend", C.c_double), ("MAX_AMP", C.c_double), ("TimeFactor", C.c_double),
    ("lam_0", C.c_double), ("StaticField", C.c_int),
    # constants the reference hard-codes
    ("tfsf_inset", C.c_int), ("box_offset", C.c_int), ("cpml_order", C.c_int),
    ("cpml_kappa_max", C.c_double), ("cpml_alpha_max", C.c_double),
    ("cpml_sigma_factor", C.c_double), ("lam_min", C.c_double), ("lam_max", C.c_double),
    ("inc_theta_deg", C.c_double), ("inc_phi_deg", C.c_double), ("polar_psi_deg", C.c_double),
    ("source_offset", C.c_int), ("dft_every", C.c_int), ("hydro_D", C.c_double),
    ("fermi_velocity", C.c_double), ("precision", C.c_int), ("fixes", C.c_int),
    # material overrides
    ("metal_custom", C.c_int), ("eps_inf", C.c_double), ("omega_D", C.c_double),
    ("gamma_D", C.c_double), ("cp_A", C.c_double * 2), ("cp_phi", C.c_double * 2),
    ("cp_Omega", C.c_double * 2), ("cp_Gamma", C.c_double * 2), ("N_EQ", C.c_double),
    # extended geometry
    ("geometry", C.c_int), ("axis", C.c_int), ("rod_length", C.c_double),
    ("rod_diameter", C.c_double), ("gap", C.c_double), ("disk_diameter", C.c_double),
    ("disk_height", C.c_double), ("pitch", C.c_double), ("disk_nx", C.c_int),
    ("disk_ny", C.c_int), ("slab_eps", C.c_double), ("slab_thickness", C.c_double),
    ("sphere_radius", C.c_double), ("sphere_cx", C.c_double), ("sphere_cy", C.c_double),
    ("sphere_cz", C.c_double),
    # probe
    ("probe_i", C.c_int), ("probe_j", C.c_int), ("probe_k", C.c_int),
    # adjoint design region
    ("design_box", C.c_int * 6),
    # periodic x and y
    ("periodic_xy", C.c_int),
]


class Params(C.Structure):
    _fields_ = _PARAM_FIELDS

    def update(self, **kw):
        for k, v in kw.items():
            if not hasattr(self, k):
                raise AttributeError(f"fdtd_params has no field {k!r}")
            cur = getattr(self, k)
            if isinstance(cur, C.Array):
                for q, x in enumerate(v):
                    cur[q] = x
            else:
                setattr(self, k, v)
        return self

    def as_dict(self):
        out = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            out[name] = list(v) if isinstance(v, C.Array) else v
        return out


class Dims(C.Structure):
    _fields_ = [
        ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("ntfsf_x", C.c_int), ("ntfsf_y", C.c_int), ("ntfsf_z", C.c_int),
        ("inc_length", C.c_int), ("m0", C.c_int),
        ("abs_start", C.c_int * 3), ("abs_end", C.c_int * 3),
        ("sca_start", C.c_int * 3), ("sca_end", C.c_int * 3),
        ("num_freq", C.c_int), ("n_metal_cells", C.c_int * 3), ("hydro", C.c_int),
        ("precision", C.c_int), ("dt", C.c_double), ("delay", C.c_double),
        ("width", C.c_double),
    ]


FDTD_FP32, FDTD_FP64 = 0, 1
FDTD_KERNEL_H_PASS, FDTD_KERNEL_E_PASS = 0, 1
GEOM_REFERENCE, GEOM_ROD_DIMER, GEOM_DISK_ARRAY, GEOM_SPHERE = 0, 1, 2, 3
FIX_BH_X_F, FIX_CE_EY_XN, FIX_HYDRO_CBRT = 1, 2, 4
STATUS = {0: "OK", 1: "INVALID", 2: "CUDA", 3: "ALLOC", 4: "IO", 5: "STATE",
          6: "NONFINITE", 7: "TIMEOUT", 8: "UNSUPPORTED"}

# the face component order of the DFT arrays (see fdtd_get_dft)
FACE_COMPONENTS = {0: (1, 2, 4, 5), 1: (0, 2, 3, 5), 2: (0, 1, 3, 4)}


class Stats(C.Structure):
    _fields_ = [("kernels", C.c_longlong), ("steps", C.c_longlong),
                ("graph_launches", C.c_longlong),
                ("h_minb", C.c_int), ("h_ty", C.c_int), ("h_kchunk", C.c_int),
                ("e_minb", C.c_int), ("e_ty", C.c_int), ("e_kchunk", C.c_int),
                ("h_ms", C.c_float), ("e_ms", C.c_float),
                ("h_staged", C.c_int), ("e_staged", C.c_int),
                ("h_stages", C.c_int), ("e_stages", C.c_int),
                ("h_eminb", C.c_int), ("h_estages", C.c_int),
                ("e_eminb", C.c_int), ("e_estages", C.c_int),
                ("h_pdl", C.c_int), ("e_pdl", C.c_int),
                ("tfsf_entries_h", C.c_longlong), ("tfsf_entries_e", C.c_longlong),
                ("dft_rows", C.c_longlong),
                ("adj_record_steps", C.c_longlong), ("adj_record_bytes", C.c_longlong),
                ("adj_checkpoints", C.c_longlong),
                ("h_tma", C.c_int), ("h_etma", C.c_int), ("e_tma", C.c_int), ("e_etma", C.c_int)]


class SnapshotLayout(C.Structure):
    """fdtd_snapshot_layout (include/fdtd_b200.h)."""
    _fields_ = [("mode", C.c_int), ("t_skip", C.c_int), ("plane_rows", C.c_int), ("plane_cols", C.c_int),
                ("aux_len", C.c_int), ("line_len", C.c_int), ("off_plane", C.c_int), ("off_plane2", C.c_int),
                ("off_aux", C.c_int), ("off_line", C.c_int), ("record", C.c_int), ("capacity", C.c_int)]


class BatchTuning(C.Structure):
    """fdtd_batch_tuning (include/fdtd_b200.h)."""
    _fields_ = [("tuned", C.c_int), ("nbuckets", C.c_int), ("edge_lo", C.c_int * 16), ("edge_hi", C.c_int * 16),
                ("members", C.c_int * 16), ("kchunk", C.c_int * 16), ("bucket_ms", C.c_float * 16),
                ("tile_x", C.c_int), ("tile_y", C.c_int), ("minb", (C.c_int * 2) * 2),
                ("stages", (C.c_int * 2) * 2)]
