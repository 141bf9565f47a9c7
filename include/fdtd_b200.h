/*
 * fdtd_b200.h -- C ABI of the B200-native FDTD time-step loop.
 *
 * The reference (jbaxt089/FDTD-CUDA) is a monolithic main() over ~700
 * globals.  This ABI exposes its entry points as functions on an opaque
 * simulation handle.  Every function returns an fdtd_status, never exits,
 * and keeps its error text for fdtd_last_error().  Plain C types only: no
 * torch or CUDA-runtime types appear in the signatures (streams are passed
 * as void* cudaStream_t).
 *
 * Reference entry point                        replaced by
 * -------------------------------------------  -----------------------------
 * READ_DATA_FILE        setup.cu:10-133        fdtd_load_input_txt
 * SETUP_CONST           setup.cu:347-510       fdtd_create (derived sizes)
 * MATERIAL_MATRIX       setup.cu:135-342       fdtd_create (rasteriser)
 * SETUP_Drude_CP        setup.cu:979-1558      fdtd_create (ADE tables)
 * SETUP_CPML            setup.cu:513-978       fdtd_create (CPML tables)
 * SETUP_TFSF            tfsf2.cu:6-56          fdtd_create (pulse, line)
 * DEF_UPDATE_COEFF_*    setup.cu:2015-2062     fdtd_create (Yee tables)
 * UPDATE_hx/hy/hz       main.cu:762-1044       fdtd_update_h
 * CORRECT_X/Y/Z         main.cu:369-758        fused into update_h/update_e
 * UPDATE_h_inc/e_inc    main.cu:2280-2337      fdtd_update_line
 * host Mur + source     main.cu:2831-2859      fdtd_update_line (on device)
 * UpdateHydroPx/Py/Pz   main.cu:1916-2276      fdtd_update_e (metal pass)
 * UPDATE_ex/ey/ez       main.cu:1048-1912      fdtd_update_e
 * ScattAbs              main.cu:35-366         fdtd_spectral_accumulate
 * CalculateAbsScatt     Spectral.cu:411-1177   fdtd_spectral_finalize
 * SNAPSHOT_*            snapshot.cu:10-180     fdtd_get_field / fdtd_probe_*
 * time loop             main.cu:2724-3175      fdtd_step
 */
#ifndef FDTD_B200_H
#define FDTD_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum fdtd_status {
  FDTD_OK = 0,
  FDTD_ERR_INVALID = 1,     /* bad argument or parameter combination */
  FDTD_ERR_CUDA = 2,        /* a CUDA runtime call failed */
  FDTD_ERR_ALLOC = 3,       /* device allocation failed or over the cap */
  FDTD_ERR_IO = 4,          /* Input.txt / output file problem */
  FDTD_ERR_STATE = 5,       /* call out of order (e.g. finalize before run) */
  FDTD_ERR_NONFINITE = 6,   /* watchdog saw NaN/Inf in the fields */
  FDTD_ERR_TIMEOUT = 7,     /* a bounded device wait gave up */
  FDTD_ERR_UNSUPPORTED = 8  /* feature outside the supported set */
} fdtd_status;

/* Arithmetic type of the fields (the reference's compile-time
 * DOUBLEPRECISION / FlOATPRECISION switch, define.h:7, global_var.h:15). */
typedef enum fdtd_precision { FDTD_FP32 = 0, FDTD_FP64 = 1 } fdtd_precision;

/* Geometry kinds.  FDTD_GEOM_REFERENCE rasterises exactly what
 * MATERIAL_MATRIX does from the Input.txt fields inf_disp_slab /
 * nano_sphere / nano_sphere_radius (setup.cu:135-342).  The others are
 * shapes the reference cannot express. */
typedef enum fdtd_geometry {
  FDTD_GEOM_REFERENCE = 0,
  FDTD_GEOM_ROD_DIMER = 1,   /* two capped rods along an axis with a gap */
  FDTD_GEOM_DISK_ARRAY = 2,  /* nx*ny disks on a dielectric slab */
  FDTD_GEOM_SPHERE = 3       /* sphere of real radius at a real centre */
} fdtd_geometry;

/* Field components, in the reference's naming. */
typedef enum fdtd_component {
  FDTD_EX = 0, FDTD_EY = 1, FDTD_EZ = 2, FDTD_HX = 3, FDTD_HY = 4, FDTD_HZ = 5
} fdtd_component;

/* Behaviours of the reference that are reproduced by default so results
 * match it bit-for-bit in structure.  Setting a bit switches to the
 * physically intended behaviour instead. */
enum fdtd_fix_bits {
  /* setup.cu:681 uploads bh_z_F (not yet computed, SETUP_CPML_X runs before
   * SETUP_CPML_Z) as bh_x_F; the reference therefore runs with bh_x_F = 0. */
  FDTD_FIX_BH_X_F = 1 << 0,
  /* main.cu:2891 passes ce_y_N where UPDATE_ey expects ce_x_N. */
  FDTD_FIX_CE_EY_XN = 1 << 1,
  /* UpdateHydroP* take the cube root with powf (FP32) even in FP64 builds
   * (main.cu:2035); the fix uses the working precision. */
  FDTD_FIX_HYDRO_CBRT = 1 << 2
};

/*
 * Parameters.  The first block mirrors the 41 positional Input.txt values in
 * file order (setup.cu:17-58).  NCELLX/Y/Z and NcpmlX/Y/Z are the raw file
 * values; the grid actually allocated is N + 2*Ncpml + 1 per axis
 * (setup.cu:377-393).  The second block turns the reference's hard-coded
 * constants into parameters; fdtd_params_default() sets them to the
 * reference's values.
 */
typedef struct fdtd_params {
  /* ---- Input.txt (setup.cu:17-58) ---- */
  int Tend;
  double dx, dy, dz;
  int num_trials, min_trials, max_trials;
  int TE_TM;
  int NCELLX, NCELLY, NCELLZ;
  int NcpmlX, NcpmlY, NcpmlZ;
  int inf_disp_slab;
  int nano_sphere;
  double nano_sphere_radius;
  int material;           /* 2 = silver, 3 = gold (setup.cu:1164-1211) */
  int first_medium;
  int inc_plane;
  int dispersive_slab;
  int NUM_freq;
  int WL_or_freq;         /* 1 = wavelength grid, else frequency grid */
  int NUM_freq_inc;
  int Tend_inc;
  int Snap_in;
  int Freq_start;
  int Test_offset;
  int Spect_loc;
  double BandWidth;
  int NONLOCAL;           /* 3 = hydrodynamic nonlocal model */
  int Diverge_Gradient;
  int t_skip, x_skip, y_skip, z_skip;
  double Nonlocalend;
  double MAX_AMP;
  double TimeFactor;
  double lam_0;
  int StaticField;

  /* ---- constants hard-coded in the reference ---- */
  int tfsf_inset;          /* 10       setup.cu:428 */
  int box_offset;          /* 5        setup.cu:435-452 (DFT boxes) */
  int cpml_order;          /* 3        setup.cu:481 */
  double cpml_kappa_max;   /* 5        setup.cu:482 */
  double cpml_alpha_max;   /* 0.05     setup.cu:485 */
  double cpml_sigma_factor;/* 0.8      setup.cu:483 (sigma_max=f(m+1)/(Z0 dx)) */
  double lam_min, lam_max; /* 200e-9 / 700e-9   main.cu:2446-2447 */
  double inc_theta_deg;    /* 0        tfsf2.cu:11-13 */
  double inc_phi_deg;      /* 0  (E along -y); 90 gives E along +x */
  double polar_psi_deg;    /* 0        main.cu:2424-2426 */
  int source_offset;       /* 50       main.cu:2851 (source at m0-50) */
  int dft_every;           /* 4        main.cu:2920 */
  double hydro_D;          /* 2        setup.cu:981 (beta^2 = 3/(D+2) vF^2) */
  double fermi_velocity;   /* 1.39e6   setup.cu:980 */
  int precision;           /* fdtd_precision */
  int fixes;               /* fdtd_fix_bits */

  /* ---- material overrides (0 = use the table for `material`) ---- */
  int metal_custom;
  double eps_inf, omega_D, gamma_D;
  double cp_A[2], cp_phi[2], cp_Omega[2], cp_Gamma[2];
  double N_EQ;             /* hydro equilibrium density */

  /* ---- extended geometry (FDTD_GEOM_*) ---- */
  int geometry;
  int axis;                /* rod axis / dimer axis: 0=x 1=y 2=z */
  double rod_length, rod_diameter, gap;
  double disk_diameter, disk_height, pitch;
  int disk_nx, disk_ny;
  double slab_eps, slab_thickness;
  double sphere_radius, sphere_cx, sphere_cy, sphere_cz; /* metres, cells */

  /* ---- probes ---- */
  int probe_i, probe_j, probe_k; /* -1 = grid centre (OUT.txt, main.cu:2732) */

  /* ---- adjoint design region (no counterpart in the reference) ---- */
  /* [i0, i1) x [j0, j1) x [k0, k1) in grid cells; empty (i1 <= i0) = none.
   * Its cells are dispersive (class `material`) for all three components;
   * fdtd_set_design blends each cell's ADE coefficients between vacuum and
   * the metal.  It must lie inside the absorption box, off the CPML. */
  int design_box[6];

  /* ---- periodic x and y (the reference's Periodic_XY path) ---- */
  /* 1 = the lateral boundaries are periodic, as in the reference's
   * Periodic_XY branches (main.cu:781-1912, real fields: no Bloch phase),
   * which its main() switches off (main.cu:2398).  The grid is NX = NCELLX,
   * NY = NCELLY (setup.cu:401-404), NZ = NCELLZ + 2 NcpmlZ + 1; NcpmlX and
   * NcpmlY must be 0 (CPML in z only), NX a multiple of 8.  The plane wave
   * enters through the lower z face of the TFSF box only (main.cu:698); the
   * spectra are the reflectance and transmittance of two xy planes
   * (Fourier_Transform, Spectral.cu:8-120, and Reflectance_XZ,
   * main.cu:3195-3320): fdtd_reflectance.  No design region, hydrodynamic
   * model or batch membership. */
  int periodic_xy;
} fdtd_params;

typedef struct fdtd_sim fdtd_sim;   /* opaque */

/* Sizes derived by setup, for callers that allocate host buffers. */
typedef struct fdtd_dims {
  int nx, ny, nz;          /* allocated grid (N + 2*Ncpml + 1) */
  int ntfsf_x, ntfsf_y, ntfsf_z;
  int inc_length, m0;
  int abs_start[3], abs_end[3], sca_start[3], sca_end[3];
  int num_freq;
  int n_metal_cells[3];    /* ex/ey/ez cells with a dispersive update */
  int hydro;               /* 1 when the hydrodynamic model is active */
  int precision;
  double dt;
  double delay, width;     /* pulse, in steps (tfsf2.cu:37-40) */
} fdtd_dims;

/* ---------------------------------------------------------------------- */
/* parameters                                                              */

/* Reference defaults for every field (Input.txt fields zeroed). */
void fdtd_params_default(fdtd_params* p);
/* sizeof(fdtd_params) as compiled into the library (ABI check). */
size_t fdtd_params_size(void);

/* READ_DATA_FILE (setup.cu:10-133): reads the 41 positional values of an
 * Input.txt into *p, leaving the other fields untouched. */
fdtd_status fdtd_load_input_txt(const char* path, fdtd_params* p);

/* Writes *p as an Input.txt the reference can read. */
fdtd_status fdtd_write_input_txt(const char* path, const fdtd_params* p);

/* Host-only queries (no GPU needed): the sizes fdtd_create would derive,
 * the material class bits it would rasterise (reference layout [i][j][k],
 * bit c set when component c is dispersive) and its coefficient tables.
 * which: 0..2 kappa_e*d (x,y,z), 3..5 kappa_h*d, 6+8*axis+slot for the CPML
 * tables be_N ce_N be_F ce_F bh_N ch_N bh_F ch_F (SETUP_CPML,
 * setup.cu:584-668), 100 = ADE scalars C_E C_E_1 C_E_2 d1..d5 d_NL
 * C1..C5 (pole 0) C1..C5 (pole 1) dt N_EQ (setup.cu:1282-1373), 101 =
 * frequencies, 102 = source pulse per step. *len gets the table length. */
fdtd_status fdtd_plan(const fdtd_params* p, fdtd_dims* out);
fdtd_status fdtd_rasterise(const fdtd_params* p, uint8_t* bits, size_t count);
fdtd_status fdtd_coefficients(const fdtd_params* p, int which, double* out,
                              size_t count, size_t* len);

/* ---------------------------------------------------------------------- */
/* life cycle                                                              */

/* SETUP_CONST + MATERIAL_MATRIX + SETUP_Drude_CP + ALLOCATE_MEM +
 * SETUP_TFSF + DEF_* + SETUP_CPML (setup.cu:135-1558, tfsf2.cu:6-56,
 * main.cu:2435-2643).  Builds every table on the host in FP64, uploads
 * them and zeroes the state on `device`. */
fdtd_status fdtd_create(const fdtd_params* p, int device, fdtd_sim** out);
fdtd_status fdtd_destroy(fdtd_sim* s);
fdtd_status fdtd_get_dims(const fdtd_sim* s, fdtd_dims* out);
/* Zero every field, auxiliary state and DFT accumulator; t = 0. */
fdtd_status fdtd_reset(fdtd_sim* s);
const char* fdtd_last_error(void);

/* ---------------------------------------------------------------------- */
/* the time step, split the way the reference launches it                  */

/* UPDATE_hx/hy/hz + the H half of CORRECT_X/Y/Z (main.cu:2735-2813). */
fdtd_status fdtd_update_h(fdtd_sim* s, void* stream);
/* UPDATE_h_inc + UPDATE_e_inc + Mur ends + source injection
 * (main.cu:2791, 2822-2859). */
fdtd_status fdtd_update_line(fdtd_sim* s, void* stream);
/* E half of CORRECT_X/Y/Z, UpdateHydroP*, UPDATE_ex/ey/ez
 * (main.cu:2798-2901). */
fdtd_status fdtd_update_e(fdtd_sim* s, void* stream);
/* ScattAbs (main.cu:2920-2934) for the current step when
 * t % dft_every == 0; advances t. */
fdtd_status fdtd_spectral_accumulate(fdtd_sim* s, void* stream);

/* The fused fast path: nsteps full time steps (H, line, E, DFT), captured
 * into CUDA graphs where the step pattern repeats. */
fdtd_status fdtd_step(fdtd_sim* s, int nsteps, void* stream);
/* Runs until t == Tend + 1 (the reference loop is t = 0..Tend inclusive). */
fdtd_status fdtd_run(fdtd_sim* s, void* stream);
fdtd_status fdtd_get_time(const fdtd_sim* s, int* t);

/* Polls the device NaN/Inf watchdog; FDTD_ERR_NONFINITE if it fired,
 * FDTD_ERR_TIMEOUT if a Yee pass gave up waiting (one second) for the
 * tensor copies of a plane (the fields are then not valid). */
fdtd_status fdtd_check(fdtd_sim* s);

/* ---------------------------------------------------------------------- */
/* spectra (CalculateAbsScatt, Spectral.cu:411-1177)                       */

/* Flushes pending DFT samples and reduces the 12 face fluxes per
 * frequency on the device in FP64.  out19 (NUM_freq x 19, row major) gets
 * the reference's ScatAbs columns: lambda, Sca, Abs, Ext, the 12 face
 * fluxes (Sca: -X +X -Y +Y -Z +Z, then Abs), |E_inc|, Re E_inc, Im E_inc. */
fdtd_status fdtd_spectral_finalize(fdtd_sim* s, double* out19);
/* Same, written as ScatAbs.<t>.txt in the reference's format. */
fdtd_status fdtd_write_scatabs(fdtd_sim* s, const char* path);
/* Periodic simulations (periodic_xy): reflectance and transmittance from
 * the DFT of Ex, Ey, Hx, Hy on two whole xy planes, the reflection plane
 * at k = Nt_z - 5 below the TFSF face (scattered field) and the
 * transmission plane at k = NZ - Nt_z - 5 (total field) (Spectral.cu:11-16).
 * Per frequency and plane P = sum Re(Ey conj(Hx) - Ex conj(Hy)) dA, as
 * Reflectance_XZ sums it (main.cu:3295-3300); R = P_refl / (A |E_s|^2)
 * and T = -P_trans / (A |E_s|^2), A the plane's area and E_s = E_inc /
 * dft_every the incident spectrum as the planes sample it (H is stored as
 * Z0 H, so a plane wave carries |E|^2 per unit area; the transmitted wave
 * runs along +z, where P < 0).
 * out7 (NUM_freq x 7): lambda, R, T, 1 - R - T, |E_inc|, Re E_inc,
 * Im E_inc.  FDTD_ERR_STATE for a simulation that is not periodic (and
 * fdtd_spectral_finalize fails for one that is). */
fdtd_status fdtd_reflectance(fdtd_sim* s, double* out7);
/* Raw DFT phasors of one face/component in the reference's layout
 * [F][a][b] (main.cu:86 ThreeDMapD(f,II,JJ,...)), FP64 re/im.
 * box: 0 = Abs, 1 = Sca.  face: 0..5 = -X +X -Y +Y -Z +Z.
 * comp: 0..3 = the face's (E_a, E_b, H_a, H_b) in the reference's order
 * (Z faces: Ex Ey Hx Hy; Y faces: Ex Ez Hx Hz; X faces: Ey Ez Hy Hz).
 * periodic_xy: box 0, face 0 = the reflection plane, 1 = the transmission
 * plane (Ex Ey Hx Hy over the whole xy plane). */
fdtd_status fdtd_get_dft(fdtd_sim* s, int box, int face, int comp,
                         double* re, double* im, size_t count);
fdtd_status fdtd_get_freqs(const fdtd_sim* s, double* freq, size_t count);
/* Analytic incident spectrum E_incident[m] (main.cu:2632-2643). */
fdtd_status fdtd_get_incident(const fdtd_sim* s, double* re, double* im,
                              size_t count);

/* ---------------------------------------------------------------------- */
/* snapshots and probes (snapshot.cu:10-180, OUT.txt main.cu:2732)         */

/* Whole component in the reference's layout [i][j][k] (z fastest), as
 * double.  count must be nx*ny*nz. */
fdtd_status fdtd_get_field(fdtd_sim* s, int comp, double* out, size_t count);
/* Overwrites a whole component from the reference layout (test hook). */
fdtd_status fdtd_set_field(fdtd_sim* s, int comp, const double* in,
                           size_t count);
/* One plane (axis 0/1/2 at `index`) of a component into a device or host
 * buffer of doubles, layout [a][b] with the remaining axes in x,y,z order.
 * Asynchronous on `stream` when dst is device memory. */
fdtd_status fdtd_snapshot_plane(fdtd_sim* s, int comp, int axis, int index,
                                double* dst, size_t count, void* stream);
/* The same plane as fdtd_snapshot_plane, with no memory allocation of any
 * kind: the plane is gathered into a fixed scratch array in the library's
 * static device memory and copied to dst (host or device) on `stream`.
 * No counterpart in the reference.  Every call synchronises `stream` before
 * it returns, whatever dst is.  Limit: count <= 1048576 cells
 * (FDTD_ERR_INVALID beyond).  The scratch is one per device and shared by
 * all simulations: calls that overlap in time on one device race and must
 * be serialised by the caller.  The scratch's device address is looked up
 * on the first call on each device and kept for the life of the process:
 * the library must not be used across a cudaDeviceReset. */
fdtd_status fdtd_snapshot_plane_static(fdtd_sim* s, int comp, int axis,
                                       int index, double* dst, size_t count,
                                       void* stream);
/* Snapshots as the reference writes them (SNAPSHOT_1D / SNAPSHOT_2D /
 * SNAPSHOT_2D_N, snapshot.cu:23-176), taken on the device by the stepper
 * after every step t with t % t_skip == 0 (main.cu:2948-2991) into a ring of
 * `capacity` records.  mode is the reference's Snap_in:
 *   1  aux lines: ey at (2, 2, k) for k = 0, z_skip, ... (aux_len values)
 *      and the incident line's E with the same step (line_len values)
 *   2  the YZ plane at x = nx/2 of |P_d| (the Drude current) and of the
 *      mean density (NDx + NDy + NDz) / 3 as the reference holds it after
 *      its step (the density from before the step), rows over y with step
 *      y_skip, columns over z with step z_skip, row major
 *   3  the aux lines, then the YZ plane of |E|
 * A record is `record` doubles: the step index t at offset 0, then the
 * parts at the offsets in the layout (-1 = absent).  0 turns snapshots
 * off.  Enabling synchronises the device.  fdtd_step fails with
 * FDTD_ERR_STATE instead of overwriting records that were not drained. */
typedef struct fdtd_snapshot_layout {
  int mode, t_skip;
  int plane_rows, plane_cols;
  int aux_len, line_len;
  int off_plane, off_plane2, off_aux, off_line;
  int record, capacity;
} fdtd_snapshot_layout;
fdtd_status fdtd_snapshots_enable(fdtd_sim* s, int mode, int capacity,
                                  fdtd_snapshot_layout* out);
/* Copies the records taken since the last drain (at most max_records, in
 * step order) to host memory, asynchronously on `stream` (pinned memory
 * for an overlapped copy); *n gets the number of records. */
fdtd_status fdtd_snapshots_drain(fdtd_sim* s, double* host, int max_records,
                                 int* n, void* stream);
/* Probe record: ex, ey, ez at the probe cell after every completed step,
 * [t][3]. n = number of steps recorded so far. */
fdtd_status fdtd_get_probe(fdtd_sim* s, double* out, size_t count, int* n);
/* Rows [t0, t0+n) of the probe record into host memory, asynchronously on
 * `stream` (the rows must belong to steps already enqueued on it). */
fdtd_status fdtd_get_probe_range(fdtd_sim* s, int t0, int n, double* out,
                                 void* stream);
/* Replaces the soft-source samples injected at steps [t0, t0+n) (the
 * reference's pulse at e_inc[m0-50], main.cu:2845-2851) from host memory,
 * asynchronously on `stream`. */
fdtd_status fdtd_set_source(fdtd_sim* s, int t0, int n, const double* pulse,
                            void* stream);

/* Counters: kernels this handle has enqueued (graph replays included). */
typedef struct fdtd_stats {
  long long kernels;
  long long steps;
  long long graph_launches;
  /* launch shapes picked by the autotuner (min CTAs/SM, tile height,
   * z-chunk) and their measured time per launch, for the H and E passes */
  int h_minb, h_ty, h_kchunk, e_minb, e_ty, e_kchunk;
  float h_ms, e_ms;
  int h_staged, e_staged;  /* 1 = shared-memory pipelined pass */
  int h_stages, e_stages;  /* its ring depth */
  /* the same two for the launch over the CPML edge tiles */
  int h_eminb, h_estages, e_eminb, e_estages;
  /* 1 = the two launches of the pass run on one stream with a programmatic
   * dependency, 0 = on two streams */
  int h_pdl, e_pdl;
  /* sizes of the step's work beside the passes, for traffic accounting:
   * TFSF table entries of the H and E shells, and DFT rows (one per
   * tangential component and flux-face cell, padding excluded) */
  long long tfsf_entries_h, tfsf_entries_e, dft_rows;
  /* adjoint (after fdtd_forward / fdtd_forward_spectra): the steps whose
   * dispersive-cell trajectory the forward recorded (the backward recomputes
   * the others from checkpoints), the record's device bytes, and the number
   * of checkpoints kept */
  long long adj_record_steps, adj_record_bytes, adj_checkpoints;
  /* how the launches of the passes stage their planes: 1 = tensor copies
   * (one thread per CTA, completion on an mbarrier), 0 = per-thread
   * cp.async; interior and edge launch of the H and E passes */
  int h_tma, h_etma, e_tma, e_etma;
} fdtd_stats;
fdtd_status fdtd_get_stats(const fdtd_sim* s, fdtd_stats* out);
/* Measurement hook (no counterpart in the reference): runs one Yee pass
 * (its interior-tile and CPML-edge-tile launches) reps times back to back,
 * after two untimed runs, on `stream` and stores its mean device time per
 * pass, from CUDA events on that stream, in *ms.  The runs change the
 * fields: call fdtd_reset before using the simulation again. */
enum {
  FDTD_KERNEL_H_PASS = 0, /* the H pass (Yee + CPML) over the whole grid */
  FDTD_KERNEL_E_PASS = 1  /* the E pass (Yee + CPML) over the whole grid,
                             dispersive cells excluded */
};
fdtd_status fdtd_time_kernel(fdtd_sim* s, int which, int reps, void* stream,
                             double* ms);
/* Material class map used by the E pass (bit0..2: ex/ey/ez dispersive),
 * reference layout, for rasteriser parity checks. */
fdtd_status fdtd_get_material(fdtd_sim* s, uint8_t* out, size_t count);

/* ---------------------------------------------------------------------- */
/* adjoint (no counterpart in the reference)                               */

/* Design region: per-cell blend rho in [0,1] between vacuum and the metal
 * for a box [i0,i1)x[j0,j1)x[k0,k1), x fastest.  Cells with rho > 0 get a
 * per-cell ADE update with linearly blended coefficients. */
fdtd_status fdtd_set_design(fdtd_sim* s, const int box[6], const float* rho,
                            size_t count);
/* Forward for the reverse sweep: zeroes the state and runs t = 0..Tend in
 * segments of checkpoint_every steps.  The last segments, as many as the
 * device memory holds (env FDTD_ADJ_RECORD_GB caps it; at least one),
 * record the dispersive cells' trajectory as they run; every earlier
 * segment starts with a copy of the state, from which the backward
 * recomputes it.  fdtd_get_stats reports the split.  out19 (NUM_freq x 19,
 * may be NULL) gets the ScatAbs table of fdtd_spectral_finalize. */
fdtd_status fdtd_forward_spectra(fdtd_sim* s, int checkpoint_every,
                                 double* out19);
/* Reverse-time adjoint of the last forward (recomputing the segments that
 * were not recorded), for the objective whose gradient with respect to the
 * ScatAbs table is dL_dspectra (NUM_freq x 19, row major): any weighted sum of the
 * scattering, absorption and extinction columns and of the 12 face
 * fluxes (columns 1-15; columns 0 and 16-18 do not depend on the fields
 * and must be zero).  dL_drho (may be NULL) has the design box's cell
 * count; dL_dparams (may be NULL) gets d/d(omega_D), d/d(gamma_D). */
fdtd_status fdtd_backward_spectra(fdtd_sim* s, const double* dL_dspectra,
                                  float* dL_drho, size_t count,
                                  double* dL_dparams);
/* The absorbed-power objective: fdtd_forward_spectra, then objective =
 * sum over the listed frequency indices of the absorption cross-section
 * sigma_abs = P_abs / I_inc (m^2), the net inward flux through the
 * absorption box, -sum_f s_f q_abs,f over its faces (ScatAbs columns
 * 10-15, s_f = -1 / +1 on the - / + face of each axis).  It is positive
 * for an absorbing structure; the reference's AbsTot column is
 * -sigma_abs for every geometry but its sphere (Spectral.cu:1163-1168). */
fdtd_status fdtd_forward(fdtd_sim* s, const int* freq_idx, int nfreq,
                         int checkpoint_every, double* objective);
/* fdtd_backward_spectra for the objective of the last fdtd_forward. */
fdtd_status fdtd_backward(fdtd_sim* s, float* dL_drho, size_t count,
                          double* dL_dparams);

/* ---------------------------------------------------------------------- */
/* batched independent simulations (no counterpart in the reference; its
 * trials loop, main.cu:2435, is sequential)                               */

typedef struct fdtd_batch fdtd_batch;
/* n independent simulations on one device, each from its own parameters
 * (grid sizes may differ); all members share precision, the hydrodynamic
 * switch, the DFT sampling period and Tend. */
fdtd_status fdtd_batch_create(const fdtd_params* ps, int n, int device,
                              fdtd_batch** out);
/* Advances every member by nsteps.  Per time step the two Yee passes of
 * all members run as one persistent kernel each, fed from a shared
 * (member, tile) work queue, and every other kernel of the step runs as one
 * launch over all members; runs of 32*dft_every steps replay a CUDA graph. */
fdtd_status fdtd_batch_step(fdtd_batch* b, int nsteps, void* stream);
/* Runs every member to Tend (fdtd_batch_step with the remaining steps). */
fdtd_status fdtd_batch_run(fdtd_batch* b, void* stream);
/* Member idx as a borrowed simulation handle (fields, probes, spectra);
 * owned by the batch, valid until fdtd_batch_destroy. */
fdtd_status fdtd_batch_sim(fdtd_batch* b, int idx, fdtd_sim** out);
/* The 19-column ScatAbs table of member idx (fdtd_spectral_finalize). */
fdtd_status fdtd_batch_spectra(fdtd_batch* b, int idx, double* out19);
/* Kernel launches and graph replays issued by the batch so far. */
fdtd_status fdtd_batch_get_stats(const fdtd_batch* b, long long* kernels,
                                 long long* graph_launches);
/* The pass launch shapes fdtd_batch_create chose (its autotuner): members
 * are bucketed by their largest edge, 16 cells a bucket ([edge_lo, edge_hi]
 * inclusive); each bucket has its own z-chunk (planes per work item),
 * timed with the bucket's members alone (bucket_ms: both passes, one step).
 * Work items are tile_x x tile_y columns; minb / stages are the register
 * cap (minimum CTAs per SM) and ring depth of each persistent launch,
 * [0 = H pass, 1 = E pass][0 = CPML edge items, 1 = interior items], timed
 * over the whole batch.  tuned = 0 when the batch kept the defaults
 * (FDTD_TUNE=0 or under 2^20 cells). */
#define FDTD_BATCH_MAX_BUCKETS 16
typedef struct fdtd_batch_tuning {
  int tuned;
  int nbuckets;
  int edge_lo[FDTD_BATCH_MAX_BUCKETS], edge_hi[FDTD_BATCH_MAX_BUCKETS];
  int members[FDTD_BATCH_MAX_BUCKETS], kchunk[FDTD_BATCH_MAX_BUCKETS];
  float bucket_ms[FDTD_BATCH_MAX_BUCKETS];
  int tile_x, tile_y;
  int minb[2][2], stages[2][2];
} fdtd_batch_tuning;
fdtd_status fdtd_batch_get_tuning(const fdtd_batch* b, fdtd_batch_tuning* out);
fdtd_status fdtd_batch_destroy(fdtd_batch* b);

#ifdef __cplusplus
}
#endif
#endif /* FDTD_B200_H */
