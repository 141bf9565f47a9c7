// Host-side setup: restates SETUP_CONST, MATERIAL_MATRIX, SETUP_Drude_CP,
// SETUP_CPML, SETUP_TFSF and DEF_UPDATE_COEFF_* of the reference in FP64.
#include "setup.h"

#include <cmath>
#include <cstdio>
#include <cstring>

namespace fdtd {

// define.h:22-29
static const double kPI = 3.1415926535897932384626433832795;
static const double kEP0 = 8.85418782E-12;
static const double kMU0 = 1.25663706E-06;
static const double kC0 = 2.99792458E+08;
static const double kZ0 = 376.730313462;
static const double kE0 = 1.60217662E-19;
static const double kME = 9.10938356E-31;

void params_default(fdtd_params* p) {
  std::memset(p, 0, sizeof(*p));
  p->num_trials = p->min_trials = p->max_trials = 1;
  p->first_medium = 1;
  p->material = 3;
  p->WL_or_freq = 1;
  p->t_skip = p->x_skip = p->y_skip = p->z_skip = 1;
  p->MAX_AMP = 1.0;
  p->TimeFactor = 1.0;
  p->tfsf_inset = 10;          // setup.cu:428
  p->box_offset = 5;           // setup.cu:435-452
  p->cpml_order = 3;           // setup.cu:481
  p->cpml_kappa_max = 5.0;     // setup.cu:482
  p->cpml_alpha_max = 0.05;    // setup.cu:485
  p->cpml_sigma_factor = 0.8;  // setup.cu:483
  p->lam_min = 200e-9;         // main.cu:2447
  p->lam_max = 700e-9;         // main.cu:2446
  p->source_offset = 50;       // main.cu:2851
  p->dft_every = 4;            // main.cu:2920
  p->hydro_D = 2.0;            // setup.cu:981
  p->fermi_velocity = 1.39e8 / 100.0;  // setup.cu:980
  p->precision = FDTD_FP64;
  p->probe_i = p->probe_j = p->probe_k = -1;
}

// The 41 positional values of Input.txt (setup.cu:17-58).
#define FDTD_INPUT_FIELDS(X)                                                               \
  X(Tend, 'd') X(dx, 'g') X(dy, 'g') X(dz, 'g') X(num_trials, 'd') X(min_trials, 'd')      \
  X(max_trials, 'd') X(TE_TM, 'd') X(NCELLX, 'd') X(NCELLY, 'd') X(NCELLZ, 'd')             \
  X(NcpmlX, 'd') X(NcpmlY, 'd') X(NcpmlZ, 'd') X(inf_disp_slab, 'd') X(nano_sphere, 'd')    \
  X(nano_sphere_radius, 'g') X(material, 'd') X(first_medium, 'd') X(inc_plane, 'd')       \
  X(dispersive_slab, 'd') X(NUM_freq, 'd') X(WL_or_freq, 'd') X(NUM_freq_inc, 'd')         \
  X(Tend_inc, 'd') X(Snap_in, 'd') X(Freq_start, 'd') X(Test_offset, 'd') X(Spect_loc, 'd') \
  X(BandWidth, 'g') X(NONLOCAL, 'd') X(Diverge_Gradient, 'd') X(t_skip, 'd') X(x_skip, 'd') \
  X(y_skip, 'd') X(z_skip, 'd') X(Nonlocalend, 'g') X(MAX_AMP, 'g') X(TimeFactor, 'g')      \
  X(lam_0, 'g') X(StaticField, 'd')

int read_input_txt(const char* path, fdtd_params* p) {
  FILE* f = std::fopen(path, "r");
  if (!f) return -1;
  char label[512];
  bool ok = std::fscanf(f, "%511s", label) == 1;
#define READ_ONE(name, kind)                                                   \
  if (ok) {                                                                    \
    if (kind == 'd') ok = std::fscanf(f, "%d %511s", (int*)(void*)&p->name, label) == 2; \
    else ok = std::fscanf(f, "%lf %511s", (double*)(void*)&p->name, label) == 2;          \
  }
  FDTD_INPUT_FIELDS(READ_ONE)
#undef READ_ONE
  std::fclose(f);
  return ok ? 0 : -2;
}

int write_input_txt(const char* path, const fdtd_params* p) {
  FILE* f = std::fopen(path, "w");
  if (!f) return -1;
  std::fprintf(f, "Input\n");
#define WRITE_ONE(name, kind)                                            \
  if (kind == 'd') std::fprintf(f, "%d %s\n", *(const int*)(const void*)&p->name, #name); \
  else std::fprintf(f, "%.17g %s\n", *(const double*)(const void*)&p->name, #name);
  FDTD_INPUT_FIELDS(WRITE_ONE)
#undef WRITE_ONE
  std::fclose(f);
  return 0;
}

// SETUP_CPML_{X,Y,Z} (setup.cu:513-978): sigma and kappa graded with
// ((Nc - i)/Nc)^m (near) or (i/Nc)^m (far), alpha graded linearly the other
// way; H points sit half a cell inside.  b = exp(-(S/K + A) dt / eps0),
// c = S (b - 1) / (K (S + K A)).
static void cpml_axis(const fdtd_params& p, double d, int Nc, int F, int N, double dt, CpmlTables& t) {
  const double m = p.cpml_order;
  const double smax = p.cpml_sigma_factor * (m + 1) / (kZ0 * d);
  const double kmax = p.cpml_kappa_max, amax = p.cpml_alpha_max;
  t.ked.assign(N, d);
  t.khd.assign(N, d);
  t.be_N.assign(Nc + 1, 0); t.ce_N.assign(Nc + 1, 0);
  t.be_F.assign(Nc + 1, 0); t.ce_F.assign(Nc + 1, 0);
  t.bh_N.assign(Nc > 0 ? Nc : 0, 0); t.ch_N.assign(Nc > 0 ? Nc : 0, 0);
  t.bh_F.assign(Nc > 0 ? Nc : 0, 0); t.ch_F.assign(Nc > 0 ? Nc : 0, 0);
  if (Nc <= 0) return;
  auto grade = [&](double xs, double xa, double& b, double& c, double& kd) {
    double S = std::pow(xs, m) * smax;
    double A = amax * std::pow(xa, 1.0);
    double K = 1 + (kmax - 1) * std::pow(xs, m);
    b = std::exp(-(S / K + A) * (dt / kEP0));
    c = (K * A + S == 0.0) ? 0.0 : S * (b - 1) / (K * (S + K * A));
    kd *= K;
  };
  const double n = Nc;
  for (int i = 0; i <= Nc; i++) grade((double)(Nc - i) / n, (double)i / n, t.be_N[i], t.ce_N[i], t.ked[i]);
  for (int i = 0; i <= Nc; i++) grade((double)i / n, (double)(Nc - i) / n, t.be_F[i], t.ce_F[i], t.ked[i + F]);
  for (int i = 0; i < Nc; i++)
    grade((n - (double)i - 0.5) / n, ((double)i + 0.5) / n, t.bh_N[i], t.ch_N[i], t.khd[i]);
  for (int i = 0; i < Nc; i++)
    grade(((double)i + 0.5) / n, (n - (double)i - 0.5) / n, t.bh_F[i], t.ch_F[i], t.khd[i + F]);
}

// Drude + 2CP material constants (setup.cu:1164-1211).
struct Metal {
  double eps_inf, wD, gam, A[2], phi[2], Om[2], Ga[2], NEQ;
};
static Metal metal_table(const fdtd_params& p) {
  Metal m;
  if (p.material == 2) {
    m = {1.4447, 1.3280e16, 9.1269e13, {-1.5951, 0.25261}, {3.1288, -1.5066},
         {8.2749e15, 6.1998e15}, {5.1770e15, 5.4126e14}, 5.541318196761572e28};
  } else {
    m = {1.1431, 1.3202e16, 1.0805e14, {0.26698, 3.0834}, {-1.2371, -1.0968},
         {3.8711e15, 4.1684e15}, {4.4642e14, 2.3555e15}, 5.476415562682574e28};
  }
  if (p.metal_custom) {
    m.eps_inf = p.eps_inf; m.wD = p.omega_D; m.gam = p.gamma_D;
    for (int q = 0; q < 2; q++) {
      m.A[q] = p.cp_A[q]; m.phi[q] = p.cp_phi[q]; m.Om[q] = p.cp_Omega[q]; m.Ga[q] = p.cp_Gamma[q];
    }
    if (p.N_EQ > 0) m.NEQ = p.N_EQ;
  }
  return m;
}

// SETUP_Drude_CP (setup.cu:1282-1373): second-order ADE recursions.
static void ade_coefficients(Setup& s) {
  const fdtd_params& p = s.p;
  const double dt = s.dt, ep0 = s.ep0;
  const Metal mt = metal_table(p);
  const double D = p.hydro_D;
  const double nl = std::sqrt((3.0 * D / (D + 2.0)) / D);
  double NONLOC = 0;
  if (p.NONLOCAL == 1 || s.hydro) NONLOC = p.fermi_velocity * nl;
  s.N_EQ = s.hydro ? mt.NEQ : 0;
  for (int q = 0; q < 2; q++) {
    double a0 = 2.0 * ep0 * mt.A[q] * mt.Om[q] * (mt.Om[q] * std::cos(mt.phi[q]) - mt.Ga[q] * std::sin(mt.phi[q]));
    double a1 = -2.0 * ep0 * mt.A[q] * mt.Om[q] * std::sin(mt.phi[q]);
    double b0 = mt.Ga[q] * mt.Ga[q] + mt.Om[q] * mt.Om[q];
    double b1 = 2.0 * mt.Ga[q], b2 = 1.0;
    double Cc = b2 / (dt * dt) + b1 / (2.0 * dt) + b0 / 4.0;
    s.C1[q] = (2 * b2 / (dt * dt) - b0 / 2.0) / Cc;
    s.C2[q] = (b1 / (2.0 * dt) - b2 / (dt * dt) - b0 / 4.0) / Cc;
    s.C3[q] = (a0 / 4.0 + a1 / (2.0 * dt)) / Cc;
    s.C4[q] = a0 / (2.0 * Cc);
    s.C5[q] = (a0 / 4.0 - a1 / (2.0 * dt)) / Cc;
  }
  s.wD = mt.wD;
  s.gam = mt.gam;
  const double dd = 1.0 / (dt * dt) + mt.gam / (2.0 * dt);
  s.d1 = 2.0 / (dd * dt * dt);
  s.d2 = (mt.gam / (2.0 * dt) - 1.0 / (dt * dt)) / dd;
  double sum;
  if (!s.hydro) {
    s.d3 = s.d5 = ep0 * mt.wD * mt.wD / (4.0 * dd);
    s.d4 = ep0 * mt.wD * mt.wD / (2.0 * dd);
    s.dNL = NONLOC * NONLOC / dd;
    sum = 0.0; sum += s.d3; sum += s.C3[0]; sum += s.C3[1];
    s.C_E = ep0 * mt.eps_inf + sum;
    sum = 0.0; sum += s.d4; sum += s.C4[0]; sum += s.C4[1];
    s.C_E_1 = -sum + ep0 * mt.eps_inf;
    sum = 0.0; sum += s.d5; sum += s.C5[0]; sum += s.C5[1];
    s.C_E_2 = sum;
  } else {
    s.d3 = -1.0 * s.e0 / (s.me) / dd / dt;
    s.d4 = 1.0 * s.e0 / (s.me) / dd / dt;
    s.d5 = -1.0 / dd;
    s.dNL = std::pow(mt.NEQ, 1.0 / 3.0) * NONLOC * NONLOC / dd;
    sum = 0.0; sum += s.C3[0]; sum += s.C3[1];
    s.C_E = ep0 * mt.eps_inf + sum;
    sum = 0.0; sum += s.C4[0]; sum += s.C4[1];
    s.C_E_1 = -sum + ep0 * mt.eps_inf;
    sum = 0.0; sum += s.C5[0]; sum += s.C5[1];
    s.C_E_2 = sum;
  }
}

// MATERIAL_MATRIX (setup.cu:135-342) for the reference geometries; the
// extended shapes test the cell centre and the three staggered E points.
static void rasterise(Setup& s) {
  const fdtd_params& p = s.p;
  const int NX = s.NX, NY = s.NY, NZ = s.NZ;
  const size_t n = (size_t)NX * NY * NZ;
  std::vector<int> centre(n);
  for (int c = 0; c < 3; c++) s.matc[c].assign(n, p.first_medium);
  auto at = [&](int i, int j, int k) { return ((size_t)i * NY + j) * NZ + k; };
  const int mat = p.material;
  if (p.geometry == FDTD_GEOM_REFERENCE) {
    const int slab = p.dispersive_slab + s.Nt[1];
    for (int i = 0; i < NX; i++)
      for (int j = 0; j < NY; j++)
        for (int k = 0; k < NZ; k++) {
          int v = p.first_medium;
          if (p.inf_disp_slab == 1 && k >= slab) v = mat;
          if (p.inf_disp_slab == 2 && k >= slab && k < slab + (int)(p.nano_sphere_radius / p.dz)) v = mat;
          for (int c = 0; c < 3; c++) s.matc[c][at(i, j, k)] = v;
        }
    if (p.nano_sphere == 1 || p.nano_sphere == 3) {
      const int r = (int)(p.nano_sphere_radius / p.dx);
      // periodic x and y: the particle rests on the slab (setup.cu:223, 268)
      const double cx = NX / 2, cy = NY / 2, cz = p.periodic_xy ? (double)(slab - r) : (double)(NZ / 2);
      const double off[3][3] = {{0.5, 0, 0}, {0, 0.5, 0}, {0, 0, 0.5}};
      for (int i = 0; i < NX; i++)
        for (int j = 0; j < NY; j++)
          for (int k = 0; k < NZ; k++)
            for (int c = 0; c < 3; c++) {
              double x = i + off[c][0] - cx, y = j + off[c][1] - cy, z = k + off[c][2] - cz;
              bool in = p.nano_sphere == 1 ? std::pow(x * x + y * y + z * z, 0.5) < r
                                           : (x * x < r * r && y * y < r * r && z * z < r * r);
              if (in) s.matc[c][at(i, j, k)] = mat;
            }
    }
    return;
  }
  const double cx = NX / 2, cy = NY / 2, cz = NZ / 2;
  const double off[3][3] = {{0.5, 0, 0}, {0, 0.5, 0}, {0, 0, 0.5}};
  for (int i = 0; i < NX; i++)
    for (int j = 0; j < NY; j++)
      for (int k = 0; k < NZ; k++)
        for (int c = 0; c < 3; c++) {
          const double x = (i + off[c][0] - cx) * p.dx, y = (j + off[c][1] - cy) * p.dy,
                       z = (k + off[c][2] - cz) * p.dz;
          bool in = false;
          if (p.geometry == FDTD_GEOM_SPHERE) {
            double X = x - p.sphere_cx, Y = y - p.sphere_cy, Z = z - p.sphere_cz;
            in = X * X + Y * Y + Z * Z < p.sphere_radius * p.sphere_radius;
          } else if (p.geometry == FDTD_GEOM_ROD_DIMER) {
            const double a = p.axis == 0 ? x : p.axis == 1 ? y : z;
            const double u = p.axis == 0 ? y : x, v = p.axis == 2 ? y : z;
            const double R = 0.5 * p.rod_diameter, Lr = p.rod_length;
            const double rr = u * u + v * v;
            for (int sg = -1; sg <= 1; sg += 2) {
              const double t = a - sg * (0.5 * p.gap + 0.5 * Lr);
              const double half = 0.5 * Lr - R;
              if (std::fabs(t) <= half) {
                if (rr < R * R) in = true;
              } else {
                const double e = std::fabs(t) - half;
                if (rr + e * e < R * R) in = true;
              }
            }
          } else if (p.geometry == FDTD_GEOM_DISK_ARRAY) {
            const double R = 0.5 * p.disk_diameter;
            if (z >= 0 && z < p.disk_height)
              for (int a = 0; a < p.disk_nx; a++)
                for (int b = 0; b < p.disk_ny; b++) {
                  double X = x - (a - 0.5 * (p.disk_nx - 1)) * p.pitch;
                  double Y = y - (b - 0.5 * (p.disk_ny - 1)) * p.pitch;
                  if (X * X + Y * Y < R * R) in = true;
                }
          }
          if (in) s.matc[c][at(i, j, k)] = mat;
        }
  // dielectric slab under the disks (no counterpart in the reference, whose
  // DIELECTRIC_SLAB is commented out, main.cu:2566): cell centres with z in
  // [-slab_thickness, 0) of the disk frame, strictly inside the TFSF box in
  // x and y (off its faces, where the incident field is added); metal wins
  // where both apply
  if (p.geometry == FDTD_GEOM_DISK_ARRAY && p.slab_thickness > 0 && p.slab_eps != 1.0)
    for (int i = s.Nt[0] + 1; i < NX - s.Nt[0] - 1; i++)
      for (int j = s.Nt[1] + 1; j < NY - s.Nt[1] - 1; j++)
        for (int k = 0; k < NZ; k++) {
          const double z = (k - cz) * p.dz;
          if (!(z >= -p.slab_thickness && z < 0)) continue;
          for (int c = 0; c < 3; c++)
            if (!is_dispersive(s.matc[c][at(i, j, k)])) s.matc[c][at(i, j, k)] = kSlabMaterial;
        }
}

const char* setup_build(const fdtd_params& pin, Setup& s) {
  s.p = pin;
  const fdtd_params& p = s.p;
  if (p.NCELLX < 1 || p.NCELLY < 1 || p.NCELLZ < 1) return "NCELLX/Y/Z must be >= 1";
  if (p.dx <= 0 || p.dy <= 0 || p.dz <= 0) return "dx, dy, dz must be > 0";
  if (p.NUM_freq < 2) return "NUM_freq must be >= 2";
  if (p.Tend < 0) return "Tend must be >= 0";
  if (p.material != 2 && p.material != 3 && !p.metal_custom) return "material must be 2 (Ag) or 3 (Au)";
  if (p.dft_every < 1) return "dft_every must be >= 1";
  if (p.BandWidth <= 0) return "BandWidth must be > 0";
  if (p.geometry == FDTD_GEOM_DISK_ARRAY && p.slab_thickness > 0 && !(p.slab_eps >= 1.0))
    return "slab_eps must be >= 1";
  if (p.precision != FDTD_FP32 && p.precision != FDTD_FP64) return "precision must be FDTD_FP32 or FDTD_FP64";
  const bool per = p.periodic_xy != 0;
  if (per) {
    if (p.NcpmlX != 0 || p.NcpmlY != 0) return "periodic_xy needs NcpmlX = NcpmlY = 0 (CPML in z only)";
    if (p.NCELLX % 8 != 0 || p.NCELLX < 8 || p.NCELLY < 2) return "periodic_xy needs NCELLX a multiple of 8 and NCELLY >= 2";
    if (p.NONLOCAL == 3) return "periodic_xy does not support the hydrodynamic model";
    const int* b = p.design_box;
    if (b[1] > b[0] || b[3] > b[2] || b[5] > b[4]) return "periodic_xy does not support a design region";
    if (std::fabs(p.inc_theta_deg) > 1e-12) return "periodic_xy needs normal incidence (inc_theta_deg = 0)";
  }
  // SETUP_CONST (setup.cu:347-510)
  s.z0 = kZ0; s.ep0 = kEP0; s.mu0 = kMU0; s.c0 = kC0; s.pi = kPI; s.e0 = kE0; s.me = kME;
  s.L = p.NCELLZ * 6;
  if (p.NCELLX == 1 || p.NCELLY == 1 || p.NCELLZ == 1) s.dt = 0.9 * p.dy / (kC0 * std::pow(2, 0.5));
  else s.dt = 0.5 * p.dy / kC0 / (double)p.TimeFactor;
  // periodic x and y: the reference drops the grid's extra cell
  // (setup.cu:401-404) and has no lateral TFSF faces (setup.cu:429)
  s.NX = per ? p.NCELLX : p.NCELLX + 2 * p.NcpmlX + 1;
  s.NY = per ? p.NCELLY : p.NCELLY + 2 * p.NcpmlY + 1;
  s.NZ = p.NCELLZ + 2 * p.NcpmlZ + 1;
  const int N3[3] = {s.NX, s.NY, s.NZ};
  const int ncp[3] = {p.NcpmlX, p.NcpmlY, p.NcpmlZ};
  for (int a = 0; a < 3; a++) {
    if (ncp[a] < 0) return "Ncpml must be >= 0";
    s.Nc[a] = ncp[a];
    s.F[a] = N3[a] - 1 - ncp[a];
    s.Nt[a] = p.tfsf_inset + ncp[a];
    if (per && a < 2) {
      // no slab along a periodic axis: every slab test (index <= Nc or
      // >= F) fails
      s.Nc[a] = -1;
      s.F[a] = N3[a] + 1;
      s.Nt[a] = 0;
      s.absS[a] = s.scaS[a] = 0;
      s.absE[a] = s.scaE[a] = N3[a];
      continue;
    }
    s.absS[a] = s.Nt[a] + p.box_offset;
    s.absE[a] = N3[a] - s.Nt[a] - p.box_offset;
    s.scaS[a] = s.Nt[a] - p.box_offset;
    s.scaE[a] = N3[a] - s.Nt[a] + p.box_offset;
    if (s.scaS[a] < 1 || s.scaE[a] > N3[a] - 1 || s.absE[a] - s.absS[a] < 2)
      return "TFSF/DFT boxes do not fit the grid";
  }
  if (per) {
    // reflection and transmission planes (Spectral.cu:11-16)
    s.k_refl = s.Nt[2] - 5;
    s.k_trans = s.NZ - s.Nt[2] - 5;
    if (s.k_refl < s.Nc[2] + 1 || s.k_trans <= s.Nt[2] || s.k_trans >= s.F[2])
      return "periodic_xy: the reflection and transmission planes do not fit between the z CPML slabs";
  }
  s.hydro = p.NONLOCAL == 3;
  s.f0 = kC0 / p.lam_0;
  // frequency grid (main.cu:2442-2464)
  const int NF = p.NUM_freq;
  s.freq.resize(NF);
  for (int i = 0; i < NF; i++) {
    if (p.WL_or_freq == 1) s.freq[i] = s.c0 / (p.lam_min + i * (p.lam_max - p.lam_min) / (NF - 1.0));
    else s.freq[i] = s.c0 / p.lam_max + i * (s.c0 / p.lam_min - s.c0 / p.lam_max) / (NF - 1.0);
  }
  ade_coefficients(s);
  // SETUP_TFSF (tfsf2.cu:6-56)
  double th = p.inc_theta_deg, ph = p.inc_phi_deg, ps = p.polar_psi_deg;
  th *= s.pi / 180.0; ph *= s.pi / 180.0; ps *= s.pi / 180.0;
  s.d1D = p.dx;
  s.m0 = (int)std::floor(s.L / 2);
  s.i0 = s.Nt[0]; s.j0 = s.Nt[1]; s.k0 = s.Nt[2];
  s.width = std::ceil((6 / (p.BandWidth * 2 * s.pi)) / s.dt);
  s.delay = 6 * s.width;
  {
    const float st = sinf((float)th), ct = cosf((float)th), sp = sinf((float)ph), cp = cosf((float)ph),
                sps = sinf((float)ps), cps = cosf((float)ps);
    volatile float t0;
    // E and H direction factors, single precision like CORRECT_* (main.cu:392)
    t0 = cps * sp; s.fe[0] = t0 - (sps * ct) * cp;
    t0 = -cps * cp; s.fe[1] = t0 - (sps * ct) * sp;
    s.fe[2] = sps * st;
    t0 = sps * sp; s.fh[0] = t0 + (cps * ct) * cp;
    t0 = -sps * cp; s.fh[1] = t0 + (cps * ct) * sp;
    s.fh[2] = -cps * st;
    s.sth = st; s.cth = ct; s.sph = sp; s.cph = cp;
  }
  if (s.m0 - p.source_offset < 1) return "source position outside the 1D line";
  // the TFSF faces must interpolate inside the line
  {
    const int far = 2 * (s.NZ - s.Nt[2] - s.k0) + 2;
    if (std::fabs(p.inc_theta_deg) < 1e-12 && s.m0 + far / 2 + 2 >= s.L) return "1D line too short for the TFSF box";
  }
  // DEF_UPDATE_COEFF_* with eps = EP0, mu = MU0, sigma = 0
  s.Cee = (1 - (s.dt * 0) / (2 * kEP0)) / (1 + (s.dt * 0) / (2 * kEP0));
  s.Ceh = (s.dt / (s.z0 * kEP0)) / ((1 + (s.dt * 0) / (2 * kEP0)));
  s.Ceh_slab = (s.dt / (s.z0 * kEP0 * p.slab_eps)) / ((1 + (s.dt * 0) / (2 * kEP0 * p.slab_eps)));
  s.Chh = (1 - (s.dt * 0) / (2 * kMU0)) / (1 + (s.dt * 0) / (2 * kMU0));
  s.Che = (s.z0 * s.dt / kMU0) / (1 + (s.dt * 0) / (2 * kMU0));
  const double dxyz[3] = {p.dx, p.dy, p.dz};
  for (int a = 0; a < 3; a++) cpml_axis(p, dxyz[a], s.Nc[a], s.F[a], N3[a], s.dt, s.cp[a]);
  // setup.cu:681 uploads bh_z_F before SETUP_CPML_Z has filled it; the
  // reference runs with bh_x_F = 0.
  if (!(p.fixes & FDTD_FIX_BH_X_F))
    for (auto& v : s.cp[0].bh_F) v = 0.0;
  rasterise(s);
  {
    // adjoint design region: dispersive for all three components
    const int* b = p.design_box;
    if (b[1] > b[0] || b[3] > b[2] || b[5] > b[4]) {
      if (!(b[1] > b[0] && b[3] > b[2] && b[5] > b[4])) return "design_box is empty along one axis";
      if (p.first_medium != 1) return "the design region blends towards vacuum: first_medium must be 1";
      for (int a = 0; a < 3; a++)
        if (b[2 * a] < s.absS[a] + 1 || b[2 * a + 1] > s.absE[a] - 1)
          return "design_box must lie inside the absorption box";
      for (int c = 0; c < 3; c++)
        for (int i = b[0]; i < b[1]; i++)
          for (int j = b[2]; j < b[3]; j++)
            for (int k = b[4]; k < b[5]; k++) s.matc[c][((size_t)i * s.NY + j) * s.NZ + k] = p.material;
    }
  }
  if (s.hydro) {
    if (p.first_medium != 1) return "hydrodynamic model needs first_medium == 1";
    for (int c = 0; c < 3; c++)
      for (int i = 0; i < s.NX; i++)
        for (int j = 0; j < s.NY; j++)
          for (int k = 0; k < s.NZ; k++) {
            int v = s.matc[c][((size_t)i * s.NY + j) * s.NZ + k];
            if (!is_dispersive(v)) continue;
            if (i < 2 || j < 2 || k < 2 || i > s.NX - 3 || j > s.NY - 3 || k > s.NZ - 3)
              return "hydrodynamic metal touches the domain boundary";
            if (i == s.Nt[0] || i == s.NX - s.Nt[0] || j == s.Nt[1] || j == s.NY - s.Nt[1] || k == s.Nt[2] ||
                k == s.NZ - s.Nt[2])
              return "hydrodynamic metal on a TFSF face is not supported";
          }
  }
  // source pulse (main.cu:2845-2848) and incident spectrum (main.cu:2632-2643)
  s.pulse.resize((size_t)p.Tend + 1);
  for (int t = 0; t <= p.Tend; t++) {
    if (p.StaticField == 0) {
      float u = (float)((double)(t - s.delay) / (double)s.width);
      s.pulse[t] = p.MAX_AMP * std::exp(-(double)powf(u, 2) / 2.0) * std::sin(2 * s.pi * s.f0 * (t)*s.dt);
    } else {
      s.pulse[t] = t < 1000.0 ? (double)p.MAX_AMP * t / 1000.0 : p.MAX_AMP * 1.0;
    }
  }
  s.Einc.assign(NF, std::complex<double>(0, 0));
  for (int t = 0; t < p.Tend; t++) {
    double pulse = s.pulse[t];
    if (p.StaticField != 0) {
      float u = (float)((double)(t - s.delay) / (double)s.width);
      pulse = p.MAX_AMP * std::exp(-(double)powf(u, 2) / 2.0) * std::sin(2 * s.pi * s.f0 * (t)*s.dt);
    }
    for (int m = 0; m < NF; m++) {
      const double th_ = 2 * s.pi * t * s.dt * s.freq[m];
      s.Einc[m] += std::complex<double>(pulse * std::cos(th_), pulse * std::sin(th_));
    }
  }
  s.probe[0] = p.probe_i >= 0 ? p.probe_i : s.NX / 2;
  s.probe[1] = p.probe_j >= 0 ? p.probe_j : s.NY / 2;
  s.probe[2] = p.probe_k >= 0 ? p.probe_k : s.NZ / 2;
  if (s.probe[0] >= s.NX || s.probe[1] >= s.NY || s.probe[2] >= s.NZ) return "probe outside the grid";
  return nullptr;
}

}  // namespace fdtd
