/*
 * oracle.c -- FP64 CPU restatement of the reference FDTD time step.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle.h).  Each function cites the
 * reference routine it restates.  Semantics chosen where the reference is
 * ill-defined are stated at the function; the product follows the same
 * definitions.
 *
 * Build: make -C oracle   (gcc -O2 -fopenmp, no FMA contraction).
 */
#include "oracle.h"

#include <complex.h>
#include <math.h>
#include <omp.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* define.h:22-29 */
static const double K_PI = 3.1415926535897932384626433832795;
static const double K_EP0 = 8.85418782E-12;
static const double K_MU0 = 1.25663706E-06;
static const double K_C0 = 2.99792458E+08;
static const double K_Z0 = 376.730313462;
static const double K_E0 = 1.60217662E-19;
static const double K_ME = 9.10938356E-31;

enum { XC = 0, YC = 1, ZC = 2 };

typedef struct {
  double *be_N, *ce_N, *be_F, *ce_F; /* Nc+1 entries (E side) */
  double *bh_N, *ch_N, *bh_F, *ch_F; /* Nc entries (H side) */
} cpml_axis;

struct orc_sim {
  fdtd_params p;
  int NX, NY, NZ;
  int Nc[3], F[3];            /* Ncpml, cpml_F_* */
  int Nt[3];                  /* Ntfsf* */
  int absS[3], absE[3], scaS[3], scaE[3];
  int per;                    /* periodic x and y (the Periodic_XY branches) */
  int k_refl, k_trans;        /* periodic: reflection and transmission planes */
  int L, m0, i0, j0, k0;
  double d1D;
  double dt, z0, ep0, mu0, c0, pi, e0, me;
  double delay, width, f0;
  size_t n;                   /* NX*NY*NZ */
  int t;
  int hydro;
  int float_dft, dft_on;
  unsigned char* dft_sel;     /* per frequency: accumulate (NULL = all) */
  /* fields, reference layout */
  double *E[3], *H[3];
  double *En[3], *En1[3];     /* e*_n, e*_n_1 */
  double *Pcp[3], *Pcp_n[3], *Pcp_n1[3];   /* [cell][2] */
  double *Pd[3], *Pd_n[3], *Pd_n1[3], *Pd_n2[3];
  double *ND[3], *NDp[3];
  int *mat, *matc[3];
  /* Yee coefficients (uniform: eps = EP0, mu = MU0, sigma = 0) */
  double Cee, Ceh, Chh, Che;
  double Ceh_slab; /* dielectric slab class (material 6, eps = slab_eps) */
  /* CPML */
  double *ked[3], *khd[3];
  cpml_axis cp[3];
  double *psiE_N[3][2], *psiE_F[3][2];  /* [component][the other axis] */
  double *psiH_N[3][2], *psiH_F[3][2];
  /* ADE */
  double C_E, C_E_1, C_E_2;
  double d1, d2, d3, d4, d5, dNL, N_EQ;
  double C1[2], C2[2], C3[2], C4[2], C5[2];
  double* rho;  /* design blend per cell (NULL: plain metal), see orc_set_design */
  /* TFSF */
  double *e_inc, *h_inc, e1, e2;
  float fe[3], fh[3];        /* E/H incident direction factors (x,y,z) */
  float sth, cth, sph, cph;  /* sinf/cosf of the incidence angles */
  /* spectra */
  int NF;
  double *freq;
  double complex *Einc;
  double *dft[2][6][4][2];   /* box, face, comp, re/im */
  int dft_a[2][6], dft_b[2][6];
  /* probe */
  int pi_, pj, pk;
  double *probe;
};

#define IDX(s, i, j, k) (((size_t)(i) * (s)->NY + (size_t)(j)) * (s)->NZ + (size_t)(k))

static int g_threads = 0;
void orc_set_threads(int n) { g_threads = n; }

/* ------------------------------------------------------------------ */
/* parameters                                                          */

/* Reference defaults for the constants the reference hard-codes
 * (setup.cu:428-509, main.cu:2446-2447, tfsf2.cu:11-13, main.cu:2851,
 * main.cu:2920, setup.cu:980-981). */
void orc_params_default(fdtd_params* p) {
  memset(p, 0, sizeof(*p));
  p->num_trials = p->min_trials = p->max_trials = 1;
  p->first_medium = 1;
  p->material = 3;
  p->WL_or_freq = 1;
  p->t_skip = p->x_skip = p->y_skip = p->z_skip = 1;
  p->MAX_AMP = 1.0;
  p->TimeFactor = 1.0;
  p->tfsf_inset = 10;
  p->box_offset = 5;
  p->cpml_order = 3;
  p->cpml_kappa_max = 5.0;
  p->cpml_alpha_max = 0.05;
  p->cpml_sigma_factor = 0.8;
  p->lam_min = 200e-9;
  p->lam_max = 700e-9;
  p->source_offset = 50;
  p->dft_every = 4;
  p->hydro_D = 2.0;
  p->fermi_velocity = 1.39e8 / 100.0;
  p->precision = FDTD_FP64;
  p->probe_i = p->probe_j = p->probe_k = -1;
}

/* READ_DATA_FILE (setup.cu:10-133): one header token, then 41
 * "value label" pairs in fixed order. */
int orc_load_input_txt(const char* path, fdtd_params* p) {
  FILE* f = fopen(path, "r");
  if (!f) return -1;
  char tok[512];
  int ok = fscanf(f, "%511s", tok) == 1;
#define RI(x) ok = ok && fscanf(f, "%d %511s", &p->x, tok) == 2
#define RD(x) ok = ok && fscanf(f, "%lf %511s", &p->x, tok) == 2
  RI(Tend); RD(dx); RD(dy); RD(dz); RI(num_trials); RI(min_trials);
  RI(max_trials); RI(TE_TM); RI(NCELLX); RI(NCELLY); RI(NCELLZ);
  RI(NcpmlX); RI(NcpmlY); RI(NcpmlZ); RI(inf_disp_slab); RI(nano_sphere);
  RD(nano_sphere_radius); RI(material); RI(first_medium); RI(inc_plane);
  RI(dispersive_slab); RI(NUM_freq); RI(WL_or_freq); RI(NUM_freq_inc);
  RI(Tend_inc); RI(Snap_in); RI(Freq_start); RI(Test_offset); RI(Spect_loc);
  RD(BandWidth); RI(NONLOCAL); RI(Diverge_Gradient); RI(t_skip); RI(x_skip);
  RI(y_skip); RI(z_skip); RD(Nonlocalend); RD(MAX_AMP); RD(TimeFactor);
  RD(lam_0); RI(StaticField);
#undef RI
#undef RD
  fclose(f);
  return ok ? 0 : -2;
}

/* ------------------------------------------------------------------ */
/* setup                                                               */

static double* zalloc(size_t n) {
  double* a = (double*)calloc(n ? n : 1, sizeof(double));
  return a;
}

/* SETUP_CPML_{X,Y,Z} (setup.cu:513-978): polynomial-graded sigma and
 * kappa, linearly graded alpha, for the E points (i = 0..Nc) and the
 * half-shifted H points (i = 0..Nc-1), near and far slabs. */
static void setup_cpml_axis(orc_sim* s, int ax, double d) {
  const fdtd_params* p = &s->p;
  int Nc = s->Nc[ax];
  int Ntot = ax == 0 ? s->NX : ax == 1 ? s->NY : s->NZ;
  double m = p->cpml_order;
  double smax = p->cpml_sigma_factor * (m + 1) / (K_Z0 * d);
  double kmax = p->cpml_kappa_max, amax = p->cpml_alpha_max;
  cpml_axis* c = &s->cp[ax];
  s->ked[ax] = zalloc(Ntot);
  s->khd[ax] = zalloc(Ntot);
  for (int i = 0; i < Ntot; i++) s->ked[ax][i] = s->khd[ax][i] = d;
  c->be_N = zalloc(Nc + 1); c->ce_N = zalloc(Nc + 1);
  c->be_F = zalloc(Nc + 1); c->ce_F = zalloc(Nc + 1);
  int nh = Nc > 0 ? Nc : 0; /* Nc = -1: a periodic axis, no slab */
  c->bh_N = zalloc(nh); c->ch_N = zalloc(nh);
  c->bh_F = zalloc(nh); c->ch_F = zalloc(nh);
  if (Nc <= 0) return;
  double dt = s->dt;
#define GRADE(xs, xa, bout, cout, kscale)                                   \
  do {                                                                      \
    double S_ = pow((xs), m) * smax;                                        \
    double A_ = amax * pow((xa), 1.0);                                      \
    double K_ = 1 + (kmax - 1) * pow((xs), m);                              \
    (bout) = exp(-(S_ / K_ + A_) * (dt / K_EP0));                           \
    (cout) = (K_ * A_ + S_ == 0.0) ? 0.0                                    \
                                   : S_ * ((bout) - 1) / (K_ * (S_ + K_ * A_)); \
    (kscale) *= K_;                                                         \
  } while (0)
  for (int i = 0; i < Nc + 1; i++)
    GRADE((double)(Nc - i) / (double)Nc, (double)i / (double)Nc, c->be_N[i],
          c->ce_N[i], s->ked[ax][i]);
  for (int i = 0; i < Nc + 1; i++)
    GRADE((double)i / (double)Nc, (double)(Nc - i) / (double)Nc, c->be_F[i],
          c->ce_F[i], s->ked[ax][i + s->F[ax]]);
  for (int i = 0; i < Nc; i++)
    GRADE(((double)Nc - (double)i - 0.5) / (double)Nc,
          ((double)i + 0.5) / (double)Nc, c->bh_N[i], c->ch_N[i],
          s->khd[ax][i]);
  for (int i = 0; i < Nc; i++)
    GRADE(((double)i + 0.5) / (double)Nc,
          ((double)Nc - (double)i - 0.5) / (double)Nc, c->bh_F[i],
          c->ch_F[i], s->khd[ax][i + s->F[ax]]);
#undef GRADE
}

/* MATERIAL_MATRIX (setup.cu:135-342) for the reference geometries, plus the
 * extended shapes (rod dimer, disk array, real-radius sphere). */
static void rasterise(orc_sim* s) {
  const fdtd_params* p = &s->p;
  int NX = s->NX, NY = s->NY, NZ = s->NZ;
  int mat = p->material, fm = p->first_medium;
  int* m[4] = {s->mat, s->matc[0], s->matc[1], s->matc[2]};
  int slab = p->dispersive_slab + s->Nt[1];
  for (int i = 0; i < NX; i++)
    for (int j = 0; j < NY; j++)
      for (int k = 0; k < NZ; k++) {
        int v = fm;
        if (p->geometry == FDTD_GEOM_REFERENCE) {
          if (p->inf_disp_slab == 1 && k >= slab) v = mat;
          if (p->inf_disp_slab == 2 && k >= slab &&
              k < slab + (int)(p->nano_sphere_radius / p->dz))
            v = mat;
        }
        for (int q = 0; q < 4; q++) m[q][IDX(s, i, j, k)] = v;
      }
  if (p->geometry == FDTD_GEOM_REFERENCE && (p->nano_sphere == 1 || p->nano_sphere == 3)) {
    int r = (int)(p->nano_sphere_radius / p->dx);
    /* periodic x and y: the particle sits on the slab (setup.cu:223, 268) */
    double cz = s->per ? (double)(slab - r) : (double)(NZ / 2), cx = NX / 2, cy = NY / 2;
    for (int i = 0; i < NX; i++)
      for (int j = 0; j < NY; j++)
        for (int k = 0; k < NZ; k++) {
          /* offsets of the cell centre and of the Ex/Ey/Ez points */
          double off[4][3] = {{0, 0, 0}, {0.5, 0, 0}, {0, 0.5, 0}, {0, 0, 0.5}};
          for (int q = 0; q < 4; q++) {
            double x = i + off[q][0] - cx, y = j + off[q][1] - cy,
                   z = k + off[q][2] - cz;
            int in;
            if (p->nano_sphere == 1)
              in = pow(x * x + y * y + z * z, 0.5) < r;
            else
              in = x * x < r * r && y * y < r * r && z * z < r * r;
            if (in) m[q][IDX(s, i, j, k)] = mat;
          }
        }
    /* dielectric slab under the disks (the reference's DIELECTRIC_SLAB is
     * commented out, main.cu:2566): cell centres with z in [-T, 0),
     * strictly inside the TFSF box in x and y; metal wins */
    if (p->geometry == FDTD_GEOM_DISK_ARRAY && p->slab_thickness > 0 && p->slab_eps != 1.0) {
      double czs = NZ / 2;
      for (int i = s->Nt[0] + 1; i < NX - s->Nt[0] - 1; i++)
        for (int j = s->Nt[1] + 1; j < NY - s->Nt[1] - 1; j++)
          for (int k = 0; k < NZ; k++) {
            double z = (k - czs) * p->dz;
            if (!(z >= -p->slab_thickness && z < 0)) continue;
            for (int q = 0; q < 4; q++)
              if (!(m[q][IDX(s, i, j, k)] > 1 && m[q][IDX(s, i, j, k)] < 6)) m[q][IDX(s, i, j, k)] = 6;
          }
    }
  } else if (p->geometry == FDTD_GEOM_REFERENCE && p->nano_sphere == 2) {
    double cz = p->dispersive_slab, cx = NX / 2, cy = NY / 2;
    for (int i = 0; i < NX; i++)
      for (int j = 0; j < NY; j++)
        for (int k = 0; k < NZ; k++)
          if (i < cx + 2 && i > cx - 2 && j < cy + 2 && j > cy - 2 && k > cz - 20)
            s->mat[IDX(s, i, j, k)] = mat;
  } else if (p->geometry != FDTD_GEOM_REFERENCE) {
    /* Extended shapes: membership of the cell centre and the three
     * staggered E points, shape coordinates in metres from the grid
     * centre (NX/2, NY/2, NZ/2 in cells). */
    double cx = NX / 2, cy = NY / 2, cz = NZ / 2;
    for (int i = 0; i < NX; i++)
      for (int j = 0; j < NY; j++)
        for (int k = 0; k < NZ; k++) {
          double off[4][3] = {{0, 0, 0}, {0.5, 0, 0}, {0, 0.5, 0}, {0, 0, 0.5}};
          for (int q = 0; q < 4; q++) {
            double x = (i + off[q][0] - cx) * p->dx;
            double y = (j + off[q][1] - cy) * p->dy;
            double z = (k + off[q][2] - cz) * p->dz;
            int in = 0;
            if (p->geometry == FDTD_GEOM_SPHERE) {
              double X = x - p->sphere_cx, Y = y - p->sphere_cy, Z = z - p->sphere_cz;
              in = X * X + Y * Y + Z * Z < p->sphere_radius * p->sphere_radius;
            } else if (p->geometry == FDTD_GEOM_ROD_DIMER) {
              /* rods along `axis`, centred at +-(gap/2 + L/2), radius R,
               * total length L including hemispherical caps */
              double a = p->axis == 0 ? x : p->axis == 1 ? y : z;
              double u = p->axis == 0 ? y : x, v = p->axis == 2 ? y : z;
              double R = 0.5 * p->rod_diameter, L = p->rod_length;
              double rr = u * u + v * v;
              for (int sgn = -1; sgn <= 1; sgn += 2) {
                double c = sgn * (0.5 * p->gap + 0.5 * L);
                double t = a - c;
                double half = 0.5 * L - R; /* cylinder half length */
                if (fabs(t) <= half) {
                  if (rr < R * R) in = 1;
                } else {
                  double e = fabs(t) - half;
                  if (rr + e * e < R * R) in = 1;
                }
              }
            } else if (p->geometry == FDTD_GEOM_DISK_ARRAY) {
              /* slab occupies z in [-T, 0), disks z in [0, h) */
              double R = 0.5 * p->disk_diameter;
              if (z >= 0 && z < p->disk_height) {
                for (int a = 0; a < p->disk_nx; a++)
                  for (int b = 0; b < p->disk_ny; b++) {
                    double X = x - (a - 0.5 * (p->disk_nx - 1)) * p->pitch;
                    double Y = y - (b - 0.5 * (p->disk_ny - 1)) * p->pitch;
                    if (X * X + Y * Y < R * R) in = 1;
                  }
              }
            }
            if (in) m[q][IDX(s, i, j, k)] = mat;
          }
        }
    /* dielectric slab under the disks (the reference's DIELECTRIC_SLAB is
     * commented out, main.cu:2566): cell centres with z in [-T, 0),
     * strictly inside the TFSF box in x and y; metal wins */
    if (p->geometry == FDTD_GEOM_DISK_ARRAY && p->slab_thickness > 0 && p->slab_eps != 1.0) {
      double czs = NZ / 2;
      for (int i = s->Nt[0] + 1; i < NX - s->Nt[0] - 1; i++)
        for (int j = s->Nt[1] + 1; j < NY - s->Nt[1] - 1; j++)
          for (int k = 0; k < NZ; k++) {
            double z = (k - czs) * p->dz;
            if (!(z >= -p->slab_thickness && z < 0)) continue;
            for (int q = 0; q < 4; q++)
              if (!(m[q][IDX(s, i, j, k)] > 1 && m[q][IDX(s, i, j, k)] < 6)) m[q][IDX(s, i, j, k)] = 6;
          }
    }
  }
}

/* SETUP_Drude_CP (setup.cu:979-1373): Drude pole + two critical points,
 * second-order ADE recursion coefficients; hydrodynamic variant when
 * NONLOCAL == 3. */
static void setup_ade(orc_sim* s) {
  const fdtd_params* p = &s->p;
  double dt = s->dt, ep0 = s->ep0;
  double D = p->hydro_D;
  double Ccoef = 3.0 * D / (D + 2.0);
  double NL_COEFF = sqrt(Ccoef / D);
  double vF = p->fermi_velocity;
  double NONLOC = 0;
  double eps_inf, wD, gam, A[2], phi[2], Om[2], Ga[2], NEQ = 0;
  if (p->material == 2) {
    eps_inf = 1.4447; wD = 1.3280e16; gam = 9.1269e13;
    A[0] = -1.5951; phi[0] = 3.1288; Om[0] = 8.2749e15; Ga[0] = 5.1770e15;
    A[1] = 0.25261; phi[1] = -1.5066; Om[1] = 6.1998e15; Ga[1] = 5.4126e14;
    NEQ = 5.541318196761572e28;
  } else {
    eps_inf = 1.1431; wD = 1.3202e16; gam = 1.0805e14;
    A[0] = 0.26698; phi[0] = -1.2371; Om[0] = 3.8711e15; Ga[0] = 4.4642e14;
    A[1] = 3.0834; phi[1] = -1.0968; Om[1] = 4.1684e15; Ga[1] = 2.3555e15;
    NEQ = 5.476415562682574e28;
  }
  if (p->metal_custom) {
    eps_inf = p->eps_inf; wD = p->omega_D; gam = p->gamma_D;
    for (int q = 0; q < 2; q++) {
      A[q] = p->cp_A[q]; phi[q] = p->cp_phi[q];
      Om[q] = p->cp_Omega[q]; Ga[q] = p->cp_Gamma[q];
    }
    if (p->N_EQ > 0) NEQ = p->N_EQ;
  }
  if (p->NONLOCAL == 1) NONLOC = vF * NL_COEFF;
  if (s->hydro) NONLOC = vF * NL_COEFF;
  s->N_EQ = s->hydro ? NEQ : 0;
  for (int q = 0; q < 2; q++) {
    double a0 = 2.0 * ep0 * A[q] * Om[q] * (Om[q] * cos(phi[q]) - Ga[q] * sin(phi[q]));
    double a1 = -2.0 * ep0 * A[q] * Om[q] * sin(phi[q]);
    double b0 = Ga[q] * Ga[q] + Om[q] * Om[q];
    double b1 = 2.0 * Ga[q];
    double b2 = 1.0;
    double Cc = b2 / (dt * dt) + b1 / (2.0 * dt) + b0 / 4.0;
    s->C1[q] = (2 * b2 / (dt * dt) - b0 / 2.0) / Cc;
    s->C2[q] = (b1 / (2.0 * dt) - b2 / (dt * dt) - b0 / 4.0) / Cc;
    s->C3[q] = (a0 / 4.0 + a1 / (2.0 * dt)) / Cc;
    s->C4[q] = a0 / (2.0 * Cc);
    s->C5[q] = (a0 / 4.0 - a1 / (2.0 * dt)) / Cc;
  }
  double dd = 1.0 / (dt * dt) + gam / (2.0 * dt);
  s->d1 = 2.0 / (dd * dt * dt);
  s->d2 = (gam / (2.0 * dt) - 1.0 / (dt * dt)) / dd;
  if (!s->hydro) {
    s->d3 = s->d5 = ep0 * wD * wD / (4.0 * dd);
    s->d4 = ep0 * wD * wD / (2.0 * dd);
    s->dNL = NONLOC * NONLOC / dd;
    double sm = 0.0;
    sm += s->d3; sm += s->C3[0]; sm += s->C3[1];
    s->C_E = ep0 * eps_inf + sm;
    sm = 0.0; sm += s->d4; sm += s->C4[0]; sm += s->C4[1];
    s->C_E_1 = -sm + ep0 * eps_inf;
    sm = 0.0; sm += s->d5; sm += s->C5[0]; sm += s->C5[1];
    s->C_E_2 = sm;
  } else {
    s->d3 = -1.0 * s->e0 / (s->me) / dd / dt;
    s->d4 = 1.0 * s->e0 / (s->me) / dd / dt;
    s->d5 = -1.0 / dd;
    s->dNL = pow(NEQ, 1.0 / 3.0) * NONLOC * NONLOC / dd;
    double sm = 0.0;
    sm += s->C3[0]; sm += s->C3[1];
    s->C_E = ep0 * eps_inf + sm;
    sm = 0.0; sm += s->C4[0]; sm += s->C4[1];
    s->C_E_1 = -sm + ep0 * eps_inf;
    sm = 0.0; sm += s->C5[0]; sm += s->C5[1];
    s->C_E_2 = sm;
  }
}

/* Source pulse (main.cu:2634-2636, 2845-2848): Gaussian envelope with the
 * exponent squared in single precision (powf), times a sine carrier. */
static double pulse_at(const orc_sim* s, int t) {
  float u = (float)((double)(t - s->delay) / (double)s->width);
  return s->p.MAX_AMP * exp(-(double)powf(u, 2) / 2.0) *
         sin(2 * s->pi * s->f0 * (t)*s->dt);
}

orc_sim* orc_create(const fdtd_params* pin, char* err) {
  orc_sim* s = (orc_sim*)calloc(1, sizeof(orc_sim));
  s->p = *pin;
  fdtd_params* p = &s->p;
#define FAIL(msg)                                 \
  do {                                            \
    if (err) snprintf(err, 256, "%s", msg);       \
    orc_destroy(s);                               \
    return NULL;                                  \
  } while (0)
  if (p->NCELLX < 1 || p->NCELLY < 1 || p->NCELLZ < 1) FAIL("grid too small");
  if (p->dx <= 0 || p->dy <= 0 || p->dz <= 0) FAIL("cell size must be > 0");
  if (p->NUM_freq < 2) FAIL("NUM_freq must be >= 2");
  if (p->material != 2 && p->material != 3 && !p->metal_custom)
    FAIL("material must be 2 (Ag) or 3 (Au)");
  /* SETUP_CONST (setup.cu:347-510) */
  s->L = p->NCELLZ * 6;
  if (p->NCELLX == 1 || p->NCELLY == 1 || p->NCELLZ == 1)
    s->dt = 0.9 * p->dy / (K_C0 * pow(2, 0.5));
  else
    s->dt = 0.5 * p->dy / K_C0 / (double)p->TimeFactor;
  s->z0 = K_Z0; s->ep0 = K_EP0; s->mu0 = K_MU0; s->c0 = K_C0; s->pi = K_PI;
  s->me = K_ME; s->e0 = K_E0;
  s->per = p->periodic_xy != 0;
  if (s->per) {
    /* Periodic_XY (setup.cu:401-404, 429): no x or y CPML, no lateral
     * TFSF faces; the plane wave enters at normal incidence */
    if (p->NcpmlX != 0 || p->NcpmlY != 0) FAIL("periodic_xy needs NcpmlX = NcpmlY = 0");
    if (p->NCELLX % 8 != 0 || p->NCELLX < 8 || p->NCELLY < 2) FAIL("periodic_xy grid");
    if (p->NONLOCAL == 3) FAIL("periodic_xy does not support the hydrodynamic model");
    if (fabs(p->inc_theta_deg) > 1e-12) FAIL("periodic_xy needs normal incidence");
  }
  /* periodic: the reference drops the grid's extra cell (setup.cu:401-404) */
  s->NX = p->NCELLX + 2 * p->NcpmlX + (s->per ? 0 : 1);
  s->NY = p->NCELLY + 2 * p->NcpmlY + (s->per ? 0 : 1);
  s->NZ = p->NCELLZ + 2 * p->NcpmlZ + 1;
  s->Nc[0] = p->NcpmlX; s->Nc[1] = p->NcpmlY; s->Nc[2] = p->NcpmlZ;
  s->F[0] = s->NX - 1 - p->NcpmlX;
  s->F[1] = s->NY - 1 - p->NcpmlY;
  s->F[2] = s->NZ - 1 - p->NcpmlZ;
  int N3[3] = {s->NX, s->NY, s->NZ};
  for (int a = 0; a < 3; a++) {
    if (s->per && a < 2) {
      /* every index of a periodic axis is updated and no slab test holds
       * (index <= Nc or >= F); the DFT planes span it */
      s->Nc[a] = -1;
      s->F[a] = N3[a] + 1;
      s->Nt[a] = 0;
      s->absS[a] = s->scaS[a] = 0;
      s->absE[a] = s->scaE[a] = N3[a];
      continue;
    }
    s->Nt[a] = p->tfsf_inset + s->Nc[a];
    s->absS[a] = s->Nt[a] + p->box_offset;
    s->absE[a] = N3[a] - s->Nt[a] - p->box_offset;
    s->scaS[a] = s->Nt[a] - p->box_offset;
    s->scaE[a] = N3[a] - s->Nt[a] + p->box_offset;
    if (s->scaS[a] < 1 || s->scaE[a] > N3[a] - 1 || s->absE[a] - s->absS[a] < 2)
      FAIL("TFSF/DFT boxes do not fit the grid");
  }
  if (s->per) {
    /* Fourier_Transform (Spectral.cu:11-16) */
    s->k_refl = s->Nt[2] - 5;
    s->k_trans = s->NZ - s->Nt[2] - 5;
    if (s->k_refl < s->Nc[2] + 1 || s->k_trans <= s->Nt[2] || s->k_trans >= s->F[2])
      FAIL("periodic_xy: the reflection and transmission planes do not fit");
  }
  s->n = (size_t)s->NX * s->NY * s->NZ;
  s->hydro = p->NONLOCAL == 3;
  s->f0 = K_C0 / p->lam_0;
  /* MATERIAL_MATRIX */
  s->mat = (int*)calloc(s->n, sizeof(int));
  for (int c = 0; c < 3; c++) s->matc[c] = (int*)calloc(s->n, sizeof(int));
  rasterise(s);
  {
    /* adjoint design region (no counterpart in the reference): dispersive
     * for all three components, class `material` */
    const int* b = p->design_box;
    if (b[1] > b[0] && b[3] > b[2] && b[5] > b[4])
      for (int c = 0; c < 3; c++)
        for (int i = b[0]; i < b[1]; i++)
          for (int j = b[2]; j < b[3]; j++)
            for (int k = b[4]; k < b[5]; k++) {
              s->matc[c][IDX(s, i, j, k)] = p->material;
              s->mat[IDX(s, i, j, k)] = p->material;
            }
  }
  if (s->hydro) {
    /* the reference reads outside its arrays when metal touches the outer
     * planes (main.cu:1950-1980 wrap and i-1 = -1); that case is rejected */
    for (int c = 0; c < 3; c++)
      for (int i = 0; i < s->NX; i++)
        for (int j = 0; j < s->NY; j++)
          for (int k = 0; k < s->NZ; k++) {
            int v = s->matc[c][IDX(s, i, j, k)];
            if (v > p->first_medium && v < 6 &&
                (i < 2 || j < 2 || k < 2 || i > s->NX - 3 || j > s->NY - 3 || k > s->NZ - 3))
              FAIL("hydrodynamic metal touches the domain boundary");
          }
  }
  /* frequency grid (main.cu:2442-2464) */
  s->NF = p->NUM_freq;
  s->freq = zalloc(s->NF);
  for (int i = 0; i < s->NF; i++) {
    if (p->WL_or_freq == 1)
      s->freq[i] = s->c0 / (p->lam_min + i * (p->lam_max - p->lam_min) / (s->NF - 1.0));
    else
      s->freq[i] = s->c0 / p->lam_max + i * (s->c0 / p->lam_min - s->c0 / p->lam_max) / (s->NF - 1.0);
  }
  setup_ade(s);
  /* SETUP_TFSF (tfsf2.cu:6-56) */
  double th = p->inc_theta_deg, ph = p->inc_phi_deg, ps = p->polar_psi_deg;
  th *= s->pi / 180.0; ph *= s->pi / 180.0; ps *= s->pi / 180.0;
  s->d1D = p->dx;
  s->m0 = (int)floor(s->L / 2);
  s->i0 = s->Nt[0]; s->j0 = s->Nt[1]; s->k0 = s->Nt[2];
  s->width = ceil((6 / (p->BandWidth * 2 * s->pi)) / s->dt);
  s->delay = 6 * s->width;
  s->e1 = s->e2 = 0;
  {
    float st = sinf((float)th), ct = cosf((float)th), sp = sinf((float)ph),
          cp = cosf((float)ph), sps = sinf((float)ps), cps = cosf((float)ps);
    /* incident E and H direction factors, single precision as in
     * CORRECT_* (main.cu:392, 407, 466, 481 and their X/Z mirrors) */
    s->fe[0] = cps * sp - sps * ct * cp;
    s->fe[1] = -cps * cp - sps * ct * sp;
    s->fe[2] = sps * st;
    s->fh[0] = sps * sp + cps * ct * cp;
    s->fh[1] = -sps * cp + cps * ct * sp;
    s->fh[2] = -cps * st;
    s->sth = st; s->cth = ct; s->sph = sp; s->cph = cp;
  }
  s->e_inc = zalloc(s->L);
  s->h_inc = zalloc(s->L);
  if (s->m0 - p->source_offset < 1) FAIL("source position outside the 1D line");
  /* Yee coefficients (DEF_UPDATE_COEFF_*, setup.cu:2015-2062) with
   * eps = EP0, mu = MU0, sigma = 0 (DEF_EPS/MU/SIGMA, setup.cu:1943-1997) */
  s->Cee = (1 - (s->dt * 0) / (2 * K_EP0)) / (1 + (s->dt * 0) / (2 * K_EP0));
  s->Ceh = (s->dt / (s->z0 * K_EP0)) / ((1 + (s->dt * 0) / (2 * K_EP0)));
  s->Ceh_slab = (s->dt / (s->z0 * K_EP0 * s->p.slab_eps)) / ((1 + (s->dt * 0) / (2 * K_EP0 * s->p.slab_eps)));
  s->Chh = (1 - (s->dt * 0) / (2 * K_MU0)) / (1 + (s->dt * 0) / (2 * K_MU0));
  s->Che = (s->z0 * s->dt / K_MU0) / (1 + (s->dt * 0) / (2 * K_MU0));
  /* CPML; order X, Z, Y as SETUP_CPML does (setup.cu:513-533) */
  setup_cpml_axis(s, 0, p->dx);
  setup_cpml_axis(s, 2, p->dz);
  setup_cpml_axis(s, 1, p->dy);
  if (!(p->fixes & FDTD_FIX_BH_X_F))
    for (int i = 0; i < s->Nc[0]; i++) s->cp[0].bh_F[i] = 0.0;
  /* fields and state */
  for (int c = 0; c < 3; c++) {
    s->E[c] = zalloc(s->n); s->H[c] = zalloc(s->n);
    s->En[c] = zalloc(s->n); s->En1[c] = zalloc(s->n);
    s->Pcp[c] = zalloc(2 * s->n); s->Pcp_n[c] = zalloc(2 * s->n);
    s->Pcp_n1[c] = zalloc(2 * s->n);
    s->Pd[c] = zalloc(s->n); s->Pd_n[c] = zalloc(s->n);
    s->Pd_n1[c] = zalloc(s->n); s->Pd_n2[c] = zalloc(s->n);
    if (s->hydro) { s->ND[c] = zalloc(s->n); s->NDp[c] = zalloc(s->n); }
  }
  /* psi arrays: E component c has psi along the two other axes */
  for (int c = 0; c < 3; c++)
    for (int q = 0; q < 2; q++) {
      int ax = (c + 1 + q) % 3; /* ex: y,z  ey: z,x  ez: x,y */
      int w = s->Nc[ax] > 0 ? s->Nc[ax] : 0;
      size_t ne = s->n / N3[ax] * (s->Nc[ax] + 1);
      size_t nh = s->n / N3[ax] * w;
      s->psiE_N[c][q] = zalloc(ne); s->psiE_F[c][q] = zalloc(ne);
      s->psiH_N[c][q] = zalloc(nh); s->psiH_F[c][q] = zalloc(nh);
    }
  /* incident spectrum (main.cu:2632-2643) */
  s->Einc = (double complex*)calloc(s->NF, sizeof(double complex));
  for (int t = 0; t < p->Tend; t++) {
    double pulse = pulse_at(s, t);
    for (int m = 0; m < s->NF; m++) {
      double th_ = 2 * s->pi * t * s->dt * s->freq[m];
      s->Einc[m] += pulse * (cos(th_) + I * sin(th_));
    }
  }
  /* DFT boxes (ScattAbs main.cu:35-366): face extents; periodic: box 0
   * faces 0 and 1 are the reflection and transmission planes */
  for (int b = 0; b < 2 && s->per; b++)
    for (int f = 0; f < 6; f++) {
      s->dft_a[b][f] = b == 0 && f < 2 ? s->NX + 1 : 0;
      s->dft_b[b][f] = b == 0 && f < 2 ? s->NY + 1 : 0;
    }
  for (int b = 0; b < 2 && !s->per; b++) {
    const int* S = b == 0 ? s->absS : s->scaS;
    const int* E = b == 0 ? s->absE : s->scaE;
    for (int f = 0; f < 6; f++) {
      int ax = f / 2;
      int a1 = ax == 0 ? 1 : 0, a2 = ax == 2 ? 1 : 2;
      s->dft_a[b][f] = E[a1] - S[a1] + 1;
      s->dft_b[b][f] = E[a2] - S[a2] + 1;
    }
  }
  s->dft_on = 1;
  /* probe (OUT.txt, main.cu:2732) */
  s->pi_ = p->probe_i >= 0 ? p->probe_i : s->NX / 2;
  s->pj = p->probe_j >= 0 ? p->probe_j : s->NY / 2;
  s->pk = p->probe_k >= 0 ? p->probe_k : s->NZ / 2;
  s->probe = zalloc((size_t)3 * (p->Tend + 2));
  return s;
#undef FAIL
}

void orc_destroy(orc_sim* s) {
  if (!s) return;
  free(s->rho);
  free(s->dft_sel);
  for (int c = 0; c < 3; c++) {
    free(s->E[c]); free(s->H[c]); free(s->En[c]); free(s->En1[c]);
    free(s->Pcp[c]); free(s->Pcp_n[c]); free(s->Pcp_n1[c]);
    free(s->Pd[c]); free(s->Pd_n[c]); free(s->Pd_n1[c]); free(s->Pd_n2[c]);
    free(s->ND[c]); free(s->NDp[c]); free(s->matc[c]);
    free(s->ked[c]); free(s->khd[c]);
    cpml_axis* a = &s->cp[c];
    free(a->be_N); free(a->ce_N); free(a->be_F); free(a->ce_F);
    free(a->bh_N); free(a->ch_N); free(a->bh_F); free(a->ch_F);
    for (int q = 0; q < 2; q++) {
      free(s->psiE_N[c][q]); free(s->psiE_F[c][q]);
      free(s->psiH_N[c][q]); free(s->psiH_F[c][q]);
    }
  }
  for (int b = 0; b < 2; b++)
    for (int f = 0; f < 6; f++)
      for (int c = 0; c < 4; c++)
        for (int r = 0; r < 2; r++) free(s->dft[b][f][c][r]);
  free(s->mat); free(s->e_inc); free(s->h_inc); free(s->freq); free(s->Einc);
  free(s->probe);
  free(s);
}

/* Design blend of the cells of params.design_box (x fastest in the box),
 * the other dispersive cells keep rho = 1.  Returns 0, or -1 for a
 * simulation without a design box or a wrong count. */
int orc_set_design(orc_sim* s, const float* rho, size_t count) {
  const int* b = s->p.design_box;
  if (!(b[1] > b[0] && b[3] > b[2] && b[5] > b[4])) return -1;
  const int bx = b[1] - b[0], by = b[3] - b[2], bz = b[5] - b[4];
  if (count != (size_t)bx * by * bz) return -1;
  if (!s->rho) {
    s->rho = (double*)malloc(s->n * sizeof(double));
    for (size_t q = 0; q < s->n; q++) s->rho[q] = 1.0;
  }
  for (int k = 0; k < bz; k++)
    for (int j = 0; j < by; j++)
      for (int i = 0; i < bx; i++)
        s->rho[IDX(s, b[0] + i, b[2] + j, b[4] + k)] = rho[((size_t)k * by + j) * bx + i];
  return 0;
}

void orc_set_float_dft(orc_sim* s, int on) { s->float_dft = on; }
void orc_set_dft_enabled(orc_sim* s, int on) { s->dft_on = on; }
int orc_set_dft_freqs(orc_sim* s, const int* idx, int n) {
  free(s->dft_sel);
  s->dft_sel = NULL;
  if (!idx || n <= 0) return 0;
  s->dft_sel = (unsigned char*)calloc((size_t)s->NF, 1);
  for (int q = 0; q < n; q++) {
    if (idx[q] < 0 || idx[q] >= s->NF) return -1;
    s->dft_sel[idx[q]] = 1;
  }
  return 0;
}
int orc_time(const orc_sim* s) { return s->t; }

/* ------------------------------------------------------------------ */
/* the time step                                                       */

/* psi index helpers: slabs keep the reference's shapes
 * (ThreeDMapD with the slab width as the size along the slab axis). */
static inline size_t pidx(const orc_sim* s, int ax, int w, int i, int j, int k) {
  if (ax == 0) return ((size_t)i * s->NY + j) * s->NZ + k;          /* [w][NY][NZ] */
  if (ax == 1) return ((size_t)i * w + j) * s->NZ + k;              /* [NX][w][NZ] */
  return ((size_t)i * s->NY + j) * w + k;                           /* [NX][NY][w] */
}

/* UPDATE_hx/hy/hz (main.cu:762-1044), non-periodic branch.  Component c is
 * updated where the index along c is < N and the other two are < N-1; the
 * CPML psi terms apply only where all three indices are < N-1. */
static void update_h(orc_sim* s) {
  int NX = s->NX, NY = s->NY, NZ = s->NZ;
  double **E = s->E, **H = s->H;
#pragma omp parallel for schedule(static)
  for (int i = 0; i < NX; i++)
    for (int j = 0; j < NY; j++)
      for (int k = 0; k < NZ; k++) {
        size_t id = IDX(s, i, j, k);
        int in3 = i < NX - 1 && j < NY - 1 && k < NZ - 1;
        /* hx: i<NX, j<NY-1, k<NZ-1 */
        if (j < NY - 1 && k < NZ - 1) {
          double dey = E[1][IDX(s, i, j, k + 1)] - E[1][id];
          double dez = E[2][IDX(s, i, j + 1, k)] - E[2][id];
          double curl = dey / s->khd[2][k] - dez / s->khd[1][j];
          H[0][id] = s->Chh * H[0][id] + s->Che * curl;
          if (in3) {
            const cpml_axis* z = &s->cp[2]; const cpml_axis* y = &s->cp[1];
            if (k < s->Nc[2]) {
              double* ps = &s->psiH_N[0][1][pidx(s, 2, s->Nc[2], i, j, k)];
              *ps = z->bh_N[k] * *ps + z->ch_N[k] * dey / s->p.dz;
              H[0][id] += s->Che * *ps;
            }
            if (k >= s->F[2]) {
              int k2 = k - s->F[2];
              double* ps = &s->psiH_F[0][1][pidx(s, 2, s->Nc[2], i, j, k2)];
              *ps = z->bh_F[k2] * *ps + z->ch_F[k2] * dey / s->p.dz;
              H[0][id] += s->Che * *ps;
            }
            if (j < s->Nc[1]) {
              double* ps = &s->psiH_N[0][0][pidx(s, 1, s->Nc[1], i, j, k)];
              *ps = y->bh_N[j] * *ps + y->ch_N[j] * dez / s->p.dy;
              H[0][id] -= s->Che * *ps;
            }
            if (j >= s->F[1]) {
              int j2 = j - s->F[1];
              double* ps = &s->psiH_F[0][0][pidx(s, 1, s->Nc[1], i, j2, k)];
              *ps = y->bh_F[j2] * *ps + y->ch_F[j2] * dez / s->p.dy;
              H[0][id] -= s->Che * *ps;
            }
          }
        }
        /* hy: i<NX-1, j<NY, k<NZ-1 */
        if (i < NX - 1 && k < NZ - 1) {
          double dez = E[2][IDX(s, i + 1, j, k)] - E[2][id];
          double dex = E[0][IDX(s, i, j, k + 1)] - E[0][id];
          double curl = dez / s->khd[0][i] - dex / s->khd[2][k];
          H[1][id] = s->Chh * H[1][id] + s->Che * curl;
          if (in3) {
            const cpml_axis* z = &s->cp[2]; const cpml_axis* x = &s->cp[0];
            if (k < s->Nc[2]) {
              double* ps = &s->psiH_N[1][0][pidx(s, 2, s->Nc[2], i, j, k)];
              *ps = z->bh_N[k] * *ps + z->ch_N[k] * dex / s->p.dz;
              H[1][id] -= s->Che * *ps;
            }
            if (k >= s->F[2]) {
              int k2 = k - s->F[2];
              double* ps = &s->psiH_F[1][0][pidx(s, 2, s->Nc[2], i, j, k2)];
              *ps = z->bh_F[k2] * *ps + z->ch_F[k2] * dex / s->p.dz;
              H[1][id] -= s->Che * *ps;
            }
            if (i < s->Nc[0]) {
              double* ps = &s->psiH_N[1][1][pidx(s, 0, s->Nc[0], i, j, k)];
              *ps = x->bh_N[i] * *ps + x->ch_N[i] * dez / s->p.dx;
              H[1][id] += s->Che * *ps;
            }
            if (i >= s->F[0]) {
              int i2 = i - s->F[0];
              double* ps = &s->psiH_F[1][1][pidx(s, 0, s->Nc[0], i2, j, k)];
              *ps = x->bh_F[i2] * *ps + x->ch_F[i2] * dez / s->p.dx;
              H[1][id] += s->Che * *ps;
            }
          }
        }
        /* hz: i<NX-1, j<NY-1, k<NZ */
        if (i < NX - 1 && j < NY - 1) {
          double dex = E[0][IDX(s, i, j + 1, k)] - E[0][id];
          double dey = E[1][IDX(s, i + 1, j, k)] - E[1][id];
          double curl = dex / s->khd[1][j] - dey / s->khd[0][i];
          H[2][id] = s->Chh * H[2][id] + s->Che * curl;
          if (in3) {
            const cpml_axis* x = &s->cp[0]; const cpml_axis* y = &s->cp[1];
            if (i < s->Nc[0]) {
              double* ps = &s->psiH_N[2][0][pidx(s, 0, s->Nc[0], i, j, k)];
              *ps = x->bh_N[i] * *ps + x->ch_N[i] * dey / s->p.dx;
              H[2][id] -= s->Che * *ps;
            }
            if (i >= s->F[0]) {
              int i2 = i - s->F[0];
              double* ps = &s->psiH_F[2][0][pidx(s, 0, s->Nc[0], i2, j, k)];
              *ps = x->bh_F[i2] * *ps + x->ch_F[i2] * dey / s->p.dx;
              H[2][id] -= s->Che * *ps;
            }
            if (j < s->Nc[1]) {
              double* ps = &s->psiH_N[2][1][pidx(s, 1, s->Nc[1], i, j, k)];
              *ps = y->bh_N[j] * *ps + y->ch_N[j] * dex / s->p.dy;
              H[2][id] += s->Che * *ps;
            }
            if (j >= s->F[1]) {
              int j2 = j - s->F[1];
              double* ps = &s->psiH_F[2][1][pidx(s, 1, s->Nc[1], i, j2, k)];
              *ps = y->bh_F[j2] * *ps + y->ch_F[j2] * dex / s->p.dy;
              H[2][id] += s->Che * *ps;
            }
          }
        }
      }
}

/* UPDATE_hx/hy/hz, Periodic_XY branches (main.cu:781-820, 877-920,
 * 962-1000): every x and y index is updated, the +x and +y neighbours of
 * the last column and row are the first (real fields: no Bloch phase).
 * hx and hy are updated for k < NZ-1 and hz for every k, as in the
 * non-periodic branch (the reference's periodic hx and hy run to k = NZ-1
 * and read E at k = NZ there, outside the array); the z CPML applies over
 * the whole plane. */
static void update_h_periodic(orc_sim* s) {
  int NX = s->NX, NY = s->NY, NZ = s->NZ;
  double **E = s->E, **H = s->H;
  const cpml_axis* z = &s->cp[2];
#pragma omp parallel for schedule(static)
  for (int i = 0; i < NX; i++)
    for (int j = 0; j < NY; j++) {
      int ip = i + 1 == NX ? 0 : i + 1, jp = j + 1 == NY ? 0 : j + 1;
      for (int k = 0; k < NZ; k++) {
        size_t id = IDX(s, i, j, k);
        if (k < NZ - 1) {
          double dey = E[1][IDX(s, i, j, k + 1)] - E[1][id];
          double dez = E[2][IDX(s, i, jp, k)] - E[2][id];
          H[0][id] = s->Chh * H[0][id] + s->Che * (dey / s->khd[2][k] - dez / s->khd[1][j]);
          double dez_x = E[2][IDX(s, ip, j, k)] - E[2][id];
          double dex = E[0][IDX(s, i, j, k + 1)] - E[0][id];
          H[1][id] = s->Chh * H[1][id] + s->Che * (dez_x / s->khd[0][i] - dex / s->khd[2][k]);
          double* p0 = NULL;
          double* p1 = NULL;
          double b = 0, c = 0;
          if (k < s->Nc[2]) {
            p0 = &s->psiH_N[0][1][pidx(s, 2, s->Nc[2], i, j, k)];
            p1 = &s->psiH_N[1][0][pidx(s, 2, s->Nc[2], i, j, k)];
            b = z->bh_N[k]; c = z->ch_N[k];
          } else if (k >= s->F[2]) {
            int k2 = k - s->F[2];
            p0 = &s->psiH_F[0][1][pidx(s, 2, s->Nc[2], i, j, k2)];
            p1 = &s->psiH_F[1][0][pidx(s, 2, s->Nc[2], i, j, k2)];
            b = z->bh_F[k2]; c = z->ch_F[k2];
          }
          if (p0) {
            *p0 = b * *p0 + c * dey / s->p.dz;
            H[0][id] += s->Che * *p0;
            *p1 = b * *p1 + c * dex / s->p.dz;
            H[1][id] -= s->Che * *p1;
          }
        }
        double dex_y = E[0][IDX(s, i, jp, k)] - E[0][id];
        double dey_x = E[1][IDX(s, ip, j, k)] - E[1][id];
        H[2][id] = s->Chh * H[2][id] + s->Che * (dex_y / s->khd[1][j] - dey_x / s->khd[0][i]);
      }
    }
}

/* Projection of a staggered point onto the incidence direction, in cells,
 * with the reference's mixed precision: a term whose offset is a whole
 * number of cells is int * float * float (single precision), a half-cell
 * offset is double * float * float; the three terms are summed left to
 * right with C promotion (CORRECT_* main.cu:388-740). hx2/hy2/hz2 are twice
 * the offsets from (i0, j0, k0). */
static double proj(const orc_sim* s, int hx2, int hy2, int hz2) {
  /* each term is (value, is_double) */
  double t[3];
  int isd[3];
  float fa[3] = {s->sth, s->sth, s->cth};
  float fb[3] = {s->cph, s->sph, 1.0f};
  int h2[3] = {hx2, hy2, hz2};
  for (int a = 0; a < 3; a++) {
    if (!(h2[a] & 1)) {
      float v = (float)(h2[a] / 2) * fa[a];
      if (a < 2) v = v * fb[a];
      t[a] = v; isd[a] = 0;
    } else {
      double v = (h2[a] * 0.5) * (double)fa[a];
      if (a < 2) v = v * (double)fb[a];
      t[a] = v; isd[a] = 1;
    }
  }
  double d;
  if (!isd[0] && !isd[1]) {
    float xy = (float)t[0] + (float)t[1];
    d = isd[2] ? (double)xy + t[2] : (double)(xy + (float)t[2]);
  } else {
    d = (t[0] + t[1]) + t[2];
  }
  return (s->p.dx / s->d1D) * d;
}

static inline double einc_at(const orc_sim* s, double d) {
  double dp = d - (int)d;
  return (1 - dp) * s->e_inc[s->m0 + (int)d] + dp * s->e_inc[s->m0 + (int)d + 1];
}
static inline double hinc_at(const orc_sim* s, double d) {
  double d2 = d + 0.5;
  double dp = d2 - (int)(d2);
  return (1 - dp) * s->h_inc[s->m0 - 1 + (int)d2] + dp * s->h_inc[s->m0 + (int)d2];
}

/* CORRECT_X / CORRECT_Y / CORRECT_Z (main.cu:369-758): the H faces use the
 * incident E line at step n, the E faces the incident H line at n+1/2.
 * Applied in the launch order X, Y, Z.  The correction of E is added
 * before the E update (main.cu:2798-2880). */
static void tfsf(orc_sim* s) {
  int NX = s->NX, NY = s->NY, NZ = s->NZ;
  int Tx = s->Nt[0], Ty = s->Nt[1], Tz = s->Nt[2];
  int i0 = s->i0, j0 = s->j0, k0 = s->k0;
  double **E = s->E, **H = s->H;
  double Che = s->Che, Ceh = s->Ceh;
  double dx = s->p.dx, dy = s->p.dy, dz = s->p.dz;
  const float* fe = s->fe; const float* fh = s->fh;
  if (s->per) {
    /* Periodic_XY: the lower z face of CORRECT_Z only (main.cu:698), over
     * the whole plane.  The reference also launches CORRECT_X and _Y, whose
     * faces then sit at i = 0 and j = 0 and write H at index -1, outside
     * its arrays; with x and y periodic the lateral faces of a box that
     * spans the period add nothing, and they are left out. */
    int k = Tz;
    for (int i = 0; i < NX; i++)
      for (int j = 0; j < NY; j++) {
        double eyi = einc_at(s, proj(s, 2 * (i - i0), 2 * (j - j0) + 1, 2 * (k - k0))) * fe[1];
        H[0][IDX(s, i, j, k - 1)] -= Che * eyi / dz;
        double exi = einc_at(s, proj(s, 2 * (i - i0) + 1, 2 * (j - j0), 2 * (k - k0))) * fe[0];
        H[1][IDX(s, i, j, k - 1)] += Che * exi / dz;
        double hxi = hinc_at(s, proj(s, 2 * (i - i0), 2 * (j - j0) + 1, 2 * (k - k0) - 1)) * fh[0];
        E[1][IDX(s, i, j, k)] -= Ceh * hxi / dz;
        double hyi = hinc_at(s, proj(s, 2 * (i - i0) + 1, 2 * (j - j0), 2 * (k - k0) - 1)) * fh[1];
        E[0][IDX(s, i, j, k)] += Ceh * hyi / dz;
      }
    return;
  }
  /* CORRECT_X */
  for (int j = Ty; j <= NY - Ty; j++)
    for (int k = Tz; k <= NZ - Tz; k++)
      for (int side = 0; side < 2; side++) {
        int i = side == 0 ? Tx : NX - Tx;
        double sg = side == 0 ? 1.0 : -1.0;
        int hi = side == 0 ? i - 1 : i;     /* H target index */
        int ie2 = side == 0 ? 2 * (i - i0) - 1 : 2 * (i - i0) + 1;
        double ezi = einc_at(s, proj(s, 2 * (i - i0), 2 * (j - j0), 2 * (k - k0) + 1)) * fe[2];
        if (k != NZ - Tz) H[1][IDX(s, hi, j, k)] -= sg * (Che * ezi / dx);
        double eyi = einc_at(s, proj(s, 2 * (i - i0), 2 * (j - j0) + 1, 2 * (k - k0))) * fe[1];
        if (j != NY - Ty) H[2][IDX(s, hi, j, k)] += sg * (Che * eyi / dx);
        double hzi = hinc_at(s, proj(s, ie2, 2 * (j - j0) + 1, 2 * (k - k0))) * fh[2];
        if (j != NY - Ty) E[1][IDX(s, i, j, k)] += sg * (Ceh * hzi / dx);
        double hyi = hinc_at(s, proj(s, ie2, 2 * (j - j0), 2 * (k - k0) + 1)) * fh[1];
        if (k != NZ - Tz) E[2][IDX(s, i, j, k)] -= sg * (Ceh * hyi / dx);
      }
  /* CORRECT_Y */
  for (int i = Tx; i <= NX - Tx; i++)
    for (int k = Tz; k <= NZ - Tz; k++)
      for (int side = 0; side < 2; side++) {
        int j = side == 0 ? Ty : NY - Ty;
        double sg = side == 0 ? 1.0 : -1.0;
        int hj = side == 0 ? j - 1 : j;
        int je2 = side == 0 ? 2 * (j - j0) - 1 : 2 * (j - j0) + 1;
        double ezi = einc_at(s, proj(s, 2 * (i - i0), 2 * (j - j0), 2 * (k - k0) + 1)) * fe[2];
        if (k != NZ - Tz) H[0][IDX(s, i, hj, k)] += sg * (Che * ezi / dy);
        double exi = einc_at(s, proj(s, 2 * (i - i0) + 1, 2 * (j - j0), 2 * (k - k0))) * fe[0];
        if (i != NX - Tx) H[2][IDX(s, i, hj, k)] -= sg * (Che * exi / dy);
        double hzi = hinc_at(s, proj(s, 2 * (i - i0) + 1, je2, 2 * (k - k0))) * fh[2];
        if (i != NX - Tx) E[0][IDX(s, i, j, k)] -= sg * (Ceh * hzi / dy);
        double hxi = hinc_at(s, proj(s, 2 * (i - i0), je2, 2 * (k - k0) + 1)) * fh[0];
        if (k != NZ - Tz) E[2][IDX(s, i, j, k)] += sg * (Ceh * hxi / dy);
      }
  /* CORRECT_Z */
  for (int i = Tx; i <= NX - Tx; i++)
    for (int j = Ty; j <= NY - Ty; j++)
      for (int side = 0; side < 2; side++) {
        int k = side == 0 ? Tz : NZ - Tz;
        double sg = side == 0 ? 1.0 : -1.0;
        int hk = side == 0 ? k - 1 : k;
        int ke2 = side == 0 ? 2 * (k - k0) - 1 : 2 * (k - k0) + 1;
        double eyi = einc_at(s, proj(s, 2 * (i - i0), 2 * (j - j0) + 1, 2 * (k - k0))) * fe[1];
        if (j != NY - Ty) H[0][IDX(s, i, j, hk)] -= sg * (Che * eyi / dz);
        double exi = einc_at(s, proj(s, 2 * (i - i0) + 1, 2 * (j - j0), 2 * (k - k0))) * fe[0];
        if (i != NX - Tx) H[1][IDX(s, i, j, hk)] += sg * (Che * exi / dz);
        double hxi = hinc_at(s, proj(s, 2 * (i - i0), 2 * (j - j0) + 1, ke2)) * fh[0];
        if (j != NY - Ty) E[1][IDX(s, i, j, k)] -= sg * (Ceh * hxi / dz);
        double hyi = hinc_at(s, proj(s, 2 * (i - i0) + 1, 2 * (j - j0), ke2)) * fh[1];
        if (i != NX - Tx) E[0][IDX(s, i, j, k)] += sg * (Ceh * hyi / dz);
      }
}

/* UPDATE_h_inc / UPDATE_e_inc (main.cu:2280-2337) and the host-side Mur
 * ends and soft source (main.cu:2831-2859). */
static void line_h(orc_sim* s) {
  double c = s->z0 * s->dt / (s->mu0 * s->d1D);
  for (int i = 0; i < s->L - 1; i++) s->h_inc[i] = s->h_inc[i] - c * (s->e_inc[i + 1] - s->e_inc[i]);
}
static void line_e(orc_sim* s) {
  double c = s->dt / (s->z0 * s->ep0 * s->d1D);
  for (int i = 1; i < s->L - 1; i++) s->e_inc[i] = s->e_inc[i] - c * (s->h_inc[i] - s->h_inc[i - 1]);
  double factor = s->c0 * s->dt;
  double r = (factor - s->d1D) / (factor + s->d1D);
  s->e_inc[0] = s->e1 + r * (s->e_inc[1] - s->e_inc[0]);
  s->e_inc[s->L - 1] = s->e2 + r * (s->e_inc[s->L - 2] - s->e_inc[s->L - 1]);
  s->e1 = s->e_inc[1];
  s->e2 = s->e_inc[s->L - 2];
  if (s->p.StaticField == 0) {
    s->e_inc[s->m0 - s->p.source_offset] += pulse_at(s, s->t);
  } else {
    double pulse = s->t < 1000.0 ? (double)s->p.MAX_AMP * s->t / 1000.0 : s->p.MAX_AMP * 1.0;
    s->e_inc[s->m0 - s->p.source_offset] += pulse;
  }
}

static inline int is_metal(const orc_sim* s, int v) { return v > 1 && v < 6; }
static inline int is_metal_hydro(const orc_sim* s, int v) {
  return v > s->p.first_medium && v < 6;
}

/* UpdateHydroPx/Py/Pz (main.cu:1916-2276): new hydrodynamic current of
 * the Drude pole from E^n, its history and the pressure term
 * d_NL (grad div J + grad div (N J)/N_EQ) / (N_EQ + N)^(1/3).  Convection
 * and Lorentz-force terms are switched off in the reference
 * (setup.cu:990-999) and are not restated. Interior-cell formula only. */
static void hydro_p(orc_sim* s) {
  int NX = s->NX, NY = s->NY, NZ = s->NZ;
  double IX = 1.0 / s->p.dx, IY = 1.0 / s->p.dy, IZ = 1.0 / s->p.dz;
  double **P = s->Pd_n, **N = s->NDp;
  double NEQ = s->N_EQ;
  int fix = s->p.fixes & FDTD_FIX_HYDRO_CBRT;
#define A(c, i, j, k) P[c][IDX(s, i, j, k)]
#define AN(c, i, j, k) (P[c][IDX(s, i, j, k)] * N[c][IDX(s, i, j, k)])
#pragma omp parallel for schedule(static)
  for (int i = 1; i < NX - 1; i++)
    for (int j = 1; j < NY - 1; j++)
      for (int k = 1; k < NZ - 1; k++) {
        size_t id = IDX(s, i, j, k);
        for (int c = 0; c < 3; c++) {
          if (!is_metal_hydro(s, s->matc[c][id])) continue;
          double gd, gd2;
          if (c == 0) {
            gd2 = IX * IX * (AN(0, i + 1, j, k) - 2.0 * AN(0, i, j, k) + AN(0, i - 1, j, k)) +
                  IX * IY * (AN(1, i + 1, j, k) - AN(1, i, j, k) - AN(1, i + 1, j - 1, k) + AN(1, i, j - 1, k)) +
                  IX * IZ * (AN(2, i + 1, j, k) - AN(2, i, j, k) - AN(2, i + 1, j, k - 1) + AN(2, i, j, k - 1));
            gd = IX * IX * (A(0, i + 1, j, k) - 2.0 * A(0, i, j, k) + A(0, i - 1, j, k)) +
                 IX * IY * (A(1, i + 1, j, k) - A(1, i, j, k) - A(1, i + 1, j - 1, k) + A(1, i, j - 1, k)) +
                 IX * IZ * (A(2, i + 1, j, k) - A(2, i, j, k) - A(2, i + 1, j, k - 1) + A(2, i, j, k - 1));
          } else if (c == 1) {
            gd2 = IY * IY * (AN(1, i, j + 1, k) - 2.0 * AN(1, i, j, k) + AN(1, i, j - 1, k)) +
                  IX * IY * (AN(0, i, j + 1, k) - AN(0, i, j, k) - AN(0, i - 1, j + 1, k) + AN(0, i - 1, j, k)) +
                  IY * IZ * (AN(2, i, j + 1, k) - AN(2, i, j, k) - AN(2, i, j + 1, k - 1) + AN(2, i, j, k - 1));
            gd = IY * IY * (A(1, i, j + 1, k) - 2.0 * A(1, i, j, k) + A(1, i, j - 1, k)) +
                 IX * IY * (A(0, i, j + 1, k) - A(0, i, j, k) - A(0, i - 1, j + 1, k) + A(0, i - 1, j, k)) +
                 IY * IZ * (A(2, i, j + 1, k) - A(2, i, j, k) - A(2, i, j + 1, k - 1) + A(2, i, j, k - 1));
          } else {
            gd2 = IZ * IZ * (AN(2, i, j, k + 1) - 2.0 * AN(2, i, j, k) + AN(2, i, j, k - 1)) +
                  IZ * IY * (AN(1, i, j, k + 1) - AN(1, i, j, k) - AN(1, i, j - 1, k + 1) + AN(1, i, j - 1, k)) +
                  IX * IZ * (AN(0, i, j, k + 1) - AN(0, i, j, k) - AN(0, i - 1, j, k + 1) + AN(0, i - 1, j, k));
            gd = IZ * IZ * (A(2, i, j, k + 1) - 2.0 * A(2, i, j, k) + A(2, i, j, k - 1)) +
                 IZ * IY * (A(1, i, j, k + 1) - A(1, i, j, k) - A(1, i, j - 1, k + 1) + A(1, i, j - 1, k)) +
                 IX * IZ * (A(0, i, j, k + 1) - A(0, i, j, k) - A(0, i - 1, j, k + 1) + A(0, i - 1, j, k));
          }
          double ND1 = NEQ + N[c][id];
          double cb = fix ? cbrt(ND1) : (double)powf((float)ND1, (float)(1.0 / 3.0));
          s->Pd[c][id] = s->d1 * P[c][id] + s->d2 * s->Pd_n1[c][id] + s->d3 * s->E[c][id] +
                         s->d4 * s->En[c][id] + s->d5 * (0.0 + (s->mu0 * s->e0 / s->me) * 0.0 / s->z0) +
                         s->dNL * (gd + gd2 / NEQ) / cb;
          /* adjoint design region (no counterpart in the reference): the
           * current and density updates scale by rho (update_e_comp) */
          if (s->rho) s->Pd[c][id] *= s->rho[id];
        }
      }
#undef A
#undef AN
}

/* Curl of H at an E point (UPDATE_e* main.cu:1173, 1476, 1767). */
static inline double curl_h(const orc_sim* s, int c, int i, int j, int k) {
  double *const *H = s->H;
  size_t id = IDX(s, i, j, k);
  /* the -x and -y neighbours; periodic x and y wrap (main.cu:1074-1081) */
  int im = s->per && i == 0 ? s->NX - 1 : i - 1;
  int jm = s->per && j == 0 ? s->NY - 1 : j - 1;
  if (c == 0)
    return (H[2][id] - H[2][IDX(s, i, jm, k)]) / s->ked[1][j] -
           (H[1][id] - H[1][IDX(s, i, j, k - 1)]) / s->ked[2][k];
  if (c == 1)
    return (H[0][id] - H[0][IDX(s, i, j, k - 1)]) / s->ked[2][k] -
           (H[2][id] - H[2][IDX(s, im, j, k)]) / s->ked[0][i];
  return (H[1][id] - H[1][IDX(s, im, j, k)]) / s->ked[0][i] -
         (H[0][id] - H[0][IDX(s, i, jm, k)]) / s->ked[1][j];
}

/* Hydrodynamic continuity for the density perturbation of component c
 * (main.cu:1222-1239, 1527-1539, 1814-1826), from the currents and
 * densities before this component's update.  The z form keeps the
 * reference's 0.5*(Vz1-Vz2) term without the density factors. */
static double hydro_nd(const orc_sim* s, int c, int i, int j, int k) {
  double *const *P = s->Pd_n, *const *N = s->NDp;
  double NEQ = s->N_EQ;
  double dt = s->dt, IX = 1.0 / s->p.dx;
#define Q(a, ii, jj, kk) P[a][IDX(s, ii, jj, kk)]
#define M(a, ii, jj, kk) N[a][IDX(s, ii, jj, kk)]
  double V1[3], V2[3], N1[3], N2[3];
  int o[3] = {c == 0, c == 1, c == 2};
  for (int a = 0; a < 3; a++) {
    if (a == c) {
      V1[a] = Q(a, i + o[0], j + o[1], k + o[2]);
      V2[a] = Q(a, i - o[0], j - o[1], k - o[2]);
      N1[a] = M(a, i + o[0], j + o[1], k + o[2]);
      N2[a] = M(a, i - o[0], j - o[1], k - o[2]);
    } else {
      int b[3] = {a == 0, a == 1, a == 2};
      V1[a] = 0.5 * (Q(a, i + o[0], j + o[1], k + o[2]) + Q(a, i, j, k));
      V2[a] = 0.5 * (Q(a, i + o[0] - b[0], j + o[1] - b[1], k + o[2] - b[2]) +
                     Q(a, i - b[0], j - b[1], k - b[2]));
      N1[a] = 0.5 * (M(a, i + o[0], j + o[1], k + o[2]) + M(a, i, j, k));
      N2[a] = 0.5 * (M(a, i + o[0] - b[0], j + o[1] - b[1], k + o[2] - b[2]) +
                     M(a, i - b[0], j - b[1], k - b[2]));
    }
  }
#undef Q
#undef M
  double nd = s->ND[c][IDX(s, i, j, k)];
  if (c == 0)
    return nd - 2.0 * dt * IX *
                    (0.5 * (N1[0] * V1[0] - N2[0] * V2[0]) + (N1[1] * V1[1] - N2[1] * V2[1]) +
                     (N1[2] * V1[2] - N2[2] * V2[2]) +
                     (0.5 * (V1[0] - V2[0]) + (V1[1] - V2[1]) + (V1[2] - V2[2])) * NEQ);
  if (c == 1)
    return nd - 2.0 * dt * IX *
                    ((N1[0] * V1[0] - N2[0] * V2[0]) + 0.5 * (N1[1] * V1[1] - N2[1] * V2[1]) +
                     (N1[2] * V1[2] - N2[2] * V2[2]) +
                     ((V1[0] - V2[0]) + 0.5 * (V1[1] - V2[1]) + (V1[2] - V2[2])) * NEQ);
  return nd - 2.0 * dt * IX *
                  ((N1[0] * V1[0] - N2[0] * V2[0]) + (N1[1] * V1[1] - N2[1] * V2[1]) +
                   0.5 * (V1[2] - V2[2]) +
                   ((V1[0] - V2[0]) + (V1[1] - V2[1]) + 0.5 * (V1[2] - V2[2])) * NEQ);
}

/* UPDATE_ex / UPDATE_ey / UPDATE_ez (main.cu:1048-1912), run one component
 * after the other as the reference launches them.  Periodic x and y
 * (main.cu:1067-1090, 1359-1380, 1663-1690): every x and y index, the -1
 * neighbours wrap (curl_h), the z CPML only.
 * Within one component the hydrodynamic neighbour reads see the state from
 * before that component's launch (the reference races there; this is the
 * outcome when reads precede the neighbours' rotations). */
static void update_e_comp(orc_sim* s, int c) {
  int NX = s->NX, NY = s->NY, NZ = s->NZ;
  int lo[3] = {c == 0 ? 0 : 1, c == 1 ? 0 : 1, c == 2 ? 0 : 1};
  int hi[2] = {NX - 1, NY - 1};
  if (s->per) { lo[0] = lo[1] = 0; hi[0] = NX; hi[1] = NY; }
  double* E = s->E[c];
  int ax1 = (c + 1) % 3, ax2 = (c + 2) % 3; /* ex: y z; ey: z x; ez: x y */
  double dsp[3] = {s->p.dx, s->p.dy, s->p.dz};
  double* dnd = NULL;
  if (s->hydro) dnd = zalloc(s->n);
#pragma omp parallel for schedule(static)
  for (int i = lo[0]; i < hi[0]; i++)
    for (int j = lo[1]; j < hi[1]; j++)
      for (int k = lo[2]; k < NZ - 1; k++) {
        size_t id = IDX(s, i, j, k);
        double curl = curl_h(s, c, i, j, k);
        int v = s->matc[c][id];
        if (is_metal(s, v)) {
          double* cpn = &s->Pcp_n[c][2 * id];
          double* cpn1 = &s->Pcp_n1[c][2 * id];
          double CP2 = 0, CP4 = 0;
          for (int q = 0; q < 2; q++) { CP2 += (s->C1[q] - 1) * cpn[q]; CP4 += (s->C2[q]) * cpn1[q]; }
          if (!s->hydro) {
            double CP1 = 0, CP3 = 0, CPNL = 0;
            CP1 += (s->d1 - 1) * s->Pd_n[c][id];
            CP3 += (s->d2) * s->Pd_n1[c][id];
            CPNL += s->dNL * 0.0;
            /* adjoint design region (no counterpart in the reference): the
             * coupling coefficients blend linearly between vacuum (rho = 0)
             * and the metal (rho = 1); the pole dynamics stay the metal's */
            double CE = s->C_E, CE1 = s->C_E_1, CE2 = s->C_E_2, D3 = s->d3, D4 = s->d4, D5 = s->d5;
            double C3[2] = {s->C3[0], s->C3[1]}, C4[2] = {s->C4[0], s->C4[1]}, C5[2] = {s->C5[0], s->C5[1]};
            if (s->rho) {
              const double r = s->rho[id], vac = K_EP0;
              CE = vac + r * (s->C_E - vac);
              CE1 = vac + r * (s->C_E_1 - vac);
              CE2 = r * s->C_E_2;
              D3 = r * s->d3; D4 = r * s->d4; D5 = r * s->d5;
              for (int q = 0; q < 2; q++) { C3[q] = r * s->C3[q]; C4[q] = r * s->C4[q]; C5[q] = r * s->C5[q]; }
            }
            s->En1[c][id] = s->En[c][id];
            s->En[c][id] = E[id];
            E[id] = (1 / CE) * (s->dt * curl / s->z0 + CE1 * s->En[c][id] -
                                CE2 * s->En1[c][id] - CP1 - CP2 - CP3 - CP4 - CPNL);
            double en = s->En[c][id], en1 = s->En1[c][id];
            double ncp[2];
            for (int q = 0; q < 2; q++)
              ncp[q] = s->C1[q] * cpn[q] + s->C2[q] * cpn1[q] + C3[q] * E[id] + C4[q] * en + C5[q] * en1;
            double npd = s->d1 * s->Pd_n[c][id] + s->d2 * s->Pd_n1[c][id] + D3 * E[id] + D4 * en +
                         D5 * en1 + s->dNL * 0.0;
            s->Pd_n1[c][id] = s->Pd_n[c][id];
            s->Pd_n[c][id] = npd;
            for (int q = 0; q < 2; q++) { cpn1[q] = cpn[q]; cpn[q] = ncp[q]; }
          } else {
            double nd = hydro_nd(s, c, i, j, k);
            /* adjoint design region (no counterpart in the reference): a
             * design cell scales its current (hydro_p) and density updates
             * by rho and blends its coupling coefficients as in the local
             * model, so that rho = 0 is a vacuum cell with J = N = 0 */
            double CE = s->C_E, CE1 = s->C_E_1, CE2 = s->C_E_2;
            double C3[2] = {s->C3[0], s->C3[1]}, C4[2] = {s->C4[0], s->C4[1]}, C5[2] = {s->C5[0], s->C5[1]};
            if (s->rho) {
              const double r = s->rho[id], vac = K_EP0;
              nd = r * nd;
              CE = vac + r * (s->C_E - vac);
              CE1 = vac + r * (s->C_E_1 - vac);
              CE2 = r * s->C_E_2;
              for (int q = 0; q < 2; q++) { C3[q] = r * s->C3[q]; C4[q] = r * s->C4[q]; C5[q] = r * s->C5[q]; }
            }
            dnd[id] = nd;
            s->En1[c][id] = s->En[c][id];
            s->En[c][id] = E[id];
            E[id] = (1 / CE) * (s->dt * curl / s->z0 + s->dt * s->Pd[c][id] * s->e0 * (s->N_EQ + nd) +
                                CE1 * s->En[c][id] - CE2 * s->En1[c][id] - CP2 - CP4);
            double en = s->En[c][id], en1 = s->En1[c][id];
            double ncp[2];
            for (int q = 0; q < 2; q++)
              ncp[q] = s->C1[q] * cpn[q] + s->C2[q] * cpn1[q] + C3[q] * E[id] + C4[q] * en + C5[q] * en1;
            for (int q = 0; q < 2; q++) { cpn1[q] = cpn[q]; cpn[q] = ncp[q]; }
          }
        } else {
          E[id] = s->Cee * E[id] + (s->mat[id] == 6 ? s->Ceh_slab : s->Ceh) * curl;
        }
        /* CPML along the two transverse axes: for ex the z then y slabs
         * (main.cu:1294-1318); ey: z then x; ez: y then x. */
        int order[2];
        if (c == 0) { order[0] = 2; order[1] = 1; }
        else if (c == 1) { order[0] = 2; order[1] = 0; }
        else { order[0] = 1; order[1] = 0; }
        for (int q = 0; q < 2; q++) {
          int ax = order[q];
          if (s->per && ax < 2) continue;  /* no x or y CPML */
          int slot = ax == ax1 ? 0 : 1;
          int idx_ax = ax == 0 ? i : ax == 1 ? j : k;
          int Nc = s->Nc[ax];
          /* derivative of the H component that pairs with this axis */
          int hc = 3 - c - ax; /* the third component */
          double dh;
          if (ax == 0) dh = s->H[hc][id] - s->H[hc][IDX(s, i - 1, j, k)];
          else if (ax == 1) dh = s->H[hc][id] - s->H[hc][IDX(s, i, j - 1, k)];
          else dh = s->H[hc][id] - s->H[hc][IDX(s, i, j, k - 1)];
          /* sign: dE_c/dt has +dH_{c+2}/d_{c+1} - dH_{c+1}/d_{c+2} */
          double sg = (ax == ax1) ? 1.0 : -1.0;
          const cpml_axis* cpa = &s->cp[ax];
          int nlim = (c == 2 && ax == 1) ? Nc : Nc + 1; /* UPDATE_ez uses j<cpml_N_Y */
          if (idx_ax < nlim) {
            const double* ceN = cpa->ce_N;
            if (c == 1 && ax == 0 && !(s->p.fixes & FDTD_FIX_CE_EY_XN)) ceN = s->cp[1].ce_N;
            double* ps = &s->psiE_N[c][slot][pidx(s, ax, Nc + 1, i, j, k)];
            *ps = cpa->be_N[idx_ax] * *ps + ceN[idx_ax] * dh / dsp[ax];
            E[id] += sg * (s->Ceh * *ps);
          }
          if (idx_ax >= s->F[ax]) {
            int i2 = idx_ax - s->F[ax];
            int ii = ax == 0 ? i2 : i, jj = ax == 1 ? i2 : j, kk = ax == 2 ? i2 : k;
            double* ps = &s->psiE_F[c][slot][pidx(s, ax, Nc + 1, ii, jj, kk)];
            *ps = cpa->be_F[i2] * *ps + cpa->ce_F[i2] * dh / dsp[ax];
            E[id] += sg * (s->Ceh * *ps);
          }
        }
      }
  if (s->hydro) {
    /* rotations after the whole component (see the function comment) */
#pragma omp parallel for schedule(static)
    for (int i = lo[0]; i < NX - 1; i++)
      for (int j = lo[1]; j < NY - 1; j++)
        for (int k = lo[2]; k < NZ - 1; k++) {
          size_t id = IDX(s, i, j, k);
          if (!is_metal(s, s->matc[c][id])) continue;
          s->Pd_n2[c][id] = s->Pd_n1[c][id];
          s->Pd_n1[c][id] = s->Pd_n[c][id];
          s->Pd_n[c][id] = s->Pd[c][id];
          double hold = s->NDp[c][id];
          s->NDp[c][id] = dnd[id];
          s->ND[c][id] = hold;
        }
    free(dnd);
  }
}

/* ScattAbs (main.cu:35-366): E sampled at (t+1) dt, H at (t+1/2) dt, the
 * four tangential components of each face at the same integer cell. */
static void dft_accumulate(orc_sim* s) {
  static const int fcomp[3][4] = {{1, 2, 4, 5}, {0, 2, 3, 5}, {0, 1, 3, 4}};
  for (int b = 0; b < 2; b++)
    for (int f = 0; f < 6; f++)
      for (int c = 0; c < 4; c++)
        for (int r = 0; r < 2; r++)
          if (!s->dft[b][f][c][r])
            s->dft[b][f][c][r] = zalloc((size_t)s->NF * s->dft_a[b][f] * s->dft_b[b][f]);
  int t = s->t;
#pragma omp parallel for schedule(dynamic)
  for (int m = 0; m < s->NF; m++) {
    if (s->dft_sel && !s->dft_sel[m]) continue;
    double ph_e = (double)(float)2.0 * s->pi * (t + 1.0) * s->dt * s->freq[m];
    double ph_h = (double)(float)2.0 * s->pi * (t + 0.5) * s->dt * s->freq[m];
    double cre = cos(ph_e), cim = sin(ph_e), hre = cos(ph_h), him = sin(ph_h);
    /* periodic x and y: Ex, Ey, Hx, Hy on the reflection and transmission
     * planes (Fourier_Transform, Spectral.cu:32-120, which is not called
     * in the reference; sampled here with the phases of the box DFT) */
    for (int f = 0; f < 2 && s->per; f++) {
      int k = f == 0 ? s->k_refl : s->k_trans;
      int A = s->dft_a[0][f], B = s->dft_b[0][f];
      for (int i = 0; i < s->NX; i++)
        for (int j = 0; j < s->NY; j++) {
          size_t id = IDX(s, i, j, k);
          size_t o = ((size_t)m * A + i) * B + j;
          for (int c = 0; c < 4; c++) {
            int comp = fcomp[2][c];
            double x = comp < 3 ? s->E[comp][id] : s->H[comp - 3][id];
            s->dft[0][f][c][0][o] += x * (comp < 3 ? cre : hre);
            s->dft[0][f][c][1][o] += x * (comp < 3 ? cim : him);
          }
        }
    }
    for (int b = 0; b < 2 && !s->per; b++) {
      const int* S = b == 0 ? s->absS : s->scaS;
      const int* En = b == 0 ? s->absE : s->scaE;
      for (int f = 0; f < 6; f++) {
        int ax = f / 2;
        int a1 = ax == 0 ? 1 : 0, a2 = ax == 2 ? 1 : 2;
        int pos = (f & 1) ? En[ax] - 1 : S[ax];
        int A = s->dft_a[b][f], B = s->dft_b[b][f];
        for (int u = S[a1]; u < En[a1]; u++)
          for (int v = S[a2]; v < En[a2]; v++) {
            int ijk[3];
            ijk[ax] = pos; ijk[a1] = u; ijk[a2] = v;
            size_t id = IDX(s, ijk[0], ijk[1], ijk[2]);
            size_t o = ((size_t)m * A + (u - S[a1])) * B + (v - S[a2]);
            for (int c = 0; c < 4; c++) {
              int comp = fcomp[ax][c];
              double x = comp < 3 ? s->E[comp][id] : s->H[comp - 3][id];
              double wr = comp < 3 ? cre : hre, wi = comp < 3 ? cim : him;
              double* R = s->dft[b][f][c][0];
              double* Im = s->dft[b][f][c][1];
              if (s->float_dft) {
                float xf = (float)x;
                R[o] = (float)((double)(float)R[o] + (double)xf * wr);
                Im[o] = (float)((double)(float)Im[o] + (double)xf * wi);
              } else {
                R[o] += x * wr;
                Im[o] += x * wi;
              }
            }
          }
      }
    }
  }
}

void orc_step(orc_sim* s) {
  if (g_threads > 0) omp_set_num_threads(g_threads);
  if (s->per) update_h_periodic(s); else update_h(s);
  line_h(s);
  tfsf(s);
  line_e(s);
  if (s->hydro) hydro_p(s);
  for (int c = 0; c < 3; c++) update_e_comp(s, c);
  if (s->dft_on && s->p.StaticField == 0 && s->t % s->p.dft_every == 0) dft_accumulate(s);
  if (s->t <= s->p.Tend) {
    size_t id = IDX(s, s->pi_, s->pj, s->pk);
    for (int c = 0; c < 3; c++) s->probe[3 * (size_t)s->t + c] = s->E[c][id];
  }
  s->t++;
}

void orc_run(orc_sim* s, int nsteps) {
  for (int q = 0; q < nsteps; q++) orc_step(s);
}

/* ------------------------------------------------------------------ */
/* spectral post (CalculateAbsScatt, Spectral.cu:411-1177)             */

int orc_spectra(orc_sim* s, double* out) {
  static const int fcomp[3][4] = {{1, 2, 4, 5}, {0, 2, 3, 5}, {0, 1, 3, 4}};
  (void)fcomp;
  if (s->per) return -1;  /* no DFT box: orc_reflectance */
  for (int b = 0; b < 2; b++)
    for (int f = 0; f < 6; f++)
      if (!s->dft[b][f][0][0]) return -1;
  double dxy = s->p.dx * s->p.dy;
  for (int m = 0; m < s->NF; m++) {
    double Q[2][6];
    double amp = cabs(s->Einc[m]);
    float ampf = (float)amp;
    for (int b = 0; b < 2; b++)
      for (int f = 0; f < 6; f++) {
        int A = s->dft_a[b][f], B = s->dft_b[b][f];
        /* CalculateAbsScatt pairs the face's tangential phasors as
         * zz = cEx*conj(HY) - cEy*conj(HX) with, per face normal,
         * Z: (Ex, Ey, Hx, Hy)  Y: (Ez, Ex, Hz, Hx)  X: (Ey, Ez, Hy, Hz)
         * in our (Ea, Eb, Ha, Hb) slots: Y faces swap a and b. */
        int ax = f / 2;
        int qx = ax == 1 ? 1 : 0, qy = ax == 1 ? 0 : 1;
        double P = 0.0;
        for (int u = 0; u < A - 1; u++)
          for (int v = 0; v < B - 1; v++) {
            size_t o = ((size_t)m * A + u) * B + v;
            double exr = s->dft[b][f][qx][0][o], exi = s->dft[b][f][qx][1][o];
            double eyr = s->dft[b][f][qy][0][o], eyi = s->dft[b][f][qy][1][o];
            double hxr = s->dft[b][f][2 + qx][0][o], hxi = s->dft[b][f][2 + qx][1][o];
            double hyr = s->dft[b][f][2 + qy][0][o], hyi = s->dft[b][f][2 + qy][1][o];
            if (s->float_dft) {
              float complex cEx = (double)((float)exr / ampf) + I * (double)((float)exi / ampf);
              float complex cEy = (double)((float)eyr / ampf) + I * (double)((float)eyi / ampf);
              float complex ccHx = (double)((float)hxr / ampf) - I * (double)((float)hxi / ampf);
              float complex ccHy = (double)((float)hyr / ampf) - I * (double)((float)hyi / ampf);
              float complex zz = cEx * ccHy - cEy * ccHx;
              P += crealf(zz) * s->p.dx * s->p.dy;
            } else {
              P += (exr * hyr + exi * hyi) - (eyr * hxr + eyi * hxi);
            }
          }
        if (s->float_dft) Q[b][f] = (float)P;
        else Q[b][f] = P * dxy / (amp * amp);
      }
    double sca = -Q[1][0] + Q[1][1] - Q[1][2] + Q[1][3] - Q[1][4] + Q[1][5];
    double ab = -Q[0][0] + Q[0][1] - Q[0][2] + Q[0][3] - Q[0][4] + Q[0][5];
    int sphere = s->p.geometry == FDTD_GEOM_REFERENCE && s->p.nano_sphere == 1;
    if (sphere) {
      double r = s->p.nano_sphere_radius;
      sca = sca / (s->pi * r * r);
      ab = -ab / (s->pi * r * r);
    }
    double* row = out + 19 * (size_t)m;
    row[0] = s->c0 / s->freq[m];
    row[1] = sca; row[2] = ab; row[3] = ab + sca;
    for (int f = 0; f < 6; f++) { row[4 + f] = Q[1][f]; row[10 + f] = Q[0][f]; }
    row[16] = amp; row[17] = creal(s->Einc[m]); row[18] = cimag(s->Einc[m]);
  }
  return 0;
}

/* ------------------------------------------------------------------ */
/* accessors                                                           */

/* Reflectance_XZ (main.cu:3195-3320) on the two planes: per frequency
 * P = sum Re(Ey conj(Hx) - Ex conj(Hy)) dA; R = P_refl / (A |E_s|^2),
 * T = -P_trans / (A |E_s|^2) with A the plane's area and E_s = E_inc /
 * dft_every, the incident spectrum as the planes see it (they are sampled
 * every dft_every steps, E_inc sums every step).  P is reset for every
 * frequency (the reference's P_t is not).  out: lambda, R, T, 1 - R - T,
 * |E_inc|, Re E_inc, Im E_inc. */
int orc_reflectance(orc_sim* s, double* out) {
  if (!s->per || !s->dft[0][0][0][0]) return -1;
  double dA = s->p.dx * s->p.dy, area = 0.0;
  for (int i = 0; i < s->NX; i++)
    for (int j = 0; j < s->NY; j++) area += dA;
  for (int m = 0; m < s->NF; m++) {
    double P[2] = {0.0, 0.0};
    for (int f = 0; f < 2; f++) {
      int A = s->dft_a[0][f], B = s->dft_b[0][f];
      for (int i = 0; i < s->NX; i++)
        for (int j = 0; j < s->NY; j++) {
          size_t o = ((size_t)m * A + i) * B + j;
          double complex cEx = s->dft[0][f][0][0][o] + I * s->dft[0][f][0][1][o];
          double complex cEy = s->dft[0][f][1][0][o] + I * s->dft[0][f][1][1][o];
          double complex ccHx = s->dft[0][f][2][0][o] - I * s->dft[0][f][2][1][o];
          double complex ccHy = s->dft[0][f][3][0][o] - I * s->dft[0][f][3][1][o];
          P[f] += creal(cEy * ccHx - cEx * ccHy) * dA;
        }
    }
    double amp = cabs(s->Einc[m]), as = amp / s->p.dft_every;
    double R = P[0] / area / (as * as), T = -P[1] / area / (as * as);
    double* row = out + 7 * (size_t)m;
    row[0] = s->c0 / s->freq[m];
    row[1] = R; row[2] = T; row[3] = 1.0 - R - T;
    row[4] = amp; row[5] = creal(s->Einc[m]); row[6] = cimag(s->Einc[m]);
  }
  return 0;
}

void orc_dims(const orc_sim* s, fdtd_dims* d) {
  memset(d, 0, sizeof(*d));
  d->nx = s->NX; d->ny = s->NY; d->nz = s->NZ;
  d->ntfsf_x = s->Nt[0]; d->ntfsf_y = s->Nt[1]; d->ntfsf_z = s->Nt[2];
  d->inc_length = s->L; d->m0 = s->m0;
  for (int a = 0; a < 3; a++) {
    d->abs_start[a] = s->absS[a]; d->abs_end[a] = s->absE[a];
    d->sca_start[a] = s->scaS[a]; d->sca_end[a] = s->scaE[a];
  }
  d->num_freq = s->NF;
  for (int c = 0; c < 3; c++) {
    int n = 0;
    for (size_t q = 0; q < s->n; q++) n += is_metal(s, s->matc[c][q]);
    d->n_metal_cells[c] = n;
  }
  d->hydro = s->hydro;
  d->precision = FDTD_FP64;
  d->dt = s->dt; d->delay = s->delay; d->width = s->width;
}

int orc_get_field(const orc_sim* s, int comp, double* out, size_t n) {
  if (comp < 0 || comp > 5 || n != s->n) return -1;
  memcpy(out, comp < 3 ? s->E[comp] : s->H[comp - 3], n * sizeof(double));
  return 0;
}
int orc_set_field(orc_sim* s, int comp, const double* in, size_t n) {
  if (comp < 0 || comp > 5 || n != s->n) return -1;
  memcpy(comp < 3 ? s->E[comp] : s->H[comp - 3], in, n * sizeof(double));
  return 0;
}
int orc_get_material(const orc_sim* s, unsigned char* bits, int* mx, int* my, int* mz, size_t n) {
  if (n != s->n) return -1;
  for (size_t q = 0; q < n; q++) {
    unsigned char b = 0;
    for (int c = 0; c < 3; c++) b |= (unsigned char)(is_metal(s, s->matc[c][q]) << c);
    if (bits) bits[q] = b;
  }
  if (mx) memcpy(mx, s->matc[0], n * sizeof(int));
  if (my) memcpy(my, s->matc[1], n * sizeof(int));
  if (mz) memcpy(mz, s->matc[2], n * sizeof(int));
  return 0;
}
int orc_get_dft(const orc_sim* s, int box, int face, int comp, double* re, double* im, size_t n) {
  if (box < 0 || box > 1 || face < 0 || face > 5 || comp < 0 || comp > 3) return -1;
  size_t need = (size_t)s->NF * s->dft_a[box][face] * s->dft_b[box][face];
  if (n != need || !s->dft[box][face][comp][0]) return -1;
  memcpy(re, s->dft[box][face][comp][0], n * sizeof(double));
  memcpy(im, s->dft[box][face][comp][1], n * sizeof(double));
  return 0;
}
int orc_get_freqs(const orc_sim* s, double* f, size_t n) {
  if (n != (size_t)s->NF) return -1;
  memcpy(f, s->freq, n * sizeof(double));
  return 0;
}
int orc_get_incident(const orc_sim* s, double* re, double* im, size_t n) {
  if (n != (size_t)s->NF) return -1;
  for (size_t m = 0; m < n; m++) { re[m] = creal(s->Einc[m]); im[m] = cimag(s->Einc[m]); }
  return 0;
}
int orc_get_state(const orc_sim* s, int which, int comp, double* out, size_t n) {
  if (n != s->n || comp < 0 || comp > 2) return -1;
  if (which < 0 || which > 2) return -1;
  const double* src = which == 0 ? s->Pd_n[comp] : which == 1 ? s->ND[comp] : s->NDp[comp];
  if (src) memcpy(out, src, n * sizeof(double));
  else memset(out, 0, n * sizeof(double)); /* no density without the hydrodynamic model */
  return 0;
}
int orc_get_line(const orc_sim* s, double* e, double* h, size_t n) {
  if (n != (size_t)s->L) return -1;
  memcpy(e, s->e_inc, n * sizeof(double));
  memcpy(h, s->h_inc, n * sizeof(double));
  return 0;
}
int orc_get_probe(const orc_sim* s, double* out, size_t n) {
  size_t m = (size_t)3 * s->t;
  if (n < m) m = n;
  memcpy(out, s->probe, m * sizeof(double));
  return (int)(m / 3);
}
int orc_get_cpml(const orc_sim* s, int which, double* out, size_t n) {
  int NN[3] = {s->NX, s->NY, s->NZ};
  if (which >= 0 && which < 6) {
    int ax = which % 3;
    const double* t = which < 3 ? s->ked[ax] : s->khd[ax];
    if (n < (size_t)NN[ax]) return -1;
    memcpy(out, t, NN[ax] * sizeof(double));
    return NN[ax];
  }
  which -= 6;
  if (which < 0 || which >= 24) return -1;
  int ax = which / 8, slot = which % 8;
  const cpml_axis* c = &s->cp[ax];
  const double* tabs[8] = {c->be_N, c->ce_N, c->be_F, c->ce_F, c->bh_N, c->ch_N, c->bh_F, c->ch_F};
  int len = slot < 4 ? s->Nc[ax] + 1 : s->Nc[ax];
  if (len < 0) len = 0;
  if (n < (size_t)len) return -1;
  memcpy(out, tabs[slot], len * sizeof(double));
  return len;
}
int orc_get_ade(const orc_sim* s, double* o, size_t n) {
  if (n < 22) return -1;
  double v[22] = {s->C_E, s->C_E_1, s->C_E_2, s->d1, s->d2, s->d3, s->d4, s->d5, s->dNL,
                  s->C1[0], s->C2[0], s->C3[0], s->C4[0], s->C5[0],
                  s->C1[1], s->C2[1], s->C3[1], s->C4[1], s->C5[1], s->dt, s->N_EQ, 0};
  memcpy(o, v, sizeof(v));
  return 22;
}
