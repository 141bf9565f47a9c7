// Host-side setup of a simulation: derived sizes, material rasterisation,
// coefficient tables, incident pulse and spectrum.  Everything is computed
// in FP64 on the host with the reference's formulas and then uploaded.
#pragma once
#include <complex>
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/fdtd_b200.h"

namespace fdtd {

struct CpmlTables {
  std::vector<double> ked, khd;              // kappa * d per index (N)
  std::vector<double> be_N, ce_N, be_F, ce_F;  // Nc+1
  std::vector<double> bh_N, ch_N, bh_F, ch_F;  // Nc
};

struct Setup {
  fdtd_params p;
  int NX = 0, NY = 0, NZ = 0;
  int Nc[3] = {0, 0, 0}, F[3] = {0, 0, 0}, Nt[3] = {0, 0, 0};
  int absS[3], absE[3], scaS[3], scaE[3];
  int k_refl = 0, k_trans = 0;  // periodic_xy: reflection and transmission planes
  int L = 0, m0 = 0, i0 = 0, j0 = 0, k0 = 0;
  double d1D = 0, dt = 0, delay = 0, width = 0, f0 = 0;
  double z0, ep0, mu0, c0, pi, e0, me;
  bool hydro = false;
  // Yee coefficients (uniform medium: eps = EP0, mu = MU0, sigma = 0)
  double Cee = 1, Ceh = 0, Chh = 1, Che = 0;
  double Ceh_slab = 0;  // E-on-H coefficient of the dielectric slab class (eps = slab_eps)
  CpmlTables cp[3];
  // ADE
  double C_E = 0, C_E_1 = 0, C_E_2 = 0, d1 = 0, d2 = 0, d3 = 0, d4 = 0, d5 = 0, dNL = 0, N_EQ = 0;
  double wD = 0, gam = 0;  // Drude plasma frequency and damping in use
  double C1[2], C2[2], C3[2], C4[2], C5[2];
  // TFSF
  float sth, cth, sph, cph, fe[3], fh[3];
  // spectra
  std::vector<double> freq;
  std::vector<std::complex<double>> Einc;
  std::vector<double> pulse;  // source value injected at step t, t = 0..Tend
  // material: per-component class (reference's mat_matrixX/Y/Z values),
  // reference layout [i][j][k]
  std::vector<int> matc[3];
  int probe[3];
};

const char* setup_build(const fdtd_params& p, Setup& s);  // nullptr on success
void params_default(fdtd_params* p);
int read_input_txt(const char* path, fdtd_params* p);
int write_input_txt(const char* path, const fdtd_params* p);

inline bool is_dispersive(int v) { return v > 1 && v < 6; }
// material value of the dielectric slab (non-dispersive, eps = slab_eps)
constexpr int kSlabMaterial = 6;

}  // namespace fdtd
