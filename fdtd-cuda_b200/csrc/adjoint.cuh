// Reverse-time discrete adjoint of the time step (no counterpart in the
// reference).  The step without the hydrodynamic model is linear in the
// state (E, H, the CPML psi, the dispersive-cell ADE states) plus sources
// that do not depend on it (TFSF corrections, the 1D line), so its adjoint
// is the transposed step run backwards:
//
//   lambda^n = M^T lambda^{n+1} + dL/dx^n,   dL/drho = sum_n lambda^{n+1} (dM/drho) x^n
//
// The transposed Yee/CPML sub-steps are written in gather form: a first
// kernel turns each updated component's adjoint into the coefficients of
// the field differences it read ("a" arrays, one per component and
// difference axis) and applies the psi recursions transposed; a second
// kernel gathers those coefficients into the adjoint of the other field
// (each difference D = F(p) - F(p - e) read by cell p contributes +a(p) to
// F(p) and -a(p) to F(p - e)).  The dispersive (design) cells transpose
// their ADE recursions locally and accumulate dL/drho and the Drude
// parameter gradients from the forward values recorded during the segment
// recompute.  Objective: any linear combination of the ScatAbs table
// (the totals and the 12 face fluxes at every frequency), each a bilinear
// form of the DFT accumulators, whose derivative enters at every DFT
// sample step.
#pragma once
#include "kernels.cuh"
#include "staged.cuh"

namespace fdtd {

template <typename T>
struct AdjView {
  T* lE[3];
  T* lH[3];
  T* lpE_N[3][2];
  T* lpE_F[3][2];
  T* lpH_N[3][2];
  T* lpH_F[3][2];
  T* a[3][2];  // difference coefficients of component c, slot q (axis (c+1+q)%3)
  // dispersive-cell adjoint states per component slot: Drude current J^{n+1}
  // and J^n, the two CP polarisations P^{n+1} and P^n, the E history
  T* lJa[3];
  T* lJb[3];
  T* lPa[3][2];
  T* lPb[3][2];
  T* lEh[3];
  double* grho[3];  // dL/drho per slot
  double* gpar;     // [2]: dL/d omega_D, dL/d gamma
  // hydrodynamic cells: adjoints of the current J and the density N of
  // component c at time m in ring slot m % 3 (FP64, like their forward state)
  double* lJ[3][3];
  double* lN[3][3];
  // hydrodynamic model: d/d gamma of d1, d2, d3, d4, dNL
  double dgam[5];
  // derivatives of the metal coefficients: [p] = d/d omega_D, d/d gamma
  T dCE[2], dCE1[2], dCE2[2], dd1[2], dd2[2], dd3[2], dd4[2], dd5[2];
  int* step;        // adjoint clock: the step being transposed
  unsigned* flags;  // per cell: adj_flags_e | adj_flags_h << 16 (adj_build_flags)
};

// psi element of component c, slot q at cell (i, j, k) for slab axis ax;
// returns nullptr outside the slab.  w = slab width (Nc+1 for E, Nc for H).
template <typename T>
__device__ __forceinline__ T* adj_psi(const SimView<T>& s, T* const* nearp, T* const* farp, int ax, bool e_extent,
                                      int i, int j, int k, int* qout) {
  const CpmlAxis<T>& a = s.cp[ax];
  const int n = ax == 0 ? i : ax == 1 ? j : k;
  const int w = e_extent ? a.Nc + 1 : a.Nc;
  if (e_extent ? n <= a.Nc : n < a.Nc) {
    *qout = n;
    return nearp[0] + slab_idx(s, ax, w, i, j, k);
  }
  if (n >= a.F) {
    const int q2 = n - a.F;
    *qout = -1 - q2;  // far side, index q2
    return farp[0] + slab_idx(s, ax, w, ax == 0 ? q2 : i, ax == 1 ? q2 : j, ax == 2 ? q2 : k);
  }
  return nullptr;
}

// E sub-step transposed, per cell: coefficients of the H differences, the
// old-E adjoint and the psi_E adjoints.  Dispersive components are left to
// adj_e_design (their coefficients are zeroed here).
template <typename T>
__global__ void adj_e_coef(const __grid_constant__ SimView<T> s, const __grid_constant__ AdjView<T> a) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long n = (long long)s.NX * s.NY * s.NZ;
  if (q >= n) return;
  const int i = (int)(q % s.NX);
  const long long r = q / s.NX;
  const int j = (int)(r % s.NY), k = (int)(r / s.NY);
  const size_t id = fidx(s.PX, s.plane, i, j, k);
  unsigned m = 0;
  if (i >= s.mat_lo[0] && i < s.mat_hi[0] && j >= s.mat_lo[1] && j < s.mat_hi[1] && k >= s.mat_lo[2] &&
      k < s.mat_hi[2])
    m = s.mat[id];
  const T cee = s.cee[m >> 3], ceh = s.ceh[m >> 3];
  const int NX = s.NX, NY = s.NY, NZ = s.NZ;
  const int ijk[3] = {i, j, k};
#pragma unroll
  for (int c = 0; c < 3; c++) {
    // active range of component c (main.cu:1172, 1476, 1767)
    bool act = true;
#pragma unroll
    for (int d = 0; d < 3; d++) {
      const int N = d == 0 ? NX : d == 1 ? NY : NZ;
      if (ijk[d] >= N - 1) act = false;
      if (d != c && ijk[d] < 1) act = false;
    }
    if (!act || (m & (1u << c))) {
      a.a[c][0][id] = T(0);
      a.a[c][1][id] = T(0);
      continue;  // not updated (or dispersive): adjoint passes through here
    }
    const T lam = a.lE[c][id];
#pragma unroll
    for (int sl = 0; sl < 2; sl++) {
      const int ax = (c + 1 + sl) % 3;
      const T sg = sl == 0 ? T(1) : T(-1);
      const CpmlAxis<T>& cp = s.cp[ax];
      const int nn = ijk[ax];
      T coef = sg * ceh * ldg(cp.inv_ked + nn) * lam;
      int qs;
      T* lp = adj_psi(s, &a.lpE_N[c][sl], &a.lpE_F[c][sl], ax, true, i, j, k, &qs);
      if (lp) {
        T b, cc;
        if (qs >= 0) {
          b = ldg(cp.be_N + qs);
          cc = ldg(((c == 1 && ax == 0) ? cp.ce_N_ey : cp.ce_N) + qs);
        } else {
          b = ldg(cp.be_F + (-1 - qs));
          cc = ldg(cp.ce_F + (-1 - qs));
        }
        const T tot = *lp + sg * ceh * lam;
        *lp = b * tot;
        coef += cc * cp.inv_d * tot;
      }
      a.a[c][sl][id] = coef;
    }
    a.lE[c][id] = cee * lam;
  }
}

// Dispersive (design) cells, transposed: one thread per (component, cell).
// The forward map is
//   nv  = (dt/z0 curl + CE1 v - CE2 e1 - (d1-1) J - d2 Jm - sum (C1q-1) Pq - C2q Pqm) / CE
//   Pq' = C1q Pq + C2q Pqm + C3q nv + C4q v + C5q e1,   J' = d1 J + d2 Jm + d3 nv + d4 v + d5 e1
// with v = E^n, e1 = E^{n-1}; the coupling coefficients are blended by rho.
template <typename T>
__global__ void adj_e_design(const __grid_constant__ SimView<T> s, const __grid_constant__ MetalView<T> m,
                             const __grid_constant__ AdjView<T> a, const T* __restrict__ rec, int rec_rows) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  int c = 0;
  while (c < 3 && q >= m.n[c]) { q -= m.n[c]; c++; }
  double gp0 = 0, gp1 = 0;
  if (c < 3) {
    const int4 e = m.cell[c][q];
    const int sl = e.w;
    const size_t id = fidx(s.PX, s.plane, e.x, e.y, e.z);
    const int n = *a.step;
    const T* r = rec + rec_row(n, m.rec_base, rec_rows) * 5 * m.rec_slots + m.rec_off[c] + sl;
    const T v = r[0], e1 = r[m.rec_slots], J = r[2 * m.rec_slots], Jm = r[3 * m.rec_slots],
            nv = r[4 * m.rec_slots];
    const T rho = m.rho[c] ? (T)m.rho[c][sl] : T(1);
    const T CE = (T)(m.vac + rho * (m.C_E - m.vac)), CE1 = (T)(m.vac + rho * (m.C_E_1 - m.vac));
    const T CE2 = (T)(rho * m.C_E_2);
    const T D3 = (T)(rho * m.d3), D4 = (T)(rho * m.d4), D5 = (T)(rho * m.d5);
    const T C3[2] = {(T)(rho * m.C3[0]), (T)(rho * m.C3[1])}, C4[2] = {(T)(rho * m.C4[0]), (T)(rho * m.C4[1])},
            C5[2] = {(T)(rho * m.C5[0]), (T)(rho * m.C5[1])};
    const T lnv = a.lE[c][id];
    const T al = a.lJa[c][sl], be = a.lJb[c][sl], ep = a.lEh[c][sl];
    const T aq[2] = {a.lPa[c][0][sl], a.lPa[c][1][sl]}, bq[2] = {a.lPb[c][0][sl], a.lPb[c][1][sl]};
    const T Lam = lnv + C3[0] * aq[0] + C3[1] * aq[1] + D3 * al;
    const T mu = Lam / CE;
    // adjoint of E^n (the field and the stored history both read it)
    a.lE[c][id] = CE1 * mu + C4[0] * aq[0] + C4[1] * aq[1] + D4 * al + ep;
    // curl(H) coefficients: nv has dt/z0 curl/CE, curl = s0 ik0 D0 + s1 ik1 D1
    const int ijk[3] = {e.x, e.y, e.z};
    const T f = m.dt / m.z0 * mu;
#pragma unroll
    for (int sq = 0; sq < 2; sq++) {
      const int ax = (c + 1 + sq) % 3;
      a.a[c][sq][id] = (sq == 0 ? f : -f) * ldg(s.cp[ax].inv_ked + ijk[ax]);
    }
    // states one step back
    a.lJa[c][sl] = be + m.d1 * al - (m.d1 - T(1)) * mu;
    a.lJb[c][sl] = m.d2 * al - m.d2 * mu;
#pragma unroll
    for (int p = 0; p < 2; p++) {
      a.lPa[c][p][sl] = bq[p] + m.C1[p] * aq[p] - (m.C1[p] - T(1)) * mu;
      a.lPb[c][p][sl] = m.C2[p] * aq[p] - m.C2[p] * mu;
    }
    a.lEh[c][sl] = -CE2 * mu + C5[0] * aq[0] + C5[1] * aq[1] + D5 * al;
    // dL/drho: every coupling coefficient is vac + rho (metal - vac)
    const double g = (double)mu * (-(double)nv * ((double)m.C_E - (double)m.vac) +
                                   (double)v * ((double)m.C_E_1 - (double)m.vac) - (double)e1 * (double)m.C_E_2) +
                     (double)aq[0] * ((double)nv * m.C3[0] + (double)v * m.C4[0] + (double)e1 * m.C5[0]) +
                     (double)aq[1] * ((double)nv * m.C3[1] + (double)v * m.C4[1] + (double)e1 * m.C5[1]) +
                     (double)al * ((double)nv * m.d3 + (double)v * m.d4 + (double)e1 * m.d5);
    a.grho[c][sl] += g;
    // Drude parameters: coupling terms scale with rho, the pole dynamics
    // (d1, d2) do not
    double gpp[2];
#pragma unroll
    for (int p = 0; p < 2; p++)
      gpp[p] = (double)rho * ((double)mu * (-(double)nv * a.dCE[p] + (double)v * a.dCE1[p] - (double)e1 * a.dCE2[p]) +
                              (double)al * ((double)nv * a.dd3[p] + (double)v * a.dd4[p] + (double)e1 * a.dd5[p])) +
               ((double)al - (double)mu) * ((double)J * a.dd1[p] + (double)Jm * a.dd2[p]);
    gp0 = gpp[0];
    gp1 = gpp[1];
  }
  // block sum of the parameter gradients
  __shared__ double red[2][32];
  for (int o = 16; o > 0; o >>= 1) {
    gp0 += __shfl_down_sync(0xffffffffu, gp0, o);
    gp1 += __shfl_down_sync(0xffffffffu, gp1, o);
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) { red[0][w] = gp0; red[1][w] = gp1; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double s0 = 0, s1 = 0;
    for (int x = 0; x < (int)(blockDim.x >> 5); x++) { s0 += red[0][x]; s1 += red[1][x]; }
    if (s0 != 0.0) atomicAdd(a.gpar, s0);
    if (s1 != 0.0) atomicAdd(a.gpar + 1, s1);
  }
}

// ---------------------------------------------------------------------
// Hydrodynamic cells, transposed.  The forward step (kernels.cuh) is three
// phases: hydro_p_ex computes J^{n+1} of every cell from J^n, J^{n-1},
// E^n, E^{n-1} and the pressure term over the neighbour slots' J^n and
// N^n, then the x cells' continuity and E update; hydro_e<1> and <2> do the
// y and z cells, whose continuity reads the x (and y) neighbours' new J and
// N.  Linearised about the recorded trajectory (MetalView::hrec, ::rec),
// the reverse step runs adj_hydro_e<2>, <1>, <0> (E update and continuity
// of each phase, in reverse order), then adj_hydro_j (the current update).
// A slot's J or N adjoint receives terms from its neighbours, added with
// FP64 atomics.  Design cells: J' = rho (update), N' = rho (update), the
// coupling coefficients blended as in the local model.
//
// Neighbour slots per cell of component c and component a (nbr, 12 per
// cell): a == c: +e_c, 0, -e_c, unused; a != c: +e_c, 0, +e_c - e_a, -e_a.

template <typename T>
__device__ __forceinline__ void adj_hydro_blend(const MetalView<T>& m, bool blend, double r, double& CE,
                                                double& CE1, double& CE2, double C3[2], double C4[2],
                                                double C5[2]) {
  CE = m.C_E; CE1 = m.C_E_1; CE2 = m.C_E_2;
#pragma unroll
  for (int q = 0; q < 2; q++) { C3[q] = m.C3[q]; C4[q] = m.C4[q]; C5[q] = m.C5[q]; }
  if (blend) {
    CE = m.vac + r * (m.C_E - m.vac);
    CE1 = m.vac + r * (m.C_E_1 - m.vac);
    CE2 = r * m.C_E_2;
#pragma unroll
    for (int q = 0; q < 2; q++) { C3[q] = r * m.C3[q]; C4[q] = r * m.C4[q]; C5[q] = r * m.C5[q]; }
  }
}

// The E update and the continuity of the cells of component c, transposed.
template <typename T, int c>
__global__ void adj_hydro_e(const __grid_constant__ SimView<T> s, const __grid_constant__ MetalView<T> m,
                            const __grid_constant__ AdjView<T> a) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= m.n[c]) return;
  const int4 e = m.cell[c][q];
  const int sl = e.w;
  const size_t id = fidx(s.PX, s.plane, e.x, e.y, e.z);
  const int n = *a.step;
  const size_t row = rec_row(n, m.rec_base, m.rec_rows);
  const long long S = m.rec_slots;
  const T* rec = m.rec + (size_t)row * 5 * S + m.rec_off[c] + sl;
  const double v = (double)rec[0], e1 = (double)rec[S], nv = (double)rec[4 * S];
  const T* h = m.hrec + (size_t)row * 6 * S;
  const long long own = m.rec_off[c] + sl;
  const double Jn1 = h[2 * S + own], Nm1 = h[3 * S + own], Nn1 = h[5 * S + own];
  const bool blend = m.rho[c] != nullptr;
  const double r = blend ? (double)m.rho[c][sl] : 1.0;
  double CE, CE1, CE2, C3[2], C4[2], C5[2];
  adj_hydro_blend(m, blend, r, CE, CE1, CE2, C3, C4, C5);
  const int r1 = (n + 1) % 3, r0 = n % 3, rm = (n + 2) % 3;
  // E update: nv = (dt/z0 curl + dt e0 J' (N_EQ + N') + CE1 v - CE2 e1 - sum (C1q-1) Pq + C2q Pqm) / CE
  const double lnv = (double)a.lE[c][id];
  const double aq[2] = {(double)a.lPa[c][0][sl], (double)a.lPa[c][1][sl]};
  const double bq[2] = {(double)a.lPb[c][0][sl], (double)a.lPb[c][1][sl]};
  const double ep = (double)a.lEh[c][sl];
  const double mu = (lnv + C3[0] * aq[0] + C3[1] * aq[1]) / CE;
  a.lE[c][id] = (T)(CE1 * mu + C4[0] * aq[0] + C4[1] * aq[1] + ep);
  const int ijk[3] = {e.x, e.y, e.z};
  const double f = m.dt / m.z0 * mu;
#pragma unroll
  for (int sq = 0; sq < 2; sq++) {
    const int ax = (c + 1 + sq) % 3;
    a.a[c][sq][id] = (T)((sq == 0 ? f : -f) * (double)ldg(s.cp[ax].inv_ked + ijk[ax]));
  }
#pragma unroll
  for (int p = 0; p < 2; p++) {
    a.lPa[c][p][sl] = (T)(bq[p] + m.C1[p] * aq[p] - (m.C1[p] - 1.0) * mu);
    a.lPb[c][p][sl] = (T)(m.C2[p] * aq[p] - m.C2[p] * mu);
  }
  a.lEh[c][sl] = (T)(-CE2 * mu + C5[0] * aq[0] + C5[1] * aq[1]);
  const double src = mu * m.dt * m.e0;
  a.lJ[c][r1][sl] += src * (m.N_EQ + Nn1);
  const double lNp = a.lN[c][r1][sl] + src * Jn1;  // complete: later phases have run
  a.lN[c][r1][sl] = 0.0;
  double g = mu * (-nv * (m.C_E - m.vac) + v * (m.C_E_1 - m.vac) - e1 * m.C_E_2);
#pragma unroll
  for (int p = 0; p < 2; p++) g += aq[p] * (nv * m.C3[p] + v * m.C4[p] + e1 * m.C5[p]);
  // continuity: N' = r (N^{n-1} - k2 B), B over the neighbours' J and N at
  // n + 1 for the components updated before c, at n for the others
  const double rl = r * lNp;
  a.lN[c][rm][sl] += rl;
  const int* nb = m.nbr[c] + (size_t)q * 12;
  double P[3][4], N[3][4];
#pragma unroll
  for (int b = 0; b < 3; b++) {
    const int vj = b < c ? 2 : 1, vn = b < c ? 5 : 4;
#pragma unroll
    for (int x = 0; x < 4; x++) {
      const int o = nb[b * 4 + x];
      P[b][x] = o >= 0 ? h[vj * S + m.rec_off[b] + o] : 0.0;
      N[b][x] = o >= 0 ? h[vn * S + m.rec_off[b] + o] : 0.0;
    }
  }
  double V1[3], V2[3], N1[3], N2[3];
#pragma unroll
  for (int b = 0; b < 3; b++) {
    if (b == c) {
      V1[b] = P[b][0]; V2[b] = P[b][2]; N1[b] = N[b][0]; N2[b] = N[b][2];
    } else {
      V1[b] = 0.5 * (P[b][0] + P[b][1]);
      V2[b] = 0.5 * (P[b][2] + P[b][3]);
      N1[b] = 0.5 * (N[b][0] + N[b][1]);
      N2[b] = 0.5 * (N[b][2] + N[b][3]);
    }
  }
  const double k2 = 2.0 * m.dt * m.inv_dx;
  double B = 0.0;
  double dN1[3], dN2[3], dV1[3], dV2[3];  // dB / d(each averaged value)
#pragma unroll
  for (int b = 0; b < 3; b++) {
    const double w = b == c ? 0.5 : 1.0;
    if (c == 2 && b == 2) {
      // the z form carries 0.5 (V1z - V2z) without the density factors
      B += 0.5 * (V1[b] - V2[b]) + 0.5 * (V1[b] - V2[b]) * m.N_EQ;
      dN1[b] = 0.0; dN2[b] = 0.0;
      dV1[b] = 0.5 + 0.5 * m.N_EQ; dV2[b] = -(0.5 + 0.5 * m.N_EQ);
    } else {
      B += w * (N1[b] * V1[b] - N2[b] * V2[b]) + w * (V1[b] - V2[b]) * m.N_EQ;
      dN1[b] = w * V1[b]; dN2[b] = -w * V2[b];
      dV1[b] = w * (N1[b] + m.N_EQ); dV2[b] = -w * (N2[b] + m.N_EQ);
    }
  }
  g += lNp * (Nm1 - k2 * B);
  const double kk = -k2 * rl;
#pragma unroll
  for (int b = 0; b < 3; b++) {
    const int ring = b < c ? r1 : r0;
    double* lJb = a.lJ[b][ring];
    double* lNb = a.lN[b][ring];
    if (b == c) {
      const int o0 = nb[b * 4 + 0], o2 = nb[b * 4 + 2];
      if (o0 >= 0) { atomicAdd(lJb + o0, kk * dV1[b]); atomicAdd(lNb + o0, kk * dN1[b]); }
      if (o2 >= 0) { atomicAdd(lJb + o2, kk * dV2[b]); atomicAdd(lNb + o2, kk * dN2[b]); }
    } else {
#pragma unroll
      for (int x = 0; x < 4; x++) {
        const int o = nb[b * 4 + x];
        if (o < 0) continue;
        const double dv = x < 2 ? dV1[b] : dV2[b], dn = x < 2 ? dN1[b] : dN2[b];
        atomicAdd(lJb + o, 0.5 * kk * dv);
        atomicAdd(lNb + o, 0.5 * kk * dn);
      }
    }
  }
  a.grho[c][sl] += g;
}

// The current update of every hydrodynamic cell, transposed:
// J' = r (d1 J + d2 Jm + d3 E + d4 Em + dNL (gd + gd2 / N_EQ) / cb), gd and
// gd2 the stencil sums of J and of J N over the neighbour slots at time n,
// cb = (N_EQ + N)^(1/3) of the cell (the reference's FP32 powf is locally
// constant in N; with the cube-root fix its derivative is kept).
template <typename T>
__global__ void adj_hydro_j(const __grid_constant__ SimView<T> s, const __grid_constant__ MetalView<T> m,
                            const __grid_constant__ AdjView<T> a) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  int c = 0;
  while (c < 3 && q >= m.n[c]) { q -= m.n[c]; c++; }
  double gg = 0.0;
  if (c < 3) {
    const int4 e = m.cell[c][q];
    const int sl = e.w;
    const size_t id = fidx(s.PX, s.plane, e.x, e.y, e.z);
    const int n = *a.step;
    const size_t row = rec_row(n, m.rec_base, m.rec_rows);
    const long long S = m.rec_slots;
    const T* rec = m.rec + (size_t)row * 5 * S + m.rec_off[c] + sl;
    const double v = (double)rec[0], e1 = (double)rec[S];
    const T* h = m.hrec + (size_t)row * 6 * S;
    const long long own = m.rec_off[c] + sl;
    const double Jm = h[own], J = h[S + own];
    const int r1 = (n + 1) % 3, r0 = n % 3, rm = (n + 2) % 3;
    const double lJp = a.lJ[c][r1][sl];
    a.lJ[c][r1][sl] = 0.0;
    const bool blend = m.rho[c] != nullptr;
    const double r = blend ? (double)m.rho[c][sl] : 1.0;
    const double rl = r * lJp;
    atomicAdd(a.lJ[c][r0] + sl, m.d1 * rl);
    a.lJ[c][rm][sl] += m.d2 * rl;
    a.lE[c][id] += (T)(m.d3 * rl);
    a.lEh[c][sl] += (T)(m.d4 * rl);
    // pressure term over the neighbour slots at time n
    const int* nb = m.nbr[c] + (size_t)q * 12;
    const double I3[3] = {m.inv_dx, m.inv_dy, m.inv_dz};
    double wgt[3][4], P[3][4], N[3][4];
#pragma unroll
    for (int b = 0; b < 3; b++) {
      const double kb = b == c ? I3[c] * I3[c] : I3[b < c ? b : c] * I3[b < c ? c : b];
      if (b == c) { wgt[b][0] = kb; wgt[b][1] = -2.0 * kb; wgt[b][2] = kb; wgt[b][3] = 0.0; }
      else { wgt[b][0] = kb; wgt[b][1] = -kb; wgt[b][2] = -kb; wgt[b][3] = kb; }
#pragma unroll
      for (int x = 0; x < 4; x++) {
        const int o = nb[b * 4 + x];
        P[b][x] = o >= 0 ? h[S + m.rec_off[b] + o] : 0.0;
        N[b][x] = o >= 0 ? h[4 * S + m.rec_off[b] + o] : 0.0;
      }
    }
    double gd = 0.0, gd2 = 0.0;
#pragma unroll
    for (int b = 0; b < 3; b++)
#pragma unroll
      for (int x = 0; x < 4; x++) { gd += wgt[b][x] * P[b][x]; gd2 += wgt[b][x] * P[b][x] * N[b][x]; }
    const double ND1 = m.N_EQ + N[c][1];
    const double cb = m.fix_cbrt ? cbrt(ND1) : (double)powf((float)ND1, (float)(1.0 / 3.0));
    const double pr = (gd + gd2 / m.N_EQ) / cb;
    const double gp = rl * m.dNL / cb;
#pragma unroll
    for (int b = 0; b < 3; b++)
#pragma unroll
      for (int x = 0; x < 4; x++) {
        const int o = nb[b * 4 + x];
        if (o < 0 || wgt[b][x] == 0.0) continue;
        atomicAdd(a.lJ[b][r0] + o, gp * wgt[b][x] * (1.0 + N[b][x] / m.N_EQ));
        atomicAdd(a.lN[b][r0] + o, gp * wgt[b][x] * P[b][x] / m.N_EQ);
      }
    if (m.fix_cbrt) atomicAdd(a.lN[c][r0] + sl, -rl * m.dNL * pr / (3.0 * ND1));
    a.grho[c][sl] += lJp * (m.d1 * J + m.d2 * Jm + m.d3 * v + m.d4 * e1 + m.dNL * pr);
    gg = rl * (a.dgam[0] * J + a.dgam[1] * Jm + a.dgam[2] * v + a.dgam[3] * e1 + a.dgam[4] * pr);
  }
  __shared__ double red[32];
  for (int o = 16; o > 0; o >>= 1) gg += __shfl_down_sync(0xffffffffu, gg, o);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) red[w] = gg;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int x = 0; x < (int)(blockDim.x >> 5); x++) t += red[x];
    if (t != 0.0) atomicAdd(a.gpar + 1, t);
  }
}

// lambda_H += gather of the E-sub-step coefficients: H component h is read
// by the E components c != h through D = H_h(p) - H_h(p - e_ax), ax the
// third axis.
template <typename T>
__global__ void adj_gather_h(const __grid_constant__ SimView<T> s, const __grid_constant__ AdjView<T> a) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long n = (long long)s.NX * s.NY * s.NZ;
  if (q >= n) return;
  const int i = (int)(q % s.NX);
  const long long r = q / s.NX;
  const int j = (int)(r % s.NY), k = (int)(r / s.NY);
  const size_t id = fidx(s.PX, s.plane, i, j, k);
  const bool nx = i + 1 < s.NX, ny = j + 1 < s.NY, nz = k + 1 < s.NZ;
  const size_t sx = 1, sy = s.PX, sz = s.plane;
  // Hx: Ey slot 0 (z), Ez slot 1 (y)
  a.lH[0][id] += a.a[1][0][id] - (nz ? a.a[1][0][id + sz] : T(0)) + a.a[2][1][id] - (ny ? a.a[2][1][id + sy] : T(0));
  // Hy: Ex slot 1 (z), Ez slot 0 (x)
  a.lH[1][id] += a.a[0][1][id] - (nz ? a.a[0][1][id + sz] : T(0)) + a.a[2][0][id] - (nx ? a.a[2][0][id + sx] : T(0));
  // Hz: Ex slot 0 (y), Ey slot 1 (x)
  a.lH[2][id] += a.a[0][0][id] - (ny ? a.a[0][0][id + sy] : T(0)) + a.a[1][1][id] - (nx ? a.a[1][1][id + sx] : T(0));
}

// H sub-step transposed, per cell: coefficients of the E differences
// D = E_e(p + e_ax) - E_e(p), the old-H adjoint and the psi_H adjoints.
template <typename T>
__global__ void adj_h_coef(const __grid_constant__ SimView<T> s, const __grid_constant__ AdjView<T> a) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long n = (long long)s.NX * s.NY * s.NZ;
  if (q >= n) return;
  const int i = (int)(q % s.NX);
  const long long r = q / s.NX;
  const int j = (int)(r % s.NY), k = (int)(r / s.NY);
  const size_t id = fidx(s.PX, s.plane, i, j, k);
  const int NX = s.NX, NY = s.NY, NZ = s.NZ;
  const int ijk[3] = {i, j, k};
  const bool cellok = i < NX - 1 && j < NY - 1 && k < NZ - 1;  // CPML range (main.cu:829)
  const T che = s.che, chh = s.chh;
#pragma unroll
  for (int h = 0; h < 3; h++) {
    // Yee range: the two other indices below N-1
    bool act = true;
#pragma unroll
    for (int d = 0; d < 3; d++) {
      const int N = d == 0 ? NX : d == 1 ? NY : NZ;
      if (d != h && ijk[d] >= N - 1) act = false;
    }
    if (!act) {
      a.a[h][0][id] = T(0);
      a.a[h][1][id] = T(0);
      continue;
    }
    const T lam = a.lH[h][id];
#pragma unroll
    for (int sl = 0; sl < 2; sl++) {
      const int ax = (h + 1 + sl) % 3;
      const T sg = sl == 0 ? T(-1) : T(1);
      const CpmlAxis<T>& cp = s.cp[ax];
      T coef = sg * che * ldg(cp.inv_khd + ijk[ax]) * lam;
      if (cellok) {
        int qs;
        T* lp = adj_psi(s, &a.lpH_N[h][sl], &a.lpH_F[h][sl], ax, false, i, j, k, &qs);
        if (lp) {
          T b, cc;
          if (qs >= 0) { b = ldg(cp.bh_N + qs); cc = ldg(cp.ch_N + qs); }
          else { b = ldg(cp.bh_F + (-1 - qs)); cc = ldg(cp.ch_F + (-1 - qs)); }
          const T tot = *lp + sg * che * lam;
          *lp = b * tot;
          coef += cc * cp.inv_d * tot;
        }
      }
      a.a[h][sl][id] = coef;
    }
    a.lH[h][id] = chh * lam;
  }
}

// lambda_E += gather of the H-sub-step coefficients: D = E_e(p + e_ax) -
// E_e(p) read by H cell p contributes +a(p - e_ax) and -a(p) to E_e(p).
template <typename T>
__global__ void adj_gather_e(const __grid_constant__ SimView<T> s, const __grid_constant__ AdjView<T> a) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long n = (long long)s.NX * s.NY * s.NZ;
  if (q >= n) return;
  const int i = (int)(q % s.NX);
  const long long r = q / s.NX;
  const int j = (int)(r % s.NY), k = (int)(r / s.NY);
  const size_t id = fidx(s.PX, s.plane, i, j, k);
  const bool px = i > 0, py = j > 0, pz = k > 0;
  const size_t sx = 1, sy = s.PX, sz = s.plane;
  // Ex: Hy slot 0 (z), Hz slot 1 (y)
  a.lE[0][id] += (pz ? a.a[1][0][id - sz] : T(0)) - a.a[1][0][id] + (py ? a.a[2][1][id - sy] : T(0)) - a.a[2][1][id];
  // Ey: Hx slot 1 (z), Hz slot 0 (x)
  a.lE[1][id] += (pz ? a.a[0][1][id - sz] : T(0)) - a.a[0][1][id] + (px ? a.a[2][0][id - sx] : T(0)) - a.a[2][0][id];
  // Ez: Hx slot 0 (y), Hy slot 1 (x)
  a.lE[2][id] += (py ? a.a[0][0][id - sy] : T(0)) - a.a[0][0][id] + (px ? a.a[1][1][id - sx] : T(0)) - a.a[1][1][id];
}

// Objective derivative at a DFT sample step n: for every flux-face cell and
// tangential component of the faces in face_mask (bit b*6+f: box b, face
// f), g = sum_m Re(P_m conj(w_m)) with w_m = exp(i 2 pi (n + delta) dt f_m)
// (delta = 1 for E, 1/2 for H) and P_m the weighted partner accumulator
// (adj_partner).
template <typename T>
__global__ void adj_source(const __grid_constant__ SimView<T> s, const __grid_constant__ DftView d,
                           const __grid_constant__ AdjView<T> a, const double2* __restrict__ P,
                           const double* __restrict__ fsel, int nsel, long long prows, unsigned face_mask) {
  const int f = blockIdx.y;  // faces 0..11 (absorption box, then scattering box)
  if (!((face_mask >> f) & 1u)) return;
  const DftFace F = d.face[f];
  const int nc = F.na * F.nb;
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nc) return;
  const int n = *a.step;
  const int u = q / F.nb, v = q - u * F.nb;
  int ijk[3];
  const int a1 = F.ax == 0 ? 1 : 0, a2 = F.ax == 2 ? 1 : 2;
  ijk[F.ax] = F.pos;
  ijk[a1] = F.s1 + u;
  ijk[a2] = F.s2 + v;
  const size_t id = fidx(s.PX, s.plane, ijk[0], ijk[1], ijk[2]);
#pragma unroll
  for (int cs = 0; cs < 4; cs++) {
    const long long row = F.row0 + (long long)cs * F.npad + q;
    const double del = cs < 2 ? 1.0 : 0.5;
    double g = 0.0;
    for (int m = 0; m < nsel; m++) {
      const double ph = (double)(float)2.0 * 3.1415926535897932384626433832795 * (n + del) * d.dt * fsel[m];
      double sv, cv;
      sincos(ph, &sv, &cv);
      const double2 p = P[(size_t)m * prows + row];
      g += p.x * cv + p.y * sv;
    }
    const int comp = F.comp[cs];
    T* dst = comp < 3 ? a.lE[comp] : a.lH[comp - 3];
    atomicAdd(dst + id, (T)g);
  }
}

// Weighted partner accumulators of the flux-face rows for the chosen
// frequencies.  Face flux Q_f(m) = sum Re(Ex conj(Hy) - Ey conj(Hx)) (per
// face pairing) is bilinear in the accumulators, so dQ/d(sample of Ex)
// pairs with Hy, etc.; wface[m * 12 + f] = dL/dQ_f(m), zero for faces the
// objective does not read.
__global__ void adj_partner(const __grid_constant__ DftView d, const int* __restrict__ sel,
                            const double* __restrict__ wface, int nsel, double2* __restrict__ P, long long prows) {
  const int f = blockIdx.y;
  const int m = blockIdx.z;
  const DftFace F = d.face[f];
  const int nc = F.na * F.nb;
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nc || m >= nsel) return;
  const int qx = F.ax == 1 ? 1 : 0, qy = F.ax == 1 ? 0 : 1;
  const double K = wface[(size_t)m * 12 + f];
  const int fm = sel[m];
#pragma unroll
  for (int cs = 0; cs < 4; cs++) {
    int ps;
    double sg;
    if (cs == qx) { ps = 2 + qy; sg = 1.0; }
    else if (cs == qy) { ps = 2 + qx; sg = -1.0; }
    else if (cs == 2 + qx) { ps = qy; sg = -1.0; }
    else { ps = qx; sg = 1.0; }
    const long long pr = F.row0 + (long long)ps * F.npad + q;
    const double re = d.acc_re[(size_t)fm * d.rows + pr], im = d.acc_im[(size_t)fm * d.rows + pr];
    P[(size_t)m * prows + F.row0 + (long long)cs * F.npad + q] = make_double2(K * sg * re, K * sg * im);
  }
}

__global__ void adj_step_back(int* step) { *step -= 1; }
__global__ void adj_set_step(int* step, int n) { *step = n; }

// ---------------------------------------------------------------------
// Fused form of the transposed Yee sub-steps.  Away from the CPML slabs and
// the dispersive cells a difference coefficient is a fixed multiple of the
// adjoint of the component that read the difference, so the gathers
// compute it on the fly from that adjoint (read with a one-cell halo)
// instead of from a coefficient array.  Only the slab cells (psi
// recursions) and the dispersive cells keep their coefficients in the
// arrays ("special" components, written by adj_e_slab / adj_h_slab and
// adj_e_design before the gathers).  The scaling of a non-special E adjoint
// by cee, which must follow every read of it by the H gather, moves into
// the E gather of the same step.  The H scaling chh is 1 (no magnetic loss
// in the reference's coefficients, setup.cu:2020), which the host checks
// before taking this path.  Per step the two gathers each read one field
// adjoint and update the other: 9 values per cell each, against 24 per
// sub-step for coefficient arrays written then gathered.  Arithmetic and
// summation order are those of adj_e_coef / adj_gather_h / adj_h_coef /
// adj_gather_e, so both forms give the same values.

// Cells of the thick shell n < lo[a] or n >= hi[a] along some axis a, each
// once: the z slabs (whole planes), then the y slabs of the other planes,
// then the x slabs of the other rows.
struct SlabShell {
  int N[3], lo[3], hi[3];
  long long n0, n1, n2;
  __host__ void init(const int n[3], const int l[3], const int h[3]) {
    for (int a = 0; a < 3; a++) {
      N[a] = n[a];
      lo[a] = std::max(0, std::min(l[a], n[a]));
      hi[a] = std::max(lo[a], std::min(h[a], n[a]));
    }
    const long long zc = lo[2] + (N[2] - hi[2]), yc = lo[1] + (N[1] - hi[1]), xc = lo[0] + (N[0] - hi[0]);
    const long long mz = hi[2] - lo[2], my = hi[1] - lo[1];
    n0 = zc * N[1] * N[0];
    n1 = mz * yc * N[0];
    n2 = mz * my * xc;
  }
  __host__ __device__ long long total() const { return n0 + n1 + n2; }
  // 32-bit index arithmetic: the host takes this path only for shells of
  // fewer than 2^32 cells
  __device__ void cell(unsigned q, int& i, int& j, int& k) const {
    const unsigned N0 = (unsigned)N[0], N1 = (unsigned)N[1];
    if (q < (unsigned)n0) {
      i = (int)(q % N0);
      const unsigned r = q / N0;
      j = (int)(r % N1);
      const int kk = (int)(r / N1);
      k = kk < lo[2] ? kk : hi[2] + (kk - lo[2]);
    } else if (q < (unsigned)(n0 + n1)) {
      q -= (unsigned)n0;
      i = (int)(q % N0);
      const unsigned r = q / N0;
      const unsigned yc = (unsigned)(lo[1] + (N[1] - hi[1]));
      const int jj = (int)(r % yc);
      k = lo[2] + (int)(r / yc);
      j = jj < lo[1] ? jj : hi[1] + (jj - lo[1]);
    } else {
      q -= (unsigned)(n0 + n1);
      const unsigned xc = (unsigned)(lo[0] + (N[0] - hi[0])), my = (unsigned)(hi[1] - lo[1]);
      const int ii = (int)(q % xc);
      const unsigned r = q / xc;
      j = lo[1] + (int)(r % my);
      k = lo[2] + (int)(r / my);
      i = ii < lo[0] ? ii : hi[0] + (ii - lo[0]);
    }
  }
};

template <typename T>
__device__ __forceinline__ unsigned adj_mat(const SimView<T>& s, int i, int j, int k, size_t id) {
  return (i >= s.mat_lo[0] && i < s.mat_hi[0] && j >= s.mat_lo[1] && j < s.mat_hi[1] && k >= s.mat_lo[2] &&
          k < s.mat_hi[2])
             ? s.mat[id]
             : 0u;
}
// active range of E component c (main.cu:1172, 1476, 1767) and of H
// component h (the two other indices below N-1)
template <typename T>
__device__ __forceinline__ bool adj_e_act(const SimView<T>& s, int c, int i, int j, int k) {
  const int ijk[3] = {i, j, k}, N[3] = {s.NX, s.NY, s.NZ};
  bool act = true;
#pragma unroll
  for (int d = 0; d < 3; d++) {
    if (ijk[d] >= N[d] - 1) act = false;
    if (d != c && ijk[d] < 1) act = false;
  }
  return act;
}
template <typename T>
__device__ __forceinline__ bool adj_h_act(const SimView<T>& s, int h, int i, int j, int k) {
  const int ijk[3] = {i, j, k}, N[3] = {s.NX, s.NY, s.NZ};
  bool act = true;
#pragma unroll
  for (int d = 0; d < 3; d++)
    if (d != h && ijk[d] >= N[d] - 1) act = false;
  return act;
}
// slab membership as adj_psi decides it (E extent Nc+1, H extent Nc)
template <typename T>
__device__ __forceinline__ bool adj_in_slab(const SimView<T>& s, int ax, int n, bool e_extent) {
  const CpmlAxis<T>& a = s.cp[ax];
  return (e_extent ? n <= a.Nc : n < a.Nc) || n >= a.F;
}
// E component c keeps its coefficients in the arrays: dispersive, or
// updated with a psi recursion in one of its two slots
template <typename T>
__device__ __forceinline__ bool adj_e_special(const SimView<T>& s, int c, int i, int j, int k, unsigned m) {
  if (m & (1u << c)) return true;
  if (!adj_e_act(s, c, i, j, k)) return false;
  const int ijk[3] = {i, j, k};
  const int a0 = (c + 1) % 3, a1 = (c + 2) % 3;
  return adj_in_slab(s, a0, ijk[a0], true) || adj_in_slab(s, a1, ijk[a1], true);
}
template <typename T>
__device__ __forceinline__ bool adj_h_special(const SimView<T>& s, int h, int i, int j, int k) {
  if (!adj_h_act(s, h, i, j, k)) return false;
  if (!(i < s.NX - 1 && j < s.NY - 1 && k < s.NZ - 1)) return false;  // CPML range (main.cu:829)
  const int ijk[3] = {i, j, k};
  const int a0 = (h + 1) % 3, a1 = (h + 2) % 3;
  return adj_in_slab(s, a0, ijk[a0], false) || adj_in_slab(s, a1, ijk[a1], false);
}

// Per-cell flags of the gathers, evaluated once per cell: bit c = E (or H)
// component c active, bit 3 + c = special; bits 8.. = the material byte.
template <typename T>
__device__ __forceinline__ unsigned adj_flags_e(const SimView<T>& s, int i, int j, int k, size_t id) {
  const unsigned m = adj_mat(s, i, j, k, id);
  const bool sl[3] = {adj_in_slab(s, 0, i, true), adj_in_slab(s, 1, j, true), adj_in_slab(s, 2, k, true)};
  unsigned f = m << 8;
#pragma unroll
  for (int c = 0; c < 3; c++) {
    const bool act = adj_e_act(s, c, i, j, k);
    const bool spec = (m & (1u << c)) || (act && (sl[(c + 1) % 3] || sl[(c + 2) % 3]));
    f |= (act ? 1u << c : 0u) | (spec ? 8u << c : 0u);
  }
  return f;
}
template <typename T>
__device__ __forceinline__ unsigned adj_flags_h(const SimView<T>& s, int i, int j, int k) {
  const bool ok = i < s.NX - 1 && j < s.NY - 1 && k < s.NZ - 1;
  const bool sl[3] = {adj_in_slab(s, 0, i, false), adj_in_slab(s, 1, j, false), adj_in_slab(s, 2, k, false)};
  unsigned f = 0;
#pragma unroll
  for (int h = 0; h < 3; h++) {
    const bool act = adj_h_act(s, h, i, j, k);
    const bool spec = act && ok && (sl[(h + 1) % 3] || sl[(h + 2) % 3]);
    f |= (act ? 1u << h : 0u) | (spec ? 8u << h : 0u);
  }
  return f;
}

// The flags of every cell, once per reverse sweep: E flags in the low
// half (material byte in bits 8..15), H flags in bits 16..21.
template <typename T>
__global__ void adj_build_flags(const __grid_constant__ SimView<T> s, unsigned* __restrict__ flags) {
  const int i = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y * 8 + threadIdx.y, k = blockIdx.z;
  if (i >= s.NX || j >= s.NY) return;
  const size_t id = fidx(s.PX, s.plane, i, j, k);
  flags[id] = adj_flags_e(s, i, j, k, id) | (adj_flags_h(s, i, j, k) << 16);
}

// Product rounded on its own (no contraction into a following add), as a
// value stored to a coefficient array is.
__device__ __forceinline__ float adj_mul(float x, float y) { return __fmul_rn(x, y); }
__device__ __forceinline__ double adj_mul(double x, double y) { return __dmul_rn(x, y); }

// Difference coefficient of E component c, slot sl (axis (c+1+sl)%3), at a
// cell: the coefficient-array value `pre` for a special component, else sg
// ceh ikd lambda_E (H: sg che ikh lambda_H), from the cell's flags
// (adj_flags_e / adj_flags_h); n = the cell's coordinate along the slot's
// axis.  lam (the component's adjoint at the cell) and pre are loaded by the
// caller beside the flags (every coefficient array spans the grid), so that
// no load waits for the flags.
template <typename T>
__device__ __forceinline__ T adj_e_coef_v(const SimView<T>& s, int c, int sl, int n, unsigned f, T lam, T pre) {
  if (f & (8u << c)) return pre;
  if (!(f & (1u << c))) return T(0);
  const int ax = (c + 1 + sl) % 3;
  const T sg = sl == 0 ? T(1) : T(-1);
  return adj_mul(sg * s.ceh[(f >> 8) >> 3] * ldg(s.cp[ax].inv_ked + n), lam);
}
template <typename T>
__device__ __forceinline__ T adj_h_coef_v(const SimView<T>& s, int h, int sl, int n, unsigned f, T lam, T pre) {
  if (f & (8u << h)) return pre;
  if (!(f & (1u << h))) return T(0);
  const int ax = (h + 1 + sl) % 3;
  const T sg = sl == 0 ? T(-1) : T(1);
  return adj_mul(sg * s.che * ldg(s.cp[ax].inv_khd + n), lam);
}

// E sub-step transposed at the special slab components (the dispersive ones
// are adj_e_design's): coefficients, psi_E adjoints, lambda_E <- cee lambda_E.
// A cell's loads (its components' adjoints, psi adjoints and slab tables)
// do not depend on one another and are all issued before the arithmetic and
// the stores, which no load of the cell reads back.
template <typename T>
__global__ void adj_e_slab(const __grid_constant__ SimView<T> s, const __grid_constant__ AdjView<T> a,
                           const SlabShell sh) {
  const unsigned q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= (unsigned)sh.total()) return;
  int i, j, k;
  sh.cell(q, i, j, k);
  const size_t id = fidx(s.PX, s.plane, i, j, k);
  const unsigned m = adj_mat(s, i, j, k, id);
  const T cee = s.cee[m >> 3], ceh = s.ceh[m >> 3];
  const int ijk[3] = {i, j, k};
  bool sp[3];
  T lam[3], ik[3][2], old[3][2], bt[3][2], ct[3][2];
  T* lp[3][2];
#pragma unroll
  for (int c = 0; c < 3; c++) {
    sp[c] = !(m & (1u << c)) && adj_e_special(s, c, i, j, k, m);
    lam[c] = sp[c] ? a.lE[c][id] : T(0);
#pragma unroll
    for (int sl = 0; sl < 2; sl++) {
      const int ax = (c + 1 + sl) % 3;
      const CpmlAxis<T>& cp = s.cp[ax];
      lp[c][sl] = nullptr;
      ik[c][sl] = old[c][sl] = bt[c][sl] = ct[c][sl] = T(0);
      if (!sp[c]) continue;
      ik[c][sl] = ldg(cp.inv_ked + ijk[ax]);
      int qs;
      lp[c][sl] = adj_psi(s, &a.lpE_N[c][sl], &a.lpE_F[c][sl], ax, true, i, j, k, &qs);
      if (lp[c][sl]) {
        if (qs >= 0) {
          bt[c][sl] = ldg(cp.be_N + qs);
          ct[c][sl] = ldg(((c == 1 && ax == 0) ? cp.ce_N_ey : cp.ce_N) + qs);
        } else {
          bt[c][sl] = ldg(cp.be_F + (-1 - qs));
          ct[c][sl] = ldg(cp.ce_F + (-1 - qs));
        }
        old[c][sl] = *lp[c][sl];
      }
    }
  }
#pragma unroll
  for (int c = 0; c < 3; c++) {
    if (!sp[c]) continue;
#pragma unroll
    for (int sl = 0; sl < 2; sl++) {
      const int ax = (c + 1 + sl) % 3;
      const T sg = sl == 0 ? T(1) : T(-1);
      T coef = sg * ceh * ik[c][sl] * lam[c];
      if (lp[c][sl]) {
        const T tot = old[c][sl] + sg * ceh * lam[c];
        *lp[c][sl] = bt[c][sl] * tot;
        coef += ct[c][sl] * s.cp[ax].inv_d * tot;
      }
      a.a[c][sl][id] = coef;
    }
    a.lE[c][id] = cee * lam[c];
  }
}

// H sub-step transposed at the special slab components: coefficients and
// psi_H adjoints (lambda_H <- chh lambda_H is the identity).  Loads first,
// as in adj_e_slab.
template <typename T>
__global__ void adj_h_slab(const __grid_constant__ SimView<T> s, const __grid_constant__ AdjView<T> a,
                           const SlabShell sh) {
  const unsigned q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= (unsigned)sh.total()) return;
  int i, j, k;
  sh.cell(q, i, j, k);
  const size_t id = fidx(s.PX, s.plane, i, j, k);
  const int ijk[3] = {i, j, k};
  const T che = s.che;
  bool sp[3];
  T lam[3], ik[3][2], old[3][2], bt[3][2], ct[3][2];
  T* lp[3][2];
#pragma unroll
  for (int h = 0; h < 3; h++) {
    sp[h] = adj_h_special(s, h, i, j, k);
    lam[h] = sp[h] ? a.lH[h][id] : T(0);
#pragma unroll
    for (int sl = 0; sl < 2; sl++) {
      const int ax = (h + 1 + sl) % 3;
      const CpmlAxis<T>& cp = s.cp[ax];
      lp[h][sl] = nullptr;
      ik[h][sl] = old[h][sl] = bt[h][sl] = ct[h][sl] = T(0);
      if (!sp[h]) continue;
      ik[h][sl] = ldg(cp.inv_khd + ijk[ax]);
      int qs;
      lp[h][sl] = adj_psi(s, &a.lpH_N[h][sl], &a.lpH_F[h][sl], ax, false, i, j, k, &qs);
      if (lp[h][sl]) {
        if (qs >= 0) { bt[h][sl] = ldg(cp.bh_N + qs); ct[h][sl] = ldg(cp.ch_N + qs); }
        else { bt[h][sl] = ldg(cp.bh_F + (-1 - qs)); ct[h][sl] = ldg(cp.ch_F + (-1 - qs)); }
        old[h][sl] = *lp[h][sl];
      }
    }
  }
#pragma unroll
  for (int h = 0; h < 3; h++) {
    if (!sp[h]) continue;
#pragma unroll
    for (int sl = 0; sl < 2; sl++) {
      const int ax = (h + 1 + sl) % 3;
      const T sg = sl == 0 ? T(-1) : T(1);
      T coef = sg * che * ik[h][sl] * lam[h];
      if (lp[h][sl]) {
        const T tot = old[h][sl] + sg * che * lam[h];
        *lp[h][sl] = bt[h][sl] * tot;
        coef += ct[h][sl] * s.cp[ax].inv_d * tot;
      }
      a.a[h][sl][id] = coef;
    }
  }
}

// A block's cells [i0, i0 + 32) x [j0, j0 + 8) x {k}, widened by the halo
// [lo_off, hi_off] on every axis, lie away from the CPML slabs (E extent),
// off the grid boundary and outside the material box: every component
// there is active, not special, with the background coefficients.
template <typename T>
__device__ __forceinline__ bool adj_block_simple(const SimView<T>& s, int i0, int j0, int k, int lo_off, int hi_off) {
  const int lo[3] = {i0 + lo_off, j0 + lo_off, k + lo_off};
  const int hi[3] = {i0 + 31 + hi_off, j0 + 7 + hi_off, k + hi_off};  // inclusive
  bool inside = true, off_mat = false;
#pragma unroll
  for (int a = 0; a < 3; a++) {
    inside = inside && lo[a] >= s.cp[a].Nc + 1 && hi[a] < s.cp[a].F;
    off_mat = off_mat || hi[a] < s.mat_lo[a] || lo[a] >= s.mat_hi[a];
  }
  return inside && off_mat;
}

// lambda_H += gather of the E-sub-step coefficients (adj_gather_h's sums),
// the non-special coefficients computed from lambda_E of the cell and of
// its +x, +y, +z neighbours.  Grid (x tiles of 32, y rows of 8, z).
// Block (x tile of 32, y row of 8, plane) of a fused gather: the launch
// grid itself, or entry blockIdx.x of a table (the blocks the staged
// gathers leave).
__device__ __forceinline__ int3 adj_block(const int4* table) {
  if (table) {
    const int4 b = table[blockIdx.x];
    return make_int3(b.x, b.y, b.z);
  }
  return make_int3((int)blockIdx.x, (int)blockIdx.y, (int)blockIdx.z);
}

template <typename T>
__global__ void __launch_bounds__(256) adj_gather_h_fused(const __grid_constant__ SimView<T> s,
                                                          const __grid_constant__ AdjView<T> a,
                                                          const int4* __restrict__ table) {
  const int3 bk = adj_block(table);
  const int i = bk.x * 32 + threadIdx.x, j = bk.y * 8 + threadIdx.y, k = bk.z;
  const size_t sx = 1, sy = s.PX, sz = s.plane;
  if (adj_block_simple(s, bk.x * 32, bk.y * 8, k, 0, 1)) {
    // the same sums with every coefficient sg ceh0 ikd lambda_E
    const size_t id = fidx(s.PX, s.plane, i, j, k);
    const T ceh = s.ceh[0];
    const T kx = ldg(s.cp[0].inv_ked + i), kx1 = ldg(s.cp[0].inv_ked + i + 1);
    const T ky = ldg(s.cp[1].inv_ked + j), ky1 = ldg(s.cp[1].inv_ked + j + 1);
    const T kz = ldg(s.cp[2].inv_ked + k), kz1 = ldg(s.cp[2].inv_ked + k + 1);
    const T* ex = a.lE[0] + id;
    const T* ey = a.lE[1] + id;
    const T* ez = a.lE[2] + id;
    const T ex0 = ex[0], ey0 = ey[0], ez0 = ez[0];
    // Hx: Ey slot 0 (axis z, sg +1), Ez slot 1 (axis y, sg -1)
    a.lH[0][id] += adj_mul(T(1) * ceh * kz, ey0) - adj_mul(T(1) * ceh * kz1, ey[sz]) +
                   adj_mul(T(-1) * ceh * ky, ez0) - adj_mul(T(-1) * ceh * ky1, ez[sy]);
    // Hy: Ex slot 1 (axis z, sg -1), Ez slot 0 (axis x, sg +1)
    a.lH[1][id] += adj_mul(T(-1) * ceh * kz, ex0) - adj_mul(T(-1) * ceh * kz1, ex[sz]) +
                   adj_mul(T(1) * ceh * kx, ez0) - adj_mul(T(1) * ceh * kx1, ez[sx]);
    // Hz: Ex slot 0 (axis y, sg +1), Ey slot 1 (axis x, sg -1)
    a.lH[2][id] += adj_mul(T(1) * ceh * ky, ex0) - adj_mul(T(1) * ceh * ky1, ex[sy]) +
                   adj_mul(T(-1) * ceh * kx, ey0) - adj_mul(T(-1) * ceh * kx1, ey[sx]);
    return;
  }
  if (i >= s.NX || j >= s.NY) return;
  const size_t id = fidx(s.PX, s.plane, i, j, k);
  const bool nx = i + 1 < s.NX, ny = j + 1 < s.NY, nz = k + 1 < s.NZ;
  // neighbour offsets, 0 past the grid (the term is dropped there)
  const size_t ox = nx ? sx : 0, oy = ny ? sy : 0, oz = nz ? sz : 0;
  const T ex0 = a.lE[0][id], ey0 = a.lE[1][id], ez0 = a.lE[2][id];
  const T exy = a.lE[0][id + oy], exz = a.lE[0][id + oz], eyx = a.lE[1][id + ox], eyz = a.lE[1][id + oz];
  const T ezx = a.lE[2][id + ox], ezy = a.lE[2][id + oy];
  const T h0 = a.lH[0][id], h1 = a.lH[1][id], h2 = a.lH[2][id];
  const unsigned f0 = a.flags[id] & 0xffffu;
  const unsigned fx = a.flags[id + ox] & 0xffffu, fy = a.flags[id + oy] & 0xffffu, fz = a.flags[id + oz] & 0xffffu;
  // the coefficient-array values of every term, loaded beside the flags
  // (used where the flags mark the component special)
  const T p10 = a.a[1][0][id], p10z = a.a[1][0][id + oz], p21 = a.a[2][1][id], p21y = a.a[2][1][id + oy];
  const T p01 = a.a[0][1][id], p01z = a.a[0][1][id + oz], p20 = a.a[2][0][id], p20x = a.a[2][0][id + ox];
  const T p00 = a.a[0][0][id], p00y = a.a[0][0][id + oy], p11 = a.a[1][1][id], p11x = a.a[1][1][id + ox];
  // Hx: Ey slot 0 (z), Ez slot 1 (y)
  a.lH[0][id] = h0 + (adj_e_coef_v(s, 1, 0, k, f0, ey0, p10) -
                      (nz ? adj_e_coef_v(s, 1, 0, k + 1, fz, eyz, p10z) : T(0)) +
                      adj_e_coef_v(s, 2, 1, j, f0, ez0, p21) -
                      (ny ? adj_e_coef_v(s, 2, 1, j + 1, fy, ezy, p21y) : T(0)));
  // Hy: Ex slot 1 (z), Ez slot 0 (x)
  a.lH[1][id] = h1 + (adj_e_coef_v(s, 0, 1, k, f0, ex0, p01) -
                      (nz ? adj_e_coef_v(s, 0, 1, k + 1, fz, exz, p01z) : T(0)) +
                      adj_e_coef_v(s, 2, 0, i, f0, ez0, p20) -
                      (nx ? adj_e_coef_v(s, 2, 0, i + 1, fx, ezx, p20x) : T(0)));
  // Hz: Ex slot 0 (y), Ey slot 1 (x)
  a.lH[2][id] = h2 + (adj_e_coef_v(s, 0, 0, j, f0, ex0, p00) -
                      (ny ? adj_e_coef_v(s, 0, 0, j + 1, fy, exy, p00y) : T(0)) +
                      adj_e_coef_v(s, 1, 1, i, f0, ey0, p11) -
                      (nx ? adj_e_coef_v(s, 1, 1, i + 1, fx, eyx, p11x) : T(0)));
}

// lambda_E <- (non-special: cee) lambda_E + gather of the H-sub-step
// coefficients (adj_gather_e's sums), the non-special ones computed from
// lambda_H of the cell and of its -x, -y, -z neighbours.
template <typename T>
__global__ void __launch_bounds__(256) adj_gather_e_fused(const __grid_constant__ SimView<T> s,
                                                          const __grid_constant__ AdjView<T> a,
                                                          const int4* __restrict__ table) {
  const int3 bk = adj_block(table);
  const int i = bk.x * 32 + threadIdx.x, j = bk.y * 8 + threadIdx.y, k = bk.z;
  const size_t sx = 1, sy = s.PX, sz = s.plane;
  if (adj_block_simple(s, bk.x * 32, bk.y * 8, k, -1, 0)) {
    // the same sums with every coefficient sg che ikh lambda_H, after
    // lambda_E <- cee0 lambda_E
    const size_t id = fidx(s.PX, s.plane, i, j, k);
    const T che = s.che, cee = s.cee[0];
    const T kx = ldg(s.cp[0].inv_khd + i), kxm = ldg(s.cp[0].inv_khd + i - 1);
    const T ky = ldg(s.cp[1].inv_khd + j), kym = ldg(s.cp[1].inv_khd + j - 1);
    const T kz = ldg(s.cp[2].inv_khd + k), kzm = ldg(s.cp[2].inv_khd + k - 1);
    const T* hx = a.lH[0] + id;
    const T* hy = a.lH[1] + id;
    const T* hz = a.lH[2] + id;
    const T hx0 = hx[0], hy0 = hy[0], hz0 = hz[0];
    T l0 = adj_mul(cee, a.lE[0][id]), l1 = adj_mul(cee, a.lE[1][id]), l2 = adj_mul(cee, a.lE[2][id]);
    // Ex: Hy slot 0 (axis z, sg -1), Hz slot 1 (axis y, sg +1)
    l0 += adj_mul(T(-1) * che * kzm, hy[-(ptrdiff_t)sz]) - adj_mul(T(-1) * che * kz, hy0) +
          adj_mul(T(1) * che * kym, hz[-(ptrdiff_t)sy]) - adj_mul(T(1) * che * ky, hz0);
    // Ey: Hx slot 1 (axis z, sg +1), Hz slot 0 (axis x, sg -1)
    l1 += adj_mul(T(1) * che * kzm, hx[-(ptrdiff_t)sz]) - adj_mul(T(1) * che * kz, hx0) +
          adj_mul(T(-1) * che * kxm, hz[-(ptrdiff_t)sx]) - adj_mul(T(-1) * che * kx, hz0);
    // Ez: Hx slot 0 (axis y, sg -1), Hy slot 1 (axis x, sg +1)
    l2 += adj_mul(T(-1) * che * kym, hx[-(ptrdiff_t)sy]) - adj_mul(T(-1) * che * ky, hx0) +
          adj_mul(T(1) * che * kxm, hy[-(ptrdiff_t)sx]) - adj_mul(T(1) * che * kx, hy0);
    a.lE[0][id] = l0;
    a.lE[1][id] = l1;
    a.lE[2][id] = l2;
    return;
  }
  if (i >= s.NX || j >= s.NY) return;
  const size_t id = fidx(s.PX, s.plane, i, j, k);
  const bool px = i > 0, py = j > 0, pz = k > 0;
  // neighbour offsets, 0 before the grid (the term is dropped there)
  const size_t ox = px ? sx : 0, oy = py ? sy : 0, oz = pz ? sz : 0;
  T l[3] = {a.lE[0][id], a.lE[1][id], a.lE[2][id]};
  const T hx0 = a.lH[0][id], hy0 = a.lH[1][id], hz0 = a.lH[2][id];
  const T hxy = a.lH[0][id - oy], hxz = a.lH[0][id - oz], hyx = a.lH[1][id - ox], hyz = a.lH[1][id - oz];
  const T hzx = a.lH[2][id - ox], hzy = a.lH[2][id - oy];
  const unsigned fw = a.flags[id];
  const unsigned fe = fw & 0xffffu;
  const T cee = s.cee[(fe >> 8) >> 3];
#pragma unroll
  for (int c = 0; c < 3; c++)
    if ((fe & (1u << c)) && !(fe & (8u << c))) l[c] = adj_mul(cee, l[c]);
  const unsigned f0 = fw >> 16;
  const unsigned fx = a.flags[id - ox] >> 16, fy = a.flags[id - oy] >> 16, fz = a.flags[id - oz] >> 16;
  // the coefficient-array values of every term, loaded beside the flags
  // (used where the flags mark the component special)
  const T p10 = a.a[1][0][id], p10z = a.a[1][0][id - oz], p21 = a.a[2][1][id], p21y = a.a[2][1][id - oy];
  const T p01 = a.a[0][1][id], p01z = a.a[0][1][id - oz], p20 = a.a[2][0][id], p20x = a.a[2][0][id - ox];
  const T p00 = a.a[0][0][id], p00y = a.a[0][0][id - oy], p11 = a.a[1][1][id], p11x = a.a[1][1][id - ox];
  // Ex: Hy slot 0 (z), Hz slot 1 (y)
  l[0] += (pz ? adj_h_coef_v(s, 1, 0, k - 1, fz, hyz, p10z) : T(0)) - adj_h_coef_v(s, 1, 0, k, f0, hy0, p10) +
          (py ? adj_h_coef_v(s, 2, 1, j - 1, fy, hzy, p21y) : T(0)) - adj_h_coef_v(s, 2, 1, j, f0, hz0, p21);
  // Ey: Hx slot 1 (z), Hz slot 0 (x)
  l[1] += (pz ? adj_h_coef_v(s, 0, 1, k - 1, fz, hxz, p01z) : T(0)) - adj_h_coef_v(s, 0, 1, k, f0, hx0, p01) +
          (px ? adj_h_coef_v(s, 2, 0, i - 1, fx, hzx, p20x) : T(0)) - adj_h_coef_v(s, 2, 0, i, f0, hz0, p20);
  // Ez: Hx slot 0 (y), Hy slot 1 (x)
  l[2] += (py ? adj_h_coef_v(s, 0, 0, j - 1, fy, hxy, p00y) : T(0)) - adj_h_coef_v(s, 0, 0, j, f0, hx0, p00) +
          (px ? adj_h_coef_v(s, 1, 1, i - 1, fx, hyx, p11x) : T(0)) - adj_h_coef_v(s, 1, 1, i, f0, hy0, p11);
#pragma unroll
  for (int c = 0; c < 3; c++) a.lE[c][id] = l[c];
}

// ---------------------------------------------------------------------
// Staged z-march form of the fused gathers: a CTA owns a 32 x 8 tile and a
// z-chunk.  The adjoint planes stream through the shared-memory ring of the
// forward passes (staged.cuh), with the same data movement: adj_gather_h
// reads lambda_E at planes k and k + 1 with the +x and +y halo and updates
// lambda_H, as the H pass reads E and updates H; adj_gather_e reads
// lambda_H at k - 1 and k with the -x and -y halo and updates lambda_E, as
// the E pass.  The tiles are those whose cells and halo lie away from the
// CPML slabs, the grid's faces and the material box, where every
// coefficient is sg ceh0 ik lambda_E (or sg che ik lambda_H).  Each
// difference term has the product and sum order of the fused gathers, so
// the results are theirs bit for bit.  The host builds the tile table and
// hands the remaining blocks to the fused gathers.
constexpr int kAdjTY = 8, kAdjS = 4, kAdjKC = 16;

template <typename T>
__global__ void __launch_bounds__(32 * kAdjTY) adj_gather_h_staged(const __grid_constant__ SimView<T> s,
                                                                   const __grid_constant__ AdjView<T> a,
                                                                   const int4* __restrict__ tiles) {
  constexpr int TY = kAdjTY, S = kAdjS;
  using L = StageLayout<T, TY>;
  constexpr unsigned SB = L::STAGE * sizeof(T);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const T* sm = reinterpret_cast<const T*>(smem_raw);
  const unsigned sbase = (unsigned)__cvta_generic_to_shared(smem_raw);
  const int4 tl = tiles[blockIdx.x];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int i0 = tl.x * 32, j0 = tl.y * TY;
  const int i = i0 + tx, j = j0 + ty;
  const int NX = s.NX, NY = s.NY, NZ = s.NZ, PX = s.PX;
  const size_t plane = s.plane;
  const int k0 = tl.z * kAdjKC, k1 = min(NZ, k0 + kAdjKC);
  CopyTasks<T, TY> tasks;
  // (the adjoint has no periodic mode)
  tasks.init(sbase, a.lE[0], a.lE[1], a.lE[2], a.lH[0], a.lH[1], a.lH[2], NX, NY, PX, plane, k0, i0, j0, 0, 0, false);
  int pnext = k0;
#pragma unroll
  for (int q = 0; q < S - 1; q++) {
    tasks.issue(q * SB, pnext++, NZ, a.lE[0], plane);
    cp_async_commit();
  }
  const T ceh = s.ceh[0];
  const T kx = ldg(s.cp[0].inv_ked + i), kx1 = ldg(s.cp[0].inv_ked + i + 1);
  const T ky = ldg(s.cp[1].inv_ked + j), ky1 = ldg(s.cp[1].inv_ked + j + 1);
  const T* __restrict__ kzp = s.cp[2].inv_ked + k0;
  const size_t id0 = fidx(PX, plane, i, j, k0);
  T* __restrict__ phx = a.lH[0] + id0;
  T* __restrict__ phy = a.lH[1] + id0;
  T* __restrict__ phz = a.lH[2] + id0;
  const int o = ty * L::HW + tx, oo = ty * 32 + tx;
  constexpr int FH = L::FH;
  for (int k = k0; k < k1;) {
#pragma unroll
    for (int u = 0; u < S; u++) {
      if (k < k1) {
        cp_async_wait<S - 3>();  // planes up to k+1 have landed
        __syncthreads();
        tasks.issue(((u + S - 1) % S) * SB, pnext++, NZ, a.lE[0], plane);
        cp_async_commit();
        const T* eh = sm + u * L::STAGE;
        const T* en = sm + ((u + 1) % S) * L::STAGE;
        const T* hown = eh + L::HALO;
        const T ex0 = eh[o], ey0 = eh[FH + o], ez0 = eh[2 * FH + o];
        const T ex_y = eh[o + L::HW], ez_y = eh[2 * FH + o + L::HW];
        const T ey_x = eh[FH + o + 1], ez_x = eh[2 * FH + o + 1];
        const T ex_z = en[o], ey_z = en[FH + o];
        const T kz = ldg(kzp), kz1 = ldg(kzp + 1);
        // Hx: Ey slot 0 (axis z, sg +1), Ez slot 1 (axis y, sg -1)
        *phx = hown[oo] + (adj_mul(T(1) * ceh * kz, ey0) - adj_mul(T(1) * ceh * kz1, ey_z) +
                           adj_mul(T(-1) * ceh * ky, ez0) - adj_mul(T(-1) * ceh * ky1, ez_y));
        // Hy: Ex slot 1 (axis z, sg -1), Ez slot 0 (axis x, sg +1)
        *phy = hown[TY * 32 + oo] + (adj_mul(T(-1) * ceh * kz, ex0) - adj_mul(T(-1) * ceh * kz1, ex_z) +
                                     adj_mul(T(1) * ceh * kx, ez0) - adj_mul(T(1) * ceh * kx1, ez_x));
        // Hz: Ex slot 0 (axis y, sg +1), Ey slot 1 (axis x, sg -1)
        *phz = hown[2 * TY * 32 + oo] + (adj_mul(T(1) * ceh * ky, ex0) - adj_mul(T(1) * ceh * ky1, ex_y) +
                                         adj_mul(T(-1) * ceh * kx, ey0) - adj_mul(T(-1) * ceh * kx1, ey_x));
        phx += plane; phy += plane; phz += plane; kzp++;
        k++;
      }
    }
  }
  cp_async_wait<0>();
}

template <typename T>
__global__ void __launch_bounds__(32 * kAdjTY) adj_gather_e_staged(const __grid_constant__ SimView<T> s,
                                                                   const __grid_constant__ AdjView<T> a,
                                                                   const int4* __restrict__ tiles) {
  constexpr int TY = kAdjTY, S = kAdjS;
  using L = StageLayout<T, TY>;
  constexpr unsigned SB = L::STAGE * sizeof(T);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const T* sm = reinterpret_cast<const T*>(smem_raw);
  const unsigned sbase = (unsigned)__cvta_generic_to_shared(smem_raw);
  const int4 tl = tiles[blockIdx.x];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int i0 = tl.x * 32, j0 = tl.y * TY;
  const int i = i0 + tx, j = j0 + ty;
  const int NX = s.NX, NY = s.NY, NZ = s.NZ, PX = s.PX;
  const size_t plane = s.plane;
  const int k0 = tl.z * kAdjKC, k1 = min(NZ, k0 + kAdjKC);
  CopyTasks<T, TY> tasks;
  // (the adjoint has no periodic mode)
  tasks.init(sbase, a.lH[0], a.lH[1], a.lH[2], a.lE[0], a.lE[1], a.lE[2], NX, NY, PX, plane, k0 - 1, i0, j0, -1, -L::CH,
             false);
  int pnext = k0 - 1;
#pragma unroll
  for (int q = 0; q < S - 1; q++) {
    tasks.issue(q * SB, pnext++, NZ, a.lH[0], plane);
    cp_async_commit();
  }
  const T che = s.che, cee = s.cee[0];
  const T kx = ldg(s.cp[0].inv_khd + i), kxm = ldg(s.cp[0].inv_khd + i - 1);
  const T ky = ldg(s.cp[1].inv_khd + j), kym = ldg(s.cp[1].inv_khd + j - 1);
  const T* __restrict__ kzp = s.cp[2].inv_khd + k0;
  const size_t id0 = fidx(PX, plane, i, j, k0);
  T* __restrict__ pex = a.lE[0] + id0;
  T* __restrict__ pey = a.lE[1] + id0;
  T* __restrict__ pez = a.lE[2] + id0;
  const int o = (ty + 1) * L::HW + tx + L::CH, oo = ty * 32 + tx;
  constexpr int FH = L::FH;
  for (int k = k0; k < k1;) {
#pragma unroll
    for (int u = 0; u < S; u++) {
      if (k < k1) {
        cp_async_wait<S - 3>();  // planes up to k have landed
        __syncthreads();
        tasks.issue(((u + S - 1) % S) * SB, pnext++, NZ, a.lH[0], plane);
        cp_async_commit();
        const T* cur = sm + ((u + 1) % S) * L::STAGE;
        const T* prv = sm + u * L::STAGE;
        const T* eown = cur + L::HALO;
        const T hx0 = cur[o], hy0 = cur[FH + o], hz0 = cur[2 * FH + o];
        const T hx_y = cur[o - L::HW], hz_y = cur[2 * FH + o - L::HW];
        const T hy_x = cur[FH + o - 1], hz_x = cur[2 * FH + o - 1];
        const T hx_z = prv[o], hy_z = prv[FH + o];
        const T kz = ldg(kzp), kzm = ldg(kzp - 1);
        T l0 = adj_mul(cee, eown[oo]), l1 = adj_mul(cee, eown[TY * 32 + oo]), l2 = adj_mul(cee, eown[2 * TY * 32 + oo]);
        // Ex: Hy slot 0 (axis z, sg -1), Hz slot 1 (axis y, sg +1)
        l0 += adj_mul(T(-1) * che * kzm, hy_z) - adj_mul(T(-1) * che * kz, hy0) +
              adj_mul(T(1) * che * kym, hz_y) - adj_mul(T(1) * che * ky, hz0);
        // Ey: Hx slot 1 (axis z, sg +1), Hz slot 0 (axis x, sg -1)
        l1 += adj_mul(T(1) * che * kzm, hx_z) - adj_mul(T(1) * che * kz, hx0) +
              adj_mul(T(-1) * che * kxm, hz_x) - adj_mul(T(-1) * che * kx, hz0);
        // Ez: Hx slot 0 (axis y, sg -1), Hy slot 1 (axis x, sg +1)
        l2 += adj_mul(T(-1) * che * kym, hx_y) - adj_mul(T(-1) * che * ky, hx0) +
              adj_mul(T(1) * che * kxm, hy_x) - adj_mul(T(1) * che * kx, hy0);
        *pex = l0;
        *pey = l1;
        *pez = l2;
        pex += plane; pey += plane; pez += plane; kzp++;
        k++;
      }
    }
  }
  cp_async_wait<0>();
}

}  // namespace fdtd
