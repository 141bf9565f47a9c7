// Internal types shared by the host runtime and the CUDA kernels.
//
// Device layout (all per-sim state lives in HBM, allocated once at create):
//   fields ex..hz      [NZ][NY][PX] of T, x fastest, PX = NX rounded up to 8
//   material bits      [NZ][NY][PX] uint8 (bit c: component c is dispersive,
//                      bits 3..7: dielectric class), read only inside the
//                      material bounding box
//   CPML psi slabs     z slabs [w][NY][PX], y slabs [NZ][w][PX],
//                      x slabs [NZ][NY][w]; w = Ncpml (H) or Ncpml+1 (E)
//   dispersive cells   compact per-component lists + SoA state per slot
//   DFT                sample ring [TB][rows] of T, accumulators
//                      [F][rows] of double (re, im)
#pragma once
#include <cstddef>
#include <cstdint>

#include "../../include/fdtd_b200.h"

namespace fdtd {

constexpr int kMaxClasses = 32;   // dielectric classes (bits 3..7)
constexpr int kSampleBlock = 32;  // DFT samples per launch period of the stepper (a graph block)
constexpr int kRingSlots = 64;    // DFT samples per FP64 contraction (one half of the ring)
static_assert(kRingSlots == 2 * kSampleBlock, "a contraction period is two launch periods");

// Step clock kept in device memory so captured graphs can be replayed.
// The DFT sample ring has two halves of kRingSlots slots: samples go into
// the half at `base`; a contraction (its "job": ring slots job_off ..
// job_off + job_n) takes one half's samples, so that it can run beside
// the steps that fill the other half.
struct DevClock {
  int t;          // steps completed by the 1D-line kernel (current step + 1)
  int nsamp;      // DFT samples in the half being filled
  int nonfinite;  // watchdog flag: bit 0 NaN/Inf seen, bit 1 a pass gave up waiting for a plane copy
  int samp_slot;  // ring slot of the current step's DFT sample
  double e1, e2;  // Mur history of the incident line ends (main.cu:2835-2838)
  int base;       // first slot of the half being filled (0 or kRingSlots)
  int cstart;     // samples of that half a flush has already contracted
  int job_off, job_n, job_reset;
  int samp_t[2 * kRingSlots];
};

// Per-axis CPML tables.  The E tables have Nc+1 entries, the H tables Nc.
template <typename T>
struct CpmlAxis {
  const T* be_N; const T* ce_N; const T* be_F; const T* ce_F;
  const T* bh_N; const T* ch_N; const T* bh_F; const T* ch_F;
  const T* ce_N_ey;  // ce_N used by Ey's near-x slab (reference passes ce_y_N)
  const T* inv_ked;  // 1/(kappa_e * d), length N
  const T* inv_khd;  // 1/(kappa_h * d), length N
  T inv_d;           // 1/d
  int Nc, F;         // slab width, first index of the far slab
};

// Incident-field geometry for the TFSF corrections (CORRECT_* main.cu:369).
struct TfsfView {
  int on;
  int Tx, Ty, Tz;      // box faces at Tx and N-Tx (etc.)
  int i0, j0, k0, m0;  // projection origin, line centre
  float sth, cth, sph, cph;  // sinf/cosf of the angles (host-computed)
  float fe[3], fh[3];        // E and H direction factors
  double dscale;             // dx / d_1D
  int closed;                // 1: all six faces; 0: the lower z face only (periodic x and y)
};

template <typename T>
struct SimView {
  int NX, NY, NZ, PX;
  size_t plane;  // NY * PX
  T* E[3];
  T* H[3];
  const uint8_t* mat;
  int mat_lo[3], mat_hi[3];  // material bounding box, [lo, hi)
  T cee[kMaxClasses], ceh[kMaxClasses];  // per dielectric class
  T chh, che;
  CpmlAxis<T> cp[3];
  T* psiE_N[3][2]; T* psiE_F[3][2];  // [component][slot]: slot 0 = axis c+1
  T* psiH_N[3][2]; T* psiH_F[3][2];
  T dxyz[3];
  TfsfView tf;
  const double* h_inc;  // incident line H (double in both precisions); the
                        // line's E is double-buffered and passed per launch
  int* nonfinite;
  const SimView* self;  // a copy of this view in device memory (cold paths)
  int periodic;         // 1: x and y wrap around (every x and y index is updated)
};

// Dispersive (Drude + 2 critical points, optionally hydrodynamic) cells.
template <typename T>
struct MetalView {
  int n[3];             // cells per component
  const int4* cell[3];  // (i, j, k, slot) per entry
  // state, SoA per component: slot-major arrays.  The E history is in the
  // field type (it holds copies of field values); the polarisations, the
  // Drude current and the hydrodynamic density are FP64 in both builds:
  // rounding them to FP32 alone shifts the absorption spectra by 1e-5 of
  // their peak
  T* en[3]; T* en1[3];
  double* cpn[3][2]; double* cpn1[3][2];
  double* pd[3][3];     // Drude current ring (n, n-1, new) indexed by step
  double* nd[3][2];     // hydro density ring
  const float* rho[3];  // design blend per slot (null: plain metal coefficients)
  double vac;           // vacuum C_E = C_E_1 = ep0, the rho = 0 end of the blend
  // forward record for the adjoint (null = off): per step t the row
  // (t - rec_base) mod rec_rows (rec_row), five values per slot,
  // [row][value][rec_off[c] + slot], value = E^n, E^{n-1}, J^n, J^{n-1},
  // E^{n+1}
  T* rec;
  int rec_rows, rec_base;
  int rec_off[3];
  long long rec_slots;
  // hydrodynamic cells: six values per slot and row (FP64 state recorded in
  // the field type), [row][value][rec_off[c] + slot], value = J^{n-1}, J^n,
  // J^{n+1}, N^{n-1}, N^n, N^{n+1}
  T* hrec;
  // hydrodynamic neighbour slots, 12 per cell (see hydro_neighbours)
  const int* nbr[3];
  // ADE coefficients, FP64 in both builds: the CP pole recursions sit close
  // to their stability limit, and rounding these to FP32 alone shifts the
  // spectra by 1e-5 to 1e-4 of their peak.  The recursions run in FP64 and
  // the state is stored in T.
  double C_E, C_E_1, C_E_2;
  double d1, d2, d3, d4, d5, dNL;
  double C1[2], C2[2], C3[2], C4[2], C5[2];
  // the hydrodynamic E source dt J e0 (N_EQ + N) and the continuity update
  // run in FP64 too (their constants are FP64)
  double dt, z0, e0, N_EQ;
  double inv_dx, inv_dy, inv_dz;
  int hydro;
  int fix_cbrt;
};

}  // namespace fdtd
