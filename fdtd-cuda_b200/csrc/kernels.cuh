// CUDA kernels of the FDTD time step (sm_100a).
//
// One time step is:
//   h_pass      UPDATE_hx/hy/hz + H CPML (staged.cuh)
//   tfsf_h      H half of CORRECT_X/Y/Z on the TFSF faces (boundary.cuh)
//   line_step   UPDATE_h_inc + UPDATE_e_inc + Mur ends + source (1 CTA)
//   tfsf_e      E half of CORRECT_X/Y/Z (boundary.cuh)
//   e_pass      UPDATE_ex/ey/ez for non-dispersive components + E CPML
//   metal_e / hydro_*   dispersive (Drude + 2CP, hydrodynamic) cells,
//               compact lists
//   dft_sample  every dft_every steps: gather the flux-plane tangential
//               components into a sample ring
//   dft_contract once a half of the ring holds kRingSlots samples: FP64
//               contraction of that half with the phasors into the
//               accumulators, beside the steps that fill the other half
// This file holds the bodies of everything but the Yee passes and the TFSF
// tables.
#pragma once
#include <cuda_runtime.h>
#include <math.h>

#include "fdtd_internal.h"

namespace fdtd {

template <typename T>
__device__ __forceinline__ T ldg(const T* p) { return __ldg(p); }

// Arithmetic with its rounding fixed: products, differences and fused
// multiply-adds that the compiler may neither contract nor split.  The Yee
// passes are written with these, so that a cell's update rounds the same
// in every launch form (the CPML-free or the CPML-edge instantiation, any
// tile shape, the batched work queue).
__device__ __forceinline__ float rmul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double rmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float rsub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double rsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float rfma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double rfma(double a, double b, double c) { return __fma_rn(a, b, c); }
// a * x - b * y with the first product fused
template <typename T>
__device__ __forceinline__ T rcurl(T x, T a, T y, T b) { return rfma(x, a, -rmul(y, b)); }

__device__ __forceinline__ size_t fidx(int PX, size_t plane, int i, int j, int k) {
  return (size_t)k * plane + (size_t)j * PX + i;
}

// ---------------------------------------------------------------------
// TFSF helpers (CORRECT_X/Y/Z, main.cu:369-758)

// Projection of a staggered point onto the incidence direction with the
// reference's mixed precision: whole-cell offsets are int*float*float in
// single precision, half-cell offsets double*float*float; summed left to
// right with C promotion.  Explicit _rn intrinsics keep the compiler from
// contracting these into FMAs, so host and device round identically.
__device__ __forceinline__ double tf_proj(const TfsfView& tf, int hx2, int hy2, int hz2) {
  int h2[3] = {hx2, hy2, hz2};
  float fa[3] = {tf.sth, tf.sth, tf.cth};
  float fb[3] = {tf.cph, tf.sph, 1.0f};
  double t[3];
  int isd[3];
#pragma unroll
  for (int a = 0; a < 3; a++) {
    if (!(h2[a] & 1)) {
      float v = __fmul_rn((float)(h2[a] / 2), fa[a]);
      if (a < 2) v = __fmul_rn(v, fb[a]);
      t[a] = v;
      isd[a] = 0;
    } else {
      double v = __dmul_rn(h2[a] * 0.5, (double)fa[a]);
      if (a < 2) v = __dmul_rn(v, (double)fb[a]);
      t[a] = v;
      isd[a] = 1;
    }
  }
  double d;
  if (!isd[0] && !isd[1]) {
    float xy = __fadd_rn((float)t[0], (float)t[1]);
    d = isd[2] ? __dadd_rn((double)xy, t[2]) : (double)__fadd_rn(xy, (float)t[2]);
  } else {
    d = __dadd_rn(__dadd_rn(t[0], t[1]), t[2]);
  }
  return __dmul_rn(tf.dscale, d);
}

// The H half of CORRECT_X/Y/Z for H component c at (i,j,k), in the
// reference's kernel order X, Y, Z: fn(sign, axis, e_component, d) per
// correction, d the projected distance on the incident line.  tfsf_tabulate
// records the line index and interpolation weight of each correction; the
// appliers add sign * che * e_inc(d) fe / d_axis.
template <typename T, typename Fn>
__device__ __forceinline__ void tfsf_h_walk(const SimView<T>& s, int c, int i, int j, int k, Fn&& fn) {
  const TfsfView& tf = s.tf;
  const int NX = s.NX, NY = s.NY, NZ = s.NZ;
  const int Tx = tf.Tx, Ty = tf.Ty, Tz = tf.Tz;
  const int di = 2 * (i - tf.i0), dj = 2 * (j - tf.j0), dk = 2 * (k - tf.k0);
  if (c == 0) {  // hx: CORRECT_Y then CORRECT_Z
    if (tf.closed && i >= Tx && i <= NX - Tx && k >= Tz && k < NZ - Tz) {
      if (j == Ty - 1) {  // source at j+1
        fn(+1, 1, 2, tf_proj(tf, di, dj + 2, dk + 1));
      } else if (j == NY - Ty) {
        fn(-1, 1, 2, tf_proj(tf, di, dj, dk + 1));
      }
    }
    if (i >= Tx && i <= NX - Tx && j >= Ty && j < NY - Ty) {
      if (k == Tz - 1) {
        fn(-1, 2, 1, tf_proj(tf, di, dj + 1, dk + 2));
      } else if (k == NZ - Tz && tf.closed) {
        fn(+1, 2, 1, tf_proj(tf, di, dj + 1, dk));
      }
    }
  } else if (c == 1) {  // hy: CORRECT_X then CORRECT_Z
    if (tf.closed && j >= Ty && j <= NY - Ty && k >= Tz && k < NZ - Tz) {
      if (i == Tx - 1) {
        fn(-1, 0, 2, tf_proj(tf, di + 2, dj, dk + 1));
      } else if (i == NX - Tx) {
        fn(+1, 0, 2, tf_proj(tf, di, dj, dk + 1));
      }
    }
    if (i >= Tx && i < NX - Tx && j >= Ty && j <= NY - Ty) {
      if (k == Tz - 1) {
        fn(+1, 2, 0, tf_proj(tf, di + 1, dj, dk + 2));
      } else if (k == NZ - Tz && tf.closed) {
        fn(-1, 2, 0, tf_proj(tf, di + 1, dj, dk));
      }
    }
  } else {  // hz: CORRECT_X then CORRECT_Y
    if (tf.closed && j >= Ty && j < NY - Ty && k >= Tz && k <= NZ - Tz) {
      if (i == Tx - 1) {
        fn(+1, 0, 1, tf_proj(tf, di + 2, dj + 1, dk));
      } else if (i == NX - Tx) {
        fn(-1, 0, 1, tf_proj(tf, di, dj + 1, dk));
      }
    }
    if (tf.closed && i >= Tx && i < NX - Tx && k >= Tz && k <= NZ - Tz) {
      if (j == Ty - 1) {
        fn(-1, 1, 0, tf_proj(tf, di + 1, dj + 2, dk));
      } else if (j == NY - Ty) {
        fn(+1, 1, 0, tf_proj(tf, di + 1, dj, dk));
      }
    }
  }
}

// The E half of CORRECT_X/Y/Z for E component c, added before its update
// (the reference launches CORRECT_* before UPDATE_e*): fn(sign, axis,
// h_component, d) per correction.
template <typename T, typename Fn>
__device__ __forceinline__ void tfsf_e_walk(const SimView<T>& s, int c, int i, int j, int k, Fn&& fn) {
  const TfsfView& tf = s.tf;
  const int NX = s.NX, NY = s.NY, NZ = s.NZ;
  const int Tx = tf.Tx, Ty = tf.Ty, Tz = tf.Tz;
  const int di = 2 * (i - tf.i0), dj = 2 * (j - tf.j0), dk = 2 * (k - tf.k0);
  if (c == 0) {  // ex: CORRECT_Y then CORRECT_Z
    if (tf.closed && i >= Tx && i < NX - Tx && k >= Tz && k <= NZ - Tz) {
      if (j == Ty) {
        fn(-1, 1, 2, tf_proj(tf, di + 1, dj - 1, dk));
      } else if (j == NY - Ty) {
        fn(+1, 1, 2, tf_proj(tf, di + 1, dj + 1, dk));
      }
    }
    if (i >= Tx && i < NX - Tx && j >= Ty && j <= NY - Ty) {
      if (k == Tz) {
        fn(+1, 2, 1, tf_proj(tf, di + 1, dj, dk - 1));
      } else if (k == NZ - Tz && tf.closed) {
        fn(-1, 2, 1, tf_proj(tf, di + 1, dj, dk + 1));
      }
    }
  } else if (c == 1) {  // ey: CORRECT_X then CORRECT_Z
    if (tf.closed && j >= Ty && j < NY - Ty && k >= Tz && k <= NZ - Tz) {
      if (i == Tx) {
        fn(+1, 0, 2, tf_proj(tf, di - 1, dj + 1, dk));
      } else if (i == NX - Tx) {
        fn(-1, 0, 2, tf_proj(tf, di + 1, dj + 1, dk));
      }
    }
    if (i >= Tx && i <= NX - Tx && j >= Ty && j < NY - Ty) {
      if (k == Tz) {
        fn(-1, 2, 0, tf_proj(tf, di, dj + 1, dk - 1));
      } else if (k == NZ - Tz && tf.closed) {
        fn(+1, 2, 0, tf_proj(tf, di, dj + 1, dk + 1));
      }
    }
  } else {  // ez: CORRECT_X then CORRECT_Y
    if (tf.closed && j >= Ty && j <= NY - Ty && k >= Tz && k < NZ - Tz) {
      if (i == Tx) {
        fn(-1, 0, 1, tf_proj(tf, di - 1, dj, dk + 1));
      } else if (i == NX - Tx) {
        fn(+1, 0, 1, tf_proj(tf, di + 1, dj, dk + 1));
      }
    }
    if (tf.closed && i >= Tx && i <= NX - Tx && k >= Tz && k < NZ - Tz) {
      if (j == Ty) {
        fn(+1, 1, 0, tf_proj(tf, di, dj - 1, dk + 1));
      } else if (j == NY - Ty) {
        fn(-1, 1, 0, tf_proj(tf, di, dj + 1, dk + 1));
      }
    }
  }
}


// ---------------------------------------------------------------------
// CPML psi helpers.  psi layouts: z slab [w][NY][PX], y slab [NZ][w][PX],
// x slab [NZ][NY][w].

template <typename T>
__device__ __forceinline__ size_t slab_idx(const SimView<T>& s, int ax, int w, int i, int j, int k) {
  if (ax == 2) return (size_t)k * s.plane + (size_t)j * s.PX + i;
  if (ax == 1) return ((size_t)k * w + j) * s.PX + i;
  return ((size_t)k * s.NY + j) * w + i;
}

// One psi recursion of an E component (UPDATE_e* CPML blocks,
// main.cu:1294-1318 and mirrors).  near_lim is Nc+1 except Ez's near-y
// slab, which the reference bounds by Nc (main.cu:1843).
template <typename T>
__device__ __forceinline__ T cpml_e(const SimView<T>& s, int c, int slot, int ax, int i, int j, int k,
                                    T diff, T v, T sg, T ceh) {
  const CpmlAxis<T>& a = s.cp[ax];
  int q = ax == 0 ? i : ax == 1 ? j : k;
  int near_lim = (c == 2 && ax == 1) ? a.Nc : a.Nc + 1;
  if (q < near_lim) {
    const T* ceN = (c == 1 && ax == 0) ? a.ce_N_ey : a.ce_N;
    T* p = s.psiE_N[c][slot] + slab_idx(s, ax, a.Nc + 1, i, j, k);
    T ps = ldg(a.be_N + q) * *p + ldg(ceN + q) * diff * a.inv_d;
    *p = ps;
    v += sg * (ceh * ps);
  }
  if (q >= a.F) {
    int q2 = q - a.F;
    int ii = ax == 0 ? q2 : i, jj = ax == 1 ? q2 : j, kk = ax == 2 ? q2 : k;
    T* p = s.psiE_F[c][slot] + slab_idx(s, ax, a.Nc + 1, ii, jj, kk);
    T ps = ldg(a.be_F + q2) * *p + ldg(a.ce_F + q2) * diff * a.inv_d;
    *p = ps;
    v += sg * (ceh * ps);
  }
  return v;
}

template <typename T>
__device__ __forceinline__ bool in_slab(const CpmlAxis<T>& a, int q) {
  return q <= a.Nc || q >= a.F;
}

template <typename T>
__device__ __forceinline__ void flag_nonfinite(const SimView<T>& s, T v) {
  if (!isfinite((double)v)) atomicOr(s.nonfinite, 1);
}

// ---------------------------------------------------------------------
// 1-D incident line (UPDATE_h_inc / UPDATE_e_inc, main.cu:2280-2337) with
// the Mur ends and the soft source that the reference applies on the host
// (main.cu:2831-2859).  One CTA.  Advances the device clock and records the
// probe (E after the previous step).
//
// The line's E is double-buffered: step t reads buffer t & 1 and writes
// the other, so the H half of the TFSF correction (which needs the line's
// E from before the update) can run after the line step, and the line step
// can run beside the H pass.  The parity comes from the device clock, so
// captured graphs replay correctly from either parity.

struct LineArgs {
  double* e_inc;        // [2][L]: the line's E, buffer t & 1 current at step t
  double* h_inc;
  int L, m0, src;
  double ch, ce, mur;
  const double* pulse;  // pulse[t], host-computed (main.cu:2845-2848)
  int tmax;             // entries in pulse
  DevClock* clk;
  double* probe;        // [t][3]
  int probe_cap;
  int dft_every;        // 0 = no DFT sampling
};

// E buffer of the line current at step parity `par` (the other one receives
// the update)
__device__ __forceinline__ double* line_e(const LineArgs& a, int par) {
  return a.e_inc + (size_t)(par & 1) * a.L;
}
// The line's E from before the update of the current step, for a kernel
// that runs before the line step of the step (after_line = 0: the clock
// still holds the step) or after it (after_line = 1: the clock holds the
// step + 1).
__device__ __forceinline__ const double* line_e_before(const LineArgs& a, int after_line) {
  return line_e(a, a.clk->t - after_line);
}

template <typename T>
__device__ __forceinline__ void line_step_body(const LineArgs& a, const SimView<T>& s, size_t probe_id) {
  const int t = a.clk->t;
  const double* ec = line_e(a, t);
  double* e = line_e(a, t + 1);
  // probe: E after step t-1 (OUT.txt records it at the top of step t)
  if (threadIdx.x < 3 && t >= 1 && t - 1 < a.probe_cap)
    a.probe[3 * (size_t)(t - 1) + threadIdx.x] = (double)s.E[threadIdx.x][probe_id];
  for (int q = threadIdx.x; q < a.L - 1; q += blockDim.x)
    a.h_inc[q] = a.h_inc[q] - a.ch * (ec[q + 1] - ec[q]);
  __syncthreads();
  for (int q = threadIdx.x + 1; q < a.L - 1; q += blockDim.x)
    e[q] = ec[q] - a.ce * (a.h_inc[q] - a.h_inc[q - 1]);
  __syncthreads();
  if (threadIdx.x == 0) {
    e[0] = a.clk->e1 + a.mur * (e[1] - ec[0]);
    e[a.L - 1] = a.clk->e2 + a.mur * (e[a.L - 2] - ec[a.L - 1]);
    a.clk->e1 = e[1];
    a.clk->e2 = e[a.L - 2];
    if (t < a.tmax) e[a.src] += a.pulse[t];
    // reserve this step's slot in the DFT sample ring (ScattAbs runs when
    // t % 4 == 0, main.cu:2920)
    if (a.dft_every > 0 && t % a.dft_every == 0) {
      const int n = a.clk->nsamp;
      if (n < kRingSlots) {
        const int slot = a.clk->base + n;
        a.clk->samp_slot = slot;
        a.clk->samp_t[slot] = t;
        a.clk->nsamp = n + 1;
      } else {
        a.clk->samp_slot = -1;  // half full: the caller skipped a contraction
      }
    }
    a.clk->t = t + 1;
  }
}
// Programmatic dependent launch.  A kernel that triggers lets the launch
// after it on its stream, when that launch carries a programmatic
// dependency, start its CTAs as soon as all of this one's have started;
// griddepcontrol.wait in the later kernel then waits for the earlier one to
// finish (and its writes to be visible).  Both are no-ops in a launch
// without a programmatic dependency.
__device__ __forceinline__ void pdl_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }

// The line step triggers at once: the H pass launched after it reads
// nothing it writes (and waits for it at its own end).
template <typename T>
__global__ void __launch_bounds__(1024) line_step(const __grid_constant__ LineArgs a, const __grid_constant__ SimView<T> s,
                                                  size_t probe_id) {
  pdl_launch_dependents();
  line_step_body(a, s, probe_id);
}

template <typename T>
__global__ void probe_record(const __grid_constant__ SimView<T> s, DevClock* clk, double* probe, int cap, size_t probe_id) {
  int t = clk->t;
  if (threadIdx.x < 3 && t >= 1 && t - 1 < cap)
    probe[3 * (size_t)(t - 1) + threadIdx.x] = (double)s.E[threadIdx.x][probe_id];
}

// ---------------------------------------------------------------------
// Dispersive cells: Drude + two critical points (UPDATE_e* metal branch,
// main.cu:1178-1219 and mirrors).  One thread per (component, cell).

template <typename T>
__device__ __forceinline__ T curl_h_at(const SimView<T>& s, int c, int i, int j, int k, T* dh_a, T* dh_b) {
  const size_t id = fidx(s.PX, s.plane, i, j, k);
  const T* hx = s.H[0];
  const T* hy = s.H[1];
  const T* hz = s.H[2];
  // offsets of the -x and -y neighbours (periodic x and y wrap around)
  const long long mx = (s.periodic && i == 0) ? -(long long)(s.NX - 1) : 1;
  const long long my = (s.periodic && j == 0) ? -(long long)(s.NY - 1) * s.PX : (long long)s.PX;
  if (c == 0) {
    T dhz = hz[id] - hz[id - my], dhy = hy[id] - hy[id - s.plane];
    *dh_a = dhz; *dh_b = dhy;  // y-slab diff, z-slab diff
    return dhz * s.cp[1].inv_ked[j] - dhy * s.cp[2].inv_ked[k];
  }
  if (c == 1) {
    T dhx = hx[id] - hx[id - s.plane], dhz = hz[id] - hz[id - mx];
    *dh_a = dhx; *dh_b = dhz;  // z-slab diff, x-slab diff
    return dhx * s.cp[2].inv_ked[k] - dhz * s.cp[0].inv_ked[i];
  }
  T dhy = hy[id] - hy[id - mx], dhx = hx[id] - hx[id - my];
  *dh_a = dhy; *dh_b = dhx;  // x-slab diff, y-slab diff
  return dhy * s.cp[0].inv_ked[i] - dhx * s.cp[1].inv_ked[j];
}

template <typename T>
__device__ __forceinline__ T cpml_e_all(const SimView<T>& s, int c, int i, int j, int k, T da, T db, T v,
                                        T ceh) {
  if (c == 0) {
    v = cpml_e(s, 0, 1, 2, i, j, k, db, v, T(-1), ceh);
    v = cpml_e(s, 0, 0, 1, i, j, k, da, v, T(1), ceh);
  } else if (c == 1) {
    v = cpml_e(s, 1, 0, 2, i, j, k, da, v, T(1), ceh);
    v = cpml_e(s, 1, 1, 0, i, j, k, db, v, T(-1), ceh);
  } else {
    v = cpml_e(s, 2, 1, 1, i, j, k, db, v, T(-1), ceh);
    v = cpml_e(s, 2, 0, 0, i, j, k, da, v, T(1), ceh);
  }
  return v;
}

// Row of step t in the adjoint's trajectory record (MetalView::rec).
__device__ __forceinline__ size_t rec_row(int t, int base, int rows) {
  const int d = (t - base) % rows;
  return (size_t)(d < 0 ? d + rows : d);
}

// Non-hydrodynamic dispersive update of all three components (they do not
// couple within a step).  pd ring: n = t%3, n-1 = (t+2)%3, new = (t+1)%3.
template <typename T>
__device__ __forceinline__ void metal_e_body(const SimView<T>& s, const MetalView<T>& m, const DevClock* clk) {
  const int t = clk->t - 1;
  const int rn = t % 3, rn1 = (t + 2) % 3, rnew = (t + 1) % 3;
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  int c = 0;
  while (c < 3 && q >= m.n[c]) { q -= m.n[c]; c++; }
  if (c >= 3) return;
  const int4 e = m.cell[c][q];
  const int i = e.x, j = e.y, k = e.z, sl = e.w;
  const size_t id = fidx(s.PX, s.plane, i, j, k);
  const unsigned mb = s.mat[id];
  const T ceh = s.ceh[mb >> 3];
  // the E half of CORRECT_* has already been added by tfsf_e_apply
  const T v = s.E[c][id];
  T da, db;
  const T curl = curl_h_at(s, c, i, j, k, &da, &db);
  const double pdn = m.pd[c][rn][sl], pdn1 = m.pd[c][rn1][sl];
  const double cpn0 = m.cpn[c][0][sl], cpn1_0 = m.cpn1[c][0][sl];
  const double cpn1 = m.cpn[c][1][sl], cpn1_1 = m.cpn1[c][1][sl];
  // the ADE recursions and their state in FP64, the fields in T
  double CP1 = 0.0, CP2 = 0.0, CP3 = 0.0, CP4 = 0.0;
  CP1 += (m.d1 - 1) * pdn;
  CP3 += m.d2 * pdn1;
  CP2 += (m.C1[0] - 1) * cpn0;
  CP2 += (m.C1[1] - 1) * cpn1;
  CP4 += m.C2[0] * cpn1_0;
  CP4 += m.C2[1] * cpn1_1;
  const T en1 = m.en[c][sl];  // e_n becomes e_n_1
  const T en = v;             // current E becomes e_n
  // coefficients coupling E to the poles; an adjoint design region blends
  // them linearly between vacuum (rho = 0) and the metal (rho = 1)
  double CE = m.C_E, CE1 = m.C_E_1, CE2 = m.C_E_2, D3 = m.d3, D4 = m.d4, D5 = m.d5;
  double C3[2] = {m.C3[0], m.C3[1]}, C4[2] = {m.C4[0], m.C4[1]}, C5[2] = {m.C5[0], m.C5[1]};
  if (m.rho[c]) {
    const double r = (double)(T)m.rho[c][sl];
    CE = m.vac + r * (m.C_E - m.vac);
    CE1 = m.vac + r * (m.C_E_1 - m.vac);
    CE2 = r * m.C_E_2;
    D3 = r * m.d3; D4 = r * m.d4; D5 = r * m.d5;
#pragma unroll
    for (int q = 0; q < 2; q++) { C3[q] = r * m.C3[q]; C4[q] = r * m.C4[q]; C5[q] = r * m.C5[q]; }
  }
  const double inv_CE = 1.0 / CE;
  const double nvd = inv_CE * ((double)(m.dt * curl / m.z0) + CE1 * en - CE2 * en1 - CP1 - CP2 - CP3 - CP4 - 0.0);
  const double ncp0 = m.C1[0] * cpn0 + m.C2[0] * cpn1_0 + C3[0] * nvd + C4[0] * en + C5[0] * en1;
  const double ncp1 = m.C1[1] * cpn1 + m.C2[1] * cpn1_1 + C3[1] * nvd + C4[1] * en + C5[1] * en1;
  const double npd = m.d1 * pdn + m.d2 * pdn1 + D3 * nvd + D4 * en + D5 * en1 + m.dNL * 0.0;
  T nv = (T)nvd;
  if (m.rec) {
    T* r = m.rec + rec_row(t, m.rec_base, m.rec_rows) * 5 * m.rec_slots + m.rec_off[c] + sl;
    r[0] = en; r[m.rec_slots] = en1; r[2 * m.rec_slots] = (T)pdn; r[3 * m.rec_slots] = (T)pdn1; r[4 * m.rec_slots] = nv;
  }
  m.en1[c][sl] = en1;
  m.en[c][sl] = en;
  m.cpn1[c][0][sl] = cpn0;
  m.cpn1[c][1][sl] = cpn1;
  m.cpn[c][0][sl] = ncp0;
  m.cpn[c][1][sl] = ncp1;
  m.pd[c][rnew][sl] = npd;
  nv = cpml_e_all(s, c, i, j, k, da, db, nv, ceh);
  if (!isfinite((double)nv)) atomicOr(s.nonfinite, 1);
  s.E[c][id] = nv;
}
template <typename T>
__global__ void metal_e(const __grid_constant__ SimView<T> s, const __grid_constant__ MetalView<T> m, const DevClock* clk) {
  pdl_launch_dependents();  // the E pass after it touches none of its cells
  metal_e_body(s, m, clk);
}

// Neighbour values of a dispersive cell for the hydrodynamic model.  nbr
// holds, per cell of component c and per component a, four slots (-1 =
// not dispersive: value 0, the reference's untouched dense arrays): for
// a == c the cells at +1, 0, -1 along c; for a != c the cells at +e_c, 0,
// +e_c - e_a and -e_a.  cphase: components below it have already rotated
// in this step (the reference launches UPDATE_ex, _ey, _ez in turn).
template <typename T, int c, int cphase>
__device__ __forceinline__ void hydro_neighbours(const MetalView<T>& m, int q, int t, double P[3][4], double N[3][4]) {
  const int* nb = m.nbr[c] + (size_t)q * 12;
#pragma unroll
  for (int a = 0; a < 3; a++) {
    const int rp = (a < cphase) ? (t + 1) % 3 : t % 3;
    const int rn = ((a < cphase) ? t + 1 : t) & 1;
#pragma unroll
    for (int x = 0; x < 4; x++) {
      const int sl = nb[a * 4 + x];
      P[a][x] = sl >= 0 ? m.pd[a][rp][sl] : 0.0;
      N[a][x] = sl >= 0 ? m.nd[a][rn][sl] : 0.0;
    }
  }
}

// UpdateHydroPx/Py/Pz (main.cu:1916-2276): the new hydrodynamic Drude
// current of one cell from E^n (after the TFSF pre-add), its history and
// the pressure term d_NL (grad div J + grad div (N J) / N_EQ) / (N_EQ +
// N)^(1/3).  Convection and Lorentz terms are off in the reference.
template <typename T, int c>
__device__ __forceinline__ double hydro_current(const MetalView<T>& m, int t, int sl, const double P[3][4],
                                                const double N[3][4], T ev, T en_prev) {
  const double IX = m.inv_dx, IY = m.inv_dy, IZ = m.inv_dz;
  const double I3[3] = {IX, IY, IZ};
  // the two other components in the reference's summation order, with
  // their mixed-derivative coefficients
  constexpr int a1 = c == 0 ? 1 : (c == 1 ? 0 : 1), a2 = c == 0 ? 2 : (c == 1 ? 2 : 0);
  const double k1 = c == 2 ? IZ * IY : I3[c < a1 ? c : a1] * I3[c < a1 ? a1 : c];
  const double k2 = I3[c < a2 ? c : a2] * I3[c < a2 ? a2 : c];
  const double Ic = I3[c];
  double PN[3][4];
#pragma unroll
  for (int a = 0; a < 3; a++)
#pragma unroll
    for (int x = 0; x < 4; x++) PN[a][x] = P[a][x] * N[a][x];
  const double gd2 = Ic * Ic * (PN[c][0] - 2.0 * PN[c][1] + PN[c][2]) +
                     k1 * (PN[a1][0] - PN[a1][1] - PN[a1][2] + PN[a1][3]) +
                     k2 * (PN[a2][0] - PN[a2][1] - PN[a2][2] + PN[a2][3]);
  const double gd = Ic * Ic * (P[c][0] - 2.0 * P[c][1] + P[c][2]) + k1 * (P[a1][0] - P[a1][1] - P[a1][2] + P[a1][3]) +
                    k2 * (P[a2][0] - P[a2][1] - P[a2][2] + P[a2][3]);
  const double ND1 = m.N_EQ + N[c][1];
  double cb;
  if (m.fix_cbrt) cb = cbrt(ND1);
  else cb = (double)powf((float)ND1, (float)(1.0 / 3.0));
  const double pn = m.pd[c][t % 3][sl], pn1 = m.pd[c][(t + 2) % 3][sl];
  return m.d1 * pn + m.d2 * pn1 + m.d3 * (double)ev + m.d4 * (double)en_prev + m.d5 * 0.0 +
         m.dNL * ((gd + gd2 / m.N_EQ) / cb);
}

// Hydrodynamic E update of one cell of component c (UPDATE_e* hydro
// branch, main.cu:1220-1271 and mirrors): continuity for the density
// perturbation, then E with the current source e0 (N_EQ + N) J.
template <typename T, int c>
__device__ __forceinline__ void hydro_e_cell(const SimView<T>& s, const MetalView<T>& m, int t, int4 e,
                                             const double P[3][4], const double N[3][4], double jd) {
  const int i = e.x, j = e.y, k = e.z, sl = e.w;
  const size_t id = fidx(s.PX, s.plane, i, j, k);
  const T ceh = s.ceh[s.mat[id] >> 3];
  double V1[3], V2[3], N1[3], N2[3];
#pragma unroll
  for (int a = 0; a < 3; a++) {
    if (a == c) {
      V1[a] = P[a][0]; V2[a] = P[a][2]; N1[a] = N[a][0]; N2[a] = N[a][2];
    } else {
      V1[a] = 0.5 * (P[a][0] + P[a][1]);
      V2[a] = 0.5 * (P[a][2] + P[a][3]);
      N1[a] = 0.5 * (N[a][0] + N[a][1]);
      N2[a] = 0.5 * (N[a][2] + N[a][3]);
    }
  }
  const double ndm1 = m.nd[c][(t + 1) & 1][sl];  // N^{n-1}
  const double k2 = 2.0 * m.dt * m.inv_dx;
  // an adjoint design cell scales its current and density updates and
  // blends its coupling coefficients by rho (rho = 0: a vacuum cell with
  // J = N = 0, as the neighbours of a non-dispersive cell see it)
  const bool blend = m.rho[c] != nullptr;
  const double r = blend ? (double)m.rho[c][sl] : 1.0;
  double nd;
  if (c == 0)
    nd = ndm1 - k2 * (0.5 * (N1[0] * V1[0] - N2[0] * V2[0]) + (N1[1] * V1[1] - N2[1] * V2[1]) +
                      (N1[2] * V1[2] - N2[2] * V2[2]) +
                      (0.5 * (V1[0] - V2[0]) + (V1[1] - V2[1]) + (V1[2] - V2[2])) * m.N_EQ);
  else if (c == 1)
    nd = ndm1 - k2 * ((N1[0] * V1[0] - N2[0] * V2[0]) + 0.5 * (N1[1] * V1[1] - N2[1] * V2[1]) +
                      (N1[2] * V1[2] - N2[2] * V2[2]) +
                      ((V1[0] - V2[0]) + 0.5 * (V1[1] - V2[1]) + (V1[2] - V2[2])) * m.N_EQ);
  else
    nd = ndm1 - k2 * ((N1[0] * V1[0] - N2[0] * V2[0]) + (N1[1] * V1[1] - N2[1] * V2[1]) +
                      0.5 * (V1[2] - V2[2]) +
                      ((V1[0] - V2[0]) + (V1[1] - V2[1]) + 0.5 * (V1[2] - V2[2])) * m.N_EQ);
  if (blend) nd = r * nd;
  const T v = s.E[c][id];
  T da, db;
  const T curl = curl_h_at(s, c, i, j, k, &da, &db);
  const double cpn0 = m.cpn[c][0][sl], cpn1_0 = m.cpn1[c][0][sl];
  const double cpn1 = m.cpn[c][1][sl], cpn1_1 = m.cpn1[c][1][sl];
  // the ADE recursions and their state in FP64, the fields in T
  double CP2 = 0.0, CP4 = 0.0;
  CP2 += (m.C1[0] - 1) * cpn0;
  CP2 += (m.C1[1] - 1) * cpn1;
  CP4 += m.C2[0] * cpn1_0;
  CP4 += m.C2[1] * cpn1_1;
  const T en1 = m.en[c][sl];
  const T en = v;
  double CE = m.C_E, CE1 = m.C_E_1, CE2 = m.C_E_2;
  double C3[2] = {m.C3[0], m.C3[1]}, C4[2] = {m.C4[0], m.C4[1]}, C5[2] = {m.C5[0], m.C5[1]};
  if (blend) {
    CE = m.vac + r * (m.C_E - m.vac);
    CE1 = m.vac + r * (m.C_E_1 - m.vac);
    CE2 = r * m.C_E_2;
#pragma unroll
    for (int q = 0; q < 2; q++) { C3[q] = r * m.C3[q]; C4[q] = r * m.C4[q]; C5[q] = r * m.C5[q]; }
  }
  const double inv_CE = 1.0 / CE;
  const double nvd = inv_CE * ((m.dt * (double)curl / m.z0 + m.dt * jd * m.e0 * (m.N_EQ + nd)) + CE1 * en -
                               CE2 * en1 - CP2 - CP4);
  const double ncp0 = m.C1[0] * cpn0 + m.C2[0] * cpn1_0 + C3[0] * nvd + C4[0] * en + C5[0] * en1;
  const double ncp1 = m.C1[1] * cpn1 + m.C2[1] * cpn1_1 + C3[1] * nvd + C4[1] * en + C5[1] * en1;
  T nv = (T)nvd;
  if (m.rec) {
    T* rr = m.rec + rec_row(t, m.rec_base, m.rec_rows) * 5 * m.rec_slots + m.rec_off[c] + sl;
    rr[0] = en; rr[m.rec_slots] = en1; rr[4 * m.rec_slots] = nv;
  }
  if (m.hrec) m.hrec[(rec_row(t, m.rec_base, m.rec_rows) * 6 + 5) * m.rec_slots + m.rec_off[c] + sl] = (T)nd;
  m.en1[c][sl] = en1;
  m.en[c][sl] = en;
  m.cpn1[c][0][sl] = cpn0;
  m.cpn1[c][1][sl] = cpn1;
  m.cpn[c][0][sl] = ncp0;
  m.cpn[c][1][sl] = ncp1;
  m.nd[c][(t + 1) & 1][sl] = nd;  // becomes "prev" after the parity flip
  nv = cpml_e_all(s, c, i, j, k, da, db, nv, ceh);
  if (!isfinite((double)nv)) atomicOr(s.nonfinite, 1);
  s.E[c][id] = nv;
}

template <typename T, int c>
__device__ __forceinline__ void hydro_p_cell(const SimView<T>& s, const MetalView<T>& m, int t, int q) {
  const int4 e = m.cell[c][q];
  double P[3][4], N[3][4];
  hydro_neighbours<T, c, 0>(m, q, t, P, N);
  const size_t id = fidx(s.PX, s.plane, e.x, e.y, e.z);
  double jd = hydro_current<T, c>(m, t, e.w, P, N, s.E[c][id], m.en[c][e.w]);
  if (m.rho[c]) jd *= (double)m.rho[c][e.w];  // adjoint design cell (see hydro_e_cell)
  if (m.hrec) {
    // J^{n-1}, J^n, J^{n+1}, N^{n-1}, N^n of the slot; N^{n+1} follows in
    // hydro_e_cell
    T* h = m.hrec + rec_row(t, m.rec_base, m.rec_rows) * 6 * m.rec_slots + m.rec_off[c] + e.w;
    const long long S = m.rec_slots;
    h[0] = (T)m.pd[c][(t + 2) % 3][e.w];
    h[S] = (T)m.pd[c][t % 3][e.w];
    h[2 * S] = (T)jd;
    h[3 * S] = (T)m.nd[c][(t + 1) & 1][e.w];
    h[4 * S] = (T)m.nd[c][t & 1][e.w];
  }
  m.pd[c][(t + 1) % 3][e.w] = jd;
  if (c == 0) hydro_e_cell<T, 0>(s, m, t, e, P, N, jd);
}

// Phase 1 of the hydrodynamic step: UpdateHydroP* for every dispersive
// cell, and the Ex update for the x cells (which needs only its own new
// current and the state from before this step).
template <typename T>
__global__ void hydro_p_ex(const __grid_constant__ SimView<T> s, const __grid_constant__ MetalView<T> m,
                           const DevClock* clk) {
  pdl_launch_dependents();  // the next phase waits for this one itself; the E pass touches none of its cells
  const int t = clk->t - 1;
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  int c = 0;
  while (c < 3 && q >= m.n[c]) { q -= m.n[c]; c++; }
  if (c >= 3) return;
  if (c == 0) hydro_p_cell<T, 0>(s, m, t, q);
  else if (c == 1) hydro_p_cell<T, 1>(s, m, t, q);
  else hydro_p_cell<T, 2>(s, m, t, q);
}

// Phases 2 and 3: the Ey, then the Ez update.
template <typename T, int c>
__global__ void hydro_e(const __grid_constant__ SimView<T> s, const __grid_constant__ MetalView<T> m,
                        const DevClock* clk) {
  pdl_launch_dependents();
  pdl_wait();  // the previous phase has finished
  const int t = clk->t - 1;
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= m.n[c]) return;
  const int4 e = m.cell[c][q];
  double P[3][4], N[3][4];
  hydro_neighbours<T, c, c>(m, q, t, P, N);
  hydro_e_cell<T, c>(s, m, t, e, P, N, m.pd[c][(t + 1) % 3][e.w]);
}

// ---------------------------------------------------------------------
// DFT flux planes (ScattAbs, main.cu:35-366).

// One flux face: component c occupies rows [row0 + c*npad, row0 + c*npad
// + na*nb), u major then v; npad rounds na*nb up to kDftRows so every
// contraction tile holds E rows only or H rows only.
struct DftFace {
  int ax, pos;          // normal axis and plane index
  int s1, s2;           // start of the two tangential axes
  int na, nb;           // extents (END - START)
  int comp[4];          // field components 0..5
  long long row0;
  long long npad;
};

struct DftView {
  int nfaces;           // 12
  DftFace face[12];
  long long rows;       // total rows
  int nf;               // frequencies
  const double* freq;
  double dt;
  double* acc_re;       // [nf][rows]
  double* acc_im;
};

template <typename T>
__device__ __forceinline__ void dft_sample_body(const SimView<T>& s, const DftView& d, T* ring, const DevClock* clk) {
  const int slot = clk->samp_slot;
  if (slot < 0 || slot >= 2 * kRingSlots) return;
  const int f = blockIdx.y;
  const DftFace F = d.face[f];
  const int n = F.na * F.nb;
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
    const int u = q / F.nb, v = q - u * F.nb;
    int ijk[3];
    const int a1 = F.ax == 0 ? 1 : 0, a2 = F.ax == 2 ? 1 : 2;
    ijk[F.ax] = F.pos;
    ijk[a1] = F.s1 + u;
    ijk[a2] = F.s2 + v;
    const size_t id = fidx(s.PX, s.plane, ijk[0], ijk[1], ijk[2]);
#pragma unroll
    for (int c = 0; c < 4; c++) {
      const int comp = F.comp[c];
      const T x = comp < 3 ? s.E[comp][id] : s.H[comp - 3][id];
      ring[(size_t)slot * d.rows + F.row0 + (size_t)c * F.npad + q] = x;
    }
  }
}
template <typename T>
__global__ void dft_sample(const __grid_constant__ SimView<T> s, const __grid_constant__ DftView d, T* ring, const DevClock* clk) {
  dft_sample_body(s, d, ring, clk);
}

// The contraction's job, set on the device before its kernels run:
//   dft_job_period  (a simulation's stepper, at the start of every
//                    contraction period) the samples of the half just
//                    filled; the other half becomes the one being filled
//   dft_job_flush   (before the spectra are read) the samples of the half
//                    being filled that no job has taken yet
//   dft_job_ready / dft_job_done  (the batch, whose members never switch
//                    halves) the half's samples once the half can no
//                    longer take another launch period, then empty it
__device__ __forceinline__ void dft_take(DevClock* clk, int upto) {
  clk->job_off = clk->base + clk->cstart;
  clk->job_n = upto - clk->cstart;
}
__global__ void dft_job_period(DevClock* clk) {
  dft_take(clk, clk->nsamp);
  clk->base ^= kRingSlots;
  clk->nsamp = 0;
  clk->cstart = 0;
}
__global__ void dft_job_flush(DevClock* clk) {
  dft_take(clk, clk->nsamp);
  clk->cstart = clk->nsamp;
}
__device__ __forceinline__ void dft_job_ready_body(DevClock* clk) {
  const bool ready = clk->nsamp > kRingSlots - kSampleBlock;
  dft_take(clk, ready ? min(kRingSlots, clk->nsamp) : clk->cstart);
  clk->job_reset = ready;
}
__device__ __forceinline__ void dft_job_done_body(DevClock* clk) {
  if (clk->job_reset) {
    clk->nsamp = 0;
    clk->cstart = 0;
    clk->job_reset = 0;
  }
}

// Phasors of the job's samples: tw[h][s][f] = exp(i 2 pi (t_s + delta_h)
// dt freq[f]) with delta = 1 for E (sampled after the E update) and 1/2 for
// H (main.cu:62-76).  [2][kRingSlots][nf] of double2; slots past the job
// hold zeros.
__device__ __forceinline__ void dft_twiddles_body(const DftView& d, const DevClock* clk, double2* tw) {
  const int n = clk->job_n;
  if (n <= 0) return;
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= 2 * kRingSlots * d.nf) return;
  const int h = q / (kRingSlots * d.nf);
  const int r = q - h * kRingSlots * d.nf;
  const int sidx = r / d.nf, f = r - sidx * d.nf;
  double c = 0, sv = 0;
  if (sidx < n) {
    const int ts = clk->samp_t[clk->job_off + sidx];
    const double ph = (double)(float)2.0 * 3.1415926535897932384626433832795 * (ts + (h ? 0.5 : 1.0)) * d.dt * d.freq[f];
    sincos(ph, &sv, &c);
  }
  tw[q] = make_double2(c, sv);
}
__global__ void dft_twiddles(const __grid_constant__ DftView d, const DevClock* clk, double2* tw) {
  dft_twiddles_body(d, clk, tw);
}

// acc[f][r] += sum_s x[s][r] tw[h(r)][s][f] in FP64, as a real matrix
// product on the FP64 tensor path (mma.sync m8n8k4 .f64): M = the real and
// imaginary parts of the phasors of 8 frequencies, K = 4 samples, N = 8 rows.
// A CTA owns kDftRows rows (all E or all H thanks to the padding) and walks
// every frequency in tiles of kDftFreqs; each of its four warps owns 32 rows
// of the tile, i.e. 2 frequency groups x {re, im} x 4 row groups = 16
// accumulator fragments.  The samples of the CTA's rows are staged once in
// shared memory, the phasors are read through L1 (a tile's phasors are 16
// KB), and the accumulators of a tile are copied into shared memory with
// cp.async while the tile's products run.  With
// kRingSlots = 64 samples per contraction the accumulator traffic (one FP64
// read and write per row and frequency) is spread over 64 samples.
constexpr int kDftRows = 128;
constexpr int kDftFreqs = 16;
constexpr int kDftXsPitch = kDftRows + 8;   // sample row pitch (elements): conflict-free B loads
constexpr int kDftAccPitch = kDftRows + 4;  // accumulator row pitch (doubles)
// dynamic shared memory of the contraction: samples (in the field type) and
// accumulators; three CTAs fit an SM in FP32, two in FP64
template <typename T>
constexpr size_t dft_smem_bytes() {
  return sizeof(T) * kRingSlots * kDftXsPitch + 2 * sizeof(double) * kDftFreqs * kDftAccPitch;
}

__device__ __forceinline__ void dft_cp_async16(void* dst, const void* src) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(src));
}

// D = A B + D for one m8n8k4 FP64 fragment: a = A[lane/4][lane%4],
// b = B[lane%4][lane/4], d = D[lane/4][2 (lane%4) + {0, 1}].
__device__ __forceinline__ void dmma_8x8x4(double& d0, double& d1, double a, double b) {
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
      : "+d"(d0), "+d"(d1)
      : "d"(a), "d"(b));
}

template <typename T>
__device__ __forceinline__ void dft_contract_body(const DftView& d, const T* ring, const DevClock* clk,
                                                  const double2* tw) {
  extern __shared__ __align__(16) unsigned char dft_smem[];
  constexpr size_t kXs = sizeof(T) * kRingSlots * kDftXsPitch;
  T(*xs)[kDftXsPitch] = reinterpret_cast<T(*)[kDftXsPitch]>(dft_smem);
  double(*ar)[kDftAccPitch] = reinterpret_cast<double(*)[kDftAccPitch]>(dft_smem + kXs);
  double(*ai)[kDftAccPitch] = ar + kDftFreqs;
  const int nsamp = clk->job_n;
  if (nsamp <= 0) return;  // an empty job adds nothing
  ring += (size_t)clk->job_off * d.rows;
  const int nk = (nsamp + 3) & ~3;  // K padded to whole m8n8k4 steps with zero samples
  const long long r0 = (long long)blockIdx.x * kDftRows;
  if (r0 >= d.rows) return;  // batched launches size the grid for the largest simulation
  // E or H rows: the tile lies inside one (face, component) block
  int h = 0;
  for (int f = 0; f < d.nfaces; f++) {
    const DftFace& F = d.face[f];
    if (r0 >= F.row0 && r0 < F.row0 + 4 * F.npad) { h = (r0 - F.row0) >= 2 * F.npad; break; }
  }
  const int tid = threadIdx.x;
  // the samples of this CTA's rows, 16 bytes per copy (rows are padded to
  // kDftRows, so every copy lies inside the ring); the K padding is zeroed
  constexpr int kPer = 16 / sizeof(T);
  for (int q = tid; q < nsamp * (kDftRows / kPer); q += 128) {
    const int sidx = q / (kDftRows / kPer), rr = kPer * (q - sidx * (kDftRows / kPer));
    dft_cp_async16(&xs[sidx][rr], ring + (size_t)sidx * d.rows + r0 + rr);
  }
  for (int q = tid; q < (nk - nsamp) * kDftRows; q += 128) xs[nsamp + q / kDftRows][q % kDftRows] = T(0);
  asm volatile("cp.async.commit_group;\n" ::);
  asm volatile("cp.async.wait_all;\n" ::);  // the barrier at the top of the tile loop publishes them
  const int lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, q4 = lane & 3;  // fragment row group and thread-in-group
  const int rw = warp * 32;                // this warp's rows within the tile
  // phasors: slots past nsamp hold zeros (dft_twiddles writes every slot)
  const double2* twh = tw + (size_t)h * kRingSlots * d.nf;
  for (int f0 = 0; f0 < d.nf; f0 += kDftFreqs) {
    __syncthreads();  // xs loaded / previous tile's accumulators consumed
    // this tile's accumulators, 16 bytes (two rows) per copy
    for (int q = tid; q < kDftFreqs * kDftRows / 2; q += 128) {
      const int fl = q / (kDftRows / 2), rr = 2 * (q - fl * (kDftRows / 2));
      if (f0 + fl < d.nf) {
        const size_t o = (size_t)(f0 + fl) * d.rows + r0 + rr;
        dft_cp_async16(&ar[fl][rr], d.acc_re + o);
        dft_cp_async16(&ai[fl][rr], d.acc_im + o);
      }
    }
    asm volatile("cp.async.commit_group;\n" ::);
    // A operands: this thread's two frequencies, clamped to the last one
    // (the rows of frequencies past nf are computed and dropped)
    const double2* tw0 = twh + min(f0 + g, d.nf - 1);
    const double2* tw1 = twh + min(f0 + 8 + g, d.nf - 1);
    // acc[fg][c][n]: frequency group fg, c = 0 re / 1 im, row group n
    double acc[2][2][4][2];
#pragma unroll
    for (int fg = 0; fg < 2; fg++)
#pragma unroll
      for (int c = 0; c < 2; c++)
#pragma unroll
        for (int n = 0; n < 4; n++) acc[fg][c][n][0] = acc[fg][c][n][1] = 0.0;
#pragma unroll 2
    for (int s0 = 0; s0 < nk; s0 += 4) {
      const double2 w0 = __ldg(tw0 + (size_t)(s0 + q4) * d.nf), w1 = __ldg(tw1 + (size_t)(s0 + q4) * d.nf);
      double b[4];
#pragma unroll
      for (int n = 0; n < 4; n++) b[n] = (double)xs[s0 + q4][rw + 8 * n + g];
#pragma unroll
      for (int n = 0; n < 4; n++) {
        dmma_8x8x4(acc[0][0][n][0], acc[0][0][n][1], w0.x, b[n]);
        dmma_8x8x4(acc[0][1][n][0], acc[0][1][n][1], w0.y, b[n]);
        dmma_8x8x4(acc[1][0][n][0], acc[1][0][n][1], w1.x, b[n]);
        dmma_8x8x4(acc[1][1][n][0], acc[1][1][n][1], w1.y, b[n]);
      }
    }
    asm volatile("cp.async.wait_all;\n" ::);
    __syncthreads();  // every thread's copies have landed
#pragma unroll
    for (int fg = 0; fg < 2; fg++) {
      const int fl = fg * 8 + g, f = f0 + fl;
      if (f >= d.nf) continue;
#pragma unroll
      for (int n = 0; n < 4; n++) {
        const int rl = rw + 8 * n + 2 * q4;
        const double2 pr = *reinterpret_cast<const double2*>(&ar[fl][rl]);
        const double2 pi = *reinterpret_cast<const double2*>(&ai[fl][rl]);
        const size_t o = (size_t)f * d.rows + r0 + rl;
        *reinterpret_cast<double2*>(d.acc_re + o) = make_double2(pr.x + acc[fg][0][n][0], pr.y + acc[fg][0][n][1]);
        *reinterpret_cast<double2*>(d.acc_im + o) = make_double2(pi.x + acc[fg][1][n][0], pi.y + acc[fg][1][n][1]);
      }
    }
  }
}
template <typename T>
__global__ void __launch_bounds__(128) dft_contract(const __grid_constant__ DftView d, const T* ring,
                                                     const DevClock* clk, const double2* tw) {
  dft_contract_body(d, ring, clk, tw);
}

// Per (box-face, frequency): sum over the face of Re(cEx conj(HY) -
// cEy conj(HX)) with the reference's component pairing
// (CalculateAbsScatt, Spectral.cu:725-1132).  Y faces swap the pair.
__global__ void flux_reduce(const __grid_constant__ DftView d, double* out /* [12][nf] */) {
  const int f = blockIdx.x, m = blockIdx.y;
  const DftFace F = d.face[f];
  const long long n = (long long)F.na * F.nb, np = F.npad;
  const int qx = F.ax == 1 ? 1 : 0, qy = F.ax == 1 ? 0 : 1;
  const double* re = d.acc_re + (size_t)m * d.rows + F.row0;
  const double* im = d.acc_im + (size_t)m * d.rows + F.row0;
  double acc = 0;
  for (long long q = threadIdx.x; q < n; q += blockDim.x) {
    const double exr = re[qx * np + q], exi = im[qx * np + q];
    const double eyr = re[qy * np + q], eyi = im[qy * np + q];
    const double hxr = re[(2 + qx) * np + q], hxi = im[(2 + qx) * np + q];
    const double hyr = re[(2 + qy) * np + q], hyi = im[(2 + qy) * np + q];
    acc += (exr * hyr + exi * hyi) - (eyr * hxr + eyi * hxi);
  }
  __shared__ double red[256];
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[(size_t)f * d.nf + m] = red[0];
}

// ---------------------------------------------------------------------
// Layout conversion between the device layout and the reference's
// [i][j][k] (z fastest) double arrays.

template <typename T>
__global__ void to_ref_layout(const T* src, double* dst, int NX, int NY, int NZ, int PX) {
  size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  size_t n = (size_t)NX * NY * NZ;
  if (q >= n) return;
  int k = q % NZ;
  size_t r = q / NZ;
  int j = r % NY;
  int i = r / NY;
  dst[q] = (double)src[((size_t)k * NY + j) * PX + i];
}
template <typename T>
__global__ void from_ref_layout(const double* src, T* dst, int NX, int NY, int NZ, int PX) {
  size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  size_t n = (size_t)NX * NY * NZ;
  if (q >= n) return;
  int k = q % NZ;
  size_t r = q / NZ;
  int j = r % NY;
  int i = r / NY;
  dst[((size_t)k * NY + j) * PX + i] = (T)src[q];
}

}  // namespace fdtd
