// CUDA kernels of the FDTD time step (sm_100a).
//
// One time step is:
//   h_pass      fused UPDATE_hx/hy/hz + H CPML + H half of CORRECT_X/Y/Z
//   line_step   UPDATE_h_inc + UPDATE_e_inc + Mur ends + source (1 CTA)
//   e_pass      E half of CORRECT_*, UPDATE_ex/ey/ez for non-dispersive
//               components + E CPML
//   metal_*     dispersive (Drude + 2CP, hydrodynamic) cells, compact list
//   dft_sample  every dft_every steps: gather the flux-plane tangential
//               components into a sample ring
//   dft_contract every kSampleBlock samples: FP64 contraction of the ring
//               with the phasors into the accumulators
// The E and H passes march along z with a 2-D (x, y) thread tile; the
// z-neighbour is carried in registers, x and y neighbours come through L1.
#pragma once
#include <cuda_runtime.h>
#include <math.h>

#include "fdtd_internal.h"

namespace fdtd {

template <typename T>
__device__ __forceinline__ T ldg(const T* p) { return __ldg(p); }

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
__device__ __noinline__ double tf_proj(const TfsfView& tf, int hx2, int hy2, int hz2) {
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

// Linear interpolation of the incident line at projected distance d
// (truncation toward zero as the reference's (int) casts).
__device__ __forceinline__ double einc_at(const double* e, int m0, double d) {
  int n = (int)d;
  double dp = d - n;
  return (1 - dp) * e[m0 + n] + dp * e[m0 + n + 1];
}
__device__ __forceinline__ double hinc_at(const double* h, int m0, double d) {
  double d2 = d + 0.5;
  int n = (int)d2;
  double dp = d2 - n;
  return (1 - dp) * h[m0 - 1 + n] + dp * h[m0 + n];
}

// The H half of CORRECT_X/Y/Z applied to H component c at (i,j,k), in the
// reference's kernel order X, Y, Z.  v is the freshly updated value.
template <typename T>
__device__ __noinline__ T tfsf_h(const SimView<T>& s, int c, int i, int j, int k, T v) {
  const TfsfView& tf = s.tf;
  const int NX = s.NX, NY = s.NY, NZ = s.NZ;
  const int Tx = tf.Tx, Ty = tf.Ty, Tz = tf.Tz;
  const int di = 2 * (i - tf.i0), dj = 2 * (j - tf.j0), dk = 2 * (k - tf.k0);
  const T che = s.che;
  const T idx_ = s.cp[0].inv_d, idy_ = s.cp[1].inv_d, idz_ = s.cp[2].inv_d;
  (void)idx_; (void)idy_; (void)idz_;
  const T dx = s.dxyz[0], dy = s.dxyz[1], dz = s.dxyz[2];
  if (c == 0) {  // hx: CORRECT_Y then CORRECT_Z
    if (i >= Tx && i <= NX - Tx && k >= Tz && k < NZ - Tz) {
      if (j == Ty - 1) {  // source at j+1
        T ez = (T)(einc_at(s.e_inc, tf.m0, tf_proj(tf, di, dj + 2, dk + 1)) * (double)tf.fe[2]);
        v += che * ez / dy;
      } else if (j == NY - Ty) {
        T ez = (T)(einc_at(s.e_inc, tf.m0, tf_proj(tf, di, dj, dk + 1)) * (double)tf.fe[2]);
        v -= che * ez / dy;
      }
    }
    if (i >= Tx && i <= NX - Tx && j >= Ty && j < NY - Ty) {
      if (k == Tz - 1) {
        T ey = (T)(einc_at(s.e_inc, tf.m0, tf_proj(tf, di, dj + 1, dk + 2)) * (double)tf.fe[1]);
        v -= che * ey / dz;
      } else if (k == NZ - Tz) {
        T ey = (T)(einc_at(s.e_inc, tf.m0, tf_proj(tf, di, dj + 1, dk)) * (double)tf.fe[1]);
        v += che * ey / dz;
      }
    }
  } else if (c == 1) {  // hy: CORRECT_X then CORRECT_Z
    if (j >= Ty && j <= NY - Ty && k >= Tz && k < NZ - Tz) {
      if (i == Tx - 1) {
        T ez = (T)(einc_at(s.e_inc, tf.m0, tf_proj(tf, di + 2, dj, dk + 1)) * (double)tf.fe[2]);
        v -= che * ez / dx;
      } else if (i == NX - Tx) {
        T ez = (T)(einc_at(s.e_inc, tf.m0, tf_proj(tf, di, dj, dk + 1)) * (double)tf.fe[2]);
        v += che * ez / dx;
      }
    }
    if (i >= Tx && i < NX - Tx && j >= Ty && j <= NY - Ty) {
      if (k == Tz - 1) {
        T ex = (T)(einc_at(s.e_inc, tf.m0, tf_proj(tf, di + 1, dj, dk + 2)) * (double)tf.fe[0]);
        v += che * ex / dz;
      } else if (k == NZ - Tz) {
        T ex = (T)(einc_at(s.e_inc, tf.m0, tf_proj(tf, di + 1, dj, dk)) * (double)tf.fe[0]);
        v -= che * ex / dz;
      }
    }
  } else {  // hz: CORRECT_X then CORRECT_Y
    if (j >= Ty && j < NY - Ty && k >= Tz && k <= NZ - Tz) {
      if (i == Tx - 1) {
        T ey = (T)(einc_at(s.e_inc, tf.m0, tf_proj(tf, di + 2, dj + 1, dk)) * (double)tf.fe[1]);
        v += che * ey / dx;
      } else if (i == NX - Tx) {
        T ey = (T)(einc_at(s.e_inc, tf.m0, tf_proj(tf, di, dj + 1, dk)) * (double)tf.fe[1]);
        v -= che * ey / dx;
      }
    }
    if (i >= Tx && i < NX - Tx && k >= Tz && k <= NZ - Tz) {
      if (j == Ty - 1) {
        T ex = (T)(einc_at(s.e_inc, tf.m0, tf_proj(tf, di + 1, dj + 2, dk)) * (double)tf.fe[0]);
        v -= che * ex / dy;
      } else if (j == NY - Ty) {
        T ex = (T)(einc_at(s.e_inc, tf.m0, tf_proj(tf, di + 1, dj, dk)) * (double)tf.fe[0]);
        v += che * ex / dy;
      }
    }
  }
  return v;
}

// The E half of CORRECT_X/Y/Z, added to E component c before its update
// (the reference launches CORRECT_* before UPDATE_e*).  ceh is the cell's
// E-on-H coefficient (the reference uses Cexh for ex and ey, Cezh for ez;
// they are equal per cell).
template <typename T>
__device__ __noinline__ T tfsf_e(const SimView<T>& s, int c, int i, int j, int k, T v, T ceh) {
  const TfsfView& tf = s.tf;
  const int NX = s.NX, NY = s.NY, NZ = s.NZ;
  const int Tx = tf.Tx, Ty = tf.Ty, Tz = tf.Tz;
  const int di = 2 * (i - tf.i0), dj = 2 * (j - tf.j0), dk = 2 * (k - tf.k0);
  const T dx = s.dxyz[0], dy = s.dxyz[1], dz = s.dxyz[2];
  if (c == 0) {  // ex: CORRECT_Y then CORRECT_Z
    if (i >= Tx && i < NX - Tx && k >= Tz && k <= NZ - Tz) {
      if (j == Ty) {
        T hz = (T)(hinc_at(s.h_inc, tf.m0, tf_proj(tf, di + 1, dj - 1, dk)) * (double)tf.fh[2]);
        v -= ceh * hz / dy;
      } else if (j == NY - Ty) {
        T hz = (T)(hinc_at(s.h_inc, tf.m0, tf_proj(tf, di + 1, dj + 1, dk)) * (double)tf.fh[2]);
        v += ceh * hz / dy;
      }
    }
    if (i >= Tx && i < NX - Tx && j >= Ty && j <= NY - Ty) {
      if (k == Tz) {
        T hy = (T)(hinc_at(s.h_inc, tf.m0, tf_proj(tf, di + 1, dj, dk - 1)) * (double)tf.fh[1]);
        v += ceh * hy / dz;
      } else if (k == NZ - Tz) {
        T hy = (T)(hinc_at(s.h_inc, tf.m0, tf_proj(tf, di + 1, dj, dk + 1)) * (double)tf.fh[1]);
        v -= ceh * hy / dz;
      }
    }
  } else if (c == 1) {  // ey: CORRECT_X then CORRECT_Z
    if (j >= Ty && j < NY - Ty && k >= Tz && k <= NZ - Tz) {
      if (i == Tx) {
        T hz = (T)(hinc_at(s.h_inc, tf.m0, tf_proj(tf, di - 1, dj + 1, dk)) * (double)tf.fh[2]);
        v += ceh * hz / dx;
      } else if (i == NX - Tx) {
        T hz = (T)(hinc_at(s.h_inc, tf.m0, tf_proj(tf, di + 1, dj + 1, dk)) * (double)tf.fh[2]);
        v -= ceh * hz / dx;
      }
    }
    if (i >= Tx && i <= NX - Tx && j >= Ty && j < NY - Ty) {
      if (k == Tz) {
        T hx = (T)(hinc_at(s.h_inc, tf.m0, tf_proj(tf, di, dj + 1, dk - 1)) * (double)tf.fh[0]);
        v -= ceh * hx / dz;
      } else if (k == NZ - Tz) {
        T hx = (T)(hinc_at(s.h_inc, tf.m0, tf_proj(tf, di, dj + 1, dk + 1)) * (double)tf.fh[0]);
        v += ceh * hx / dz;
      }
    }
  } else {  // ez: CORRECT_X then CORRECT_Y
    if (j >= Ty && j <= NY - Ty && k >= Tz && k < NZ - Tz) {
      if (i == Tx) {
        T hy = (T)(hinc_at(s.h_inc, tf.m0, tf_proj(tf, di - 1, dj, dk + 1)) * (double)tf.fh[1]);
        v -= ceh * hy / dx;
      } else if (i == NX - Tx) {
        T hy = (T)(hinc_at(s.h_inc, tf.m0, tf_proj(tf, di + 1, dj, dk + 1)) * (double)tf.fh[1]);
        v += ceh * hy / dx;
      }
    }
    if (i >= Tx && i <= NX - Tx && k >= Tz && k < NZ - Tz) {
      if (j == Ty) {
        T hx = (T)(hinc_at(s.h_inc, tf.m0, tf_proj(tf, di, dj - 1, dk + 1)) * (double)tf.fh[0]);
        v += ceh * hx / dy;
      } else if (j == NY - Ty) {
        T hx = (T)(hinc_at(s.h_inc, tf.m0, tf_proj(tf, di, dj + 1, dk + 1)) * (double)tf.fh[0]);
        v -= ceh * hx / dy;
      }
    }
  }
  return v;
}

__device__ __forceinline__ bool near_tfsf_h(const TfsfView& tf, int NX, int NY, int NZ, int i, int j, int k) {
  return tf.on && (i == tf.Tx - 1 || i == NX - tf.Tx || j == tf.Ty - 1 || j == NY - tf.Ty ||
                   k == tf.Tz - 1 || k == NZ - tf.Tz);
}
__device__ __forceinline__ bool near_tfsf_e(const TfsfView& tf, int NX, int NY, int NZ, int i, int j, int k) {
  return tf.on && (i == tf.Tx || i == NX - tf.Tx || j == tf.Ty || j == NY - tf.Ty || k == tf.Tz ||
                   k == NZ - tf.Tz);
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

// One psi recursion of an H component along axis ax, applied with sign sg
// (UPDATE_h* CPML blocks, main.cu:829-861 and mirrors).
template <typename T>
__device__ __forceinline__ T cpml_h(const SimView<T>& s, int c, int slot, int ax, int i, int j, int k,
                                    T diff, T v, T sg) {
  const CpmlAxis<T>& a = s.cp[ax];
  int q = ax == 0 ? i : ax == 1 ? j : k;
  if (q < a.Nc) {
    T* p = s.psiH_N[c][slot] + slab_idx(s, ax, a.Nc, i, j, k);
    T ps = ldg(a.bh_N + q) * *p + ldg(a.ch_N + q) * diff * a.inv_d;
    *p = ps;
    v += sg * (s.che * ps);
  }
  if (q >= a.F) {
    int q2 = q - a.F;
    int ii = ax == 0 ? q2 : i, jj = ax == 1 ? q2 : j, kk = ax == 2 ? q2 : k;
    T* p = s.psiH_F[c][slot] + slab_idx(s, ax, a.Nc, ii, jj, kk);
    T ps = ldg(a.bh_F + q2) * *p + ldg(a.ch_F + q2) * diff * a.inv_d;
    *p = ps;
    v += sg * (s.che * ps);
  }
  return v;
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
// H pass: UPDATE_hx/hy/hz (main.cu:762-1044) fused, + H CPML + H TFSF.

template <typename T>
__global__ void __launch_bounds__(256) h_pass(SimView<T> s, int kchunk) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int NX = s.NX, NY = s.NY, NZ = s.NZ, PX = s.PX;
  if (i >= NX || j >= NY) return;
  const int k0 = blockIdx.z * kchunk;
  const int k1 = min(NZ, k0 + kchunk);
  const size_t plane = s.plane;
  const T* __restrict__ ex = s.E[0];
  const T* __restrict__ ey = s.E[1];
  const T* __restrict__ ez = s.E[2];
  T* __restrict__ hx = s.H[0];
  T* __restrict__ hy = s.H[1];
  T* __restrict__ hz = s.H[2];
  const bool hasx = i + 1 < NX, hasy = j + 1 < NY;
  const bool xs = in_slab(s.cp[0], i), ys = in_slab(s.cp[1], j);
  const T ikx = ldg(s.cp[0].inv_khd + i), iky = ldg(s.cp[1].inv_khd + j);
  size_t id = fidx(PX, plane, i, j, k0);
  T exk = ldg(ex + id), eyk = ldg(ey + id);
  const T che = s.che, chh = s.chh;
  for (int k = k0; k < k1; k++, id += plane) {
    const bool hask = k + 1 < NZ;
    const T exk1 = hask ? ldg(ex + id + plane) : T(0);
    const T eyk1 = hask ? ldg(ey + id + plane) : T(0);
    const T ezk = ldg(ez + id);
    const T ez_j = hasy ? ldg(ez + id + PX) : T(0);
    const T ex_j = hasy ? ldg(ex + id + PX) : T(0);
    const T ey_i = hasx ? ldg(ey + id + 1) : T(0);
    const T ez_i = hasx ? ldg(ez + id + 1) : T(0);
    const T ikz = ldg(s.cp[2].inv_khd + k);
    const bool in3 = hasx && hasy && hask;
    const bool zs = in_slab(s.cp[2], k);
    const bool tf = near_tfsf_h(s.tf, NX, NY, NZ, i, j, k);
    if (hasy && hask) {  // hx
      const T dey = eyk1 - eyk, dez = ez_j - ezk;
      T v = chh * hx[id] + che * (dey * ikz - dez * iky);
      if (in3 && (zs || ys)) {
        v = cpml_h(s, 0, 1, 2, i, j, k, dey, v, T(1));
        v = cpml_h(s, 0, 0, 1, i, j, k, dez, v, T(-1));
      }
      if (tf) v = tfsf_h(s, 0, i, j, k, v);
      hx[id] = v;
    }
    if (hasx && hask) {  // hy
      const T dez = ez_i - ezk, dex = exk1 - exk;
      T v = chh * hy[id] + che * (dez * ikx - dex * ikz);
      if (in3 && (zs || xs)) {
        v = cpml_h(s, 1, 0, 2, i, j, k, dex, v, T(-1));
        v = cpml_h(s, 1, 1, 0, i, j, k, dez, v, T(1));
      }
      if (tf) v = tfsf_h(s, 1, i, j, k, v);
      hy[id] = v;
    }
    if (hasx && hasy) {  // hz
      const T dex = ex_j - exk, dey = ey_i - eyk;
      T v = chh * hz[id] + che * (dex * iky - dey * ikx);
      if (in3 && (xs || ys)) {
        v = cpml_h(s, 2, 0, 0, i, j, k, dey, v, T(-1));
        v = cpml_h(s, 2, 1, 1, i, j, k, dex, v, T(1));
      }
      if (tf) v = tfsf_h(s, 2, i, j, k, v);
      hz[id] = v;
    }
    exk = exk1;
    eyk = eyk1;
  }
}

// ---------------------------------------------------------------------
// E pass: UPDATE_ex/ey/ez (main.cu:1048-1912) for non-dispersive
// components, with the E half of the TFSF added first and the E CPML after.
// Dispersive components are left untouched for metal_e*.

template <typename T>
__global__ void __launch_bounds__(256) e_pass(SimView<T> s, int kchunk) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int NX = s.NX, NY = s.NY, NZ = s.NZ, PX = s.PX;
  if (i >= NX || j >= NY) return;
  const int k0 = blockIdx.z * kchunk;
  const int k1 = min(NZ, k0 + kchunk);
  const size_t plane = s.plane;
  T* __restrict__ ex = s.E[0];
  T* __restrict__ ey = s.E[1];
  T* __restrict__ ez = s.E[2];
  const T* __restrict__ hx = s.H[0];
  const T* __restrict__ hy = s.H[1];
  const T* __restrict__ hz = s.H[2];
  const bool hasx = i > 0, hasy = j > 0;
  const bool okx = i < NX - 1, oky = j < NY - 1;
  const bool xs = in_slab(s.cp[0], i), ys = in_slab(s.cp[1], j);
  const T ikx = ldg(s.cp[0].inv_ked + i), iky = ldg(s.cp[1].inv_ked + j);
  const bool inbox_xy = i >= s.mat_lo[0] && i < s.mat_hi[0] && j >= s.mat_lo[1] && j < s.mat_hi[1];
  size_t id = fidx(PX, plane, i, j, k0);
  T hxm = k0 > 0 ? ldg(hx + id - plane) : T(0);
  T hym = k0 > 0 ? ldg(hy + id - plane) : T(0);
  int bad = 0;
  for (int k = k0; k < k1; k++, id += plane) {
    const T hxk = ldg(hx + id), hyk = ldg(hy + id), hzk = ldg(hz + id);
    const T hz_j = hasy ? ldg(hz + id - PX) : T(0);
    const T hx_j = hasy ? ldg(hx + id - PX) : T(0);
    const T hz_i = hasx ? ldg(hz + id - 1) : T(0);
    const T hy_i = hasx ? ldg(hy + id - 1) : T(0);
    const T ikz = ldg(s.cp[2].inv_ked + k);
    const bool okz = k < NZ - 1, hasz = k > 0;
    unsigned m = 0;
    if (inbox_xy && k >= s.mat_lo[2] && k < s.mat_hi[2]) m = s.mat[id];
    const int cls = m >> 3;
    const T cee = s.cee[cls], ceh = s.ceh[cls];
    const bool zs = in_slab(s.cp[2], k);
    const bool tf = near_tfsf_e(s.tf, NX, NY, NZ, i, j, k);
    if (okx && hasy && oky && hasz && okz && !(m & 1)) {  // ex
      const T dhz = hzk - hz_j, dhy = hyk - hym;
      T v = ex[id];
      if (tf) v = tfsf_e(s, 0, i, j, k, v, ceh);
      v = cee * v + ceh * (dhz * iky - dhy * ikz);
      if (zs || ys) {
        v = cpml_e(s, 0, 1, 2, i, j, k, dhy, v, T(-1), ceh);
        v = cpml_e(s, 0, 0, 1, i, j, k, dhz, v, T(1), ceh);
      }
      bad |= !isfinite((double)v);
      ex[id] = v;
    }
    if (hasx && okx && oky && hasz && okz && !(m & 2)) {  // ey
      const T dhx = hxk - hxm, dhz = hzk - hz_i;
      T v = ey[id];
      if (tf) v = tfsf_e(s, 1, i, j, k, v, ceh);
      v = cee * v + ceh * (dhx * ikz - dhz * ikx);
      if (zs || xs) {
        v = cpml_e(s, 1, 0, 2, i, j, k, dhx, v, T(1), ceh);
        v = cpml_e(s, 1, 1, 0, i, j, k, dhz, v, T(-1), ceh);
      }
      bad |= !isfinite((double)v);
      ey[id] = v;
    }
    if (hasx && okx && hasy && oky && okz && !(m & 4)) {  // ez
      const T dhy = hyk - hy_i, dhx = hxk - hx_j;
      T v = ez[id];
      if (tf) v = tfsf_e(s, 2, i, j, k, v, ceh);
      v = cee * v + ceh * (dhy * ikx - dhx * iky);
      if (ys || xs) {
        v = cpml_e(s, 2, 1, 1, i, j, k, dhx, v, T(-1), ceh);
        v = cpml_e(s, 2, 0, 0, i, j, k, dhy, v, T(1), ceh);
      }
      bad |= !isfinite((double)v);
      ez[id] = v;
    }
    hxm = hxk;
    hym = hyk;
  }
  if (bad) atomicOr(s.nonfinite, 1);
}

// ---------------------------------------------------------------------
// 1-D incident line (UPDATE_h_inc / UPDATE_e_inc, main.cu:2280-2337) with
// the Mur ends and the soft source that the reference applies on the host
// (main.cu:2831-2859).  One CTA.  Advances the device clock and records the
// probe (E after the previous step).

struct LineArgs {
  double* e_inc;
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

template <typename T>
__global__ void __launch_bounds__(1024) line_step(LineArgs a, SimView<T> s, size_t probe_id) {
  const int t = a.clk->t;
  // probe: E after step t-1 (OUT.txt records it at the top of step t)
  if (threadIdx.x < 3 && t >= 1 && t - 1 < a.probe_cap)
    a.probe[3 * (size_t)(t - 1) + threadIdx.x] = (double)s.E[threadIdx.x][probe_id];
  for (int q = threadIdx.x; q < a.L - 1; q += blockDim.x)
    a.h_inc[q] = a.h_inc[q] - a.ch * (a.e_inc[q + 1] - a.e_inc[q]);
  __syncthreads();
  for (int q = threadIdx.x + 1; q < a.L - 1; q += blockDim.x)
    a.e_inc[q] = a.e_inc[q] - a.ce * (a.h_inc[q] - a.h_inc[q - 1]);
  __syncthreads();
  if (threadIdx.x == 0) {
    double* e = a.e_inc;
    e[0] = a.clk->e1 + a.mur * (e[1] - e[0]);
    e[a.L - 1] = a.clk->e2 + a.mur * (e[a.L - 2] - e[a.L - 1]);
    a.clk->e1 = e[1];
    a.clk->e2 = e[a.L - 2];
    if (t < a.tmax) e[a.src] += a.pulse[t];
    // reserve this step's slot in the DFT sample ring (ScattAbs runs when
    // t % 4 == 0, main.cu:2920)
    if (a.dft_every > 0 && t % a.dft_every == 0) {
      const int slot = a.clk->nsamp;
      if (slot < kSampleBlock) {
        a.clk->samp_slot = slot;
        a.clk->samp_t[slot] = t;
        a.clk->nsamp = slot + 1;
      } else {
        a.clk->samp_slot = -1;  // ring full: the caller skipped a contraction
      }
    }
    a.clk->t = t + 1;
  }
}

template <typename T>
__global__ void probe_record(SimView<T> s, DevClock* clk, double* probe, int cap, size_t probe_id) {
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
  if (c == 0) {
    T dhz = hz[id] - hz[id - s.PX], dhy = hy[id] - hy[id - s.plane];
    *dh_a = dhz; *dh_b = dhy;  // y-slab diff, z-slab diff
    return dhz * s.cp[1].inv_ked[j] - dhy * s.cp[2].inv_ked[k];
  }
  if (c == 1) {
    T dhx = hx[id] - hx[id - s.plane], dhz = hz[id] - hz[id - 1];
    *dh_a = dhx; *dh_b = dhz;  // z-slab diff, x-slab diff
    return dhx * s.cp[2].inv_ked[k] - dhz * s.cp[0].inv_ked[i];
  }
  T dhy = hy[id] - hy[id - 1], dhx = hx[id] - hx[id - s.PX];
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

// Non-hydrodynamic dispersive update of all three components (they do not
// couple within a step).  pd ring: n = t%3, n-1 = (t+2)%3, new = (t+1)%3.
template <typename T>
__global__ void metal_e(SimView<T> s, MetalView<T> m, const DevClock* clk) {
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
  T v = s.E[c][id];
  if (near_tfsf_e(s.tf, s.NX, s.NY, s.NZ, i, j, k)) v = tfsf_e(s, c, i, j, k, v, ceh);
  T da, db;
  const T curl = curl_h_at(s, c, i, j, k, &da, &db);
  const T pdn = m.pd[c][rn][sl], pdn1 = m.pd[c][rn1][sl];
  const T cpn0 = m.cpn[c][0][sl], cpn1_0 = m.cpn1[c][0][sl];
  const T cpn1 = m.cpn[c][1][sl], cpn1_1 = m.cpn1[c][1][sl];
  T CP1 = T(0), CP2 = T(0), CP3 = T(0), CP4 = T(0);
  CP1 += (m.d1 - 1) * pdn;
  CP3 += m.d2 * pdn1;
  CP2 += (m.C1[0] - 1) * cpn0;
  CP2 += (m.C1[1] - 1) * cpn1;
  CP4 += m.C2[0] * cpn1_0;
  CP4 += m.C2[1] * cpn1_1;
  const T en1 = m.en[c][sl];  // e_n becomes e_n_1
  const T en = v;             // current E becomes e_n
  const T inv_CE = T(1) / m.C_E;
  T nv = inv_CE * (m.dt * curl / m.z0 + m.C_E_1 * en - m.C_E_2 * en1 - CP1 - CP2 - CP3 - CP4 - T(0));
  const T ncp0 = m.C1[0] * cpn0 + m.C2[0] * cpn1_0 + m.C3[0] * nv + m.C4[0] * en + m.C5[0] * en1;
  const T ncp1 = m.C1[1] * cpn1 + m.C2[1] * cpn1_1 + m.C3[1] * nv + m.C4[1] * en + m.C5[1] * en1;
  const T npd = m.d1 * pdn + m.d2 * pdn1 + m.d3 * nv + m.d4 * en + m.d5 * en1 + m.dNL * T(0);
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

// Slot lookup over the dispersive bounding box; -1 outside the metal.
template <typename T>
__device__ __forceinline__ int slot_of(const MetalView<T>& m, int a, int i, int j, int k) {
  int x = i - m.box_lo[0], y = j - m.box_lo[1], z = k - m.box_lo[2];
  if (x < 0 || y < 0 || z < 0 || x >= m.box_dim[0] || y >= m.box_dim[1] || z >= m.box_dim[2]) return -1;
  return m.slot_map[a][((size_t)z * m.box_dim[1] + y) * m.box_dim[0] + x];
}

// Ring position of component a's "current" Drude current and density as
// seen during component c's phase of step t (components before c have
// already rotated, as the reference's sequential launches imply).
template <typename T>
__device__ __forceinline__ T pd_cur(const MetalView<T>& m, int a, int c, int t, int i, int j, int k) {
  int sl = slot_of(m, a, i, j, k);
  if (sl < 0) return T(0);
  int r = (a < c) ? (t + 1) % 3 : t % 3;
  return m.pd[a][r][sl];
}
template <typename T>
__device__ __forceinline__ T nd_cur(const MetalView<T>& m, int a, int c, int t, int i, int j, int k) {
  int sl = slot_of(m, a, i, j, k);
  if (sl < 0) return T(0);
  int r = ((a < c) ? (t + 1) : t) & 1;
  return m.nd[a][r][sl];
}

// UpdateHydroPx/Py/Pz (main.cu:1916-2276): new hydrodynamic Drude current of
// every dispersive cell from E^n (after the TFSF pre-add), its history and
// the pressure term.  Convection and Lorentz terms are off in the reference.
template <typename T>
__global__ void hydro_p(SimView<T> s, MetalView<T> m, const DevClock* clk) {
  const int t = clk->t - 1;
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  int c = 0;
  while (c < 3 && q >= m.n[c]) { q -= m.n[c]; c++; }
  if (c >= 3) return;
  const int4 e = m.cell[c][q];
  const int i = e.x, j = e.y, k = e.z, sl = e.w;
  const size_t id = fidx(s.PX, s.plane, i, j, k);
  const T IX = m.inv_dx, IY = m.inv_dy, IZ = m.inv_dz;
#define PA(a, ii, jj, kk) pd_cur(m, a, 0, t, ii, jj, kk)
#define NA(a, ii, jj, kk) nd_cur(m, a, 0, t, ii, jj, kk)
#define PN(a, ii, jj, kk) (PA(a, ii, jj, kk) * NA(a, ii, jj, kk))
  T gd, gd2;
  if (c == 0) {
    gd2 = IX * IX * (PN(0, i + 1, j, k) - T(2) * PN(0, i, j, k) + PN(0, i - 1, j, k)) +
          IX * IY * (PN(1, i + 1, j, k) - PN(1, i, j, k) - PN(1, i + 1, j - 1, k) + PN(1, i, j - 1, k)) +
          IX * IZ * (PN(2, i + 1, j, k) - PN(2, i, j, k) - PN(2, i + 1, j, k - 1) + PN(2, i, j, k - 1));
    gd = IX * IX * (PA(0, i + 1, j, k) - T(2) * PA(0, i, j, k) + PA(0, i - 1, j, k)) +
         IX * IY * (PA(1, i + 1, j, k) - PA(1, i, j, k) - PA(1, i + 1, j - 1, k) + PA(1, i, j - 1, k)) +
         IX * IZ * (PA(2, i + 1, j, k) - PA(2, i, j, k) - PA(2, i + 1, j, k - 1) + PA(2, i, j, k - 1));
  } else if (c == 1) {
    gd2 = IY * IY * (PN(1, i, j + 1, k) - T(2) * PN(1, i, j, k) + PN(1, i, j - 1, k)) +
          IX * IY * (PN(0, i, j + 1, k) - PN(0, i, j, k) - PN(0, i - 1, j + 1, k) + PN(0, i - 1, j, k)) +
          IY * IZ * (PN(2, i, j + 1, k) - PN(2, i, j, k) - PN(2, i, j + 1, k - 1) + PN(2, i, j, k - 1));
    gd = IY * IY * (PA(1, i, j + 1, k) - T(2) * PA(1, i, j, k) + PA(1, i, j - 1, k)) +
         IX * IY * (PA(0, i, j + 1, k) - PA(0, i, j, k) - PA(0, i - 1, j + 1, k) + PA(0, i - 1, j, k)) +
         IY * IZ * (PA(2, i, j + 1, k) - PA(2, i, j, k) - PA(2, i, j + 1, k - 1) + PA(2, i, j, k - 1));
  } else {
    gd2 = IZ * IZ * (PN(2, i, j, k + 1) - T(2) * PN(2, i, j, k) + PN(2, i, j, k - 1)) +
          IZ * IY * (PN(1, i, j, k + 1) - PN(1, i, j, k) - PN(1, i, j - 1, k + 1) + PN(1, i, j - 1, k)) +
          IX * IZ * (PN(0, i, j, k + 1) - PN(0, i, j, k) - PN(0, i - 1, j, k + 1) + PN(0, i - 1, j, k));
    gd = IZ * IZ * (PA(2, i, j, k + 1) - T(2) * PA(2, i, j, k) + PA(2, i, j, k - 1)) +
         IZ * IY * (PA(1, i, j, k + 1) - PA(1, i, j, k) - PA(1, i, j - 1, k + 1) + PA(1, i, j - 1, k)) +
         IX * IZ * (PA(0, i, j, k + 1) - PA(0, i, j, k) - PA(0, i - 1, j, k + 1) + PA(0, i - 1, j, k));
  }
#undef PA
#undef NA
#undef PN
  const T nd_prev = m.nd[c][t & 1][sl];
  const T ND1 = m.N_EQ + nd_prev;
  T cb;
  if (m.fix_cbrt) cb = (T)cbrt((double)ND1);
  else cb = (T)powf((float)ND1, (float)(1.0 / 3.0));
  // E^n after the TFSF pre-add: dispersive cells never sit on the TFSF faces
  // in the hydrodynamic model (checked at create), so E is read as stored.
  const T ev = s.E[c][id];
  const T pn = m.pd[c][t % 3][sl], pn1 = m.pd[c][(t + 2) % 3][sl];
  const T npd = m.d1 * pn + m.d2 * pn1 + m.d3 * ev + m.d4 * m.en[c][sl] + m.d5 * T(0) +
                m.dNL * (gd + gd2 / m.N_EQ) / cb;
  m.pd[c][(t + 1) % 3][sl] = npd;
}

// Hydrodynamic E update of component c (UPDATE_e* hydro branch,
// main.cu:1220-1271 and mirrors): continuity for the density
// perturbation, then E with the current source e0 (N_EQ + N) J.
template <typename T>
__global__ void metal_e_hydro(SimView<T> s, MetalView<T> m, const DevClock* clk, int c) {
  const int t = clk->t - 1;
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= m.n[c]) return;
  const int4 e = m.cell[c][q];
  const int i = e.x, j = e.y, k = e.z, sl = e.w;
  const size_t id = fidx(s.PX, s.plane, i, j, k);
  const unsigned mb = s.mat[id];
  const T ceh = s.ceh[mb >> 3];
  // continuity
  T V1[3], V2[3], N1[3], N2[3];
  const int o0 = c == 0, o1 = c == 1, o2 = c == 2;
#pragma unroll
  for (int a = 0; a < 3; a++) {
    if (a == c) {
      V1[a] = pd_cur(m, a, c, t, i + o0, j + o1, k + o2);
      V2[a] = pd_cur(m, a, c, t, i - o0, j - o1, k - o2);
      N1[a] = nd_cur(m, a, c, t, i + o0, j + o1, k + o2);
      N2[a] = nd_cur(m, a, c, t, i - o0, j - o1, k - o2);
    } else {
      const int b0 = a == 0, b1 = a == 1, b2 = a == 2;
      V1[a] = T(0.5) * (pd_cur(m, a, c, t, i + o0, j + o1, k + o2) + pd_cur(m, a, c, t, i, j, k));
      V2[a] = T(0.5) * (pd_cur(m, a, c, t, i + o0 - b0, j + o1 - b1, k + o2 - b2) +
                        pd_cur(m, a, c, t, i - b0, j - b1, k - b2));
      N1[a] = T(0.5) * (nd_cur(m, a, c, t, i + o0, j + o1, k + o2) + nd_cur(m, a, c, t, i, j, k));
      N2[a] = T(0.5) * (nd_cur(m, a, c, t, i + o0 - b0, j + o1 - b1, k + o2 - b2) +
                        nd_cur(m, a, c, t, i - b0, j - b1, k - b2));
    }
  }
  const T ndm1 = m.nd[c][(t + 1) & 1][sl];  // N^{n-1}
  const T k2 = T(2) * m.dt * m.inv_dx;
  T nd;
  if (c == 0)
    nd = ndm1 - k2 * (T(0.5) * (N1[0] * V1[0] - N2[0] * V2[0]) + (N1[1] * V1[1] - N2[1] * V2[1]) +
                      (N1[2] * V1[2] - N2[2] * V2[2]) +
                      (T(0.5) * (V1[0] - V2[0]) + (V1[1] - V2[1]) + (V1[2] - V2[2])) * m.N_EQ);
  else if (c == 1)
    nd = ndm1 - k2 * ((N1[0] * V1[0] - N2[0] * V2[0]) + T(0.5) * (N1[1] * V1[1] - N2[1] * V2[1]) +
                      (N1[2] * V1[2] - N2[2] * V2[2]) +
                      ((V1[0] - V2[0]) + T(0.5) * (V1[1] - V2[1]) + (V1[2] - V2[2])) * m.N_EQ);
  else
    nd = ndm1 - k2 * ((N1[0] * V1[0] - N2[0] * V2[0]) + (N1[1] * V1[1] - N2[1] * V2[1]) +
                      T(0.5) * (V1[2] - V2[2]) +
                      ((V1[0] - V2[0]) + (V1[1] - V2[1]) + T(0.5) * (V1[2] - V2[2])) * m.N_EQ);
  // E update
  const T v = s.E[c][id];
  T da, db;
  const T curl = curl_h_at(s, c, i, j, k, &da, &db);
  const T cpn0 = m.cpn[c][0][sl], cpn1_0 = m.cpn1[c][0][sl];
  const T cpn1 = m.cpn[c][1][sl], cpn1_1 = m.cpn1[c][1][sl];
  T CP2 = T(0), CP4 = T(0);
  CP2 += (m.C1[0] - 1) * cpn0;
  CP2 += (m.C1[1] - 1) * cpn1;
  CP4 += m.C2[0] * cpn1_0;
  CP4 += m.C2[1] * cpn1_1;
  const T en1 = m.en[c][sl];
  const T en = v;
  const T jd = m.pd[c][(t + 1) % 3][sl];  // current from hydro_p
  const T inv_CE = T(1) / m.C_E;
  T nv = inv_CE * (m.dt * curl / m.z0 + m.dt * jd * m.e0 * (m.N_EQ + nd) + m.C_E_1 * en - m.C_E_2 * en1 - CP2 -
                   CP4);
  const T ncp0 = m.C1[0] * cpn0 + m.C2[0] * cpn1_0 + m.C3[0] * nv + m.C4[0] * en + m.C5[0] * en1;
  const T ncp1 = m.C1[1] * cpn1 + m.C2[1] * cpn1_1 + m.C3[1] * nv + m.C4[1] * en + m.C5[1] * en1;
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

// ---------------------------------------------------------------------
// DFT flux planes (ScattAbs, main.cu:35-366).

// One flux face: rows [row0, row0 + 4*na*nb), component-major, then u, v.
struct DftFace {
  int ax, pos;          // normal axis and plane index
  int s1, s2;           // start of the two tangential axes
  int na, nb;           // extents (END - START)
  int comp[4];          // field components 0..5
  long long row0;
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
__global__ void dft_sample(SimView<T> s, DftView d, T* ring, const DevClock* clk) {
  const int slot = clk->samp_slot;
  if (slot < 0 || slot >= kSampleBlock) return;
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
      ring[(size_t)slot * d.rows + F.row0 + (size_t)c * n + q] = x;
    }
  }
}

// acc[f][r] += sum_s x[s][r] * exp(i 2 pi (t_s + delta) dt freq[f]), delta =
// 1 for E rows and 1/2 for H rows (main.cu:62-76), in FP64.  Block: 128
// rows x one frequency tile; the tile's phasors live in shared memory.
constexpr int kDftRows = 128;
constexpr int kDftFreqs = 16;

template <typename T>
__global__ void __launch_bounds__(kDftRows) dft_contract(DftView d, const T* ring, DevClock* clk, int nsamp_arg) {
  __shared__ double cs[2][kSampleBlock][kDftFreqs];  // E/H cos
  __shared__ double sn[2][kSampleBlock][kDftFreqs];
  const int nsamp = min(kSampleBlock, nsamp_arg > 0 ? nsamp_arg : clk->nsamp);
  const int f0 = blockIdx.y * kDftFreqs;
  const int nfl = min(kDftFreqs, d.nf - f0);
  for (int q = threadIdx.x; q < 2 * kSampleBlock * kDftFreqs; q += blockDim.x) {
    const int h = q / (kSampleBlock * kDftFreqs);
    const int r = q - h * kSampleBlock * kDftFreqs;
    const int sidx = r / kDftFreqs, fl = r - sidx * kDftFreqs;
    double c = 0, sv = 0;
    if (sidx < nsamp && fl < nfl) {
      const int ts = clk->samp_t[sidx];
      const double ph = (double)(float)2.0 * 3.1415926535897932384626433832795 * (ts + (h ? 0.5 : 1.0)) * d.dt *
                        d.freq[f0 + fl];
      sincos(ph, &sv, &c);
    }
    cs[h][sidx][fl] = c;
    sn[h][sidx][fl] = sv;
  }
  __syncthreads();
  const long long r = (long long)blockIdx.x * kDftRows + threadIdx.x;
  if (r >= d.rows) return;
  // which face / component this row belongs to (E or H twiddles)
  int h = 0;
  for (int f = 0; f < d.nfaces; f++) {
    const long long n = (long long)d.face[f].na * d.face[f].nb;
    if (r >= d.face[f].row0 && r < d.face[f].row0 + 4 * n) {
      h = (r - d.face[f].row0) >= 2 * n;
      break;
    }
  }
  double x[kSampleBlock];
#pragma unroll
  for (int q = 0; q < kSampleBlock; q++) x[q] = q < nsamp ? (double)ring[(size_t)q * d.rows + r] : 0.0;
  for (int fl = 0; fl < nfl; fl++) {
    double re = 0, im = 0;
#pragma unroll
    for (int q = 0; q < kSampleBlock; q++) {
      re = fma(x[q], cs[h][q][fl], re);
      im = fma(x[q], sn[h][q][fl], im);
    }
    const size_t o = (size_t)(f0 + fl) * d.rows + r;
    d.acc_re[o] += re;
    d.acc_im[o] += im;
  }
}

__global__ void dft_reset_count(DevClock* clk) { clk->nsamp = 0; }

// Per (box-face, frequency): sum over the face of Re(cEx conj(HY) -
// cEy conj(HX)) with the reference's component pairing
// (CalculateAbsScatt, Spectral.cu:725-1132).  Y faces swap the pair.
__global__ void flux_reduce(DftView d, double* out /* [12][nf] */) {
  const int f = blockIdx.x, m = blockIdx.y;
  const DftFace F = d.face[f];
  const long long n = (long long)F.na * F.nb;
  const int qx = F.ax == 1 ? 1 : 0, qy = F.ax == 1 ? 0 : 1;
  const double* re = d.acc_re + (size_t)m * d.rows + F.row0;
  const double* im = d.acc_im + (size_t)m * d.rows + F.row0;
  double acc = 0;
  for (long long q = threadIdx.x; q < n; q += blockDim.x) {
    const double exr = re[qx * n + q], exi = im[qx * n + q];
    const double eyr = re[qy * n + q], eyi = im[qy * n + q];
    const double hxr = re[(2 + qx) * n + q], hxi = im[(2 + qx) * n + q];
    const double hyr = re[(2 + qy) * n + q], hyi = im[(2 + qy) * n + q];
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
