// TFSF work of the time step, on the cells that need it only:
//   tfsf_tabulate                 at create: the corrections of CORRECT_X/Y/Z
//                                 (main.cu:369-758) on the TFSF box faces
//   tfsf_h_apply / tfsf_e_apply   every step: after the H update for H,
//                                 before the E update for E
// Splitting these off keeps the Yee passes branch-free: x is the warp
// dimension, so the x faces would otherwise make two warps of every row
// execute the face code.
#pragma once
#include <algorithm>

#include "kernels.cuh"

namespace fdtd {

// Cells on the shell of the box [lo, hi] per axis, each once: the two x
// faces, then the y faces without their x edges, then the z faces without
// x and y edges.
struct ShellCells {
  int lo[3], hi[3];
  long long n0, n1, n2;
  __host__ void init(const int l[3], const int h[3]) {
    for (int a = 0; a < 3; a++) { lo[a] = l[a]; hi[a] = h[a]; }
    const long long ex = hi[0] - lo[0] + 1, ey = hi[1] - lo[1] + 1, ez = hi[2] - lo[2] + 1;
    n0 = 2 * ey * ez;
    n1 = 2 * (ex - 2 > 0 ? ex - 2 : 0) * ez;
    n2 = 2 * (ex - 2 > 0 ? ex - 2 : 0) * (ey - 2 > 0 ? ey - 2 : 0);
  }
  __host__ __device__ long long total() const { return n0 + n1 + n2; }
  __device__ void cell(long long q, int& i, int& j, int& k) const {
    const int ey = hi[1] - lo[1] + 1, ex2 = hi[0] - lo[0] - 1, ey2 = hi[1] - lo[1] - 1;
    if (q < n0) {
      j = lo[1] + (int)(q % ey);
      const long long r = q / ey;
      k = lo[2] + (int)(r / 2);
      i = (r & 1) ? hi[0] : lo[0];
    } else if (q < n0 + n1) {
      q -= n0;
      i = lo[0] + 1 + (int)(q % ex2);
      const long long r = q / ex2;
      k = lo[2] + (int)(r / 2);
      j = (r & 1) ? hi[1] : lo[1];
    } else {
      q -= n0 + n1;
      i = lo[0] + 1 + (int)(q % ex2);
      const long long r = q / ex2;
      j = lo[1] + 1 + (int)((r / 2) % ey2);
      k = (r & 1) ? hi[2] : lo[2];
    }
  }
};

// TFSF corrections tabulated once at create: per face cell and component
// with at least one correction, up to two (line index, weight, meta) terms
// in the reference's order; meta = (sign > 0) | axis << 1 | component << 3.
// A term whose polarisation factor is exactly zero (the incident field has
// no such component, e.g. E_z and H_z of a wave along z) adds a signed zero
// and is left out.
// Applying a term adds sign * coefficient * (interpolated incident value)
// * (polarisation factor) / d_axis, the arithmetic of the walk forms in
// kernels.cuh with the projection and the truncation already done.
// The table is one 16-byte entry per corrected component (cell offset, the
// two term numbers, component | terms << 2 | dielectric class << 8) and a
// table of the distinct terms: a plane wave's terms depend on the face cell
// only through its projection on the incidence direction, so at normal
// incidence a face holds a few hundred distinct terms for its ~10^5 cells.
struct TfsfTerm {
  double dp;  // interpolation weight of the right point
  int idx;    // line index of the left point
  int meta;
};
struct TfsfTable {
  int n;                  // entries
  const uint4* ent;       // (cell offset, term 0, term 1, component | terms << 2 | class << 8)
  const TfsfTerm* term;   // distinct terms
};

// dense build: slot (q, c) of shell cell q and component c
template <typename T>
__global__ void tfsf_tabulate(const SimView<T>* __restrict__ gv, const ShellCells sh, int efield, unsigned* id,
                              unsigned* cn, int* idx0, int* idx1, double* dp0, double* dp1,
                              unsigned char* m0, unsigned char* m1) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= sh.total()) return;
  const SimView<T>& g = *gv;
  int i, j, k;
  sh.cell(q, i, j, k);
  const size_t cell = fidx(g.PX, g.plane, i, j, k);
  // the E corrections take the cell's dielectric class coefficient
  unsigned cls = 0;
  if (efield && i >= g.mat_lo[0] && i < g.mat_hi[0] && j >= g.mat_lo[1] && j < g.mat_hi[1] && k >= g.mat_lo[2] &&
      k < g.mat_hi[2])
    cls = (unsigned)g.mat[cell] >> 3;
  for (int c = 0; c < 3; c++) {
    int nt = 0;
    int ix[2] = {0, 0};
    double w[2] = {0, 0};
    unsigned char mm[2] = {0, 0};
    const float* fac = efield ? g.tf.fh : g.tf.fe;
    auto rec = [&](int sg, int ax, int f, double d) {
      if (fac[f] == 0.0f) return;
      if (nt < 2) {
        if (efield) {  // hinc_at
          const double d2 = d + 0.5;
          const int n = (int)d2;
          ix[nt] = g.tf.m0 - 1 + n;
          w[nt] = d2 - n;
        } else {  // einc_at
          const int n = (int)d;
          ix[nt] = g.tf.m0 + n;
          w[nt] = d - n;
        }
        mm[nt] = (unsigned char)((sg > 0 ? 1 : 0) | (ax << 1) | (f << 3));
      }
      nt++;
    };
    if (efield) tfsf_e_walk(g, c, i, j, k, rec);
    else tfsf_h_walk(g, c, i, j, k, rec);
    const size_t o = (size_t)q * 3 + c;
    id[o] = (unsigned)cell;
    cn[o] = (unsigned)c | ((unsigned)min(nt, 3) << 2) | (cls << 8);  // 3 terms would be a bug: flagged, not applied
    idx0[o] = ix[0]; idx1[o] = ix[1];
    dp0[o] = w[0]; dp1[o] = w[1];
    m0[o] = mm[0]; m1[o] = mm[1];
  }
}

template <typename T>
__device__ __forceinline__ T tfsf_term(const double* line, const float* dir, const TfsfTerm& t, T v, T coef,
                                       const T* dd) {
  const unsigned meta = (unsigned)t.meta;
  const T x = (T)(((1 - t.dp) * line[t.idx] + t.dp * line[t.idx + 1]) * (double)dir[meta >> 3]);
  const int ax = (meta >> 1) & 3;
  if (meta & 1) v += coef * x / dd[ax];
  else v -= coef * x / dd[ax];
  return v;
}

// Entry g of the H table: e_line is the incident line's E from before this
// step's line update.
template <typename T>
__device__ __forceinline__ void tfsf_h_entry(const SimView<T>& s, const TfsfTable& tb, int g, const double* e_line) {
  const uint4 e = tb.ent[g];
  const int c = e.w & 3, nt = (e.w >> 2) & 3;
  const T dd[3] = {s.dxyz[0], s.dxyz[1], s.dxyz[2]};
  T v = s.H[c][e.x];
  v = tfsf_term(e_line, s.tf.fe, tb.term[e.y], v, s.che, dd);
  if (nt > 1) v = tfsf_term(e_line, s.tf.fe, tb.term[e.z], v, s.che, dd);
  s.H[c][e.x] = v;
}

// Entry g of the E table (the line's H after this step's line update).
template <typename T>
__device__ __forceinline__ void tfsf_e_entry(const SimView<T>& s, const TfsfTable& tb, int g) {
  const uint4 e = tb.ent[g];
  const int c = e.w & 3, nt = (e.w >> 2) & 3;
  const T ceh = s.ceh[e.w >> 8];
  const T dd[3] = {s.dxyz[0], s.dxyz[1], s.dxyz[2]};
  T v = s.E[c][e.x];
  v = tfsf_term(s.h_inc, s.tf.fh, tb.term[e.y], v, ceh, dd);
  if (nt > 1) v = tfsf_term(s.h_inc, s.tf.fh, tb.term[e.z], v, ceh, dd);
  s.E[c][e.x] = v;
}

// The halves as separate launches (the split per-half entry points) and
// fused: the H entries write H face cells from the line's E, the E entries
// write E face cells from the line's H, so one launch can run both once
// the line step is done.  Thread g < th.n takes H entry g, the rest the E
// entries.
template <typename T>
__device__ __forceinline__ void tfsf_h_apply_body(const SimView<T>& s, const TfsfTable& tb, const LineArgs& line) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g < tb.n) tfsf_h_entry(s, tb, g, line_e_before(line, 0));
}
template <typename T>
__device__ __forceinline__ void tfsf_e_apply_body(const SimView<T>& s, const TfsfTable& tb) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g < tb.n) tfsf_e_entry(s, tb, g);
}
template <typename T>
__device__ __forceinline__ void tfsf_apply_body(const SimView<T>& s, const TfsfTable& th, const TfsfTable& te,
                                                const LineArgs& line) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g < th.n) tfsf_h_entry(s, th, g, line_e_before(line, 1));
  else if (g - th.n < te.n) tfsf_e_entry(s, te, g - th.n);
}
template <typename T>
__global__ void tfsf_h_apply(const __grid_constant__ SimView<T> s, const __grid_constant__ TfsfTable tb,
                             const __grid_constant__ LineArgs line) {
  tfsf_h_apply_body(s, tb, line);
}
template <typename T>
__global__ void tfsf_e_apply(const __grid_constant__ SimView<T> s, const __grid_constant__ TfsfTable tb) {
  tfsf_e_apply_body(s, tb);
}
template <typename T>
__global__ void tfsf_apply(const __grid_constant__ SimView<T> s, const __grid_constant__ TfsfTable th,
                           const __grid_constant__ TfsfTable te, const __grid_constant__ LineArgs line) {
  tfsf_apply_body(s, th, te, line);
}

}  // namespace fdtd
