// TFSF work of the time step, on the cells that need it only:
//   tfsf_h_faces / tfsf_e_faces   CORRECT_X/Y/Z (main.cu:369-758) on the
//                                 cells of the TFSF box faces: after the H
//                                 update for H, before the E update for E
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

template <typename T>
__device__ __forceinline__ void tfsf_h_faces_body(const SimView<T>& g, const ShellCells& sh) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= sh.total()) return;
  int i, j, k;
  sh.cell(q, i, j, k);
  const size_t id = fidx(g.PX, g.plane, i, j, k);
#pragma unroll
  for (int c = 0; c < 3; c++) {
    g.H[c][id] = tfsf_h(g, c, i, j, k, g.H[c][id]);
  }
}
template <typename T>
__global__ void tfsf_h_faces(const SimView<T>* __restrict__ gv, const ShellCells sh) {
  tfsf_h_faces_body(*gv, sh);
}

template <typename T>
__device__ __forceinline__ void tfsf_e_faces_body(const SimView<T>& g, const ShellCells& sh) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= sh.total()) return;
  int i, j, k;
  sh.cell(q, i, j, k);
  const size_t id = fidx(g.PX, g.plane, i, j, k);
  unsigned m = 0;
  if (i >= g.mat_lo[0] && i < g.mat_hi[0] && j >= g.mat_lo[1] && j < g.mat_hi[1] && k >= g.mat_lo[2] &&
      k < g.mat_hi[2])
    m = g.mat[id];
  const T ceh = g.ceh[m >> 3];
#pragma unroll
  for (int c = 0; c < 3; c++) {
    g.E[c][id] = tfsf_e(g, c, i, j, k, g.E[c][id], ceh);
  }
}
template <typename T>
__global__ void tfsf_e_faces(const SimView<T>* __restrict__ gv, const ShellCells sh) {
  tfsf_e_faces_body(*gv, sh);
}

}  // namespace fdtd
