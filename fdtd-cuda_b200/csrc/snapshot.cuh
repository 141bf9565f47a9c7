// Snapshots as the reference writes them (SNAPSHOT_1D, SNAPSHOT_2D and
// SNAPSHOT_2D_N, snapshot.cu:23-176), taken on the device by the stepper
// after every step t with t % t_skip == 0 (the schedule of main.cu:2948-2991)
// into a ring of records that the host drains asynchronously.
//
// One record holds the step index and, by the reference's Snap_in mode:
//   1  the aux lines: ey at (2, 2, k) and the incident line's E, both with
//      step z_skip (SNAPSHOT_1D)
//   2  the YZ plane at x = NX/2 of |P_d| and of (NDx + NDy + NDz) / 3 (the
//      reference copies its Drude currents into the host E arrays before
//      SNAPSHOT_2D, main.cu:2960-2962; its NDx after the swap at the end of
//      its E update holds the density from before the step, main.cu:1267-1269)
//   3  the aux lines, then the YZ plane of |E| (SNAPSHOT_1D, SNAPSHOT_2D)
// Planes run over y with step y_skip (rows) and z with step z_skip
// (columns), values in FP64.
#pragma once
#include "kernels.cuh"

namespace fdtd {

struct SnapArgs {
  int mode;                 // Snap_in: 1, 2 or 3
  int t_skip, y_skip, z_skip;
  int xc;                   // x index of the YZ plane
  int rows, cols;           // plane extent
  int aux_len, line_len;    // aux line lengths
  int rec;                  // doubles per record
  int cap;                  // records in the ring
  int off_plane, off_plane2, off_aux, off_line;  // offsets in a record, -1 = absent
  const int* pslot;         // [rows * cols][3]: dispersive slot per component, -1 = none
  double* ring;             // [cap][rec]
};

template <typename T>
__global__ void snap_gather(const __grid_constant__ SimView<T> s, const __grid_constant__ MetalView<T> m,
                            const __grid_constant__ LineArgs line, const __grid_constant__ SnapArgs a) {
  const int tn = line.clk->t;  // the step just completed is tn - 1
  const int t = tn - 1;
  if (t < 0 || t % a.t_skip) return;
  double* r = a.ring + (size_t)((t / a.t_skip) % a.cap) * a.rec;
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q == 0) r[0] = (double)t;
  if (a.off_plane >= 0 && q < a.rows * a.cols) {
    const int j = (q / a.cols) * a.y_skip, k = (q % a.cols) * a.z_skip;
    if (a.mode == 3) {
      const size_t id = fidx(s.PX, s.plane, a.xc, j, k);
      const double ex = (double)s.E[0][id], ey = (double)s.E[1][id], ez = (double)s.E[2][id];
      r[a.off_plane + q] = sqrt(ex * ex + ey * ey + ez * ez);
    } else {
      const int* ps = a.pslot + (size_t)q * 3;
      double p[3], nd[3];
#pragma unroll
      for (int c = 0; c < 3; c++) {
        const int sl = ps[c];
        p[c] = sl >= 0 ? m.pd[c][(t + 1) % 3][sl] : 0.0;
        nd[c] = (sl >= 0 && m.hydro) ? m.nd[c][t & 1][sl] : 0.0;
      }
      r[a.off_plane + q] = sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
      r[a.off_plane2 + q] = (nd[0] + nd[1] + nd[2]) / 3.0;
    }
  }
  if (a.off_aux >= 0 && q < a.aux_len) r[a.off_aux + q] = (double)s.E[1][fidx(s.PX, s.plane, 2, 2, q * a.z_skip)];
  if (a.off_line >= 0 && q < a.line_len) r[a.off_line + q] = line_e(line, tn)[(size_t)q * a.z_skip];
}

}  // namespace fdtd
