// Shared-memory-staged E and H passes: the Yee updates of all cells with the
// CPML psi recursions of the six absorbing slabs fused in (UPDATE_hx/hy/hz
// and UPDATE_ex/ey/ez with their CPML blocks; the TFSF corrections and the
// dispersive cells are applied by the kernels of boundary.cuh and
// kernels.cuh).
//
// Each CTA owns a 32 x TY tile of (x, y) columns and marches along z through
// its z-chunk.  The planes it needs are streamed into a ring of S shared-
// memory stages, so two planes of loads are in flight while a third is
// computed, independent of occupancy: either every thread issues a share of
// the plane's 16-byte cp.async copies, or one thread issues the plane's six
// tensor copies (cp.async.bulk.tensor, completing on the stage's mbarrier);
// the autotuner picks per launch.  Per plane a stage holds
//   the "halo" family  (3 components, TY+1 rows, 32+CH columns): the field
//                      read at the +-1 neighbours (E in the H pass, H in the
//                      E pass), CH = 16 bytes / sizeof(T) columns of x halo
//   the "own" family   (3 components, TY rows, 32 columns): the field being
//                      updated
// Out-of-grid rows, columns and planes are zero-filled by the copy (the
// reference's PEC outer boundary).
//
// CPML: a z-slab plane is uniform across the CTA and a y-slab row across a
// warp; only the x slabs split a warp (lanes 0..Nc of the first x tile and
// the last lanes of the last).  The psi values of a cell for plane k+1 are
// loaded into registers while plane k is computed, so their DRAM latency
// overlaps one plane of work; every psi element belongs to one cell and is
// read and written only by that cell's thread.
#pragma once
#include <cuda.h>

#include "kernels.cuh"

namespace fdtd {

// Which CPML slab a cell index lies in (side: 0 none, 1 near, 2 far), the
// index inside it and the recursion coefficients there.  E extent: index <=
// Nc or >= F; H extent: index < Nc or >= F.
template <typename T>
struct SlabAt {
  int side;
  int q;
  T b, c;
};

template <typename T>
__device__ __forceinline__ SlabAt<T> slab_e(const CpmlAxis<T>& a, int n, const T* ceN) {
  SlabAt<T> r;
  r.side = 0; r.q = 0; r.b = T(0); r.c = T(0);
  if (n < a.Nc + 1) { r.side = 1; r.q = n; r.b = ldg(a.be_N + n); r.c = ldg(ceN + n); }
  else if (n >= a.F) { r.side = 2; r.q = n - a.F; r.b = ldg(a.be_F + r.q); r.c = ldg(a.ce_F + r.q); }
  return r;
}
template <typename T>
__device__ __forceinline__ SlabAt<T> slab_h(const CpmlAxis<T>& a, int n) {
  SlabAt<T> r;
  r.side = 0; r.q = 0; r.b = T(0); r.c = T(0);
  if (n < a.Nc) { r.side = 1; r.q = n; r.b = ldg(a.bh_N + n); r.c = ldg(a.ch_N + n); }
  else if (n >= a.F) { r.side = 2; r.q = n - a.F; r.b = ldg(a.bh_F + r.q); r.c = ldg(a.ch_F + r.q); }
  return r;
}

// psi <- b psi + c diff / d (the reference's recursion, main.cu:829-861 and
// 1294-1318); stores and returns the new psi
template <typename T>
__device__ __forceinline__ T psi_apply(T* p, T old, T b, T c, T diff, T inv_d) {
  const T ps = rfma(b, old, rmul(rmul(c, diff), inv_d));
  *p = ps;
  return ps;
}


__device__ __forceinline__ void cp_async16(unsigned dst, const void* src, int src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src), "r"(src_bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// Tensor-copy staging (the alternative to the per-thread cp.async tasks):
// one thread of the CTA moves each plane's six component tiles with
// cp.async.bulk.tensor into the stage and the copies complete on that
// stage's mbarrier; every thread waits on the barrier's phase.  The tensor
// maps describe each component array as a {PX, NY, NZ} box; the halo
// family's tile is (32 + CH) x (TY + 1), the own family's 32 x TY, and
// rows or columns outside the arrays read as zero.  No multicast.
struct TmaMaps {
  CUtensorMap halo[3];
  CUtensorMap own[3];
  // test switch (FDTD_TMA_STALL_TEST=1): the issuing thread issues nothing,
  // so that every wait runs out and the timeout path is exercised
  int stall;
};

__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
}
// makes the initialised barriers visible to the tensor-copy unit
__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(unsigned bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(bar) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
  return t;
}
// Waits for the phase of the given parity to complete, for one second at
// most; false when it gave up.
__device__ __forceinline__ bool mbar_wait(unsigned bar, unsigned parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  for (;;) {
    if (mbar_try_wait(bar, parity)) return true;
    if (global_ns() - t0 > 1000000000ull) return false;
  }
}
__device__ __forceinline__ void tma_load_3d(unsigned dst, const CUtensorMap* map, int x, int y, int z, unsigned bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];\n" ::"r"(
          dst),
      "l"(map), "r"(x), "r"(y), "r"(z), "r"(bar)
      : "memory");
}

// Which tile a CTA of a pass owns: a box launch (grid = box of tiles,
// origin added) or a table launch (one (bx, by, bz) entry per CTA).  The
// passes are launched twice per half step: the interior box, whose tiles
// touch no CPML slab and use the PML-free instantiation, and the table of
// the remaining tiles.
struct TileMap {
  int ox, oy, oz;
  const int4* table;
};
__device__ __forceinline__ void tile_of(const TileMap& tm, int& bx, int& by, int& bz) {
  if (tm.table) {
    const int4 t = tm.table[blockIdx.x];
    bx = t.x; by = t.y; bz = t.z;
  } else {
    bx = tm.ox + (int)blockIdx.x; by = tm.oy + (int)blockIdx.y; bz = tm.oz + (int)blockIdx.z;
  }
}

// One stage of the ring: the three halo-family components ((TY + 1) rows of
// HW, each component block starting on a 128-byte boundary, which a tensor
// copy's destination needs), then the three own-family components (TY rows
// of 32).
template <typename T, int TY>
struct StageLayout {
  static constexpr int CH = 16 / (int)sizeof(T);   // elements per 16-byte chunk
  static constexpr int HW = 32 + CH;               // halo row width
  static constexpr int NCH_HALO = HW / CH;         // chunks per halo row
  static constexpr int NCH_OWN = 32 / CH;          // chunks per own row
  static constexpr int AL = 128 / (int)sizeof(T);  // elements per 128 bytes
  static constexpr int FH = ((TY + 1) * HW + AL - 1) / AL * AL;  // halo component stride
  static constexpr int HALO = 3 * FH;              // elements per stage
  static constexpr int OWN = 3 * TY * 32;
  static constexpr int STAGE = HALO + OWN;
  static constexpr int TASKS_HALO = 3 * (TY + 1) * NCH_HALO;
  static constexpr int TASKS_OWN = 3 * TY * NCH_OWN;
  static constexpr int TASKS = TASKS_HALO + TASKS_OWN;
  static constexpr int NTHR = 32 * TY;
  static constexpr int MAXT = (TASKS + NTHR - 1) / NTHR;  // copy tasks per thread
};

// The 16-byte copies one thread issues for every plane, resolved once: the
// shared-memory byte address inside stage 0, the source of the next plane
// to issue (advanced by one plane per issue) and whether the row and column
// lie inside the grid (zero fill otherwise).
template <typename T, int TY>
struct CopyTasks {
  using L = StageLayout<T, TY>;
  unsigned dst[L::MAXT];
  const T* src[L::MAXT];
  bool ok[L::MAXT];
  bool has[L::MAXT];

  __device__ __forceinline__ void init(unsigned sbase, const T* h0, const T* h1, const T* h2, const T* o0,
                                       const T* o1, const T* o2, int NX, int NY, int PX, size_t plane, int p0,
                                       int i0, int j0, int halo_row0, int halo_col0, bool per) {
    const int tid = threadIdx.y * 32 + threadIdx.x;
#pragma unroll
    for (int t = 0; t < L::MAXT; t++) {
      const int q = tid + t * L::NTHR;
      has[t] = q < L::TASKS;
      dst[t] = sbase;
      src[t] = h0;
      ok[t] = false;
      if (!has[t]) continue;
      int a, r, ch, gj, gi, d;
      const T* base;
      if (q < L::TASKS_HALO) {
        a = q / ((TY + 1) * L::NCH_HALO);
        const int rem = q - a * (TY + 1) * L::NCH_HALO;
        r = rem / L::NCH_HALO;
        ch = rem - r * L::NCH_HALO;
        gj = j0 + halo_row0 + r;
        gi = i0 + halo_col0 + ch * L::CH;
        d = a * L::FH + r * L::HW + ch * L::CH;
        base = a == 0 ? h0 : a == 1 ? h1 : h2;
        if (per) {
          // periodic x and y: the halo row -1 is row NY-1, row NY is row 0,
          // and the halo chunks left of column 0 or at column NX come from
          // the other side (NX is a multiple of the chunk width, so no chunk
          // straddles the seam)
          if (gj == -1) gj = NY - 1; else if (gj == NY) gj = 0;
          if (gi < 0) gi += NX; else if (gi >= NX && gi < NX + L::CH) gi -= NX;
        }
      } else {
        const int q2 = q - L::TASKS_HALO;
        a = q2 / (TY * L::NCH_OWN);
        const int rem = q2 - a * TY * L::NCH_OWN;
        r = rem / L::NCH_OWN;
        ch = rem - r * L::NCH_OWN;
        gj = j0 + r;
        gi = i0 + ch * L::CH;
        d = L::HALO + (a * TY + r) * 32 + ch * L::CH;
        base = a == 0 ? o0 : a == 1 ? o1 : o2;
      }
      dst[t] = sbase + (unsigned)(d * (int)sizeof(T));
      ok[t] = gj >= 0 && gj < NY && gi >= 0 && gi < PX;
      // plane p0 may be -1 (the E pass starts one plane below its chunk);
      // the pointer is only dereferenced for planes inside the grid
      if (ok[t]) src[t] = base + ((long long)p0 * (long long)plane + (long long)gj * PX + gi);
    }
  }

  // the next plane (number p; outside [0, NZ) zero-fills) into the stage
  // at byte offset soff
  __device__ __forceinline__ void issue(unsigned soff, int p, int NZ, const T* any, size_t plane) {
    const bool pz = (unsigned)p < (unsigned)NZ;
#pragma unroll
    for (int t = 0; t < L::MAXT; t++) {
      if (!has[t]) continue;
      const bool g = pz && ok[t];
      cp_async16(dst[t] + soff, g ? src[t] : any, g ? 16 : 0);
      src[t] += plane;
    }
  }
};

// The stage ring filled by tensor copies.  The S mbarriers (one per stage,
// arrival count 1) sit after the ring; a stage's barrier completes one
// phase per plane copied into it, so the parity a wait needs is the lowest
// bit of the stage's use count.  Only thread (0, 0) issues.  Planes beyond
// the last one the chunk reads are not copied, so every copy issued is
// waited for inside the plane loop; a plane outside [0, NZ) is not copied
// either (no value computed from it is stored) and its phase completes by
// a plain arrival.  A wait gives up after a second: the thread sets bit 2
// of the watchdog word and skips its later waits, the issuing thread stops
// issuing and, before the CTA ends, waits (again for a second at most) for
// the copies it has in flight.
template <typename T, int TY, int S>
struct TmaRing {
  using L = StageLayout<T, TY>;
  static constexpr unsigned SB = L::STAGE * sizeof(T);
  static constexpr unsigned HB = (TY + 1) * L::HW * sizeof(T);  // bytes of one halo tile
  static constexpr unsigned OB = TY * 32 * sizeof(T);           // bytes of one own tile
  unsigned sbase, bar0;
  int hx, hy, i0, j0;  // tile origins of the halo and own families
  int pfirst, plast;   // first and last plane of the chunk's ring
  int pdone;           // one past the last plane issued
  bool lead, bad;

  __device__ __forceinline__ void init(unsigned sbase_, int hx_, int hy_, int i0_, int j0_, int pfirst_,
                                       int plast_, int* flag) {
    sbase = sbase_;
    bar0 = sbase + S * SB;
    hx = hx_; hy = hy_; i0 = i0_; j0 = j0_;
    pfirst = pdone = pfirst_;
    plast = plast_;
    lead = threadIdx.x == 0 && threadIdx.y == 0;
    bad = false;
    if (lead) {
#pragma unroll
      for (int q = 0; q < S; q++) mbar_init(bar0 + 8 * q, 1);
      mbar_fence_init();
      // the tile destinations need 128-byte alignment
      if (sbase & 127) {
        bad = true;
        atomicOr(flag, 2);
      }
    }
    __syncthreads();
  }
  __device__ __forceinline__ void issue(const TmaMaps& m, int st, int p, int NZ) {
    if (!lead || bad || p > plast || m.stall) return;
    const unsigned bar = bar0 + 8 * st, stage = sbase + st * SB;
    pdone = p + 1;
    if ((unsigned)p >= (unsigned)NZ) {
      mbar_arrive(bar);
      return;
    }
    mbar_expect_tx(bar, 3 * (HB + OB));
#pragma unroll
    for (int a = 0; a < 3; a++) tma_load_3d(stage + a * L::FH * sizeof(T), &m.halo[a], hx, hy, p, bar);
#pragma unroll
    for (int a = 0; a < 3; a++)
      tma_load_3d(stage + (L::HALO + a * TY * 32) * sizeof(T), &m.own[a], i0, j0, p, bar);
  }
  __device__ __forceinline__ void wait(int st, int use, int* flag) {
    if (bad) return;
    if (!mbar_wait(bar0 + 8 * st, (unsigned)use & 1u)) {
      bad = true;
      atomicOr(flag, 2);
    }
  }
  __device__ __forceinline__ void drain() {
    if (!lead || !bad) return;
#pragma unroll
    for (int st = 0; st < S; st++) {
      const int n = pdone > pfirst + st ? (pdone - pfirst - st + S - 1) / S : 0;  // planes issued into st
      if (n > 0) mbar_wait(bar0 + 8 * st, (unsigned)(n - 1) & 1u);
    }
  }
};

// ---------------------------------------------------------------------
// H pass (UPDATE_hx/hy/hz, main.cu:762-1044).
// Needs E at k and k+1 (halo family) and H at k (own family).  hx is
// updated where j < NY-1 and k < NZ-1, hy where i < NX-1 and k < NZ-1, hz
// where i < NX-1 and j < NY-1; the CPML terms apply where all three indices
// are below N-1 (main.cu:829), per axis in the order z, x, y (hx: z then y;
// hy: z then x; hz: x then y).  The stage ring is counted from the chunk's
// first plane and the plane loop is unrolled by S, so every stage offset is
// a compile-time constant.
template <typename T, int TY, int S, bool PML, bool TMA = false>
__device__ __forceinline__ void h_pass_tile(const SimView<T>& s, int kchunk, int bx, int by, int bz,
                                            const TmaMaps* maps = nullptr) {
  using L = StageLayout<T, TY>;
  constexpr unsigned SB = L::STAGE * sizeof(T);  // stage bytes
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const T* sm = reinterpret_cast<const T*>(smem_raw);
  const unsigned sbase = (unsigned)__cvta_generic_to_shared(smem_raw);
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int i0 = bx * 32, j0 = by * TY;
  const int i = i0 + tx, j = j0 + ty;
  const int NX = s.NX, NY = s.NY, NZ = s.NZ, PX = s.PX;
  const size_t plane = s.plane;
  const int k0 = bz * kchunk;
  const int k1 = min(NZ, k0 + kchunk);
  const T* any = s.E[0];
  CopyTasks<T, TY> tasks;
  TmaRing<T, TY, S> ring;
  int pnext = k0;
  if constexpr (TMA) {
    ring.init(sbase, i0, j0, i0, j0, k0, k1, s.nonfinite);  // planes k0 .. k1
#pragma unroll
    for (int q = 0; q < S - 1; q++) ring.issue(*maps, q, pnext++, NZ);
  } else {
    tasks.init(sbase, s.E[0], s.E[1], s.E[2], s.H[0], s.H[1], s.H[2], NX, NY, PX, plane, k0, i0, j0, 0, 0,
               s.periodic != 0);
#pragma unroll
    for (int q = 0; q < S - 1; q++) {  // prologue: planes k0 .. k0+S-2 into stages 0 .. S-2
      tasks.issue(q * SB, pnext++, NZ, any, plane);
      cp_async_commit();
    }
  }
  const bool live = i < NX && j < NY;
  // periodic x and y: every column has its +x and +y neighbour
  const bool per = s.periodic != 0;
  const bool hasx = per || i + 1 < NX, hasy = per || j + 1 < NY;
  const T ikx = live ? ldg(s.cp[0].inv_khd + i) : T(0);
  const T iky = live ? ldg(s.cp[1].inv_khd + j) : T(0);
  const T* __restrict__ ikzp = s.cp[2].inv_khd + k0;
  const T che = s.che, chh = s.chh;
  const size_t id0 = fidx(PX, plane, i, j, k0);
  T* __restrict__ phx = s.H[0] + id0;
  T* __restrict__ phy = s.H[1] + id0;
  T* __restrict__ phz = s.H[2] + id0;
  const int o = ty * L::HW + tx, oo = ty * 32 + tx;
  constexpr int FH = L::FH;  // one halo component
  // CPML of this column: x and y slabs are fixed, z slabs follow the plane
  const bool pml_xy = PML && live && hasx && hasy;  // i < NX-1 and j < NY-1 (any column when periodic)
  SlabAt<T> sx, sy;
  sx.side = sy.side = 0; sx.q = sy.q = 0; sx.b = sx.c = sy.b = sy.c = T(0);
  if (pml_xy) { sx = slab_h(s.cp[0], i); sy = slab_h(s.cp[1], j); }
  const T idx_ = s.cp[0].inv_d, idy_ = s.cp[1].inv_d, idz_ = s.cp[2].inv_d;
  const int Ncz = s.cp[2].Nc, Fz = s.cp[2].F;
  // psi offsets in 32 bits; near and far slabs are contiguous (near first)
  const unsigned xstep = (unsigned)NY * (unsigned)s.cp[0].Nc, ystep = (unsigned)s.cp[1].Nc * (unsigned)PX;
  const unsigned plane32 = (unsigned)plane, jrow = (unsigned)j * (unsigned)PX + (unsigned)i;
  T* bx0 = nullptr;  // psi_hy(x) at plane 0
  T* bx1 = nullptr;  // psi_hz(x)
  T* by0 = nullptr;  // psi_hx(y)
  T* by1 = nullptr;  // psi_hz(y)
  if (sx.side) {
    const size_t q = (size_t)j * s.cp[0].Nc + sx.q;
    bx0 = (sx.side == 1 ? s.psiH_N[1][1] : s.psiH_F[1][1]) + q;
    bx1 = (sx.side == 1 ? s.psiH_N[2][0] : s.psiH_F[2][0]) + q;
  }
  if (sy.side) {
    const size_t q = (size_t)sy.q * PX + i;
    by0 = (sy.side == 1 ? s.psiH_N[0][0] : s.psiH_F[0][0]) + q;
    by1 = (sy.side == 1 ? s.psiH_N[2][1] : s.psiH_F[2][1]) + q;
  }
  T* const pz0 = s.psiH_N[0][1];  // psi_hx(z)
  T* const pz1 = s.psiH_N[1][0];  // psi_hy(z)
  // z-slab plane of the psi arrays (near 0..Nc-1, far Nc..) and of the
  // bh/ch tables (near 0..Nc-1, far Nc+1..: the tables hold Nc+1 entries a
  // side); -1 outside the slabs
  auto zq = [&](int kk) -> int { return kk < Ncz ? kk : (kk >= Fz ? kk - Fz + Ncz : -1); };
  unsigned ox = (unsigned)k0 * xstep, oy = (unsigned)k0 * ystep;  // x/y psi offsets of plane k
  // psi of the next plane, prefetched one plane ahead
  T nz0 = 0, nz1 = 0, nx0 = 0, nx1 = 0, ny0 = 0, ny1 = 0;
  auto fetch = [&](int kk, unsigned oxk, unsigned oyk) {
    if (!pml_xy || kk >= NZ - 1) return;
    const int q = zq(kk);
    if (q >= 0) {
      const unsigned off = (unsigned)q * plane32 + jrow;
      nz0 = pz0[off];
      nz1 = pz1[off];
    }
    if (sx.side) { nx0 = bx0[oxk]; nx1 = bx1[oxk]; }
    if (sy.side) { ny0 = by0[oyk]; ny1 = by1[oyk]; }
  };
  fetch(k0, ox, oy);
  // Ex, Ey of plane k+1 read in one plane are plane k's in the next (kept
  // in registers), and 1/(kappa dz) of the next plane is loaded ahead
  T cex = T(0), cey = T(0);
  bool carry = false;
  T ikz_next = ldg(ikzp);
  int use = 0;  // ring passes completed (the use count of stage u)
  for (int k = k0; k < k1; use++) {
#pragma unroll
    for (int u = 0; u < S; u++) {
      if (k < k1) {
        const T cz0 = nz0, cz1 = nz1, cx0 = nx0, cx1 = nx1, cy0 = ny0, cy1 = ny1;
        if (k + 1 < k1) fetch(k + 1, ox + xstep, oy + ystep);
        const T ikz = ikz_next;
        if (k + 1 < k1) ikz_next = ldg(ikzp + 1);
        // planes k and k+1 (stages u and u+1) have landed; then stage
        // (u+S-1)%S, which held plane k-1 (last read in the previous
        // iteration), takes plane k+S-1
        if constexpr (TMA) {
          ring.wait(u, use, s.nonfinite);
          ring.wait((u + 1) % S, u + 1 < S ? use : use + 1, s.nonfinite);
          __syncthreads();
          ring.issue(*maps, (u + S - 1) % S, pnext++, NZ);
        } else {
          cp_async_wait<S - 3>();
          __syncthreads();
          tasks.issue(((u + S - 1) % S) * SB, pnext++, NZ, any, plane);
          cp_async_commit();
        }
        if (live) {
          const T* eh = sm + u * L::STAGE;
          const T* en = sm + ((u + 1) % S) * L::STAGE;
          const T* hown = eh + L::HALO;
          const T exk = carry ? cex : eh[o], eyk = carry ? cey : eh[FH + o], ezk = eh[2 * FH + o];
          const T ex_j = eh[o + L::HW], ez_j = eh[2 * FH + o + L::HW];
          const T ey_i = eh[FH + o + 1], ez_i = eh[2 * FH + o + 1];
          const T exk1 = en[o], eyk1 = en[FH + o];
          cex = exk1;
          cey = eyk1;
          carry = true;
          const bool hask = k + 1 < NZ;
          T vx = rfma(che, rcurl(rsub(eyk1, eyk), ikz, rsub(ez_j, ezk), iky), rmul(chh, hown[oo]));
          T vy = rfma(che, rcurl(rsub(ez_i, ezk), ikx, rsub(exk1, exk), ikz), rmul(chh, hown[TY * 32 + oo]));
          T vz = rfma(che, rcurl(rsub(ex_j, exk), iky, rsub(ey_i, eyk), ikx), rmul(chh, hown[2 * TY * 32 + oo]));
          if (pml_xy && hask) {
            const int q = zq(k);
            if (q >= 0) {
              const unsigned off = (unsigned)q * plane32 + jrow;
              const int qt = q < Ncz ? q : q + 1;  // table index (Nc+1 entries a side)
              const T b = ldg(s.cp[2].bh_N + qt);
              const T c = ldg(s.cp[2].ch_N + qt);
              vx = rfma(che, psi_apply(pz0 + off, cz0, b, c, rsub(eyk1, eyk), idz_), vx);
              vy = rfma(-che, psi_apply(pz1 + off, cz1, b, c, rsub(exk1, exk), idz_), vy);
            }
            if (sx.side) {
              vy = rfma(che, psi_apply(bx0 + ox, cx0, sx.b, sx.c, rsub(ez_i, ezk), idx_), vy);
              vz = rfma(-che, psi_apply(bx1 + ox, cx1, sx.b, sx.c, rsub(ey_i, eyk), idx_), vz);
            }
            if (sy.side) {
              vx = rfma(-che, psi_apply(by0 + oy, cy0, sy.b, sy.c, rsub(ez_j, ezk), idy_), vx);
              vz = rfma(che, psi_apply(by1 + oy, cy1, sy.b, sy.c, rsub(ex_j, exk), idy_), vz);
            }
          }
          if (hasy && hask) *phx = vx;
          if (hasx && hask) *phy = vy;
          if (hasx && hasy) *phz = vz;
        }
        phx += plane; phy += plane; phz += plane; ikzp++;
        if (PML) { ox += xstep; oy += ystep; }
        k++;
      }
    }
  }
  if constexpr (TMA) ring.drain();
  else cp_async_wait<0>();
}
// Programmatic dependent launch of the two launches of a pass on one
// stream (the CPML edge tiles, then the interior box): the first lets the
// second start its CTAs as soon as all of its own are running, so the
// second fills the first's tail, and the second waits, after its own work,
// for the first to finish, so that its completion implies both.  The two
// launches touch disjoint cells and read only the other field.  The first
// may itself carry a programmatic dependency on the kernels before it on
// the stream (the 1D line before the H pass, the dispersive kernels before
// the E pass), which touch none of the pass's cells.

template <typename T, int TY, int S, int MINB, bool PML>
__global__ void __launch_bounds__(32 * TY, MINB) h_pass_s(const __grid_constant__ SimView<T> s, int kchunk,
                                                      const __grid_constant__ TileMap tm) {
  pdl_launch_dependents();
  int bx, by, bz;
  tile_of(tm, bx, by, bz);
  h_pass_tile<T, TY, S, PML>(s, kchunk, bx, by, bz);
  pdl_wait();
}
// The same with tensor-copy staging.
template <typename T, int TY, int S, int MINB, bool PML>
__global__ void __launch_bounds__(32 * TY, MINB) h_pass_t(const __grid_constant__ SimView<T> s, int kchunk,
                                                      const __grid_constant__ TileMap tm,
                                                      const __grid_constant__ TmaMaps maps) {
  pdl_launch_dependents();
  int bx, by, bz;
  tile_of(tm, bx, by, bz);
  h_pass_tile<T, TY, S, PML, true>(s, kchunk, bx, by, bz, &maps);
  pdl_wait();
}

// Batched form: a persistent grid that takes (simulation, tile) work items
// from a queue shared by every simulation of a batch; the views live in
// device memory, one per simulation, and every item carries the z-chunk of
// its simulation's size bucket.
template <typename T, int TY, int S, int MINB, bool PML>
__global__ void __launch_bounds__(32 * TY, MINB) h_pass_batch(const SimView<T>* __restrict__ views,
                                                           const int4* __restrict__ items, int nitems,
                                                           int* __restrict__ queue) {
  __shared__ int next;
  pdl_launch_dependents();  // the second launch of the pass may fill this one's tail
  for (;;) {
    __syncthreads();  // the previous item is finished with the stage ring and with next
    if (threadIdx.x == 0 && threadIdx.y == 0) next = atomicAdd(queue, 1);
    __syncthreads();
    const int it = next;
    if (it >= nitems) {
      pdl_wait();
      return;
    }
    const int4 w = items[it];  // (simulation | z-chunk << 20, bx, by, bz)
    h_pass_tile<T, TY, S, PML>(views[w.x & 0xFFFFF], w.x >> 20, w.y, w.z, w.w);
  }
}

// ---------------------------------------------------------------------
// E pass (UPDATE_ex/ey/ez, main.cu:1048-1912).
// Needs H at k and k-1 (halo family, one row/column of -1 halo) and E at k
// (own family).  Dispersive components are skipped (the dispersive-cell
// kernels update them, CPML included); dielectric classes select their
// coefficients.  CPML per axis in the order z, y, x (ex: z then y; ey: z
// then x; ez: y then x).  The stage ring is counted from plane k0-1.
template <typename T, int TY, int S, bool PML, bool TMA = false>
__device__ __forceinline__ void e_pass_tile(const SimView<T>& s, int kchunk, int bx, int by, int bz,
                                            const TmaMaps* maps = nullptr) {
  using L = StageLayout<T, TY>;
  constexpr unsigned SB = L::STAGE * sizeof(T);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const T* sm = reinterpret_cast<const T*>(smem_raw);
  const unsigned sbase = (unsigned)__cvta_generic_to_shared(smem_raw);
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int i0 = bx * 32, j0 = by * TY;
  const int i = i0 + tx, j = j0 + ty;
  const int NX = s.NX, NY = s.NY, NZ = s.NZ, PX = s.PX;
  const size_t plane = s.plane;
  const int k0 = bz * kchunk;
  const int k1 = min(NZ, k0 + kchunk);
  const T* any = s.H[0];
  CopyTasks<T, TY> tasks;
  TmaRing<T, TY, S> ring;
  int pnext = k0 - 1;
  if constexpr (TMA) {
    ring.init(sbase, i0 - L::CH, j0 - 1, i0, j0, k0 - 1, k1 - 1, s.nonfinite);  // planes k0-1 .. k1-1
#pragma unroll
    for (int q = 0; q < S - 1; q++) ring.issue(*maps, q, pnext++, NZ);
  } else {
    tasks.init(sbase, s.H[0], s.H[1], s.H[2], s.E[0], s.E[1], s.E[2], NX, NY, PX, plane, k0 - 1, i0, j0, -1,
               -L::CH, s.periodic != 0);
#pragma unroll
    for (int q = 0; q < S - 1; q++) {  // prologue: planes k0-1 .. k0+S-3 into stages 0 .. S-2
      tasks.issue(q * SB, pnext++, NZ, any, plane);
      cp_async_commit();
    }
  }
  const bool live = i < NX && j < NY;
  // active-range masks of ex, ey, ez in this column (main.cu:1172, 1476, 1767)
  // (periodic x and y: every column, main.cu:1072, 1364, 1668)
  const bool per = s.periodic != 0;
  const bool okx = i < NX - 1, oky = j < NY - 1;
  const bool colx = live && (per || (okx && j > 0 && oky));
  const bool coly = live && (per || (i > 0 && okx && oky));
  const bool colz = live && (per || (i > 0 && okx && j > 0 && oky));
  const T ikx = live ? ldg(s.cp[0].inv_ked + i) : T(0);
  const T iky = live ? ldg(s.cp[1].inv_ked + j) : T(0);
  const T* __restrict__ ikzp = s.cp[2].inv_ked + k0;
  const int mlo_z = s.mat_lo[2], mhi_z = s.mat_hi[2];
  const bool inbox_xy = i >= s.mat_lo[0] && i < s.mat_hi[0] && j >= s.mat_lo[1] && j < s.mat_hi[1];
  const T cee0 = s.cee[0], ceh0 = s.ceh[0];
  const size_t id0 = fidx(PX, plane, i, j, k0);
  T* __restrict__ pex = s.E[0] + id0;
  T* __restrict__ pey = s.E[1] + id0;
  T* __restrict__ pez = s.E[2] + id0;
  const int o = (ty + 1) * L::HW + tx + L::CH, oo = ty * 32 + tx;
  constexpr int FH = L::FH;
  // CPML of this column: x and y slabs are fixed, z slabs follow the plane
  const bool pml_xy = PML && live && (per || (okx && oky));  // i < NX-1 and j < NY-1 (any column when periodic)
  SlabAt<T> sx, sy;
  sx.side = sy.side = 0; sx.q = sy.q = 0; sx.b = sx.c = sy.b = sy.c = T(0);
  T cx_ey = T(0);
  if (pml_xy) {
    sy = slab_e(s.cp[1], j, s.cp[1].ce_N);
    sx = slab_e(s.cp[0], i, s.cp[0].ce_N);
    // Ey's near-x slab takes ce_y_N in the reference (main.cu:2891)
    cx_ey = sx.side == 1 ? ldg(s.cp[0].ce_N_ey + sx.q) : sx.c;
  }
  const T idx_ = s.cp[0].inv_d, idy_ = s.cp[1].inv_d, idz_ = s.cp[2].inv_d;
  const int Ncz = s.cp[2].Nc, Fz = s.cp[2].F;
  // psi offsets in 32 bits; near and far slabs are contiguous (near first)
  const unsigned xstep = (unsigned)NY * (unsigned)(s.cp[0].Nc + 1), ystep = (unsigned)(s.cp[1].Nc + 1) * (unsigned)PX;
  const unsigned plane32 = (unsigned)plane, jrow = (unsigned)j * (unsigned)PX + (unsigned)i;
  T* bx0 = nullptr;  // psi_ey(x) at plane 0
  T* bx1 = nullptr;  // psi_ez(x)
  T* by0 = nullptr;  // psi_ex(y)
  T* by1 = nullptr;  // psi_ez(y)
  if (sx.side) {
    const size_t q = (size_t)j * (s.cp[0].Nc + 1) + sx.q;
    bx0 = (sx.side == 1 ? s.psiE_N[1][1] : s.psiE_F[1][1]) + q;
    bx1 = (sx.side == 1 ? s.psiE_N[2][0] : s.psiE_F[2][0]) + q;
  }
  if (sy.side) {
    const size_t q = (size_t)sy.q * PX + i;
    by0 = (sy.side == 1 ? s.psiE_N[0][0] : s.psiE_F[0][0]) + q;
    by1 = (sy.side == 1 ? s.psiE_N[2][1] : s.psiE_F[2][1]) + q;
  }
  T* const pz0 = s.psiE_N[0][1];  // psi_ex(z)
  T* const pz1 = s.psiE_N[1][0];  // psi_ey(z)
  // z-slab index of a plane (near 0..Nc, far Nc+1..), -1 outside: indexes
  // the psi planes and the be/ce tables alike
  auto zq = [&](int kk) -> int { return kk <= Ncz ? kk : (kk >= Fz ? kk - Fz + Ncz + 1 : -1); };
  unsigned ox = (unsigned)k0 * xstep, oy = (unsigned)k0 * ystep;  // x/y psi offsets of plane k
  T nz0 = 0, nz1 = 0, nx0 = 0, nx1 = 0, ny0 = 0, ny1 = 0;
  auto fetch = [&](int kk, unsigned oxk, unsigned oyk) {
    if (!pml_xy || kk >= NZ - 1) return;
    const int q = zq(kk);
    if (q >= 0) {
      const unsigned off = (unsigned)q * plane32 + jrow;
      nz0 = pz0[off];
      nz1 = pz1[off];
    }
    if (sx.side) { nx0 = bx0[oxk]; nx1 = bx1[oxk]; }
    if (sy.side) { ny0 = by0[oyk]; ny1 = by1[oyk]; }
  };
  fetch(k0, ox, oy);
  T check = T(0);
  // Hx, Hy of plane k are plane k-1's in the next plane (kept in
  // registers), and 1/(kappa dz) of the next plane is loaded ahead
  T chx = T(0), chy = T(0);
  bool carry = false;
  T ikz_next = ldg(ikzp);
  int use = 0;  // ring passes completed (the use count of stage u)
  for (int k = k0; k < k1; use++) {
#pragma unroll
    for (int u = 0; u < S; u++) {
      if (k < k1) {
        const T cz0 = nz0, cz1 = nz1, cx0 = nx0, cx1 = nx1, cy0 = ny0, cy1 = ny1;
        if (k + 1 < k1) fetch(k + 1, ox + xstep, oy + ystep);
        const T ikz = ikz_next;
        if (k + 1 < k1) ikz_next = ldg(ikzp + 1);
        // planes k-1 and k (stages u and u+1) have landed; then stage
        // (u+S-1)%S, which held plane k-2 (last read in the previous
        // iteration), takes plane k+S-2
        if constexpr (TMA) {
          ring.wait(u, use, s.nonfinite);
          ring.wait((u + 1) % S, u + 1 < S ? use : use + 1, s.nonfinite);
          __syncthreads();
          ring.issue(*maps, (u + S - 1) % S, pnext++, NZ);
        } else {
          cp_async_wait<S - 3>();
          __syncthreads();
          tasks.issue(((u + S - 1) % S) * SB, pnext++, NZ, any, plane);
          cp_async_commit();
        }
        if (live) {
          const T* cur = sm + ((u + 1) % S) * L::STAGE;
          const T* prv = sm + u * L::STAGE;
          const T hxk = cur[o], hyk = cur[FH + o], hzk = cur[2 * FH + o];
          const T hx_j = cur[o - L::HW], hz_j = cur[2 * FH + o - L::HW];
          const T hy_i = cur[FH + o - 1], hz_i = cur[2 * FH + o - 1];
          const T hxm = carry ? chx : prv[o], hym = carry ? chy : prv[FH + o];
          chx = hxk;
          chy = hyk;
          carry = true;
          const T* eown = cur + L::HALO;
          const bool okz = k < NZ - 1, hasz = k > 0;
          unsigned m = 0;
          T cee = cee0, ceh = ceh0;
          if (inbox_xy && k >= mlo_z && k < mhi_z) {
            m = s.mat[id0 + (size_t)(k - k0) * plane];
            if (m >> 3) {
              cee = s.cee[m >> 3];
              ceh = s.ceh[m >> 3];
            }
          }
          T vx = rfma(ceh, rcurl(rsub(hzk, hz_j), iky, rsub(hyk, hym), ikz), rmul(cee, eown[oo]));
          T vy = rfma(ceh, rcurl(rsub(hxk, hxm), ikz, rsub(hzk, hz_i), ikx), rmul(cee, eown[TY * 32 + oo]));
          T vz = rfma(ceh, rcurl(rsub(hyk, hy_i), ikx, rsub(hxk, hx_j), iky), rmul(cee, eown[2 * TY * 32 + oo]));
          const bool wx = colx && hasz && okz && !(m & 1);
          const bool wy = coly && hasz && okz && !(m & 2);
          const bool wz = colz && okz && !(m & 4);
          if (pml_xy && okz) {
            const int q = zq(k);
            if (q >= 0) {
              const unsigned off = (unsigned)q * plane32 + jrow;
              const T b = ldg(s.cp[2].be_N + q);  // be_N then be_F
              const T c = ldg(s.cp[2].ce_N + q);  // ce_N then ce_F
              if (wx) vx = rfma(-ceh, psi_apply(pz0 + off, cz0, b, c, rsub(hyk, hym), idz_), vx);
              if (wy) vy = rfma(ceh, psi_apply(pz1 + off, cz1, b, c, rsub(hxk, hxm), idz_), vy);
            }
            if (sy.side) {
              if (wx) vx = rfma(ceh, psi_apply(by0 + oy, cy0, sy.b, sy.c, rsub(hzk, hz_j), idy_), vx);
              if (wz) vz = rfma(-ceh, psi_apply(by1 + oy, cy1, sy.b, sy.c, rsub(hxk, hx_j), idy_), vz);
            }
            if (sx.side) {
              if (wy) vy = rfma(-ceh, psi_apply(bx0 + ox, cx0, sx.b, cx_ey, rsub(hzk, hz_i), idx_), vy);
              if (wz) vz = rfma(ceh, psi_apply(bx1 + ox, cx1, sx.b, sx.c, rsub(hyk, hy_i), idx_), vz);
            }
          }
          if (wx) { *pex = vx; check += vx; }
          if (wy) { *pey = vy; check += vy; }
          if (wz) { *pez = vz; check += vz; }
        }
        pex += plane; pey += plane; pez += plane; ikzp++;
        if (PML) { ox += xstep; oy += ystep; }
        k++;
      }
    }
  }
  if constexpr (TMA) ring.drain();
  else cp_async_wait<0>();
  // NaN/Inf watchdog: a non-finite value makes the running sum non-finite
  if (!isfinite(check)) atomicOr(s.nonfinite, 1);
}
template <typename T, int TY, int S, int MINB, bool PML>
__global__ void __launch_bounds__(32 * TY, MINB) e_pass_s(const __grid_constant__ SimView<T> s, int kchunk,
                                                      const __grid_constant__ TileMap tm) {
  pdl_launch_dependents();
  int bx, by, bz;
  tile_of(tm, bx, by, bz);
  e_pass_tile<T, TY, S, PML>(s, kchunk, bx, by, bz);
  pdl_wait();
}
template <typename T, int TY, int S, int MINB, bool PML>
__global__ void __launch_bounds__(32 * TY, MINB) e_pass_t(const __grid_constant__ SimView<T> s, int kchunk,
                                                      const __grid_constant__ TileMap tm,
                                                      const __grid_constant__ TmaMaps maps) {
  pdl_launch_dependents();
  int bx, by, bz;
  tile_of(tm, bx, by, bz);
  e_pass_tile<T, TY, S, PML, true>(s, kchunk, bx, by, bz, &maps);
  pdl_wait();
}

// Batched form: a persistent grid that takes (simulation, tile) work items
// from a queue shared by every simulation of a batch; the views live in
// device memory, one per simulation, and every item carries the z-chunk of
// its simulation's size bucket.
template <typename T, int TY, int S, int MINB, bool PML>
__global__ void __launch_bounds__(32 * TY, MINB) e_pass_batch(const SimView<T>* __restrict__ views,
                                                           const int4* __restrict__ items, int nitems,
                                                           int* __restrict__ queue) {
  __shared__ int next;
  pdl_launch_dependents();  // the second launch of the pass may fill this one's tail
  for (;;) {
    __syncthreads();  // the previous item is finished with the stage ring and with next
    if (threadIdx.x == 0 && threadIdx.y == 0) next = atomicAdd(queue, 1);
    __syncthreads();
    const int it = next;
    if (it >= nitems) {
      pdl_wait();
      return;
    }
    const int4 w = items[it];  // (simulation | z-chunk << 20, bx, by, bz)
    e_pass_tile<T, TY, S, PML>(views[w.x & 0xFFFFF], w.x >> 20, w.y, w.z, w.w);
  }
}

}  // namespace fdtd
