// C ABI of the B200-native FDTD time step: simulation handle, device state,
// launch sequencing (direct and CUDA-graph replay), spectra, snapshots.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/fdtd_b200.h"
#include "kernels.cuh"
#include "staged.cuh"
#include "boundary.cuh"
#include "adjoint.cuh"
#include "snapshot.cuh"
#include "setup.h"

using namespace fdtd;

static thread_local std::string g_err;

static fdtd_status fail(fdtd_status st, const std::string& msg) {
  g_err = msg;
  return st;
}

#define CUDA_TRY(expr)                                                                          \
  do {                                                                                          \
    cudaError_t e_ = (expr);                                                                    \
    if (e_ != cudaSuccess)                                                                      \
      return fail(FDTD_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_));          \
  } while (0)

namespace {

// A device allocation that frees itself.
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
  cudaError_t alloc(size_t n) {
    bytes = n;
    cudaError_t e = cudaMalloc(&p, n ? n : 16);
    if (e == cudaSuccess) e = cudaMemset(p, 0, n ? n : 16);
    return e;
  }
  template <typename U>
  U* as() const { return static_cast<U*>(p); }
};

}  // namespace

struct fdtd_sim {
  Setup su;
  int device = 0;
  bool fp64 = true;
  int NX, NY, NZ, PX;
  size_t plane, ncell;
  int kchunk = 32;
  // launch shape of the E and H passes, chosen by tune_passes()
  // staged = shared-memory pipelined kernels (minb unused), else the plain
  // register z-march
  // launch shape of one pass: tile height and z-chunk shared by its two
  // launches, register cap (min CTAs/SM) and ring depth per launch
  // (interior tiles: minb/stages, CPML edge tiles: eminb/estages)
  // pdl = 1: the edge and interior launches of a pass go on one stream
  // with a programmatic dependency instead of on two streams
  struct PassCfg { int minb = 1, ty = 4, kchunk = 16, staged = 1, stages = 4, eminb = 1, estages = 4, pdl = 0, tma = 0, etma = 0; float ms = 0; };
  // pass tiles for one (tile height, z-chunk): the interior box of tiles
  // that touch no CPML slab and the table of the others
  struct TileSet {
    int ty = 0, kchunk = 0;
    dim3 inner;
    TileMap inner_map{0, 0, 0, nullptr}, edge_map{0, 0, 0, nullptr};
    unsigned nedge = 0;
  };
  std::vector<TileSet> tilesets;
  // tensor maps of the field arrays for the tensor-copy staging of the
  // passes, one set per tile height (0 = the encoder is not available)
  struct TmaSet {
    int ty = 0;
    TmaMaps h, e;  // H pass: halo E, own H; E pass: halo H, own E
  };
  std::vector<TmaSet> tmasets;
  int tma_avail = -1;  // -1 not yet known
  ShellCells shell_h, shell_e;
  TfsfTable tf_h{}, tf_e{};  // tabulated TFSF corrections of the two shells
  const void* dview = nullptr;  // device copy of the view
  PassCfg hcfg, ecfg;
  bool tuned = false;
  // device state
  std::vector<std::unique_ptr<DevBuf>> bufs;
  void* E[3];
  void* H[3];
  uint8_t* mat = nullptr;
  int mat_lo[3], mat_hi[3];
  DevClock* clk = nullptr;
  double* e_inc = nullptr;
  double* h_inc = nullptr;
  double* pulse = nullptr;
  double* probe = nullptr;
  int probe_cap = 0;
  size_t probe_id = 0;
  void* tables = nullptr;  // CPML tables of both precisions live here
  // dispersive cells
  int nmetal[3] = {0, 0, 0};
  int4* mcell[3] = {nullptr, nullptr, nullptr};
  int* nbr[3] = {nullptr, nullptr, nullptr};  // hydrodynamic neighbour slots
  // DFT
  DftView dft;
  void* ring = nullptr;
  double* flux = nullptr;  // [12][nf]
  double2* twiddles = nullptr;  // [2][kRingSlots][nf]
  bool dft_on = true;
  int host_nsamp = 0;  // DFT samples into the contraction period (0 .. kRingSlots - 1)
  // views (one of them is used, by precision)
  SimView<float> vf;
  SimView<double> vd;
  MetalView<float> mf;
  MetalView<double> md;
  LineArgs line;
  // host step counter
  int t = 0;
  // kernels enqueued by this handle (graph replays counted per node)
  long long kernels = 0, steps_done = 0, graph_launches = 0;
  // graph replays of the two launch periods of a DFT contraction period
  // (the first forks the contraction of the last period's samples);
  // graph_epoch counts the times captured graphs were dropped because the
  // step's launches changed
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  long long graph_kernels_p[2] = {0, 0};
  int graph_len = 0, graph_epoch = 0;
  // the DFT contraction beside the steps: its stream and fork/join events,
  // and whether a forked contraction still has to be joined
  cudaStream_t side_dft = nullptr;
  cudaEvent_t dft_fork_ev = nullptr, dft_join_ev = nullptr;
  bool dft_pending = false;
  cudaStream_t graph_stream = nullptr;
  bool use_graphs = true;

  // snapshots taken by the stepper (fdtd_snapshots_enable / _drain):
  // records [snap_first, produced) exist, [snap_drained, produced) wait
  SnapArgs snap{};
  bool snap_on = false;
  long long snap_first = 0, snap_drained = 0;

  // adjoint design region (fdtd_set_design / fdtd_forward / fdtd_backward)
  bool has_design = false;
  int dbox[6] = {0, 0, 0, 0, 0, 0};
  std::vector<int> dslot[3];     // design-box cell (x fastest) -> slot of component c, -1 none
  float* rho_d[3] = {nullptr, nullptr, nullptr};  // blend per slot of component c
  bool pml_metal = false;        // a dispersive cell lies in a CPML slab
  struct Adjoint;
  std::unique_ptr<Adjoint> adj;
  ~fdtd_sim();

  // side stream on which a pass's edge-tile launch runs beside its
  // interior launch (fork/join by events, also inside graph capture)
  cudaStream_t side = nullptr;
  cudaEvent_t fork_ev = nullptr, join_ev = nullptr;
  // second side stream: the dispersive-cell kernels beside the E pass and
  // the 1D line beside the H pass, when a pass's launches use two streams
  // (they touch nothing the pass touches)
  cudaStream_t side2 = nullptr;
  cudaEvent_t fork2_ev = nullptr, join2_ev = nullptr;
  cudaEvent_t fork3_ev = nullptr, join3_ev = nullptr;  // the line step beside the H pass

  void destroy_streams() {
    for (auto& g : graph)
      if (g) cudaGraphExecDestroy(g);
    if (side_dft) cudaStreamDestroy(side_dft);
    if (dft_fork_ev) cudaEventDestroy(dft_fork_ev);
    if (dft_join_ev) cudaEventDestroy(dft_join_ev);
    if (graph_stream) cudaStreamDestroy(graph_stream);
    if (side) cudaStreamDestroy(side);
    if (fork_ev) cudaEventDestroy(fork_ev);
    if (join_ev) cudaEventDestroy(join_ev);
    if (side2) cudaStreamDestroy(side2);
    if (fork2_ev) cudaEventDestroy(fork2_ev);
    if (join2_ev) cudaEventDestroy(join2_ev);
    if (fork3_ev) cudaEventDestroy(fork3_ev);
    if (join3_ev) cudaEventDestroy(join3_ev);
  }

  // buffers that fdtd_reset zeroes (fields, psi, dispersive state, DFT,
  // clock, incident line, probe); tables are not listed
  std::vector<std::pair<void*, size_t>> state;

  template <typename U>
  cudaError_t alloc(U** out, size_t count, bool is_state = false) {
    auto b = std::make_unique<DevBuf>();
    cudaError_t e = b->alloc(count * sizeof(U));
    if (e != cudaSuccess) return e;
    *out = b->as<U>();
    if (is_state) state.emplace_back(b->p, b->bytes);
    bufs.push_back(std::move(b));
    return cudaSuccess;
  }
};

// ---------------------------------------------------------------------
// parameters

extern "C" void fdtd_params_default(fdtd_params* p) { params_default(p); }

extern "C" size_t fdtd_params_size(void) { return sizeof(fdtd_params); }

extern "C" fdtd_status fdtd_load_input_txt(const char* path, fdtd_params* p) {
  if (!path || !p) return fail(FDTD_ERR_INVALID, "null argument");
  int rc = read_input_txt(path, p);
  if (rc == -1) return fail(FDTD_ERR_IO, std::string("cannot open ") + path);
  if (rc != 0) return fail(FDTD_ERR_IO, std::string("malformed Input.txt: ") + path);
  return FDTD_OK;
}

extern "C" fdtd_status fdtd_write_input_txt(const char* path, const fdtd_params* p) {
  if (!path || !p) return fail(FDTD_ERR_INVALID, "null argument");
  if (write_input_txt(path, p) != 0) return fail(FDTD_ERR_IO, std::string("cannot write ") + path);
  return FDTD_OK;
}

extern "C" const char* fdtd_last_error(void) { return g_err.c_str(); }

static void fill_dims(const Setup& su, fdtd_dims* d) {
  std::memset(d, 0, sizeof(*d));
  d->nx = su.NX; d->ny = su.NY; d->nz = su.NZ;
  d->ntfsf_x = su.Nt[0]; d->ntfsf_y = su.Nt[1]; d->ntfsf_z = su.Nt[2];
  d->inc_length = su.L; d->m0 = su.m0;
  for (int a = 0; a < 3; a++) {
    d->abs_start[a] = su.absS[a]; d->abs_end[a] = su.absE[a];
    d->sca_start[a] = su.scaS[a]; d->sca_end[a] = su.scaE[a];
  }
  d->num_freq = su.p.NUM_freq;
  const size_t n = (size_t)su.NX * su.NY * su.NZ;
  for (int c = 0; c < 3; c++) {
    int cnt = 0;
    for (size_t q = 0; q < n; q++) cnt += is_dispersive(su.matc[c][q]);
    d->n_metal_cells[c] = cnt;
  }
  d->hydro = su.hydro;
  d->precision = su.p.precision;
  d->dt = su.dt; d->delay = su.delay; d->width = su.width;
}

extern "C" fdtd_status fdtd_plan(const fdtd_params* p, fdtd_dims* out) {
  if (!p || !out) return fail(FDTD_ERR_INVALID, "null argument");
  Setup su;
  if (const char* msg = setup_build(*p, su)) return fail(FDTD_ERR_INVALID, msg);
  fill_dims(su, out);
  return FDTD_OK;
}

extern "C" fdtd_status fdtd_rasterise(const fdtd_params* p, uint8_t* bits, size_t count) {
  if (!p || !bits) return fail(FDTD_ERR_INVALID, "null argument");
  Setup su;
  if (const char* msg = setup_build(*p, su)) return fail(FDTD_ERR_INVALID, msg);
  const size_t n = (size_t)su.NX * su.NY * su.NZ;
  if (count != n) return fail(FDTD_ERR_INVALID, "count must be nx*ny*nz");
  for (size_t q = 0; q < n; q++) {
    uint8_t b = 0;
    for (int c = 0; c < 3; c++) b |= (uint8_t)(is_dispersive(su.matc[c][q]) << c);
    bits[q] = b;
  }
  return FDTD_OK;
}

extern "C" fdtd_status fdtd_coefficients(const fdtd_params* p, int which, double* out, size_t count,
                                         size_t* len) {
  if (!p || !out || !len) return fail(FDTD_ERR_INVALID, "null argument");
  Setup su;
  if (const char* msg = setup_build(*p, su)) return fail(FDTD_ERR_INVALID, msg);
  std::vector<double> v;
  if (which >= 0 && which < 6) {
    v = which < 3 ? su.cp[which].ked : su.cp[which - 3].khd;
  } else if (which >= 6 && which < 30) {
    const CpmlTables& t = su.cp[(which - 6) / 8];
    const std::vector<double>* tabs[8] = {&t.be_N, &t.ce_N, &t.be_F, &t.ce_F, &t.bh_N, &t.ch_N, &t.bh_F, &t.ch_F};
    v = *tabs[(which - 6) % 8];
  } else if (which == 100) {
    v = {su.C_E, su.C_E_1, su.C_E_2, su.d1, su.d2, su.d3, su.d4, su.d5, su.dNL,
         su.C1[0], su.C2[0], su.C3[0], su.C4[0], su.C5[0],
         su.C1[1], su.C2[1], su.C3[1], su.C4[1], su.C5[1], su.dt, su.N_EQ, 0.0};
  } else if (which == 101) {
    v = su.freq;
  } else if (which == 102) {
    v = su.pulse;
  } else {
    return fail(FDTD_ERR_INVALID, "unknown table");
  }
  *len = v.size();
  if (count < v.size()) return fail(FDTD_ERR_INVALID, "output buffer too small");
  std::memcpy(out, v.data(), v.size() * sizeof(double));
  return FDTD_OK;
}

// ---------------------------------------------------------------------
// create

template <typename T>
static fdtd_status upload(T* dst, const std::vector<double>& src) {
  std::vector<T> tmp(src.begin(), src.end());
  if (!tmp.empty()) CUDA_TRY(cudaMemcpy(dst, tmp.data(), tmp.size() * sizeof(T), cudaMemcpyHostToDevice));
  return FDTD_OK;
}

template <typename T>
static fdtd_status build_views(fdtd_sim* s) {
  const Setup& su = s->su;
  SimView<T>& v = *reinterpret_cast<SimView<T>*>(std::is_same<T, float>::value ? (void*)&s->vf : (void*)&s->vd);
  MetalView<T>& m = *reinterpret_cast<MetalView<T>*>(std::is_same<T, float>::value ? (void*)&s->mf : (void*)&s->md);
  std::memset(&v, 0, sizeof(v));
  std::memset(&m, 0, sizeof(m));
  v.NX = s->NX; v.NY = s->NY; v.NZ = s->NZ; v.PX = s->PX; v.plane = s->plane;
  for (int c = 0; c < 3; c++) { v.E[c] = (T*)s->E[c]; v.H[c] = (T*)s->H[c]; }
  v.mat = s->mat;
  for (int a = 0; a < 3; a++) { v.mat_lo[a] = s->mat_lo[a]; v.mat_hi[a] = s->mat_hi[a]; }
  for (int q = 0; q < kMaxClasses; q++) { v.cee[q] = (T)su.Cee; v.ceh[q] = (T)su.Ceh; }
  v.ceh[1] = (T)su.Ceh_slab;  // class 1: the dielectric slab (Cee = 1: no conductivity)
  v.chh = (T)su.Chh; v.che = (T)su.Che;
  const double dxyz[3] = {su.p.dx, su.p.dy, su.p.dz};
  const int N3[3] = {s->NX, s->NY, s->NZ};
  for (int a = 0; a < 3; a++) {
    const CpmlTables& t = su.cp[a];
    const int Nc = su.Nc[a];
    T* base;
    const size_t need = 8 * (size_t)(Nc + 1) + (size_t)(Nc + 1) + 2 * (size_t)N3[a];
    cudaError_t e = s->alloc(&base, need);
    if (e != cudaSuccess) return fail(FDTD_ERR_ALLOC, cudaGetErrorString(e));
    T* q = base;
    auto put = [&](const std::vector<double>& src, size_t len) -> T* {
      T* at = q;
      std::vector<double> pad(src);
      pad.resize(len, 0.0);
      upload<T>(at, pad);
      q += len;
      return at;
    };
    CpmlAxis<T>& ca = v.cp[a];
    // near then far, each Nc+1 entries, so that one index walks both slabs
    ca.be_N = put(t.be_N, Nc + 1); ca.be_F = put(t.be_F, Nc + 1);
    ca.ce_N = put(t.ce_N, Nc + 1); ca.ce_F = put(t.ce_F, Nc + 1);
    ca.bh_N = put(t.bh_N, Nc + 1); ca.bh_F = put(t.bh_F, Nc + 1);
    ca.ch_N = put(t.ch_N, Nc + 1); ca.ch_F = put(t.ch_F, Nc + 1);
    std::vector<double> ik(N3[a]), ih(N3[a]);
    for (int i = 0; i < N3[a]; i++) { ik[i] = 1.0 / t.ked[i]; ih[i] = 1.0 / t.khd[i]; }
    ca.inv_ked = put(ik, N3[a]);
    ca.inv_khd = put(ih, N3[a]);
    ca.inv_d = (T)(1.0 / dxyz[a]);
    ca.Nc = Nc;
    ca.F = su.F[a];
    v.dxyz[a] = (T)dxyz[a];
    // Ey's near-x slab reads ce_y_N in the reference (main.cu:2891)
    if (a == 0) {
      const std::vector<double>& src = (su.p.fixes & FDTD_FIX_CE_EY_XN) ? su.cp[0].ce_N : su.cp[1].ce_N;
      std::vector<double> pad(src);
      pad.resize(Nc + 1, 0.0);
      T* at = q;
      upload<T>(at, pad);
      q += Nc + 1;
      ca.ce_N_ey = at;
    }
  }
  v.cp[1].ce_N_ey = v.cp[1].ce_N;
  v.cp[2].ce_N_ey = v.cp[2].ce_N;
  // psi slabs
  for (int c = 0; c < 3; c++)
    for (int slot = 0; slot < 2; slot++) {
      const int ax = (c + 1 + slot) % 3;
      const int Nc = std::max(su.Nc[ax], 0);  // -1 along a periodic axis: no slab
      size_t cells_e, cells_h;
      if (ax == 2) { cells_e = (size_t)(Nc + 1) * s->plane; cells_h = (size_t)Nc * s->plane; }
      else if (ax == 1) { cells_e = (size_t)s->NZ * (Nc + 1) * s->PX; cells_h = (size_t)s->NZ * Nc * s->PX; }
      else { cells_e = (size_t)s->NZ * s->NY * (Nc + 1); cells_h = (size_t)s->NZ * s->NY * Nc; }
      // near slab then far slab in one allocation (the passes index both
      // from the near pointer)
      T *a1, *a3;
      cudaError_t e;
      if ((e = s->alloc(&a1, 2 * cells_e, true)) != cudaSuccess || (e = s->alloc(&a3, 2 * cells_h, true)) != cudaSuccess)
        return fail(FDTD_ERR_ALLOC, cudaGetErrorString(e));
      v.psiE_N[c][slot] = a1; v.psiE_F[c][slot] = a1 + cells_e;
      v.psiH_N[c][slot] = a3; v.psiH_F[c][slot] = a3 + cells_h;
    }
  // TFSF
  TfsfView& tf = v.tf;
  tf.on = 1;
  tf.Tx = su.Nt[0]; tf.Ty = su.Nt[1]; tf.Tz = su.Nt[2];
  tf.i0 = su.i0; tf.j0 = su.j0; tf.k0 = su.k0; tf.m0 = su.m0;
  tf.sth = su.sth; tf.cth = su.cth; tf.sph = su.sph; tf.cph = su.cph;
  for (int c = 0; c < 3; c++) { tf.fe[c] = su.fe[c]; tf.fh[c] = su.fh[c]; }
  tf.dscale = su.p.dx / su.d1D;
  tf.closed = su.p.periodic_xy ? 0 : 1;  // periodic: the lower z face only (main.cu:698)
  v.periodic = su.p.periodic_xy ? 1 : 0;
  v.h_inc = s->h_inc;
  v.nonfinite = &s->clk->nonfinite;
  // dispersive cells
  for (int c = 0; c < 3; c++) { m.n[c] = s->nmetal[c]; m.cell[c] = s->mcell[c]; }
  size_t maxn = std::max(s->nmetal[0], std::max(s->nmetal[1], s->nmetal[2]));
  if (maxn > 0) {
    // per component: en, en1 in T; cpn[2], cpn1[2], pd[3], nd[2] in FP64
    T* st;
    double* sd;
    cudaError_t e = s->alloc(&st, (size_t)3 * 2 * maxn, true);
    if (e == cudaSuccess) e = s->alloc(&sd, (size_t)3 * 9 * maxn, true);
    if (e != cudaSuccess) return fail(FDTD_ERR_ALLOC, cudaGetErrorString(e));
    for (int c = 0; c < 3; c++) {
      T* b = st + (size_t)c * 2 * maxn;
      double* d = sd + (size_t)c * 9 * maxn;
      m.en[c] = b; m.en1[c] = b + maxn;
      m.cpn[c][0] = d; m.cpn[c][1] = d + maxn;
      m.cpn1[c][0] = d + 2 * maxn; m.cpn1[c][1] = d + 3 * maxn;
      m.pd[c][0] = d + 4 * maxn; m.pd[c][1] = d + 5 * maxn; m.pd[c][2] = d + 6 * maxn;
      m.nd[c][0] = d + 7 * maxn; m.nd[c][1] = d + 8 * maxn;
      m.nbr[c] = s->nbr[c];
    }
  }
  m.C_E = su.C_E; m.C_E_1 = su.C_E_1; m.C_E_2 = su.C_E_2;
  m.d1 = su.d1; m.d2 = su.d2; m.d3 = su.d3; m.d4 = su.d4; m.d5 = su.d5; m.dNL = su.dNL;
  for (int q = 0; q < 2; q++) {
    m.C1[q] = su.C1[q]; m.C2[q] = su.C2[q]; m.C3[q] = su.C3[q]; m.C4[q] = su.C4[q]; m.C5[q] = su.C5[q];
  }
  m.dt = su.dt; m.z0 = su.z0; m.e0 = su.e0; m.N_EQ = su.N_EQ;
  m.inv_dx = 1.0 / su.p.dx; m.inv_dy = 1.0 / su.p.dy; m.inv_dz = 1.0 / su.p.dz;
  m.hydro = su.hydro;
  m.vac = su.ep0;
  for (int c = 0; c < 3; c++) { m.rho[c] = nullptr; m.rec_off[c] = 0; }
  m.rec = nullptr;
  m.hrec = nullptr;
  m.rec_rows = 1;
  m.rec_slots = 0;
  m.fix_cbrt = (su.p.fixes & FDTD_FIX_HYDRO_CBRT) ? 1 : 0;
  // device copy of the view, read by the cold TFSF helpers of the staged
  // passes (keeps the kernel parameter from escaping to memory)
  {
    SimView<T>* dv;
    cudaError_t e = s->alloc(&dv, 1);
    if (e != cudaSuccess) return fail(FDTD_ERR_ALLOC, cudaGetErrorString(e));
    v.self = dv;
    s->dview = dv;
    CUDA_TRY(cudaMemcpy(dv, &v, sizeof(v), cudaMemcpyHostToDevice));
  }
  // DFT sample ring: two halves of kRingSlots samples
  if (s->dft.rows > 0) {
    T* r;
    cudaError_t e = s->alloc(&r, (size_t)2 * kRingSlots * s->dft.rows, true);
    if (e != cudaSuccess) return fail(FDTD_ERR_ALLOC, cudaGetErrorString(e));
    s->ring = r;
  }
  return FDTD_OK;
}

template <typename T>
static fdtd_status tune_passes(fdtd_sim* s, bool time_variants);

// Tabulates the TFSF corrections of one shell (tfsf_tabulate on the device,
// so the projections round exactly as in the applying kernels), keeps the
// (cell, component) groups that have terms and uploads them packed.
template <typename T>
static fdtd_status build_tfsf_table(fdtd_sim* s, const ShellCells& sh, int efield, TfsfTable& out) {
  const long long nq = sh.total();
  out = TfsfTable{};
  if (nq <= 0) return FDTD_OK;
  const size_t n = (size_t)nq * 3;
  DevBuf b;
  const size_t bytes = n * (4 + 4 + 4 + 4 + 8 + 8 + 1 + 1);
  CUDA_TRY(b.alloc(bytes));
  char* p = static_cast<char*>(b.p);
  double* dp0 = reinterpret_cast<double*>(p);
  double* dp1 = dp0 + n;
  unsigned* id = reinterpret_cast<unsigned*>(dp1 + n);
  unsigned* cn = id + n;
  int* i0 = reinterpret_cast<int*>(cn + n);
  int* i1 = i0 + n;
  unsigned char* m0 = reinterpret_cast<unsigned char*>(i1 + n);
  unsigned char* m1 = m0 + n;
  tfsf_tabulate<T><<<(unsigned)((nq + 127) / 128), 128>>>(static_cast<const SimView<T>*>(s->dview), sh, efield, id,
                                                          cn, i0, i1, dp0, dp1, m0, m1);
  CUDA_TRY(cudaGetLastError());
  std::vector<char> h(bytes);
  CUDA_TRY(cudaMemcpy(h.data(), b.p, bytes, cudaMemcpyDeviceToHost));
  const double* hdp[2] = {reinterpret_cast<const double*>(h.data()), reinterpret_cast<const double*>(h.data()) + n};
  const unsigned* hid = reinterpret_cast<const unsigned*>(hdp[1] + n);
  const unsigned* hcn = hid + n;
  const int* hix[2] = {reinterpret_cast<const int*>(hcn + n), reinterpret_cast<const int*>(hcn + n) + n};
  const unsigned char* hm[2] = {reinterpret_cast<const unsigned char*>(hix[1] + n),
                                reinterpret_cast<const unsigned char*>(hix[1] + n) + n};
  // entries, with every term numbered in a table of the distinct terms
  struct Key {
    long long idx_meta;
    unsigned long long dp_bits;
    bool operator==(const Key& o) const { return idx_meta == o.idx_meta && dp_bits == o.dp_bits; }
  };
  struct KeyHash {
    size_t operator()(const Key& k) const {
      return std::hash<unsigned long long>()(k.dp_bits * 0x9E3779B97F4A7C15ull ^ (unsigned long long)k.idx_meta);
    }
  };
  std::unordered_map<Key, unsigned, KeyHash> seen;
  std::vector<TfsfTerm> terms;
  std::vector<uint4> ent;
  auto term_of = [&](size_t q, int t) -> unsigned {
    Key key{(long long)hix[t][q] << 8 | hm[t][q], 0};
    std::memcpy(&key.dp_bits, &hdp[t][q], sizeof(double));
    auto it = seen.find(key);
    if (it != seen.end()) return it->second;
    const unsigned k = (unsigned)terms.size();
    terms.push_back(TfsfTerm{hdp[t][q], hix[t][q], (int)hm[t][q]});
    seen.emplace(key, k);
    return k;
  };
  for (size_t q = 0; q < n; q++) {
    const unsigned nt = (hcn[q] >> 2) & 3;
    if (nt == 0) continue;
    if (nt > 2) return fail(FDTD_ERR_INVALID, "a TFSF face cell has more than two corrections");
    const unsigned t0 = term_of(q, 0), t1 = nt > 1 ? term_of(q, 1) : t0;
    ent.push_back(make_uint4(hid[q], t0, t1, hcn[q]));
  }
  const size_t m = ent.size();
  out.n = (int)m;
  if (m == 0) return FDTD_OK;
  uint4* dent;
  TfsfTerm* dterm;
  CUDA_TRY(s->alloc(&dent, m));
  CUDA_TRY(s->alloc(&dterm, terms.size()));
  CUDA_TRY(cudaMemcpy(dent, ent.data(), m * sizeof(uint4), cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMemcpy(dterm, terms.data(), terms.size() * sizeof(TfsfTerm), cudaMemcpyHostToDevice));
  out.ent = dent;
  out.term = dterm;
  return FDTD_OK;
}

static fdtd_status create_impl(const fdtd_params* p, int device, fdtd_sim** out, bool tune = true) {
  auto s = std::make_unique<fdtd_sim>();
  if (const char* msg = setup_build(*p, s->su)) return fail(FDTD_ERR_INVALID, msg);
  const Setup& su = s->su;
  s->device = device;
  s->fp64 = su.p.precision == FDTD_FP64;
  CUDA_TRY(cudaSetDevice(device));
  s->NX = su.NX; s->NY = su.NY; s->NZ = su.NZ;
  s->PX = (su.NX + 7) / 8 * 8;
  s->plane = (size_t)s->NY * s->PX;
  s->ncell = s->plane * s->NZ;
  s->kchunk = s->NZ >= 192 ? 32 : 16;
  s->hcfg.kchunk = s->ecfg.kchunk = s->kchunk;
  const size_t es = s->fp64 ? 8 : 4;
  // fields
  for (int c = 0; c < 3; c++) {
    char* a;
    char* b;
    cudaError_t e;
    if ((e = s->alloc(&a, s->ncell * es, true)) != cudaSuccess || (e = s->alloc(&b, s->ncell * es, true)) != cudaSuccess)
      return fail(FDTD_ERR_ALLOC, std::string("field allocation: ") + cudaGetErrorString(e));
    s->E[c] = a;
    s->H[c] = b;
  }
  CUDA_TRY(s->alloc(&s->clk, 1, true));
  CUDA_TRY(s->alloc(&s->e_inc, 2 * (size_t)su.L, true));  // two buffers, by step parity
  CUDA_TRY(s->alloc(&s->h_inc, su.L, true));
  CUDA_TRY(s->alloc(&s->pulse, su.pulse.size()));
  CUDA_TRY(cudaMemcpy(s->pulse, su.pulse.data(), su.pulse.size() * sizeof(double), cudaMemcpyHostToDevice));
  s->probe_cap = su.p.Tend + 2;
  CUDA_TRY(s->alloc(&s->probe, (size_t)3 * s->probe_cap, true));
  s->probe_id = (size_t)su.probe[2] * s->plane + (size_t)su.probe[1] * s->PX + su.probe[0];
  // material bits in device layout + dispersive cell lists
  {
    std::vector<uint8_t> bits(s->ncell, 0);
    int lo[3] = {s->NX, s->NY, s->NZ}, hi[3] = {0, 0, 0};
    std::vector<int4> cells[3];
    for (int k = 0; k < s->NZ; k++)
      for (int j = 0; j < s->NY; j++)
        for (int i = 0; i < s->NX; i++) {
          const size_t r = ((size_t)i * s->NY + j) * s->NZ + k;
          uint8_t b = 0;
          // class 1: the dielectric slab (any component on the slab)
          for (int c = 0; c < 3; c++)
            if (su.matc[c][r] == kSlabMaterial) b = (uint8_t)(1u << 3);
          for (int c = 0; c < 3; c++)
            if (is_dispersive(su.matc[c][r])) {
              b |= (uint8_t)(1u << c);
              // only cells the reference's UPDATE_e* touches: index along c
              // below N-1, the other two strictly inside (main.cu:1172,
              // 1476, 1767); the curl there reads the -1 neighbours
              const int q[3] = {i, j, k};
              const int N3[3] = {s->NX, s->NY, s->NZ};
              bool active = true;
              for (int a = 0; a < 3; a++) {
                if (su.p.periodic_xy && a < 2) continue;  // x and y wrap around
                if (q[a] >= N3[a] - 1) active = false;
                if (a != c && q[a] < 1) active = false;
              }
              if (active) cells[c].push_back(make_int4(i, j, k, (int)cells[c].size()));
            }
          if (b) {
            bits[(size_t)k * s->plane + (size_t)j * s->PX + i] = b;
            lo[0] = std::min(lo[0], i); lo[1] = std::min(lo[1], j); lo[2] = std::min(lo[2], k);
            hi[0] = std::max(hi[0], i + 1); hi[1] = std::max(hi[1], j + 1); hi[2] = std::max(hi[2], k + 1);
          }
        }
    for (int a = 0; a < 3; a++) {
      if (hi[a] <= lo[a]) { lo[a] = 0; hi[a] = 0; }
      s->mat_lo[a] = lo[a];
      s->mat_hi[a] = hi[a];
    }
    // adjoint design box: slot of every box cell per component, blend
    // arrays (rho = 1 until fdtd_set_design), and whether any dispersive
    // cell sits in a CPML slab (the adjoint leaves those out)
    {
      const int* b = su.p.design_box;
      s->has_design = b[1] > b[0] && b[3] > b[2] && b[5] > b[4];
      for (int c = 0; c < 3 && s->has_design; c++) {
        for (int a = 0; a < 6; a++) s->dbox[a] = b[a];
        const int bx = b[1] - b[0], by = b[3] - b[2];
        s->dslot[c].assign((size_t)bx * by * (b[5] - b[4]), -1);
        for (const int4& e : cells[c])
          if (e.x >= b[0] && e.x < b[1] && e.y >= b[2] && e.y < b[3] && e.z >= b[4] && e.z < b[5])
            s->dslot[c][((size_t)(e.z - b[4]) * by + (e.y - b[2])) * bx + (e.x - b[0])] = e.w;
        if (!cells[c].empty()) {
          std::vector<float> ones(cells[c].size(), 1.0f);
          CUDA_TRY(s->alloc(&s->rho_d[c], ones.size()));
          CUDA_TRY(cudaMemcpy(s->rho_d[c], ones.data(), ones.size() * sizeof(float), cudaMemcpyHostToDevice));
        }
      }
      for (int c = 0; c < 3; c++)
        for (const int4& e : cells[c]) {
          const int q[3] = {e.x, e.y, e.z};
          for (int a = 0; a < 3; a++)
            if (su.Nc[a] >= 0 && (q[a] <= su.Nc[a] + 1 || q[a] >= su.F[a] - 1)) s->pml_metal = true;
        }
    }
    CUDA_TRY(s->alloc(&s->mat, s->ncell));
    CUDA_TRY(cudaMemcpy(s->mat, bits.data(), s->ncell, cudaMemcpyHostToDevice));
    // slot lookup over the bounding box grown by one cell, used here to
    // resolve each dispersive cell's hydrodynamic neighbours once
    int box_lo[3], box_dim[3];
    for (int a = 0; a < 3; a++) {
      box_lo[a] = std::max(0, lo[a] - 1);
      int h = std::min(a == 0 ? s->NX : a == 1 ? s->NY : s->NZ, hi[a] + 1);
      box_dim[a] = std::max(0, h - box_lo[a]);
    }
    const size_t nbox = (size_t)box_dim[0] * box_dim[1] * box_dim[2];
    std::vector<int> map[3];
    auto slot = [&](int a, int i, int j, int k) -> int {
      const int x = i - box_lo[0], y = j - box_lo[1], z = k - box_lo[2];
      if (x < 0 || y < 0 || z < 0 || x >= box_dim[0] || y >= box_dim[1] || z >= box_dim[2]) return -1;
      return map[a][((size_t)z * box_dim[1] + y) * box_dim[0] + x];
    };
    for (int c = 0; c < 3; c++) {
      s->nmetal[c] = (int)cells[c].size();
      map[c].assign(nbox, -1);
      for (const int4& e : cells[c])
        map[c][((size_t)(e.z - box_lo[2]) * box_dim[1] + (e.y - box_lo[1])) * box_dim[0] + (e.x - box_lo[0])] = e.w;
    }
    for (int c = 0; c < 3; c++) {
      if (cells[c].empty()) continue;
      CUDA_TRY(s->alloc(&s->mcell[c], cells[c].size()));
      CUDA_TRY(cudaMemcpy(s->mcell[c], cells[c].data(), cells[c].size() * sizeof(int4), cudaMemcpyHostToDevice));
      // per cell and component a: a == c -> +e_c, 0, -e_c, unused;
      // a != c -> +e_c, 0, +e_c - e_a, -e_a
      std::vector<int> nb(cells[c].size() * 12, -1);
      const int oc[3] = {c == 0, c == 1, c == 2};
      for (size_t q = 0; q < cells[c].size(); q++) {
        const int4 e = cells[c][q];
        int* o = nb.data() + q * 12;
        for (int a = 0; a < 3; a++) {
          const int ob[3] = {a == 0, a == 1, a == 2};
          o[a * 4 + 0] = slot(a, e.x + oc[0], e.y + oc[1], e.z + oc[2]);
          o[a * 4 + 1] = slot(a, e.x, e.y, e.z);
          if (a == c) {
            o[a * 4 + 2] = slot(a, e.x - oc[0], e.y - oc[1], e.z - oc[2]);
          } else {
            o[a * 4 + 2] = slot(a, e.x + oc[0] - ob[0], e.y + oc[1] - ob[1], e.z + oc[2] - ob[2]);
            o[a * 4 + 3] = slot(a, e.x - ob[0], e.y - ob[1], e.z - ob[2]);
          }
        }
      }
      CUDA_TRY(s->alloc(&s->nbr[c], nb.size()));
      CUDA_TRY(cudaMemcpy(s->nbr[c], nb.data(), nb.size() * sizeof(int), cudaMemcpyHostToDevice));
    }
  }
  // DFT faces: box b (0 Abs, 1 Sca), face f (-X +X -Y +Y -Z +Z)
  {
    static const int fcomp[3][4] = {{1, 2, 4, 5}, {0, 2, 3, 5}, {0, 1, 3, 4}};
    DftView& d = s->dft;
    std::memset(&d, 0, sizeof(d));
    d.nfaces = su.p.periodic_xy ? 2 : 12;
    long long row = 0;
    // periodic x and y: the reflection and the transmission plane, whole
    // xy planes (Spectral.cu:11-16, 32-120)
    for (int f = 0; su.p.periodic_xy && f < 2; f++) {
      DftFace& F = d.face[f];
      F.ax = 2;
      F.pos = f == 0 ? su.k_refl : su.k_trans;
      F.s1 = 0; F.s2 = 0;
      F.na = s->NX; F.nb = s->NY;
      for (int c = 0; c < 4; c++) F.comp[c] = fcomp[2][c];
      F.row0 = row;
      F.npad = ((long long)F.na * F.nb + kDftRows - 1) / kDftRows * kDftRows;
      row += 4LL * F.npad;
    }
    for (int b = 0; b < 2 && !su.p.periodic_xy; b++) {
      const int* S = b == 0 ? su.absS : su.scaS;
      const int* En = b == 0 ? su.absE : su.scaE;
      for (int f = 0; f < 6; f++) {
        DftFace& F = d.face[b * 6 + f];
        F.ax = f / 2;
        const int a1 = F.ax == 0 ? 1 : 0, a2 = F.ax == 2 ? 1 : 2;
        F.pos = (f & 1) ? En[F.ax] - 1 : S[F.ax];
        F.s1 = S[a1]; F.s2 = S[a2];
        F.na = En[a1] - S[a1]; F.nb = En[a2] - S[a2];
        for (int c = 0; c < 4; c++) F.comp[c] = fcomp[F.ax][c];
        F.row0 = row;
        F.npad = ((long long)F.na * F.nb + kDftRows - 1) / kDftRows * kDftRows;
        row += 4LL * F.npad;
      }
    }
    d.rows = row;
    d.nf = su.p.NUM_freq;
    d.dt = su.dt;
    double* fq;
    CUDA_TRY(s->alloc(&fq, d.nf));
    CUDA_TRY(cudaMemcpy(fq, su.freq.data(), d.nf * sizeof(double), cudaMemcpyHostToDevice));
    d.freq = fq;
    cudaError_t e;
    if ((e = s->alloc(&d.acc_re, (size_t)d.nf * d.rows, true)) != cudaSuccess ||
        (e = s->alloc(&d.acc_im, (size_t)d.nf * d.rows, true)) != cudaSuccess)
      return fail(FDTD_ERR_ALLOC, std::string("DFT accumulators: ") + cudaGetErrorString(e));
    CUDA_TRY(s->alloc(&s->flux, (size_t)12 * d.nf));
    CUDA_TRY(s->alloc(&s->twiddles, (size_t)2 * kRingSlots * d.nf));
  }
  s->dft_on = su.p.StaticField == 0;
  // CPML slab cells and TFSF shells
  {
    int lo[3], hi[3];
    if (su.p.periodic_xy) {
      // the lower z face only: planes Nt_z - 1 (H) and Nt_z (E), every cell
      // of both once (a box two planes thick is all shell)
      const int l[3] = {0, 0, su.Nt[2] - 1}, h[3] = {s->NX - 1, s->NY - 1, su.Nt[2]};
      s->shell_h.init(l, h);
      s->shell_e.init(l, h);
    } else {
      for (int a = 0; a < 3; a++) { lo[a] = su.Nt[a] - 1; hi[a] = (a == 0 ? s->NX : a == 1 ? s->NY : s->NZ) - su.Nt[a]; }
      s->shell_h.init(lo, hi);
      for (int a = 0; a < 3; a++) lo[a] = su.Nt[a];
      s->shell_e.init(lo, hi);
    }
  }
  fdtd_status st = s->fp64 ? build_views<double>(s.get()) : build_views<float>(s.get());
  if (st != FDTD_OK) return st;
  st = s->fp64 ? build_tfsf_table<double>(s.get(), s->shell_h, 0, s->tf_h)
              : build_tfsf_table<float>(s.get(), s->shell_h, 0, s->tf_h);
  if (st != FDTD_OK) return st;
  st = s->fp64 ? build_tfsf_table<double>(s.get(), s->shell_e, 1, s->tf_e)
              : build_tfsf_table<float>(s.get(), s->shell_e, 1, s->tf_e);
  if (st != FDTD_OK) return st;
  if (s->has_design)
    for (int c = 0; c < 3; c++) {
      if (s->fp64) s->md.rho[c] = s->rho_d[c]; else s->mf.rho[c] = s->rho_d[c];
    }
  // line
  LineArgs& L = s->line;
  L.e_inc = s->e_inc; L.h_inc = s->h_inc; L.L = su.L; L.m0 = su.m0; L.src = su.m0 - su.p.source_offset;
  L.ch = su.z0 * su.dt / (su.mu0 * su.d1D);
  L.ce = su.dt / (su.z0 * su.ep0 * su.d1D);
  const double factor = su.c0 * su.dt;
  L.mur = (factor - su.d1D) / (factor + su.d1D);
  L.pulse = s->pulse; L.tmax = (int)su.pulse.size();
  L.clk = s->clk; L.probe = s->probe; L.probe_cap = s->probe_cap;
  L.dft_every = s->dft_on ? su.p.dft_every : 0;
  CUDA_TRY(cudaStreamCreateWithFlags(&s->side, cudaStreamNonBlocking));
  CUDA_TRY(cudaStreamCreateWithFlags(&s->side2, cudaStreamNonBlocking));
  CUDA_TRY(cudaStreamCreateWithFlags(&s->side_dft, cudaStreamNonBlocking));
  CUDA_TRY(cudaEventCreateWithFlags(&s->dft_fork_ev, cudaEventDisableTiming));
  CUDA_TRY(cudaEventCreateWithFlags(&s->dft_join_ev, cudaEventDisableTiming));
  CUDA_TRY(cudaEventCreateWithFlags(&s->fork2_ev, cudaEventDisableTiming));
  CUDA_TRY(cudaEventCreateWithFlags(&s->join2_ev, cudaEventDisableTiming));
  CUDA_TRY(cudaEventCreateWithFlags(&s->fork3_ev, cudaEventDisableTiming));
  CUDA_TRY(cudaEventCreateWithFlags(&s->join3_ev, cudaEventDisableTiming));
  CUDA_TRY(cudaEventCreateWithFlags(&s->fork_ev, cudaEventDisableTiming));
  CUDA_TRY(cudaEventCreateWithFlags(&s->join_ev, cudaEventDisableTiming));
  CUDA_TRY(cudaDeviceSynchronize());
  st = s->fp64 ? tune_passes<double>(s.get(), tune) : tune_passes<float>(s.get(), tune);
  if (st != FDTD_OK) return st;
  *out = s.release();
  return FDTD_OK;
}

extern "C" fdtd_status fdtd_create(const fdtd_params* p, int device, fdtd_sim** out) {
  if (!p || !out) return fail(FDTD_ERR_INVALID, "null argument");
  *out = nullptr;
  try {
    return create_impl(p, device, out);
  } catch (const std::bad_alloc&) {
    return fail(FDTD_ERR_ALLOC, "host allocation failed");
  }
}

extern "C" fdtd_status fdtd_destroy(fdtd_sim* s) {
  if (!s) return FDTD_OK;
  cudaSetDevice(s->device);
  cudaDeviceSynchronize();
  delete s;
  return FDTD_OK;
}

extern "C" fdtd_status fdtd_get_dims(const fdtd_sim* s, fdtd_dims* d) {
  if (!s || !d) return fail(FDTD_ERR_INVALID, "null argument");
  fill_dims(s->su, d);
  return FDTD_OK;
}

extern "C" fdtd_status fdtd_reset(fdtd_sim* s) {
  if (!s) return fail(FDTD_ERR_INVALID, "null argument");
  CUDA_TRY(cudaSetDevice(s->device));
  CUDA_TRY(cudaDeviceSynchronize());
  for (const auto& b : s->state) CUDA_TRY(cudaMemset(b.first, 0, b.second));
  s->t = 0;
  s->host_nsamp = 0;
  s->dft_pending = false;
  s->snap_first = s->snap_drained = 0;
  return FDTD_OK;
}

// ---------------------------------------------------------------------
// launches

template <typename T>
static SimView<T>& view(fdtd_sim* s);
template <>
SimView<float>& view<float>(fdtd_sim* s) { return s->vf; }
template <>
SimView<double>& view<double>(fdtd_sim* s) { return s->vd; }
template <typename T>
static MetalView<T>& mview(fdtd_sim* s);
template <>
MetalView<float>& mview<float>(fdtd_sim* s) { return s->mf; }
template <>
MetalView<double>& mview<double>(fdtd_sim* s) { return s->md; }

template <typename T, int TY, int S>
static size_t staged_smem() {
  return (size_t)S * StageLayout<T, TY>::STAGE * sizeof(T) + (size_t)S * 8;  // ring + its mbarriers
}

// The tensor maps of one tile height: each field component as a {PX, NY,
// NZ} array (row and plane pitches in bytes), the halo family's tile
// (32 + CH) x (TY + 1) and the own family's 32 x TY, zero fill outside.
// Null when the driver's encoder is not available or refuses a map (the
// passes then stage with cp.async).
using EncodeTiledFn = decltype(&cuTensorMapEncodeTiled);
static EncodeTiledFn tensor_map_encoder() {
  static EncodeTiledFn fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  return fn;
}
template <typename T>
static const fdtd_sim::TmaSet* tma_maps(fdtd_sim* s, int ty) {
  if (s->tma_avail == 0) return nullptr;
  for (const auto& m : s->tmasets)
    if (m.ty == ty) return &m;
  EncodeTiledFn enc = tensor_map_encoder();
  if (!enc || s->su.p.periodic_xy) {
    s->tma_avail = 0;
    return nullptr;
  }
  constexpr int CH = 16 / (int)sizeof(T);
  const CUtensorMapDataType dt = sizeof(T) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  const cuuint64_t dims[3] = {(cuuint64_t)s->PX, (cuuint64_t)s->NY, (cuuint64_t)s->NZ};
  const cuuint64_t strides[2] = {(cuuint64_t)s->PX * sizeof(T), (cuuint64_t)s->plane * sizeof(T)};
  const cuuint32_t halo_box[3] = {(cuuint32_t)(32 + CH), (cuuint32_t)(ty + 1), 1};
  const cuuint32_t own_box[3] = {32, (cuuint32_t)ty, 1};
  const cuuint32_t unit[3] = {1, 1, 1};
  fdtd_sim::TmaSet m;
  m.ty = ty;
  m.h.stall = m.e.stall = 0;
  bool ok = true;
  auto encode = [&](CUtensorMap* map, const void* base, const cuuint32_t* box) {
    ok = ok && enc(map, dt, 3, const_cast<void*>(base), dims, strides, box, unit, CU_TENSOR_MAP_INTERLEAVE_NONE,
                   CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
  };
  for (int a = 0; a < 3; a++) {
    encode(&m.h.halo[a], s->E[a], halo_box);
    encode(&m.h.own[a], s->H[a], own_box);
    encode(&m.e.halo[a], s->H[a], halo_box);
    encode(&m.e.own[a], s->E[a], own_box);
  }
  if (!ok) {
    s->tma_avail = 0;
    return nullptr;
  }
  s->tma_avail = 1;
  s->tmasets.push_back(m);
  return &s->tmasets.back();
}

// Staged-pass variants: tile height TY, a register cap given as the
// minimum number of resident CTAs per SM (MINB; 1 = no cap) and the ring
// depth S (S-2 planes of lookahead beyond the ones in use).
#define FDTD_STAGED_VARIANTS(X) X(4, 1, 4) X(4, 6, 4) X(4, 8, 4) X(8, 3, 4) X(4, 6, 6)

// Opt the staged kernels into more than 48 KB of dynamic shared memory once.
template <typename T>
static void staged_attributes() {
  static bool done = false;
  if (done) return;
#define FDTD_ATTR(TY, MB, S)                                                                         \
  cudaFuncSetAttribute(h_pass_s<T, TY, S, MB, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,   \
                       (int)staged_smem<T, TY, S>());                                                \
  cudaFuncSetAttribute(h_pass_s<T, TY, S, MB, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,    \
                       (int)staged_smem<T, TY, S>());                                                \
  cudaFuncSetAttribute(e_pass_s<T, TY, S, MB, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,   \
                       (int)staged_smem<T, TY, S>());                                                \
  cudaFuncSetAttribute(e_pass_s<T, TY, S, MB, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,    \
                       (int)staged_smem<T, TY, S>());                                                \
  cudaFuncSetAttribute(h_pass_t<T, TY, S, MB, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,   \
                       (int)staged_smem<T, TY, S>());                                                \
  cudaFuncSetAttribute(h_pass_t<T, TY, S, MB, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,    \
                       (int)staged_smem<T, TY, S>());                                                \
  cudaFuncSetAttribute(e_pass_t<T, TY, S, MB, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,   \
                       (int)staged_smem<T, TY, S>());                                                \
  cudaFuncSetAttribute(e_pass_t<T, TY, S, MB, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,    \
                       (int)staged_smem<T, TY, S>());
  FDTD_STAGED_VARIANTS(FDTD_ATTR)
#undef FDTD_ATTR
  cudaFuncSetAttribute(dft_contract<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dft_smem_bytes<T>());
  done = true;
}

// Interior box and edge table of the pass tiles for a tile height and
// z-chunk.  A tile is interior when none of its cells lies in a CPML slab
// of the E extent (index <= Nc or >= F, a superset of the H extent).
static fdtd_status build_tiles(fdtd_sim* s, int ty, int kc) {
  for (const auto& t : s->tilesets)
    if (t.ty == ty && t.kchunk == kc) return FDTD_OK;
  fdtd_sim::TileSet ts;
  ts.ty = ty; ts.kchunk = kc;
  const int nb[3] = {(s->NX + 31) / 32, (s->NY + ty - 1) / ty, (s->NZ + kc - 1) / kc};
  const int w[3] = {32, ty, kc};
  int lo[3], hi[3];  // interior tile range [lo, hi)
  for (int a = 0; a < 3; a++) {
    const int Nc = s->su.Nc[a], F = s->su.F[a];
    lo[a] = (Nc + 1 + w[a] - 1) / w[a];
    hi[a] = F >= w[a] ? (F - w[a]) / w[a] + 1 : 0;
    hi[a] = std::min(hi[a], nb[a]);
    if (hi[a] < lo[a]) hi[a] = lo[a];
  }
  const bool inner = hi[0] > lo[0] && hi[1] > lo[1] && hi[2] > lo[2];
  ts.inner = inner ? dim3(hi[0] - lo[0], hi[1] - lo[1], hi[2] - lo[2]) : dim3(0, 0, 0);
  ts.inner_map = TileMap{lo[0], lo[1], lo[2], nullptr};
  std::vector<int4> edge;
  for (int bz = 0; bz < nb[2]; bz++)
    for (int by = 0; by < nb[1]; by++)
      for (int bx = 0; bx < nb[0]; bx++) {
        const bool in = inner && bx >= lo[0] && bx < hi[0] && by >= lo[1] && by < hi[1] && bz >= lo[2] && bz < hi[2];
        if (!in) edge.push_back(make_int4(bx, by, bz, 0));
      }
  ts.nedge = (unsigned)edge.size();
  if (!edge.empty()) {
    int4* d;
    CUDA_TRY(s->alloc(&d, edge.size()));
    CUDA_TRY(cudaMemcpy(d, edge.data(), edge.size() * sizeof(int4), cudaMemcpyHostToDevice));
    ts.edge_map = TileMap{0, 0, 0, d};
  }
  s->tilesets.push_back(ts);
  return FDTD_OK;
}
static const fdtd_sim::TileSet& tiles(const fdtd_sim* s, const fdtd_sim::PassCfg& c) {
  for (const auto& t : s->tilesets)
    if (t.ty == c.ty && t.kchunk == c.kchunk) return t;
  return s->tilesets.front();  // unreachable: every configuration is built at create
}

// One launch of a pass variant over a tile map (box grid or table): the
// cp.async or (tma) the tensor-copy staging, optionally (pdl) with a
// programmatic dependency on the launch before it on the stream.
template <typename T, bool PML, bool EPASS>
static void launch_variant(fdtd_sim* s, int ty, int mb, int sg, bool tma, dim3 g, const TileMap& tm, int kchunk,
                           cudaStream_t st, bool pdl = false) {
  const fdtd_sim::TmaSet* maps = tma ? tma_maps<T>(s, ty) : nullptr;
  // FDTD_TMA_STALL_TEST=1: the launch's copies are never issued (its waits
  // time out; fdtd_check then reports FDTD_ERR_TIMEOUT)
  fdtd_sim::TmaSet stalled;
  const char* stall_env = std::getenv("FDTD_TMA_STALL_TEST");
  if (maps && stall_env && stall_env[0] == '1') {
    stalled = *maps;
    stalled.h.stall = stalled.e.stall = 1;
    maps = &stalled;
  }
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
#define FDTD_LAUNCH(TY, MB, S)                                                                             \
  if (ty == TY && mb == MB && sg == S) {                                                                   \
    cudaLaunchConfig_t cfg = {};                                                                           \
    cfg.gridDim = g; cfg.blockDim = dim3(32, TY); cfg.dynamicSmemBytes = staged_smem<T, TY, S>(); cfg.stream = st; \
    cfg.attrs = at; cfg.numAttrs = pdl ? 1 : 0;                                                            \
    if (maps && EPASS) cudaLaunchKernelEx(&cfg, e_pass_t<T, TY, S, MB, PML>, view<T>(s), kchunk, tm, maps->e); \
    else if (maps) cudaLaunchKernelEx(&cfg, h_pass_t<T, TY, S, MB, PML>, view<T>(s), kchunk, tm, maps->h);  \
    else if (EPASS) cudaLaunchKernelEx(&cfg, e_pass_s<T, TY, S, MB, PML>, view<T>(s), kchunk, tm);           \
    else cudaLaunchKernelEx(&cfg, h_pass_s<T, TY, S, MB, PML>, view<T>(s), kchunk, tm);                      \
    return;                                                                                                \
  }
  FDTD_STAGED_VARIANTS(FDTD_LAUNCH)
#undef FDTD_LAUNCH
}
template <typename T, bool PML>
static void launch_h_variant(fdtd_sim* s, int ty, int mb, int sg, bool tma, dim3 g, const TileMap& tm, int kchunk,
                             cudaStream_t st, bool pdl = false) {
  launch_variant<T, PML, false>(s, ty, mb, sg, tma, g, tm, kchunk, st, pdl);
}
template <typename T, bool PML>
static void launch_e_variant(fdtd_sim* s, int ty, int mb, int sg, bool tma, dim3 g, const TileMap& tm, int kchunk,
                             cudaStream_t st, bool pdl = false) {
  launch_variant<T, PML, true>(s, ty, mb, sg, tma, g, tm, kchunk, st, pdl);
}

// Launches one pass as its interior box (PML-free) and its edge table so
// that the two overlap: the edge launch on the side stream, or (c.pdl) the
// edge launch then the interior launch with a programmatic dependency on
// one stream; returns the number of launches.
// chained (one-stream configurations only): the launch before this pass on
// `st` triggers early and touches none of the pass's cells, so the pass's
// first launch carries a programmatic dependency on it too.
template <typename T, bool EPASS>
static int launch_pass_cfg(fdtd_sim* s, const fdtd_sim::PassCfg& c, cudaStream_t st, bool chained = false) {
  const fdtd_sim::TileSet& ts = tiles(s, c);
  if (c.pdl && ((ts.inner.x && ts.nedge) || chained)) {
    bool dep = chained;
    if (ts.nedge) {
      if (EPASS) launch_e_variant<T, true>(s, c.ty, c.eminb, c.estages, c.etma, dim3(ts.nedge), ts.edge_map, c.kchunk, st, dep);
      else launch_h_variant<T, true>(s, c.ty, c.eminb, c.estages, c.etma, dim3(ts.nedge), ts.edge_map, c.kchunk, st, dep);
      dep = true;
    }
    if (ts.inner.x) {
      if (EPASS) launch_e_variant<T, false>(s, c.ty, c.minb, c.stages, c.tma, ts.inner, ts.inner_map, c.kchunk, st, dep);
      else launch_h_variant<T, false>(s, c.ty, c.minb, c.stages, c.tma, ts.inner, ts.inner_map, c.kchunk, st, dep);
    }
    return (ts.inner.x ? 1 : 0) + (ts.nedge ? 1 : 0);
  }
  const bool fork = ts.inner.x && ts.nedge;
  cudaStream_t est = st;
  if (fork) {
    cudaEventRecord(s->fork_ev, st);
    cudaStreamWaitEvent(s->side, s->fork_ev, 0);
    est = s->side;
  }
  if (ts.nedge) {
    if (EPASS) launch_e_variant<T, true>(s, c.ty, c.eminb, c.estages, c.etma, dim3(ts.nedge), ts.edge_map, c.kchunk, est);
    else launch_h_variant<T, true>(s, c.ty, c.eminb, c.estages, c.etma, dim3(ts.nedge), ts.edge_map, c.kchunk, est);
  }
  if (ts.inner.x) {
    if (EPASS) launch_e_variant<T, false>(s, c.ty, c.minb, c.stages, c.tma, ts.inner, ts.inner_map, c.kchunk, st);
    else launch_h_variant<T, false>(s, c.ty, c.minb, c.stages, c.tma, ts.inner, ts.inner_map, c.kchunk, st);
  }
  if (fork) {
    cudaEventRecord(s->join_ev, s->side);
    cudaStreamWaitEvent(st, s->join_ev, 0);
  }
  return (ts.inner.x ? 1 : 0) + (ts.nedge ? 1 : 0);
}
template <typename T>
static int launch_h_cfg(fdtd_sim* s, const fdtd_sim::PassCfg& c, cudaStream_t st, bool chained = false) {
  return launch_pass_cfg<T, false>(s, c, st, chained);
}
template <typename T>
static int launch_e_cfg(fdtd_sim* s, const fdtd_sim::PassCfg& c, cudaStream_t st, bool chained = false) {
  return launch_pass_cfg<T, true>(s, c, st, chained);
}

// Autotuner: times every launch shape of the E and H passes on the zero
// state (which they leave at zero: no source has run yet) and keeps the
// fastest.  Shapes: minimum CTAs per SM (register cap) x tile height x
// z-chunk.  FDTD_TUNE=0 keeps the defaults.
template <typename T>
static fdtd_status tune_passes(fdtd_sim* s, bool time_variants) {
  staged_attributes<T>();
  // defaults; FDTD_PASS=staged:TY:MINB:KCHUNK[:STAGES] forces a variant,
  // FDTD_TUNE=0 skips the timing, small grids are not worth timing
  fdtd_sim::PassCfg def;
  def.staged = 1; def.ty = 4; def.minb = 1; def.stages = 4; def.kchunk = 16;
  const char* force = std::getenv("FDTD_PASS");
  if (force) {
    const char* c = std::strchr(force, ':');
    int ty, mb, kc;
    int sg = 4;
    if (c && std::sscanf(c + 1, "%d:%d:%d:%d", &ty, &mb, &kc, &sg) >= 3) {
      def.ty = ty; def.minb = mb; def.kchunk = kc; def.stages = sg;
    }
  }
  {
    bool known = false;
#define FDTD_KNOWN(TY, MB, S) known = known || (def.ty == TY && def.minb == MB && def.stages == S);
    FDTD_STAGED_VARIANTS(FDTD_KNOWN)
#undef FDTD_KNOWN
    if (!known || def.kchunk < 1) return fail(FDTD_ERR_INVALID, "FDTD_PASS names a pass variant that is not built");
  }
  def.eminb = def.minb;
  def.estages = def.stages;
  // FDTD_TMA=0 / 1 fixes the staging of both launches (cp.async / tensor
  // copies) instead of timing both
  const char* tma_env = std::getenv("FDTD_TMA");
  const int tma_force = tma_env && (tma_env[0] == '0' || tma_env[0] == '1') ? tma_env[0] - '0' : -1;
  if (tma_force == 1 && tma_maps<T>(s, def.ty)) def.tma = def.etma = 1;
  // FDTD_PDL=0 / 1 fixes how the two launches of a pass overlap (two
  // streams / one stream with a programmatic dependency) instead of timing
  // both
  const char* pdl_env = std::getenv("FDTD_PDL");
  const int pdl_force = pdl_env && (pdl_env[0] == '0' || pdl_env[0] == '1') ? pdl_env[0] - '0' : -1;
  if (pdl_force >= 0) def.pdl = pdl_force;
  s->hcfg = s->ecfg = def;
  {
    const fdtd_status st = build_tiles(s, def.ty, def.kchunk);
    if (st != FDTD_OK) return st;
  }
  const char* env = std::getenv("FDTD_TUNE");
  if (!time_variants || (env && env[0] == '0') || force || s->ncell < (size_t)(1 << 18)) {
    s->tuned = true;
    return FDTD_OK;
  }
  cudaEvent_t a, b;
  CUDA_TRY(cudaEventCreate(&a));
  CUDA_TRY(cudaEventCreate(&b));
  const char* venv = std::getenv("FDTD_TUNE_VERBOSE");
  const bool verbose = venv && venv[0] == '1';
  // per (tile height, z-chunk): the fastest interior variant and the
  // fastest edge variant, each timed alone; the pair with the smallest sum
  const int variants[][3] = {{4, 1, 4}, {4, 6, 4}, {4, 8, 4}, {8, 3, 4}, {4, 6, 6}};
  for (int pass = 0; pass < 2; pass++) {
    // one candidate per (tile height, z-chunk): its fastest launch shapes
    std::vector<fdtd_sim::PassCfg> cands;
    for (int ty : {4, 8})
      for (int kc : {8, 16, 32}) {
        if (kc > 2 * s->NZ) continue;
        const fdtd_status st = build_tiles(s, ty, kc);
        if (st != FDTD_OK) return st;
        fdtd_sim::PassCfg probe;
        probe.ty = ty; probe.kchunk = kc;
        const fdtd_sim::TileSet& ts = tiles(s, probe);
        float bin = ts.inner.x ? 1e30f : 0.f, bed = ts.nedge ? 1e30f : 0.f;
        int in_mb = 1, in_sg = 4, ed_mb = 1, ed_sg = 4, in_tma = 0, ed_tma = 0;
        bool any = false;
        const bool tma_ok = tma_force != 0 && tma_maps<T>(s, ty) != nullptr;
        for (const auto& v : variants)
        for (int tm = tma_force == 1 && tma_ok ? 1 : 0; tm < (tma_ok ? 2 : 1); tm++) {
          if (v[0] != ty) continue;
          const size_t sm = sizeof(T) * (size_t)v[2] * (ty == 4 ? StageLayout<T, 4>::STAGE : StageLayout<T, 8>::STAGE);
          if (sm * std::max(1, v[1]) > 220 * 1024) continue;
          any = true;
          for (int part = 0; part < 2; part++) {
            if (part == 0 ? !ts.inner.x : !ts.nedge) continue;
            auto go = [&]() {
              if (part == 0) {
                if (pass == 0) launch_h_variant<T, false>(s, ty, v[1], v[2], tm, ts.inner, ts.inner_map, kc, 0);
                else launch_e_variant<T, false>(s, ty, v[1], v[2], tm, ts.inner, ts.inner_map, kc, 0);
              } else {
                if (pass == 0) launch_h_variant<T, true>(s, ty, v[1], v[2], tm, dim3(ts.nedge), ts.edge_map, kc, 0);
                else launch_e_variant<T, true>(s, ty, v[1], v[2], tm, dim3(ts.nedge), ts.edge_map, kc, 0);
              }
            };
            go();
            CUDA_TRY(cudaEventRecord(a));
            for (int r = 0; r < 3; r++) go();
            CUDA_TRY(cudaEventRecord(b));
            CUDA_TRY(cudaEventSynchronize(b));
            float ms;
            CUDA_TRY(cudaEventElapsedTime(&ms, a, b));
            ms /= 3;
            if (verbose)
              std::fprintf(stderr, "[fdtd tune] %s %s minb=%d ty=%d kchunk=%d stages=%d %s %.4f ms\n",
                           pass == 0 ? "H" : "E", part == 0 ? "interior" : "edge", v[1], ty, kc, v[2],
                           tm ? "tensor-copy" : "cp.async", ms);
            if (part == 0 && ms < bin) { bin = ms; in_mb = v[1]; in_sg = v[2]; in_tma = tm; }
            if (part == 1 && ms < bed) { bed = ms; ed_mb = v[1]; ed_sg = v[2]; ed_tma = tm; }
          }
        }
        if (!any) continue;
        fdtd_sim::PassCfg cand;
        cand.staged = 1; cand.ty = ty; cand.kchunk = kc;
        cand.minb = in_mb; cand.stages = in_sg; cand.eminb = ed_mb; cand.estages = ed_sg;
        cand.tma = in_tma; cand.etma = ed_tma;
        cand.ms = bin + bed;
        cands.push_back(cand);
      }
    // the fastest candidates by the sum of their launches' times, timed
    // again as whole passes (both launches together, on two streams or on
    // one stream with a programmatic dependency, more repetitions): the
    // launches overlap, and one noisy part time must not decide
    if (cands.empty()) continue;  // no variant fits: the defaults stay
    std::sort(cands.begin(), cands.end(),
              [](const fdtd_sim::PassCfg& x, const fdtd_sim::PassCfg& y) { return x.ms < y.ms; });
    if (cands.size() > 3) cands.resize(3);
    fdtd_sim::PassCfg best = cands.front();
    best.pdl = pdl_force >= 0 ? pdl_force : 0;
    float best_ms = 1e30f;
    for (fdtd_sim::PassCfg c : cands) {
      for (int mode = 0; mode < 2; mode++) {
        if (pdl_force >= 0 && mode != pdl_force) continue;
        c.pdl = mode;
        auto go = [&]() {
          if (pass == 0) launch_pass_cfg<T, false>(s, c, 0);
          else launch_pass_cfg<T, true>(s, c, 0);
        };
        go();
        go();
        CUDA_TRY(cudaEventRecord(a));
        for (int r = 0; r < 10; r++) go();
        CUDA_TRY(cudaEventRecord(b));
        CUDA_TRY(cudaEventSynchronize(b));
        float ms;
        CUDA_TRY(cudaEventElapsedTime(&ms, a, b));
        ms /= 10;
        if (verbose)
          std::fprintf(stderr, "[fdtd tune] %s pass ty=%d kchunk=%d, %s: %.4f ms\n", pass == 0 ? "H" : "E", c.ty,
                       c.kchunk, mode ? "one stream, programmatic dependency" : "two streams", ms);
        if (ms < best_ms) {
          best_ms = ms;
          best = c;
          best.ms = ms;
        }
      }
    }
    (pass == 0 ? s->hcfg : s->ecfg) = best;
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  CUDA_TRY(cudaGetLastError());
  s->tuned = true;
  return FDTD_OK;
}

// A launch on `st` that, when pdl is set, carries a programmatic dependency
// on the launch before it on the stream: it may start once every CTA of
// that launch has started, and orders itself with griddepcontrol.wait.
template <typename... P, typename... A>
static void launch_ex(bool pdl, void (*kern)(P...), dim3 g, dim3 blk, size_t smem, cudaStream_t st, A&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = g;
  cfg.blockDim = blk;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = pdl ? 1 : 0;
  cudaLaunchKernelEx(&cfg, kern, std::forward<A>(args)...);
}

// The split per-half entry points (fdtd_update_h / _line / _e) launch the
// H pass + the H half of CORRECT_*, the line, then the E half + the E pass.
template <typename T>
static void launch_h(fdtd_sim* s, cudaStream_t st) {
  s->kernels += launch_h_cfg<T>(s, s->hcfg, st);
  const int nf = s->tf_h.n;
  if (nf > 0) {
    tfsf_h_apply<T><<<(unsigned)((nf + 255) / 256), 256, 0, st>>>(view<T>(s), s->tf_h, s->line);
    s->kernels++;
  }
}
template <typename T>
static void launch_line(fdtd_sim* s, cudaStream_t st) {
  line_step<T><<<1, 1024, 0, st>>>(s->line, view<T>(s), s->probe_id);
  s->kernels++;
}
template <typename T>
static void launch_metal(fdtd_sim* s, cudaStream_t st, bool chained = false);
template <typename T>
static void launch_e_pass(fdtd_sim* s, cudaStream_t st);

template <typename T>
static void launch_e(fdtd_sim* s, cudaStream_t st) {
  const int nf = s->tf_e.n;
  // E half of CORRECT_* before the update (main.cu:2798-2813)
  if (nf > 0) {
    tfsf_e_apply<T><<<(unsigned)((nf + 255) / 256), 256, 0, st>>>(view<T>(s), s->tf_e);
    s->kernels++;
  }
  launch_e_pass<T>(s, st);
}

// The fused step's TFSF: both halves in one launch, after the line step.
template <typename T>
static void launch_tfsf(fdtd_sim* s, cudaStream_t st) {
  const int nf = s->tf_h.n + s->tf_e.n;
  if (nf > 0) {
    tfsf_apply<T><<<(unsigned)((nf + 255) / 256), 256, 0, st>>>(view<T>(s), s->tf_h, s->tf_e, s->line);
    s->kernels++;
  }
}

template <typename T>
static void launch_e_pass(fdtd_sim* s, cudaStream_t st) {
  // The dispersive components (Drude + 2CP, hydrodynamic current) run beside
  // the E pass: the pass skips them, reads no dispersive E component and
  // writes none, and the dispersive kernels read E^n of their own cells and
  // the final H only.
  const bool metal = s->nmetal[0] + s->nmetal[1] + s->nmetal[2] > 0;
  if (metal && s->ecfg.pdl) {
    // one stream, without a fork: the dispersive kernels, then the pass,
    // each launch with a programmatic dependency on the one before (a
    // dispersive phase waits for the previous phase at its start, the pass
    // for the dispersive kernels at its end)
    launch_metal<T>(s, st, true);
    s->kernels += launch_e_cfg<T>(s, s->ecfg, st, true);
    return;
  }
  if (metal) {
    cudaEventRecord(s->fork2_ev, st);
    cudaStreamWaitEvent(s->side2, s->fork2_ev, 0);
    launch_metal<T>(s, s->side2);
  }
  s->kernels += launch_e_cfg<T>(s, s->ecfg, st);
  if (metal) {
    cudaEventRecord(s->join2_ev, s->side2);
    cudaStreamWaitEvent(st, s->join2_ev, 0);
  }
}

// The dispersive cells' kernels; chained: the hydrodynamic phases after the
// first carry a programmatic dependency on the phase before (they wait for
// it at their start).
template <typename T>
static void launch_metal(fdtd_sim* s, cudaStream_t st, bool chained) {
  const int ntot = s->nmetal[0] + s->nmetal[1] + s->nmetal[2];
  if (ntot == 0) return;
  if (!s->su.hydro) {
    metal_e<T><<<(ntot + 127) / 128, 128, 0, st>>>(view<T>(s), mview<T>(s), s->clk);
    s->kernels++;
  } else {
    // UpdateHydroP* of every cell fused with the Ex update, then Ey, Ez
    hydro_p_ex<T><<<(ntot + 127) / 128, 128, 0, st>>>(view<T>(s), mview<T>(s), s->clk);
    s->kernels++;
    if (s->nmetal[1] > 0) {
      launch_ex(chained, hydro_e<T, 1>, dim3((s->nmetal[1] + 127) / 128), dim3(128), 0, st, view<T>(s), mview<T>(s),
                (const DevClock*)s->clk);
      s->kernels++;
    }
    if (s->nmetal[2] > 0) {
      launch_ex(chained, hydro_e<T, 2>, dim3((s->nmetal[2] + 127) / 128), dim3(128), 0, st, view<T>(s), mview<T>(s),
                (const DevClock*)s->clk);
      s->kernels++;
    }
  }
}
template <typename T>
static void launch_sample(fdtd_sim* s, cudaStream_t st) {
  int maxn = 0;
  for (int f = 0; f < s->dft.nfaces; f++) maxn = std::max(maxn, s->dft.face[f].na * s->dft.face[f].nb);
  dim3 g((maxn + 255) / 256, s->dft.nfaces);
  dft_sample<T><<<g, 256, 0, st>>>(view<T>(s), s->dft, (T*)s->ring, s->clk);
  s->kernels++;
}
// The contraction of the clock's job (dft_job_*): phasors, then the FP64
// product into the accumulators.
template <typename T>
static void launch_contract(fdtd_sim* s, cudaStream_t st) {
  const int ntw = 2 * kRingSlots * s->dft.nf;
  dft_twiddles<<<(ntw + 255) / 256, 256, 0, st>>>(s->dft, s->clk, s->twiddles);
  dft_contract<T><<<(unsigned)(s->dft.rows / kDftRows), 128, dft_smem_bytes<T>(), st>>>(
      s->dft, (const T*)s->ring, s->clk, s->twiddles);
  s->kernels += 2;
}

// A contraction period is kRingSlots samples, two launch periods.  Its first
// sample step, before its line step reserves a ring slot, switches the
// ring's halves and forks the contraction of the half the last period
// filled onto the DFT stream, where it runs beside the steps (it touches
// only that half, the phasors and the accumulators).
template <typename T>
static void dft_period_begin(fdtd_sim* s, cudaStream_t st) {
  if (s->line.dft_every <= 0 || s->t % s->line.dft_every != 0 || s->host_nsamp != 0) return;
  dft_job_period<<<1, 1, 0, st>>>(s->clk);
  cudaEventRecord(s->dft_fork_ev, st);
  cudaStreamWaitEvent(s->side_dft, s->dft_fork_ev, 0);
  launch_contract<T>(s, s->side_dft);
  cudaEventRecord(s->dft_join_ev, s->side_dft);
  s->dft_pending = true;
  s->kernels++;
}

// One DFT sample of the step; the end of the first launch period of a
// contraction period joins the forked contraction, so each captured launch
// period is self-contained.
template <typename T>
static void sample_and_contract(fdtd_sim* s, cudaStream_t st) {
  launch_sample<T>(s, st);
  if (++s->host_nsamp == kSampleBlock && s->dft_pending) {
    cudaStreamWaitEvent(st, s->dft_join_ev, 0);
    s->dft_pending = false;
  }
  if (s->host_nsamp == kRingSlots) s->host_nsamp = 0;
}

// One full step.  The 1-D line step runs beside the H pass (on the second
// side stream, or before it on the same stream with the pass launched as a
// programmatic dependent when the pass's launches run on one stream): it
// reads the line, E at the probe cell and the clock, none of which the H
// pass touches, and writes the line's other E buffer, so the H half of
// CORRECT_* still sees the line's E from before the update, as in the
// reference's order (UPDATE_h*, CORRECT_* H, UPDATE_h_inc/e_inc, CORRECT_* E,
// UPDATE_e*).  Both TFSF halves then run as one launch.  Host
// mirrors of the clock decide which optional kernels run; the kernels read
// t from the device.
template <typename T>
static void enqueue_step(fdtd_sim* s, cudaStream_t st) {
  dft_period_begin<T>(s, st);
  if (s->hcfg.pdl) {
    // one stream, without a fork: the line, then the H pass with a
    // programmatic dependency on it (the pass starts at once and waits for
    // the line at its end)
    launch_line<T>(s, st);
    s->kernels += launch_h_cfg<T>(s, s->hcfg, st, true);
  } else {
    cudaEventRecord(s->fork3_ev, st);
    cudaStreamWaitEvent(s->side2, s->fork3_ev, 0);
    launch_line<T>(s, s->side2);
    s->kernels += launch_h_cfg<T>(s, s->hcfg, st);
    cudaEventRecord(s->join3_ev, s->side2);
    cudaStreamWaitEvent(st, s->join3_ev, 0);
  }
  launch_tfsf<T>(s, st);
  launch_e_pass<T>(s, st);
  if (s->line.dft_every > 0 && s->t % s->line.dft_every == 0) sample_and_contract<T>(s, st);
  if (s->snap_on) {
    const int n = std::max(s->snap.rows * s->snap.cols, std::max(s->snap.aux_len, s->snap.line_len));
    snap_gather<T><<<(unsigned)((n + 255) / 256), 256, 0, st>>>(view<T>(s), mview<T>(s), s->line, s->snap);
    s->kernels++;
  }
  s->t++;
}

// Snapshot records the steps [0, t) have produced (every t_skip-th step).
static long long snap_produced(const fdtd_sim* s, long long t) {
  return t > 0 ? (t - 1) / s->snap.t_skip + 1 : 0;
}

// Scheduling priorities inside a captured step graph (the graph is then
// instantiated to use its nodes' priorities): every kernel but the DFT
// contraction's (phasors and product) runs at the device's highest
// priority, so that the contraction forked beside the steps yields SM room
// to them; the contraction only has to end within its launch period.  On
// the 256^3 workload this shortens the block that carries the contraction
// by 0.8 ms (of 44).  FDTD_GRAPH_PRIORITY=0 leaves every node at its
// stream's priority.  Returns whether any node got a priority.
template <typename T>
static bool graph_priorities(cudaGraph_t g) {
  const char* env = std::getenv("FDTD_GRAPH_PRIORITY");
  if (env && env[0] == '0') return false;
  int least = 0, greatest = 0;
  if (cudaDeviceGetStreamPriorityRange(&least, &greatest) != cudaSuccess || least == greatest) return false;
  size_t n = 0;
  if (cudaGraphGetNodes(g, nullptr, &n) != cudaSuccess || n == 0) return false;
  std::vector<cudaGraphNode_t> nodes(n);
  if (cudaGraphGetNodes(g, nodes.data(), &n) != cudaSuccess) return false;
  const void* dft[2] = {reinterpret_cast<const void*>(dft_contract<T>), reinterpret_cast<const void*>(dft_twiddles)};
  bool any = false, failed = false;
  for (size_t i = 0; i < n; i++) {
    cudaGraphNodeType ty;
    if (cudaGraphNodeGetType(nodes[i], &ty) != cudaSuccess || ty != cudaGraphNodeTypeKernel) continue;
    cudaKernelNodeParams p;
    if (cudaGraphKernelNodeGetParams(nodes[i], &p) != cudaSuccess) { failed = true; continue; }
    if (p.func == dft[0] || p.func == dft[1]) continue;
    cudaKernelNodeAttrValue v = {};
    v.priority = greatest;
    if (cudaGraphKernelNodeSetAttribute(nodes[i], cudaKernelNodeAttributePriority, &v) != cudaSuccess) failed = true;
    else any = true;
  }
  if (failed) cudaGetLastError();  // a node keeps its stream's priority; nothing else depends on it
  return any;
}

template <typename T>
static fdtd_status step_impl(fdtd_sim* s, int nsteps, cudaStream_t st) {
  if (s->snap_on && snap_produced(s, (long long)s->t + nsteps) - s->snap_drained > s->snap.cap)
    return fail(FDTD_ERR_STATE, "the snapshot ring would overflow: drain it (fdtd_snapshots_drain) or step fewer "
                                "steps at a time");
  const int every = s->line.dft_every > 0 ? s->line.dft_every : 1;
  const int G = every * kSampleBlock;  // launch pattern period
  int done = 0;
  while (done < nsteps) {
    // the two launch periods of a contraction period have their own graphs
    const int ph = s->line.dft_every > 0 ? s->host_nsamp / kSampleBlock : 0;
    const bool aligned =
        s->t % G == 0 && s->host_nsamp % kSampleBlock == 0 && !s->dft_pending && nsteps - done >= G;
    if (s->use_graphs && aligned) {
      if (!s->graph[ph]) {
        // capture one period on a private stream, then replay it
        if (!s->graph_stream) CUDA_TRY(cudaStreamCreateWithFlags(&s->graph_stream, cudaStreamNonBlocking));
        cudaGraph_t g;
        const int t_save = s->t, n_save = s->host_nsamp;
        const long long k_save = s->kernels;
        CUDA_TRY(cudaStreamBeginCapture(s->graph_stream, cudaStreamCaptureModeThreadLocal));
        for (int q = 0; q < G; q++) enqueue_step<T>(s, s->graph_stream);
        CUDA_TRY(cudaStreamEndCapture(s->graph_stream, &g));
        s->graph_kernels_p[ph] = s->kernels - k_save;
        s->kernels = k_save;
        s->t = t_save;
        s->host_nsamp = n_save;
        const unsigned long long iflags = graph_priorities<T>(g) ? cudaGraphInstantiateFlagUseNodePriority : 0;
        cudaError_t e = cudaGraphInstantiateWithFlags(&s->graph[ph], g, iflags);
        cudaGraphDestroy(g);
        CUDA_TRY(e);
        s->graph_len = G;
      }
      CUDA_TRY(cudaGraphLaunch(s->graph[ph], st));
      s->kernels += s->graph_kernels_p[ph];
      s->graph_launches++;
      s->t += G;
      if (s->line.dft_every > 0) s->host_nsamp = (s->host_nsamp + kSampleBlock) % kRingSlots;
      done += G;
    } else {
      enqueue_step<T>(s, st);
      done++;
    }
  }
  s->steps_done += nsteps;
  CUDA_TRY(cudaGetLastError());
  return FDTD_OK;
}

static cudaStream_t as_stream(void* p) { return reinterpret_cast<cudaStream_t>(p); }

extern "C" fdtd_status fdtd_step(fdtd_sim* s, int nsteps, void* stream) {
  if (!s || nsteps < 0) return fail(FDTD_ERR_INVALID, "bad argument");
  CUDA_TRY(cudaSetDevice(s->device));
  return s->fp64 ? step_impl<double>(s, nsteps, as_stream(stream)) : step_impl<float>(s, nsteps, as_stream(stream));
}

extern "C" fdtd_status fdtd_run(fdtd_sim* s, void* stream) {
  if (!s) return fail(FDTD_ERR_INVALID, "null argument");
  const int left = s->su.p.Tend + 1 - s->t;
  if (left <= 0) return FDTD_OK;
  return fdtd_step(s, left, stream);
}

extern "C" fdtd_status fdtd_update_h(fdtd_sim* s, void* stream) {
  if (!s) return fail(FDTD_ERR_INVALID, "null argument");
  CUDA_TRY(cudaSetDevice(s->device));
  if (s->fp64) launch_h<double>(s, as_stream(stream)); else launch_h<float>(s, as_stream(stream));
  CUDA_TRY(cudaGetLastError());
  return FDTD_OK;
}
extern "C" fdtd_status fdtd_update_line(fdtd_sim* s, void* stream) {
  if (!s) return fail(FDTD_ERR_INVALID, "null argument");
  CUDA_TRY(cudaSetDevice(s->device));
  if (s->fp64) {
    dft_period_begin<double>(s, as_stream(stream));
    launch_line<double>(s, as_stream(stream));
  } else {
    dft_period_begin<float>(s, as_stream(stream));
    launch_line<float>(s, as_stream(stream));
  }
  CUDA_TRY(cudaGetLastError());
  return FDTD_OK;
}
extern "C" fdtd_status fdtd_update_e(fdtd_sim* s, void* stream) {
  if (!s) return fail(FDTD_ERR_INVALID, "null argument");
  CUDA_TRY(cudaSetDevice(s->device));
  if (s->fp64) launch_e<double>(s, as_stream(stream)); else launch_e<float>(s, as_stream(stream));
  CUDA_TRY(cudaGetLastError());
  return FDTD_OK;
}
extern "C" fdtd_status fdtd_spectral_accumulate(fdtd_sim* s, void* stream) {
  if (!s) return fail(FDTD_ERR_INVALID, "null argument");
  CUDA_TRY(cudaSetDevice(s->device));
  cudaStream_t st = as_stream(stream);
  if (s->line.dft_every > 0 && s->t % s->line.dft_every == 0) {
    if (s->fp64) sample_and_contract<double>(s, st); else sample_and_contract<float>(s, st);
  }
  s->t++;
  CUDA_TRY(cudaGetLastError());
  return FDTD_OK;
}

template <typename T>
static int launch_one(fdtd_sim* s, int which, cudaStream_t st) {
  return which == FDTD_KERNEL_H_PASS ? launch_h_cfg<T>(s, s->hcfg, st) : launch_e_cfg<T>(s, s->ecfg, st);
}

extern "C" fdtd_status fdtd_time_kernel(fdtd_sim* s, int which, int reps, void* stream, double* ms) {
  if (!s || !ms || reps <= 0) return fail(FDTD_ERR_INVALID, "bad argument");
  if (which != FDTD_KERNEL_H_PASS && which != FDTD_KERNEL_E_PASS) return fail(FDTD_ERR_INVALID, "unknown kernel");
  CUDA_TRY(cudaSetDevice(s->device));
  cudaStream_t st = as_stream(stream);
  cudaEvent_t a, b;
  CUDA_TRY(cudaEventCreate(&a));
  CUDA_TRY(cudaEventCreate(&b));
  for (int r = 0; r < 2; r++) {  // warm-up
    s->kernels += s->fp64 ? launch_one<double>(s, which, st) : launch_one<float>(s, which, st);
  }
  cudaEventRecord(a, st);
  for (int r = 0; r < reps; r++) {
    s->kernels += s->fp64 ? launch_one<double>(s, which, st) : launch_one<float>(s, which, st);
  }
  cudaEventRecord(b, st);
  cudaError_t e = cudaEventSynchronize(b);
  float t = 0.f;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&t, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (e != cudaSuccess) return fail(FDTD_ERR_CUDA, cudaGetErrorString(e));
  *ms = (double)t / reps;
  return FDTD_OK;
}

extern "C" fdtd_status fdtd_get_time(const fdtd_sim* s, int* t) {
  if (!s || !t) return fail(FDTD_ERR_INVALID, "null argument");
  *t = s->t;
  return FDTD_OK;
}

extern "C" fdtd_status fdtd_check(fdtd_sim* s) {
  if (!s) return fail(FDTD_ERR_INVALID, "null argument");
  CUDA_TRY(cudaSetDevice(s->device));
  DevClock c;
  CUDA_TRY(cudaMemcpy(&c, s->clk, sizeof(c), cudaMemcpyDeviceToHost));
  if (c.nonfinite & 2) return fail(FDTD_ERR_TIMEOUT, "a Yee pass gave up waiting for its plane copies");
  if (c.nonfinite) return fail(FDTD_ERR_NONFINITE, "non-finite field value detected");
  return FDTD_OK;
}

// ---------------------------------------------------------------------
// spectra

// Contracts the samples of the ring half being filled that no contraction
// has taken (nothing when there are none); the stepper's contraction period
// goes on where it was.  The callers have synchronised the device, so no
// forked contraction is in flight.
static fdtd_status flush_dft(fdtd_sim* s) {
  if (s->dft.rows > 0 && s->line.dft_every > 0) {
    dft_job_flush<<<1, 1>>>(s->clk);
    if (s->fp64) launch_contract<double>(s, 0); else launch_contract<float>(s, 0);
  }
  CUDA_TRY(cudaGetLastError());
  return FDTD_OK;
}

extern "C" fdtd_status fdtd_spectral_finalize(fdtd_sim* s, double* out) {
  if (!s || !out) return fail(FDTD_ERR_INVALID, "null argument");
  CUDA_TRY(cudaSetDevice(s->device));
  CUDA_TRY(cudaDeviceSynchronize());
  if (s->su.p.periodic_xy)
    return fail(FDTD_ERR_STATE, "a periodic_xy simulation has no DFT box: fdtd_reflectance gives its spectra");
  fdtd_status st = flush_dft(s);
  if (st != FDTD_OK) return st;
  const int nf = s->dft.nf;
  flux_reduce<<<dim3(12, nf), 256>>>(s->dft, s->flux);
  CUDA_TRY(cudaGetLastError());
  std::vector<double> Q((size_t)12 * nf);
  CUDA_TRY(cudaMemcpy(Q.data(), s->flux, Q.size() * sizeof(double), cudaMemcpyDeviceToHost));
  const Setup& su = s->su;
  const double dxy = su.p.dx * su.p.dy;
  const bool sphere = su.p.geometry == FDTD_GEOM_REFERENCE && su.p.nano_sphere == 1;
  for (int m = 0; m < nf; m++) {
    const double amp = std::abs(su.Einc[m]);
    double q[2][6];
    for (int b = 0; b < 2; b++)
      for (int f = 0; f < 6; f++) q[b][f] = Q[(size_t)(b * 6 + f) * nf + m] * dxy / (amp * amp);
    double sca = -q[1][0] + q[1][1] - q[1][2] + q[1][3] - q[1][4] + q[1][5];
    double ab = -q[0][0] + q[0][1] - q[0][2] + q[0][3] - q[0][4] + q[0][5];
    if (sphere) {
      const double r = su.p.nano_sphere_radius;
      sca = sca / (su.pi * r * r);
      ab = -ab / (su.pi * r * r);
    }
    double* row = out + 19 * (size_t)m;
    row[0] = su.c0 / su.freq[m];
    row[1] = sca; row[2] = ab; row[3] = ab + sca;
    for (int f = 0; f < 6; f++) { row[4 + f] = q[1][f]; row[10 + f] = q[0][f]; }
    row[16] = amp; row[17] = su.Einc[m].real(); row[18] = su.Einc[m].imag();
  }
  return FDTD_OK;
}

extern "C" fdtd_status fdtd_write_scatabs(fdtd_sim* s, const char* path) {
  if (!s || !path) return fail(FDTD_ERR_INVALID, "null argument");
  std::vector<double> rows((size_t)19 * s->dft.nf);
  fdtd_status st = fdtd_spectral_finalize(s, rows.data());
  if (st != FDTD_OK) return st;
  FILE* f = std::fopen(path, "w");
  if (!f) return fail(FDTD_ERR_IO, std::string("cannot write ") + path);
  for (int m = 0; m < s->dft.nf; m++) {
    for (int c = 0; c < 19; c++) std::fprintf(f, c == 18 ? "%e\n" : "%e\t", rows[(size_t)19 * m + c]);
  }
  std::fclose(f);
  return FDTD_OK;
}

// R and T of a periodic simulation (Reflectance_XZ, main.cu:3195-3320):
// per frequency P = sum Re(Ey conj(Hx) - Ex conj(Hy)) dA over the
// reflection plane (scattered field: the reflected wave, P > 0) and the
// transmission plane (total field: the transmitted wave, P < 0), over the
// plane's area and |E_inc / dft_every|^2 (the planes are sampled every
// dft_every steps, E_inc sums every step).  flux_reduce sums Re(Ex conj(Hy)
// - Ey conj(Hx)) = -P / dA per plane.
extern "C" fdtd_status fdtd_reflectance(fdtd_sim* s, double* out) {
  if (!s || !out) return fail(FDTD_ERR_INVALID, "null argument");
  if (!s->su.p.periodic_xy) return fail(FDTD_ERR_STATE, "fdtd_reflectance needs a periodic_xy simulation");
  CUDA_TRY(cudaSetDevice(s->device));
  CUDA_TRY(cudaDeviceSynchronize());
  fdtd_status st = flush_dft(s);
  if (st != FDTD_OK) return st;
  const int nf = s->dft.nf;
  flux_reduce<<<dim3(2, nf), 256>>>(s->dft, s->flux);
  CUDA_TRY(cudaGetLastError());
  std::vector<double> Q((size_t)2 * nf);
  CUDA_TRY(cudaMemcpy(Q.data(), s->flux, Q.size() * sizeof(double), cudaMemcpyDeviceToHost));
  const Setup& su = s->su;
  const double cells = (double)s->NX * s->NY;  // area / (dx dy)
  for (int m = 0; m < nf; m++) {
    const double amp = std::abs(su.Einc[m]), as = amp / su.p.dft_every;
    const double inc = cells * as * as;
    const double R = -Q[m] / inc, T = Q[(size_t)nf + m] / inc;
    double* row = out + 7 * (size_t)m;
    row[0] = su.c0 / su.freq[m];
    row[1] = R; row[2] = T; row[3] = 1.0 - R - T;
    row[4] = amp; row[5] = su.Einc[m].real(); row[6] = su.Einc[m].imag();
  }
  return FDTD_OK;
}

extern "C" fdtd_status fdtd_get_dft(fdtd_sim* s, int box, int face, int comp, double* re, double* im,
                                    size_t count) {
  if (!s || !re || !im || box < 0 || box > 1 || face < 0 || face > 5 || comp < 0 || comp > 3)
    return fail(FDTD_ERR_INVALID, "bad argument");
  CUDA_TRY(cudaSetDevice(s->device));
  CUDA_TRY(cudaDeviceSynchronize());
  if (s->su.p.periodic_xy && (box != 0 || face > 1))
    return fail(FDTD_ERR_INVALID, "periodic_xy: box 0, face 0 (reflection plane) or 1 (transmission plane)");
  fdtd_status st = flush_dft(s);
  if (st != FDTD_OK) return st;
  const DftFace& F = s->dft.face[box * 6 + face];
  const int A = F.na + 1, B = F.nb + 1, nf = s->dft.nf;
  if (count != (size_t)nf * A * B) return fail(FDTD_ERR_INVALID, "count must be NUM_freq*(na+1)*(nb+1)");
  std::memset(re, 0, count * sizeof(double));
  std::memset(im, 0, count * sizeof(double));
  const size_t n = (size_t)F.na * F.nb;
  std::vector<double> r(n), i(n);
  for (int m = 0; m < nf; m++) {
    const size_t off = (size_t)m * s->dft.rows + F.row0 + (size_t)comp * F.npad;
    CUDA_TRY(cudaMemcpy(r.data(), s->dft.acc_re + off, n * sizeof(double), cudaMemcpyDeviceToHost));
    CUDA_TRY(cudaMemcpy(i.data(), s->dft.acc_im + off, n * sizeof(double), cudaMemcpyDeviceToHost));
    for (int u = 0; u < F.na; u++)
      for (int v = 0; v < F.nb; v++) {
        re[((size_t)m * A + u) * B + v] = r[(size_t)u * F.nb + v];
        im[((size_t)m * A + u) * B + v] = i[(size_t)u * F.nb + v];
      }
  }
  return FDTD_OK;
}

extern "C" fdtd_status fdtd_get_freqs(const fdtd_sim* s, double* freq, size_t count) {
  if (!s || !freq || count != s->su.freq.size()) return fail(FDTD_ERR_INVALID, "bad argument");
  std::memcpy(freq, s->su.freq.data(), count * sizeof(double));
  return FDTD_OK;
}

extern "C" fdtd_status fdtd_get_incident(const fdtd_sim* s, double* re, double* im, size_t count) {
  if (!s || !re || !im || count != s->su.Einc.size()) return fail(FDTD_ERR_INVALID, "bad argument");
  for (size_t m = 0; m < count; m++) { re[m] = s->su.Einc[m].real(); im[m] = s->su.Einc[m].imag(); }
  return FDTD_OK;
}

// ---------------------------------------------------------------------
// fields, snapshots, probes

static void* comp_ptr(fdtd_sim* s, int comp) { return comp < 3 ? s->E[comp] : s->H[comp - 3]; }

extern "C" fdtd_status fdtd_get_field(fdtd_sim* s, int comp, double* out, size_t count) {
  if (!s || !out || comp < 0 || comp > 5) return fail(FDTD_ERR_INVALID, "bad argument");
  const size_t n = (size_t)s->NX * s->NY * s->NZ;
  if (count != n) return fail(FDTD_ERR_INVALID, "count must be nx*ny*nz");
  CUDA_TRY(cudaSetDevice(s->device));
  double* tmp;
  CUDA_TRY(cudaMalloc(&tmp, n * sizeof(double)));
  const unsigned g = (unsigned)((n + 255) / 256);
  if (s->fp64) to_ref_layout<double><<<g, 256>>>((const double*)comp_ptr(s, comp), tmp, s->NX, s->NY, s->NZ, s->PX);
  else to_ref_layout<float><<<g, 256>>>((const float*)comp_ptr(s, comp), tmp, s->NX, s->NY, s->NZ, s->PX);
  cudaError_t e = cudaMemcpy(out, tmp, n * sizeof(double), cudaMemcpyDeviceToHost);
  cudaFree(tmp);
  CUDA_TRY(e);
  return FDTD_OK;
}

extern "C" fdtd_status fdtd_set_field(fdtd_sim* s, int comp, const double* in, size_t count) {
  if (!s || !in || comp < 0 || comp > 5) return fail(FDTD_ERR_INVALID, "bad argument");
  const size_t n = (size_t)s->NX * s->NY * s->NZ;
  if (count != n) return fail(FDTD_ERR_INVALID, "count must be nx*ny*nz");
  CUDA_TRY(cudaSetDevice(s->device));
  double* tmp;
  CUDA_TRY(cudaMalloc(&tmp, n * sizeof(double)));
  cudaError_t e = cudaMemcpy(tmp, in, n * sizeof(double), cudaMemcpyHostToDevice);
  const unsigned g = (unsigned)((n + 255) / 256);
  if (e == cudaSuccess) {
    if (s->fp64) from_ref_layout<double><<<g, 256>>>(tmp, (double*)comp_ptr(s, comp), s->NX, s->NY, s->NZ, s->PX);
    else from_ref_layout<float><<<g, 256>>>(tmp, (float*)comp_ptr(s, comp), s->NX, s->NY, s->NZ, s->PX);
    e = cudaDeviceSynchronize();
  }
  cudaFree(tmp);
  CUDA_TRY(e);
  return FDTD_OK;
}

template <typename T>
__global__ void plane_gather(const T* src, double* dst, int NX, int NY, int NZ, int PX, int axis, int index) {
  const int na = axis == 0 ? NY : NX;
  const int nb = axis == 2 ? NY : NZ;
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= na * nb) return;
  const int a = q / nb, b = q - a * nb;
  int i, j, k;
  if (axis == 0) { i = index; j = a; k = b; }
  else if (axis == 1) { i = a; j = index; k = b; }
  else { i = a; j = b; k = index; }
  dst[q] = (double)src[((size_t)k * NY + j) * PX + i];
}

extern "C" fdtd_status fdtd_snapshot_plane(fdtd_sim* s, int comp, int axis, int index, double* dst, size_t count,
                                           void* stream) {
  if (!s || !dst || comp < 0 || comp > 5 || axis < 0 || axis > 2) return fail(FDTD_ERR_INVALID, "bad argument");
  const int N3[3] = {s->NX, s->NY, s->NZ};
  if (index < 0 || index >= N3[axis]) return fail(FDTD_ERR_INVALID, "plane index outside the grid");
  const int na = axis == 0 ? s->NY : s->NX, nb = axis == 2 ? s->NY : s->NZ;
  if (count != (size_t)na * nb) return fail(FDTD_ERR_INVALID, "count must match the plane size");
  CUDA_TRY(cudaSetDevice(s->device));
  cudaPointerAttributes at;
  CUDA_TRY(cudaPointerGetAttributes(&at, dst));
  const bool on_dev = at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
  cudaStream_t st = as_stream(stream);
  double* tgt = dst;
  if (!on_dev) CUDA_TRY(cudaMalloc(&tgt, count * sizeof(double)));
  const unsigned g = (unsigned)((count + 255) / 256);
  if (s->fp64)
    plane_gather<double><<<g, 256, 0, st>>>((const double*)comp_ptr(s, comp), tgt, s->NX, s->NY, s->NZ, s->PX, axis,
                                            index);
  else
    plane_gather<float><<<g, 256, 0, st>>>((const float*)comp_ptr(s, comp), tgt, s->NX, s->NY, s->NZ, s->PX, axis,
                                           index);
  if (!on_dev) {
    cudaError_t e = cudaMemcpyAsync(dst, tgt, count * sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    cudaFree(tgt);
    CUDA_TRY(e);
  }
  CUDA_TRY(cudaGetLastError());
  return FDTD_OK;
}

// ---------------------------------------------------------------------
// Plane snapshot that allocates nothing.  fdtd_snapshot_plane needs a
// temporary device buffer for a host destination; its cudaMalloc/cudaFree
// pair synchronises the whole device and can fail once the simulation has
// filled the GPU.  A snapshot writer called every few hundred steps inside
// a pipelined time loop, or a host that sized the grid to the device memory,
// cannot afford either, so this variant gathers into one fixed scratch array
// in the module's static device memory instead.
//
// Limits and rules: a plane of at most kPlaneScratchCells cells; nothing in
// the scratch has to start at zero (the gather writes every element that is
// copied back); the scratch is one per device, shared by every simulation
// in the process, so calls that overlap in time on the same device (from
// several host threads, or on streams that run concurrently) race on it and
// must be serialised by the caller.  Every call synchronises its stream
// (also for a device destination).  The first call on each device resolves
// the scratch address with cudaGetSymbolAddress and keeps it for the life
// of the process; a cudaDeviceReset would leave the kept address stale, so
// the library must not be used across one.
constexpr size_t kPlaneScratchCells = (size_t)1 << 20;  // 8 MiB of doubles
static __device__ __align__(256) double g_plane_scratch[kPlaneScratchCells];

static fdtd_status plane_scratch(int device, double** out) {
  constexpr int kMaxDevices = 64;
  static std::mutex mu;
  static double* ptr[kMaxDevices] = {};
  if (device < 0 || device >= kMaxDevices) return fail(FDTD_ERR_INVALID, "device index out of range");
  std::lock_guard<std::mutex> lock(mu);
  if (!ptr[device]) {
    // the device is current (the caller set it)
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_plane_scratch);
    if (e != cudaSuccess || !p) return fail(FDTD_ERR_CUDA, std::string("scratch address: ") + cudaGetErrorString(e));
    ptr[device] = static_cast<double*>(p);
  }
  *out = ptr[device];
  return FDTD_OK;
}

extern "C" fdtd_status fdtd_snapshot_plane_static(fdtd_sim* s, int comp, int axis, int index, double* dst,
                                                  size_t count, void* stream) {
  if (!s || !dst || comp < 0 || comp > 5 || axis < 0 || axis > 2) return fail(FDTD_ERR_INVALID, "bad argument");
  const int N3[3] = {s->NX, s->NY, s->NZ};
  if (index < 0 || index >= N3[axis]) return fail(FDTD_ERR_INVALID, "plane index outside the grid");
  const int na = axis == 0 ? s->NY : s->NX, nb = axis == 2 ? s->NY : s->NZ;
  if (count != (size_t)na * nb) return fail(FDTD_ERR_INVALID, "count must match the plane size");
  if (count > kPlaneScratchCells)
    return fail(FDTD_ERR_INVALID, "plane of " + std::to_string(count) + " cells exceeds the " +
                                      std::to_string(kPlaneScratchCells) +
                                      "-cell scratch of fdtd_snapshot_plane_static; use fdtd_snapshot_plane");
  CUDA_TRY(cudaSetDevice(s->device));
  double* scratch = nullptr;
  const fdtd_status st0 = plane_scratch(s->device, &scratch);
  if (st0 != FDTD_OK) return st0;
  cudaStream_t st = as_stream(stream);
  const unsigned g = (unsigned)((count + 255) / 256);
  if (s->fp64)
    plane_gather<double><<<g, 256, 0, st>>>((const double*)comp_ptr(s, comp), scratch, s->NX, s->NY, s->NZ, s->PX,
                                            axis, index);
  else
    plane_gather<float><<<g, 256, 0, st>>>((const float*)comp_ptr(s, comp), scratch, s->NX, s->NY, s->NZ, s->PX,
                                           axis, index);
  CUDA_TRY(cudaGetLastError());
  s->kernels++;
  CUDA_TRY(cudaMemcpyAsync(dst, scratch, count * sizeof(double), cudaMemcpyDefault, st));
  CUDA_TRY(cudaStreamSynchronize(st));
  return FDTD_OK;
}

extern "C" fdtd_status fdtd_get_probe(fdtd_sim* s, double* out, size_t count, int* n) {
  if (!s || !out || !n) return fail(FDTD_ERR_INVALID, "null argument");
  CUDA_TRY(cudaSetDevice(s->device));
  // record the E of the last completed step (the line kernel records
  // the previous step at the start of each new one)
  if (s->fp64) probe_record<double><<<1, 32>>>(s->vd, s->clk, s->probe, s->probe_cap, s->probe_id);
  else probe_record<float><<<1, 32>>>(s->vf, s->clk, s->probe, s->probe_cap, s->probe_id);
  CUDA_TRY(cudaDeviceSynchronize());
  size_t have = (size_t)3 * std::min(s->t, s->probe_cap);
  size_t m = std::min(have, count);
  CUDA_TRY(cudaMemcpy(out, s->probe, m * sizeof(double), cudaMemcpyDeviceToHost));
  *n = (int)(m / 3);
  return FDTD_OK;
}

extern "C" fdtd_status fdtd_get_probe_range(fdtd_sim* s, int t0, int n, double* out, void* stream) {
  if (!s || !out || t0 < 0 || n < 0 || t0 + n > s->probe_cap) return fail(FDTD_ERR_INVALID, "bad probe range");
  CUDA_TRY(cudaSetDevice(s->device));
  cudaStream_t st = as_stream(stream);
  if (t0 + n >= s->t) {  // the last step's row is written by the next line kernel
    if (s->fp64) probe_record<double><<<1, 32, 0, st>>>(s->vd, s->clk, s->probe, s->probe_cap, s->probe_id);
    else probe_record<float><<<1, 32, 0, st>>>(s->vf, s->clk, s->probe, s->probe_cap, s->probe_id);
    s->kernels++;
  }
  CUDA_TRY(cudaMemcpyAsync(out, s->probe + (size_t)3 * t0, (size_t)3 * n * sizeof(double), cudaMemcpyDeviceToHost, st));
  return FDTD_OK;
}

extern "C" fdtd_status fdtd_set_source(fdtd_sim* s, int t0, int n, const double* pulse, void* stream) {
  if (!s || !pulse || t0 < 0 || n < 0 || (size_t)t0 + n > s->su.pulse.size())
    return fail(FDTD_ERR_INVALID, "source range outside [0, Tend]");
  CUDA_TRY(cudaSetDevice(s->device));
  CUDA_TRY(cudaMemcpyAsync(s->pulse + t0, pulse, (size_t)n * sizeof(double), cudaMemcpyHostToDevice, as_stream(stream)));
  return FDTD_OK;
}

// the adjoint's part of the statistics (adjoint_host.cuh)
static void adj_stats(const fdtd_sim* s, fdtd_stats* out);

extern "C" fdtd_status fdtd_get_stats(const fdtd_sim* s, fdtd_stats* out) {
  if (!s || !out) return fail(FDTD_ERR_INVALID, "null argument");
  out->kernels = s->kernels;
  out->steps = s->steps_done;
  out->graph_launches = s->graph_launches;
  out->h_minb = s->hcfg.minb; out->h_ty = s->hcfg.ty; out->h_kchunk = s->hcfg.kchunk;
  out->e_minb = s->ecfg.minb; out->e_ty = s->ecfg.ty; out->e_kchunk = s->ecfg.kchunk;
  out->h_ms = s->hcfg.ms; out->e_ms = s->ecfg.ms;
  out->h_staged = s->hcfg.staged; out->e_staged = s->ecfg.staged;
  out->h_stages = s->hcfg.stages; out->e_stages = s->ecfg.stages;
  out->h_eminb = s->hcfg.eminb; out->h_estages = s->hcfg.estages;
  out->e_eminb = s->ecfg.eminb; out->e_estages = s->ecfg.estages;
  out->h_pdl = s->hcfg.pdl; out->e_pdl = s->ecfg.pdl;
  out->h_tma = s->hcfg.tma; out->h_etma = s->hcfg.etma;
  out->e_tma = s->ecfg.tma; out->e_etma = s->ecfg.etma;
  out->tfsf_entries_h = s->tf_h.n;
  out->tfsf_entries_e = s->tf_e.n;
  long long rows = 0;
  for (int f = 0; f < s->dft.nfaces; f++) rows += 4LL * s->dft.face[f].na * s->dft.face[f].nb;
  out->dft_rows = rows;
  adj_stats(s, out);
  return FDTD_OK;
}

extern "C" fdtd_status fdtd_get_material(fdtd_sim* s, uint8_t* out, size_t count) {
  if (!s || !out) return fail(FDTD_ERR_INVALID, "null argument");
  const size_t n = (size_t)s->NX * s->NY * s->NZ;
  if (count != n) return fail(FDTD_ERR_INVALID, "count must be nx*ny*nz");
  for (int i = 0; i < s->NX; i++)
    for (int j = 0; j < s->NY; j++)
      for (int k = 0; k < s->NZ; k++) {
        const size_t r = ((size_t)i * s->NY + j) * s->NZ + k;
        uint8_t b = 0;
        for (int c = 0; c < 3; c++) b |= (uint8_t)(is_dispersive(s->su.matc[c][r]) << c);
        out[r] = b;
      }
  return FDTD_OK;
}

// ---------------------------------------------------------------------
// snapshots (snapshot.cuh)

extern "C" fdtd_status fdtd_snapshots_enable(fdtd_sim* s, int mode, int capacity, fdtd_snapshot_layout* out) {
  if (!s) return fail(FDTD_ERR_INVALID, "null argument");
  if (mode < 0 || mode > 3) return fail(FDTD_ERR_INVALID, "mode must be 0 (off) or Snap_in 1, 2 or 3");
  CUDA_TRY(cudaSetDevice(s->device));
  CUDA_TRY(cudaDeviceSynchronize());
  // a captured step graph holds the step's launches: capture it again
  for (auto& g : s->graph)
    if (g) {
      cudaGraphExecDestroy(g);
      g = nullptr;
    }
  s->graph_epoch++;
  s->snap_on = false;
  if (mode == 0) {
    if (out) std::memset(out, 0, sizeof(*out));
    return FDTD_OK;
  }
  if (capacity <= 0) return fail(FDTD_ERR_INVALID, "capacity must be positive");
  const fdtd_params& p = s->su.p;
  if (p.t_skip <= 0 || p.y_skip <= 0 || p.z_skip <= 0) return fail(FDTD_ERR_INVALID, "t_skip, y_skip, z_skip must be positive");
  SnapArgs a{};
  a.mode = mode;
  a.t_skip = p.t_skip; a.y_skip = p.y_skip; a.z_skip = p.z_skip;
  a.xc = s->NX / 2;
  a.rows = (s->NY + p.y_skip - 1) / p.y_skip;
  a.cols = (s->NZ + p.z_skip - 1) / p.z_skip;
  a.off_plane = a.off_plane2 = a.off_aux = a.off_line = -1;
  int rec = 1;  // the step index
  if (mode == 1 || mode == 3) {
    a.aux_len = (s->NZ + p.z_skip - 1) / p.z_skip;
    a.line_len = (s->line.L + p.z_skip - 1) / p.z_skip;
    a.off_aux = rec; rec += a.aux_len;
    a.off_line = rec; rec += a.line_len;
  }
  if (mode == 3) { a.off_plane = rec; rec += a.rows * a.cols; }
  if (mode == 2) {
    a.off_plane = rec; rec += a.rows * a.cols;
    a.off_plane2 = rec; rec += a.rows * a.cols;
    // dispersive slot of every plane cell per component
    std::vector<int> ps((size_t)a.rows * a.cols * 3, -1);
    for (int c = 0; c < 3; c++) {
      if (s->nmetal[c] == 0) continue;
      std::vector<int4> cells(s->nmetal[c]);
      CUDA_TRY(cudaMemcpy(cells.data(), s->mcell[c], cells.size() * sizeof(int4), cudaMemcpyDeviceToHost));
      for (const int4& e : cells)
        if (e.x == a.xc && e.y % p.y_skip == 0 && e.z % p.z_skip == 0)
          ps[((size_t)(e.y / p.y_skip) * a.cols + e.z / p.z_skip) * 3 + c] = e.w;
    }
    int* d;
    CUDA_TRY(s->alloc(&d, ps.size()));
    CUDA_TRY(cudaMemcpy(d, ps.data(), ps.size() * sizeof(int), cudaMemcpyHostToDevice));
    a.pslot = d;
  }
  a.rec = rec;
  a.cap = capacity;
  double* ring;
  CUDA_TRY(s->alloc(&ring, (size_t)rec * capacity));
  a.ring = ring;
  s->snap = a;
  s->snap_on = true;
  s->snap_first = s->snap_drained = snap_produced(s, s->t);
  if (out) {
    out->mode = mode;
    out->t_skip = a.t_skip;
    out->plane_rows = mode >= 2 ? a.rows : 0;
    out->plane_cols = mode >= 2 ? a.cols : 0;
    out->aux_len = mode != 2 ? a.aux_len : 0;
    out->line_len = mode != 2 ? a.line_len : 0;
    out->off_plane = a.off_plane; out->off_plane2 = a.off_plane2;
    out->off_aux = a.off_aux; out->off_line = a.off_line;
    out->record = rec;
    out->capacity = capacity;
  }
  return FDTD_OK;
}

extern "C" fdtd_status fdtd_snapshots_drain(fdtd_sim* s, double* host, int max_records, int* n, void* stream) {
  if (!s || !host || !n || max_records < 0) return fail(FDTD_ERR_INVALID, "bad argument");
  if (!s->snap_on) return fail(FDTD_ERR_STATE, "snapshots are not enabled");
  CUDA_TRY(cudaSetDevice(s->device));
  const long long have = snap_produced(s, s->t) - s->snap_drained;
  const int m = (int)std::min<long long>(have, max_records);
  cudaStream_t st = as_stream(stream);
  const SnapArgs& a = s->snap;
  int done = 0;
  while (done < m) {
    const long long r = s->snap_drained + done;
    const int slot = (int)(r % a.cap);
    const int run = std::min(m - done, a.cap - slot);  // contiguous up to the ring's end
    CUDA_TRY(cudaMemcpyAsync(host + (size_t)done * a.rec, a.ring + (size_t)slot * a.rec,
                             (size_t)run * a.rec * sizeof(double), cudaMemcpyDeviceToHost, st));
    done += run;
  }
  s->snap_drained += m;
  *n = m;
  return FDTD_OK;
}

#include "batch.cuh"
#include "adjoint_host.cuh"
