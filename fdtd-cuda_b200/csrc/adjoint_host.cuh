// Host side of the adjoint (no counterpart in the reference): design-region
// blend, forward run with field checkpoints, and the reverse sweep with
// segment recompute.  Included at the end of fdtd.cu (it uses the
// simulation internals defined there).
//
// The transposed Yee and CPML operators need no forward values (the step is
// linear with fixed coefficients), so the reverse sweep needs, per step, only
// the dispersive cells' local values (their trajectory record).
// fdtd_forward runs the whole time loop from zero fields in segments of
// checkpoint_every steps.  The last segments, as many as the record budget
// holds (all of them when it fits), record their trajectory as they run;
// every earlier segment starts with a copy of the state (fields, psi,
// dispersive-cell states, incident line, clock) set aside.  fdtd_backward
// walks the segments from the last: a recorded segment goes straight into
// its transposed steps; an earlier one first restores its checkpoint and
// recomputes its steps with DFT sampling off while the dispersive-cell
// kernels record, into the rows the later segments no longer need.

struct fdtd_sim::Adjoint {
  std::vector<std::unique_ptr<DevBuf>> bufs;
  // checkpoints
  std::vector<std::pair<void*, size_t>> ck_bufs;  // state buffers that are checkpointed
  size_t ck_bytes = 0;
  std::unique_ptr<DevBuf> ck;  // nseg * ck_bytes
  int every = 0, nseg = 0, tend = 0;
  // trajectory record: rows = nrec * every, the last nrec segments recorded
  // by the forward (their first step rec_base), the others recomputed
  int nrec = 0, rows = 0, rec_base = 0;
  size_t rec_bytes = 0;
  // graphs of the two launch periods of the recording forward (the main
  // step graphs do not record), with the generation of the main graphs they
  // match
  cudaGraphExec_t g_fwd[2] = {nullptr, nullptr};
  long long g_fwd_kernels[2] = {0, 0};
  int g_fwd_len = 0, g_fwd_epoch = -1;
  // objective: weights on the ScatAbs table (fdtd_forward's own, for
  // fdtd_backward), the frequencies with a nonzero weight and the faces the
  // objective reads (bit b*6+f)
  std::vector<double> G;
  std::vector<int> sel;
  unsigned face_mask = 0;
  double objective = 0;
  bool forward_done = false, has_objective = false;
  std::unique_ptr<DevBuf> P, fsel;  // weighted partner accumulators; face weights, frequencies
  bool obj_is_G = false;  // the partner accumulators are those of G
  struct ObjSig {
    int nsel = -1;
    unsigned mask = 0;
    const void* P = nullptr;
    const void* fsel = nullptr;
    bool operator==(const ObjSig& o) const { return nsel == o.nsel && mask == o.mask && P == o.P && fsel == o.fsel; }
  } sig;
  // adjoint state (allocated on the first backward)
  bool ready = false;
  void* view = nullptr;  // AdjView<T> on the host, as bytes
  std::vector<char> view_bytes;
  std::vector<std::pair<void*, size_t>> zero;  // buffers zeroed before each sweep
  void* rec = nullptr;
  void* hrec = nullptr;  // hydrodynamic cells' record (MetalView::hrec)
  long long rec_slots = 0;
  int rec_off[3] = {0, 0, 0};
  double* grho[3] = {nullptr, nullptr, nullptr};
  double* gpar = nullptr;
  int* step = nullptr;
  // gather tables per gather (0 = H, 1 = E): the staged tiles and the
  // one-plane blocks of the other tiles, which the fused gathers take
  std::unique_ptr<DevBuf> gtab[2][2];
  int ngt[2][2] = {{0, 0}, {0, 0}};
  bool tabs = false;
  // graphs of one full segment: the recompute (DFT off, recording on) and
  // the reverse sweep; replayed for every full segment
  cudaGraphExec_t g_rec = nullptr, g_adj = nullptr;
  cudaStream_t cap = nullptr;

  void drop_graphs() {
    if (g_rec) cudaGraphExecDestroy(g_rec);
    if (g_adj) cudaGraphExecDestroy(g_adj);
    for (auto& g : g_fwd)
      if (g) cudaGraphExecDestroy(g);
    g_rec = g_adj = g_fwd[0] = g_fwd[1] = nullptr;
  }
  ~Adjoint() {
    drop_graphs();
    if (cap) cudaStreamDestroy(cap);
  }

  template <typename U>
  cudaError_t alloc(U** out, size_t count, bool zeroed_each_sweep) {
    auto b = std::make_unique<DevBuf>();
    cudaError_t e = b->alloc(count * sizeof(U));
    if (e != cudaSuccess) return e;
    *out = b->as<U>();
    if (zeroed_each_sweep) zero.emplace_back(b->p, b->bytes);
    bufs.push_back(std::move(b));
    return cudaSuccess;
  }
};

fdtd_sim::~fdtd_sim() { destroy_streams(); }

extern "C" fdtd_status fdtd_set_design(fdtd_sim* s, const int box[6], const float* rho, size_t count) {
  if (!s || !box || !rho) return fail(FDTD_ERR_INVALID, "null argument");
  if (!s->has_design) return fail(FDTD_ERR_STATE, "the simulation was created without params.design_box");
  for (int a = 0; a < 6; a++)
    if (box[a] != s->dbox[a]) return fail(FDTD_ERR_INVALID, "box differs from params.design_box");
  const size_t nb = s->dslot[0].size();
  if (count != nb) return fail(FDTD_ERR_INVALID, "count must be the design box's cell count");
  for (size_t q = 0; q < nb; q++)
    if (!(rho[q] >= 0.0f && rho[q] <= 1.0f)) return fail(FDTD_ERR_INVALID, "rho must lie in [0, 1]");
  CUDA_TRY(cudaSetDevice(s->device));
  CUDA_TRY(cudaDeviceSynchronize());
  for (int c = 0; c < 3; c++) {
    if (!s->rho_d[c]) continue;
    std::vector<float> h(s->nmetal[c], 1.0f);
    for (size_t q = 0; q < nb; q++)
      if (s->dslot[c][q] >= 0) h[s->dslot[c][q]] = rho[q];
    CUDA_TRY(cudaMemcpy(s->rho_d[c], h.data(), h.size() * sizeof(float), cudaMemcpyHostToDevice));
  }
  if (s->adj) s->adj->forward_done = false;
  return FDTD_OK;
}

static fdtd_status adj_checks(fdtd_sim* s) {
  if (!s->has_design) return fail(FDTD_ERR_STATE, "the simulation was created without params.design_box");
  if (s->pml_metal) return fail(FDTD_ERR_UNSUPPORTED, "the adjoint needs every dispersive cell outside the CPML");
  if (!s->dft_on || s->line.dft_every <= 0) return fail(FDTD_ERR_STATE, "the objective needs the DFT (StaticField = 0)");
  return FDTD_OK;
}

template <typename T>
static fdtd_status adj_prepare(fdtd_sim* s);

static void adj_stats(const fdtd_sim* s, fdtd_stats* out) {
  out->adj_record_steps = out->adj_record_bytes = out->adj_checkpoints = 0;
  if (!s->adj || !s->adj->forward_done) return;
  const fdtd_sim::Adjoint& A = *s->adj;
  out->adj_record_steps = A.tend + 1 - A.rec_base;
  out->adj_record_bytes = (long long)A.rec_bytes;
  out->adj_checkpoints = A.nseg - A.nrec;
}

// The record rows of the forward: nrec segments, as many as the budget
// holds (FDTD_ADJ_RECORD_GB, else 60% of the device's memory and all but 4
// GB of what is free), at least one.  Reallocated only when the depth
// changes; the graphs hold the record's address.
template <typename T>
static fdtd_status adj_record_alloc(fdtd_sim* s) {
  fdtd_sim::Adjoint& A = *s->adj;
  const size_t per_row = (size_t)A.rec_slots * (5 + (s->su.hydro ? 6 : 0)) * sizeof(T);
  const size_t per_seg = per_row * (size_t)A.every;
  size_t free_b = 0, total_b = 0;
  CUDA_TRY(cudaMemGetInfo(&free_b, &total_b));
  const size_t avail = free_b + A.rec_bytes;  // the current record is given back
  const size_t reserve = (size_t)4 << 30;
  double budget = std::min(0.6 * (double)total_b, avail > reserve ? (double)(avail - reserve) : 0.0);
  if (const char* e = std::getenv("FDTD_ADJ_RECORD_GB")) budget = std::min(budget, std::atof(e) * (double)(1ull << 30));
  const int nrec = std::max(1, std::min(A.nseg, (int)(budget / (double)std::max<size_t>(per_seg, 1))));
  if (nrec == A.nrec && A.rec) return FDTD_OK;
  A.drop_graphs();
  for (auto it = A.bufs.begin(); it != A.bufs.end();) {
    if ((*it)->p == A.rec || (A.hrec && (*it)->p == A.hrec)) it = A.bufs.erase(it);
    else ++it;
  }
  A.rec = nullptr;
  A.hrec = nullptr;
  A.rec_bytes = 0;
  A.nrec = nrec;
  A.rows = nrec * A.every;
  T* rec;
  CUDA_TRY(A.alloc(&rec, (size_t)A.rows * 5 * A.rec_slots, false));
  A.rec = rec;
  A.rec_bytes = (size_t)A.rows * 5 * A.rec_slots * sizeof(T);
  if (s->su.hydro) {
    T* hr;
    CUDA_TRY(A.alloc(&hr, (size_t)A.rows * 6 * A.rec_slots, false));
    A.hrec = hr;
    A.rec_bytes += (size_t)A.rows * 6 * A.rec_slots * sizeof(T);
  }
  return FDTD_OK;
}

// Points the dispersive-cell kernels at the record (or off, rec == nullptr).
template <typename T>
static void adj_record_view(fdtd_sim* s, bool on) {
  fdtd_sim::Adjoint& A = *s->adj;
  MetalView<T>& m = mview<T>(s);
  m.rec = on ? static_cast<T*>(A.rec) : nullptr;
  m.hrec = on ? static_cast<T*>(A.hrec) : nullptr;
  m.rec_rows = A.rows;
  m.rec_base = A.rec_base;
  m.rec_slots = A.rec_slots;
  for (int c = 0; c < 3; c++) m.rec_off[c] = A.rec_off[c];
}

// The forward: every field, auxiliary state and accumulator zeroed, then
// the whole time loop t = 0..Tend in segments of checkpoint_every steps,
// with a copy of the state (without the DFT accumulators, the sample ring
// and the probe record) at the start of every segment that is not
// recorded.  The DFT accumulators of the run stay in place for the
// objective.
template <typename T>
static fdtd_status adj_forward_run_t(fdtd_sim* s, int checkpoint_every) {
  fdtd_sim::Adjoint& A = *s->adj;
  A.forward_done = false;
  A.has_objective = false;
  if (A.every != checkpoint_every) {
    A.drop_graphs();  // they hold the segment length
    A.ready = false;  // the record depth follows the segment
    A.nrec = 0;
  }
  fdtd_status st = fdtd_reset(s);
  if (st != FDTD_OK) return st;
  CUDA_TRY(cudaSetDevice(s->device));
  A.ck_bufs.clear();
  A.ck_bytes = 0;
  const void* skip[4] = {s->dft.acc_re, s->dft.acc_im, s->ring, s->probe};
  for (const auto& b : s->state) {
    bool keep = true;
    for (const void* k : skip) keep = keep && b.first != k;
    if (keep) { A.ck_bufs.push_back(b); A.ck_bytes += (b.second + 255) / 256 * 256; }
  }
  A.every = checkpoint_every;
  A.tend = s->su.p.Tend;
  const int total = A.tend + 1;
  A.nseg = (total + A.every - 1) / A.every;
  if (!A.ready) {
    st = adj_prepare<T>(s);
    if (st != FDTD_OK) return st;
  }
  st = adj_record_alloc<T>(s);
  if (st != FDTD_OK) return st;
  const int nck = A.nseg - A.nrec;  // segments that are recomputed
  A.rec_base = nck * A.every;
  const size_t need = (size_t)nck * A.ck_bytes;
  if (need > 0 && (!A.ck || A.ck->bytes < need)) {
    A.ck.reset();
    auto b = std::make_unique<DevBuf>();
    CUDA_TRY(b->alloc(need));
    A.ck = std::move(b);
  }
  for (int seg = 0; seg < nck; seg++) {
    char* dst = static_cast<char*>(A.ck->p) + (size_t)seg * A.ck_bytes;
    for (const auto& b : A.ck_bufs) {
      CUDA_TRY(cudaMemcpyAsync(dst, b.first, b.second, cudaMemcpyDeviceToDevice, 0));
      dst += (b.second + 255) / 256 * 256;
    }
    st = fdtd_step(s, A.every, nullptr);
    if (st != FDTD_OK) return st;
  }
  // the recorded segments, with their own step graph
  if (A.g_fwd_epoch != s->graph_epoch)
    for (auto& g : A.g_fwd)
      if (g) {
        cudaGraphExecDestroy(g);
        g = nullptr;
      }
  adj_record_view<T>(s, true);
  auto swap_graphs = [&]() {
    for (int q = 0; q < 2; q++) {
      std::swap(s->graph[q], A.g_fwd[q]);
      std::swap(s->graph_kernels_p[q], A.g_fwd_kernels[q]);
    }
    std::swap(s->graph_len, A.g_fwd_len);
  };
  swap_graphs();
  st = fdtd_step(s, total - A.rec_base, nullptr);
  swap_graphs();
  A.g_fwd_epoch = s->graph_epoch;
  adj_record_view<T>(s, false);
  if (st != FDTD_OK) return st;
  CUDA_TRY(cudaDeviceSynchronize());
  A.forward_done = true;
  return FDTD_OK;
}
static fdtd_status adj_forward_run(fdtd_sim* s, int checkpoint_every) {
  if (!s->adj) s->adj = std::make_unique<fdtd_sim::Adjoint>();
  return s->fp64 ? adj_forward_run_t<double>(s, checkpoint_every) : adj_forward_run_t<float>(s, checkpoint_every);
}

// The objective L = sum_m sum_c G[m][c] spectra[m][c] over the ScatAbs
// table of fdtd_spectral_finalize.  Its columns are linear in the 12 face
// fluxes Q_f(m) (flux_reduce) scaled by dxy / |E_inc(m)|^2:
//   faces   col 4 + f = q_sca,f, col 10 + f = q_abs,f
//   totals  col 1 = sum_f s_f q_sca,f (/ pi r^2 for the reference's
//           sphere), col 2 = sum_f s_f q_abs,f (x -1 / pi r^2 for the
//           sphere), col 3 = col 1 + col 2, with s_f = -1, +1 for the -, +
//           face of each axis (Spectral.cu:1145-1168),
// so dL/dQ_f(m) follows from G by the chain rule.  Frequencies whose
// weights are all zero are dropped; the partner accumulators of the rest
// are built for the reverse sweep.
static fdtd_status adj_objective(fdtd_sim* s, const double* G) {
  fdtd_sim::Adjoint& A = *s->adj;
  const int nf = s->dft.nf;
  const Setup& su = s->su;
  for (int m = 0; m < nf; m++) {
    const double* g = G + (size_t)m * 19;
    if (g[0] != 0.0 || g[16] != 0.0 || g[17] != 0.0 || g[18] != 0.0)
      return fail(FDTD_ERR_INVALID, "dL_dspectra: columns 0 and 16-18 (wavelength, incident field) must be zero");
    for (int c = 1; c < 16; c++)
      if (!std::isfinite(g[c])) return fail(FDTD_ERR_INVALID, "dL_dspectra holds a non-finite value");
  }
  const bool sphere = su.p.geometry == FDTD_GEOM_REFERENCE && su.p.nano_sphere == 1;
  const double area = sphere ? su.pi * su.p.nano_sphere_radius * su.p.nano_sphere_radius : 1.0;
  const double sca_scale = sphere ? 1.0 / area : 1.0, abs_scale = sphere ? -1.0 / area : 1.0;
  const double dxy = su.p.dx * su.p.dy;
  A.sel.clear();
  std::vector<double> wface, fs;
  unsigned mask = 0;
  for (int m = 0; m < nf; m++) {
    const double* g = G + (size_t)m * 19;
    const double amp = std::abs(su.Einc[m]);
    const double w = dxy / (amp * amp);
    double k[12];
    bool any = false;
    for (int b = 0; b < 2; b++)
      for (int f = 0; f < 6; f++) {
        const double sf = (f & 1) ? 1.0 : -1.0;
        const double v = b == 1 ? g[4 + f] + sf * (g[1] + g[3]) * sca_scale
                                : g[10 + f] + sf * (g[2] + g[3]) * abs_scale;
        k[b * 6 + f] = w * v;
        if (v != 0.0) { any = true; mask |= 1u << (b * 6 + f); }
      }
    if (!any) continue;
    A.sel.push_back(m);
    wface.insert(wface.end(), k, k + 12);
    fs.push_back(su.freq[m]);
  }
  const int nsel = (int)A.sel.size();
  A.face_mask = mask;
  A.has_objective = true;
  if (nsel == 0) return FDTD_OK;
  // partner accumulators and the frequency list, kept across calls (an
  // allocation per call would synchronise the device)
  const size_t pbytes = (size_t)nsel * s->dft.rows * sizeof(double2);
  const size_t fbytes = (size_t)nsel * (13 * sizeof(double) + sizeof(int));
  if (!A.P || A.P->bytes < pbytes) {
    A.P.reset();
    auto b = std::make_unique<DevBuf>();
    CUDA_TRY(b->alloc(pbytes));
    A.P = std::move(b);
  }
  if (!A.fsel || A.fsel->bytes < fbytes) {
    A.fsel.reset();
    auto b = std::make_unique<DevBuf>();
    CUDA_TRY(b->alloc(fbytes));
    A.fsel = std::move(b);
  }
  double* dw = static_cast<double*>(A.fsel->p);
  double* dfs = dw + (size_t)nsel * 12;
  int* dsel = reinterpret_cast<int*>(dfs + nsel);
  CUDA_TRY(cudaMemcpy(dw, wface.data(), wface.size() * sizeof(double), cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMemcpy(dfs, fs.data(), nsel * sizeof(double), cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMemcpy(dsel, A.sel.data(), nsel * sizeof(int), cudaMemcpyHostToDevice));
  int maxn = 0;
  for (int f = 0; f < 12; f++) maxn = std::max(maxn, s->dft.face[f].na * s->dft.face[f].nb);
  adj_partner<<<dim3((maxn + 255) / 256, 12, nsel), 256>>>(s->dft, dsel, dw, nsel, static_cast<double2*>(A.P->p),
                                                           s->dft.rows);
  // the reverse-sweep graph holds the selection's size, face mask and
  // buffers (their contents are read at replay)
  const fdtd_sim::Adjoint::ObjSig sig{nsel, mask, A.P->p, A.fsel->p};
  if (!(sig == A.sig)) A.drop_graphs();
  A.sig = sig;
  CUDA_TRY(cudaGetLastError());
  CUDA_TRY(cudaDeviceSynchronize());
  return FDTD_OK;
}

extern "C" fdtd_status fdtd_forward_spectra(fdtd_sim* s, int checkpoint_every, double* out19) {
  if (!s || checkpoint_every <= 0) return fail(FDTD_ERR_INVALID, "bad argument");
  fdtd_status st = adj_checks(s);
  if (st != FDTD_OK) return st;
  st = adj_forward_run(s, checkpoint_every);
  if (st != FDTD_OK) return st;
  s->adj->G.clear();  // no objective of its own: fdtd_backward_spectra supplies one
  if (out19) return fdtd_spectral_finalize(s, out19);
  return FDTD_OK;
}

extern "C" fdtd_status fdtd_forward(fdtd_sim* s, const int* freq_idx, int nfreq, int checkpoint_every,
                                    double* objective) {
  if (!s || !freq_idx || nfreq <= 0 || checkpoint_every <= 0 || !objective)
    return fail(FDTD_ERR_INVALID, "bad argument");
  fdtd_status st = adj_checks(s);
  if (st != FDTD_OK) return st;
  const int nf = s->dft.nf;
  for (int m = 0; m < nfreq; m++)
    if (freq_idx[m] < 0 || freq_idx[m] >= nf) return fail(FDTD_ERR_INVALID, "frequency index out of range");
  st = adj_forward_run(s, checkpoint_every);
  if (st != FDTD_OK) return st;
  std::vector<double> rows((size_t)nf * 19);
  st = fdtd_spectral_finalize(s, rows.data());
  if (st != FDTD_OK) return st;
  // absorption cross-section sigma_abs(m) = P_abs / I_inc: the net inward
  // flux through the absorption box, -sum_f s_f q_abs,f (positive for an
  // absorbing structure whatever the geometry)
  fdtd_sim::Adjoint& A = *s->adj;
  A.G.assign((size_t)nf * 19, 0.0);
  double L = 0;
  for (int q = 0; q < nfreq; q++) {
    const int m = freq_idx[q];
    for (int f = 0; f < 6; f++) {
      const double w = (f & 1) ? -1.0 : 1.0;
      A.G[(size_t)m * 19 + 10 + f] += w;
      L += w * rows[(size_t)m * 19 + 10 + f];
    }
  }
  A.objective = L;
  *objective = L;
  st = adj_objective(s, A.G.data());
  A.obj_is_G = st == FDTD_OK;
  return st;
}

template <typename T>
static fdtd_status adj_prepare(fdtd_sim* s) {
  fdtd_sim::Adjoint& A = *s->adj;
  A.drop_graphs();  // they hold the buffers released here
  A.bufs.clear();  // a re-preparation (another checkpoint interval) starts afresh
  A.zero.clear();
  A.rec = nullptr;  // the record goes with them (adj_record_alloc makes it again)
  A.hrec = nullptr;
  A.rec_bytes = 0;
  A.nrec = 0;
  AdjView<T> a;
  std::memset(&a, 0, sizeof(a));
  const size_t nc = s->ncell;
  for (int c = 0; c < 3; c++) {
    CUDA_TRY(A.alloc(&a.lE[c], nc, true));
    CUDA_TRY(A.alloc(&a.lH[c], nc, true));
    for (int q = 0; q < 2; q++) CUDA_TRY(A.alloc(&a.a[c][q], nc, false));
  }
  // psi adjoints, the shapes of the psi slabs
  const Setup& su = s->su;
  for (int c = 0; c < 3; c++)
    for (int slot = 0; slot < 2; slot++) {
      const int ax = (c + 1 + slot) % 3;
      const int Nc = su.Nc[ax];
      size_t ce, ch;
      if (ax == 2) { ce = (size_t)(Nc + 1) * s->plane; ch = (size_t)Nc * s->plane; }
      else if (ax == 1) { ce = (size_t)s->NZ * (Nc + 1) * s->PX; ch = (size_t)s->NZ * Nc * s->PX; }
      else { ce = (size_t)s->NZ * s->NY * (Nc + 1); ch = (size_t)s->NZ * s->NY * Nc; }
      CUDA_TRY(A.alloc(&a.lpE_N[c][slot], ce, true));
      CUDA_TRY(A.alloc(&a.lpE_F[c][slot], ce, true));
      CUDA_TRY(A.alloc(&a.lpH_N[c][slot], ch, true));
      CUDA_TRY(A.alloc(&a.lpH_F[c][slot], ch, true));
    }
  long long slots = 0;
  for (int c = 0; c < 3; c++) {
    const size_t n = std::max(1, s->nmetal[c]);
    CUDA_TRY(A.alloc(&a.lJa[c], n, true));
    CUDA_TRY(A.alloc(&a.lJb[c], n, true));
    CUDA_TRY(A.alloc(&a.lEh[c], n, true));
    for (int q = 0; q < 2; q++) {
      CUDA_TRY(A.alloc(&a.lPa[c][q], n, true));
      CUDA_TRY(A.alloc(&a.lPb[c][q], n, true));
    }
    CUDA_TRY(A.alloc(&a.grho[c], n, true));
    A.grho[c] = a.grho[c];
    A.rec_off[c] = (int)slots;
    slots += s->nmetal[c];
  }
  if (su.hydro) {
    for (int c = 0; c < 3; c++)
      for (int r = 0; r < 3; r++) {
        CUDA_TRY(A.alloc(&a.lJ[c][r], std::max(1, s->nmetal[c]), true));
        CUDA_TRY(A.alloc(&a.lN[c][r], std::max(1, s->nmetal[c]), true));
      }
  }
  CUDA_TRY(A.alloc(&a.gpar, 2, true));
  A.gpar = a.gpar;
  CUDA_TRY(A.alloc(&a.step, 1, false));
  CUDA_TRY(A.alloc(&a.flags, s->ncell, false));
  A.step = a.step;
  A.rec_slots = std::max(1LL, slots);  // the record itself: adj_record_alloc
  // derivatives of the metal's coupling and dynamics coefficients with
  // respect to omega_D and gamma (ade_coefficients, non-hydrodynamic form)
  const double dt = su.dt, wD = su.wD, gam = su.gam;
  const double dd = 1.0 / (dt * dt) + gam / (2.0 * dt), g1 = 1.0 / (2.0 * dt);
  const double dd3[2] = {2.0 * su.d3 / wD, -su.d3 * g1 / dd};
  const double dd4[2] = {2.0 * su.d4 / wD, -su.d4 * g1 / dd};
  const double dd5[2] = {2.0 * su.d5 / wD, -su.d5 * g1 / dd};
  const double dd1[2] = {0.0, -su.d1 * g1 / dd};
  const double dd2[2] = {0.0, g1 * (1.0 - su.d2) / dd};
  for (int p = 0; p < 2; p++) {
    a.dd1[p] = (T)dd1[p]; a.dd2[p] = (T)dd2[p];
    a.dd3[p] = (T)dd3[p]; a.dd4[p] = (T)dd4[p]; a.dd5[p] = (T)dd5[p];
    a.dCE[p] = (T)dd3[p]; a.dCE1[p] = (T)(-dd4[p]); a.dCE2[p] = (T)dd5[p];
  }
  // hydrodynamic model: gamma enters d1..d4 and dNL through dd (omega_D does
  // not enter; the equilibrium density N_EQ is its own constant)
  a.dgam[0] = -su.d1 * g1 / dd;
  a.dgam[1] = g1 * (1.0 - su.d2) / dd;
  a.dgam[2] = -su.d3 * g1 / dd;
  a.dgam[3] = -su.d4 * g1 / dd;
  a.dgam[4] = -su.dNL * g1 / dd;
  A.view_bytes.assign(reinterpret_cast<const char*>(&a), reinterpret_cast<const char*>(&a) + sizeof(a));
  A.ready = true;
  return FDTD_OK;
}

template <typename T>
static fdtd_status adj_sweep(fdtd_sim* s) {
  fdtd_sim::Adjoint& A = *s->adj;
  const AdjView<T>& a = *reinterpret_cast<const AdjView<T>*>(A.view_bytes.data());
  for (const auto& z : A.zero) CUDA_TRY(cudaMemset(z.first, 0, z.second));
  MetalView<T>& m = mview<T>(s);
  adj_record_view<T>(s, true);
  const int every_dft = s->line.dft_every;
  const bool graphs = s->use_graphs, snaps = s->snap_on;
  s->line.dft_every = 0;  // the recompute needs no DFT samples
  s->snap_on = false;     // nor snapshots
  s->use_graphs = false;
  const long long ncell = (long long)s->NX * s->NY * s->NZ;
  const unsigned gc = (unsigned)((ncell + 255) / 256);
  const int ntot = s->nmetal[0] + s->nmetal[1] + s->nmetal[2];
  int maxn = 0;
  for (int f = 0; f < 12; f++) maxn = std::max(maxn, s->dft.face[f].na * s->dft.face[f].nb);
  const int nsel = (int)A.sel.size();
  const double* fsel = static_cast<const double*>(A.fsel->p) + (size_t)nsel * 12;
  const int total = A.tend + 1;
  // fused gathers (the default; FDTD_ADJ_FUSED=0 selects the coefficient
  // arrays everywhere) need chh == 1
  const char* fenv = std::getenv("FDTD_ADJ_FUSED");
  bool fused = s->su.Chh == 1.0 && !(fenv && fenv[0] == '0');
  SlabShell she, shh;
  {
    const int n3[3] = {s->NX, s->NY, s->NZ};
    int lo_e[3], lo_h[3], hi[3];
    for (int ax = 0; ax < 3; ax++) {
      lo_e[ax] = s->su.Nc[ax] + 1;
      lo_h[ax] = s->su.Nc[ax];
      hi[ax] = s->su.F[ax];
    }
    she.init(n3, lo_e, hi);
    shh.init(n3, lo_h, hi);
    if (she.total() >= (1LL << 32) || shh.total() >= (1LL << 32)) fused = false;  // 32-bit shell indices
  }
  const dim3 gtile((unsigned)((s->NX + 31) / 32), (unsigned)((s->NY + 7) / 8), (unsigned)s->NZ);
  if (fused) adj_build_flags<T><<<gtile, dim3(32, 8)>>>(view<T>(s), a.flags);
  // staged tiles: 32 x kAdjTY x kAdjKC boxes whose cells and halo (+1 for
  // the H gather, -1 for the E gather) lie away from the CPML slabs, the
  // grid's faces and the material box; the other tiles go to the fused
  // gathers, one plane per block.  A tile keeps a CTA on 16 planes: on a
  // small grid too few of them would run (fewer than 4 a multiprocessor),
  // and the fused gathers win there; FDTD_ADJ_STAGED=1 / 0 forces either.
  const char* senv = std::getenv("FDTD_ADJ_STAGED");
  int nsm = 148;
  CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, s->device));
  const long long ntiles =
      (long long)((s->NX + 31) / 32) * ((s->NY + 7) / 8) * ((s->NZ + kAdjKC - 1) / kAdjKC);
  const bool staged = fused && (senv ? senv[0] != '0' : ntiles >= 4LL * nsm);
  if (staged && !A.tabs) {
    static_assert(kAdjTY == 8, "the staged tiles and the fused gathers' blocks share the 32 x 8 xy grid");
    const int nbx = (s->NX + 31) / 32, nby = (s->NY + 7) / 8, nbz = (s->NZ + kAdjKC - 1) / kAdjKC;
    for (int g = 0; g < 2; g++) {
      const int lo_off = g == 0 ? 0 : -1, hi_off = g == 0 ? 1 : 0;
      std::vector<int4> v[2];
      for (int bz = 0; bz < nbz; bz++)
        for (int by = 0; by < nby; by++)
          for (int bx = 0; bx < nbx; bx++) {
            const int lo[3] = {bx * 32 + lo_off, by * 8 + lo_off, bz * kAdjKC + lo_off};
            const int hi[3] = {bx * 32 + 31 + hi_off, by * 8 + 7 + hi_off,
                               std::min(s->NZ, (bz + 1) * kAdjKC) - 1 + hi_off};
            bool inside = true, off_mat = false;
            for (int ax = 0; ax < 3; ax++) {
              inside = inside && lo[ax] >= s->su.Nc[ax] + 1 && hi[ax] < s->su.F[ax];
              off_mat = off_mat || hi[ax] < s->mat_lo[ax] || lo[ax] >= s->mat_hi[ax];
            }
            if (inside && off_mat) {
              v[0].push_back(make_int4(bx, by, bz, 0));
            } else {
              for (int k = bz * kAdjKC; k < std::min(s->NZ, (bz + 1) * kAdjKC); k++) v[1].push_back(make_int4(bx, by, k, 0));
            }
          }
      for (int q = 0; q < 2; q++) {
        auto b = std::make_unique<DevBuf>();
        CUDA_TRY(b->alloc(std::max<size_t>(1, v[q].size()) * sizeof(int4)));
        if (!v[q].empty()) CUDA_TRY(cudaMemcpy(b->p, v[q].data(), v[q].size() * sizeof(int4), cudaMemcpyHostToDevice));
        A.gtab[g][q] = std::move(b);
        A.ngt[g][q] = (int)v[q].size();
      }
    }
    const int smem = (int)(kAdjS * StageLayout<T, kAdjTY>::STAGE * sizeof(T));
    CUDA_TRY(cudaFuncSetAttribute(adj_gather_h_staged<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    CUDA_TRY(cudaFuncSetAttribute(adj_gather_e_staged<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    A.tabs = true;
  }
  const size_t gsmem = kAdjS * StageLayout<T, kAdjTY>::STAGE * sizeof(T);
  // one gather: the staged tiles and the fused blocks (disjoint outputs,
  // inputs they do not write); returns the launches
  auto gather = [&](int g, cudaStream_t stream) -> int {
    if (!staged) {
      if (g == 0) adj_gather_h_fused<T><<<gtile, dim3(32, 8), 0, stream>>>(view<T>(s), a, nullptr);
      else adj_gather_e_fused<T><<<gtile, dim3(32, 8), 0, stream>>>(view<T>(s), a, nullptr);
      return 1;
    }
    int k = 0;
    const int4* tt = static_cast<const int4*>(A.gtab[g][0]->p);
    const int4* lt = static_cast<const int4*>(A.gtab[g][1]->p);
    const int* n = A.ngt[g];
    if (n[1]) {
      if (g == 0) adj_gather_h_fused<T><<<n[1], dim3(32, 8), 0, stream>>>(view<T>(s), a, lt);
      else adj_gather_e_fused<T><<<n[1], dim3(32, 8), 0, stream>>>(view<T>(s), a, lt);
      k++;
    }
    if (n[0]) {
      if (g == 0) adj_gather_h_staged<T><<<n[0], dim3(32, kAdjTY), gsmem, stream>>>(view<T>(s), a, tt);
      else adj_gather_e_staged<T><<<n[0], dim3(32, kAdjTY), gsmem, stream>>>(view<T>(s), a, tt);
      k++;
    }
    return k;
  };
  // the dispersive cells' transposed update: the local model in one
  // launch; the hydrodynamic model as its three phases in reverse order,
  // then the current update
  const bool hydro = s->su.hydro;
  auto launch_design = [&](cudaStream_t stream) -> int {
    if (!hydro) {
      adj_e_design<T><<<(ntot + 127) / 128, 128, 0, stream>>>(view<T>(s), m, a, static_cast<const T*>(A.rec), A.rows);
      return 1;
    }
    int k = 0;
    if (s->nmetal[2] > 0) { adj_hydro_e<T, 2><<<(s->nmetal[2] + 127) / 128, 128, 0, stream>>>(view<T>(s), m, a); k++; }
    if (s->nmetal[1] > 0) { adj_hydro_e<T, 1><<<(s->nmetal[1] + 127) / 128, 128, 0, stream>>>(view<T>(s), m, a); k++; }
    if (s->nmetal[0] > 0) { adj_hydro_e<T, 0><<<(s->nmetal[0] + 127) / 128, 128, 0, stream>>>(view<T>(s), m, a); k++; }
    adj_hydro_j<T><<<(ntot + 127) / 128, 128, 0, stream>>>(view<T>(s), m, a);
    return k + 1;
  };
  auto adj_step = [&](int n, cudaStream_t stream) {
    if (n % every_dft == 0)
      adj_source<T><<<dim3((maxn + 255) / 256, 12), 256, 0, stream>>>(view<T>(s), s->dft, a,
                                                                       static_cast<const double2*>(A.P->p), fsel,
                                                                       nsel, s->dft.rows, A.face_mask);
    if (fused) {
      if (she.total() > 0)
        adj_e_slab<T><<<(unsigned)((she.total() + 255) / 256), 256, 0, stream>>>(view<T>(s), a, she);
      const int kd = ntot > 0 ? launch_design(stream) : 0;
      const int kg = gather(0, stream);
      if (shh.total() > 0)
        adj_h_slab<T><<<(unsigned)((shh.total() + 255) / 256), 256, 0, stream>>>(view<T>(s), a, shh);
      const int kg2 = gather(1, stream);
      adj_step_back<<<1, 1, 0, stream>>>(A.step);
      return 1 + kg + kg2 + (she.total() > 0) + (shh.total() > 0) + kd + (n % every_dft == 0);
    }
    adj_e_coef<T><<<gc, 256, 0, stream>>>(view<T>(s), a);
    const int kd = ntot > 0 ? launch_design(stream) : 0;
    adj_gather_h<T><<<gc, 256, 0, stream>>>(view<T>(s), a);
    adj_h_coef<T><<<gc, 256, 0, stream>>>(view<T>(s), a);
    adj_gather_e<T><<<gc, 256, 0, stream>>>(view<T>(s), a);
    adj_step_back<<<1, 1, 0, stream>>>(A.step);
    return 5 + kd + (n % every_dft == 0);
  };
  if (!A.cap) CUDA_TRY(cudaStreamCreateWithFlags(&A.cap, cudaStreamNonBlocking));
  fdtd_status st = FDTD_OK;
  for (int seg = A.nseg - 1; seg >= 0 && st == FDTD_OK; seg--) {
    const int n0 = seg * A.every, n1 = std::min(total, n0 + A.every);
    const bool full = n1 - n0 == A.every;
    // a segment the forward recorded goes straight into its reverse sweep;
    // an earlier one restores its checkpoint and recomputes, recording into
    // the rows of the segments already swept
    const bool recorded = seg >= A.nseg - A.nrec;
    if (!recorded) {
      const char* src = static_cast<const char*>(A.ck->p) + (size_t)seg * A.ck_bytes;
      for (const auto& b : A.ck_bufs) {
        CUDA_TRY(cudaMemcpyAsync(b.first, src, b.second, cudaMemcpyDeviceToDevice, 0));
        src += (b.second + 255) / 256 * 256;
      }
      s->t = n0;
      s->host_nsamp = 0;
    }
    if (recorded) {
      // nothing to recompute
    } else if (full) {
      if (!A.g_rec) {
        cudaGraph_t g;
        const long long k0 = s->kernels;
        CUDA_TRY(cudaStreamBeginCapture(A.cap, cudaStreamCaptureModeThreadLocal));
        for (int q = 0; q < A.every; q++) enqueue_step<T>(s, A.cap);
        CUDA_TRY(cudaStreamEndCapture(A.cap, &g));
        s->kernels = k0;
        s->t = n0;
        const cudaError_t e = cudaGraphInstantiate(&A.g_rec, g, 0);
        cudaGraphDestroy(g);
        CUDA_TRY(e);
      }
      CUDA_TRY(cudaGraphLaunch(A.g_rec, 0));
      s->t = n1;
    } else {
      st = step_impl<T>(s, n1 - n0, 0);
      if (st != FDTD_OK) break;
    }
    adj_set_step<<<1, 1>>>(A.step, n1 - 1);
    // the reverse sweep; a full segment starting on a DFT sample step has
    // the same launch pattern every time
    if (full && n0 % every_dft == 0) {
      if (!A.g_adj) {
        cudaGraph_t g;
        CUDA_TRY(cudaStreamBeginCapture(A.cap, cudaStreamCaptureModeThreadLocal));
        for (int n = n1 - 1; n >= n0; n--) adj_step(n, A.cap);
        CUDA_TRY(cudaStreamEndCapture(A.cap, &g));
        const cudaError_t e = cudaGraphInstantiate(&A.g_adj, g, 0);
        cudaGraphDestroy(g);
        CUDA_TRY(e);
      }
      CUDA_TRY(cudaGraphLaunch(A.g_adj, 0));
    } else {
      for (int n = n1 - 1; n >= n0; n--) s->kernels += adj_step(n, 0);
    }
    CUDA_TRY(cudaGetLastError());
  }
  m.rec = nullptr;
  m.hrec = nullptr;
  s->line.dft_every = every_dft;
  s->use_graphs = graphs;
  s->snap_on = snaps;
  CUDA_TRY(cudaDeviceSynchronize());
  return st;
}

static fdtd_status adj_backward(fdtd_sim* s, float* dL_drho, size_t count, double* dL_dparams) {
  if (dL_drho && count != s->dslot[0].size()) return fail(FDTD_ERR_INVALID, "count must be the design box's cell count");
  fdtd_sim::Adjoint& A = *s->adj;
  if (A.sel.empty()) {  // the objective reads no field: every gradient is zero
    if (dL_drho) std::fill(dL_drho, dL_drho + count, 0.0f);
    if (dL_dparams) dL_dparams[0] = dL_dparams[1] = 0.0;
    return FDTD_OK;
  }
  // the forward prepared the adjoint state and made the record
  if (!A.ready || !A.rec) return fail(FDTD_ERR_STATE, "the adjoint state is missing: run the forward again");
  fdtd_status st = s->fp64 ? adj_sweep<double>(s) : adj_sweep<float>(s);
  if (st != FDTD_OK) return st;
  if (dL_drho) {
    std::vector<double> g[3];
    for (int c = 0; c < 3; c++) {
      g[c].resize(std::max(1, s->nmetal[c]));
      CUDA_TRY(cudaMemcpy(g[c].data(), A.grho[c], g[c].size() * sizeof(double), cudaMemcpyDeviceToHost));
    }
    for (size_t q = 0; q < count; q++) {
      double v = 0;
      for (int c = 0; c < 3; c++)
        if (s->dslot[c][q] >= 0) v += g[c][s->dslot[c][q]];
      dL_drho[q] = (float)v;
    }
  }
  if (dL_dparams) CUDA_TRY(cudaMemcpy(dL_dparams, A.gpar, 2 * sizeof(double), cudaMemcpyDeviceToHost));
  return FDTD_OK;
}

extern "C" fdtd_status fdtd_backward(fdtd_sim* s, float* dL_drho, size_t count, double* dL_dparams) {
  if (!s) return fail(FDTD_ERR_INVALID, "null argument");
  fdtd_status st = adj_checks(s);
  if (st != FDTD_OK) return st;
  if (!s->adj || !s->adj->forward_done) return fail(FDTD_ERR_STATE, "fdtd_backward needs a completed fdtd_forward");
  if (s->adj->G.empty()) return fail(FDTD_ERR_STATE, "fdtd_backward needs the objective of fdtd_forward "
                                                     "(after fdtd_forward_spectra use fdtd_backward_spectra)");
  CUDA_TRY(cudaSetDevice(s->device));
  CUDA_TRY(cudaDeviceSynchronize());
  if (!s->adj->has_objective || !s->adj->obj_is_G) {
    st = adj_objective(s, s->adj->G.data());
    if (st != FDTD_OK) return st;
    s->adj->obj_is_G = true;
  }
  return adj_backward(s, dL_drho, count, dL_dparams);
}

extern "C" fdtd_status fdtd_backward_spectra(fdtd_sim* s, const double* dL_dspectra, float* dL_drho, size_t count,
                                             double* dL_dparams) {
  if (!s || !dL_dspectra) return fail(FDTD_ERR_INVALID, "null argument");
  fdtd_status st = adj_checks(s);
  if (st != FDTD_OK) return st;
  if (!s->adj || !s->adj->forward_done)
    return fail(FDTD_ERR_STATE, "fdtd_backward_spectra needs a completed fdtd_forward_spectra or fdtd_forward");
  CUDA_TRY(cudaSetDevice(s->device));
  CUDA_TRY(cudaDeviceSynchronize());
  s->adj->obj_is_G = false;
  st = adj_objective(s, dL_dspectra);
  if (st != FDTD_OK) return st;
  return adj_backward(s, dL_drho, count, dL_dparams);
}
