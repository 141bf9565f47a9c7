// Batched independent simulations (no counterpart in the reference: its
// trials loop, main.cu:2435, runs one simulation after another, and FP64
// builds allow one trial, main.cu:2386-2389).
//
// Every member is an ordinary fdtd_sim (its own fields, tables, DFT and
// clock); the batch adds, in device memory, one descriptor per member and
// one list of (member, tile) work items for the Yee passes.  A time step of
// the whole batch is
//   h_pass_batch      two persistent grids: the CPML-free tiles of all
//                     members from one queue, the CPML edge tiles from another
//   line_step         one launch, one CTA per member (double-buffered line E)
//   tfsf_apply        both TFSF halves, one launch, blockIdx.y = member
//   (hydrodynamic members: their three dispersive kernels, per member)
//   e_pass_batch      two persistent grids as for H
//   metal_e           one launch
//   dft_sample        one launch every dft_every steps, blockIdx.z = member
//   twiddles + contraction + reset, one launch each, every 32 samples
// so the launch count per step does not grow with the member count, and
// small members that could not fill the GPU alone share it.  Runs of
// 32 * dft_every steps are captured into one CUDA graph and replayed.
//
// This file is included at the end of fdtd.cu (it uses the simulation
// internals defined there).

namespace fdtd {

template <typename T>
struct BatchSim {
  SimView<T> v;
  MetalView<T> m;
  LineArgs line;
  DftView dft;
  ShellCells sh_h, sh_e;
  TfsfTable tf_h, tf_e;
  T* ring;
  double2* tw;
  DevClock* clk;
  size_t probe_id;
};

template <typename T>
__global__ void tfsf_apply_batch(const BatchSim<T>* __restrict__ b) {
  const BatchSim<T>& x = b[blockIdx.y];
  tfsf_apply_body(x.v, x.tf_h, x.tf_e, x.line);
}
template <typename T>
__global__ void __launch_bounds__(1024) line_step_batch(const BatchSim<T>* __restrict__ b) {
  const BatchSim<T>& x = b[blockIdx.y];
  line_step_body(x.line, x.v, x.probe_id);
}
template <typename T>
__global__ void metal_e_batch(const BatchSim<T>* __restrict__ b) {
  const BatchSim<T>& x = b[blockIdx.y];
  metal_e_body(x.v, x.m, x.clk);
}
template <typename T>
__global__ void dft_sample_batch(const BatchSim<T>* __restrict__ b) {
  const BatchSim<T>& x = b[blockIdx.z];
  dft_sample_body(x.v, x.dft, x.ring, x.clk);
}
template <typename T>
__global__ void dft_twiddles_batch(const BatchSim<T>* __restrict__ b) {
  const BatchSim<T>& x = b[blockIdx.y];
  dft_twiddles_body(x.dft, x.clk, x.tw, 0);
}
template <typename T>
__global__ void __launch_bounds__(128) dft_contract_batch(const BatchSim<T>* __restrict__ b) {
  const BatchSim<T>& x = b[blockIdx.y];
  dft_contract_body(x.dft, x.ring, x.clk, x.tw, 0);
}
// a flush before the spectra are read goes through the member's own
// contraction kernels (fdtd_spectral_finalize)
template <typename T>
__global__ void dft_reset_batch(const BatchSim<T>* __restrict__ b) {
  DevClock* clk = b[blockIdx.y].clk;
  if (dft_ring_ready(clk, 0)) clk->nsamp = 0;
}

}  // namespace fdtd

// The batch shares one pass launch shape: 32 x 4 tiles, 4-stage ring, six
// CTAs per SM, 16-plane z-chunks.
constexpr int kBatchTY = 4, kBatchS = 4, kBatchMinB = 6, kBatchKChunk = 16;

struct fdtd_batch {
  int device = 0;
  bool fp64 = false, hydro = false;
  std::vector<std::unique_ptr<fdtd_sim>> sims;
  std::vector<std::unique_ptr<DevBuf>> bufs;
  void* descs = nullptr;  // BatchSim<T>[n]
  void* views = nullptr;  // SimView<T>[n]
  int4* items = nullptr;  // (member, bx, by, bz)
  int* queue = nullptr;   // [4] work counters: H edge, H interior, E edge, E interior
  int nedge = 0, ninner = 0, grid_pass = 0, grid_inner = 0;
  unsigned g_f = 0, g_m = 0, g_s = 0, g_tw = 0, g_c = 0;
  int t = 0, host_nsamp = 0, dft_every = 0, tend = 0;
  long long kernels = 0, graph_launches = 0, graph_kernels = 0;
  cudaGraphExec_t graph = nullptr;
  cudaStream_t cap = nullptr;

  ~fdtd_batch() {
    if (graph) cudaGraphExecDestroy(graph);
    if (cap) cudaStreamDestroy(cap);
  }
  template <typename U>
  cudaError_t alloc(U** out, size_t count) {
    auto b = std::make_unique<DevBuf>();
    cudaError_t e = b->alloc(count * sizeof(U));
    if (e != cudaSuccess) return e;
    *out = static_cast<U*>(b->p);
    bufs.push_back(std::move(b));
    return cudaSuccess;
  }
};

template <typename T>
static fdtd_status batch_build(fdtd_batch* b) {
  const int n = (int)b->sims.size();
  std::vector<BatchSim<T>> d(n);
  std::vector<SimView<T>> v(n);
  std::vector<int4> items, inner;
  for (int i = 0; i < n; i++) {
    fdtd_sim* s = b->sims[i].get();
    BatchSim<T>& x = d[i];
    x.v = view<T>(s);
    x.m = mview<T>(s);
    x.line = s->line;
    x.dft = s->dft;
    x.sh_h = s->shell_h;
    x.sh_e = s->shell_e;
    x.tf_h = s->tf_h;
    x.tf_e = s->tf_e;
    x.ring = static_cast<T*>(s->ring);
    x.tw = s->twiddles;
    x.clk = s->clk;
    x.probe_id = s->probe_id;
    v[i] = x.v;
    const int nbx = (s->NX + 31) / 32, nby = (s->NY + kBatchTY - 1) / kBatchTY;
    const int nbz = (s->NZ + kBatchKChunk - 1) / kBatchKChunk;
    // tiles that touch no CPML slab go to the PML-free queue (the same
    // rule as build_tiles)
    const int nb3[3] = {nbx, nby, nbz}, w3[3] = {32, kBatchTY, kBatchKChunk};
    int lo[3], hi[3];
    for (int a = 0; a < 3; a++) {
      const int Nc = s->su.Nc[a], F = s->su.F[a];
      lo[a] = (Nc + 1 + w3[a] - 1) / w3[a];
      hi[a] = std::min(F >= w3[a] ? (F - w3[a]) / w3[a] + 1 : 0, nb3[a]);
    }
    for (int bz = 0; bz < nbz; bz++)
      for (int by = 0; by < nby; by++)
        for (int bx = 0; bx < nbx; bx++) {
          const bool in = bx >= lo[0] && bx < hi[0] && by >= lo[1] && by < hi[1] && bz >= lo[2] && bz < hi[2];
          (in ? inner : items).push_back(make_int4(i, bx, by, bz));
        }
    auto blocks = [](long long cells, int per) { return (unsigned)((cells + per - 1) / per); };
    b->g_f = std::max(b->g_f, blocks((long long)s->tf_h.n + s->tf_e.n, 256));
    b->g_m = std::max(b->g_m, blocks((long long)s->nmetal[0] + s->nmetal[1] + s->nmetal[2], 128));
    int maxn = 0;
    for (int f = 0; f < 12; f++) maxn = std::max(maxn, s->dft.face[f].na * s->dft.face[f].nb);
    b->g_s = std::max(b->g_s, blocks(maxn, 256));
    b->g_tw = std::max(b->g_tw, blocks(2LL * kRingSlots * s->dft.nf, 256));
    b->g_c = std::max(b->g_c, (unsigned)(s->dft.rows / kDftRows));
  }
  BatchSim<T>* dd;
  SimView<T>* dv;
  CUDA_TRY(b->alloc(&dd, n));
  CUDA_TRY(b->alloc(&dv, n));
  b->nedge = (int)items.size();
  b->ninner = (int)inner.size();
  items.insert(items.end(), inner.begin(), inner.end());  // edge items first, then interior
  CUDA_TRY(b->alloc(&b->items, items.size()));
  CUDA_TRY(b->alloc(&b->queue, 4));
  CUDA_TRY(cudaMemcpy(dd, d.data(), n * sizeof(BatchSim<T>), cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMemcpy(dv, v.data(), n * sizeof(SimView<T>), cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMemcpy(b->items, items.data(), items.size() * sizeof(int4), cudaMemcpyHostToDevice));
  b->descs = dd;
  b->views = dv;

  // persistent grids: every CTA slot of the GPU once
  const size_t smem = staged_smem<T, kBatchTY, kBatchS>();
  int sms = 0;
  CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device));
  auto slots = [&](auto kern, int& out) -> fdtd_status {
    CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per = 0;
    CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, 32 * kBatchTY, smem));
    out = std::max(out, std::max(1, per) * sms);
    return FDTD_OK;
  };
  fdtd_status st;
  if ((st = slots(h_pass_batch<T, kBatchTY, kBatchS, kBatchMinB, true>, b->grid_pass)) != FDTD_OK) return st;
  if ((st = slots(e_pass_batch<T, kBatchTY, kBatchS, kBatchMinB, true>, b->grid_pass)) != FDTD_OK) return st;
  if ((st = slots(h_pass_batch<T, kBatchTY, kBatchS, kBatchMinB, false>, b->grid_inner)) != FDTD_OK) return st;
  if ((st = slots(e_pass_batch<T, kBatchTY, kBatchS, kBatchMinB, false>, b->grid_inner)) != FDTD_OK) return st;
  CUDA_TRY(cudaFuncSetAttribute(dft_contract_batch<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)dft_smem_bytes<T>()));
  return FDTD_OK;
}

// A launch with a programmatic dependency on the launch before it on the
// stream (both persistent pass launches of a half step: the second fills
// the tail of the first).
template <typename... P, typename... A>
static void launch_dependent(void (*kern)(P...), dim3 g, dim3 blk, size_t smem, cudaStream_t st, A&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = g;
  cfg.blockDim = blk;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, kern, std::forward<A>(args)...);
}

template <typename T>
static void batch_enqueue_step(fdtd_batch* b, cudaStream_t st) {
  const int n = (int)b->sims.size();
  const BatchSim<T>* d = static_cast<const BatchSim<T>*>(b->descs);
  const SimView<T>* v = static_cast<const SimView<T>*>(b->views);
  const size_t smem = staged_smem<T, kBatchTY, kBatchS>();
  const dim3 pb(32, kBatchTY);
  const int4* inner_items = b->items + b->nedge;
  cudaMemsetAsync(b->queue, 0, 4 * sizeof(int), st);
  int k = 0;
  // each pass: the CPML edge items, then the CPML-free items with a
  // programmatic dependency (they touch disjoint cells)
  if (b->nedge) {
    h_pass_batch<T, kBatchTY, kBatchS, kBatchMinB, true><<<b->grid_pass, pb, smem, st>>>(v, b->items, b->nedge,
                                                                                       b->queue, kBatchKChunk);
    k++;
  }
  if (b->ninner) {
    launch_dependent(h_pass_batch<T, kBatchTY, kBatchS, kBatchMinB, false>, dim3(b->grid_inner), pb, smem, st, v,
                     inner_items, b->ninner, b->queue + 1, (int)kBatchKChunk);
    k++;
  }
  // the line step writes the line's other E buffer, so the fused TFSF launch
  // after it still applies the H half with the line's E from before it
  line_step_batch<T><<<dim3(1, n), 1024, 0, st>>>(d);
  k++;
  if (b->g_f) { tfsf_apply_batch<T><<<dim3(b->g_f, n), 256, 0, st>>>(d); k++; }
  if (b->hydro)
    for (auto& s : b->sims) {
      const long long k0 = s->kernels;
      launch_metal<T>(s.get(), st);  // UpdateHydroP* read E^n here
      k += (int)(s->kernels - k0);
    }
  if (b->nedge) {
    e_pass_batch<T, kBatchTY, kBatchS, kBatchMinB, true><<<b->grid_pass, pb, smem, st>>>(v, b->items, b->nedge,
                                                                                       b->queue + 2, kBatchKChunk);
    k++;
  }
  if (b->ninner) {
    launch_dependent(e_pass_batch<T, kBatchTY, kBatchS, kBatchMinB, false>, dim3(b->grid_inner), pb, smem, st, v,
                     inner_items, b->ninner, b->queue + 3, (int)kBatchKChunk);
    k++;
  }
  if (!b->hydro && b->g_m) { metal_e_batch<T><<<dim3(b->g_m, n), 128, 0, st>>>(d); k++; }
  if (b->dft_every > 0 && b->t % b->dft_every == 0) {
    dft_sample_batch<T><<<dim3(b->g_s, 12, n), 256, 0, st>>>(d);
    k++;
    if (++b->host_nsamp == kSampleBlock) {
      // the members' rings fill together: these contract once they are full
      dft_twiddles_batch<T><<<dim3(b->g_tw, n), 256, 0, st>>>(d);
      dft_contract_batch<T><<<dim3(b->g_c, n), 128, dft_smem_bytes<T>(), st>>>(d);
      dft_reset_batch<T><<<dim3(1, n), 1, 0, st>>>(d);
      k += 3;
      b->host_nsamp = 0;
    }
  }
  b->kernels += k;
  b->t++;
}

template <typename T>
static fdtd_status batch_step(fdtd_batch* b, int nsteps, cudaStream_t st) {
  const int every = b->dft_every > 0 ? b->dft_every : 1;
  const int G = every * kSampleBlock;
  int done = 0;
  while (done < nsteps) {
    const bool aligned = b->t % G == 0 && b->host_nsamp == 0 && nsteps - done >= G;
    if (aligned) {
      if (!b->graph) {
        if (!b->cap) CUDA_TRY(cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking));
        cudaGraph_t g;
        const int t_save = b->t, n_save = b->host_nsamp;
        const long long k_save = b->kernels;
        CUDA_TRY(cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal));
        for (int q = 0; q < G; q++) batch_enqueue_step<T>(b, b->cap);
        CUDA_TRY(cudaStreamEndCapture(b->cap, &g));
        b->graph_kernels = b->kernels - k_save;
        b->kernels = k_save;
        b->t = t_save;
        b->host_nsamp = n_save;
        cudaError_t e = cudaGraphInstantiate(&b->graph, g, 0);
        cudaGraphDestroy(g);
        CUDA_TRY(e);
      }
      CUDA_TRY(cudaGraphLaunch(b->graph, st));
      b->kernels += b->graph_kernels;
      b->graph_launches++;
      b->t += G;
      done += G;
    } else {
      batch_enqueue_step<T>(b, st);
      done++;
    }
  }
  // the members' host mirrors follow the batch clock
  for (auto& s : b->sims) {
    s->t = b->t;
    s->host_nsamp = b->host_nsamp;
    s->steps_done += nsteps;
  }
  CUDA_TRY(cudaGetLastError());
  return FDTD_OK;
}

static fdtd_status batch_create_impl(const fdtd_params* ps, int n, int device, fdtd_batch** out) {
  if (!ps || !out || n <= 0) return fail(FDTD_ERR_INVALID, "bad argument");
  auto b = std::make_unique<fdtd_batch>();
  b->device = device;
  CUDA_TRY(cudaSetDevice(device));
  for (int i = 0; i < n; i++) {
    fdtd_sim* s = nullptr;
    const fdtd_status st = create_impl(&ps[i], device, &s, /*tune*/ false);
    if (st != FDTD_OK) return fail(st, "batch member " + std::to_string(i) + ": " + g_err);
    b->sims.emplace_back(s);
    if (i == 0) {
      b->fp64 = s->fp64;
      b->hydro = s->su.hydro;
      b->dft_every = s->line.dft_every;
      b->tend = s->su.p.Tend;
    } else if (s->fp64 != b->fp64 || s->su.hydro != b->hydro || s->line.dft_every != b->dft_every ||
               s->su.p.Tend != b->tend) {
      return fail(FDTD_ERR_INVALID, "batch members must share precision, hydrodynamic model, "
                                    "DFT sampling period and Tend (member " + std::to_string(i) + ")");
    }
  }
  const fdtd_status st = b->fp64 ? batch_build<double>(b.get()) : batch_build<float>(b.get());
  if (st != FDTD_OK) return st;
  CUDA_TRY(cudaDeviceSynchronize());
  *out = b.release();
  return FDTD_OK;
}

extern "C" fdtd_status fdtd_batch_create(const fdtd_params* ps, int n, int device, fdtd_batch** out) {
  try {
    return batch_create_impl(ps, n, device, out);
  } catch (const std::bad_alloc&) {
    return fail(FDTD_ERR_ALLOC, "host allocation failed");
  }
}

extern "C" fdtd_status fdtd_batch_step(fdtd_batch* b, int nsteps, void* stream) {
  if (!b || nsteps < 0) return fail(FDTD_ERR_INVALID, "bad argument");
  CUDA_TRY(cudaSetDevice(b->device));
  return b->fp64 ? batch_step<double>(b, nsteps, as_stream(stream)) : batch_step<float>(b, nsteps, as_stream(stream));
}

extern "C" fdtd_status fdtd_batch_run(fdtd_batch* b, void* stream) {
  if (!b) return fail(FDTD_ERR_INVALID, "null argument");
  const int left = b->tend + 1 - b->t;
  if (left <= 0) return FDTD_OK;
  return fdtd_batch_step(b, left, stream);
}

extern "C" fdtd_status fdtd_batch_sim(fdtd_batch* b, int idx, fdtd_sim** out) {
  if (!b || !out || idx < 0 || idx >= (int)b->sims.size()) return fail(FDTD_ERR_INVALID, "bad argument");
  *out = b->sims[idx].get();
  return FDTD_OK;
}

extern "C" fdtd_status fdtd_batch_spectra(fdtd_batch* b, int idx, double* out19) {
  if (!b || !out19 || idx < 0 || idx >= (int)b->sims.size()) return fail(FDTD_ERR_INVALID, "bad argument");
  return fdtd_spectral_finalize(b->sims[idx].get(), out19);
}

extern "C" fdtd_status fdtd_batch_get_stats(const fdtd_batch* b, long long* kernels, long long* graph_launches) {
  if (!b) return fail(FDTD_ERR_INVALID, "null argument");
  if (kernels) *kernels = b->kernels;
  if (graph_launches) *graph_launches = b->graph_launches;
  return FDTD_OK;
}

extern "C" fdtd_status fdtd_batch_destroy(fdtd_batch* b) {
  if (!b) return FDTD_OK;
  cudaSetDevice(b->device);
  cudaDeviceSynchronize();
  delete b;
  return FDTD_OK;
}
