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
//   the DFT contraction (job, phasors, product, reset), one launch each,
//                     every 32 samples; it contracts each member's first
//                     ring half once that holds 64 samples
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
// The members keep filling the first half of their rings: every launch
// period each member's job is its samples once the half cannot take
// another period (dft_job_ready_body), contracted, then the half emptied.
// A flush before the spectra are read goes through the member's own
// contraction kernels (fdtd_spectral_finalize) and takes the samples no job
// has taken.
template <typename T>
__global__ void dft_job_ready_batch(const BatchSim<T>* __restrict__ b) {
  dft_job_ready_body(b[blockIdx.y].clk);
}
template <typename T>
__global__ void dft_twiddles_batch(const BatchSim<T>* __restrict__ b) {
  const BatchSim<T>& x = b[blockIdx.y];
  dft_twiddles_body(x.dft, x.clk, x.tw);
}
template <typename T>
__global__ void __launch_bounds__(128) dft_contract_batch(const BatchSim<T>* __restrict__ b) {
  const BatchSim<T>& x = b[blockIdx.y];
  dft_contract_body(x.dft, x.ring, x.clk, x.tw);
}
template <typename T>
__global__ void dft_job_done_batch(const BatchSim<T>* __restrict__ b) {
  dft_job_done_body(b[blockIdx.y].clk);
}

}  // namespace fdtd

// Pass launch shapes of the batch.  Work items are 32 x 4 tiles (TY = 4 for
// every launch, so that the CPML-edge and CPML-free item lists partition
// the cells); each size bucket of members has its own z-chunk, carried by
// its items; the edge and the interior launch of each pass have their own
// kernel variant (register cap MINB and ring depth S).  fdtd_batch_create
// times the choices (batch_tune).
constexpr int kBatchTY = 4;
#define FDTD_BATCH_VARIANTS(X) X(1, 4) X(6, 4) X(8, 4) X(6, 6)
constexpr int kBatchVariants = 4;
static const int kBatchVar[kBatchVariants][2] = {{1, 4}, {6, 4}, {8, 4}, {6, 6}};  // (MINB, S)
constexpr int kBatchBucket = 16;  // members bucketed by their largest edge, 16 cells a bucket
constexpr int kBatchMaxBuckets = FDTD_BATCH_MAX_BUCKETS;

struct fdtd_batch {
  int device = 0;
  bool fp64 = false, hydro = false;
  std::vector<std::unique_ptr<fdtd_sim>> sims;
  std::vector<std::unique_ptr<DevBuf>> bufs;
  void* descs = nullptr;  // BatchSim<T>[n]
  void* views = nullptr;  // SimView<T>[n]
  int4* items = nullptr;  // (member | z-chunk << 20, bx, by, bz): edge items, then interior items
  int* queue = nullptr;   // [4] work counters: H edge, H interior, E edge, E interior
  int nedge = 0, ninner = 0;
  size_t items_cap = 0;
  // size buckets and the z-chunk of each; member -> bucket
  int nbuckets = 0;
  int bucket_lo[kBatchMaxBuckets] = {}, bucket_members[kBatchMaxBuckets] = {}, bucket_kc[kBatchMaxBuckets] = {};
  float bucket_ms[kBatchMaxBuckets] = {};
  std::vector<int> member_bucket;
  // kernel variant (index into kBatchVar) and persistent grid per launch:
  // [pass H / E][edge / interior]
  int var[2][2] = {{1, 1}, {1, 1}};
  int grid[2][2] = {{0, 0}, {0, 0}};
  int sms = 0;
  bool tuned = false;
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

// Work items of member i with z-chunk kc: the tiles that touch no CPML slab
// go to `inner` (the rule of build_tiles), the others to `edge`.
static void batch_member_items(const fdtd_sim* s, int i, int kc, std::vector<int4>& edge, std::vector<int4>& inner) {
  const int nbx = (s->NX + 31) / 32, nby = (s->NY + kBatchTY - 1) / kBatchTY, nbz = (s->NZ + kc - 1) / kc;
  const int nb3[3] = {nbx, nby, nbz}, w3[3] = {32, kBatchTY, kc};
  int lo[3], hi[3];
  for (int a = 0; a < 3; a++) {
    const int Nc = s->su.Nc[a], F = s->su.F[a];
    lo[a] = (Nc + 1 + w3[a] - 1) / w3[a];
    hi[a] = std::min(F >= w3[a] ? (F - w3[a]) / w3[a] + 1 : 0, nb3[a]);
  }
  const int tag = i | (kc << 20);
  for (int bz = 0; bz < nbz; bz++)
    for (int by = 0; by < nby; by++)
      for (int bx = 0; bx < nbx; bx++) {
        const bool in = bx >= lo[0] && bx < hi[0] && by >= lo[1] && by < hi[1] && bz >= lo[2] && bz < hi[2];
        (in ? inner : edge).push_back(make_int4(tag, bx, by, bz));
      }
}

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
  CUDA_TRY(b->alloc(&b->queue, 4));
  CUDA_TRY(cudaMemcpy(dd, d.data(), n * sizeof(BatchSim<T>), cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMemcpy(dv, v.data(), n * sizeof(SimView<T>), cudaMemcpyHostToDevice));
  b->descs = dd;
  b->views = dv;
  // size buckets by the largest edge, z-chunk 16 until tuned
  b->member_bucket.assign(n, 0);
  std::vector<int> key(n);
  for (int i = 0; i < n; i++) {
    const fdtd_sim* s = b->sims[i].get();
    key[i] = (std::max(s->NX, std::max(s->NY, s->NZ)) - 1) / kBatchBucket;
  }
  std::vector<int> keys(key);
  std::sort(keys.begin(), keys.end());
  keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
  if ((int)keys.size() > kBatchMaxBuckets) {  // merge the largest ones into the last bucket
    keys.resize(kBatchMaxBuckets);
  }
  b->nbuckets = (int)keys.size();
  for (int q = 0; q < b->nbuckets; q++) {
    b->bucket_lo[q] = keys[q] * kBatchBucket + 1;
    b->bucket_kc[q] = 16;
    b->bucket_members[q] = 0;
  }
  for (int i = 0; i < n; i++) {
    int q = (int)(std::lower_bound(keys.begin(), keys.end(), key[i]) - keys.begin());
    q = std::min(q, b->nbuckets - 1);
    b->member_bucket[i] = q;
    b->bucket_members[q]++;
  }
  CUDA_TRY(cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, b->device));
  // every batch pass variant may take more than 48 KB of shared memory
#define FDTD_BATCH_ATTR(MB, S)                                                                                  \
  CUDA_TRY(cudaFuncSetAttribute(h_pass_batch<T, kBatchTY, S, MB, true>,                                         \
                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)staged_smem<T, kBatchTY, S>())); \
  CUDA_TRY(cudaFuncSetAttribute(h_pass_batch<T, kBatchTY, S, MB, false>,                                        \
                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)staged_smem<T, kBatchTY, S>())); \
  CUDA_TRY(cudaFuncSetAttribute(e_pass_batch<T, kBatchTY, S, MB, true>,                                         \
                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)staged_smem<T, kBatchTY, S>())); \
  CUDA_TRY(cudaFuncSetAttribute(e_pass_batch<T, kBatchTY, S, MB, false>,                                        \
                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)staged_smem<T, kBatchTY, S>()));
  FDTD_BATCH_VARIANTS(FDTD_BATCH_ATTR)
#undef FDTD_BATCH_ATTR
  CUDA_TRY(cudaFuncSetAttribute(dft_contract_batch<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)dft_smem_bytes<T>()));
  return FDTD_OK;
}

// Persistent grid of one pass launch: every CTA slot of the GPU once.
template <typename T, bool EPASS, bool PML>
static int batch_grid(fdtd_batch* b, int var) {
  int per = 0;
  const int mb = kBatchVar[var][0], sg = kBatchVar[var][1];
#define FDTD_BATCH_OCC(MB, S)                                                                                   \
  if (mb == MB && sg == S) {                                                                                     \
    if (EPASS)                                                                                                  \
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, e_pass_batch<T, kBatchTY, S, MB, PML>, 32 * kBatchTY,  \
                                                    staged_smem<T, kBatchTY, S>());                             \
    else                                                                                                        \
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, h_pass_batch<T, kBatchTY, S, MB, PML>, 32 * kBatchTY,  \
                                                    staged_smem<T, kBatchTY, S>());                             \
  }
  FDTD_BATCH_VARIANTS(FDTD_BATCH_OCC)
#undef FDTD_BATCH_OCC
  return std::max(1, per) * b->sms;
}

// The item lists for the current per-bucket z-chunks, uploaded (edge items
// first, then interior items).
static fdtd_status batch_upload_items(fdtd_batch* b, const std::vector<int>* only_bucket_members = nullptr) {
  std::vector<int4> edge, inner;
  const int n = (int)b->sims.size();
  for (int i = 0; i < n; i++) {
    if (only_bucket_members && std::find(only_bucket_members->begin(), only_bucket_members->end(), i) ==
                                   only_bucket_members->end())
      continue;
    batch_member_items(b->sims[i].get(), i, b->bucket_kc[b->member_bucket[i]], edge, inner);
  }
  b->nedge = (int)edge.size();
  b->ninner = (int)inner.size();
  edge.insert(edge.end(), inner.begin(), inner.end());
  if (edge.empty()) return FDTD_OK;
  // one buffer, kept and grown: the graph of the step holds its address
  static_assert(sizeof(int4) == 16, "int4 items");
  if (!b->items || b->items_cap < edge.size()) {
    int4* d;
    CUDA_TRY(b->alloc(&d, edge.size()));
    b->items = d;
    b->items_cap = edge.size();
  }
  CUDA_TRY(cudaMemcpy(b->items, edge.data(), edge.size() * sizeof(int4), cudaMemcpyHostToDevice));
  return FDTD_OK;
}

// One persistent pass launch of variant `var` over items [off, off + n),
// counting its work from queue; pdl = a programmatic dependency on the
// launch before it on the stream.
template <typename T, bool EPASS, bool PML>
static void batch_pass_launch(fdtd_batch* b, int var, int grid, int off, int n, int* queue, cudaStream_t st,
                              bool pdl) {
  const SimView<T>* v = static_cast<const SimView<T>*>(b->views);
  const int4* items = b->items + off;
  const int mb = kBatchVar[var][0], sg = kBatchVar[var][1];
#define FDTD_BATCH_LAUNCH(MB, S)                                                                              \
  if (mb == MB && sg == S) {                                                                                   \
    const size_t smem = staged_smem<T, kBatchTY, S>();                                                        \
    if (EPASS) {                                                                                              \
      if (pdl) launch_ex(true, e_pass_batch<T, kBatchTY, S, MB, PML>, dim3(grid), dim3(32, kBatchTY), smem,  \
                                st, v, items, n, queue);                                                      \
      else e_pass_batch<T, kBatchTY, S, MB, PML><<<grid, dim3(32, kBatchTY), smem, st>>>(v, items, n, queue); \
    } else {                                                                                                  \
      if (pdl) launch_ex(true, h_pass_batch<T, kBatchTY, S, MB, PML>, dim3(grid), dim3(32, kBatchTY), smem,  \
                                st, v, items, n, queue);                                                      \
      else h_pass_batch<T, kBatchTY, S, MB, PML><<<grid, dim3(32, kBatchTY), smem, st>>>(v, items, n, queue); \
    }                                                                                                         \
  }
  FDTD_BATCH_VARIANTS(FDTD_BATCH_LAUNCH)
#undef FDTD_BATCH_LAUNCH
}

// One pass of every member: the CPML edge items, then the CPML-free items
// with a programmatic dependency (they touch disjoint cells); returns the
// number of launches.
template <typename T, bool EPASS>
static int batch_pass(fdtd_batch* b, int* queue, cudaStream_t st) {
  const int p = EPASS ? 1 : 0;
  int k = 0;
  if (b->nedge) {
    batch_pass_launch<T, EPASS, true>(b, b->var[p][0], b->grid[p][0], 0, b->nedge, queue, st, false);
    k++;
  }
  if (b->ninner) {
    batch_pass_launch<T, EPASS, false>(b, b->var[p][1], b->grid[p][1], b->nedge, b->ninner, queue + 1, st, true);
    k++;
  }
  return k;
}

template <typename T>
static void batch_enqueue_step(fdtd_batch* b, cudaStream_t st) {
  const int n = (int)b->sims.size();
  const BatchSim<T>* d = static_cast<const BatchSim<T>*>(b->descs);
  cudaMemsetAsync(b->queue, 0, 4 * sizeof(int), st);
  int k = batch_pass<T, false>(b, b->queue, st);
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
  k += batch_pass<T, true>(b, b->queue + 2, st);
  if (!b->hydro && b->g_m) { metal_e_batch<T><<<dim3(b->g_m, n), 128, 0, st>>>(d); k++; }
  if (b->dft_every > 0 && b->t % b->dft_every == 0) {
    dft_sample_batch<T><<<dim3(b->g_s, 12, n), 256, 0, st>>>(d);
    k++;
    if (++b->host_nsamp == kSampleBlock) {
      // the members' rings fill together: these contract once they are full
      dft_job_ready_batch<T><<<dim3(1, n), 1, 0, st>>>(d);
      dft_twiddles_batch<T><<<dim3(b->g_tw, n), 256, 0, st>>>(d);
      dft_contract_batch<T><<<dim3(b->g_c, n), 128, dft_smem_bytes<T>(), st>>>(d);
      dft_job_done_batch<T><<<dim3(1, n), 1, 0, st>>>(d);
      k += 4;
      b->host_nsamp = 0;
    }
  }
  b->kernels += k;
  b->t++;
}

// Mean device time of `reps` runs of both passes (H and E, each its edge
// and interior launch) over the current item lists, after one untimed run.
// On the zero state the passes leave the fields at zero.
template <typename T>
static fdtd_status batch_time_passes(fdtd_batch* b, int reps, float* ms) {
  cudaEvent_t e0, e1;
  CUDA_TRY(cudaEventCreate(&e0));
  CUDA_TRY(cudaEventCreate(&e1));
  auto go = [&]() {
    cudaMemsetAsync(b->queue, 0, 4 * sizeof(int), 0);
    batch_pass<T, false>(b, b->queue, 0);
    batch_pass<T, true>(b, b->queue + 2, 0);
  };
  go();
  cudaEventRecord(e0, 0);
  for (int r = 0; r < reps; r++) go();
  cudaEventRecord(e1, 0);
  cudaError_t e = cudaEventSynchronize(e1);
  float t = 0.f;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&t, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (e != cudaSuccess) return fail(FDTD_ERR_CUDA, std::string("batch tuning: ") + cudaGetErrorString(e));
  *ms = t / reps;
  return FDTD_OK;
}

// The autotuner of the batch's passes (no counterpart in the reference):
// per size bucket the z-chunk (8, 16 or 32 planes) with the bucket's
// members alone, then per launch (H / E pass, edge / interior items) the
// kernel variant over the whole batch.  FDTD_TUNE=0, or a batch under 2^20
// cells, keeps z-chunk 16 and variant (MINB 6, S 4) everywhere.
template <typename T>
static fdtd_status batch_tune(fdtd_batch* b) {
  for (int p = 0; p < 2; p++)
    for (int q = 0; q < 2; q++) b->var[p][q] = 1;
  auto grids = [&]() {
    b->grid[0][0] = batch_grid<T, false, true>(b, b->var[0][0]);
    b->grid[0][1] = batch_grid<T, false, false>(b, b->var[0][1]);
    b->grid[1][0] = batch_grid<T, true, true>(b, b->var[1][0]);
    b->grid[1][1] = batch_grid<T, true, false>(b, b->var[1][1]);
  };
  grids();
  long long cells = 0;
  for (const auto& s : b->sims) cells += s->ncell;
  const char* env = std::getenv("FDTD_TUNE");
  fdtd_status st;
  if ((env && env[0] == '0') || cells < (1LL << 20)) return batch_upload_items(b);
  const int n = (int)b->sims.size();
  // z-chunk per bucket, its members alone
  for (int q = 0; q < b->nbuckets; q++) {
    std::vector<int> mem;
    for (int i = 0; i < n; i++)
      if (b->member_bucket[i] == q) mem.push_back(i);
    float best = 1e30f;
    int best_kc = 16;
    for (int kc : {8, 16, 32}) {
      b->bucket_kc[q] = kc;
      if ((st = batch_upload_items(b, &mem)) != FDTD_OK) return st;
      float ms;
      if ((st = batch_time_passes<T>(b, 3, &ms)) != FDTD_OK) return st;
      if (ms < best) { best = ms; best_kc = kc; }
    }
    b->bucket_kc[q] = best_kc;
    b->bucket_ms[q] = best;
  }
  if ((st = batch_upload_items(b)) != FDTD_OK) return st;
  // the variant of each launch, the others held
  for (int p = 0; p < 2; p++)
    for (int e = 0; e < 2; e++) {
      float best = 1e30f;
      int best_v = b->var[p][e];
      for (int v = 0; v < kBatchVariants; v++) {
        b->var[p][e] = v;
        grids();
        float ms;
        if ((st = batch_time_passes<T>(b, 3, &ms)) != FDTD_OK) return st;
        if (ms < best) { best = ms; best_v = v; }
      }
      b->var[p][e] = best_v;
      grids();
    }
  b->tuned = true;
  CUDA_TRY(cudaGetLastError());
  return FDTD_OK;
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
  for (int i = 0; i < n; i++)
    if (ps[i].periodic_xy) return fail(FDTD_ERR_UNSUPPORTED, "periodic_xy simulations do not batch (member " + std::to_string(i) + ")");
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
  fdtd_status st = b->fp64 ? batch_build<double>(b.get()) : batch_build<float>(b.get());
  if (st != FDTD_OK) return st;
  st = b->fp64 ? batch_tune<double>(b.get()) : batch_tune<float>(b.get());
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

extern "C" fdtd_status fdtd_batch_get_tuning(const fdtd_batch* b, fdtd_batch_tuning* out) {
  if (!b || !out) return fail(FDTD_ERR_INVALID, "null argument");
  std::memset(out, 0, sizeof(*out));
  out->tuned = b->tuned ? 1 : 0;
  out->nbuckets = b->nbuckets;
  for (int q = 0; q < b->nbuckets; q++) {
    out->edge_lo[q] = b->bucket_lo[q];
    out->edge_hi[q] = q + 1 < b->nbuckets ? b->bucket_lo[q + 1] - 1 : INT_MAX;
    out->members[q] = b->bucket_members[q];
    out->kchunk[q] = b->bucket_kc[q];
    out->bucket_ms[q] = b->bucket_ms[q];
  }
  out->tile_x = 32;
  out->tile_y = kBatchTY;
  for (int p = 0; p < 2; p++)
    for (int e = 0; e < 2; e++) {
      out->minb[p][e] = kBatchVar[b->var[p][e]][0];
      out->stages[p][e] = kBatchVar[b->var[p][e]][1];
    }
  return FDTD_OK;
}

extern "C" fdtd_status fdtd_batch_destroy(fdtd_batch* b) {
  if (!b) return FDTD_OK;
  cudaSetDevice(b->device);
  cudaDeviceSynchronize();
  delete b;
  return FDTD_OK;
}
