// npom_batch.cuh -- an ensemble of members advanced together, one launch per
// phase (included by npom_kernels.cu inside its anonymous namespace, after
// the one-member launchers, whose phase bodies it reuses).
//
// A batch is a set of members of one core, each with its own grid size,
// state and workspace, advanced over the same clock.  Every phase of the
// internal step is ONE launch over all members: the blocks of a launch are
// dealt to the members in contiguous ranges (a prefix table per launch
// shape); a block finds its member by binary search, copies the member's
// launch context into shared memory and runs the one-member phase body at
// its member-local index.  So every member computes bitwise what it
// computes when advanced alone, wherever no reduction spans blocks.
//
//   external subcycle (explicit core): one launch per substep phase over
//     all members (NPOM_BATCH_SUBCYCLE=phases, the default), or one
//     cooperative launch for the whole subcycle in which each member's
//     blocks meet at their own grid barrier (=coop);
//   PCG (semi-implicit core): one cluster launch per cluster shape (8 or
//     16 CTAs, Sy in shared or global memory), one cluster per member
//     whose interior fits a cluster layout (the member's own layout, as
//     when it runs alone); one cooperative launch for the other members,
//     each on its own share of the co-resident blocks (at most
//     NPOM_BATCH_PCG_BLOCKS each when set) with its own grid barrier.  The
//     FP64 dot products of the cooperative form are summed per block, so a
//     member that gets fewer blocks than it gets alone sums them in another
//     order (results agree to rounding, not bitwise);
//   A1 and B5 (kb == 16): the flux-once tiles of every member in one
//     launch (bitwise the point kernels' values), with one rows-per-tile
//     value for the whole batch;
//   the step is captured once as a CUDA graph per value of do_internal and
//   replayed (steps whose ramp is 1 for every member).
#pragma once

constexpr int kMaxBatch = NPOM_MAX_BATCH;

enum BatchShape { BS_POINTS = 0, BS_LANES, BS_COLS, BS_CELLS, BS_A1T, BS_B5T, BS_SUB, BS_PCG, BS_NSHAPES };
constexpr int kBatchThreads[BS_NSHAPES] = {kThreads, kThreads, 128, kThreads, kA1Threads, kB5Threads,
                                           kThreads, kThreads};

struct BatchTable {
  int count[BS_NSHAPES];                 // members (slots) of each shape
  int member[BS_NSHAPES][kMaxBatch];     // slot -> member
  int start[BS_NSHAPES][kMaxBatch + 1];  // slot -> first block; start[count] = blocks of the launch
  // cluster PCG groups g = (nc > 8) + 2 * sy_global: members, CTAs per cluster
  int clu_count[4], clu_nc[4];
  int clu_member[4][kMaxBatch];
  int tile_strips[2][kMaxBatch];         // flux-once A1 / B5 tiles: column strips of each member
  int tile_ichunk[2];                    // rows per tile (one value for all members)
  int nm;
  ClusterLayout L[kMaxBatch];
  Ctx ctx[kMaxBatch];
};

// per-step values of every member, a kernel argument of every launch
struct BatchStep {
  float ramp[kMaxBatch];
  int do_internal;
};

__device__ __forceinline__ void batch_copy_ctx(const Ctx *src, Ctx &dst) {
  const unsigned *s = reinterpret_cast<const unsigned *>(src);
  unsigned *d = reinterpret_cast<unsigned *>(&dst);
  for (int w = threadIdx.x; w < (int)(sizeof(Ctx) / 4); w += blockDim.x) d[w] = s[w];
}

// The member of this block in launch shape S: its context into sc (with the
// step's values; for the cooperative shapes L2 loads and the member's block
// range as its grid).  Returns the block index within the member.
template <int S>
__device__ __forceinline__ int batch_enter(const BatchTable *t, const BatchStep &v, Ctx &sc, int *member = nullptr) {
  __shared__ int s_slot;
  if (threadIdx.x == 0) {
    const int *st = t->start[S];
    int lo = 0, hi = t->count[S] - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (st[mid] <= (int)blockIdx.x) lo = mid;
      else hi = mid - 1;
    }
    s_slot = lo;
  }
  __syncthreads();
  const int slot = s_slot;
  const int m = t->member[S][slot];
  if (member) *member = m;
  batch_copy_ctx(&t->ctx[m], sc);
  __syncthreads();
  if (threadIdx.x == 0) {
    sc.ramp = v.ramp[m];
    sc.do_internal = v.do_internal;
    if (S == BS_SUB || S == BS_PCG) {
      sc.coh = 1;
      sc.grid_base = t->start[S][slot];
      sc.grid_blocks = t->start[S][slot + 1] - t->start[S][slot];
    }
  }
  __syncthreads();
  return (int)blockIdx.x - t->start[S][slot];
}

template <int PH>
__global__ void __launch_bounds__(kThreads) kb_points(const BatchTable *t, BatchStep v) {
  __shared__ Ctx sc;
  const int lb = batch_enter<BS_POINTS>(t, v, sc);
  points_body<PH>(sc, (size_t)lb * blockDim.x + threadIdx.x);
}

template <int PH>
__global__ void __launch_bounds__(kThreads) kb_lanes(const BatchTable *t, BatchStep v) {
  __shared__ Ctx sc;
  const int lb = batch_enter<BS_LANES>(t, v, sc);
  lanes_body<PH>(sc, lb * blockDim.x + threadIdx.x);
}

template <int PH>
__global__ void __launch_bounds__(128) kb_cols(const BatchTable *t, BatchStep v) {
  __shared__ Ctx sc;
  const int lb = batch_enter<BS_COLS>(t, v, sc);
  cols_body<PH>(sc, lb * blockDim.x + threadIdx.x);
}

// thread-per-column PROFT with 16 levels at compile time (k_cols_b6_kb16)
__global__ void __launch_bounds__(128) kb_cols_b6_kb16(const BatchTable *t, BatchStep v) {
  __shared__ Ctx sc;
  const int lb = batch_enter<BS_COLS>(t, v, sc);
  const int col = lb * blockDim.x + threadIdx.x;
  if (col < sc.im * sc.jm) phase_b6_column<16>(sc, col / sc.jm, col % sc.jm);
}

template <int PH>
__global__ void __launch_bounds__(kThreads) kb_cells(const BatchTable *t, BatchStep v) {
  __shared__ Ctx sc;
  const int lb = batch_enter<BS_CELLS>(t, v, sc);
  cells_body<PH>(sc, lb * blockDim.x + threadIdx.x);
}

// the flux-once A1 / B5 tiles of every member: block lb of a member is
// strip lb % strips, row chunk lb / strips
__global__ void __launch_bounds__(kA1Threads) kb_a1_tiles(const BatchTable *t, BatchStep v) {
  __shared__ Ctx sc;
  int m = 0;
  const int lb = batch_enter<BS_A1T>(t, v, sc, &m);
  const int st = t->tile_strips[0][m];
  a1_tiles_body(sc, t->tile_ichunk[0], lb % st, lb / st);
}

__global__ void __launch_bounds__(kB5Threads) kb_b5_tiles(const BatchTable *t, BatchStep v) {
  __shared__ Ctx sc;
  int m = 0;
  const int lb = batch_enter<BS_B5T>(t, v, sc, &m);
  const int st = t->tile_strips[1][m];
  b5_tiles_body(sc, t->tile_ichunk[1], lb % st, lb / st);
}

__global__ void __launch_bounds__(kThreads) kb_ext(const BatchTable *t, BatchStep v, int phase, int iext, int adv) {
  __shared__ Ctx sc;
  const int lb = batch_enter<BS_CELLS>(t, v, sc);
  ext_phase_body(sc, phase, iext, adv, lb * blockDim.x + threadIdx.x);
}

__global__ void __launch_bounds__(kThreads) kb_mpdata(const BatchTable *t, BatchStep v, int pass, int itera) {
  __shared__ Ctx sc;
  const int lb = batch_enter<BS_POINTS>(t, v, sc);
  mpdata_body(sc, pass, itera, (size_t)lb * blockDim.x + threadIdx.x);
}

__global__ void __launch_bounds__(kThreads) kb_subcycle(const BatchTable *t, BatchStep v) {
  __shared__ Ctx sc;
  batch_enter<BS_SUB>(t, v, sc);
  subcycle_coop_body(sc);
}

__global__ void __launch_bounds__(kThreads) kb_pcg(const BatchTable *t, BatchStep v, int with_rhs, int with_post) {
  __shared__ Ctx sc;
  batch_enter<BS_PCG>(t, v, sc);
  pcg_coop_body<true>(sc, with_rhs, with_post);
}

// cluster group g of the table: consecutive clusters of clu_nc[g] CTAs,
// one member each (SYG: the group's layouts read Sy from global memory)
template <bool SYG>
__global__ void __launch_bounds__(kClusterThreads, 1)
    kb_pcg_cluster(const BatchTable *t, BatchStep v, int g, int with_rhs, int with_post) {
  extern __shared__ __align__(16) float sm[];
  __shared__ Ctx sc;
  __shared__ ClusterLayout sL;
  const int m = t->clu_member[g][blockIdx.x / t->clu_nc[g]];
  batch_copy_ctx(&t->ctx[m], sc);
  if (threadIdx.x == 0) sL = t->L[m];
  __syncthreads();
  if (threadIdx.x == 0) {
    sc.ramp = v.ramp[m];
    sc.do_internal = v.do_internal;
  }
  __syncthreads();
  pcg_cluster_body<SYG>(sc, sL, sm, with_rhs, with_post);
}

// clears words [0, words) of the control block of every member (the
// barrier's arrival counter before a cooperative launch; at the start of a
// call also the solve counter)
__global__ void kb_reset_sync(const BatchTable *t, int words) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= t->nm) return;
  for (int w = 0; w < words; ++w) t->ctx[m].sync[w] = 0u;
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
constexpr size_t kBatchStaticSmem = sizeof(Ctx) + sizeof(ClusterLayout) + 64;

struct BatchPlan {
  int device = -1, core = 0, nm = 0;
  std::vector<Ctx> key;
  BatchTable *d_table = nullptr;
  int blocks[BS_NSHAPES] = {};
  int clu_count[4] = {}, clu_nc[4] = {};
  size_t clu_smem[4] = {};
  bool lanes = false, b6_cols = false;
  bool kb16 = false;      // every member has 16 levels (batch_uniform: one kb)
  bool a1_tiles = false, b5_tiles = false;
  bool sub_req = false;   // NPOM_BATCH_SUBCYCLE=coop when the plan was made
  bool sub_coop = false;  // the cooperative subcycle is in use
  int nadv = 1, nitera = 0, mode = 3, isplit = 0, ispadv = 1;
  cudaGraphExec_t graph[2] = {nullptr, nullptr};  // per do_internal
  bool capture_failed = false;
};

std::mutex g_batch_mutex;
std::vector<BatchPlan *> g_batch_plans;
constexpr size_t kBatchPlanCache = 16;

// kernels launched by the last npom_step_batch call of this process
long long g_batch_launches = 0;

// the batched explicit subcycle as one cooperative launch: NPOM_BATCH_SUBCYCLE
// =coop, or the grid-barrier subcycle form in the first member's tuning
bool batch_subcycle_coop(const Ctx &c0) {
  const char *env = getenv("NPOM_BATCH_SUBCYCLE");
  if (env) return std::strcmp(env, "coop") == 0;
  return c0.tune.subcycle_form == 2;
}

// blocks of a cooperative launch of fn dealt to the members in proportion to
// their work (at least one each, at most what covers the work); false when
// the members outnumber the co-resident blocks
bool batch_coop_shares(const void *fn, const std::vector<int> &members, const std::vector<size_t> &work,
                       int start[], int *total, int max_per_member = NPOM_MAX_COOP_BLOCKS) {
  int dev = 0, sms = 0, per_sm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return false;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return false;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kThreads, 0) != cudaSuccess) return false;
  const int cap = per_sm * sms;
  const int n = (int)members.size();
  if (n == 0) {
    start[0] = 0;
    *total = 0;
    return true;
  }
  if (n > cap) return false;
  size_t sum = 0;
  for (size_t w : work) sum += w;
  int at = 0;
  for (int s = 0; s < n; ++s) {
    start[s] = at;
    const double share = (double)(cap - n) * (double)work[s] / (double)(sum ? sum : 1);
    int b = 1 + (int)share;
    b = std::min(b, std::max(1, blocks_for(work[s], kThreads)));
    b = std::min(b, std::min(max_per_member, NPOM_MAX_COOP_BLOCKS));
    at += b;
  }
  start[n] = at;
  *total = at;
  return at <= cap;
}

const void *batch_cluster_fn(int g) {
  return g >= 2 ? (const void *)kb_pcg_cluster<true> : (const void *)kb_pcg_cluster<false>;
}

cudaError_t make_batch_plan(const std::vector<Ctx> &ctx, int core, BatchPlan *P) {
  const int nm = (int)ctx.size();
  P->nm = nm;
  P->core = core;
  P->key = ctx;
  cudaError_t e = cudaGetDevice(&P->device);
  if (e != cudaSuccess) return e;
  const int dev = P->device;
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  const Ctx &c0 = ctx[0];
  P->lanes = c0.kb == KL && lanes_enabled(c0);
  P->kb16 = c0.kb == 16;
  P->nadv = c0.k.nadv;
  P->nitera = c0.k.nitera;
  P->mode = c0.k.mode;
  P->isplit = c0.k.isplit;
  P->ispadv = c0.k.ispadv;
  std::vector<unsigned char> host(sizeof(BatchTable), 0);
  BatchTable *T = reinterpret_cast<BatchTable *>(host.data());
  T->nm = nm;
  size_t columns = 0;
  for (int m = 0; m < nm; ++m) {
    T->ctx[m] = ctx[m];
    columns += (size_t)ctx[m].im * ctx[m].jm;
  }
  P->b6_cols = !P->lanes || columns >= kProftThreadColumns;
  // flux-once tiles for A1 and B5 (kb == 16; B5 not in mode 4 nor with
  // MPDATA); NPOM_A1=points / NPOM_B5=points keep the point kernels.  Rows
  // per tile: about 16 tiles per SM over the whole batch
  {
    const char *ea = getenv("NPOM_A1"), *eb = getenv("NPOM_B5");
    const bool a1_points = ea ? std::strcmp(ea, "points") == 0 : c0.tune.a1_form == 1;
    const bool b5_points = eb ? std::strcmp(eb, "points") == 0 : c0.tune.b5_form == 1;
    P->a1_tiles = c0.kb == 16 && !a1_points;
    P->b5_tiles = c0.kb == 16 && c0.k.mode != 4 && c0.k.nadv != 2 && !b5_points;
    const int per_sm = c0.tune.tile_blocks_per_sm > 0 ? c0.tune.tile_blocks_per_sm : 16;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    for (int g = 0; g < 2; ++g) {
      const int cols = g == 0 ? kA1Cols : kB5Cols;
      size_t rows = 0;
      for (int m = 0; m < nm; ++m) rows += (size_t)ctx[m].im * ((ctx[m].jm + cols - 1) / cols);
      const int ichunk = std::max(2, (int)((rows + per_sm * (size_t)sms - 1) / (per_sm * (size_t)sms)));
      T->tile_ichunk[g] = ichunk;
      const int S = g == 0 ? BS_A1T : BS_B5T;
      int at = 0;
      T->count[S] = nm;
      for (int m = 0; m < nm; ++m) {
        const int strips = (ctx[m].jm + cols - 1) / cols;
        T->tile_strips[g][m] = strips;
        T->member[S][m] = m;
        T->start[S][m] = at;
        at += strips * ((ctx[m].im + ichunk - 1) / ichunk);
      }
      T->start[S][nm] = at;
      P->blocks[S] = at;
    }
  }
  // the plain shapes: every member, blocks to cover its work
  for (int S = BS_POINTS; S <= BS_CELLS; ++S) {
    int at = 0;
    T->count[S] = nm;
    for (int m = 0; m < nm; ++m) {
      const size_t ncol = (size_t)ctx[m].im * ctx[m].jm;
      const size_t work = S == BS_POINTS ? ncol * ctx[m].kb : (S == BS_LANES ? ncol * KL : ncol);
      T->member[S][m] = m;
      T->start[S][m] = at;
      at += std::max(1, blocks_for(work, kBatchThreads[S]));
    }
    T->start[S][nm] = at;
    P->blocks[S] = at;
  }
  P->sub_req = batch_subcycle_coop(c0);
  if (core == NPOM_CORE_EXPLICIT) {
    P->sub_coop = P->sub_req;
    if (P->sub_coop) {
      std::vector<int> mem;
      std::vector<size_t> work;
      for (int m = 0; m < nm; ++m) {
        mem.push_back(m);
        work.push_back((size_t)ctx[m].im * ctx[m].jm);
      }
      int total = 0;
      if (batch_coop_shares((const void *)kb_subcycle, mem, work, T->start[BS_SUB], &total)) {
        T->count[BS_SUB] = nm;
        for (int m = 0; m < nm; ++m) T->member[BS_SUB][m] = m;
        P->blocks[BS_SUB] = total;
      } else {
        P->sub_coop = false;
      }
    }
  } else {
    // the member's own cluster layout where it has one (8 CTAs first, as
    // alone), else the cooperative form
    int optin = 0;
    e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (e != cudaSuccess) return e;
    std::vector<int> coop;
    std::vector<size_t> work;
    for (int m = 0; m < nm; ++m) {
      ClusterLayout L{};
      const bool fits = pcg_cluster_layout(ctx[m], &L) && L.bytes() + kBatchStaticSmem <= (size_t)optin;
      if (fits) {
        const int g = (L.nc > 8 ? 1 : 0) + (L.sy_global ? 2 : 0);
        T->L[m] = L;
        T->clu_member[g][T->clu_count[g]++] = m;
        T->clu_nc[g] = L.nc;
        P->clu_smem[g] = std::max(P->clu_smem[g], L.bytes());
      } else {
        coop.push_back(m);
        work.push_back(pcg_coop_work(ctx[m]));
      }
    }
    for (int g = 0; g < 4; ++g) {
      P->clu_count[g] = T->clu_count[g];
      P->clu_nc[g] = T->clu_nc[g];
      if (P->clu_count[g] == 0) continue;
      // the attribute only grows (plans made earlier keep their launches
      // valid); a cluster shape that cannot be resident sends its members
      // to the cooperative form
      static int smem_set[64][2] = {};
      const int v = g >> 1;
      const void *fn = batch_cluster_fn(g);
      const int smem = (int)P->clu_smem[g];
      if (smem > smem_set[dev][v]) {
        e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        if (e != cudaSuccess) return e;
        smem_set[dev][v] = smem;
      }
      if (P->clu_nc[g] > 8) {
        e = cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
        if (e != cudaSuccess) return e;
      }
      if (cluster_launchable(fn, P->clu_nc[g], (size_t)smem)) continue;
      for (int q = 0; q < T->clu_count[g]; ++q) {
        const int m = T->clu_member[g][q];
        coop.push_back(m);
        work.push_back(pcg_coop_work(ctx[m]));
      }
      T->clu_count[g] = P->clu_count[g] = 0;
    }
    int total = 0;
    // NPOM_BATCH_PCG_BLOCKS caps the blocks of each member's cooperative
    // solve (its barrier waits hold their SMs)
    const char *cap_env = getenv("NPOM_BATCH_PCG_BLOCKS");
    const int cap = cap_env ? std::max(1, atoi(cap_env)) : c0.tune.batch_pcg_blocks;
    const int per_member = cap > 0 ? std::min(cap, NPOM_MAX_COOP_BLOCKS) : NPOM_MAX_COOP_BLOCKS;
    if (!batch_coop_shares((const void *)kb_pcg, coop, work, T->start[BS_PCG], &total, per_member))
      return cudaErrorInvalidValue;
    T->count[BS_PCG] = (int)coop.size();
    for (size_t s = 0; s < coop.size(); ++s) T->member[BS_PCG][s] = coop[s];
    P->blocks[BS_PCG] = total;
  }
  e = cudaMalloc(&P->d_table, sizeof(BatchTable));
  if (e == cudaSuccess) e = cudaMemcpy(P->d_table, T, sizeof(BatchTable), cudaMemcpyHostToDevice);
  return e;
}

void destroy_batch_plan(BatchPlan *P) {
  for (auto &g : P->graph)
    if (g) cudaGraphExecDestroy(g);
  if (P->d_table) cudaFree(P->d_table);
  delete P;
}

cudaError_t batch_launch_coop(const void *fn, int blocks, void **args, const BatchPlan &P, cudaStream_t s) {
  kb_reset_sync<<<(P.nm + 63) / 64, 64, 0, s>>>(P.d_table, 1);
  return cudaLaunchCooperativeKernel(fn, dim3(blocks), dim3(kThreads), args, 0, s);
}

template <int PH>
void batch_cols(const BatchPlan &P, const BatchStep &v, cudaStream_t s) {
  if (P.lanes && !(PH == CP_B6 && P.b6_cols)) kb_lanes<PH><<<P.blocks[BS_LANES], kThreads, 0, s>>>(P.d_table, v);
  else if (PH == CP_B6 && P.kb16) kb_cols_b6_kb16<<<P.blocks[BS_COLS], 128, 0, s>>>(P.d_table, v);
  else kb_cols<PH><<<P.blocks[BS_COLS], 128, 0, s>>>(P.d_table, v);
}

template <int PH>
void batch_points(const BatchPlan &P, const BatchStep &v, cudaStream_t s) {
  kb_points<PH><<<P.blocks[BS_POINTS], kThreads, 0, s>>>(P.d_table, v);
}

template <int PH>
void batch_cells(const BatchPlan &P, const BatchStep &v, cudaStream_t s) {
  kb_cells<PH><<<P.blocks[BS_CELLS], kThreads, 0, s>>>(P.d_table, v);
}

cudaError_t batch_subcycle(const BatchPlan &P, const BatchStep &v, cudaStream_t s) {
  if (P.sub_coop) {
    const BatchTable *t = P.d_table;
    BatchStep vv = v;
    void *args[] = {(void *)&t, &vv};
    return batch_launch_coop((const void *)kb_subcycle, P.blocks[BS_SUB], args, P, s);
  }
  for (int iext = 1; iext <= P.isplit; ++iext) {
    const int adv = (iext % P.ispadv) == 0;
    for (int ph = 1; ph <= 3; ++ph) kb_ext<<<P.blocks[BS_CELLS], kThreads, 0, s>>>(P.d_table, v, ph, iext, adv);
  }
  return cudaGetLastError();
}

cudaError_t batch_pcg(const BatchPlan &P, const BatchStep &v, cudaStream_t s) {
  const BatchTable *t = P.d_table;
  BatchStep vv = v;
  int with_rhs = 1, with_post = 1;
  for (int g = 0; g < 4; ++g) {
    if (P.clu_count[g] == 0) continue;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(P.clu_count[g] * P.clu_nc[g]);
    cfg.blockDim = dim3(kClusterThreads);
    cfg.dynamicSmemBytes = P.clu_smem[g];
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = P.clu_nc[g];
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaError_t e = g >= 2 ? cudaLaunchKernelEx(&cfg, kb_pcg_cluster<true>, t, vv, g, with_rhs, with_post)
                           : cudaLaunchKernelEx(&cfg, kb_pcg_cluster<false>, t, vv, g, with_rhs, with_post);
    if (e != cudaSuccess) return e;
  }
  if (P.blocks[BS_PCG] > 0) {
    void *args[] = {(void *)&t, &vv, &with_rhs, &with_post};
    return batch_launch_coop((const void *)kb_pcg, P.blocks[BS_PCG], args, P, s);
  }
  return cudaSuccess;
}

// one internal step of every member (the order of enqueue_step)
cudaError_t enqueue_batch_step(const BatchPlan &P, const BatchStep &v, cudaStream_t s) {
  if (P.a1_tiles) kb_a1_tiles<<<P.blocks[BS_A1T], kA1Threads, 0, s>>>(P.d_table, v);
  else batch_points<PP_A1>(P, v, s);
  batch_cols<CP_A2>(P, v, s);
  batch_cells<XP_A3>(P, v, s);
  cudaError_t e;
  if (P.core == NPOM_CORE_IMPLICIT) {
    e = batch_pcg(P, v, s);
    if (e != cudaSuccess) return e;
    batch_cells<XP_I5>(P, v, s);
  } else {
    e = batch_subcycle(P, v, s);
    if (e != cudaSuccess) return e;
  }
  if (v.do_internal) {
    batch_cols<CP_B1>(P, v, s);
    batch_cols<CP_B2A>(P, v, s);
    batch_points<PP_B2B>(P, v, s);
    batch_cols<CP_B3>(P, v, s);
    batch_points<PP_B4>(P, v, s);
    if (P.nadv == 2 && P.mode != 4) {
      const BatchTable *t = P.d_table;
      const int g = P.blocks[BS_POINTS];
      kb_mpdata<<<g, kThreads, 0, s>>>(t, v, MP_FILTER, 0);
      kb_mpdata<<<g, kThreads, 0, s>>>(t, v, MP_INIT, 0);
      for (int it = 1; it <= P.nitera; ++it) {
        kb_mpdata<<<g, kThreads, 0, s>>>(t, v, MP_UPWIND, it);
        kb_mpdata<<<g, kThreads, 0, s>>>(t, v, MP_FORECAST, it);
        kb_mpdata<<<g, kThreads, 0, s>>>(t, v, MP_ANTIDIFF, it);
      }
      kb_mpdata<<<g, kThreads, 0, s>>>(t, v, MP_DIFFUSION, 0);
      kb_mpdata<<<g, kThreads, 0, s>>>(t, v, MP_FINISH, 0);
    } else if (P.b5_tiles) {
      kb_b5_tiles<<<P.blocks[BS_B5T], kB5Threads, 0, s>>>(P.d_table, v);
    } else {
      batch_points<PP_B5>(P, v, s);
    }
    batch_cols<CP_B6>(P, v, s);
    batch_points<PP_B7>(P, v, s);
    batch_cols<CP_B8>(P, v, s);
  }
  batch_cols<CP_B9>(P, v, s);
  return cudaGetLastError();
}

// kernels enqueue_batch_step launches for one step
int batch_step_launches(const BatchPlan &P, int do_internal) {
  int n = 3 + 1;  // A1 A2 A3, B9
  if (P.core == NPOM_CORE_IMPLICIT) {
    for (int g = 0; g < 4; ++g) n += P.clu_count[g] > 0;
    n += (P.blocks[BS_PCG] > 0 ? 2 : 0) + 1;
  } else {
    n += P.sub_coop ? 2 : 3 * P.isplit;
  }
  if (do_internal) n += 8 + ((P.nadv == 2 && P.mode != 4) ? 4 + 3 * P.nitera : 1);
  return n;
}

// replays (capturing on first use) the graph of one step with ramp 1
// everywhere; *launched false when it could not be captured
cudaError_t batch_step_graph(BatchPlan &P, const BatchStep &v, cudaStream_t s, bool *launched) {
  *launched = false;
  cudaGraphExec_t &exec = P.graph[v.do_internal ? 1 : 0];
  if (!exec) {
    if (P.capture_failed) return cudaSuccess;
    std::lock_guard<std::mutex> lock(g_graph_mutex);  // the capture stream is shared
    const int dev = P.device;
    if (!g_capture_stream[dev]) {
      cudaError_t e = cudaStreamCreateWithFlags(&g_capture_stream[dev], cudaStreamNonBlocking);
      if (e != cudaSuccess) return e;
    }
    cudaStream_t cs = g_capture_stream[dev];
    cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return e;
    cudaError_t le = enqueue_batch_step(P, v, cs);
    cudaGraph_t graph = nullptr;
    e = cudaStreamEndCapture(cs, &graph);
    if (le != cudaSuccess || e != cudaSuccess || !graph) {
      if (graph) cudaGraphDestroy(graph);
      cudaGetLastError();
      P.capture_failed = true;
      return cudaSuccess;
    }
    e = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) {
      exec = nullptr;
      cudaGetLastError();
      P.capture_failed = true;
      return cudaSuccess;
    }
  }
  cudaError_t e = cudaGraphLaunch(exec, s);
  *launched = (e == cudaSuccess);
  return e;
}

// the members of one call: one core, one level count, one subcycle and one
// tracer-advection setting (the launches of a step are shared)
bool batch_uniform(const npom_params *const *p, int nm) {
  for (int m = 1; m < nm; ++m) {
    const npom_params *a = p[0], *b = p[m];
    if (b->core != a->core || b->kb != a->kb || b->isplit != a->isplit || b->ispadv != a->ispadv ||
        b->mode != a->mode || b->nadv != a->nadv || b->nitera != a->nitera || b->device != a->device)
      return false;
  }
  // the POM08-WAD PROFQ has no lane body, which the batched column phases
  // use, and the seamount boundary's Orlanski passes and the periodic-x
  // halo copies are not batched
  for (int m = 0; m < nm; ++m)
    if (p[m]->profq_form != NPOM_PROFQ_PRODUCTION || p[m]->obc_form != NPOM_OBC_NATIVE || p[m]->periodic_x)
      return false;
  return true;
}

npom_status run_batch_steps(int nm, const npom_params *const *p, float *const *const *fields,
                            const npom_workspace *const *ws, const npom_clock *clk, void *stream) {
  if (nm <= 0 || nm > kMaxBatch || !p || !fields || !ws || !clk || clk->nsteps < 0) return NPOM_ERR_ARG;
  for (int m = 0; m < nm; ++m)
    if (!p[m] || !check_args_dev(p[m], fields[m], ws[m])) return NPOM_ERR_ARG;
  if (!batch_uniform(p, nm)) return NPOM_ERR_ARG;
  const int core = p[0]->core;
  if (core != NPOM_CORE_EXPLICIT && core != NPOM_CORE_IMPLICIT) return NPOM_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  std::vector<Ctx> ctx(nm);
  for (int m = 0; m < nm; ++m) ctx[m] = make_ctx(p[m], fields[m], ws[m]);
  const bool sub_req = batch_subcycle_coop(ctx[0]);
  std::lock_guard<std::mutex> lock(g_batch_mutex);
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return NPOM_ERR_CUDA;
  BatchPlan *P = nullptr;
  for (BatchPlan *q : g_batch_plans) {
    if (q->device == dev && q->core == core && q->nm == nm && q->sub_req == sub_req &&
        std::memcmp(q->key.data(), ctx.data(), nm * sizeof(Ctx)) == 0) {
      P = q;
      break;
    }
  }
  if (!P) {
    if (g_batch_plans.size() >= kBatchPlanCache) {
      if (cudaDeviceSynchronize() != cudaSuccess) return NPOM_ERR_CUDA;
      destroy_batch_plan(g_batch_plans.front());
      g_batch_plans.erase(g_batch_plans.begin());
    }
    P = new BatchPlan();
    if (make_batch_plan(ctx, core, P) != cudaSuccess) {
      destroy_batch_plan(P);
      cudaGetLastError();
      return NPOM_ERR_CUDA;
    }
    g_batch_plans.push_back(P);
  }
  // a barrier that timed out may leave its arrival counter non-zero;
  // sync[2] counts the PCG solves of this call
  kb_reset_sync<<<(nm + 63) / 64, 64, 0, s>>>(P->d_table, 4);
  BatchStep v{};
  long long launches = 1;
  if (core == NPOM_CORE_IMPLICIT) {
    batch_cells<XP_COEF>(*P, v, s);
    ++launches;
  }
  const bool graphs = graphs_enabled();
  for (int n = 0; n < clk->nsteps; ++n) {
    const int iint = clk->first_iint + n;
    bool all_one = true;
    for (int m = 0; m < nm; ++m) {
      const double time = p[m]->dti * iint * 1.0 / 86400.0 + clk->time0;
      v.ramp[m] = ramp_of(p[m], time);
      all_one = all_one && v.ramp[m] == 1.0f;
    }
    v.do_internal = ((iint != 1 || clk->time0 != 0.0) && p[0]->mode != 2) ? 1 : 0;
    launches += batch_step_launches(*P, v.do_internal);
    bool done = false;
    if (graphs && all_one) {
      if (batch_step_graph(*P, v, s, &done) != cudaSuccess) return NPOM_ERR_CUDA;
    }
    if (!done && enqueue_batch_step(*P, v, s) != cudaSuccess) return NPOM_ERR_CUDA;
  }
  g_batch_launches = launches;
  return cudaGetLastError() == cudaSuccess ? NPOM_OK : NPOM_ERR_CUDA;
}
