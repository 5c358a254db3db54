// npom_adjoint_launch.cuh -- kernels and host driver of the explicit-core
// step adjoint (included by npom_kernels.cu, which provides the forward
// launchers).  One call differentiates one internal step: it recomputes the
// step phase by phase from the checkpointed state, saving every field a
// phase overwrites, then walks the phases backwards: restore the phase's
// inputs, move the cotangents of what it wrote, run its adjoint.

// Forward of one external-substep phase, one launch per phase (the fused
// subcycle kernel computes the same values; this form leaves a point to
// save the state between phases).
__global__ void __launch_bounds__(kThreads) k_ext_fwd(Ctx c, int phase, int iext, int adv) {
  const int n = c.im * c.jm;
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  const int i = q / c.jm, j = q % c.jm;
  if (phase == AP_E1) ext_phase1_cell(c, i, j, adv != 0);
  else if (phase == AP_E2) (void)ext_phase2_cell(c, i, j, iext);
  else ext_phase3_cell(c, i, j, iext);
}

// the reverse of one MPDATA pass of B5 (plan phase ph, iteration it)
__global__ void __launch_bounds__(kThreads) k_adj_mpdata(Ctx c, Adj a, int ph, int it) {
  const size_t n = (size_t)c.im * c.jm * c.kb;
  size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const int k = (int)(p % c.kb);
  const size_t col = p / c.kb;
  mp_phase_adj(c, a, ph, it, (int)(col / c.jm), (int)(col % c.jm), k);
}

template <int PH>
__global__ void __launch_bounds__(kThreads) k_adj_points(Ctx c, Adj a) {
  const size_t n = (size_t)c.im * c.jm * c.kb;
  size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const int k = (int)(p % c.kb);
  const size_t col = p / c.kb;
  const int j = (int)(col % c.jm), i = (int)(col / c.jm);
  if (PH == AP_A1) phase_a1_point_adj(c, a, i, j, k);
  else if (PH == AP_B2B) phase_b2b_point_adj(c, a, i, j, k);
  else if (PH == AP_B4) phase_b4_point_adj(c, a, i, j, k);
  else if (PH == AP_B5) phase_b5_point_adj(c, a, i, j, k);
  else if (PH == AP_B7) phase_b7_point_adj(c, a, i, j, k);
}

// column adjoints with their level arrays sized KM (16 for the common
// kb = 16, so that they stay in registers and L1)
template <int PH, int KM>
__device__ __forceinline__ void adj_column(const Ctx &c, const Adj &a, int i, int j) {
  if (PH == AP_A2) phase_a2_column_adj<KM>(c, a, i, j);
  else if (PH == AP_B1) phase_b1_column_adj<KM>(c, a, i, j);
  else if (PH == AP_B2A) phase_b2a_column_adj<KM>(c, a, i, j);
  else if (PH == AP_B3) phase_b3_column_adj<KM>(c, a, i, j);
  else if (PH == AP_B6) phase_b6_column_adj<KM>(c, a, i, j);
  else if (PH == AP_B8) phase_b8_column_adj<KM>(c, a, i, j);
  else if (PH == AP_B9) phase_b9_column_adj<KM>(c, a, i, j);
}

template <int PH, int KM>
__global__ void __launch_bounds__(128) k_adj_cols_t(Ctx c, Adj a) {
  const int n = c.im * c.jm;
  int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= n) return;
  const int j = col % c.jm, i = col / c.jm;
  adj_column<PH, KM>(c, a, i, j);
}

// B8's adjoint on two threads per column, u and v (adjacent lanes)
template <int KM>
__global__ void __launch_bounds__(128) k_adj_b8_split(Ctx c, Adj a) {
  const int n = 2 * c.im * c.jm;
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  const int col = q >> 1;
  phase_b8_comp_adj<KM>(c, a, q & 1, col / c.jm, col % c.jm);
}

template <int PH>
void launch_adj_cols(const Ctx &c, const Adj &a, cudaStream_t s) {
  const unsigned g = (unsigned)((c.im * c.jm + 127) / 128);
  if (c.kb == 16) k_adj_cols_t<PH, 16><<<g, 128, 0, s>>>(c, a);
  else k_adj_cols_t<PH, KMAX><<<g, 128, 0, s>>>(c, a);
}

__global__ void __launch_bounds__(kThreads) k_adj_cells(Ctx c, Adj a, int phase, int iext, int adv) {
  const int n = c.im * c.jm;
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  const int i = q / c.jm, j = q % c.jm;
  if (phase == AP_A3) phase_a3_cell_adj(c, a, i, j);
  else if (phase == AP_I5) phase_i5_cell_adj(c, a, i, j);
  else if (phase == AP_E1) ext_phase1_cell_adj(c, a, i, j, adv != 0);
  else if (phase == AP_E2) ext_phase2_cell_adj(c, a, i, j, iext);
  else ext_phase3_cell_adj(c, a, i, j, iext);
}

// The barrier between the phases of the fused external-subcycle adjoint
// kernels: the hardware cluster barrier (one cluster, up to 16,384 cells)
// or the counting grid barrier of a cooperative launch (larger grids; its
// wait is bounded and a timeout sets NPOM_DEV_TIMEOUT).
template <bool GRID>
__device__ __forceinline__ bool ext_sync(const Ctx &c) {
  if (GRID) return grid_barrier(c);
  cgx::this_cluster().sync();
  return true;
}

// The whole external subcycle of the recomputation in one launch: before
// each phase every thread saves the values of the fields the phase
// overwrites at the cells it computes (the same thread-to-cell map, so no
// barrier is needed between save and compute), then computes the phase; a
// barrier separates the phases.  Loads go through L2 (Ctx::coh).  save is
// the first external-phase record of the plan; records follow in plan order.
template <int T, bool GRID>
__global__ void __launch_bounds__(T, GRID ? 0 : 1) k_adj_ext_forward(Ctx c, float *save) {
  const size_t ncell = (size_t)c.im * c.jm;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  float *out = save;
  for (int iext = 1; iext <= c.k.isplit; ++iext) {
    const bool adv = (iext % c.k.ispadv) == 0;
    for (int ph = 1; ph <= 3; ++ph) {
      int fl[10];
      const int nf = ext_phase_fields(iext, ph, c.k.isplit, c.k.ispadv, fl);
      for (int e = 0; e < nf; ++e) {
        const float *src = c.F[fl[e]];
        for (size_t q = tid; q < ncell; q += stride) out[(size_t)e * ncell + q] = __ldcg(src + q);
      }
      out += (size_t)nf * ncell;
      for (size_t q = tid; q < ncell; q += stride) {
        const int i = (int)(q / c.jm), j = (int)(q % c.jm);
        if (ph == 1) ext_phase1_cell(c, i, j, adv);
        else if (ph == 2) (void)ext_phase2_cell(c, i, j, iext);
        else ext_phase3_cell(c, i, j, iext);
      }
      if (!ext_sync<GRID>(c)) return;
    }
  }
}

// The reverse sweep of the external subcycle in one launch: for each phase
// from the last, restore its inputs and move the cotangents of what it
// wrote (each thread its own cells), barrier, the phase's adjoint (scatters
// are atomics in L2; every other read goes through L2 or is of a value the
// thread itself moved), barrier.  Phase 3's adjoint needs neither: at a
// cell it reads and scatters the fields that phase 3 wrote (and that its
// restore and move touch) only at that cell, and elf of its west and south
// neighbours, which phase 3 does not write; phase 2's restore and move
// (uaf, vaf, etf) likewise touch only values that phase 3's adjoint reads
// or scatters at the same cell.  The same thread handles a cell in all
// these loops, so restore 3, adjoint 3 and restore 2 run without a
// barrier between them.
template <int T, bool GRID>
__global__ void __launch_bounds__(T, GRID ? 0 : 1) k_adj_ext_reverse(Ctx c, Adj a, const float *save_end) {
  const size_t ncell = (size_t)c.im * c.jm;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const float *in = save_end;
  for (int iext = c.k.isplit; iext >= 1; --iext) {
    const bool adv = (iext % c.k.ispadv) == 0;
    for (int ph = 3; ph >= 1; --ph) {
      int fl[10];
      const int nf = ext_phase_fields(iext, ph, c.k.isplit, c.k.ispadv, fl);
      in -= (size_t)nf * ncell;
      for (int e = 0; e < nf; ++e) {
        float *dst = c.F[fl[e]], *g = a.G[fl[e]], *l = a.L[fl[e]];
        for (size_t q = tid; q < ncell; q += stride) {
          dst[q] = in[(size_t)e * ncell + q];
          l[q] = __ldcg(g + q);
          g[q] = 0.0f;
        }
      }
      if (ph != 3 && !ext_sync<GRID>(c)) return;
      for (size_t q = tid; q < ncell; q += stride) {
        const int i = (int)(q / c.jm), j = (int)(q % c.jm);
        if (ph == 3) ext_phase3_cell_adj(c, a, i, j, iext);
        else if (ph == 2) ext_phase2_cell_adj(c, a, i, j, iext);
        else ext_phase1_cell_adj(c, a, i, j, adv);
      }
      if (ph != 3 && !ext_sync<GRID>(c)) return;
    }
  }
}

const void *const kAdjExtForward[3] = {(const void *)k_adj_ext_forward<256, false>,
                                       (const void *)k_adj_ext_forward<512, false>,
                                       (const void *)k_adj_ext_forward<1024, false>};
const void *const kAdjExtReverse[3] = {(const void *)k_adj_ext_reverse<256, false>,
                                       (const void *)k_adj_ext_reverse<512, false>,
                                       (const void *)k_adj_ext_reverse<1024, false>};
const void *const kAdjExtForwardGrid = (const void *)k_adj_ext_forward<kThreads, true>;
const void *const kAdjExtReverseGrid = (const void *)k_adj_ext_reverse<kThreads, true>;

// Launch shape of the fused external-subcycle adjoint kernels, decided
// outside any capture: < 0 a cluster shape (encode_cluster, both kernels
// get the one that fits both), > 0 cooperative grid blocks (larger grids),
// 0 one launch per substep phase (NPOM_ADJ_EXT=phases, or no fit).
// NPOM_ADJ_EXT=grid forces the cooperative form on small grids too.
int plan_adj_ext(const Ctx &c) {
  const char *env = getenv("NPOM_ADJ_EXT");
  if (env && std::strcmp(env, "phases") == 0) return 0;
  const bool grid = (env && std::strcmp(env, "grid") == 0);
  const size_t ncell = (size_t)c.im * c.jm;
  if (!grid && ncell <= kSubClusterCells) {
    int f = 0, r = 0;
    if (plan_cluster(kAdjExtForward, ncell, &f) == cudaSuccess &&
        plan_cluster(kAdjExtReverse, ncell, &r) == cudaSuccess)
      return cluster_ctas(f) <= cluster_ctas(r) ? f : r;
    cudaGetLastError();
  }
  int bf = 0, br = 0;
  if (coop_blocks(kAdjExtForwardGrid, ncell, &bf) != cudaSuccess ||
      coop_blocks(kAdjExtReverseGrid, ncell, &br) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return std::min(bf, br);
}

// Implicit free surface, forward: the solution x of the PCG (run without its
// post step) is kept in xs; then the Shapiro filter (gamma 0) and masks of
// the post step, d = h + elf, ring values -- the same arithmetic as
// k_pcg_cluster's post step.
// The forward solve (with its rhs set-up, no post step) without solving:
// the stored transports of the set-up, and elf = the raw solution the
// forward pass kept (ring 0).  The solve is deterministic, so this writes
// what run_pcg(with_rhs, no post) writes to the fields the step reads.
__global__ void __launch_bounds__(kThreads) k_imp_replay(Ctx c, const float *x) {
  const int n = c.im * c.jm;
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  const int i = q / c.jm, j = q % c.jm;
  P2(fluxua, i, j) = rhs_fluxua(c, i, j);
  P2(fluxva, i, j) = rhs_fluxva(c, i, j);
  P2(elf, i, j) = interior(c, i, j) ? x[q] : 0.0f;
}

__global__ void __launch_bounds__(kThreads) k_imp_post(Ctx c, const float *xs) {
  const int n = c.im * c.jm;
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  const int i = q / c.jm, j = q % c.jm;
  if (!interior(c, i, j)) {
    P2(elf, i, j) = 0.0f;
    P2(d, i, j) = F2(h, i, j);
    return;
  }
  const int jm = c.jm;
  const float x0 = xs[q];
  const float xn = (j + 1 < jm - 1) ? xs[q + 1] : 0.0f;
  const float xsv = (j - 1 > 0) ? xs[q - 1] : 0.0f;
  const float xe = (i + 1 < c.im - 1) ? xs[q + jm] : 0.0f;
  const float xw = (i - 1 > 0) ? xs[q - jm] : 0.0f;
  const float smv = x0 + c.k.bshap_q * (xe + xw + xn + xsv - 4.0f * x0);
  const float fsm = F2(fsm, i, j);
  const float ev = (smv * fsm) * fsm;
  if (!(fabsf(ev) <= 3.0e38f)) atomicOr(c.status, NPOM_DEV_NONFINITE);
  P2(d, i, j) = F2(h, i, j) + ev;
  P2(elf, i, j) = ev;
}

__global__ void __launch_bounds__(kThreads) k_imp_post_grad(Ctx c, Adj a, float *g) {
  const int n = c.im * c.jm;
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  g[q] = imp_post_grad(c, a, q / c.jm, q % c.jm);
}

__global__ void __launch_bounds__(kThreads) k_imp_rhs_adj(Ctx c, Adj a, const float *lam, const float *gd) {
  const int n = c.im * c.jm;
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  imp_rhs_cell_adj(c, a, q / c.jm, q % c.jm, lam, gd);
}

// save[off_e ...] = F[fld_e] for every field e of a phase (blockIdx.y = e)
__global__ void k_save_fields(Ctx c, AdjPhaseRec r, float *save) {
  const int e = blockIdx.y;
  if (e >= r.n) return;
  const int f = r.fld[e];
  const size_t n = adj_field_len(c, f);
  const float *src = adj_fptr(c, f);
  float *dst = save + r.off[e];
  for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x)
    dst[q] = src[q];
}

// F[fld_e] = save; and for moved fields L = G, G = 0
__global__ void k_restore_move(Ctx c, Adj a, AdjPhaseRec r, const float *save) {
  const int e = blockIdx.y;
  if (e >= r.n) return;
  const int f = r.fld[e];
  const size_t n = adj_field_len(c, f);
  const float *src = save + r.off[e];
  float *dst = adj_fptr(c, f);
  const bool mv = r.move[e] != 0;
  float *g = a.G[f], *l = a.L[f];
  for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
    dst[q] = src[q];
    if (mv) {
      l[q] = g[q];
      g[q] = 0.0f;
    }
  }
}

dim3 field_list_grid(const Ctx &c, const AdjPhaseRec &r) {
  size_t n = 0;
  for (int e = 0; e < r.n; ++e) n = std::max(n, adj_field_len(c, r.fld[e]));
  const size_t blocks = std::min<size_t>((n + kThreads - 1) / kThreads, 4 * 148);
  return dim3((unsigned)std::max<size_t>(blocks, 1), (unsigned)std::max(r.n, 1));
}

struct ImpScratch {
  const float *xsaved;  // the forward solve's raw solution, or null (solve again)
  float *xs, *g, *lam, *gd;
};

void launch_fwd_phase(const Ctx &c, const AdjPhaseRec &r, const PcgPlan &pplan, const ImpScratch &is,
                      cudaStream_t s) {
  const int ncell = c.im * c.jm;
  const unsigned gx = (unsigned)((ncell + kThreads - 1) / kThreads);
  switch (r.phase) {
    case AP_EI:
      if (is.xsaved) {
        k_imp_replay<<<gx, kThreads, 0, s>>>(c, is.xsaved);
      } else {
        cudaMemsetAsync(c.sync, 0, 4 * sizeof(unsigned int), s);
        run_pcg(c, pplan, 1, 0, s);
      }
      cudaMemcpyAsync(is.xs, c.F[NPOM_F_elf], (size_t)ncell * sizeof(float), cudaMemcpyDeviceToDevice, s);
      k_imp_post<<<gx, kThreads, 0, s>>>(c, is.xs);
      break;
    case AP_I5: launch_cells<XP_I5>(c, s); break;
    case AP_A1: launch_a1(c, s); break;
    case AP_A2: launch_cols<CP_A2>(c, s); break;
    case AP_A3: launch_cells<XP_A3>(c, s); break;
    case AP_E1:
    case AP_E2:
    case AP_E3: {
      const int n = c.im * c.jm;
      k_ext_fwd<<<(n + kThreads - 1) / kThreads, kThreads, 0, s>>>(c, r.phase, r.iext, r.adv);
      break;
    }
    case AP_B1: launch_cols<CP_B1>(c, s); break;
    case AP_B2A: launch_cols<CP_B2A>(c, s); break;
    case AP_B2B: launch_points<PP_B2B>(c, s); break;
    case AP_B3: launch_cols<CP_B3>(c, s); break;
    case AP_B4: launch_points<PP_B4>(c, s); break;
    case AP_B5: launch_b5(c, s); break;
    case AP_B6: launch_cols<CP_B6>(c, s); break;
    case AP_B7: launch_points<PP_B7>(c, s); break;
    case AP_B8: launch_cols<CP_B8>(c, s); break;
    case AP_B9: launch_cols<CP_B9>(c, s); break;
    case AP_MQ:
    case AP_MINIT:
    case AP_MUP:
    case AP_MFC:
    case AP_MAD:
    case AP_MDIF:
    case AP_MFIN: {
      const size_t n = (size_t)c.im * c.jm * c.kb;
      k_mpdata<<<(unsigned)((n + kThreads - 1) / kThreads), kThreads, 0, s>>>(c, mp_pass_of(r.phase), r.iext);
      break;
    }
  }
}

npom_status launch_adj_phase(const npom_params *p, const npom_workspace *ws, const Ctx &c, const Adj &a,
                             const AdjPhaseRec &r, const ImpScratch &is, cudaStream_t s) {
  const size_t np = (size_t)c.im * c.jm * c.kb;
  const int ncol = c.im * c.jm;
  const unsigned gp = (unsigned)((np + kThreads - 1) / kThreads), gx = (unsigned)((ncol + kThreads - 1) / kThreads);
  switch (r.phase) {
    case AP_EI: {
      // elf/d of the post step -> g = dJ/dx; the solve's adjoint gives
      // lambda = A^-T g and dJ/dd; then the rhs and the transports
      // (no host read-back: a non-finite cotangent propagates into the
      // gradients, as under the reference's autograd)
      k_imp_post_grad<<<gx, kThreads, 0, s>>>(c, a, is.g);
      if (enqueue_adj_prep(c, ws, is.g, 0, s) != cudaSuccess ||
          enqueue_adj_solve(c, ws, is.xs, is.lam, is.gd, s) != cudaSuccess)
        return NPOM_ERR_CUDA;
      k_imp_rhs_adj<<<gx, kThreads, 0, s>>>(c, a, is.lam, is.gd);
      break;
    }
    case AP_I5: k_adj_cells<<<gx, kThreads, 0, s>>>(c, a, r.phase, 0, 0); break;
    case AP_A1: k_adj_points<AP_A1><<<gp, kThreads, 0, s>>>(c, a); break;
    case AP_A2: launch_adj_cols<AP_A2>(c, a, s); break;
    case AP_A3:
    case AP_E1:
    case AP_E2:
    case AP_E3: k_adj_cells<<<gx, kThreads, 0, s>>>(c, a, r.phase, r.iext, r.adv); break;
    case AP_B1: launch_adj_cols<AP_B1>(c, a, s); break;
    case AP_B2A: launch_adj_cols<AP_B2A>(c, a, s); break;
    case AP_B2B: k_adj_points<AP_B2B><<<gp, kThreads, 0, s>>>(c, a); break;
    case AP_B3: launch_adj_cols<AP_B3>(c, a, s); break;
    case AP_B4: k_adj_points<AP_B4><<<gp, kThreads, 0, s>>>(c, a); break;
    case AP_B5: k_adj_points<AP_B5><<<gp, kThreads, 0, s>>>(c, a); break;
    case AP_B6: launch_adj_cols<AP_B6>(c, a, s); break;
    case AP_B7: k_adj_points<AP_B7><<<gp, kThreads, 0, s>>>(c, a); break;
    case AP_B8: {
      const unsigned g = (unsigned)((2 * c.im * c.jm + 127) / 128);
      if (c.kb == 16) k_adj_b8_split<16><<<g, 128, 0, s>>>(c, a);
      else k_adj_b8_split<KMAX><<<g, 128, 0, s>>>(c, a);
      break;
    }
    case AP_B9: launch_adj_cols<AP_B9>(c, a, s); break;
    case AP_MQ:
    case AP_MINIT:
    case AP_MUP:
    case AP_MFC:
    case AP_MAD:
    case AP_MDIF:
    case AP_MFIN: k_adj_mpdata<<<gp, kThreads, 0, s>>>(c, a, r.phase, r.iext); break;
  }
  return NPOM_OK;
}

npom_status enqueue_step_adjoint(const npom_params *p, const npom_workspace *ws, const Ctx &c, const Adj &a,
                                 const AdjPhaseRec *plan, int np, const ImpScratch &is, float *scratch,
                                 float *save, int core, cudaStream_t s);
npom_status step_adjoint_graph(const npom_params *p, const npom_workspace *ws, const Ctx &c, const Adj &a,
                               const AdjPhaseRec *plan, int np, const ImpScratch &is, float *scratch, float *save,
                               cudaStream_t s, bool *launched);

npom_status run_step_adjoint(const npom_params *p, float *const *fields, const npom_workspace *ws,
                             const npom_clock *clk, float *const *grads, const npom_adjoint_ws *aws, int core,
                             cudaStream_t s) {
  if (!check_args_dev(p, fields, ws) || !clk || clk->nsteps != 1 || !grads || !aws || !aws->save) return NPOM_ERR_ARG;
  if (p->core != core || !adj_supported(p) || p->isplit > 4096) return NPOM_ERR_ARG;
  for (int f = 0; f < NPOM_NFIELDS; ++f)
    if (!grads[f] || !aws->lam[f]) return NPOM_ERR_ARG;
  Ctx c = make_ctx(p, fields, ws);
  c.coh = 0;
  const int iint = clk->first_iint;
  const double time = p->dti * iint * 1.0 / 86400.0 + clk->time0;
  c.ramp = ramp_of(p, time);
  c.do_internal = (iint != 1 || clk->time0 != 0.0) ? 1 : 0;
  Adj a;
  for (int f = 0; f < NPOM_NFIELDS; ++f) {
    a.G[f] = grads[f];
    a.L[f] = aws->lam[f];
  }
  std::vector<AdjPhaseRec> plan((size_t)adj_plan_capacity(p->isplit, p->nitera));
  size_t need = 0;
  const int np = adj_step_plan(c, plan.data(), (int)plan.size(), &need);
  const size_t ncell = (size_t)c.im * c.jm;
  if (need + adj_scratch_floats(c) > aws->save_floats) return NPOM_ERR_ARG;
  float *scratch = aws->save + need;
  adj_bind_scratch(c, a, scratch);
  ImpScratch is;
  is.xsaved = core == NPOM_CORE_IMPLICIT ? aws->pcg_x : nullptr;
  is.xs = scratch + (size_t)(2 * AW_COUNT) * ncell;
  is.g = is.xs + ncell;
  is.lam = is.g + ncell;
  is.gd = is.lam + ncell;
  if (graphs_enabled()) {
    bool done = false;
    const npom_status st = step_adjoint_graph(p, ws, c, a, plan.data(), np, is, scratch, aws->save, s, &done);
    if (st != NPOM_OK || done) return st;
  }
  return enqueue_step_adjoint(p, ws, c, a, plan.data(), np, is, scratch, aws->save, core, s);
}

// The launches of one step adjoint (recompute with saves, then the reverse
// walk) on s.
npom_status enqueue_step_adjoint(const npom_params *p, const npom_workspace *ws, const Ctx &c, const Adj &a,
                                 const AdjPhaseRec *plan, int np, const ImpScratch &is, float *scratch,
                                 float *save, int core, cudaStream_t s) {
  const size_t ncell = (size_t)c.im * c.jm;
  // workspace and MPDATA cotangents live inside one step
  if (cudaMemsetAsync(scratch, 0, (size_t)AW_COUNT * ncell * sizeof(float), s) != cudaSuccess) return NPOM_ERR_CUDA;
  if (adj_mp_zero_floats(c) &&
      cudaMemsetAsync(scratch + adj_mp_offset(c), 0, adj_mp_zero_floats(c) * sizeof(float), s) != cudaSuccess)
    return NPOM_ERR_CUDA;
  PcgPlan pplan{};
  if (core == NPOM_CORE_IMPLICIT) {
    if (plan_pcg(c, &pplan) != cudaSuccess) return NPOM_ERR_CUDA;
    launch_cells<XP_COEF>(c, s);
  }
  // the external-subcycle records sit together in the plan: [e0, e1)
  int e0 = np, e1 = np;
  for (int q = 0; q < np; ++q)
    if (plan[q].phase == AP_E1 || plan[q].phase == AP_E2 || plan[q].phase == AP_E3) {
      e0 = std::min(e0, q);
      e1 = q + 1;
    }
  const int ext_shape = e0 < e1 ? plan_adj_ext(c) : 0;
  const int ext_threads = ext_shape < 0 ? cluster_threads(ext_shape) : 0;
  const int ext_t = ext_threads == 256 ? 0 : (ext_threads == 512 ? 1 : 2);
  const bool ext_fused = ext_shape != 0;
  const int ext_ctas = ext_shape < 0 ? cluster_ctas(ext_shape) : 0;
  Ctx cc = c;
  cc.coh = 1;
  Adj aa = a;
  float *ext_save = e0 < e1 ? save + plan[e0].off[0] : nullptr;
  const float *ext_end = e0 < e1 ? save + plan[e1 - 1].off[plan[e1 - 1].n - 1] +
                                       adj_field_len(c, plan[e1 - 1].fld[plan[e1 - 1].n - 1])
                                 : nullptr;
  for (int q = 0; q < np; ++q) {
    if (ext_fused && q >= e0 && q < e1) {
      if (q == e0) {
        void *args[] = {&cc, &ext_save};
        const cudaError_t e = ext_shape < 0
                                  ? launch_cluster(kAdjExtForward[ext_t], ext_ctas, ext_threads, args, s)
                                  : launch_coop(kAdjExtForwardGrid, ext_shape, args, c.sync, s);
        if (e != cudaSuccess) return NPOM_ERR_CUDA;
      }
      continue;
    }
    k_save_fields<<<field_list_grid(c, plan[q]), kThreads, 0, s>>>(c, plan[q], save);
    launch_fwd_phase(c, plan[q], pplan, is, s);
  }
  for (int q = np - 1; q >= 0; --q) {
    if (ext_fused && q >= e0 && q < e1) {
      if (q == e0) {
        void *args[] = {&cc, &aa, &ext_end};
        const cudaError_t e = ext_shape < 0
                                  ? launch_cluster(kAdjExtReverse[ext_t], ext_ctas, ext_threads, args, s)
                                  : launch_coop(kAdjExtReverseGrid, ext_shape, args, c.sync, s);
        if (e != cudaSuccess) return NPOM_ERR_CUDA;
      }
      continue;
    }
    k_restore_move<<<field_list_grid(c, plan[q]), kThreads, 0, s>>>(c, a, plan[q], save);
    const npom_status st = launch_adj_phase(p, ws, c, a, plan[q], is, s);
    if (st != NPOM_OK) return st;
  }
  return cudaGetLastError() == cudaSuccess ? NPOM_OK : NPOM_ERR_CUDA;
}

// CUDA graphs of the explicit step adjoint: the launch sequence is fixed
// by the context (pointers, constants, ramp, do_internal), the cotangent
// and lambda pointers and the save buffer, so the steps of a backward pass
// (and, as the allocator hands back the same buffers, the next passes)
// replay one graph instead of enqueueing several hundred kernels from the
// host.  Both cores: the adjoint of the free-surface solve keeps its rhs
// scale on the device.
struct AdjGraphKey {
  Ctx c;
  Adj a;
  float *save;
  const float *xsaved;
};

struct AdjGraphEntry {
  int device;
  AdjGraphKey key;
  cudaGraphExec_t exec;
};

std::mutex g_adj_graph_mutex;
std::vector<AdjGraphEntry> g_adj_graphs;
bool g_adj_capture_failed[64] = {};
constexpr size_t kAdjGraphCache = 64;

npom_status step_adjoint_graph(const npom_params *p, const npom_workspace *ws, const Ctx &c, const Adj &a,
                               const AdjPhaseRec *plan, int np, const ImpScratch &is, float *scratch, float *save,
                               cudaStream_t s, bool *launched) {
  *launched = false;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return NPOM_OK;
  AdjGraphKey key;
  std::memset(&key, 0, sizeof(key));
  key.c = c;
  key.a = a;
  key.save = save;
  key.xsaved = is.xsaved;
  std::lock_guard<std::mutex> lock(g_adj_graph_mutex);
  for (auto &g : g_adj_graphs) {
    if (g.device == dev && std::memcmp(&g.key, &key, sizeof(key)) == 0) {
      if (cudaGraphLaunch(g.exec, s) != cudaSuccess) return NPOM_ERR_CUDA;
      *launched = true;
      return NPOM_OK;
    }
  }
  if (g_adj_capture_failed[dev]) return NPOM_OK;
  std::lock_guard<std::mutex> glock(g_graph_mutex);  // the capture stream is shared
  if (!g_capture_stream[dev] && cudaStreamCreateWithFlags(&g_capture_stream[dev], cudaStreamNonBlocking) != cudaSuccess)
    return NPOM_ERR_CUDA;
  cudaStream_t cs = g_capture_stream[dev];
  if (cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return NPOM_ERR_CUDA;
  const npom_status le = enqueue_step_adjoint(p, ws, c, a, plan, np, is, scratch, save, p->core, cs);
  cudaGraph_t graph = nullptr;
  const cudaError_t e = cudaStreamEndCapture(cs, &graph);
  cudaGraphExec_t exec = nullptr;
  if (le != NPOM_OK || e != cudaSuccess || !graph || cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess) {
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
    g_adj_capture_failed[dev] = true;
    return NPOM_OK;  // not captured: the caller launches directly
  }
  cudaGraphDestroy(graph);
  if (g_adj_graphs.size() >= kAdjGraphCache) {
    // a replaced graph may still be in flight on some stream
    if (cudaDeviceSynchronize() != cudaSuccess) return NPOM_ERR_CUDA;
    cudaGraphExecDestroy(g_adj_graphs.front().exec);
    g_adj_graphs.erase(g_adj_graphs.begin());
  }
  g_adj_graphs.push_back(AdjGraphEntry{dev, key, exec});
  if (cudaGraphLaunch(exec, s) != cudaSuccess) return NPOM_ERR_CUDA;
  *launched = true;
  return NPOM_OK;
}

// ---------------------------------------------------------------------------
// Stand-alone DENS and BAROPG with their adjoints (the core's dens() and
// baropg() operator methods and the corrector coupling: explicit
// momentum.py:467-700, hybrid/sparse_coupling.py:10-82).
// ---------------------------------------------------------------------------

// rho_out = DENS(t, s) on levels < kb-1, the ghost level copied from F rho
__global__ void __launch_bounds__(kThreads) k_dens(Ctx c, const float *t, const float *s, float *rho_out) {
  const size_t n = (size_t)c.im * c.jm * c.kb;
  const size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const int k = (int)(p % c.kb);
  const size_t col = p / c.kb;
  const int j = (int)(col % c.jm), i = (int)(col / c.jm);
  rho_out[p] = k < c.kb - 1 ? dens_point(c, t[p], s[p], i, j, k) : F3(rho, i, j, k);
}

__global__ void __launch_bounds__(kThreads) k_dens_adj(Ctx c, const float *t, const float *s, const float *g,
                                                       float *gt, float *gs, float *grho) {
  const size_t n = (size_t)c.im * c.jm * c.kb;
  const size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const int k = (int)(p % c.kb);
  const size_t col = p / c.kb;
  const int j = (int)(col % c.jm), i = (int)(col / c.jm);
  if (k < c.kb - 1) {
    float dt_, ds_;
    dens_point_adj(c, t[p], s[p], i, j, k, dt_, ds_);
    gt[p] = g[p] * dt_;
    gs[p] = g[p] * ds_;
    grho[p] = 0.0f;
  } else {
    gt[p] = 0.0f;
    gs[p] = 0.0f;
    grho[p] = g[p];
  }
}

// BAROPG of the column with c.F[rho]/[rmean]/[drhox]/[drhoy] pointing at
// the caller's arrays; rho_out = (rho - rmean) + rmean, the reference's
// round trip
__global__ void __launch_bounds__(128) k_baropg(Ctx c, float *rho_out) {
  const int n = c.im * c.jm;
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= n) return;
  const int j = col % c.jm, i = col / c.jm;
  baropg_column(c, i, j);
  for (int k = 0; k < c.kb; ++k) {
    const float rm = F3(rmean, i, j, k);
    rho_out[NPOM_I3(c, i, j, k)] = (F3(rho, i, j, k) - rm) + rm;
  }
}

template <int KM>
__global__ void __launch_bounds__(128) k_baropg_adj(Ctx c, Adj a, const float *gx, const float *gy) {
  const int n = c.im * c.jm;
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= n) return;
  const int j = col % c.jm, i = col / c.jm;
  if (!interior(c, i, j)) return;
  float lx[KM], ly[KM];
  for (int k = 0; k < c.kb; ++k) {
    lx[k] = gx[NPOM_I3(c, i, j, k)];
    ly[k] = gy[NPOM_I3(c, i, j, k)];
  }
  baropg_column_adj<KM>(c, a, i, j, lx, ly);
}

bool fields_ok(const npom_params *p, float *const *fields) {
  if (!p || !fields || p->im < 3 || p->jm < 3 || p->kb < 3 || p->kb > KMAX) return false;
  for (int f = 0; f < NPOM_NFIELDS; ++f)
    if (!fields[f]) return false;
  return cudaSetDevice(p->device) == cudaSuccess;
}

Ctx fields_ctx(const npom_params *p, float *const *fields) {
  Ctx c;
  std::memset(&c, 0, sizeof(c));
  c.im = p->im;
  c.jm = p->jm;
  c.kb = p->kb;
  for (int f = 0; f < NPOM_NFIELDS; ++f) c.F[f] = fields[f];
  c.k = make_consts(*p);
  c.ramp = 1.0f;
  c.do_internal = 1;
  return c;
}
