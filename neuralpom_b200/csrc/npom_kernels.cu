// npom_kernels.cu -- CUDA kernels for sm_100a and the C ABI of include/npom.h.
//
// A step is a fixed sequence of launches on the caller's stream:
//
//   A1  points   forcing + ADVCT                              (all cores)
//   A2  columns  BAROPG + Smagorinsky + depth integrals
//   A3  cells    rho round trip + ADVAVE + predictor (implicit)
//   E   coop     explicit: fused 30-substep external mode (3 grid barriers
//                per substep); implicit: fused PCG free-surface solve
//   I5  cells    implicit corrector + Robert-Asselin + shifts
//   B1..B9       internal mode (skipped on the very first step from rest)
//
// The cooperative kernels (PCG, external subcycle) keep every block resident
// (cudaLaunchCooperativeKernel) and synchronise through a counting grid
// barrier whose waits are bounded in time: a wait that runs out sets
// NPOM_DEV_TIMEOUT and the kernel returns instead of hanging.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include "npom_phases_int.cuh"
#include "npom_host.cuh"
#include "npom_pcg_cluster.cuh"
#include "npom_lanes.cuh"
#include "npom_adjoint.cuh"
#include "npom_mpdata.cuh"
#include "npom_mpdata_adjoint.cuh"

using namespace npom;

namespace {

constexpr int kThreads = 256;

// ---------------------------------------------------------------------------
// generic launch shapes
// ---------------------------------------------------------------------------
enum PointPhase { PP_A1 = 0, PP_B2B = 1, PP_B4 = 2, PP_B5 = 3, PP_B7 = 4 };
enum ColPhase { CP_A2 = 0, CP_B1 = 1, CP_B2A = 2, CP_B3 = 3, CP_B6 = 4, CP_B8 = 5, CP_B9 = 6 };
enum CellPhase { XP_A3 = 0, XP_I5 = 1, XP_COEF = 2, XP_I5A = 3 };

// The bodies below map one thread index of a phase onto its grid point,
// column or cell; the one-member kernels and the batched kernels (many
// members in one launch) call the same bodies.
template <int PH>
__device__ __forceinline__ void points_body(const Ctx &c, size_t p) {
  const size_t n = (size_t)c.im * c.jm * c.kb;
  if (p >= n) return;
  int k = (int)(p % c.kb);
  size_t col = p / c.kb;
  int j = (int)(col % c.jm);
  int i = (int)(col / c.jm);
  if (PH == PP_A1) {
    float ax, ay, cv;
    advct_point(c, i, j, k, ax, ay, cv);
    P3(advx, i, j, k) = ax;
    P3(advy, i, j, k) = ay;
    P3(curv, i, j, k) = cv;
    if (k == 0) forcing_cell(c, i, j);
  } else if (PH == PP_B2B) {
    phase_b2b_point(c, i, j, k);
  } else if (PH == PP_B4) {
    phase_b4_point(c, i, j, k);
  } else if (PH == PP_B5) {
    phase_b5_point(c, i, j, k);
  } else if (PH == PP_B7) {
    phase_b7_point(c, i, j, k);
  }
}

template <int PH>
__global__ void __launch_bounds__(kThreads) k_points(Ctx c) {
  points_body<PH>(c, (size_t)blockIdx.x * blockDim.x + threadIdx.x);
}

template <int PH>
__device__ __forceinline__ void cols_body(const Ctx &c, int col) {
  const int n = c.im * c.jm;
  if (col >= n) return;
  int j = col % c.jm, i = col / c.jm;
  if (PH == CP_A2) phase_a2_column(c, i, j);
  else if (PH == CP_B1) phase_b1_column(c, i, j);
  else if (PH == CP_B2A) phase_b2a_column(c, i, j);
  else if (PH == CP_B3) phase_b3_column(c, i, j);
  else if (PH == CP_B6) phase_b6_column(c, i, j);
  else if (PH == CP_B8) phase_b8_column(c, i, j);
  else if (PH == CP_B9) phase_b9_column(c, i, j);
}

template <int PH>
__global__ void __launch_bounds__(128) k_cols(Ctx c) {
  cols_body<PH>(c, blockIdx.x * blockDim.x + threadIdx.x);
}

// PROFT one thread per column at kb == 16: the level loops unroll and the
// column stays in registers
__global__ void __launch_bounds__(128) k_cols_b6_kb16(Ctx c) {
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col < c.im * c.jm) phase_b6_column<16>(c, col / c.jm, col % c.jm);
}

// One 16-lane segment per water column (kb == 16).  Threads past the last
// column work on a copy of it and store nothing, so that every shuffle sees
// all 32 lanes of its warp.
template <int PH>
__device__ __forceinline__ void lanes_body(const Ctx &c, int p) {
  const int ncol = c.im * c.jm;
  int col = p >> 4;
  const int k = p & (KL - 1);
  const bool st = col < ncol;
  if (!st) col = ncol - 1;
  const int j = col % c.jm, i = col / c.jm;
  if (PH == CP_A2) lane_a2(c, i, j, k, st);
  else if (PH == CP_B1) lane_b1(c, i, j, k, st);
  else if (PH == CP_B2A) lane_b2a(c, i, j, k, st);
  else if (PH == CP_B3) lane_b3(c, i, j, k, st);
  else if (PH == CP_B6) lane_b6(c, i, j, k, st);
  else if (PH == CP_B8) lane_b8(c, i, j, k, st);
  else if (PH == CP_B9) lane_b9(c, i, j, k, st);
}

template <int PH>
__global__ void __launch_bounds__(kThreads) k_lanes(Ctx c) {
  lanes_body<PH>(c, blockIdx.x * blockDim.x + threadIdx.x);
}

template <int PH>
__device__ __forceinline__ void cells_body(const Ctx &c, int cell) {
  const int n = c.im * c.jm;
  if (cell >= n) return;
  int j = cell % c.jm, i = cell / c.jm;
  if (PH == XP_A3) {
    phase_a3_cell(c, i, j);
  } else if (PH == XP_I5) {
    if (phase_i5_cell(c, i, j)) atomicOr(c.status, NPOM_DEV_VMAX);
  } else if (PH == XP_COEF) {
    elliptic_coeff_cell(c, i, j);
  } else if (PH == XP_I5A) {
    phase_i5a_cell(c, i, j);
  }
}

template <int PH>
__global__ void __launch_bounds__(kThreads) k_cells(Ctx c) {
  cells_body<PH>(c, blockIdx.x * blockDim.x + threadIdx.x);
}

// A1 on large grids: every face flux of ADVCT computed once.  A block holds
// kA1Cols output columns j (plus one halo column on each side) x 16 levels
// and marches along i: the x-direction fluxes and the previous row's
// curvature stay in registers, the y-direction fluxes and the curvature of
// neighbouring columns pass through shared memory.  Each flux is the same
// helper call, and the output expressions keep the point kernel's order,
// so the results are bitwise those of k_points<PP_A1>.
constexpr int kA1Cols = 16;
constexpr int kA1Threads = 16 * (kA1Cols + 2);

// strip bx of kA1Cols columns, rows [by * ichunk, (by + 1) * ichunk)
__device__ __forceinline__ void a1_tiles_body(const Ctx &c, int ichunk, int bx, int by) {
  __shared__ float s_yu[kA1Cols + 2][16], s_yv[kA1Cols + 2][16], s_cv[kA1Cols + 2][16];
  const int k = threadIdx.x & 15;
  const int r = threadIdx.x >> 4;  // row r holds column j0 - 1 + r
  const int j = bx * kA1Cols - 1 + r;
  const int i0 = by * ichunk, i1 = min(c.im, i0 + ichunk);
  const bool jin = j >= 0 && j < c.jm;
  const bool out_row = jin && r >= 1 && r <= kA1Cols;
  const bool lev = k < c.kb - 1;
  const int jc = jin ? j : 0;
  // the values of row i0 - 1 that the first output row needs
  float xu_prev = (jin && lev) ? advct_xflux_u(c, i0 - 1, jc, k) : 0.0f;
  float xv_cur = (jin && lev) ? advct_xflux_v(c, i0, jc, k) : 0.0f;
  float cv_prev = (jin && lev) ? advct_curv(c, i0 - 1, jc, k) : 0.0f;
  for (int i = i0; i < i1; ++i) {
    float xu = 0.0f, xv_next = 0.0f, yu = 0.0f, yv = 0.0f, cv = 0.0f;
    if (jin && lev) {
      xu = advct_xflux_u(c, i, jc, k);
      if (i + 1 < c.im) xv_next = advct_xflux_v(c, i + 1, jc, k);
      yu = advct_yflux_u(c, i, jc, k);
      yv = advct_yflux_v(c, i, jc, k);
      cv = advct_curv(c, i, jc, k);
    }
    s_yu[r][k] = yu;
    s_yv[r][k] = yv;
    s_cv[r][k] = cv;
    __syncthreads();
    if (out_row) {
      float ax = 0.0f, ay = 0.0f, co = 0.0f;
      if (lev && interior(c, i, j)) {
        co = cv;
        ax = xu - xu_prev + s_yu[r + 1][k] - yu;
        if (i >= 2) {
          float tc1 = cv * F2(dt, i, j) * (F3(v, i, j + 1, k) + F3(v, i, j, k));
          float tc2 = cv_prev * F2(dt, i - 1, j) * (F3(v, i - 1, j + 1, k) + F3(v, i - 1, j, k));
          ax -= F2(aru, i, j) * 0.25f * (tc1 + tc2);
        }
        ay = xv_next - xv_cur + yv - s_yv[r - 1][k];
        if (j >= 2) {
          float tc1 = cv * F2(dt, i, j) * (F3(u, i + 1, j, k) + F3(u, i, j, k));
          float tc2 = s_cv[r - 1][k] * F2(dt, i, j - 1) * (F3(u, i + 1, j - 1, k) + F3(u, i, j - 1, k));
          ay += F2(arv, i, j) * 0.25f * (tc1 + tc2);
        }
      }
      P3(advx, i, j, k) = ax;
      P3(advy, i, j, k) = ay;
      P3(curv, i, j, k) = co;
      if (k == 0) forcing_cell(c, i, j);
    }
    __syncthreads();
    xu_prev = xu;
    xv_cur = xv_next;
    cv_prev = cv;
  }
}

__global__ void __launch_bounds__(kA1Threads) k_a1_tiles(Ctx c, int ichunk) {
  a1_tiles_body(c, ichunk, blockIdx.x, blockIdx.y);
}

// B5 on large grids: the ADVT1 face fluxes of T and S computed once per
// face.  A block holds kB5Cols output columns (plus the column above) x 16
// levels and marches along i; the x-face fluxes stay in registers, the
// y-face fluxes of the column above pass through shared memory.  The output
// expressions are those of phase_b5_point, so the results are bitwise equal.
constexpr int kB5Cols = 16;
constexpr int kB5Threads = 16 * (kB5Cols + 1);

// strip bx of kB5Cols columns, rows [by * ichunk, (by + 1) * ichunk)
__device__ __forceinline__ void b5_tiles_body(const Ctx &c, int ichunk, int bx, int by) {
  __shared__ float s_yt[kB5Cols + 1][16], s_ys[kB5Cols + 1][16];
  const int k = threadIdx.x & 15;
  const int r = threadIdx.x >> 4;  // row r holds column j0 + r
  const int j = bx * kB5Cols + r;
  const int i0 = by * ichunk, i1 = min(c.im, i0 + ichunk);
  const bool jin = j < c.jm;
  const bool out_row = jin && r < kB5Cols;
  const bool lev = k < c.kb - 1;
  const int jc = jin ? j : 0;
  const float *t = c.F[NPOM_F_t], *tb = c.F[NPOM_F_tb], *tcl = c.F[NPOM_F_tclim];
  const float *sv = c.F[NPOM_F_s], *sb = c.F[NPOM_F_sb], *scl = c.F[NPOM_F_sclim];
  // x-face fluxes at i0 (faces exist for 1 <= i <= im-1)
  float xt = 0.0f, xs = 0.0f;
  if (jin && lev && i0 >= 1) {
    xt = advt1_xflux(c, t, tb, tcl, i0, jc, k);
    xs = advt1_xflux(c, sv, sb, scl, i0, jc, k);
  }
  for (int i = i0; i < i1; ++i) {
    float xt_n = 0.0f, xs_n = 0.0f, yt = 0.0f, ys = 0.0f;
    if (jin && lev) {
      if (i + 1 < c.im) {
        xt_n = advt1_xflux(c, t, tb, tcl, i + 1, jc, k);
        xs_n = advt1_xflux(c, sv, sb, scl, i + 1, jc, k);
      }
      if (jc >= 1) {
        yt = advt1_yflux(c, t, tb, tcl, i, jc, k);
        ys = advt1_yflux(c, sv, sb, scl, i, jc, k);
      }
    }
    s_yt[r][k] = yt;
    s_ys[r][k] = ys;
    __syncthreads();
    if (out_row) {
      phase_b5_filter(c, i, j, k);
      float tf_ = 0.0f, sf_ = 0.0f;
      if (lev && interior(c, i, j)) {
        tf_ = advt1_finish(c, t, tb, i, j, k, xt_n - xt + s_yt[r + 1][k] - yt);
        sf_ = advt1_finish(c, sv, sb, i, j, k, xs_n - xs + s_ys[r + 1][k] - ys);
      }
      phase_b5_store(c, i, j, k, tf_, sf_);
    }
    __syncthreads();
    xt = xt_n;
    xs = xs_n;
  }
}

__global__ void __launch_bounds__(kB5Threads) k_b5_tiles(Ctx c, int ichunk) {
  b5_tiles_body(c, ichunk, blockIdx.x, blockIdx.y);
}

// ---------------------------------------------------------------------------
// bounded grid barrier (all blocks co-resident: cooperative launch)
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned long long globaltimer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

constexpr unsigned long long kBarrierTimeoutNs = 2000000000ull;  // 2 s

// block count and block index within the blocks of this context
__device__ __forceinline__ unsigned vgrid(const Ctx &c) {
  return c.grid_blocks ? (unsigned)c.grid_blocks : gridDim.x;
}
__device__ __forceinline__ unsigned vblock(const Ctx &c) { return blockIdx.x - (unsigned)c.grid_base; }

// sync[0] counts arrivals and only grows during a launch (the host clears it
// before every cooperative launch): barrier b of the launch is complete when
// the count reaches (b + 1) * G (G the blocks of the context), so each
// block waits for the next
// multiple of the grid size above its own arrival.  One atomic per block
// and no reset inside the kernel keep each barrier at two serial L2 round
// trips.  Returns false after a timeout (or once any block has timed out);
// the caller then returns.
//
// Ordering: the block barrier orders every thread's writes before thread
// 0's arrival, a release at GPU scope; thread 0 polls with acquire loads,
// and the closing block barrier orders the acquire before every thread's
// later reads (which in the cooperative kernels go through L2).  The
// release/acquire pair replaces two full fences.
__device__ __forceinline__ unsigned int atom_add_release_gpu(unsigned int *p, unsigned int v) {
  unsigned int old;
  asm volatile("atom.add.release.gpu.global.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
  return old;
}
__device__ __forceinline__ unsigned int ld_acquire_gpu(const unsigned int *p) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ bool grid_barrier(const Ctx &c) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    ok = 1;
    const unsigned int arrived = atom_add_release_gpu(c.sync, 1u);
    const unsigned int G = vgrid(c);
    const unsigned int target = (arrived / G + 1u) * G;
    unsigned long long t0 = globaltimer_ns();
    unsigned int spins = 0;
    while ((int)(ld_acquire_gpu(c.sync) - target) < 0) {
      if ((++spins & 63u) == 0) {
        if (*(volatile unsigned int *)c.status & NPOM_DEV_TIMEOUT) {
          ok = 0;
          break;
        }
        if (globaltimer_ns() - t0 > kBarrierTimeoutNs) {
          atomicOr(c.status, NPOM_DEV_TIMEOUT);
          ok = 0;
          break;
        }
      }
    }
  }
  __syncthreads();
  return ok != 0;
}

// block-wide FP64 sum of three values, result written to partials[slot*G+b]
__device__ void block_sum3(const Ctx &c, double a0, double a1, double a2, int s0, int s1, int s2) {
  __shared__ double red[3][kThreads / 32];
  for (int off = 16; off > 0; off >>= 1) {
    a0 += __shfl_down_sync(0xffffffffu, a0, off);
    a1 += __shfl_down_sync(0xffffffffu, a1, off);
    a2 += __shfl_down_sync(0xffffffffu, a2, off);
  }
  int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) {
    red[0][w] = a0;
    red[1][w] = a1;
    red[2][w] = a2;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double t0 = 0.0, t1 = 0.0, t2 = 0.0;
    for (int q = 0; q < (int)(blockDim.x >> 5); ++q) {
      t0 += red[0][q];
      t1 += red[1][q];
      t2 += red[2][q];
    }
    const int G = vgrid(c), b = vblock(c);
    if (s0 >= 0) c.partials[s0 * G + b] = t0;
    if (s1 >= 0) c.partials[s1 * G + b] = t1;
    if (s2 >= 0) c.partials[s2 * G + b] = t2;
  }
  __syncthreads();
}

// sum of one partial slot over blocks, identical in every block
// (warp 0: lane l sums the partials l, l + 32, ... in order, then a fixed
// shuffle tree; the loads of the lanes are in flight together)
__device__ double grid_total(const Ctx &c, int slot) {
  __shared__ double tot;
  if (threadIdx.x < 32) {
    double t = 0.0;
    const int G = vgrid(c);
    for (int b = threadIdx.x; b < G; b += 32) t += __ldcg(c.partials + slot * G + b);
    for (int off = 16; off > 0; off >>= 1) t += __shfl_down_sync(0xffffffffu, t, off);
    if (threadIdx.x == 0) tot = t;
  }
  __syncthreads();
  double r = tot;
  __syncthreads();
  return r;
}

// The DST stages of the spectral preconditioner (dst_stage_i / dst_stage_j:
// out = Sx src along i, out = src Sy along j) over the ni x nj interior, in
// tiles of kDstRows x kDstCols outputs per block (one per thread): chunks of
// kDstChunk terms of both operands are staged in shared memory by coalesced
// loads, then every thread sums its output's terms in FP64 in index order,
// the order of dst_stage_i / dst_stage_j (so the values are theirs).  The
// tiles are dealt to the blocks of the context; epi(a, b, value) stores.
constexpr int kDstRows = 8, kDstCols = 32, kDstChunk = 64;
static_assert(kDstRows * kDstCols == kThreads, "one output per thread");
// dst_row_pairs (below): rows per group, largest interior side
constexpr int kDstBandRows = 4, kDstBandMax = 384;
constexpr int kDstTileFloats = kDstRows * (kDstChunk + 1) + kDstChunk * (kDstCols + 1);
constexpr int kDstSmemFloats =
    kDstTileFloats > 2 * kDstBandRows * kDstBandMax ? kDstTileFloats : 2 * kDstBandRows * kDstBandMax;

// The one shared-memory buffer of every DST stage instantiation of a kernel
// (a function-local static array of a non-template function is one array
// per kernel; arrays declared in the templates would be one per
// instantiation).
__device__ __forceinline__ float *dst_smem() {
  __shared__ float buf[kDstSmemFloats];
  return buf;
}

// SHARED: the staging arrays in dst_smem(), the buffer that dst_row_pairs
// also uses (kernels that compile both forms); otherwise arrays of each
// instantiation, as the one-member kernel has them.
template <bool ALONG_I, bool SHARED, class Epi>
__device__ __forceinline__ void dst_tiles(const Ctx &c, const float *src, bool src_is_grid, Epi &&epi) {
  float(*lt)[kDstChunk + 1];
  float(*rt)[kDstCols + 1];
  if constexpr (SHARED) {
    lt = reinterpret_cast<float(*)[kDstChunk + 1]>(dst_smem());
    rt = reinterpret_cast<float(*)[kDstCols + 1]>(dst_smem() + kDstRows * (kDstChunk + 1));
  } else {
    __shared__ float lt_own[kDstRows][kDstChunk + 1];
    __shared__ float rt_own[kDstChunk][kDstCols + 1];
    lt = lt_own;
    rt = rt_own;
  }
  // rows: the solve's unknowns (with periodic x the unique columns, Sx the
  // Hartley matrix of the period)
  const int i0 = pcg_i0(c), ni = c.im - 2 * i0, nj = c.jm - 2;
  const int K = ALONG_I ? ni : nj;
  const float *sx = c.W[NPOM_W_sx], *sy = c.W[NPOM_W_sy];
  const int tiles_b = (nj + kDstCols - 1) / kDstCols;
  const int tiles = ((ni + kDstRows - 1) / kDstRows) * tiles_b;
  const int tr = threadIdx.x / kDstCols, tc = threadIdx.x % kDstCols;
  for (int tile = (int)vblock(c); tile < tiles; tile += (int)vgrid(c)) {
    const int a0 = (tile / tiles_b) * kDstRows, b0 = (tile % tiles_b) * kDstCols;
    double acc = 0.0;
    for (int m0 = 0; m0 < K; m0 += kDstChunk) {
      const int mc = min(kDstChunk, K - m0);
      __syncthreads();  // the previous chunk is consumed
      for (int e = threadIdx.x; e < kDstRows * kDstChunk; e += blockDim.x) {
        const int r = e / kDstChunk, k = e % kDstChunk;
        float v = 0.0f;
        if (a0 + r < ni && k < mc)
          v = ALONG_I ? __ldcg(sx + (size_t)(a0 + r) * ni + m0 + k) : __ldcg(src + (size_t)(a0 + r) * nj + m0 + k);
        lt[r][k] = v;
      }
      for (int e = threadIdx.x; e < kDstChunk * kDstCols; e += blockDim.x) {
        const int k = e / kDstCols, col = e % kDstCols;
        float v = 0.0f;
        if (k < mc && b0 + col < nj) {
          if (!ALONG_I) v = __ldcg(sy + (size_t)(m0 + k) * nj + b0 + col);
          else if (src_is_grid) v = __ldcg(src + NPOM_I2(c, m0 + k + i0, b0 + col + 1));
          else v = __ldcg(src + (size_t)(m0 + k) * nj + b0 + col);
        }
        rt[k][col] = v;
      }
      __syncthreads();
      for (int k = 0; k < mc; ++k) acc += (double)lt[tr][k] * (double)rt[k][tc];
    }
    const int a = a0 + tr, b = b0 + tc;
    if (a < ni && b < nj) epi(a, b, (float)acc);
  }
}

// The DST stages in pairs (i-stage then j-stage) over bands of whole rows:
// the rows of the interior are split into one contiguous band per block of
// the context, and a block takes its band kDstBandRows rows at a time.  For
// each group it computes the i-stage row(s) mid[q][b] = sum_m Sx[a][m] src(m, b)
// over every column b, keeps them in shared memory, and then the j-stage
// sum_b mid[q][b] Sy[b][l] of the same rows, so no grid barrier separates
// the two stages.  Every output sums its terms in FP64 in index order, as
// dst_tiles does, so the values are the same bits.  src(m, b) gives the
// i-stage operand, epi(a, l, value) stores the j-stage output.  Interiors up
// to kDstBandMax in either direction (larger ones use dst_tiles).
// Used by the batched solve only.  Each thread runs its FP64 sums over L2
// loads with few in flight, which one member alone does not hide (by timing,
// not profiled: 177x161 alone 3.2 ms per step with the tiles, 4.0 with the
// pairs); in a batch the other members' blocks hide that latency and the
// two barriers saved per iteration win (64 mixed members: 8.4 -> 8.8
// member-days/s).
template <class Src, class Epi>
__device__ __forceinline__ void dst_row_pairs(const Ctx &c, Src &&src, Epi &&epi) {
  float(*sxr)[kDstBandMax] = reinterpret_cast<float(*)[kDstBandMax]>(dst_smem());
  float(*mid)[kDstBandMax] = reinterpret_cast<float(*)[kDstBandMax]>(dst_smem() + kDstBandRows * kDstBandMax);
  const int i0 = pcg_i0(c), ni = c.im - 2 * i0, nj = c.jm - 2;
  const float *sx = c.W[NPOM_W_sx], *sy = c.W[NPOM_W_sy];
  const int G = (int)vgrid(c), band = (ni + G - 1) / G;
  const int a_beg = (int)vblock(c) * band, a_end = min(ni, a_beg + band);
  for (int a0 = a_beg; a0 < a_end; a0 += kDstBandRows) {
    const int nr = min(kDstBandRows, a_end - a0);
    __syncthreads();  // the previous group is consumed
    for (int e = threadIdx.x; e < kDstBandRows * ni; e += blockDim.x) {
      const int q = e / ni, m = e - q * ni;
      sxr[q][m] = q < nr ? __ldcg(sx + (size_t)(a0 + q) * ni + m) : 0.0f;
    }
    __syncthreads();
    for (int b = threadIdx.x; b < nj; b += blockDim.x) {
      double acc[kDstBandRows];
#pragma unroll
      for (int q = 0; q < kDstBandRows; ++q) acc[q] = 0.0;
#pragma unroll 4
      for (int m = 0; m < ni; ++m) {
        const double v = (double)src(m, b);
#pragma unroll
        for (int q = 0; q < kDstBandRows; ++q) acc[q] += (double)sxr[q][m] * v;
      }
#pragma unroll
      for (int q = 0; q < kDstBandRows; ++q) mid[q][b] = (float)acc[q];
    }
    __syncthreads();
    for (int l = threadIdx.x; l < nj; l += blockDim.x) {
      double acc[kDstBandRows];
#pragma unroll
      for (int q = 0; q < kDstBandRows; ++q) acc[q] = 0.0;
#pragma unroll 4
      for (int b = 0; b < nj; ++b) {
        const double w = (double)__ldcg(sy + (size_t)b * nj + l);
#pragma unroll
        for (int q = 0; q < kDstBandRows; ++q) acc[q] += (double)mid[q][b] * w;
      }
#pragma unroll
      for (int q = 0; q < kDstBandRows; ++q)
        if (q < nr) epi(a0 + q, l, (float)acc[q]);
    }
  }
}

// z = M^-1 r over the interior; returns after its own trailing barrier.
// Accumulates r.z into *rz of this thread.  ROWS: the DST stages in row
// pairs (one grid barrier instead of three; the batched solve).
template <bool ROWS>
__device__ bool precondition(const Ctx &c, double &rz) {
  const int nj = c.jm - 2, i0 = pcg_i0(c);
  const size_t nint = (size_t)(c.im - 2 * i0) * nj;
  const size_t stride = (size_t)vgrid(c) * blockDim.x;
  const size_t tid = (size_t)vblock(c) * blockDim.x + threadIdx.x;
  float *zv = c.W[NPOM_W_zv];
  const float *r = c.W[NPOM_W_r];
  rz = 0.0;
  if (c.k.eta_precond == NPOM_PRECOND_SPECTRAL) {
    float *t1 = c.W[NPOM_W_t1], *t2 = c.W[NPOM_W_t2];
    const float *ie = c.W[NPOM_W_inv_eigs];
    const float inv_scale = c.k.inverse_scale;
    if (ROWS && c.im - 2 * i0 <= kDstBandMax && nj <= kDstBandMax) {
      // two stages per pass: one grid barrier instead of three
      dst_row_pairs(
          c, [&](int m, int b) { return __ldcg(r + NPOM_I2(c, m + i0, b + 1)); },
          [&](int a, int b, float v) {
            const size_t q = (size_t)a * nj + b;
            t2[q] = v * __ldcg(ie + q);
          });
      if (!grid_barrier(c)) return false;
      dst_row_pairs(
          c, [&](int m, int b) { return __ldcg(t2 + (size_t)m * nj + b); },
          [&](int a, int b, float v) {
            const float zval = v / inv_scale;
            const size_t o = NPOM_I2(c, a + i0, b + 1);
            zv[o] = zval;
            rz += (double)__ldcg(r + o) * (double)zval;
          });
      return true;
    }
    dst_tiles<true, ROWS>(c, r, true, [&](int a, int b, float v) { t1[(size_t)a * nj + b] = v; });
    if (!grid_barrier(c)) return false;
    dst_tiles<false, ROWS>(c, t1, false, [&](int a, int b, float v) {
      const size_t q = (size_t)a * nj + b;
      t2[q] = v * __ldcg(ie + q);
    });
    if (!grid_barrier(c)) return false;
    dst_tiles<true, ROWS>(c, t2, false, [&](int a, int b, float v) { t1[(size_t)a * nj + b] = v; });
    if (!grid_barrier(c)) return false;
    dst_tiles<false, ROWS>(c, t1, false, [&](int a, int b, float v) {
      const float zval = v / inv_scale;
      const size_t o = NPOM_I2(c, a + i0, b + 1);
      zv[o] = zval;
      rz += (double)__ldcg(r + o) * (double)zval;
    });
  } else {
    for (size_t q = tid; q < nint; q += stride) {
      int a = (int)(q / nj), b = (int)(q % nj);
      size_t o = NPOM_I2(c, a + i0, b + 1);
      float rv = __ldcg(r + o);
      float zval = rv / (__ldcg(c.W[NPOM_W_diag] + o) + 1e-30f);
      zv[o] = zval;
      rz += (double)rv * (double)zval;
    }
  }
  return true;
}

// Fused PCG free-surface solve (core.py:460-589, eager branch), followed by
// the Shapiro filter and closed-basin bcond 1 (core.py:893-916) and
// d = h + elf.  Iterations -> c.cg_iters[c.sync[2]++] (one slot per solve
// of the call).  ROWS as for precondition: the same values either way.
template <bool ROWS>
__device__ __forceinline__ void pcg_coop_body(const Ctx &c, int with_rhs, int with_post) {
  // unknowns: rows i0 .. im-1-i0 (the interior, or the unique columns of a
  // periodic-x basin)
  const int im = c.im, jm = c.jm, i0 = pcg_i0(c), nj = jm - 2;
  const size_t ncell = (size_t)im * jm, nint = (size_t)(im - 2 * i0) * nj;
  const size_t stride = (size_t)vgrid(c) * blockDim.x;
  const size_t tid = (size_t)vblock(c) * blockDim.x + threadIdx.x;
  float *x = c.W[NPOM_W_x], *r = c.W[NPOM_W_r], *p = c.W[NPOM_W_p], *zv = c.W[NPOM_W_zv];
  float *ap = c.W[NPOM_W_ap], *rhs = c.W[NPOM_W_rhs];
  const float *elf = c.F[NPOM_F_elf];
  // With the spectral preconditioner the Jacobi-diagonal plane is free and
  // holds the next search direction: the update p' = p * beta + z is then
  // computed inside the next operator apply (from the unchanged p and z)
  // instead of being stored first, which saves one grid barrier per
  // iteration with the same values.
  float *pnext = c.k.eta_precond == NPOM_PRECOND_SPECTRAL ? c.W[NPOM_W_diag] : nullptr;
  // setup: rhs (+ stored transports), initial guess with zero ring, zeroed
  // ring of every work vector
  for (size_t q = tid; q < ncell; q += stride) {
    int i = (int)(q / jm), j = (int)(q % jm);
    if (with_rhs) {
      rhs[q] = rhs_cell(c, i, j);
      P2(fluxua, i, j) = rhs_fluxua(c, i, j);
      P2(fluxva, i, j) = rhs_fluxva(c, i, j);
    } else if (!interior(c, i, j)) {
      rhs[q] = 0.0f;
    }
    bool in = interior(c, i, j);
    x[q] = in ? __ldcg(elf + q) : 0.0f;
    if (!in) {
      r[q] = 0.0f;
      p[q] = 0.0f;
      zv[q] = 0.0f;
      ap[q] = 0.0f;
      if (pnext) pnext[q] = 0.0f;
    }
  }
  if (!grid_barrier(c)) return;
  double rr = 0.0;
  for (size_t q = tid; q < nint; q += stride) {
    int i = (int)(q / nj) + i0, j = (int)(q % nj) + 1;
    size_t o = NPOM_I2(c, i, j);
    float a = elliptic_apply_cell(c, x, i, j);
    float rv = __ldcg(rhs + o) - a;
    r[o] = rv;
    rr += (double)rv * (double)rv;
    if (c.k.eta_precond != NPOM_PRECOND_SPECTRAL) c.W[NPOM_W_diag][o] = jacobi_diag_cell(c, i, j);
  }
  block_sum3(c, rr, 0.0, 0.0, 1, -1, -1);
  if (!grid_barrier(c)) return;
  double rz;
  if (!precondition<ROWS>(c, rz)) return;
  block_sum3(c, rz, 0.0, 0.0, 2, -1, -1);
  if (!grid_barrier(c)) return;
  double rs0 = grid_total(c, 1);
  double rho_old = grid_total(c, 2);
  for (size_t q = tid; q < nint; q += stride) {
    size_t o = NPOM_I2(c, (int)(q / nj) + i0, (int)(q % nj) + 1);
    p[o] = __ldcg(zv + o);
  }
  const double tol = pcg_abs_tol(c), tol_sq = tol * tol;
  const double rel_sq = c.k.eta_rel_tol * c.k.eta_rel_tol * (rs0 > 1e-30 ? rs0 : 1e-30);
  int its = 0;
  bool converged = false;
  if (!grid_barrier(c)) return;
  bool pending = false;  // p' = p * beta_p + z not stored yet
  float beta_p = 0.0f;
  for (int it = 1; it <= c.k.eta_max_iter; ++it) {
    double pap = 0.0;
    for (size_t q = tid; q < nint; q += stride) {
      int i = (int)(q / nj) + i0, j = (int)(q % nj) + 1;
      size_t o = NPOM_I2(c, i, j);
      float a, pv;
      if (pending) {
        a = elliptic_apply_cell_pz(c, p, zv, beta_p, i, j, &pv);
        pnext[o] = pv;  // read back by this thread only until the next barrier
      } else {
        a = elliptic_apply_cell(c, p, i, j);
        pv = __ldcg(p + o);
      }
      ap[o] = a;
      pap += (double)pv * (double)a;
    }
    if (pending) {
      float *t = p;
      p = pnext;
      pnext = t;
      pending = false;
    }
    block_sum3(c, pap, 0.0, 0.0, 0, -1, -1);
    if (!grid_barrier(c)) return;
    double denom = grid_total(c, 0);
    float alpha = (float)(rho_old / (denom + 1e-30));
    double rs = 0.0;
    for (size_t q = tid; q < nint; q += stride) {
      size_t o = NPOM_I2(c, (int)(q / nj) + i0, (int)(q % nj) + 1);
      x[o] = __ldcg(x + o) + alpha * __ldcg(p + o);
      float rv = __ldcg(r + o) - alpha * __ldcg(ap + o);
      r[o] = rv;
      rs += (double)rv * (double)rv;
    }
    block_sum3(c, rs, 0.0, 0.0, 1, -1, -1);
    if (!grid_barrier(c)) return;
    double rsn = grid_total(c, 1);
    its = it;
    if (rsn <= tol_sq || rsn <= rel_sq || rsn <= 1e-30) {
      converged = true;
      break;
    }
    if (!precondition<ROWS>(c, rz)) return;
    block_sum3(c, rz, 0.0, 0.0, 2, -1, -1);
    if (!grid_barrier(c)) return;
    double rho_new = grid_total(c, 2);
    float beta = (float)(rho_new / (rho_old + 1e-30));
    rho_old = rho_new;
    if (pnext) {
      pending = true;
      beta_p = beta;
      continue;
    }
    for (size_t q = tid; q < nint; q += stride) {
      size_t o = NPOM_I2(c, (int)(q / nj) + i0, (int)(q % nj) + 1);
      p[o] = __ldcg(p + o) * beta + __ldcg(zv + o);
    }
    if (!grid_barrier(c)) return;
  }
  if (tid == 0) {
    unsigned int slot = c.sync[2];
    c.cg_iters[slot] = its;
    c.sync[2] = slot + 1;
    if (!converged) atomicOr(c.status, NPOM_DEV_PCG_MAXIT);
  }
  if (!grid_barrier(c)) return;
  if (!with_post) {
    // raw solution into elf (the ring of x is zero; with periodic x the
    // halo columns are the copies of their unique columns)
    for (size_t q = tid; q < ncell; q += stride) {
      size_t src = q;
      if (c.k.periodic_x) {
        const int i = (int)(q / jm), j = (int)(q % jm);
        const int iw = i < 2 ? i + im - 4 : (i > im - 3 ? i - (im - 4) : i);
        src = NPOM_I2(c, iw, j);
      }
      c.F[NPOM_F_elf][q] = __ldcg(x + src);
    }
    return;
  }
  for (size_t q = tid; q < ncell; q += stride) {
    int i = (int)(q / jm), j = (int)(q % jm);
    float e = 0.0f;
    if (interior(c, i, j)) {
      float x0 = __ldcg(x + q);
      const size_t qe = NPOM_I2(c, pcg_east(c, i), j), qw = NPOM_I2(c, pcg_west(c, i), j);
      float sm = x0 + c.k.bshap_q * (__ldcg(x + qe) + __ldcg(x + qw) + __ldcg(x + q + 1) + __ldcg(x + q - 1) - 4.0f * x0);
      float fsm = F2(fsm, i, j);
      e = (sm * fsm) * fsm;
      if (!(fabsf(e) <= 3.0e38f)) atomicOr(c.status, NPOM_DEV_NONFINITE);
    }
    c.F[NPOM_F_elf][q] = e;
    c.F[NPOM_F_d][q] = F2(h, i, j) + e;
  }
}

template <bool ROWS>
__global__ void __launch_bounds__(kThreads) k_pcg(Ctx c, int with_rhs, int with_post) {
  pcg_coop_body<ROWS>(c, with_rhs, with_post);
}

// The tide policies' free-surface solve on the semi-implicit core
// (coastal_boundary.py:31-54, jzb_boundary.py:150-197), one cooperative
// launch: the RHS and stored transports as the production solve sets them
// up, then CG without preconditioner on the free nodes (the interior sea
// cells that are not tide cells) for the homogeneous problem A x = b,
// b = rhs - A(lift) (the tidal lift), with the cell areas as dot-product
// weights (FP64 sums), x0 = 0, at most min(max_iter, 500) iterations,
// stopping at the top of an iteration once rr <= max(1e-30, 1e-24 rr0);
// the count it + 1 goes to the iteration history; then elf = x + lift
// with the step's bcond 1 (policy_elf).  The depth is not updated (the
// step copy keeps the old d for the corrector).  Three grid barriers per
// iteration.
__device__ __forceinline__ void cg_policy_body(const Ctx &c) {
  const int im = c.im, jm = c.jm;
  const size_t ncell = (size_t)im * jm;
  const size_t stride = (size_t)vgrid(c) * blockDim.x;
  const size_t tid = (size_t)vblock(c) * blockDim.x + threadIdx.x;
  float *x = c.W[NPOM_W_x], *r = c.W[NPOM_W_r], *p = c.W[NPOM_W_p], *ap = c.W[NPOM_W_ap];
  float *rhs = c.W[NPOM_W_rhs], *lift = c.W[NPOM_W_zv];
  for (size_t q = tid; q < ncell; q += stride) {
    const int i = (int)(q / jm), j = (int)(q % jm);
    rhs[q] = rhs_cell(c, i, j);
    P2(fluxua, i, j) = rhs_fluxua(c, i, j);
    P2(fluxva, i, j) = rhs_fluxva(c, i, j);
    lift[q] = policy_lift(c, i, j);
  }
  if (!grid_barrier(c)) return;
  double rr = 0.0;
  for (size_t q = tid; q < ncell; q += stride) {
    const int i = (int)(q / jm), j = (int)(q % jm);
    const bool fixed = policy_fixed(c, i, j);
    const float b = fixed ? 0.0f : __ldcg(rhs + q) - elliptic_apply_cell(c, lift, i, j);
    x[q] = 0.0f;
    r[q] = b;
    p[q] = b;
    const float w = fixed ? 0.0f : F2(art, i, j);
    rr += (double)(w * b) * (double)b;
  }
  block_sum3(c, rr, 0.0, 0.0, 1, -1, -1);
  if (!grid_barrier(c)) return;
  rr = grid_total(c, 1);
  const double thr = fmax(1e-30, rr * 1e-24);
  const int nmax = c.k.eta_max_iter < 500 ? c.k.eta_max_iter : 500;
  int its = nmax;
  for (int it = 0; it < nmax; ++it) {
    if (rr <= thr) {
      its = it + 1;
      break;
    }
    double den = 0.0;
    for (size_t q = tid; q < ncell; q += stride) {
      const int i = (int)(q / jm), j = (int)(q % jm);
      const bool fixed = policy_fixed(c, i, j);
      const float a = fixed ? 0.0f : elliptic_apply_cell(c, p, i, j);
      ap[q] = a;
      const float w = fixed ? 0.0f : F2(art, i, j);
      den += (double)(w * __ldcg(p + q)) * (double)a;
    }
    block_sum3(c, den, 0.0, 0.0, 0, -1, -1);
    if (!grid_barrier(c)) return;
    const float alpha = (float)(rr / (grid_total(c, 0) + 1e-40));
    double nw = 0.0;
    for (size_t q = tid; q < ncell; q += stride) {
      const int i = (int)(q / jm), j = (int)(q % jm);
      x[q] = __ldcg(x + q) + alpha * __ldcg(p + q);
      const float rv = __ldcg(r + q) - alpha * __ldcg(ap + q);
      r[q] = rv;
      const float w = policy_fixed(c, i, j) ? 0.0f : F2(art, i, j);
      nw += (double)(w * rv) * (double)rv;
    }
    block_sum3(c, nw, 0.0, 0.0, 1, -1, -1);
    if (!grid_barrier(c)) return;
    nw = grid_total(c, 1);
    const float beta = (float)(nw / (rr + 1e-40));
    for (size_t q = tid; q < ncell; q += stride) p[q] = __ldcg(r + q) + beta * __ldcg(p + q);
    rr = nw;
    if (!grid_barrier(c)) return;
  }
  if (tid == 0) {
    unsigned int slot = c.sync[2];
    c.cg_iters[slot] = its;
    c.sync[2] = slot + 1;
  }
  for (size_t q = tid; q < ncell; q += stride) {
    const int i = (int)(q / jm), j = (int)(q % jm);
    const float e = policy_elf(c, x, i, j);
    if (!(fabsf(e) <= 3.0e38f)) atomicOr(c.status, NPOM_DEV_NONFINITE);
    P2(elf, i, j) = e;
  }
}

__global__ void __launch_bounds__(kThreads) k_cg_policy(Ctx c) { cg_policy_body(c); }

// block-wide FP64 maximum of a non-negative value into partials[slot*G+b]
__device__ void block_max(const Ctx &c, double a, int slot) {
  __shared__ double red[kThreads / 32];
  for (int off = 16; off > 0; off >>= 1) a = fmax(a, __shfl_down_sync(0xffffffffu, a, off));
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) red[w] = a;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int q = 0; q < (int)(blockDim.x >> 5); ++q) t = fmax(t, red[q]);
    c.partials[slot * vgrid(c) + vblock(c)] = t;
  }
  __syncthreads();
}

// maximum of one partial slot over blocks, identical in every block
__device__ double grid_max(const Ctx &c, int slot) {
  __shared__ double tot;
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (unsigned b = 0; b < vgrid(c); ++b) t = fmax(t, __ldcg(c.partials + slot * vgrid(c) + b));
    tot = t;
  }
  __syncthreads();
  const double r = tot;
  __syncthreads();
  return r;
}

// The seamount policy's free-surface solve on the semi-implicit core
// (seamount_boundary.py:57-103), one cooperative launch in FP64 on the
// robin planes (x, r, p, Ap, and the Picard guess G = ghost(x)): the step's
// RHS and stored transports as the production solve sets them up; x0 = el
// on the unknowns; up to 6 Picard iterations on the boundary depth, each a
// CG (at most 300 iterations, stopping at the top of an iteration once
// rr <= max(1e-28, 1e-22 rr0), rr0 = max(sum area b^2, 1e-40)) for the
// Robin operator of that guess, warm-started from x; done when
// max |ghost(x) - G| < 1e-11 m.  A non-positive or non-finite p.Ap sets
// NPOM_DEV_NONFINITE and stops; Picard iterations that do not converge
// set NPOM_DEV_PCG_MAXIT (the policy raises for both).  The CG iterations
// of all Picard passes go to the iteration history.  Then elf (sea_elf);
// the depth keeps its old value for the corrector.
__device__ __forceinline__ void robin_picard_body(const Ctx &c) {
  const int im = c.im, jm = c.jm;
  const size_t ncell = (size_t)im * jm;
  const size_t stride = (size_t)vgrid(c) * blockDim.x;
  const size_t tid = (size_t)vblock(c) * blockDim.x + threadIdx.x;
  double *X = c.robin, *R = c.robin + ncell, *P = c.robin + 2 * ncell, *AP = c.robin + 3 * ncell;
  double *G = c.robin + 4 * ncell;
  float *rhs = c.W[NPOM_W_rhs];
  for (size_t q = tid; q < ncell; q += stride) {
    const int i = (int)(q / jm), j = (int)(q % jm);
    rhs[q] = rhs_cell(c, i, j);
    P2(fluxua, i, j) = rhs_fluxua(c, i, j);
    P2(fluxva, i, j) = rhs_fluxva(c, i, j);
    X[q] = sea_free(c, i, j) ? (double)F2(el, i, j) : 0.0;
  }
  if (!grid_barrier(c)) return;
  bool converged = false;
  int total = 0;
  for (int nl = 0; nl < 6 && !converged; ++nl) {
    for (size_t q = tid; q < ncell; q += stride) G[q] = sea_ghost(c, X, (int)(q / jm), (int)(q % jm));
    if (!grid_barrier(c)) return;
    double rr = 0.0, bb = 0.0;
    for (size_t q = tid; q < ncell; q += stride) {
      const int i = (int)(q / jm), j = (int)(q % jm);
      const double b = sea_rhs(c, rhs, G, i, j);
      const double rv = b - sea_robin_op(c, X, G, i, j);
      R[q] = rv;
      P[q] = rv;
      const double area = sea_free(c, i, j) ? (double)F2(art, i, j) : 0.0;
      rr += area * rv * rv;
      bb += area * b * b;
    }
    block_sum3(c, rr, bb, 0.0, 1, 2, -1);
    if (!grid_barrier(c)) return;
    rr = grid_total(c, 1);
    const double rr0 = fmax(grid_total(c, 2), 1e-40);
    const double thr = fmax(1e-28, rr0 * 1e-22);
    for (int it = 0; it < 300; ++it) {
      if (rr <= thr) break;
      double den = 0.0;
      for (size_t q = tid; q < ncell; q += stride) {
        const int i = (int)(q / jm), j = (int)(q % jm);
        const double a = sea_robin_op(c, P, G, i, j);
        AP[q] = a;
        const double area = sea_free(c, i, j) ? (double)F2(art, i, j) : 0.0;
        den += area * __ldcg(P + q) * a;
      }
      block_sum3(c, den, 0.0, 0.0, 0, -1, -1);
      if (!grid_barrier(c)) return;
      den = grid_total(c, 0);
      if (!(den > 0.0) || !(den < 1.0e308)) {
        if (tid == 0) atomicOr(c.status, NPOM_DEV_NONFINITE);
        return;
      }
      const double a = rr / den;
      double nw = 0.0;
      for (size_t q = tid; q < ncell; q += stride) {
        const int i = (int)(q / jm), j = (int)(q % jm);
        X[q] = __ldcg(X + q) + a * __ldcg(P + q);
        const double rv = __ldcg(R + q) - a * __ldcg(AP + q);
        R[q] = rv;
        const double area = sea_free(c, i, j) ? (double)F2(art, i, j) : 0.0;
        nw += area * rv * rv;
      }
      block_sum3(c, nw, 0.0, 0.0, 1, -1, -1);
      if (!grid_barrier(c)) return;
      nw = grid_total(c, 1);
      const double beta = nw / fmax(rr, 1e-40);
      for (size_t q = tid; q < ncell; q += stride) P[q] = __ldcg(R + q) + beta * __ldcg(P + q);
      rr = nw;
      ++total;
      if (!grid_barrier(c)) return;
    }
    double change = 0.0;
    for (size_t q = tid; q < ncell; q += stride) {
      const int i = (int)(q / jm), j = (int)(q % jm);
      change = fmax(change, fabs(sea_ghost(c, X, i, j) - __ldcg(G + q)));
    }
    block_max(c, change, 3);
    if (!grid_barrier(c)) return;
    converged = grid_max(c, 3) < 1e-11;
  }
  if (tid == 0) {
    unsigned int slot = c.sync[2];
    c.cg_iters[slot] = total;
    c.sync[2] = slot + 1;
    if (!converged) atomicOr(c.status, NPOM_DEV_PCG_MAXIT);
  }
  for (size_t q = tid; q < ncell; q += stride) {
    const int i = (int)(q / jm), j = (int)(q % jm);
    const float e = sea_elf(c, X, i, j);
    if (!(fabsf(e) <= 3.0e38f)) atomicOr(c.status, NPOM_DEV_NONFINITE);
    P2(elf, i, j) = e;
  }
}

__global__ void __launch_bounds__(kThreads) k_robin_picard(Ctx c) { robin_picard_body(c); }

// the seamount policy's body continuity: the transports, then etf
__global__ void __launch_bounds__(kThreads) k_sea_continuity(Ctx c, int which) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= c.im * c.jm) return;
  const int i = q / c.jm, j = q % c.jm;
  if (which == 0) sea_transport_cell(c, i, j);
  else P2(etf, i, j) = sea_etf_cell(c, i, j);
}

// The coastal policy's bcond 2 lines (policy_bc2_line): jm + im lines
__global__ void __launch_bounds__(kThreads) k_policy_bc2(Ctx c, int which) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < c.jm + c.im) policy_bc2_line(c, t, which);
}

void launch_policy_bc2(const Ctx &c, int which, cudaStream_t s) {
  if (!c.k.obc_coastal || c.k.obc_jzb) return;
  const int n = c.jm + c.im;
  k_policy_bc2<<<(n + kThreads - 1) / kThreads, kThreads, 0, s>>>(c, which);
}

// Fused external mode of the explicit core: isplit substeps, three phases
// each (explicit/time_loop.py:292-431).
__device__ __forceinline__ void subcycle_coop_body(const Ctx &c) {
  const size_t ncell = (size_t)c.im * c.jm;
  const size_t stride = (size_t)vgrid(c) * blockDim.x;
  const size_t tid = (size_t)vblock(c) * blockDim.x + threadIdx.x;
  for (int iext = 1; iext <= c.k.isplit; ++iext) {
    bool adv = (iext % c.k.ispadv) == 0;
    for (size_t q = tid; q < ncell; q += stride) ext_phase1_cell(c, (int)(q / c.jm), (int)(q % c.jm), adv, iext);
    if (!grid_barrier(c)) return;
    bool exceed = false;
    for (size_t q = tid; q < ncell; q += stride) exceed |= ext_phase2_cell(c, (int)(q / c.jm), (int)(q % c.jm), iext);
    if (exceed) atomicOr(c.status, NPOM_DEV_VMAX);
    if (!grid_barrier(c)) return;
    for (size_t q = tid; q < ncell; q += stride) ext_phase3_cell(c, (int)(q / c.jm), (int)(q % c.jm), iext);
    if (!grid_barrier(c)) return;
  }
}

__global__ void __launch_bounds__(kThreads) k_subcycle(Ctx c) { subcycle_coop_body(c); }

// The same subcycle for grids of up to kSubClusterCells cells, on one
// thread-block cluster of at most 16 CTAs of 256, 512 or 1024 threads (the
// fewest that give every cell its own thread): the three phases of a
// substep are separated by the hardware cluster barrier (release/acquire at
// cluster scope covers the global-memory state; loads bypass L1) instead of
// the global-memory grid barrier, about a fifth of its latency.  Every CTA
// runs the same loop, so every barrier is reached by all of them.
constexpr int kSubClusterMax = 16;
constexpr size_t kSubClusterCells = (size_t)kSubClusterMax * 1024;

template <int T>
__global__ void __launch_bounds__(T, 1) k_subcycle_cluster(Ctx c) {
  cgx::cluster_group cl = cgx::this_cluster();
  const size_t ncell = (size_t)c.im * c.jm;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  for (int iext = 1; iext <= c.k.isplit; ++iext) {
    bool adv = (iext % c.k.ispadv) == 0;
    for (size_t q = tid; q < ncell; q += stride) ext_phase1_cell(c, (int)(q / c.jm), (int)(q % c.jm), adv, iext);
    cl.sync();
    bool exceed = false;
    for (size_t q = tid; q < ncell; q += stride) exceed |= ext_phase2_cell(c, (int)(q / c.jm), (int)(q % c.jm), iext);
    if (exceed) atomicOr(c.status, NPOM_DEV_VMAX);
    cl.sync();
    for (size_t q = tid; q < ncell; q += stride) ext_phase3_cell(c, (int)(q / c.jm), (int)(q % c.jm), iext);
    cl.sync();
  }
}

// A cluster launch shape, encoded as a negative int (positive values are
// grid-barrier block counts): -(ctas * 4 + log2(threads / 256)).
int encode_cluster(int ctas, int threads) { return -(ctas * 4 + (threads == 256 ? 0 : (threads == 512 ? 1 : 2))); }
int cluster_ctas(int code) { return (-code) / 4; }
int cluster_threads(int code) { return 256 << ((-code) % 4); }

cudaError_t launch_cluster(const void *fn, int ctas, int threads, void **args, cudaStream_t s) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(ctas);
  cfg.blockDim = dim3(threads);
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = ctas;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelExC(&cfg, fn, args);
}

// Shape of one cluster covering ncell cells with the kernel instance fn[t]
// of 256 << t threads: the fewest threads per CTA that give each cell its
// own thread, halving the CTA count while the cluster does not fit on a GPC.
// Sets the non-portable cluster-size attribute once per kernel and device.
cudaError_t plan_cluster(const void *const fn[3], size_t ncell, int *out) {
  const int t = ncell <= 16 * 256 ? 0 : (ncell <= 16 * 512 ? 1 : 2);
  const int threads = 256 << t;
  static std::mutex mu;
  static std::vector<std::pair<const void *, int>> done;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  {
    std::lock_guard<std::mutex> lock(mu);
    bool seen = false;
    for (auto &d : done) seen |= (d.first == fn[t] && d.second == dev);
    if (!seen) {
      e = cudaFuncSetAttribute(fn[t], cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
      if (e != cudaSuccess) return e;
      done.emplace_back(fn[t], dev);
    }
  }
  int ctas = (int)std::max<size_t>(1, std::min<size_t>(kSubClusterMax, (ncell + threads - 1) / threads));
  for (; ctas > 1; ctas /= 2) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(ctas);
    cfg.blockDim = dim3(threads);
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = ctas;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int nclusters = 0;
    e = cudaOccupancyMaxActiveClusters(&nclusters, fn[t], &cfg);
    if (e == cudaSuccess && nclusters > 0) break;
    cudaGetLastError();
  }
  *out = encode_cluster(ctas, threads);
  return cudaSuccess;
}

const void *const kSubcycleCluster[3] = {(const void *)k_subcycle_cluster<256>, (const void *)k_subcycle_cluster<512>,
                                         (const void *)k_subcycle_cluster<1024>};

// PROFT over independent columns (TracersMixin.proft, any kb <= KMAX)
__global__ void __launch_bounds__(128) k_proft(int ncol, int kb, const float *f_in, const float *wfsurf,
                                               const float *fsurf, int nbc, const float *h, const float *etf,
                                               float dti2, const float *dz, const float *dzz, const float *swrad,
                                               int ntp, const float *kh, float umol, const float *z, float *f_out,
                                               float *dh_out) {
  int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= ncol) return;
  ProftCol q;
  q.f = f_in + (size_t)col * kb;
  float tmp[KMAX];
  q.out = tmp;
  q.kh = kh + (size_t)col * kb;
  q.dz = dz;
  q.dzz = dzz;
  q.z = z;
  q.kb = kb;
  q.nbc = nbc;
  q.ntp = ntp;
  q.dti2 = dti2;
  q.umol = umol;
  q.h = h[col];
  q.etf = etf[col];
  q.swrad = swrad[col];
  q.wfsurf = wfsurf[col];
  q.fsurf = fsurf[col];
  float dh = proft_column(q);
  for (int k = 0; k < kb; ++k) f_out[(size_t)col * kb + k] = tmp[k];
  dh_out[col] = dh;
}

// ---------------------------------------------------------------------------
// host helpers
// ---------------------------------------------------------------------------
bool check_args_dev(const npom_params *p, float *const *fields, const npom_workspace *ws) {
  if (!check_args(p, fields, ws)) return false;
  return cudaSetDevice(p->device) == cudaSuccess;
}

int blocks_for(size_t n, int threads) { return (int)((n + threads - 1) / threads); }

cudaError_t coop_blocks(const void *fn, size_t work, int *out) {
  int dev = 0, sms = 0, per_sm = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return e;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kThreads, 0);
  if (e != cudaSuccess) return e;
  int want = std::max(1, blocks_for(work, kThreads));
  int cap = std::max(1, std::min(per_sm * sms, NPOM_MAX_COOP_BLOCKS));
  *out = std::min(want, cap);
  return cudaSuccess;
}

// Clears the barrier's arrival counter, then launches with every block
// co-resident.
cudaError_t launch_coop(const void *fn, int blocks, void **args, unsigned int *counter, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(unsigned int), s);
  if (e != cudaSuccess) return e;
  return cudaLaunchCooperativeKernel(fn, dim3(blocks), dim3(kThreads), args, 0, s);
}

template <int PH>
void launch_points(const Ctx &c, cudaStream_t s) {
  size_t n = (size_t)c.im * c.jm * c.kb;
  k_points<PH><<<blocks_for(n, kThreads), kThreads, 0, s>>>(c);
}
// Column phases: with kb == 16 one 16-lane segment per column (lane = level,
// npom_lanes.cuh); otherwise one thread per column.  NPOM_LANES=0 forces the
// thread-per-column bodies.
bool lanes_enabled(const Ctx &c) {
  if (c.kb != KL) return false;
  const char *env = getenv("NPOM_LANES");
  if (env) return std::strcmp(env, "0") != 0;
  return c.tune.column_form != 2;
}

// Columns from which PROFT runs one thread per column: its lane form issues
// every step of the sequential sweeps for the whole segment (~70x the
// instructions per column), which only pays while columns are too few to
// fill the GPU.  With 16 levels fixed at compile time (k_cols_b6_kb16) the
// thread-per-column form is the faster one at every size measured (90x82:
// 18.9 against 28.3 us; 354x322: 73 against 215 us).  Both forms compute
// bitwise the same values.
constexpr size_t kProftThreadColumns = 16384;

template <int PH>
void launch_cols(const Ctx &c, cudaStream_t s) {
  size_t n = (size_t)c.im * c.jm;
  const bool proft_threads =
      PH == CP_B6 && (n >= kProftThreadColumns || c.kb == 16) && c.tune.column_form != 1;
  // the POM08-WAD PROFQ has only the thread-per-column body
  const bool pom08 = PH == CP_B3 && c.k.profq_pom08;
  if (lanes_enabled(c) && !proft_threads && !pom08) {
    k_lanes<PH><<<blocks_for(n * KL, kThreads), kThreads, 0, s>>>(c);
  } else if (PH == CP_B6 && c.kb == 16) {
    k_cols_b6_kb16<<<blocks_for(n, 128), 128, 0, s>>>(c);
  } else {
    k_cols<PH><<<blocks_for(n, 128), 128, 0, s>>>(c);
  }
}
template <int PH>
void launch_cells(const Ctx &c, cudaStream_t s) {
  size_t n = (size_t)c.im * c.jm;
  k_cells<PH><<<blocks_for(n, kThreads), kThreads, 0, s>>>(c);
}

// Cluster PCG when the interior fits in one cluster's shared memory (8 CTAs,
// or 16 with the non-portable cluster size), first with the Sy fragment
// table in shared memory, then with Sy read from global memory (128x112
// interiors); NPOM_PCG=coop forces the grid-barrier kernel,
// NPOM_PCG_CTAS=16 prefers the 16-CTA cluster.
bool pcg_cluster_layout(const Ctx &c, ClusterLayout *out) {
  // periodic x: the cooperative grid form, whose operator wraps its x
  // neighbours (the cluster forms' slabs assume the Dirichlet ring)
  if (c.k.periodic_x) return false;
  const char *env = getenv("NPOM_PCG");
  if (env && std::strcmp(env, "coop") == 0) return false;
  if (!env && c.tune.pcg_form == 3) return false;
  int dev = 0, optin = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return false;
  if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess) return false;
  const char *ctas = getenv("NPOM_PCG_CTAS");
  const bool prefer16 = ctas ? std::strcmp(ctas, "16") == 0 : c.tune.pcg_ctas == 16;
  // the replicated-residual form where its extra full-grid copy fits, with
  // its exchanges by bulk copies and mbarriers where the rows allow them;
  // NPOM_PCG=sync keeps the replicated form with cluster barriers,
  // NPOM_PCG=pushed the pushed-residual form (four barriers), for comparisons
  const bool spectral = c.k.eta_precond == NPOM_PRECOND_SPECTRAL;
  const bool pushed = env ? std::strcmp(env, "pushed") == 0 : c.tune.pcg_form == 1;
  const bool sync = env ? std::strcmp(env, "sync") == 0 : c.tune.pcg_form == 2;
  const bool allow_rep = spectral && !pushed;
  const bool allow_bulk = allow_rep && !sync;
  const bool forms[3][2] = {{true, true}, {true, false}, {false, false}};  // (replicated, bulk)
  for (bool sy_global : {false, true}) {
    for (int nc : {prefer16 ? 16 : 8, prefer16 ? 8 : 16}) {
      for (const auto &f : forms) {
        if ((f[0] && !allow_rep) || (f[1] && !allow_bulk)) continue;
        ClusterLayout L = cluster_layout(c.im, c.jm, nc, sy_global, f[0], f[1]);
        if (f[1] && !L.bulk) continue;
        if (L.fits && L.bytes() <= (size_t)optin) {
          *out = L;
          return true;
        }
      }
    }
  }
  return false;
}

// Kernel attributes are set once per device (not inside graph captures).
// The cluster PCG kernel instance of a layout.
const void *pcg_cluster_fn(const ClusterLayout &L) {
  return L.sy_global ? (const void *)k_pcg_cluster<true> : (const void *)k_pcg_cluster<false>;
}

bool ensure_cluster_attrs(const ClusterLayout &L) {
  static std::mutex mu;
  static int smem_set[64][2] = {};
  static bool nonportable[64][2] = {};
  std::lock_guard<std::mutex> lock(mu);
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return false;
  const void *fn = pcg_cluster_fn(L);
  const int v = L.sy_global ? 1 : 0;
  if ((int)L.bytes() > smem_set[dev][v]) {
    if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.bytes()) != cudaSuccess)
      return false;
    smem_set[dev][v] = (int)L.bytes();
  }
  if (L.nc > 8 && !nonportable[dev][v]) {
    if (cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) return false;
    nonportable[dev][v] = true;
  }
  return true;
}

cudaError_t run_pcg_cluster(const Ctx &c, const ClusterLayout &L, int with_rhs, int with_post, cudaStream_t s) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(L.nc);
  cfg.blockDim = dim3(kClusterThreads);
  cfg.dynamicSmemBytes = L.bytes();
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = L.nc;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if (L.sy_global) return cudaLaunchKernelEx(&cfg, k_pcg_cluster<true>, c, L, with_rhs, with_post);
  return cudaLaunchKernelEx(&cfg, k_pcg_cluster<false>, c, L, with_rhs, with_post);
}

// Launch shape of the PCG for this grid, decided outside any capture.
struct PcgPlan {
  bool cluster;
  ClusterLayout L;
  int coop_blocks;
};

// true when at least one cluster of nc CTAs of kClusterThreads with smem
// bytes of dynamic shared memory can be resident (attributes already set)
bool cluster_launchable(const void *fn, int nc, size_t smem) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(nc);
  cfg.blockDim = dim3(kClusterThreads);
  cfg.dynamicSmemBytes = smem;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = nc;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int n = 0;
  if (cudaOccupancyMaxActiveClusters(&n, fn, &cfg) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return n > 0;
}

// Work of the grid-barrier PCG in threads: one per interior cell, and at
// least one block per DST tile (a block holding two tiles would double
// every DST stage).
// The one-member cooperative solve: DST stages as tiles; NPOM_PCG_DST=rows
// selects the batched solve's row pairs (the same values), for comparisons.
const void *pcg_coop_fn() {
  const char *e = getenv("NPOM_PCG_DST");
  return (e && std::strcmp(e, "rows") == 0) ? (const void *)k_pcg<true> : (const void *)k_pcg<false>;
}

size_t pcg_coop_work(const Ctx &c) {
  const size_t ni = (size_t)(c.im - 2), nj = (size_t)(c.jm - 2);
  size_t work = ni * nj;
  if (c.k.eta_precond == NPOM_PRECOND_SPECTRAL) {
    const size_t tiles = ((ni + kDstRows - 1) / kDstRows) * ((nj + kDstCols - 1) / kDstCols);
    work = std::max(work, tiles * (size_t)kThreads);
  }
  return work;
}

cudaError_t plan_pcg(const Ctx &c, PcgPlan *plan) {
  plan->coop_blocks = 0;
  if (c.k.obc_coastal) {
    // the tide policies' own solve (k_cg_policy)
    plan->cluster = false;
    return coop_blocks((const void *)k_cg_policy, (size_t)c.im * c.jm, &plan->coop_blocks);
  }
  if (c.k.sea_implicit) {
    // the seamount policy's Robin / Picard solve (k_robin_picard)
    plan->cluster = false;
    return coop_blocks((const void *)k_robin_picard, (size_t)c.im * c.jm, &plan->coop_blocks);
  }
  plan->cluster = pcg_cluster_layout(c, &plan->L) && ensure_cluster_attrs(plan->L) &&
                  cluster_launchable(pcg_cluster_fn(plan->L), plan->L.nc, plan->L.bytes());
  if (plan->cluster) return cudaSuccess;
  return coop_blocks(pcg_coop_fn(), pcg_coop_work(c), &plan->coop_blocks);
}

cudaError_t run_pcg(Ctx c, const PcgPlan &plan, int with_rhs, int with_post, cudaStream_t s) {
  if (c.k.obc_coastal || c.k.sea_implicit) {
    // the policy solves always set up their RHS and apply their bcond 1
    c.coh = 1;
    void *args[] = {&c};
    return launch_coop(c.k.sea_implicit ? (const void *)k_robin_picard : (const void *)k_cg_policy,
                       plan.coop_blocks, args, c.sync, s);
  }
  if (plan.cluster) return run_pcg_cluster(c, plan.L, with_rhs, with_post, s);
  c.coh = 1;
  void *args[] = {&c, &with_rhs, &with_post};
  return launch_coop(pcg_coop_fn(), plan.coop_blocks, args, c.sync, s);
}

// Launch shape of the explicit subcycle, decided outside any capture:
// > 0 grid-barrier blocks, < 0 a cluster shape (encode_cluster), 0 one
// launch per substep phase.  NPOM_SUBCYCLE=grid forces the grid-barrier
// form on small grids too; NPOM_SUBCYCLE=phases the per-phase launches,
// which need no co-residency (for many members advanced concurrently on
// one GPU, where a cooperative grid may not find all its blocks resident);
// NPOM_SUBCYCLE=nocoop the cluster form up to kSubClusterCellsShared cells
// (up to four cells per thread: one 16-SM cluster per member leaves the
// rest of the GPU to the other members), else the per-phase launches (a
// cluster is co-scheduled by the hardware, a cooperative grid is not when
// other streams hold SMs).
constexpr size_t kSubClusterCellsShared = 4 * kSubClusterCells;

cudaError_t plan_subcycle(const Ctx &c, int *out) {
  const size_t ncell = (size_t)c.im * c.jm;
  const char *env = getenv("NPOM_SUBCYCLE");
  const int form = c.tune.subcycle_form;
  const bool nocoop = env && std::strcmp(env, "nocoop") == 0;
  const bool phases = env ? std::strcmp(env, "phases") == 0 : form == 3;
  if (phases || (nocoop && ncell > kSubClusterCellsShared)) {
    *out = 0;
    return cudaSuccess;
  }
  if (nocoop) return plan_cluster(kSubcycleCluster, ncell, out);
  const bool grid = env ? std::strcmp(env, "grid") == 0 : form == 2;
  if (!grid && ncell <= kSubClusterCells) return plan_cluster(kSubcycleCluster, ncell, out);
  return coop_blocks((const void *)k_subcycle, ncell, out);
}

// one phase (1, 2, 3) of one external substep at cell q
__device__ __forceinline__ void ext_phase_body(const Ctx &c, int phase, int iext, int adv, int q) {
  if (q >= c.im * c.jm) return;
  const int i = q / c.jm, j = q % c.jm;
  if (phase == 1) ext_phase1_cell(c, i, j, adv != 0, iext);
  else if (phase == 2) {
    if (ext_phase2_cell(c, i, j, iext)) atomicOr(c.status, NPOM_DEV_VMAX);
  } else ext_phase3_cell(c, i, j, iext);
}

__global__ void __launch_bounds__(kThreads) k_ext_phase(Ctx c, int phase, int iext, int adv) {
  ext_phase_body(c, phase, iext, adv, blockIdx.x * blockDim.x + threadIdx.x);
}

cudaError_t run_subcycle(Ctx c, int blocks, cudaStream_t s) {
  if (blocks == 0) {
    const int n = c.im * c.jm;
    const unsigned g = (unsigned)((n + kThreads - 1) / kThreads);
    for (int iext = 1; iext <= c.k.isplit; ++iext) {
      const int adv = (iext % c.k.ispadv) == 0;
      for (int ph = 1; ph <= 3; ++ph) k_ext_phase<<<g, kThreads, 0, s>>>(c, ph, iext, adv);
    }
    return cudaGetLastError();
  }
  c.coh = 1;
  void *args[] = {&c};
  if (blocks < 0) {
    const int threads = cluster_threads(blocks);
    const int t = threads == 256 ? 0 : (threads == 512 ? 1 : 2);
    return launch_cluster(kSubcycleCluster[t], cluster_ctas(blocks), threads, args, s);
  }
  return launch_coop((const void *)k_subcycle, blocks, args, c.sync, s);
}

void launch_b5(const Ctx &c, cudaStream_t s);

// The seamount policy's Orlanski edges, one thread per (j, k): which 0 the
// u edges (bcond 3, after B8), 1 the T/S edges (bcond 4, after B6).
__global__ void __launch_bounds__(kThreads) k_obc_seamount(Ctx c, int which) {
  const int n = c.jm * c.kb;
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  if (which == 0) obc_seamount_u_point(c, q / c.kb, q % c.kb);
  else obc_seamount_ts_point(c, q / c.kb, q % c.kb);
}

void launch_obc_seamount(const Ctx &c, int which, cudaStream_t s) {
  if (!c.k.obc_seamount) return;
  const int n = c.jm * c.kb;
  k_obc_seamount<<<(n + kThreads - 1) / kThreads, kThreads, 0, s>>>(c, which);
}

// The periodic-x halo copy after a phase: in every plane of the state (the
// 2-D geometry and state, the 3-D state) and the workspace planes that
// carry values from one phase to the next, columns 0, 1 take im-4, im-3
// and columns im-2, im-1 take 2, 3.  Sources are unique columns and
// destinations halo columns (im >= 8), so the copies are independent.
// Planes are (i, j[, k]) with i slowest: a column is jm*depth contiguous
// floats.  blockIdx.y is the plane.
constexpr int kWrapGeom = NPOM_F_north_e - NPOM_F_h + 1;
constexpr int kWrap3d = NPOM_F_curv - NPOM_F_u + 1;
constexpr int kWrap2d = NPOM_F_ssurf - NPOM_F_el + 1;
constexpr int kWrapPlanes = kWrapGeom + kWrap3d + kWrap2d + 5;

// the workspace planes read by a later phase: us, vs, den_u, den_v, d_baro
__device__ __forceinline__ int wrap_ws(int w) {
  return w == 0 ? NPOM_W_us : w == 1 ? NPOM_W_vs : w == 2 ? NPOM_W_den_u : w == 3 ? NPOM_W_den_v : NPOM_W_d_baro;
}

__global__ void __launch_bounds__(kThreads) k_wrap_x(Ctx c) {
  const int slot = blockIdx.y;
  float *a;
  int depth = 1;
  if (slot < kWrapGeom) {
    a = c.F[NPOM_F_h + slot];
  } else if (slot < kWrapGeom + kWrap3d) {
    a = c.F[NPOM_F_u + slot - kWrapGeom];
    depth = c.kb;
  } else if (slot < kWrapGeom + kWrap3d + kWrap2d) {
    a = c.F[NPOM_F_el + slot - kWrapGeom - kWrap3d];
  } else {
    a = c.W[wrap_ws(slot - kWrapGeom - kWrap3d - kWrap2d)];
  }
  const size_t col = (size_t)c.jm * depth;
  const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= 4 * col) return;
  const int which = (int)(e / col);
  const size_t off = e - (size_t)which * col;
  const int im = c.im;
  const int dst = which == 0 ? 0 : which == 1 ? 1 : which == 2 ? im - 2 : im - 1;
  const int src = which == 0 ? im - 4 : which == 1 ? im - 3 : which == 2 ? 2 : 3;
  a[(size_t)dst * col + off] = a[(size_t)src * col + off];
}

void launch_wrap_x(const Ctx &c, cudaStream_t s) {
  if (!c.k.periodic_x) return;
  const size_t n = 4 * (size_t)c.jm * c.kb;
  k_wrap_x<<<dim3((unsigned)((n + kThreads - 1) / kThreads), kWrapPlanes), kThreads, 0, s>>>(c);
}

void internal_mode(const Ctx &c, cudaStream_t s) {
  launch_cols<CP_B1>(c, s);
  launch_wrap_x(c, s);
  launch_cols<CP_B2A>(c, s);
  launch_wrap_x(c, s);
  launch_points<PP_B2B>(c, s);
  launch_wrap_x(c, s);
  launch_cols<CP_B3>(c, s);
  launch_wrap_x(c, s);
  launch_points<PP_B4>(c, s);
  launch_wrap_x(c, s);
  launch_b5(c, s);
  launch_wrap_x(c, s);
  launch_cols<CP_B6>(c, s);
  launch_wrap_x(c, s);
  launch_obc_seamount(c, 1, s);
  launch_points<PP_B7>(c, s);
  launch_wrap_x(c, s);
  launch_cols<CP_B8>(c, s);
  launch_wrap_x(c, s);
  launch_obc_seamount(c, 0, s);
}

// Enqueue one internal step (all its kernels) on s.
// A1 runs as flux-once tiles from kTileCells cells on (kb == 16; the point
// kernel below that, where it has more threads in flight); NPOM_A1=tiles or
// NPOM_A1=points forces either form.
constexpr size_t kTileCells = 16384;

void launch_a1(const Ctx &c, cudaStream_t s) {
  const size_t ncell = (size_t)c.im * c.jm;
  const char *env = getenv("NPOM_A1");
  bool tiles = c.kb == 16 && ncell >= kTileCells;
  if (!env && c.tune.a1_form) tiles = c.kb == 16 && c.tune.a1_form == 2;
  if (env && c.kb == 16 && std::strcmp(env, "tiles") == 0) tiles = true;
  if (env && std::strcmp(env, "points") == 0) tiles = false;
  if (!tiles) {
    launch_points<PP_A1>(c, s);
    return;
  }
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int strips = (c.jm + kA1Cols - 1) / kA1Cols;
  // short marches, many blocks: ~16 blocks per SM (measured best at 354x322)
  const int per_sm = c.tune.tile_blocks_per_sm > 0 ? c.tune.tile_blocks_per_sm : 16;
  const int want = std::max(1, (per_sm * sms + strips - 1) / strips);
  const int ichunk = std::max(2, (c.im + want - 1) / want);
  const int chunks = (c.im + ichunk - 1) / ichunk;
  k_a1_tiles<<<dim3(strips, chunks), kA1Threads, 0, s>>>(c, ichunk);
}

// B5 the same way: flux-once tiles from kTileCells cells on (kb == 16, not
// in mode 4); NPOM_B5=tiles or NPOM_B5=points forces either form.
__device__ __forceinline__ void mpdata_body(const Ctx &c, int pass, int itera, size_t p) {
  const size_t n = (size_t)c.im * c.jm * c.kb;
  if (p >= n) return;
  const int k = (int)(p % c.kb);
  const size_t col = p / c.kb;
  phase_b5_mpdata_point(c, pass, itera, (int)(col / c.jm), (int)(col % c.jm), k);
}

__global__ void __launch_bounds__(kThreads) k_mpdata(Ctx c, int pass, int itera) {
  mpdata_body(c, pass, itera, (size_t)blockIdx.x * blockDim.x + threadIdx.x);
}

// B5 with MPDATA tracer advection (nadv 2): the filter, then ADVT2's passes
// for T and S together, nitera iterations
void launch_b5_mpdata(const Ctx &c, cudaStream_t s) {
  const size_t n = (size_t)c.im * c.jm * c.kb;
  const unsigned g = (unsigned)((n + kThreads - 1) / kThreads);
  k_mpdata<<<g, kThreads, 0, s>>>(c, MP_FILTER, 0);
  k_mpdata<<<g, kThreads, 0, s>>>(c, MP_INIT, 0);
  for (int it = 1; it <= c.k.nitera; ++it) {
    k_mpdata<<<g, kThreads, 0, s>>>(c, MP_UPWIND, it);
    k_mpdata<<<g, kThreads, 0, s>>>(c, MP_FORECAST, it);
    k_mpdata<<<g, kThreads, 0, s>>>(c, MP_ANTIDIFF, it);
  }
  k_mpdata<<<g, kThreads, 0, s>>>(c, MP_DIFFUSION, 0);
  k_mpdata<<<g, kThreads, 0, s>>>(c, MP_FINISH, 0);
}

void launch_b5(const Ctx &c, cudaStream_t s) {
  if (c.k.nadv == 2 && c.k.mode != 4) {
    launch_b5_mpdata(c, s);
    return;
  }
  const size_t ncell = (size_t)c.im * c.jm;
  const char *env = getenv("NPOM_B5");
  bool tiles = c.kb == 16 && c.k.mode != 4 && ncell >= kTileCells;
  if (!env && c.tune.b5_form) tiles = c.kb == 16 && c.k.mode != 4 && c.tune.b5_form == 2;
  if (env && c.kb == 16 && c.k.mode != 4 && std::strcmp(env, "tiles") == 0) tiles = true;
  if (env && std::strcmp(env, "points") == 0) tiles = false;
  if (!tiles) {
    launch_points<PP_B5>(c, s);
    return;
  }
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int strips = (c.jm + kB5Cols - 1) / kB5Cols;
  const int per_sm = c.tune.tile_blocks_per_sm > 0 ? c.tune.tile_blocks_per_sm : 16;
  const int want = std::max(1, (per_sm * sms + strips - 1) / strips);
  const int ichunk = std::max(2, (c.im + want - 1) / want);
  const int chunks = (c.im + ichunk - 1) / ichunk;
  k_b5_tiles<<<dim3(strips, chunks), kB5Threads, 0, s>>>(c, ichunk);
}

__global__ void __launch_bounds__(kThreads) k_cbc_coastal(Ctx c) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q < c.im * c.jm) cbc_coastal_cell(c, q / c.jm, q % c.jm);
}

cudaError_t enqueue_step(const Ctx &c, int core, const PcgPlan &plan, int sub_blocks, cudaStream_t s) {
  launch_a1(c, s);
  launch_wrap_x(c, s);
  launch_cols<CP_A2>(c, s);
  launch_wrap_x(c, s);
  launch_cells<XP_A3>(c, s);
  launch_wrap_x(c, s);
  cudaError_t e;
  if (core == NPOM_CORE_IMPLICIT) {
    launch_policy_bc2(c, 0, s);
    e = run_pcg(c, plan, 1, 1, s);
    if (e != cudaSuccess) return e;
    launch_wrap_x(c, s);
    if (c.k.obc_coastal || c.k.sea_implicit) {
      // the policies: corrector with bcond 2 first, then the filter and
      // shifts; then the tide policies' cbc from the new depth
      // (coastal_implicit_time_loop.py:351-352), the seamount policy's body
      // continuity (seamount_boundary.py:26-42)
      launch_cells<XP_I5A>(c, s);
      launch_policy_bc2(c, 1, s);
    }
    launch_cells<XP_I5>(c, s);
    launch_wrap_x(c, s);
    const int n2 = c.im * c.jm;
    if (c.k.obc_coastal) k_cbc_coastal<<<(n2 + kThreads - 1) / kThreads, kThreads, 0, s>>>(c);
    if (c.k.sea_implicit) {
      k_sea_continuity<<<(n2 + kThreads - 1) / kThreads, kThreads, 0, s>>>(c, 0);
      k_sea_continuity<<<(n2 + kThreads - 1) / kThreads, kThreads, 0, s>>>(c, 1);
    }
  } else {
    e = run_subcycle(c, sub_blocks, s);
    if (e != cudaSuccess) return e;
    if (c.k.obc_coastal) {
      const int n = c.im * c.jm;
      k_cbc_coastal<<<(n + kThreads - 1) / kThreads, kThreads, 0, s>>>(c);
    }
  }
  if (c.do_internal) internal_mode(c, s);
  launch_cols<CP_B9>(c, s);
  launch_wrap_x(c, s);
  return cudaGetLastError();
}


// CUDA graphs of one internal step, keyed by the launch context (pointers,
// settings, ramp, do_internal) and device.  Steps with ramp < 1 (the first
// inertial period from rest) launch directly; every other step replays a
// cached graph, which removes the host launch cost of the ~15 kernels.
// The cache holds kGraphCache graphs (every member of a 64-member ensemble
// on one device keeps its graph, with room for both values of do_internal
// and both cores); past that the oldest is destroyed.
constexpr size_t kGraphCache = 256;

struct GraphEntry {
  int device;
  int core;
  int sub_blocks;
  Ctx key;
  cudaGraphExec_t exec;
};

std::mutex g_graph_mutex;
std::vector<GraphEntry> g_graphs;
cudaStream_t g_capture_stream[64] = {nullptr};
bool g_capture_failed[64][2] = {};

bool graphs_enabled() {
  const char *env = getenv("NPOM_GRAPH");
  return !(env && std::strcmp(env, "0") == 0);
}

cudaError_t launch_step_graph(const Ctx &c, int core, const PcgPlan &plan, int sub_blocks, cudaStream_t s,
                              bool *launched) {
  *launched = false;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= 64) return e;
  std::lock_guard<std::mutex> lock(g_graph_mutex);
  for (auto &g : g_graphs) {
    if (g.device == dev && g.core == core && g.sub_blocks == sub_blocks && std::memcmp(&g.key, &c, sizeof(Ctx)) == 0) {
      e = cudaGraphLaunch(g.exec, s);
      *launched = (e == cudaSuccess);
      return e;
    }
  }
  if (g_capture_failed[dev][core]) return cudaSuccess;
  if (!g_capture_stream[dev]) {
    e = cudaStreamCreateWithFlags(&g_capture_stream[dev], cudaStreamNonBlocking);
    if (e != cudaSuccess) return e;
  }
  cudaStream_t cs = g_capture_stream[dev];
  e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return e;
  cudaError_t le = enqueue_step(c, core, plan, sub_blocks, cs);
  cudaGraph_t graph = nullptr;
  e = cudaStreamEndCapture(cs, &graph);
  if (le != cudaSuccess || e != cudaSuccess || !graph) {
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
    g_capture_failed[dev][core] = true;
    return cudaSuccess;  // not captured: the caller launches directly
  }
  cudaGraphExec_t exec = nullptr;
  e = cudaGraphInstantiate(&exec, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) {
    cudaGetLastError();
    g_capture_failed[dev][core] = true;
    return cudaSuccess;
  }
  if (g_graphs.size() >= kGraphCache) {
    cudaGraphExecDestroy(g_graphs.front().exec);
    g_graphs.erase(g_graphs.begin());
  }
  g_graphs.push_back(GraphEntry{dev, core, sub_blocks, c, exec});
  e = cudaGraphLaunch(exec, s);
  *launched = (e == cudaSuccess);
  return e;
}

npom_status run_steps(const npom_params *p, float *const *fields, const npom_workspace *ws, const npom_clock *clk,
                      void *stream, int core) {
  if (!check_args_dev(p, fields, ws) || !clk || clk->nsteps < 0 || p->core != core) return NPOM_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  Ctx c = make_ctx(p, fields, ws);
  // a barrier that timed out may leave its arrival counter non-zero;
  // sync[2] counts the PCG solves of this call
  if (cudaMemsetAsync(ws->sync, 0, 4 * sizeof(unsigned int), s) != cudaSuccess) return NPOM_ERR_CUDA;
  PcgPlan plan{};
  int sub_blocks = 0;
  if (core == NPOM_CORE_IMPLICIT) {
    if (plan_pcg(c, &plan) != cudaSuccess) return NPOM_ERR_CUDA;
    launch_cells<XP_COEF>(c, s);
  } else {
    if (plan_subcycle(c, &sub_blocks) != cudaSuccess) return NPOM_ERR_CUDA;
  }
  const bool graphs = graphs_enabled();
  for (int n = 0; n < clk->nsteps; ++n) {
    int iint = clk->first_iint + n;
    double time = p->dti * iint * 1.0 / 86400.0 + clk->time0;
    c.ramp = ramp_of(p, time);
    c.do_internal = ((iint != 1 || clk->time0 != 0.0) && p->mode != 2) ? 1 : 0;
    // the coastal policy's tide time of the step's first substep (its
    // launches change every step: no graph replay).  Other steps keep 0:
    // the context is the key of the step graphs
    // (the semi-implicit core's solve time: time * 86400 - dte)
    c.tide_t0 = !c.k.obc_coastal ? 0.0 : time * 86400.0 - (core == NPOM_CORE_IMPLICIT ? p->dte : p->dti);
    bool done = false;
    if (graphs && c.ramp == 1.0f && !c.k.obc_coastal) {
      if (launch_step_graph(c, core, plan, sub_blocks, s, &done) != cudaSuccess) return NPOM_ERR_CUDA;
    }
    if (!done && enqueue_step(c, core, plan, sub_blocks, s) != cudaSuccess) return NPOM_ERR_CUDA;
  }
  return cudaGetLastError() == cudaSuccess ? NPOM_OK : NPOM_ERR_CUDA;
}

cudaError_t enqueue_adj_prep(const Ctx &c, const npom_workspace *ws, const float *grad_x, int flag, cudaStream_t s);
cudaError_t enqueue_adj_solve(const Ctx &c, const npom_workspace *ws, const float *x, float *grad_rhs, float *grad_d,
                              cudaStream_t s);

#include "npom_adjoint_launch.cuh"

// The bounded waits, run out on purpose (npom_wait_selftest): one block of
// a virtual two-block grid at the grid barrier -- the second block never
// arrives -- and one CTA at an exchange mbarrier whose bytes never come.
__global__ void __launch_bounds__(kThreads) k_selftest_grid_wait(unsigned int *sync, unsigned int *status) {
  Ctx c;
  memset(&c, 0, sizeof(c));
  c.sync = sync;
  c.status = status;
  c.grid_blocks = 2;
  c.grid_base = 0;
  (void)grid_barrier(c);
}

__global__ void __launch_bounds__(kClusterThreads) k_selftest_exchange_wait(unsigned int *status) {
  __shared__ uint64_t mb;
  if (threadIdx.x == 0) {
    mb_init(&mb, 1);
    mb_init_fence();
  }
  __syncthreads();
  if (threadIdx.x == 0) mb_expect(&mb, 16);
  (void)xb_wait(&mb, 0, status);
}
#include "npom_batch.cuh"

const char *kFieldNames[] = {
#define NPOM_X_NAME(n) #n,
    NPOM_FIELD_LIST(NPOM_X_NAME)
#undef NPOM_X_NAME
};
const char *kWsNames[] = {
#define NPOM_X_NAME(n) #n,
    NPOM_WS_LIST(NPOM_X_NAME)
#undef NPOM_X_NAME
};
const char *kPhaseNames[] = {"A1_forcing_advct", "A2_baropg_smag_means", "A3_advave_predictor", "E_external",
                             "I5_corrector_filter", "B1_barotropic_fix",  "B2A_vertvl",          "B2B_advq",
                             "B3_profq",            "B4_edges_bcond6",    "B5_qfilter_advt1",    "B6_proft",
                             "B7_tsfilter_dens",    "B8_advuv_profuv",    "B9_velfilter_shift"};
constexpr int kNumPhases = (int)(sizeof(kPhaseNames) / sizeof(kPhaseNames[0]));

// ---------------------------------------------------------------------------
// adjoint of the free-surface solve (implicit_p0_fixed/core.py:24-59 backward,
// :231-252 _solve_implicit_eta_adjoint, :645-675 depth adjoint)
// ---------------------------------------------------------------------------

// rhs = g / area into the rhs workspace; max |rhs| as float bits (a
// non-negative float orders like its bit pattern, NaN above infinity)
// (flag: non-finite values set NPOM_DEV_NONFINITE in the status word)
__global__ void k_adj_prep(Ctx c, const float *g, unsigned int *maxbits, int flag) {
  const size_t n = (size_t)c.im * c.jm;
  unsigned int m = 0u;
  for (size_t o = blockIdx.x * (size_t)blockDim.x + threadIdx.x; o < n; o += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(o / c.jm), j = (int)(o - (size_t)i * c.jm);
    const float v = g[o] / adj_area(c, i, j);
    c.W[NPOM_W_rhs][o] = v;
    const float a = fabsf(v);
    if (flag && !(a <= 3.4028235e38f)) atomicOr(c.status, NPOM_DEV_NONFINITE);
    m = max(m, __float_as_uint(a));
  }
  m = __reduce_max_sync(0xffffffffu, m);
  if ((threadIdx.x & 31) == 0) atomicMax(maxbits, m);
}

// normalised rhs (rhs / scale) and a zero initial guess; the scale from
// the bits k_adj_prep stored
__global__ void k_adj_scale(Ctx c, const unsigned int *scale_bits, float *x) {
  const size_t n = (size_t)c.im * c.jm;
  const float scale = adj_scale_of(scale_bits);
  for (size_t o = blockIdx.x * (size_t)blockDim.x + threadIdx.x; o < n; o += (size_t)gridDim.x * blockDim.x) {
    c.W[NPOM_W_rhs][o] = c.W[NPOM_W_rhs][o] / scale;
    x[o] = 0.0f;
  }
}

// grad_d = -(depth adjoint), gathered per cell in the reference's order
// (adj_grad_d_cell)
__global__ void k_adj_grad_d(Ctx c, const float *x, const float *sol, const unsigned int *scale_bits,
                             float *grad_d) {
  const size_t n = (size_t)c.im * c.jm;
  const float scale = adj_scale_of(scale_bits);
  for (size_t o = blockIdx.x * (size_t)blockDim.x + threadIdx.x; o < n; o += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(o / c.jm), j = (int)(o - (size_t)i * c.jm);
    grad_d[o] = adj_grad_d_cell(c, x, sol, scale, i, j);
  }
}

// lambda = solution * area * scale, in place
__global__ void k_adj_lambda(Ctx c, const unsigned int *scale_bits, float *sol) {
  const size_t n = (size_t)c.im * c.jm;
  const float scale = adj_scale_of(scale_bits);
  for (size_t o = blockIdx.x * (size_t)blockDim.x + threadIdx.x; o < n; o += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(o / c.jm), j = (int)(o - (size_t)i * c.jm);
    sol[o] = (sol[o] * adj_area(c, i, j)) * scale;
  }
}

// The adjoint solve on s: rhs = g / area and its scale (prep), then
// rhs / scale, the coefficients, the PCG from a zero guess with the
// scaled absolute tolerance, grad_d and lambda.  The scale stays on the
// device (ws->sync[3]: the float bits of max |g / area|), so nothing is
// read back to the host.
cudaError_t enqueue_adj_prep(const Ctx &c, const npom_workspace *ws, const float *grad_x, int flag, cudaStream_t s) {
  const size_t n = (size_t)c.im * c.jm;
  const int blocks = std::max(1, std::min(blocks_for(n, kThreads), 1024));
  cudaError_t e = cudaMemsetAsync(ws->sync, 0, 4 * sizeof(unsigned int), s);
  if (e != cudaSuccess) return e;
  k_adj_prep<<<blocks, kThreads, 0, s>>>(c, grad_x, ws->sync + 3, flag);
  return cudaGetLastError();
}

cudaError_t enqueue_adj_solve(const Ctx &c, const npom_workspace *ws, const float *x, float *grad_rhs, float *grad_d,
                              cudaStream_t s) {
  const size_t n = (size_t)c.im * c.jm;
  const int blocks = std::max(1, std::min(blocks_for(n, kThreads), 1024));
  const unsigned int *bits = ws->sync + 3;
  k_adj_scale<<<blocks, kThreads, 0, s>>>(c, bits, grad_rhs);
  launch_cells<XP_COEF>(c, s);
  Ctx ca = c;
  ca.F[NPOM_F_elf] = grad_rhs;  // zero guess in, A^-1 (g/area/scale) out
  ca.tol_scale_bits = bits;     // the forward's stopping test on the scaled system
  PcgPlan plan{};
  cudaError_t e = plan_pcg(ca, &plan);
  if (e != cudaSuccess) return e;
  e = run_pcg(ca, plan, 0, 0, s);
  if (e != cudaSuccess) return e;
  k_adj_grad_d<<<blocks, kThreads, 0, s>>>(c, x, grad_rhs, bits, grad_d);
  k_adj_lambda<<<blocks, kThreads, 0, s>>>(c, bits, grad_rhs);
  return cudaGetLastError();
}

}  // namespace



// ---------------------------------------------------------------------------
// Scratch of npom_pcg_solve_static: the solve's work planes, FP64 partials
// and control words in this module's own device memory (one copy per
// device), for callers that cannot allocate device memory -- a host ocean
// model that owns only its state arrays and has no device allocator of its
// own (a Fortran or C POM driver linked against this library), or a
// real-time loop that forbids allocation once it has started.  The
// address is looked up on the first call per device (and again when the
// calling context of that device changes), so that first call should come
// before any stream capture; calls on one device share the scratch and must
// not overlap.
// ---------------------------------------------------------------------------
constexpr size_t kStaticCells = NPOM_STATIC_MAX_CELLS;
constexpr int kStaticPlanes = 15;  // rhs x r p zv ap ce cw cn cs inv_art diag t1 t2 + one never touched
constexpr size_t kStaticPlaneBytes = (size_t)kStaticPlanes * kStaticCells * sizeof(float);
constexpr size_t kStaticPartialBytes = 4 * (size_t)NPOM_MAX_COOP_BLOCKS * sizeof(double);
constexpr size_t kStaticCtrlWords = 8;  // barrier counter, generation, solve counter, spare, status, iterations, pad
constexpr size_t kStaticBytes = kStaticPlaneBytes + kStaticPartialBytes + kStaticCtrlWords * sizeof(unsigned int);

static __device__ __align__(256) unsigned char g_pcg_scratch[kStaticBytes];

namespace {

std::mutex g_static_mutex;
// One entry per device: the context the address was looked up in (the
// calling thread's current context) and the address.  A call from another
// context of the device (after cudaDeviceReset, or a non-primary context
// made current by the caller) looks the symbol up again.
void *g_static_ctx[64] = {};
unsigned char *g_static_addr[64] = {};

// The calling thread's current driver context, through the runtime's driver
// entry point (no link against libcuda); null if it cannot be resolved.
void *current_context() {
  typedef int (*get_current_fn)(void **);
  static get_current_fn fn = nullptr;
  static bool looked_up = false;
  if (!looked_up) {
    void *f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<get_current_fn>(f);
    looked_up = true;
  }
  void *ctx = nullptr;
  if (!fn || fn(&ctx) != 0) return nullptr;
  return ctx;
}

// Device address of g_pcg_scratch on `dev`, which must be current.
cudaError_t static_scratch(int dev, unsigned char **out) {
  if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_static_mutex);
  void *ctx = current_context();
  if (!g_static_addr[dev] || !ctx || ctx != g_static_ctx[dev]) {
    unsigned char *ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress((void **)&ptr, g_pcg_scratch);
    if (e != cudaSuccess) return e;
    g_static_addr[dev] = ptr;
    g_static_ctx[dev] = ctx;
  }
  *out = g_static_addr[dev];
  return cudaSuccess;
}

}  // namespace

extern "C" {

int npom_abi_version(void) { return 1; }
int npom_field_count(void) { return NPOM_NFIELDS; }
const char *npom_field_name(int index) { return (index >= 0 && index < NPOM_NFIELDS) ? kFieldNames[index] : nullptr; }
int npom_ws_count(void) { return NPOM_NWS; }
const char *npom_ws_name(int index) { return (index >= 0 && index < NPOM_NWS) ? kWsNames[index] : nullptr; }
size_t npom_params_size(void) { return sizeof(npom_params); }
size_t npom_workspace_struct_size(void) { return sizeof(npom_workspace); }
int npom_phase_count(void) { return kNumPhases; }
const char *npom_phase_name(int index) { return (index >= 0 && index < kNumPhases) ? kPhaseNames[index] : nullptr; }

npom_status npom_step_explicit(const npom_params *p, float *const *fields, const npom_workspace *ws,
                               const npom_clock *clk, void *stream) {
  return run_steps(p, fields, ws, clk, stream, NPOM_CORE_EXPLICIT);
}

npom_status npom_step_batch(int32_t nmembers, const npom_params *const *params, float *const *const *fields,
                            const npom_workspace *const *ws, const npom_clock *clk, void *stream) {
  return run_batch_steps(nmembers, params, fields, ws, clk, stream);
}

long long npom_batch_launches(void) {
  std::lock_guard<std::mutex> lock(g_batch_mutex);
  return g_batch_launches;
}

npom_status npom_step_implicit(const npom_params *p, float *const *fields, const npom_workspace *ws,
                               const npom_clock *clk, void *stream) {
  return run_steps(p, fields, ws, clk, stream, NPOM_CORE_IMPLICIT);
}

size_t npom_adjoint_save_floats(const npom_params *p) {
  if (!p || p->im < 3 || p->jm < 3 || p->kb < 3 || p->isplit < 1 || p->isplit > 4096 || p->ispadv < 1) return 0;
  Ctx c;
  std::memset(&c, 0, sizeof(c));
  c.im = p->im;
  c.jm = p->jm;
  c.kb = p->kb;
  c.k = make_consts(*p);
  c.do_internal = 1;
  std::vector<AdjPhaseRec> plan((size_t)adj_plan_capacity(p->isplit, p->nitera));
  size_t need = 0;
  adj_step_plan(c, plan.data(), (int)plan.size(), &need);
  return need + adj_scratch_floats(c);
}

npom_status npom_step_explicit_adjoint(const npom_params *p, float *const *fields, const npom_workspace *ws,
                                       const npom_clock *clk, float *const *grads, const npom_adjoint_ws *aws,
                                       void *stream) {
  return run_step_adjoint(p, fields, ws, clk, grads, aws, NPOM_CORE_EXPLICIT, (cudaStream_t)stream);
}

npom_status npom_step_implicit_adjoint(const npom_params *p, float *const *fields, const npom_workspace *ws,
                                       const npom_clock *clk, float *const *grads, const npom_adjoint_ws *aws,
                                       void *stream) {
  return run_step_adjoint(p, fields, ws, clk, grads, aws, NPOM_CORE_IMPLICIT, (cudaStream_t)stream);
}

npom_status npom_dens(const npom_params *p, float *const *fields, const float *t, const float *s, float *rho_out,
                      void *stream) {
  if (!fields_ok(p, fields) || !t || !s || !rho_out) return NPOM_ERR_ARG;
  Ctx c = fields_ctx(p, fields);
  const size_t n = (size_t)c.im * c.jm * c.kb;
  k_dens<<<(unsigned)((n + kThreads - 1) / kThreads), kThreads, 0, (cudaStream_t)stream>>>(c, t, s, rho_out);
  return cudaGetLastError() == cudaSuccess ? NPOM_OK : NPOM_ERR_CUDA;
}

npom_status npom_dens_adjoint(const npom_params *p, float *const *fields, const float *t, const float *s,
                              const float *grad_rho, float *grad_t, float *grad_s, float *grad_rho_in, void *stream) {
  if (!fields_ok(p, fields) || !t || !s || !grad_rho || !grad_t || !grad_s || !grad_rho_in) return NPOM_ERR_ARG;
  Ctx c = fields_ctx(p, fields);
  const size_t n = (size_t)c.im * c.jm * c.kb;
  k_dens_adj<<<(unsigned)((n + kThreads - 1) / kThreads), kThreads, 0, (cudaStream_t)stream>>>(
      c, t, s, grad_rho, grad_t, grad_s, grad_rho_in);
  return cudaGetLastError() == cudaSuccess ? NPOM_OK : NPOM_ERR_CUDA;
}

npom_status npom_baropg(const npom_params *p, float *const *fields, const float *rho, const float *rmean, double ramp,
                        float *rho_out, float *drhox, float *drhoy, void *stream) {
  if (!fields_ok(p, fields) || !rho || !rmean || !rho_out || !drhox || !drhoy) return NPOM_ERR_ARG;
  Ctx c = fields_ctx(p, fields);
  c.F[NPOM_F_rho] = const_cast<float *>(rho);
  c.F[NPOM_F_rmean] = const_cast<float *>(rmean);
  c.F[NPOM_F_drhox] = drhox;
  c.F[NPOM_F_drhoy] = drhoy;
  c.ramp = (float)ramp;
  const int n = c.im * c.jm;
  k_baropg<<<(n + 127) / 128, 128, 0, (cudaStream_t)stream>>>(c, rho_out);
  return cudaGetLastError() == cudaSuccess ? NPOM_OK : NPOM_ERR_CUDA;
}

npom_status npom_baropg_adjoint(const npom_params *p, float *const *fields, const float *rho, const float *rmean,
                                double ramp, const float *grad_drhox, const float *grad_drhoy, float *grad_rho,
                                float *grad_dt, void *stream) {
  if (!fields_ok(p, fields) || !rho || !rmean || !grad_drhox || !grad_drhoy || !grad_rho || !grad_dt)
    return NPOM_ERR_ARG;
  Ctx c = fields_ctx(p, fields);
  c.F[NPOM_F_rho] = const_cast<float *>(rho);
  c.F[NPOM_F_rmean] = const_cast<float *>(rmean);
  c.ramp = (float)ramp;
  Adj a;
  std::memset(&a, 0, sizeof(a));
  a.G[NPOM_F_rho] = grad_rho;  // accumulated: the caller zeroes or seeds them
  a.G[NPOM_F_dt] = grad_dt;
  const int n = c.im * c.jm;
  cudaStream_t s = (cudaStream_t)stream;
  if (c.kb == 16) k_baropg_adj<16><<<(n + 127) / 128, 128, 0, s>>>(c, a, grad_drhox, grad_drhoy);
  else k_baropg_adj<KMAX><<<(n + 127) / 128, 128, 0, s>>>(c, a, grad_drhox, grad_drhoy);
  return cudaGetLastError() == cudaSuccess ? NPOM_OK : NPOM_ERR_CUDA;
}

npom_status npom_run_phase(const npom_params *p, float *const *fields, const npom_workspace *ws, int phase,
                           double ramp, void *stream) {
  if (!check_args_dev(p, fields, ws) || phase < 0 || phase >= kNumPhases) return NPOM_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  Ctx c = make_ctx(p, fields, ws);
  c.ramp = (float)ramp;
  c.do_internal = 1;
  cudaError_t e = cudaSuccess;
  switch (phase) {
    case 0: launch_a1(c, s); break;
    case 1: launch_cols<CP_A2>(c, s); break;
    case 2:
      launch_cells<XP_A3>(c, s);
      if (p->core == NPOM_CORE_IMPLICIT) launch_policy_bc2(c, 0, s);
      break;
    case 3:
      if (cudaMemsetAsync(ws->sync, 0, 4 * sizeof(unsigned int), s) != cudaSuccess) return NPOM_ERR_CUDA;
      if (p->core == NPOM_CORE_IMPLICIT) {
        PcgPlan plan{};
        e = plan_pcg(c, &plan);
        if (e == cudaSuccess) {
          launch_cells<XP_COEF>(c, s);
          e = run_pcg(c, plan, 1, 1, s);
        }
      } else {
        int blocks = 0;
        e = plan_subcycle(c, &blocks);
        if (e == cudaSuccess) e = run_subcycle(c, blocks, s);
      }
      break;
    case 4: {
      const bool pol = (c.k.obc_coastal || c.k.sea_implicit) && p->core == NPOM_CORE_IMPLICIT;
      if (pol) {
        launch_cells<XP_I5A>(c, s);
        launch_policy_bc2(c, 1, s);
      }
      launch_cells<XP_I5>(c, s);
      const int n = c.im * c.jm;
      if (pol && c.k.obc_coastal) k_cbc_coastal<<<(n + kThreads - 1) / kThreads, kThreads, 0, s>>>(c);
      if (pol && c.k.sea_implicit) {
        k_sea_continuity<<<(n + kThreads - 1) / kThreads, kThreads, 0, s>>>(c, 0);
        k_sea_continuity<<<(n + kThreads - 1) / kThreads, kThreads, 0, s>>>(c, 1);
      }
      break;
    }
    case 5: launch_cols<CP_B1>(c, s); break;
    case 6: launch_cols<CP_B2A>(c, s); break;
    case 7: launch_points<PP_B2B>(c, s); break;
    case 8: launch_cols<CP_B3>(c, s); break;
    case 9: launch_points<PP_B4>(c, s); break;
    case 10: launch_b5(c, s); break;
    case 11:
      launch_cols<CP_B6>(c, s);
      launch_obc_seamount(c, 1, s);
      break;
    case 12: launch_points<PP_B7>(c, s); break;
    case 13:
      launch_cols<CP_B8>(c, s);
      launch_obc_seamount(c, 0, s);
      break;
    case 14: launch_cols<CP_B9>(c, s); break;
  }
  if (e != cudaSuccess) return NPOM_ERR_CUDA;
  launch_wrap_x(c, s);  // the phase's periodic-x halo copy, as in the step
  return cudaGetLastError() == cudaSuccess ? NPOM_OK : NPOM_ERR_CUDA;
}

npom_status npom_proft(int ncol, int kb, const float *f_in, const float *wfsurf, const float *fsurf, int nbc,
                       const float *h, const float *etf, double dti2, const float *dz, const float *dzz,
                       const float *swrad, int ntp, const float *kh, double umol, const float *z, float *f_out,
                       float *dh_out, void *stream) {
  if (ncol < 0 || kb < 3 || kb > KMAX || nbc < 1 || nbc > 4 || ntp < 1 || ntp > 5) return NPOM_ERR_ARG;
  if (ncol == 0) return NPOM_OK;
  if (!f_in || !wfsurf || !fsurf || !h || !etf || !dz || !dzz || !swrad || !kh || !z || !f_out || !dh_out)
    return NPOM_ERR_ARG;
  k_proft<<<blocks_for((size_t)ncol, 128), 128, 0, (cudaStream_t)stream>>>(
      ncol, kb, f_in, wfsurf, fsurf, nbc, h, etf, (float)dti2, dz, dzz, swrad, ntp, kh, (float)umol, z, f_out, dh_out);
  return cudaGetLastError() == cudaSuccess ? NPOM_OK : NPOM_ERR_CUDA;
}

npom_status npom_pcg_solve(const npom_params *p, float *const *fields, const npom_workspace *ws, void *stream) {
  // (the case policies' solves belong to their step: they build their RHS
  // from its predictor)
  if (!check_args_dev(p, fields, ws) || p->core != NPOM_CORE_IMPLICIT || p->obc_form != NPOM_OBC_NATIVE)
    return NPOM_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  Ctx c = make_ctx(p, fields, ws);
  if (cudaMemsetAsync(ws->sync, 0, 4 * sizeof(unsigned int), s) != cudaSuccess) return NPOM_ERR_CUDA;
  PcgPlan plan{};
  cudaError_t e = plan_pcg(c, &plan);
  if (e != cudaSuccess) return NPOM_ERR_CUDA;
  launch_cells<XP_COEF>(c, s);
  e = run_pcg(c, plan, 0, 0, s);
  if (e != cudaSuccess) return NPOM_ERR_CUDA;
  return cudaGetLastError() == cudaSuccess ? NPOM_OK : NPOM_ERR_CUDA;
}

npom_status npom_pcg_adjoint(const npom_params *p, float *const *fields, const npom_workspace *ws,
                             const float *grad_x, const float *x, const float *d2d, float *grad_rhs, float *grad_d,
                             void *stream) {
  if (!check_args_dev(p, fields, ws) || p->core != NPOM_CORE_IMPLICIT || p->obc_form != NPOM_OBC_NATIVE || !grad_x ||
      !x || !d2d || !grad_rhs || !grad_d)
    return NPOM_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  Ctx c = make_ctx(p, fields, ws);
  c.F[NPOM_F_d] = const_cast<float *>(d2d);
  if (enqueue_adj_prep(c, ws, grad_x, 1, s) != cudaSuccess) return NPOM_ERR_CUDA;
  // a non-finite cotangent is reported before any solve (one host sync)
  unsigned int status = 0u;
  if (cudaMemcpyAsync(&status, ws->status, sizeof(status), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return NPOM_ERR_CUDA;
  if (status & NPOM_DEV_NONFINITE) return NPOM_ERR_DEVICE;
  if (enqueue_adj_solve(c, ws, x, grad_rhs, grad_d, s) != cudaSuccess) return NPOM_ERR_CUDA;
  return NPOM_OK;
}

npom_status npom_pcg_solve_static(const npom_params *p, float *const *fields, const float *rhs, const float *sx,
                                  const float *sy, const float *inv_eigs, int *iters_out, unsigned int *status_out,
                                  void *stream) {
  if (!p || !fields || !rhs || p->core != NPOM_CORE_IMPLICIT || p->obc_form != NPOM_OBC_NATIVE || p->im < 3 ||
      p->jm < 3)
    return NPOM_ERR_ARG;
  if (p->eta_precond == NPOM_PRECOND_SPECTRAL && (!sx || !sy || !inv_eigs)) return NPOM_ERR_ARG;
  const size_t ncell = (size_t)p->im * p->jm;
  if (ncell > kStaticCells) return NPOM_ERR_TOO_LARGE;
  if (cudaSetDevice(p->device) != cudaSuccess) return NPOM_ERR_CUDA;
  unsigned char *base = nullptr;
  if (static_scratch(p->device, &base) != cudaSuccess) return NPOM_ERR_CUDA;
  // a workspace view: the inputs are read in place, everything the solve
  // writes lands in the scratch
  float *planes = reinterpret_cast<float *>(base);
  int next = 0;
  auto plane = [&]() { return planes + (size_t)(next++) * kStaticCells; };
  npom_workspace ws{};
  for (int w : {NPOM_W_rhs, NPOM_W_x, NPOM_W_r, NPOM_W_p, NPOM_W_zv, NPOM_W_ap, NPOM_W_ce, NPOM_W_cw, NPOM_W_cn,
                NPOM_W_cs, NPOM_W_inv_art, NPOM_W_diag, NPOM_W_t1, NPOM_W_t2})
    ws.buf[w] = plane();
  float *untouched = plane();  // predictor planes: the solve reads and writes none of them
  for (int w : {NPOM_W_us, NPOM_W_vs, NPOM_W_den_u, NPOM_W_den_v, NPOM_W_d_baro}) ws.buf[w] = untouched;
  ws.buf[NPOM_W_sx] = const_cast<float *>(sx ? sx : untouched);
  ws.buf[NPOM_W_sy] = const_cast<float *>(sy ? sy : untouched);
  ws.buf[NPOM_W_inv_eigs] = const_cast<float *>(inv_eigs ? inv_eigs : untouched);
  ws.partials = reinterpret_cast<double *>(base + kStaticPlaneBytes);
  unsigned int *ctrl = reinterpret_cast<unsigned int *>(base + kStaticPlaneBytes + kStaticPartialBytes);
  ws.sync = ctrl;
  ws.status = ctrl + 4;
  ws.cg_iters = reinterpret_cast<int *>(ctrl + 5);
  if (!check_args(p, fields, &ws)) return NPOM_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  // the control words (barrier counter, solve counter, status) must start
  // at zero: cleared on every call; every other scratch word is written by
  // the solve before it is read
  if (cudaMemsetAsync(ctrl, 0, kStaticCtrlWords * sizeof(unsigned int), s) != cudaSuccess) return NPOM_ERR_CUDA;
  if (cudaMemcpyAsync(ws.buf[NPOM_W_rhs], rhs, ncell * sizeof(float), cudaMemcpyDeviceToDevice, s) != cudaSuccess)
    return NPOM_ERR_CUDA;
  Ctx c = make_ctx(p, fields, &ws);
  PcgPlan plan{};
  if (plan_pcg(c, &plan) != cudaSuccess) return NPOM_ERR_CUDA;
  launch_cells<XP_COEF>(c, s);
  if (run_pcg(c, plan, 0, 0, s) != cudaSuccess) return NPOM_ERR_CUDA;
  if (iters_out && cudaMemcpyAsync(iters_out, ws.cg_iters, sizeof(int), cudaMemcpyDeviceToDevice, s) != cudaSuccess)
    return NPOM_ERR_CUDA;
  if (status_out &&
      cudaMemcpyAsync(status_out, ws.status, sizeof(unsigned int), cudaMemcpyDeviceToDevice, s) != cudaSuccess)
    return NPOM_ERR_CUDA;
  return cudaGetLastError() == cudaSuccess ? NPOM_OK : NPOM_ERR_CUDA;
}

npom_status npom_wait_selftest(int which, const npom_workspace *ws, void *stream) {
  if (!ws || !ws->sync || !ws->status || (which != 0 && which != 1)) return NPOM_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  if (cudaMemsetAsync(ws->sync, 0, 4 * sizeof(unsigned int), s) != cudaSuccess) return NPOM_ERR_CUDA;
  if (which == 0) k_selftest_grid_wait<<<1, kThreads, 0, s>>>(ws->sync, ws->status);
  else k_selftest_exchange_wait<<<1, kClusterThreads, 0, s>>>(ws->status);
  return cudaGetLastError() == cudaSuccess ? NPOM_OK : NPOM_ERR_CUDA;
}

npom_status npom_status_read(const npom_workspace *ws, int clear, unsigned int *out_bits, void *stream) {
  if (!ws || !ws->status || !out_bits) return NPOM_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  unsigned int bits = 0;
  if (cudaMemcpyAsync(&bits, ws->status, sizeof(bits), cudaMemcpyDeviceToHost, s) != cudaSuccess) return NPOM_ERR_CUDA;
  if (cudaStreamSynchronize(s) != cudaSuccess) return NPOM_ERR_CUDA;
  if (clear && cudaMemsetAsync(ws->status, 0, sizeof(unsigned int), s) != cudaSuccess) return NPOM_ERR_CUDA;
  *out_bits = bits;
  return NPOM_OK;
}

}  // extern "C"
