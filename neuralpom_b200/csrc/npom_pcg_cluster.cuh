// npom_pcg_cluster.cuh -- the free-surface PCG solve on one thread-block
// cluster (distributed shared memory), for grids whose interior fits in the
// cluster's shared memory (90x82 needs ~191 KB per CTA with 8 CTAs).
//
// The interior rows are split into NC slabs, one per CTA.  Every PCG vector,
// the operator coefficients of the slab, its rows of the DST-I matrix Sx,
// the whole Sy and the slab's inverse eigenvalues live in shared memory for
// the whole solve.
//
// Data moves between CTAs only by remote STORES issued by the producer (a
// remote load stalls its warp for the DSMEM round trip; a store does not):
//   * the residual r and the half-transformed coefficients cm are pushed,
//     row by row as they are produced, into every CTA's full-grid copy (gr,
//     gc), which the i-direction DST stages then read locally;
//   * the first and last z rows of a slab are pushed into the neighbours' z
//     halo (zh), from which each CTA advances its own copy of the p halo rows
//     with the same expression the owner uses (p = p*beta + z), so the halo
//     of p never has to be fetched;
//   * every warp pushes its FP64 partial of a dot product into a slot of
//     every CTA; after the cluster barrier each warp sums the NC x warps
//     partials in a fixed order with a butterfly, so every warp of every CTA
//     holds bitwise the same total and takes the same convergence decision.
// The cluster barrier (release/acquire) that follows each producer phase is
// what makes the pushed data visible.
//
// Two loop forms, with the same vectors bit for bit:
//   * replicated residual (layouts with room for a third full-grid copy, gap:
//     90x82 on 8 CTAs): the operator product Ap is pushed into every CTA's
//     gap together with the p.Ap partials, and every CTA then advances the
//     WHOLE residual copy gr itself, r = r - alpha*Ap with the owner's own
//     expression on the same bits.  The residual never travels and its norm
//     is summed by every CTA over the whole grid in one fixed order (the same
//     bits everywhere, so every CTA stops at the same iteration).  Three
//     cluster barriers per iteration: p.Ap, the DST transpose, r.z;
//   * pushed residual (larger interiors): the new r rows are pushed into gr
//     and the r.r partials reduced; four cluster barriers per iteration.
//
// Arithmetic follows implicit_p0_fixed/core.py:460-589 (eager PCG) and
// :591-639 (operator), :762-773 (spectral preconditioner, the DSTs as dense
// sine-matrix products), :893-916 (Shapiro filter and bcond 1).  The masks
// dum/dvm of the operator are 0/1 and are folded into the metric ratios
// (exact for 0/1 masks).
//
// The four DST stages are small dense products per CTA (slab rows <= 16,
// K and N <= a few hundred) and run on the tensor cores as m16n8k8 TF32
// MMAs in the 3xTF32 form: every FP32 operand x is split into a TF32 head
// hi = rna(x) and a TF32 tail lo = rna(x - hi), and hi*hi + hi*lo + lo*hi
// is accumulated in FP32 (the lo*lo term, 2^-22 relative, is dropped).  The
// result is an FP32 product of FP32 accuracy, like the reference's dense
// matmul; neither reproduces the other's blocking order bit for bit.  The
// constant operands (the slab's Sx rows, Sy) are split once per solve and
// kept in shared memory in fragment order, one 16-byte load per lane per
// k-step; the i-stage writes its result directly in the A-fragment order of
// the j-stage.
#pragma once

#include <cooperative_groups.h>

#include "npom_phases_ext.cuh"

namespace npom {

namespace cgx = cooperative_groups;

constexpr int kClusterThreads = 512;
constexpr int kClusterWarps = kClusterThreads / 32;
constexpr int kRedSlots = 5;  // pap, r.r, r.z, r0.r0, and one CTA-local slot for block totals

struct ClusterLayout {
  int ni, nj, nc, rows;  // interior size, CTAs, rows per CTA (<= 16: one MMA row tile)
  int kti, nt;           // k-tiles of the i-stage (ceil(ni/8)); column tiles (ceil(nj/8)) = k-tiles of the j-stage
  int gp;                // row pitch of gr/gc: >= 8*nt and 8 or 24 (mod 32), conflict-free B-fragment loads
  // float offsets in dynamic shared memory
  int x, r, z, ap, rhs, p, zh, h4, c4, iart, ie, gr, gc, sxf, syf, t1f;
  int gap;         // full-grid copy of Ap (replicated-residual form), -1 when absent
  int st1, st2;    // bulk form: the slab rows of Ap and of the half-transformed field at pitch gp
  int floats;
  bool fits;       // rows <= 16 and one column tile per warp
  bool sy_global;  // Sy read from global memory in the j-stages (no room for its fragments)
  bool bulk;       // exchanges by bulk copies and mbarriers (replicated form, nj % 4 == 0)
  __host__ __device__ size_t red_doubles() const { return (size_t)kRedSlots * nc * kClusterWarps; }
  // three mbarriers (one per exchange) after the reduction slots in the bulk form
  size_t bytes() const {
    return (size_t)floats * sizeof(float) + red_doubles() * sizeof(double) + (bulk ? 4 * sizeof(uint64_t) : 0);
  }
};

inline ClusterLayout cluster_layout(int im, int jm, int nc, bool sy_global = false, bool replicated = false,
                                    bool bulk = false) {
  ClusterLayout L;
  L.sy_global = sy_global;
  // the replicated and bulk forms keep Sy in shared memory (their loops are
  // compiled for that placement only)
  if (sy_global) replicated = bulk = false;
  L.bulk = bulk && replicated && ((jm - 2) % 4 == 0);
  L.ni = im - 2;
  L.nj = jm - 2;
  L.nc = nc;
  L.rows = (L.ni + nc - 1) / nc;
  L.kti = (L.ni + 7) >> 3;
  L.nt = (L.nj + 7) >> 3;
  L.gp = 8 * L.nt;
  while (L.gp % 32 != 8 && L.gp % 32 != 24) L.gp += 8;
  L.fits = L.rows <= 16 && L.nt <= kClusterWarps;
  const int rn = L.rows * L.nj;
  int o = 0;
  auto take = [&](int n) {
    int at = o;
    o += (n + 3) & ~3;
    return at;
  };
  // bulk form: r and ap are the staging rows of its exchanges after the
  // set-up (pitch gp), so they hold rows*gp floats
  const int rstage = L.bulk ? L.rows * L.gp : rn;
  L.x = take(rn);
  L.r = take(rstage);
  L.z = take(rn);
  L.ap = take(rstage);
  L.rhs = take(rn);
  L.p = take((L.rows + 2) * L.nj);
  L.zh = take(2 * L.nj);
  L.h4 = take(4 * rn);  // (he, hw, hn, hs) per cell
  L.c4 = take(4 * rn);  // metric ratios times the masks (ce, cw, cn, cs)
  L.iart = take(rn);
  L.ie = take(rn);                         // inverse eigenvalues of the slab (Jacobi: the diagonal)
  L.gr = take(8 * L.kti * L.gp);           // full residual, zero-padded rows/columns
  L.gc = take(8 * L.kti * L.gp);           // full half-transformed field
  L.sxf = take(L.kti * 32 * 8);            // Sx slab as A fragments: per k-tile 32 lanes x hi4, then 32 x lo4
  // Sy as B fragments: (hi x2, lo x2) per lane, k-tile, column tile
  L.syf = sy_global ? -1 : take(L.nt * L.nt * 32 * 4);
  L.t1f = take(L.nt * 32 * 4);             // i-stage result as A fragments of the j-stage
  L.gap = replicated ? take(8 * L.kti * L.gp) : -1;  // full Ap, zero-padded like gr
  L.st1 = L.bulk ? L.ap : -1;  // Ap rows sent to every CTA's gap
  L.st2 = L.bulk ? L.r : -1;   // half-transformed rows sent to every CTA's gc
  L.floats = o;
  return L;
}

// Warp partial of a dot product, pushed into slot `slot` of every CTA.
__device__ __forceinline__ void cl_push_partial(cgx::cluster_group &cl, double v, double *red, int slot, int nc,
                                                int rank) {
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane < nc) {
    double *dst = cl.map_shared_rank(red, lane);
    dst[(slot * nc + rank) * kClusterWarps + w] = v;
  }
}

// After the cluster barrier: the cluster total of slot `slot`, the same
// bits in every warp of every CTA.
__device__ __forceinline__ double cl_partial_total(const double *red, int slot, int nc) {
  const int lane = threadIdx.x & 31;
  double t = 0.0;
  if (lane < kClusterWarps)
    for (int q = 0; q < nc; ++q) t += red[(slot * nc + q) * kClusterWarps + lane];
  for (int off = 16; off > 0; off >>= 1) t += __shfl_xor_sync(0xffffffffu, t, off);
  return t;
}

// CTA total of every thread's v, the same bits in every warp (a fixed
// butterfly in each warp, then the warp totals in a fixed butterfly); slot
// holds kClusterWarps doubles of this CTA.  Contains a __syncthreads.
__device__ __forceinline__ double cl_block_total(double v, double *slot) {
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) slot[w] = v;
  __syncthreads();
  double t = lane < kClusterWarps ? slot[lane] : 0.0;
  for (int off = 16; off > 0; off >>= 1) t += __shfl_xor_sync(0xffffffffu, t, off);
  return t;
}

// ---- exchanges by bulk copies and mbarriers (the bulk form) ----------------
// A producer hands data to every consumer with cp.async.bulk (shared::cta
// -> shared::cluster) or st.async, both completing on the CONSUMER's
// mbarrier with the number of bytes delivered; a consumer waits only for the
// bytes it expects (mbarrier.try_wait with acquire at cluster scope).  No
// thread issues the per-element remote stores, and no cluster barrier (with
// its release fence over every outstanding remote store) is needed.  Every
// wait is bounded: after kExchangeTimeoutNs the CTA records NPOM_DEV_TIMEOUT
// and leaves the PCG loop.
constexpr unsigned long long kExchangeTimeoutNs = 500000000ull;

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// the shared::cluster address of the same offset in CTA `rank` of the cluster
__device__ __forceinline__ uint32_t cluster_addr(uint32_t local, int rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(local), "r"(rank));
  return r;
}

__device__ __forceinline__ void mb_init(uint64_t *mb, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mb)), "r"(count) : "memory");
}

__device__ __forceinline__ void mb_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// this CTA's own arrival on its mbarrier for the current phase, with the
// bytes that the phase's producers will deliver
__device__ __forceinline__ void mb_expect(uint64_t *mb, uint32_t bytes) {
  uint64_t state;
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 %0, [%1], %2;"
               : "=l"(state)
               : "r"(smem_u32(mb)), "r"(bytes)
               : "memory");
  (void)state;
}

__device__ __forceinline__ bool mb_try_wait(uint64_t *mb, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(mb)), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// generic-proxy writes of this thread to shared memory, ordered before the
// bulk copies (async proxy) issued after the next barrier
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void bulk_s2s(uint32_t dst_cluster, uint32_t src_cta, uint32_t bytes,
                                         uint32_t mbar_cluster) {
  asm volatile("cp.async.bulk.shared::cluster.shared::cta.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
               ::"r"(dst_cluster), "r"(src_cta), "r"(bytes), "r"(mbar_cluster)
               : "memory");
}

__device__ __forceinline__ void st_async_f64(uint32_t dst_cluster, double v, uint32_t mbar_cluster) {
  asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.b64 [%0], %1, [%2];"
               ::"r"(dst_cluster), "l"((unsigned long long)__double_as_longlong(v)), "r"(mbar_cluster)
               : "memory");
}

// Every thread waits for the phase of parity `parity` (bounded); the
// outcome is made uniform over the CTA, so all its threads take the same
// branch afterwards.  Returns false (and records NPOM_DEV_TIMEOUT) if a
// thread of the CTA gave up.
__device__ __forceinline__ bool xb_wait(uint64_t *mb, uint32_t parity, unsigned int *status) {
  bool ok = mb_try_wait(mb, parity);
  if (!ok) {
    const unsigned long long t0 = global_ns();
    for (unsigned n = 0;; ++n) {
      if (mb_try_wait(mb, parity)) {
        ok = true;
        break;
      }
      if ((n & 63u) == 63u && global_ns() - t0 > kExchangeTimeoutNs) {
        atomicOr(status, NPOM_DEV_TIMEOUT);
        break;
      }
    }
  }
  return __syncthreads_or(ok ? 0 : 1) == 0;
}

// Warp partial of a dot product (the same butterfly as cl_push_partial),
// stored by st.async into slot `slot` of every CTA, counted on that CTA's
// mbarrier mb.
__device__ __forceinline__ void xb_push_partial(double v, double *red, int slot, int nc, int rank, uint64_t *mb) {
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane < nc)
    st_async_f64(cluster_addr(smem_u32(red + (slot * nc + rank) * kClusterWarps + w), lane), v,
                 cluster_addr(smem_u32(mb), lane));
}

// The slab rows at src (pitch gp, nr rows) into rows a0.. of the full-grid
// copy at dst in every CTA (one bulk copy per CTA, issued by one thread),
// counted on the mbarrier mb of each.  The caller made src visible to the
// async proxy and synchronised the CTA.
__device__ __forceinline__ void xb_send_slab(const ClusterLayout &L, float *sm, int src, int dst, int a0, int nr,
                                             uint64_t *mb) {
  if (threadIdx.x != 0 || nr <= 0) return;
  const uint32_t s = smem_u32(sm + src), d = smem_u32(sm + dst + a0 * L.gp), b = smem_u32(mb);
  const uint32_t bytes = (uint32_t)(nr * L.gp * (int)sizeof(float));
  for (int q = 0; q < L.nc; ++q) bulk_s2s(cluster_addr(d, q), s, bytes, cluster_addr(b, q));
}

// fetch halo rows of p from the neighbouring CTAs (zero outside the domain);
// used for the initial residual and the final filter only
__device__ __forceinline__ void cl_halo(cgx::cluster_group &cl, const ClusterLayout &L, float *sm, int rank, int nr) {
  float *p = sm + L.p;
  for (int b = threadIdx.x; b < 2 * L.nj; b += blockDim.x) {
    bool top = b < L.nj;
    int col = top ? b : b - L.nj;
    float v = 0.0f;
    if (top) {
      if (rank > 0) {
        const float *rp = cl.map_shared_rank(sm + L.p, rank - 1);
        v = rp[(L.rows) * L.nj + col];  // last own row of the previous CTA
      }
      p[col] = v;
    } else {
      int q = rank + 1;
      if (q < L.nc && (q * L.rows) < L.ni) {
        const float *rp = cl.map_shared_rank(sm + L.p, q);
        v = rp[1 * L.nj + col];  // first own row of the next CTA
      }
      p[(nr + 1) * L.nj + col] = v;
    }
  }
}

// ap = A p on the slab (p has its halo rows in place); returns this thread's
// share of p.Ap when asked
__device__ __forceinline__ double cl_spmv(const ClusterLayout &L, float *sm, float coeff, int nr, float *out,
                                          bool dot_with_p, int opitch = -1) {
  const int op = opitch < 0 ? L.nj : opitch;
  const float *p = sm + L.p;
  const float4 *h4 = reinterpret_cast<const float4 *>(sm + L.h4);
  const float4 *c4 = reinterpret_cast<const float4 *>(sm + L.c4);
  double acc = 0.0;
  const int n = nr * L.nj;
  for (int e = threadIdx.x; e < n; e += blockDim.x) {
    int ra = e / L.nj, b = e - ra * L.nj;
    const float *pr = p + (ra + 1) * L.nj;
    float ev = pr[b];
    float e_e = pr[b + L.nj];
    float e_w = pr[b - L.nj];
    float e_n = (b + 1 < L.nj) ? pr[b + 1] : 0.0f;
    float e_s = (b > 0) ? pr[b - 1] : 0.0f;
    float4 h = h4[e], cc = c4[e];
    float fe = h.x * (e_e - ev) * cc.x;
    float fw = h.y * (ev - e_w) * cc.y;
    float fn = h.z * (e_n - ev) * cc.z;
    float fs = h.w * (ev - e_s) * cc.w;
    float div = (fe - fw + fn - fs) * sm[L.iart + e];
    float a = ev - coeff * div;
    out[ra * op + b] = a;
    if (dot_with_p) acc += (double)ev * (double)a;
  }
  return acc;
}

// push the slab rows held at src (pitch nj) into every CTA's full-grid copy
// at dst (pitch gp), sixteen bytes per store when rows allow it
__device__ __forceinline__ void cl_push_slab(cgx::cluster_group &cl, const ClusterLayout &L, float *sm, int src,
                                             int dst, int a0, int nr) {
  const int nj = L.nj;
  if ((nj & 3) == 0) {
    const int nj4 = nj >> 2;
    for (int e4 = threadIdx.x; e4 < nr * nj4; e4 += blockDim.x) {
      const int ra = e4 / nj4, b = 4 * (e4 - ra * nj4);
      const float4 v = *reinterpret_cast<const float4 *>(sm + src + ra * nj + b);
      const int at = (a0 + ra) * L.gp + b;
      for (int q = 0; q < L.nc; ++q) *reinterpret_cast<float4 *>(cl.map_shared_rank(sm + dst, q) + at) = v;
    }
  } else {
    for (int e = threadIdx.x; e < nr * nj; e += blockDim.x) {
      const int ra = e / nj, b = e - ra * nj;
      const float v = sm[src + e];
      const int at = (a0 + ra) * L.gp + b;
      for (int q = 0; q < L.nc; ++q) cl.map_shared_rank(sm + dst, q)[at] = v;
    }
  }
}

__device__ __forceinline__ unsigned tf32_rna(float x) {
  unsigned r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

__device__ __forceinline__ void tf32_split(float x, unsigned &hi, unsigned &lo) {
  hi = tf32_rna(x);
  lo = tf32_rna(x - __uint_as_float(hi));
}

// d += a * b, m16n8k8, TF32 inputs, FP32 accumulators
__device__ __forceinline__ void mma_tf32(float (&d)[4], unsigned a0, unsigned a1, unsigned a2, unsigned a3,
                                         unsigned b0, unsigned b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// Fragment coordinates of lane: g = lane/4 (rows g and g+8 of A and C,
// column g of B), t = lane%4 (k = t and t+4 of A and B, columns 2t and 2t+1
// of C).

// i-stage: T[r][n] = sum_m Sx[a0+r][m] G[m][n] for the slab rows r < 16 and
// the column tile of this warp; T goes to t1f in the A-fragment order of
// the j-stage (its k index is n).
__device__ __forceinline__ void cl_dst_i(const ClusterLayout &L, float *sm, const float *G) {
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (w >= L.nt) return;
  const int g = lane >> 2, t = lane & 3, n0 = 8 * w;
  const float4 *af = reinterpret_cast<const float4 *>(sm + L.sxf);
  float hh[4] = {0.f, 0.f, 0.f, 0.f}, hl[4] = {0.f, 0.f, 0.f, 0.f}, lh[4] = {0.f, 0.f, 0.f, 0.f};
  const float *bcol = G + n0 + g;
#pragma unroll 2
  for (int kt = 0; kt < L.kti; ++kt) {
    const float4 ah = af[(2 * kt) * 32 + lane], al = af[(2 * kt + 1) * 32 + lane];
    unsigned bh0, bl0, bh1, bl1;
    tf32_split(bcol[(8 * kt + t) * L.gp], bh0, bl0);
    tf32_split(bcol[(8 * kt + t + 4) * L.gp], bh1, bl1);
    const unsigned a0 = __float_as_uint(ah.x), a1 = __float_as_uint(ah.y), a2 = __float_as_uint(ah.z),
                   a3 = __float_as_uint(ah.w);
    mma_tf32(hh, a0, a1, a2, a3, bh0, bh1);
    mma_tf32(hl, a0, a1, a2, a3, bl0, bl1);
    mma_tf32(lh, __float_as_uint(al.x), __float_as_uint(al.y), __float_as_uint(al.z), __float_as_uint(al.w), bh0,
             bh1);
  }
  float *tf = sm + L.t1f;
  // C element (row, col kk = 2t or 2t+1 of the tile) -> A fragment of k-tile w
  // of the j-stage: lane 4*(row%8) + kk%4, slot (row>=8) + 2*(kk>=4)
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int row8 = q >> 1, kk = 2 * t + (q & 1);
    const float v = (lh[q] + hl[q]) + hh[q];
    tf[(w * 32 + 4 * g + (kk & 3)) * 4 + row8 + 2 * (kk >> 2)] = v;
  }
}

// j-stage: C[r][l] = sum_b T[r][b] Sy[b][l] for the column tile of this
// warp; epi(row, col, value) for the rows < nr and columns < nj.  With
// SYG (layouts with sy_global) the B operand comes from Sy in global memory
// (syg): the lane's
// values of every k-tile of the warp's column tile are loaded up front and
// split as the fragment table splits them, so the products are the same.
template <bool SYG, class Epi>
__device__ __forceinline__ void cl_dst_j(const ClusterLayout &L, float *sm, int nr, const float *syg, Epi &&epi) {
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (w >= L.nt) return;
  const int g = lane >> 2, t = lane & 3;
  const float4 *af = reinterpret_cast<const float4 *>(sm + L.t1f);
  float hh[4] = {0.f, 0.f, 0.f, 0.f}, hl[4] = {0.f, 0.f, 0.f, 0.f}, lh[4] = {0.f, 0.f, 0.f, 0.f};
  if (SYG) {
    const int col = 8 * w + g, nj = L.nj;
    float v0[kClusterWarps], v1[kClusterWarps];
#pragma unroll
    for (int kt = 0; kt < kClusterWarps; ++kt) {
      const int b0 = 8 * kt + t, b1 = b0 + 4;
      v0[kt] = (kt < L.nt && b0 < nj && col < nj) ? __ldg(syg + (size_t)b0 * nj + col) : 0.0f;
      v1[kt] = (kt < L.nt && b1 < nj && col < nj) ? __ldg(syg + (size_t)b1 * nj + col) : 0.0f;
    }
#pragma unroll
    for (int kt = 0; kt < kClusterWarps; ++kt) {
      if (kt < L.nt) {
        const float4 av = af[kt * 32 + lane];
        unsigned ah0, al0, ah1, al1, ah2, al2, ah3, al3, bh0, bl0, bh1, bl1;
        tf32_split(av.x, ah0, al0);
        tf32_split(av.y, ah1, al1);
        tf32_split(av.z, ah2, al2);
        tf32_split(av.w, ah3, al3);
        tf32_split(v0[kt], bh0, bl0);
        tf32_split(v1[kt], bh1, bl1);
        mma_tf32(hh, ah0, ah1, ah2, ah3, bh0, bh1);
        mma_tf32(hl, ah0, ah1, ah2, ah3, bl0, bl1);
        mma_tf32(lh, al0, al1, al2, al3, bh0, bh1);
      }
    }
  } else {
    const float4 *bf = reinterpret_cast<const float4 *>(sm + L.syf);
  #pragma unroll 2
    for (int kt = 0; kt < L.nt; ++kt) {
      const float4 av = af[kt * 32 + lane];
      const float4 b = bf[(kt * L.nt + w) * 32 + lane];
      unsigned ah0, al0, ah1, al1, ah2, al2, ah3, al3;
      tf32_split(av.x, ah0, al0);
      tf32_split(av.y, ah1, al1);
      tf32_split(av.z, ah2, al2);
      tf32_split(av.w, ah3, al3);
      const unsigned bh0 = __float_as_uint(b.x), bh1 = __float_as_uint(b.y);
      mma_tf32(hh, ah0, ah1, ah2, ah3, bh0, bh1);
      mma_tf32(hl, ah0, ah1, ah2, ah3, __float_as_uint(b.z), __float_as_uint(b.w));
      mma_tf32(lh, al0, al1, al2, al3, bh0, bh1);
    }
  }
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const int row = g + 8 * (q >> 1), col = 8 * w + 2 * t + (q & 1);
    if (row < nr && col < L.nj) epi(row, col, (lh[q] + hl[q]) + hh[q]);
  }
}

// z = M^-1 r for the slab, with r already pushed into every CTA's gr (and
// the cluster barrier after the push passed).  Pushes the half-transformed
// field into gc (one cluster barrier inside), writes z, pushes the z rows
// that neighbours keep as halo and returns this thread's share of r.z.
template <bool SYG>
__device__ __forceinline__ double cl_precondition(cgx::cluster_group &cl, const ClusterLayout &L, float *sm, int nr,
                                                  int rank, int a0, float inverse_scale, bool spectral,
                                                  const float *syg) {
  const int nj = L.nj;
  float *z = sm + L.z;
  const float *r = sm + L.r;
  const float *ie = sm + L.ie;
  const bool up = rank > 0 && nr > 0;
  const bool down = (rank + 1) < L.nc && (rank + 1) * L.rows < L.ni;
  double rz = 0.0;
  auto finish = [&](int ra, int l, float zv) {
    const int e = ra * nj + l;
    z[e] = zv;
    rz += (double)r[e] * (double)zv;
    if (ra == 0 && up) cl.map_shared_rank(sm + L.zh, rank - 1)[nj + l] = zv;
    if (ra == nr - 1 && down) cl.map_shared_rank(sm + L.zh, rank + 1)[l] = zv;
  };
  if (!spectral) {
    for (int e = threadIdx.x; e < nr * nj; e += blockDim.x) {
      int ra = e / nj;
      finish(ra, e - ra * nj, r[e] / (ie[e] + 1e-30f));
    }
    return rz;
  }
  cl_dst_i(L, sm, sm + L.gr);
  __syncthreads();
  // DST along j times the inverse eigenvalues, pushed into every CTA's gc
  // (staged in the ap slab, free until the next operator apply)
  float *stage = sm + L.ap;
  cl_dst_j<SYG>(L, sm, nr, syg, [&](int ra, int l, float acc) { stage[ra * nj + l] = acc * ie[ra * nj + l]; });
  __syncthreads();
  cl_push_slab(cl, L, sm, L.ap, L.gc, a0, nr);
  cl.sync();  // gc complete in every CTA
  cl_dst_i(L, sm, sm + L.gc);
  __syncthreads();
  // DST along j divided by the scale: z
  cl_dst_j<SYG>(L, sm, nr, syg, [&](int ra, int l, float acc) { finish(ra, l, acc / inverse_scale); });
  return rz;
}

// Bulk form of cl_precondition (spectral only): the half-transformed slab
// goes to every CTA's gc by bulk copies counted on mbarrier mb[1]; r is read
// from the whole-residual copy gr.  Writes z (no halo push: the caller's
// r.z exchange carries the halo rows) and returns this thread's share of
// r.z.  `failed` is set (uniformly over the CTA) if the wait gave up.
template <bool SYG>
__device__ __forceinline__ double cl_precondition_bulk(const ClusterLayout &L, float *sm, int nr, int a0,
                                                       float inverse_scale, const float *syg, uint64_t *mb,
                                                       unsigned &ph1, unsigned int *status, bool &failed) {
  const int nj = L.nj, gp = L.gp;
  float *z = sm + L.z;
  const float *gr = sm + L.gr;
  const float *ie = sm + L.ie;
  float *stage = sm + L.st2;
  double rz = 0.0;
  cl_dst_i(L, sm, sm + L.gr);
  __syncthreads();
  cl_dst_j<SYG>(L, sm, nr, syg, [&](int ra, int l, float acc) { stage[ra * gp + l] = acc * ie[ra * nj + l]; });
  fence_proxy_async_smem();
  __syncthreads();
  if (threadIdx.x == 0) mb_expect(mb + 1, (uint32_t)(L.ni * gp * (int)sizeof(float)));
  xb_send_slab(L, sm, L.st2, L.gc, a0, nr, mb + 1);
  if (!xb_wait(mb + 1, ph1, status)) failed = true;
  ph1 ^= 1u;
  if (failed) return 0.0;
  cl_dst_i(L, sm, sm + L.gc);
  __syncthreads();
  cl_dst_j<SYG>(L, sm, nr, syg, [&](int ra, int l, float acc) {
    const float zv = acc / inverse_scale;
    z[ra * nj + l] = zv;
    rz += (double)gr[(a0 + ra) * gp + l] * (double)zv;
  });
  return rz;
}

// Bulk form of the r.z exchange: the z rows that the neighbours keep as
// halo (first row up, last row down) and every warp's r.z partial, counted
// on mbarrier mb[2]; the caller wrote z in every thread.
__device__ __forceinline__ void xb_exchange_rz(const ClusterLayout &L, float *sm, double rz, double *red, int nr,
                                               int rank, bool has_up, bool has_down, uint64_t *mb, unsigned &ph2,
                                               unsigned int *status, bool &failed) {
  const int nj = L.nj, nc = L.nc;
  fence_proxy_async_smem();
  __syncthreads();
  if (threadIdx.x == 0) {
    const uint32_t row = (uint32_t)(nj * (int)sizeof(float));
    mb_expect(mb + 2, (uint32_t)(nc * kClusterWarps * (int)sizeof(double)) + (has_up ? row : 0u) +
                          (has_down ? row : 0u));
    const uint32_t bar = smem_u32(mb + 2);
    if (has_up)  // first own row -> the lower halo of the CTA above
      bulk_s2s(cluster_addr(smem_u32(sm + L.zh + nj), rank - 1), smem_u32(sm + L.z), row,
               cluster_addr(bar, rank - 1));
    if (has_down)  // last own row -> the upper halo of the CTA below
      bulk_s2s(cluster_addr(smem_u32(sm + L.zh), rank + 1), smem_u32(sm + L.z + (nr - 1) * nj), row,
               cluster_addr(bar, rank + 1));
  }
  xb_push_partial(rz, red, 2, nc, rank, mb + 2);
  if (!xb_wait(mb + 2, ph2, status)) failed = true;
  ph2 ^= 1u;
}

// The rhs scale of the adjoint solve from its float bits (clamp_min(1); a
// NaN gives 1, as on the host), and the PCG's absolute tolerance.
__device__ __forceinline__ float adj_scale_of(const unsigned int *bits) {
  const float a = __uint_as_float(*bits);
  return a > 1.0f ? a : 1.0f;
}
__device__ __forceinline__ double pcg_abs_tol(const Ctx &c) {
  return c.tol_scale_bits ? c.k.eta_tol / (double)adj_scale_of(c.tol_scale_bits) : c.k.eta_tol;
}

// The solve of one member on the cluster of this block; sm is the dynamic
// shared memory of the layout L.
template <bool SYG>
__device__ __forceinline__ void pcg_cluster_body(const Ctx &c, const ClusterLayout &L, float *sm, int with_rhs,
                                                 int with_post) {
  double *red = reinterpret_cast<double *>(sm + L.floats);
  uint64_t *mb = reinterpret_cast<uint64_t *>(red + L.red_doubles());  // bulk form: three mbarriers
  unsigned ph0 = 0u, ph1 = 0u, ph2 = 0u;
  bool failed = false;
  if (L.bulk && threadIdx.x == 0) {
    for (int k = 0; k < 3; ++k) mb_init(mb + k, 1u);
    mb_init_fence();  // visible cluster-wide before the set-up's first cluster barrier
  }
  cgx::cluster_group cl = cgx::this_cluster();
  const int rank = (int)cl.block_rank();
  const int im = c.im, jm = c.jm, nj = L.nj, nc = L.nc;
  const int a0 = rank * L.rows;
  const int nr = max(0, min(L.rows, L.ni - a0));
  const int n = nr * nj;
  const bool spectral = c.k.eta_precond == NPOM_PRECOND_SPECTRAL;
  const float coeff = c.k.implicit_coeff;
  const bool has_up = rank > 0 && nr > 0;
  const bool has_down = (rank + 1) < nc && (rank + 1) * L.rows < L.ni;

  // ---- set-up: stored transports (whole grid, strided over the cluster)
  const int gt = rank * blockDim.x + threadIdx.x, gs = nc * blockDim.x;
  if (with_rhs) {
    for (int q = gt; q < im * jm; q += gs) {
      int i = q / jm, j = q - i * jm;
      P2(fluxua, i, j) = rhs_fluxua(c, i, j);
      P2(fluxva, i, j) = rhs_fluxva(c, i, j);
    }
  }
  // ---- slab: coefficients, rhs, initial guess, DST blocks
  const float *dd = c.F[NPOM_F_d];
  float4 *h4 = reinterpret_cast<float4 *>(sm + L.h4);
  float4 *c4 = reinterpret_cast<float4 *>(sm + L.c4);
  for (int e = threadIdx.x; e < n; e += blockDim.x) {
    int ra = e / nj, b = e - ra * nj;
    int i = a0 + ra + 1, j = b + 1;
    size_t o = NPOM_I2(c, i, j);
    float d0 = dd[o];
    h4[e] = make_float4(0.5f * (dd[o + jm] + d0), 0.5f * (d0 + dd[o - jm]), 0.5f * (dd[o + 1] + d0),
                        0.5f * (d0 + dd[o - 1]));
    float dx_e = 0.5f * (F2(dx, i + 1, j) + F2(dx, i, j));
    float dx_w = 0.5f * (F2(dx, i, j) + F2(dx, i - 1, j));
    float dy_e = 0.5f * (F2(dy, i + 1, j) + F2(dy, i, j));
    float dy_w = 0.5f * (F2(dy, i, j) + F2(dy, i - 1, j));
    float dy_n = 0.5f * (F2(dy, i, j + 1) + F2(dy, i, j));
    float dy_s = 0.5f * (F2(dy, i, j) + F2(dy, i, j - 1));
    float dx_n = 0.5f * (F2(dx, i, j + 1) + F2(dx, i, j));
    float dx_s = 0.5f * (F2(dx, i, j) + F2(dx, i, j - 1));
    c4[e] = make_float4((dy_e / (dx_e + 1e-20f)) * F2(dum, i + 1, j), (dy_w / (dx_w + 1e-20f)) * F2(dum, i, j),
                        (dx_n / (dy_n + 1e-20f)) * F2(dvm, i, j + 1), (dx_s / (dy_s + 1e-20f)) * F2(dvm, i, j));
    sm[L.iart + e] = 1.0f / (F2(art, i, j) + 1e-20f);
    sm[L.rhs + e] = with_rhs ? rhs_cell(c, i, j) : c.W[NPOM_W_rhs][o];
    sm[L.x + e] = F2(elf, i, j);
    if (spectral) sm[L.ie + e] = c.W[NPOM_W_inv_eigs][(size_t)(a0 + ra) * nj + b];
  }
  for (int b = threadIdx.x; b < 2 * nj; b += blockDim.x) sm[L.zh + b] = 0.0f;
  if (L.bulk) fence_proxy_async_smem();
  if (spectral) {
    const float *sx = c.W[NPOM_W_sx], *sy = c.W[NPOM_W_sy];
    const int ni = L.ni;
    // padding rows/columns of the full-grid copies stay zero
    for (int e = threadIdx.x; e < 8 * L.kti * L.gp; e += blockDim.x) {
      sm[L.gr + e] = 0.0f;
      sm[L.gc + e] = 0.0f;
      if (L.gap >= 0) sm[L.gap + e] = 0.0f;
    }
    if (L.bulk) fence_proxy_async_smem();  // gc and gap are written by bulk copies from here on
    // Sx rows of the slab as split A fragments (zero outside the slab)
    for (int f = threadIdx.x; f < L.kti * 32; f += blockDim.x) {
      const int kt = f >> 5, lane = f & 31, g = lane >> 2, t = lane & 3;
      float v[4];
      for (int q = 0; q < 4; ++q) {
        const int row = g + 8 * (q & 1), m = 8 * kt + t + 4 * (q >> 1);
        v[q] = (row < nr && m < ni) ? sx[(size_t)(a0 + row) * ni + m] : 0.0f;
      }
      unsigned hi[4], lo[4];
      for (int q = 0; q < 4; ++q) tf32_split(v[q], hi[q], lo[q]);
      float4 *dst = reinterpret_cast<float4 *>(sm + L.sxf) + (2 * kt) * 32 + lane;
      dst[0] = make_float4(__uint_as_float(hi[0]), __uint_as_float(hi[1]), __uint_as_float(hi[2]), __uint_as_float(hi[3]));
      dst[32] = make_float4(__uint_as_float(lo[0]), __uint_as_float(lo[1]), __uint_as_float(lo[2]), __uint_as_float(lo[3]));
    }
    // Sy as split B fragments (kept in global memory with sy_global)
    for (int f = threadIdx.x; !SYG && f < L.nt * L.nt * 32; f += blockDim.x) {
      const int lane = f & 31, tile = f >> 5, kt = tile / L.nt, ct = tile - kt * L.nt, g = lane >> 2, t = lane & 3;
      const int col = 8 * ct + g, b0 = 8 * kt + t, b1 = b0 + 4;
      const float v0 = (b0 < nj && col < nj) ? sy[(size_t)b0 * nj + col] : 0.0f;
      const float v1 = (b1 < nj && col < nj) ? sy[(size_t)b1 * nj + col] : 0.0f;
      unsigned h0, l0, h1, l1;
      tf32_split(v0, h0, l0);
      tf32_split(v1, h1, l1);
      reinterpret_cast<float4 *>(sm + L.syf)[f] =
          make_float4(__uint_as_float(h0), __uint_as_float(h1), __uint_as_float(l0), __uint_as_float(l1));
    }
  }
  __syncthreads();
  if (!spectral) {
    // Jacobi diagonal (core.py:677-700), kept where the eigenvalues would be
    for (int e = threadIdx.x; e < n; e += blockDim.x) {
      float4 h = h4[e], cc = c4[e];
      sm[L.ie + e] = 1.0f + coeff * sm[L.iart + e] * (h.x * cc.x + h.y * cc.y + h.z * cc.z + h.w * cc.w);
    }
  }
  // r = rhs - A x  (x goes through the halo buffer)
  for (int e = threadIdx.x; e < n; e += blockDim.x) sm[L.p + nj + e] = sm[L.x + e];
  cl.sync();  // x slabs complete; zh zeroed everywhere before any push
  cl_halo(cl, L, sm, rank, nr);
  __syncthreads();
  cl_spmv(L, sm, coeff, nr, sm + L.ap, false);
  double rr = 0.0;
  for (int e = threadIdx.x; e < n; e += blockDim.x) {
    float rv = sm[L.rhs + e] - sm[L.ap + e];
    sm[L.r + e] = rv;
    rr += (double)rv * (double)rv;
  }
  __syncthreads();
  if (spectral) cl_push_slab(cl, L, sm, L.r, L.gr, a0, nr);
  cl_push_partial(cl, rr, red, 3, nc, rank);
  cl.sync();  // r pushed everywhere; neighbours' x halo reads done
  const double rs0 = cl_partial_total(red, 3, nc);
  double rz = 0.0;
  if constexpr (!SYG) {
    if (L.bulk) {
      // the set-up is done with the r and ap slabs: from here on they are the
      // staging rows (pitch gp) of the exchanges, whose padding columns must
      // stay zero (they land in the zero-padded full-grid copies)
      for (int e = threadIdx.x; e < L.rows * L.gp; e += blockDim.x) {
        sm[L.st1 + e] = 0.0f;
        sm[L.st2 + e] = 0.0f;
      }
      fence_proxy_async_smem();
      __syncthreads();
      rz = cl_precondition_bulk<SYG>(L, sm, nr, a0, c.k.inverse_scale, c.W[NPOM_W_sy], mb, ph1, c.status, failed);
      if (!failed) xb_exchange_rz(L, sm, rz, red, nr, rank, has_up, has_down, mb, ph2, c.status, failed);
    }
  }
  if (!L.bulk) {
    rz = cl_precondition<SYG>(cl, L, sm, nr, rank, a0, c.k.inverse_scale, spectral, c.W[NPOM_W_sy]);
    cl_push_partial(cl, rz, red, 2, nc, rank);
    cl.sync();  // z halo rows and r.z partials in place
  }
  double rho_old = cl_partial_total(red, 2, nc);
  float *p = sm + L.p;
  for (int e = threadIdx.x; e < n; e += blockDim.x) p[nj + e] = sm[L.z + e];
  for (int b = threadIdx.x; b < nj; b += blockDim.x) {
    p[b] = has_up ? sm[L.zh + b] : 0.0f;
    p[(nr + 1) * nj + b] = has_down ? sm[L.zh + nj + b] : 0.0f;
  }
  const double tol = pcg_abs_tol(c), tol_sq = tol * tol;
  const double rel_sq = c.k.eta_rel_tol * c.k.eta_rel_tol * (rs0 > 1e-30 ? rs0 : 1e-30);
  int its = 0;
  bool converged = false;
  __syncthreads();  // p and its halo rows complete in this CTA
  const bool replicated = spectral && L.gap >= 0 && !L.bulk;
  if constexpr (!SYG) {
  for (int it = 1; L.bulk && !failed && it <= c.k.eta_max_iter; ++it) {
    // ---- bulk form: the replicated-residual iteration, exchanges by bulk
    // copies counted on mbarriers (no cluster barrier in the loop)
    double pap = cl_spmv(L, sm, coeff, nr, sm + L.st1, true, L.gp);
    fence_proxy_async_smem();
    __syncthreads();  // the Ap slab complete (and visible to the async proxy) before it is sent
    if (threadIdx.x == 0)
      mb_expect(mb, (uint32_t)(L.ni * L.gp * (int)sizeof(float) + nc * kClusterWarps * (int)sizeof(double)));
    xb_send_slab(L, sm, L.st1, L.gap, a0, nr, mb);
    xb_push_partial(pap, red, 0, nc, rank, mb);
    if (!xb_wait(mb, ph0, c.status)) failed = true;
    ph0 ^= 1u;
    if (failed) break;
    const double denom = cl_partial_total(red, 0, nc);
    const float alpha = (float)(rho_old / (denom + 1e-30));
    for (int e = threadIdx.x; e < n; e += blockDim.x) sm[L.x + e] = sm[L.x + e] + alpha * p[nj + e];
    float4 *gr4 = reinterpret_cast<float4 *>(sm + L.gr);
    const float4 *ga4 = reinterpret_cast<const float4 *>(sm + L.gap);
    double rs = 0.0;
    for (int e4 = threadIdx.x; e4 < 2 * L.kti * L.gp; e4 += blockDim.x) {
      float4 rv = gr4[e4];
      const float4 av = ga4[e4];
      rv.x = rv.x - alpha * av.x;
      rv.y = rv.y - alpha * av.y;
      rv.z = rv.z - alpha * av.z;
      rv.w = rv.w - alpha * av.w;
      gr4[e4] = rv;
      rs += (double)rv.x * (double)rv.x;
      rs += (double)rv.y * (double)rv.y;
      rs += (double)rv.z * (double)rv.z;
      rs += (double)rv.w * (double)rv.w;
    }
    const double rsn = cl_block_total(rs, red + (size_t)4 * nc * kClusterWarps);  // gr complete after this
    its = it;
    if (rsn <= tol_sq || rsn <= rel_sq || rsn <= 1e-30) {
      converged = true;
      break;
    }
    rz = cl_precondition_bulk<SYG>(L, sm, nr, a0, c.k.inverse_scale, c.W[NPOM_W_sy], mb, ph1, c.status, failed);
    if (failed) break;
    xb_exchange_rz(L, sm, rz, red, nr, rank, has_up, has_down, mb, ph2, c.status, failed);
    if (failed) break;
    const double rho_new = cl_partial_total(red, 2, nc);
    const float beta = (float)(rho_new / (rho_old + 1e-30));
    for (int e = threadIdx.x; e < n; e += blockDim.x) {
      float *pp = p + nj + e;
      *pp = *pp * beta + sm[L.z + e];
    }
    for (int b = threadIdx.x; b < nj; b += blockDim.x) {
      if (has_up) p[b] = p[b] * beta + sm[L.zh + b];
      if (has_down) p[(nr + 1) * nj + b] = p[(nr + 1) * nj + b] * beta + sm[L.zh + nj + b];
    }
    rho_old = rho_new;
    __syncthreads();
  }
  for (int it = 1; replicated && it <= c.k.eta_max_iter; ++it) {
    // ---- replicated-residual form: three cluster barriers per iteration
    double pap = cl_spmv(L, sm, coeff, nr, sm + L.ap, true);
    __syncthreads();  // the Ap slab complete before it is pushed
    cl_push_slab(cl, L, sm, L.ap, L.gap, a0, nr);
    cl_push_partial(cl, pap, red, 0, nc, rank);
    cl.sync();  // Ap rows and p.Ap partials in every CTA
    const double denom = cl_partial_total(red, 0, nc);
    const float alpha = (float)(rho_old / (denom + 1e-30));
    for (int e = threadIdx.x; e < n; e += blockDim.x) sm[L.x + e] = sm[L.x + e] + alpha * p[nj + e];
    // the whole residual, in every CTA, with the owner's expression
    float4 *gr4 = reinterpret_cast<float4 *>(sm + L.gr);
    const float4 *ga4 = reinterpret_cast<const float4 *>(sm + L.gap);
    double rs = 0.0;
    for (int e4 = threadIdx.x; e4 < 2 * L.kti * L.gp; e4 += blockDim.x) {
      float4 rv = gr4[e4];
      const float4 av = ga4[e4];
      rv.x = rv.x - alpha * av.x;
      rv.y = rv.y - alpha * av.y;
      rv.z = rv.z - alpha * av.z;
      rv.w = rv.w - alpha * av.w;
      gr4[e4] = rv;
      rs += (double)rv.x * (double)rv.x;
      rs += (double)rv.y * (double)rv.y;
      rs += (double)rv.z * (double)rv.z;
      rs += (double)rv.w * (double)rv.w;
    }
    const double rsn = cl_block_total(rs, red + (size_t)4 * nc * kClusterWarps);  // gr complete after this
    its = it;
    if (rsn <= tol_sq || rsn <= rel_sq || rsn <= 1e-30) {
      converged = true;
      break;
    }
    for (int e = threadIdx.x; e < n; e += blockDim.x) {
      const int ra = e / nj;
      sm[L.r + e] = sm[L.gr + (a0 + ra) * L.gp + (e - ra * nj)];
    }
    rz = cl_precondition<SYG>(cl, L, sm, nr, rank, a0, c.k.inverse_scale, spectral, c.W[NPOM_W_sy]);
    cl_push_partial(cl, rz, red, 2, nc, rank);
    cl.sync();  // z halo rows and r.z partials in place
    const double rho_new = cl_partial_total(red, 2, nc);
    const float beta = (float)(rho_new / (rho_old + 1e-30));
    for (int e = threadIdx.x; e < n; e += blockDim.x) {
      float *pp = p + nj + e;
      *pp = *pp * beta + sm[L.z + e];
    }
    for (int b = threadIdx.x; b < nj; b += blockDim.x) {
      if (has_up) p[b] = p[b] * beta + sm[L.zh + b];
      if (has_down) p[(nr + 1) * nj + b] = p[(nr + 1) * nj + b] * beta + sm[L.zh + nj + b];
    }
    rho_old = rho_new;
    __syncthreads();
  }
  }  // !SYG: bulk and replicated forms
  for (int it = 1; !replicated && !L.bulk && it <= c.k.eta_max_iter; ++it) {
    // ---- pushed-residual form: four cluster barriers per iteration
    double pap = cl_spmv(L, sm, coeff, nr, sm + L.ap, true);
    cl_push_partial(cl, pap, red, 0, nc, rank);
    cl.sync();
    const double denom = cl_partial_total(red, 0, nc);
    const float alpha = (float)(rho_old / (denom + 1e-30));
    double rs = 0.0;
    if ((nj & 3) == 0) {
      // four cells per thread: the new r goes out to every CTA in one
      // sixteen-byte store per destination
      for (int e = 4 * threadIdx.x; e < n; e += 4 * blockDim.x) {
        const float4 pv = *reinterpret_cast<const float4 *>(p + nj + e);
        const float4 av = *reinterpret_cast<const float4 *>(sm + L.ap + e);
        float4 xv = *reinterpret_cast<const float4 *>(sm + L.x + e);
        float4 rv = *reinterpret_cast<const float4 *>(sm + L.r + e);
        xv.x = xv.x + alpha * pv.x;
        xv.y = xv.y + alpha * pv.y;
        xv.z = xv.z + alpha * pv.z;
        xv.w = xv.w + alpha * pv.w;
        rv.x = rv.x - alpha * av.x;
        rv.y = rv.y - alpha * av.y;
        rv.z = rv.z - alpha * av.z;
        rv.w = rv.w - alpha * av.w;
        *reinterpret_cast<float4 *>(sm + L.x + e) = xv;
        *reinterpret_cast<float4 *>(sm + L.r + e) = rv;
        rs += (double)rv.x * (double)rv.x;
        rs += (double)rv.y * (double)rv.y;
        rs += (double)rv.z * (double)rv.z;
        rs += (double)rv.w * (double)rv.w;
        if (spectral) {
          const int ra = e / nj, at = (a0 + ra) * L.gp + (e - ra * nj);
          for (int q = 0; q < nc; ++q) *reinterpret_cast<float4 *>(cl.map_shared_rank(sm + L.gr, q) + at) = rv;
        }
      }
    } else {
      for (int e = threadIdx.x; e < n; e += blockDim.x) {
        float pv = p[nj + e];
        sm[L.x + e] = sm[L.x + e] + alpha * pv;
        float rv = sm[L.r + e] - alpha * sm[L.ap + e];
        sm[L.r + e] = rv;
        rs += (double)rv * (double)rv;
      }
      __syncthreads();
      if (spectral) cl_push_slab(cl, L, sm, L.r, L.gr, a0, nr);
    }
    cl_push_partial(cl, rs, red, 1, nc, rank);
    cl.sync();
    const double rsn = cl_partial_total(red, 1, nc);
    its = it;
    if (rsn <= tol_sq || rsn <= rel_sq || rsn <= 1e-30) {
      converged = true;
      break;
    }
    rz = cl_precondition<SYG>(cl, L, sm, nr, rank, a0, c.k.inverse_scale, spectral, c.W[NPOM_W_sy]);
    cl_push_partial(cl, rz, red, 2, nc, rank);
    cl.sync();
    const double rho_new = cl_partial_total(red, 2, nc);
    const float beta = (float)(rho_new / (rho_old + 1e-30));
    for (int e = threadIdx.x; e < n; e += blockDim.x) {
      float *pp = p + nj + e;
      *pp = *pp * beta + sm[L.z + e];
    }
    // the halo rows follow the owner's own update p = p*beta + z
    for (int b = threadIdx.x; b < nj; b += blockDim.x) {
      if (has_up) p[b] = p[b] * beta + sm[L.zh + b];
      if (has_down) p[(nr + 1) * nj + b] = p[(nr + 1) * nj + b] * beta + sm[L.zh + nj + b];
    }
    rho_old = rho_new;
    __syncthreads();
  }
  if (rank == 0 && threadIdx.x == 0) {
    // one slot per step of the call: sync[2] counts the solves
    unsigned int slot = c.sync[2];
    c.cg_iters[slot] = its;
    c.sync[2] = slot + 1;
    if (!converged) atomicOr(c.status, NPOM_DEV_PCG_MAXIT);
  }
  // ---- solution: Shapiro filter + closed-basin bcond 1, d = h + elf
  for (int e = threadIdx.x; e < n; e += blockDim.x) p[nj + e] = sm[L.x + e];
  cl.sync();
  cl_halo(cl, L, sm, rank, nr);
  __syncthreads();
  for (int e = threadIdx.x; e < n; e += blockDim.x) {
    int ra = e / nj, b = e - ra * nj;
    int i = a0 + ra + 1, j = b + 1;
    const float *pr = p + (ra + 1) * nj;
    float x0 = pr[b];
    float ev;
    if (with_post) {
      float xn = (b + 1 < nj) ? pr[b + 1] : 0.0f;
      float xs = (b > 0) ? pr[b - 1] : 0.0f;
      float smv = x0 + c.k.bshap_q * (pr[b + nj] + pr[b - nj] + xn + xs - 4.0f * x0);
      float fsm = F2(fsm, i, j);
      ev = (smv * fsm) * fsm;
      if (!(fabsf(ev) <= 3.0e38f)) atomicOr(c.status, NPOM_DEV_NONFINITE);
      P2(d, i, j) = F2(h, i, j) + ev;
    } else {
      ev = x0;
    }
    P2(elf, i, j) = ev;
    c.W[NPOM_W_x][NPOM_I2(c, i, j)] = x0;  // the raw solution, as the grid-barrier form leaves it
  }
  // ring cells
  for (int q = gt; q < 2 * (im + jm); q += gs) {
    int i, j;
    if (q < im) { i = q; j = 0; }
    else if (q < 2 * im) { i = q - im; j = jm - 1; }
    else if (q < 2 * im + jm) { i = 0; j = q - 2 * im; }
    else { i = im - 1; j = q - 2 * im - jm; }
    P2(elf, i, j) = 0.0f;
    c.W[NPOM_W_x][NPOM_I2(c, i, j)] = 0.0f;
    if (with_post) P2(d, i, j) = F2(h, i, j);
  }
  cl.sync();  // no CTA exits while others may still read its shared memory
}

// SYG: the layout reads Sy from global memory (L.sy_global)
template <bool SYG>
__global__ void __launch_bounds__(kClusterThreads, 1)
    k_pcg_cluster(Ctx c, ClusterLayout L, int with_rhs, int with_post) {
  extern __shared__ __align__(16) float sm[];
  pcg_cluster_body<SYG>(c, L, sm, with_rhs, with_post);
}

}  // namespace npom
