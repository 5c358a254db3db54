// npom_pcg_cluster.cuh -- the free-surface PCG solve on one thread-block
// cluster (distributed shared memory), for grids whose interior fits in the
// cluster's shared memory (90x82 needs ~140 KB per CTA with 8 CTAs).
//
// The interior rows are split into NC slabs, one per CTA.  Every PCG vector,
// the operator coefficients of the slab, its rows of the DST-I matrix Sx
// (stored transposed), the whole Sy and the slab's inverse eigenvalues live
// in shared memory for the whole solve.  Neighbour rows of p (the 5-point
// stencil halo) and the full residual / spectral coefficients needed by the
// i-direction DSTs are read from the other CTAs through DSMEM; reductions
// combine per-CTA FP64 partials read the same way, in rank order, so every
// CTA takes identical convergence decisions.  Cluster barriers separate the
// phases: five per iteration.  The DST stages are register-blocked over four
// rows of the slab (one shared-memory load of the data operand per four
// fused products).
//
// Arithmetic follows implicit_p0_fixed/core.py:460-589 (eager PCG) and
// :591-639 (operator), :762-773 (spectral preconditioner, the DSTs as dense
// sine-matrix products), :893-916 (Shapiro filter and bcond 1).
#pragma once

#include <cooperative_groups.h>

#include "npom_phases_ext.cuh"

namespace npom {

namespace cgx = cooperative_groups;

constexpr int kClusterThreads = 1024;

struct ClusterLayout {
  int ni, nj, nc, rows, rp;  // interior size, CTAs, rows per CTA (rp: padded to 4)
  // float offsets in dynamic shared memory
  int x, r, z, ap, rhs, p, he, hw, hn, hs, ce, cw, cn, cs, me, mw, mn, ms, iart, t1, cm, g, sxt, sy, ie, ks;
  int floats;
  size_t bytes() const { return (size_t)floats * sizeof(float) + 64 * sizeof(double); }
};

inline ClusterLayout cluster_layout(int im, int jm, int nc) {
  ClusterLayout L;
  L.ni = im - 2;
  L.nj = jm - 2;
  L.nc = nc;
  L.rows = (L.ni + nc - 1) / nc;
  L.rp = (L.rows + 3) & ~3;
  const int rn = L.rows * L.nj;
  int o = 0;
  auto take = [&](int n) {
    int at = o;
    o += (n + 3) & ~3;
    return at;
  };
  L.x = take(rn);
  L.r = take(rn);
  L.z = take(rn);
  L.ap = take(rn);
  L.rhs = take(rn);
  L.p = take((L.rows + 2) * L.nj);
  L.he = take(rn);
  L.hw = take(rn);
  L.hn = take(rn);
  L.hs = take(rn);
  L.ce = take(rn);
  L.cw = take(rn);
  L.cn = take(rn);
  L.cs = take(rn);
  L.me = take(rn);
  L.mw = take(rn);
  L.mn = take(rn);
  L.ms = take(rn);
  L.iart = take(rn);
  L.t1 = take(L.nj * L.rp);  // transposed [b][row]; Jacobi keeps its diagonal here
  L.cm = take(rn);
  L.g = take(L.ni * L.nj);
  L.sxt = take(L.ni * L.rp);  // Sx rows of the slab, transposed [m][row]
  L.sy = take(L.nj * L.nj);
  L.ie = take(rn);
  L.ks = take(4 * kClusterThreads);  // split-K partials of the DST stages (float4 each)
  L.floats = o;
  return L;
}

// block-wide FP64 sum (fixed shuffle tree); the CTA's total is left in
// part[slot] by warp 0
__device__ __forceinline__ void cl_block_sum(double v, double *red, double *part, int slot) {
  for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) red[w] = v;
  __syncthreads();
  if (w == 0) {
    const int nw = (int)(blockDim.x >> 5);
    double t = lane < nw ? red[lane] : 0.0;
    for (int off = 16; off > 0; off >>= 1) t += __shfl_down_sync(0xffffffffu, t, off);
    if (lane == 0) part[slot] = t;
  }
}

// after a cluster barrier: sum of part[slot] over the cluster.  Warp 0 reads
// the nc partials in parallel and reduces them with the same shuffle tree in
// every CTA, so all CTAs obtain bitwise the same total.
__device__ __forceinline__ double cl_total(cgx::cluster_group &cl, double *part, int slot, int nc, double *bcast) {
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x;
    double t = lane < nc ? *cl.map_shared_rank(part + slot, lane) : 0.0;
    for (int off = 16; off > 0; off >>= 1) t += __shfl_down_sync(0xffffffffu, t, off);
    if (lane == 0) bcast[slot] = t;
  }
  __syncthreads();
  return bcast[slot];
}

// g <- all rows of the slab array at src_off (row length nj) of every CTA:
// the slab of CTA q is contiguous and lands at row q*rows of g
__device__ __forceinline__ void cl_gather(cgx::cluster_group &cl, const ClusterLayout &L, float *sm, int src_off,
                                          float *g) {
  const int nj = L.nj;
  for (int q = 0; q < L.nc; ++q) {
    const int nrq = min(L.rows, L.ni - q * L.rows);
    if (nrq <= 0) break;
    const float *remote = cl.map_shared_rank(sm + src_off, q);
    float *dst = g + (size_t)q * L.rows * nj;
    if ((nj & 3) == 0) {
      const int n4 = (nrq * nj) >> 2;
      const float4 *r4 = reinterpret_cast<const float4 *>(remote);
      float4 *d4 = reinterpret_cast<float4 *>(dst);
      for (int f = threadIdx.x; f < n4; f += blockDim.x) d4[f] = r4[f];
    } else {
      for (int e = threadIdx.x; e < nrq * nj; e += blockDim.x) dst[e] = remote[e];
    }
  }
}

// fetch halo rows of p from the neighbouring CTAs (zero outside the domain)
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

// ap = A p on the slab (p has its halo rows in place)
__device__ __forceinline__ double cl_spmv(const ClusterLayout &L, float *sm, float coeff, int nr, float *out,
                                          bool dot_with_p) {
  const float *p = sm + L.p;
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
    float fe = sm[L.he + e] * (e_e - ev) * sm[L.ce + e] * sm[L.me + e];
    float fw = sm[L.hw + e] * (ev - e_w) * sm[L.cw + e] * sm[L.mw + e];
    float fn = sm[L.hn + e] * (e_n - ev) * sm[L.cn + e] * sm[L.mn + e];
    float fs = sm[L.hs + e] * (ev - e_s) * sm[L.cs + e] * sm[L.ms + e];
    float div = (fe - fw + fn - fs) * sm[L.iart + e];
    float a = ev - coeff * div;
    out[e] = a;
    if (dot_with_p) acc += (double)ev * (double)a;
  }
  return acc;
}

// The two DST stages compute, for every output group (four slab rows x one
// column), a length-K dot product.  The K range is split KS ways so that all
// warps of the CTA work (KS * groups <= blockDim); the KS partial float4s are
// then summed in split order.
__device__ __forceinline__ int cl_splits(int ng) {
  int ks = (int)blockDim.x / (ng > 0 ? ng : 1);
  return ks < 1 ? 1 : (ks > 8 ? 8 : ks);
}

// DST along i: t1T[b][4g..4g+3] = sum_m Sx[row][m] g[m][b]
__device__ __forceinline__ void cl_dst_i(const ClusterLayout &L, float *sm, int nr) {
  const int nj = L.nj, rp = L.rp, groups = (nr + 3) >> 2, ng = groups * nj;
  const int ks = cl_splits(ng), mlen = (L.ni + ks - 1) / ks;
  const float *g = sm + L.g, *sxt = sm + L.sxt;
  float4 *part = reinterpret_cast<float4 *>(sm + L.ks);
  for (int t = threadIdx.x; t < ng * ks; t += blockDim.x) {
    int s = t / ng, og = t - s * ng;
    int grp = og / nj, b = og - grp * nj;
    int m0 = s * mlen, m1 = min(L.ni, m0 + mlen);
    float a0 = 0.0f, a1 = 0.0f, a2 = 0.0f, a3 = 0.0f;
    const float *sc = sxt + 4 * grp;
#pragma unroll 4
    for (int m = m0; m < m1; ++m) {
      float gv = g[m * nj + b];
      float4 sv = *reinterpret_cast<const float4 *>(sc + m * rp);
      a0 += sv.x * gv;
      a1 += sv.y * gv;
      a2 += sv.z * gv;
      a3 += sv.w * gv;
    }
    part[t] = make_float4(a0, a1, a2, a3);
  }
  __syncthreads();
  float *t1 = sm + L.t1;
  for (int og = threadIdx.x; og < ng; og += blockDim.x) {
    float4 v = part[og];
    for (int s = 1; s < ks; ++s) {
      float4 w = part[s * ng + og];
      v.x += w.x;
      v.y += w.y;
      v.z += w.z;
      v.w += w.w;
    }
    int grp = og / nj, b = og - grp * nj;
    *reinterpret_cast<float4 *>(t1 + b * rp + 4 * grp) = v;
  }
}

// DST along j: out[row][l] = (sum_b t1T[b][row] Sy[b][l]) times scale[row][l]
// (the inverse eigenvalues) or divided by div; accumulates r.out into rz
__device__ __forceinline__ void cl_dst_j(const ClusterLayout &L, float *sm, int nr, float *out, const float *scale,
                                         float div, const float *r, double &rz) {
  const int nj = L.nj, rp = L.rp, groups = (nr + 3) >> 2, ng = groups * nj;
  const int ks = cl_splits(ng), blen = (nj + ks - 1) / ks;
  const float *t1 = sm + L.t1, *sy = sm + L.sy;
  float4 *part = reinterpret_cast<float4 *>(sm + L.ks);
  for (int t = threadIdx.x; t < ng * ks; t += blockDim.x) {
    int s = t / ng, og = t - s * ng;
    int grp = og / nj, l = og - grp * nj;
    int b0 = s * blen, b1 = min(nj, b0 + blen);
    float a0 = 0.0f, a1 = 0.0f, a2 = 0.0f, a3 = 0.0f;
    const float *tc = t1 + 4 * grp;
#pragma unroll 4
    for (int b = b0; b < b1; ++b) {
      float syv = sy[b * nj + l];
      float4 tv = *reinterpret_cast<const float4 *>(tc + b * rp);
      a0 += tv.x * syv;
      a1 += tv.y * syv;
      a2 += tv.z * syv;
      a3 += tv.w * syv;
    }
    part[t] = make_float4(a0, a1, a2, a3);
  }
  __syncthreads();
  for (int og = threadIdx.x; og < ng; og += blockDim.x) {
    float4 v = part[og];
    for (int s = 1; s < ks; ++s) {
      float4 w = part[s * ng + og];
      v.x += w.x;
      v.y += w.y;
      v.z += w.z;
      v.w += w.w;
    }
    int grp = og / nj, l = og - grp * nj;
    float acc[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      int ra = 4 * grp + q;
      if (ra < nr) {
        int e = ra * nj + l;
        float val = scale ? acc[q] * scale[e] : acc[q] / div;
        out[e] = val;
        if (r) rz += (double)r[e] * (double)val;
      }
    }
  }
}

// z = M^-1 r: two cluster-wide gathers, one cluster barrier inside; returns
// this thread's share of r.z.  Every CTA's r slab must be final on entry.
__device__ __forceinline__ double cl_precondition(cgx::cluster_group &cl, const ClusterLayout &L, float *sm, int nr,
                                                  float inverse_scale, bool spectral) {
  const int n = nr * L.nj;
  float *z = sm + L.z;
  const float *r = sm + L.r;
  double rz = 0.0;
  if (!spectral) {
    // Jacobi: the diagonal is kept in the t1 slab
    for (int e = threadIdx.x; e < n; e += blockDim.x) {
      float zv = r[e] / (sm[L.t1 + e] + 1e-30f);
      z[e] = zv;
      rz += (double)r[e] * (double)zv;
    }
    return rz;
  }
  cl_gather(cl, L, sm, L.r, sm + L.g);
  __syncthreads();
  cl_dst_i(L, sm, nr);
  __syncthreads();
  double unused = 0.0;
  cl_dst_j(L, sm, nr, sm + L.cm, sm + L.ie, 1.0f, nullptr, unused);
  cl.sync();
  cl_gather(cl, L, sm, L.cm, sm + L.g);
  __syncthreads();
  cl_dst_i(L, sm, nr);
  __syncthreads();
  cl_dst_j(L, sm, nr, z, nullptr, inverse_scale, r, rz);
  return rz;
}

__global__ void __launch_bounds__(kClusterThreads, 1)
    k_pcg_cluster(Ctx c, ClusterLayout L, int with_rhs, int with_post) {
  extern __shared__ __align__(16) float sm[];
  double *red = reinterpret_cast<double *>(sm + L.floats);  // 32 doubles
  double *part = red + 32;                                    // 8 slots
  double *bcast = part + 8;                                   // 8 slots
  cgx::cluster_group cl = cgx::this_cluster();
  const int rank = (int)cl.block_rank();
  const int im = c.im, jm = c.jm, nj = L.nj;
  const int a0 = rank * L.rows;
  const int nr = max(0, min(L.rows, L.ni - a0));
  const int n = nr * nj;
  const bool spectral = c.k.eta_precond == NPOM_PRECOND_SPECTRAL;
  const float coeff = c.k.implicit_coeff;

  // ---- set-up: stored transports (whole grid, strided over the cluster)
  const int gt = rank * blockDim.x + threadIdx.x, gs = L.nc * blockDim.x;
  if (with_rhs) {
    for (int q = gt; q < im * jm; q += gs) {
      int i = q / jm, j = q - i * jm;
      P2(fluxua, i, j) = rhs_fluxua(c, i, j);
      P2(fluxva, i, j) = rhs_fluxva(c, i, j);
    }
  }
  // ---- slab: coefficients, rhs, initial guess, DST blocks
  const float *dd = c.F[NPOM_F_d];
  for (int e = threadIdx.x; e < n; e += blockDim.x) {
    int ra = e / nj, b = e - ra * nj;
    int i = a0 + ra + 1, j = b + 1;
    size_t o = NPOM_I2(c, i, j);
    float d0 = dd[o];
    sm[L.he + e] = 0.5f * (dd[o + jm] + d0);
    sm[L.hw + e] = 0.5f * (d0 + dd[o - jm]);
    sm[L.hn + e] = 0.5f * (dd[o + 1] + d0);
    sm[L.hs + e] = 0.5f * (d0 + dd[o - 1]);
    float dx_e = 0.5f * (F2(dx, i + 1, j) + F2(dx, i, j));
    float dx_w = 0.5f * (F2(dx, i, j) + F2(dx, i - 1, j));
    float dy_e = 0.5f * (F2(dy, i + 1, j) + F2(dy, i, j));
    float dy_w = 0.5f * (F2(dy, i, j) + F2(dy, i - 1, j));
    float dy_n = 0.5f * (F2(dy, i, j + 1) + F2(dy, i, j));
    float dy_s = 0.5f * (F2(dy, i, j) + F2(dy, i, j - 1));
    float dx_n = 0.5f * (F2(dx, i, j + 1) + F2(dx, i, j));
    float dx_s = 0.5f * (F2(dx, i, j) + F2(dx, i, j - 1));
    sm[L.ce + e] = dy_e / (dx_e + 1e-20f);
    sm[L.cw + e] = dy_w / (dx_w + 1e-20f);
    sm[L.cn + e] = dx_n / (dy_n + 1e-20f);
    sm[L.cs + e] = dx_s / (dy_s + 1e-20f);
    sm[L.me + e] = F2(dum, i + 1, j);
    sm[L.mw + e] = F2(dum, i, j);
    sm[L.mn + e] = F2(dvm, i, j + 1);
    sm[L.ms + e] = F2(dvm, i, j);
    sm[L.iart + e] = 1.0f / (F2(art, i, j) + 1e-20f);
    sm[L.rhs + e] = with_rhs ? rhs_cell(c, i, j) : c.W[NPOM_W_rhs][o];
    sm[L.x + e] = F2(elf, i, j);
    if (spectral) sm[L.ie + e] = c.W[NPOM_W_inv_eigs][(size_t)(a0 + ra) * nj + b];
  }
  if (spectral) {
    // Sx rows of the slab, transposed, zero-padded to rp rows
    for (int e = threadIdx.x; e < L.ni * L.rp; e += blockDim.x) {
      int m = e / L.rp, q = e - m * L.rp;
      sm[L.sxt + e] = (q < nr) ? c.W[NPOM_W_sx][(size_t)(a0 + q) * L.ni + m] : 0.0f;
    }
    for (int e = threadIdx.x; e < nj * nj; e += blockDim.x) sm[L.sy + e] = c.W[NPOM_W_sy][e];
  }
  __syncthreads();
  if (!spectral) {
    // Jacobi diagonal (core.py:677-700) into the t1 slab
    for (int e = threadIdx.x; e < n; e += blockDim.x)
      sm[L.t1 + e] = 1.0f + coeff * sm[L.iart + e] *
                                (sm[L.he + e] * sm[L.ce + e] * sm[L.me + e] + sm[L.hw + e] * sm[L.cw + e] * sm[L.mw + e] +
                                 sm[L.hn + e] * sm[L.cn + e] * sm[L.mn + e] + sm[L.hs + e] * sm[L.cs + e] * sm[L.ms + e]);
  }
  // r = rhs - A x  (x goes through the halo buffer)
  for (int e = threadIdx.x; e < n; e += blockDim.x) sm[L.p + nj + e] = sm[L.x + e];
  cl.sync();
  cl_halo(cl, L, sm, rank, nr);
  __syncthreads();
  cl_spmv(L, sm, coeff, nr, sm + L.ap, false);
  __syncthreads();
  double rr = 0.0;
  for (int e = threadIdx.x; e < n; e += blockDim.x) {
    float rv = sm[L.rhs + e] - sm[L.ap + e];
    sm[L.r + e] = rv;
    rr += (double)rv * (double)rv;
  }
  cl_block_sum(rr, red, part, 0);
  cl.sync();  // r complete in every CTA
  double rs0 = cl_total(cl, part, 0, L.nc, bcast);
  double rz = cl_precondition(cl, L, sm, nr, c.k.inverse_scale, spectral);
  __syncthreads();
  cl_block_sum(rz, red, part, 1);
  cl.sync();
  double rho_old = cl_total(cl, part, 1, L.nc, bcast);
  for (int e = threadIdx.x; e < n; e += blockDim.x) sm[L.p + nj + e] = sm[L.z + e];
  const double tol_sq = c.k.eta_tol * c.k.eta_tol;
  const double rel_sq = c.k.eta_rel_tol * c.k.eta_rel_tol * (rs0 > 1e-30 ? rs0 : 1e-30);
  int its = 0;
  bool converged = false;
  cl.sync();  // p slabs complete
  for (int it = 1; it <= c.k.eta_max_iter; ++it) {
    cl_halo(cl, L, sm, rank, nr);
    __syncthreads();
    double pap = cl_spmv(L, sm, coeff, nr, sm + L.ap, true);
    cl_block_sum(pap, red, part, 2);
    cl.sync();
    double denom = cl_total(cl, part, 2, L.nc, bcast);
    float alpha = (float)(rho_old / (denom + 1e-30));
    double rs = 0.0;
    for (int e = threadIdx.x; e < n; e += blockDim.x) {
      float pv = sm[L.p + nj + e];
      sm[L.x + e] = sm[L.x + e] + alpha * pv;
      float rv = sm[L.r + e] - alpha * sm[L.ap + e];
      sm[L.r + e] = rv;
      rs += (double)rv * (double)rv;
    }
    cl_block_sum(rs, red, part, 3);
    cl.sync();
    double rsn = cl_total(cl, part, 3, L.nc, bcast);
    its = it;
    if (rsn <= tol_sq || rsn <= rel_sq || rsn <= 1e-30) {
      converged = true;
      break;
    }
    rz = cl_precondition(cl, L, sm, nr, c.k.inverse_scale, spectral);
    __syncthreads();
    cl_block_sum(rz, red, part, 4);
    cl.sync();
    double rho_new = cl_total(cl, part, 4, L.nc, bcast);
    float beta = (float)(rho_new / (rho_old + 1e-30));
    for (int e = threadIdx.x; e < n; e += blockDim.x) {
      float *pp = sm + L.p + nj + e;
      *pp = *pp * beta + sm[L.z + e];
    }
    rho_old = rho_new;
    cl.sync();  // p slabs complete before the next halo fetch
  }
  if (rank == 0 && threadIdx.x == 0) {
    // one slot per step of the call: sync[2] counts the solves
    unsigned int slot = c.sync[2];
    c.cg_iters[slot] = its;
    c.sync[2] = slot + 1;
    if (!converged) atomicOr(c.status, NPOM_DEV_PCG_MAXIT);
  }
  // ---- solution: Shapiro filter + closed-basin bcond 1, d = h + elf
  for (int e = threadIdx.x; e < n; e += blockDim.x) sm[L.p + nj + e] = sm[L.x + e];
  cl.sync();
  cl_halo(cl, L, sm, rank, nr);
  __syncthreads();
  for (int e = threadIdx.x; e < n; e += blockDim.x) {
    int ra = e / nj, b = e - ra * nj;
    int i = a0 + ra + 1, j = b + 1;
    const float *pr = sm + L.p + (ra + 1) * nj;
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
  }
  // ring cells
  for (int q = gt; q < 2 * (im + jm); q += gs) {
    int i, j;
    if (q < im) { i = q; j = 0; }
    else if (q < 2 * im) { i = q - im; j = jm - 1; }
    else if (q < 2 * im + jm) { i = 0; j = q - 2 * im; }
    else { i = im - 1; j = q - 2 * im - jm; }
    P2(elf, i, j) = 0.0f;
    if (with_post) P2(d, i, j) = F2(h, i, j);
  }
  cl.sync();  // no CTA exits while others may still read its shared memory
}

}  // namespace npom
