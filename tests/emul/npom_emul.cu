// npom_emul.cu -- CPU emulation of the device phases, for tests only.
//
// Compiles the very same __host__ __device__ phase bodies as the CUDA
// library (neuralpom_b200/csrc) for the host and runs each phase as a loop
// over its points / columns / cells, in the order the kernels launch them.
// The cooperative kernels (PCG, explicit subcycle) are restated with the
// grid barriers replaced by the end of each loop.  This checks the index
// logic of every phase against the oracle on a machine without a GPU; it is
// not part of the product library and is never loaded by neuralpom_b200.
#include <algorithm>
#include <cmath>
#include <cstring>

#include <vector>

#include "../../neuralpom_b200/csrc/npom_host.cuh"
#include "../../neuralpom_b200/csrc/npom_adjoint.cuh"
#include "../../neuralpom_b200/csrc/npom_mpdata.cuh"
#include "../../neuralpom_b200/csrc/npom_mpdata_adjoint.cuh"

using namespace npom;

namespace {

template <class F>
void each_point(const Ctx &c, F f) {
  for (int i = 0; i < c.im; ++i)
    for (int j = 0; j < c.jm; ++j)
      for (int k = 0; k < c.kb; ++k) f(i, j, k);
}
template <class F>
void each_cell(const Ctx &c, F f) {
  for (int i = 0; i < c.im; ++i)
    for (int j = 0; j < c.jm; ++j) f(i, j);
}

void a1(const Ctx &c) {
  each_point(c, [&](int i, int j, int k) {
    float ax, ay, cv;
    advct_point(c, i, j, k, ax, ay, cv);
    P3(advx, i, j, k) = ax;
    P3(advy, i, j, k) = ay;
    P3(curv, i, j, k) = cv;
    if (k == 0) forcing_cell(c, i, j);
  });
}

// the periodic-x halo copy after a phase (k_wrap_x): every plane of the
// state and the workspace planes a later phase reads
void wrap_x(const Ctx &c) {
  if (!c.k.periodic_x) return;
  auto copy = [&](float *a, int depth) {
    const size_t col = (size_t)c.jm * depth;
    const int dst[4] = {0, 1, c.im - 2, c.im - 1}, src[4] = {c.im - 4, c.im - 3, 2, 3};
    for (int w = 0; w < 4; ++w) std::memcpy(a + dst[w] * col, a + src[w] * col, col * sizeof(float));
  };
  for (int f = NPOM_F_h; f <= NPOM_F_north_e; ++f) copy(c.F[f], 1);
  for (int f = NPOM_F_u; f <= NPOM_F_curv; ++f) copy(c.F[f], c.kb);
  for (int f = NPOM_F_el; f <= NPOM_F_ssurf; ++f) copy(c.F[f], 1);
  for (int w : {NPOM_W_us, NPOM_W_vs, NPOM_W_den_u, NPOM_W_den_v, NPOM_W_d_baro}) copy(c.W[w], 1);
}

// dot product over the unknowns of the free-surface solve
double dot_int(const Ctx &c, const float *a, const float *b) {
  double s = 0.0;
  for (int i = pcg_i0(c); i < c.im - pcg_i0(c); ++i)
    for (int j = 1; j < c.jm - 1; ++j) {
      size_t o = NPOM_I2(c, i, j);
      s += (double)a[o] * (double)b[o];
    }
  return s;
}

void precondition(const Ctx &c) {
  int ni = c.im - 2;
  const int nj = c.jm - 2;
  float *zv = c.W[NPOM_W_zv];
  const float *r = c.W[NPOM_W_r];
  if (c.k.eta_precond == NPOM_PRECOND_SPECTRAL) {
    float *t1 = c.W[NPOM_W_t1], *t2 = c.W[NPOM_W_t2];
    const int i0 = pcg_i0(c);
    ni = c.im - 2 * i0;
    for (int a = 0; a < ni; ++a)
      for (int b = 0; b < nj; ++b) t1[(size_t)a * nj + b] = dst_stage_i(c, r, true, a, b);
    for (int a = 0; a < ni; ++a)
      for (int b = 0; b < nj; ++b)
        t2[(size_t)a * nj + b] = dst_stage_j(c, t1, a, b) * c.W[NPOM_W_inv_eigs][(size_t)a * nj + b];
    for (int a = 0; a < ni; ++a)
      for (int b = 0; b < nj; ++b) t1[(size_t)a * nj + b] = dst_stage_i(c, t2, false, a, b);
    for (int a = 0; a < ni; ++a)
      for (int b = 0; b < nj; ++b) zv[NPOM_I2(c, a + i0, b + 1)] = dst_stage_j(c, t1, a, b) / c.k.inverse_scale;
  } else {
    for (int i = pcg_i0(c); i < c.im - pcg_i0(c); ++i)
      for (int j = 1; j < c.jm - 1; ++j) {
        size_t o = NPOM_I2(c, i, j);
        zv[o] = r[o] / (c.W[NPOM_W_diag][o] + 1e-30f);
      }
  }
}

void pcg(const Ctx &c, int step, int with_rhs, int with_post) {
  const int im = c.im, jm = c.jm, i0 = pcg_i0(c);
  float *x = c.W[NPOM_W_x], *r = c.W[NPOM_W_r], *p = c.W[NPOM_W_p], *zv = c.W[NPOM_W_zv];
  float *ap = c.W[NPOM_W_ap], *rhs = c.W[NPOM_W_rhs];
  each_cell(c, [&](int i, int j) {
    size_t q = NPOM_I2(c, i, j);
    if (with_rhs) rhs[q] = rhs_cell(c, i, j);
    else if (!interior(c, i, j)) rhs[q] = 0.0f;
  });
  if (with_rhs)
    each_cell(c, [&](int i, int j) {
      P2(fluxua, i, j) = rhs_fluxua(c, i, j);
      P2(fluxva, i, j) = rhs_fluxva(c, i, j);
    });
  each_cell(c, [&](int i, int j) {
    size_t q = NPOM_I2(c, i, j);
    bool in = interior(c, i, j);
    x[q] = in ? c.F[NPOM_F_elf][q] : 0.0f;
    if (!in) r[q] = p[q] = zv[q] = ap[q] = 0.0f;
  });
  for (int i = i0; i < im - i0; ++i)
    for (int j = 1; j < jm - 1; ++j) {
      size_t o = NPOM_I2(c, i, j);
      r[o] = rhs[o] - elliptic_apply_cell(c, x, i, j);
      if (c.k.eta_precond != NPOM_PRECOND_SPECTRAL) c.W[NPOM_W_diag][o] = jacobi_diag_cell(c, i, j);
    }
  double rs0 = dot_int(c, r, r);
  precondition(c);
  double rho_old = dot_int(c, r, zv);
  for (int i = i0; i < im - i0; ++i)
    for (int j = 1; j < jm - 1; ++j) p[NPOM_I2(c, i, j)] = zv[NPOM_I2(c, i, j)];
  const double tol_sq = c.k.eta_tol * c.k.eta_tol;
  const double rel_sq = c.k.eta_rel_tol * c.k.eta_rel_tol * (rs0 > 1e-30 ? rs0 : 1e-30);
  int its = 0;
  bool conv = false;
  for (int it = 1; it <= c.k.eta_max_iter; ++it) {
    for (int i = i0; i < im - i0; ++i)
      for (int j = 1; j < jm - 1; ++j) ap[NPOM_I2(c, i, j)] = elliptic_apply_cell(c, p, i, j);
    double denom = dot_int(c, p, ap);
    float alpha = (float)(rho_old / (denom + 1e-30));
    for (int i = i0; i < im - i0; ++i)
      for (int j = 1; j < jm - 1; ++j) {
        size_t o = NPOM_I2(c, i, j);
        x[o] = x[o] + alpha * p[o];
        r[o] = r[o] - alpha * ap[o];
      }
    double rs = dot_int(c, r, r);
    its = it;
    if (rs <= tol_sq || rs <= rel_sq || rs <= 1e-30) {
      conv = true;
      break;
    }
    precondition(c);
    double rho_new = dot_int(c, r, zv);
    float beta = (float)(rho_new / (rho_old + 1e-30));
    for (int i = i0; i < im - i0; ++i)
      for (int j = 1; j < jm - 1; ++j) {
        size_t o = NPOM_I2(c, i, j);
        p[o] = p[o] * beta + zv[o];
      }
    rho_old = rho_new;
  }
  c.cg_iters[step] = its;
  if (!conv) *c.status |= NPOM_DEV_PCG_MAXIT;
  if (!with_post) {
    each_cell(c, [&](int i, int j) {
      const int iw = !c.k.periodic_x ? i : i < 2 ? i + im - 4 : (i > im - 3 ? i - (im - 4) : i);
      P2(elf, i, j) = x[NPOM_I2(c, iw, j)];
    });
    return;
  }
  each_cell(c, [&](int i, int j) {
    size_t q = NPOM_I2(c, i, j);
    float e = 0.0f;
    if (interior(c, i, j)) {
      float x0 = x[q];
      const size_t qe = NPOM_I2(c, pcg_east(c, i), j), qw = NPOM_I2(c, pcg_west(c, i), j);
      float sm = x0 + c.k.bshap_q * (x[qe] + x[qw] + x[q + 1] + x[q - 1] - 4.0f * x0);
      float fsm = F2(fsm, i, j);
      e = (sm * fsm) * fsm;
    }
    P2(elf, i, j) = e;
    P2(d, i, j) = F2(h, i, j) + e;
  });
}

// the tide policies' free-surface solve (k_cg_policy), sequentially
void cg_policy(const Ctx &c, int step) {
  const int im = c.im, jm = c.jm;
  float *x = c.W[NPOM_W_x], *r = c.W[NPOM_W_r], *p = c.W[NPOM_W_p], *ap = c.W[NPOM_W_ap];
  float *rhs = c.W[NPOM_W_rhs], *lift = c.W[NPOM_W_zv];
  each_cell(c, [&](int i, int j) {
    const size_t q = NPOM_I2(c, i, j);
    rhs[q] = rhs_cell(c, i, j);
    lift[q] = policy_lift(c, i, j);
  });
  each_cell(c, [&](int i, int j) {
    P2(fluxua, i, j) = rhs_fluxua(c, i, j);
    P2(fluxva, i, j) = rhs_fluxva(c, i, j);
  });
  auto wdot = [&](const float *a, const float *b) {
    double s = 0.0;
    for (int i = 0; i < im; ++i)
      for (int j = 0; j < jm; ++j) {
        const size_t q = NPOM_I2(c, i, j);
        const float w = policy_fixed(c, i, j) ? 0.0f : F2(art, i, j);
        s += (double)(w * a[q]) * (double)b[q];
      }
    return s;
  };
  each_cell(c, [&](int i, int j) {
    const size_t q = NPOM_I2(c, i, j);
    const float b = policy_fixed(c, i, j) ? 0.0f : rhs[q] - elliptic_apply_cell(c, lift, i, j);
    x[q] = 0.0f;
    r[q] = b;
    p[q] = b;
  });
  double rr = wdot(r, r);
  const double thr = std::max(1e-30, rr * 1e-24);
  const int nmax = std::min(c.k.eta_max_iter, 500);
  int its = nmax;
  for (int it = 0; it < nmax; ++it) {
    if (rr <= thr) {
      its = it + 1;
      break;
    }
    each_cell(c, [&](int i, int j) {
      ap[NPOM_I2(c, i, j)] = policy_fixed(c, i, j) ? 0.0f : elliptic_apply_cell(c, p, i, j);
    });
    const float alpha = (float)(rr / (wdot(p, ap) + 1e-40));
    each_cell(c, [&](int i, int j) {
      const size_t q = NPOM_I2(c, i, j);
      x[q] = x[q] + alpha * p[q];
      r[q] = r[q] - alpha * ap[q];
    });
    const double nw = wdot(r, r);
    const float beta = (float)(nw / (rr + 1e-40));
    each_cell(c, [&](int i, int j) {
      const size_t q = NPOM_I2(c, i, j);
      p[q] = r[q] + beta * p[q];
    });
    rr = nw;
  }
  c.cg_iters[step] = its;
  std::vector<float> e((size_t)im * jm);
  each_cell(c, [&](int i, int j) { e[NPOM_I2(c, i, j)] = policy_elf(c, x, i, j); });
  std::memcpy(c.F[NPOM_F_elf], e.data(), e.size() * sizeof(float));
}

// the seamount policy's Picard / Robin solve (k_robin_picard), sequentially
void robin_picard(const Ctx &c, int step) {
  const int im = c.im, jm = c.jm;
  const size_t ncell = (size_t)im * jm;
  double *X = c.robin, *R = c.robin + ncell, *P = c.robin + 2 * ncell, *AP = c.robin + 3 * ncell;
  double *G = c.robin + 4 * ncell;
  float *rhs = c.W[NPOM_W_rhs];
  each_cell(c, [&](int i, int j) { rhs[NPOM_I2(c, i, j)] = rhs_cell(c, i, j); });
  each_cell(c, [&](int i, int j) {
    P2(fluxua, i, j) = rhs_fluxua(c, i, j);
    P2(fluxva, i, j) = rhs_fluxva(c, i, j);
    X[NPOM_I2(c, i, j)] = sea_free(c, i, j) ? (double)F2(el, i, j) : 0.0;
  });
  auto area = [&](int i, int j) { return sea_free(c, i, j) ? (double)F2(art, i, j) : 0.0; };
  bool converged = false;
  int total = 0;
  for (int nl = 0; nl < 6 && !converged; ++nl) {
    each_cell(c, [&](int i, int j) { G[NPOM_I2(c, i, j)] = sea_ghost(c, X, i, j); });
    double rr = 0.0, bb = 0.0;
    each_cell(c, [&](int i, int j) {
      const size_t q = NPOM_I2(c, i, j);
      const double b = sea_rhs(c, rhs, G, i, j);
      R[q] = b - sea_robin_op(c, X, G, i, j);
      P[q] = R[q];
      rr += area(i, j) * R[q] * R[q];
      bb += area(i, j) * b * b;
    });
    const double thr = std::max(1e-28, std::max(bb, 1e-40) * 1e-22);
    for (int it = 0; it < 300; ++it) {
      if (rr <= thr) break;
      double den = 0.0;
      each_cell(c, [&](int i, int j) {
        const size_t q = NPOM_I2(c, i, j);
        AP[q] = sea_robin_op(c, P, G, i, j);
        den += area(i, j) * P[q] * AP[q];
      });
      if (!(den > 0.0) || !(den < 1.0e308)) {
        *c.status |= NPOM_DEV_NONFINITE;
        return;
      }
      const double a = rr / den;
      double nw = 0.0;
      each_cell(c, [&](int i, int j) {
        const size_t q = NPOM_I2(c, i, j);
        X[q] = X[q] + a * P[q];
        R[q] = R[q] - a * AP[q];
        nw += area(i, j) * R[q] * R[q];
      });
      const double beta = nw / std::max(rr, 1e-40);
      each_cell(c, [&](int i, int j) {
        const size_t q = NPOM_I2(c, i, j);
        P[q] = R[q] + beta * P[q];
      });
      rr = nw;
      ++total;
    }
    double change = 0.0;
    each_cell(c, [&](int i, int j) {
      change = std::max(change, std::fabs(sea_ghost(c, X, i, j) - G[NPOM_I2(c, i, j)]));
    });
    converged = change < 1e-11;
  }
  c.cg_iters[step] = total;
  if (!converged) *c.status |= NPOM_DEV_PCG_MAXIT;
  each_cell(c, [&](int i, int j) { P2(elf, i, j) = sea_elf(c, X, i, j); });
}

void policy_lines(const Ctx &c, int which) {
  if (!c.k.obc_coastal || c.k.obc_jzb) return;
  for (int t = 0; t < c.jm + c.im; ++t) policy_bc2_line(c, t, which);
}

void subcycle(const Ctx &c) {
  for (int iext = 1; iext <= c.k.isplit; ++iext) {
    bool adv = (iext % c.k.ispadv) == 0;
    each_cell(c, [&](int i, int j) { ext_phase1_cell(c, i, j, adv, iext); });
    each_cell(c, [&](int i, int j) {
      if (ext_phase2_cell(c, i, j, iext)) *c.status |= NPOM_DEV_VMAX;
    });
    each_cell(c, [&](int i, int j) { ext_phase3_cell(c, i, j, iext); });
  }
}

void run_phase(const Ctx &c, const npom_params *p, int phase) {
  switch (phase) {
    case 0: a1(c); break;
    case 1: each_cell(c, [&](int i, int j) { phase_a2_column(c, i, j); }); break;
    case 2:
      each_cell(c, [&](int i, int j) { phase_a3_cell(c, i, j); });
      if (p->core == NPOM_CORE_IMPLICIT) policy_lines(c, 0);
      break;
    case 3:
      if (p->core == NPOM_CORE_IMPLICIT) {
        each_cell(c, [&](int i, int j) { elliptic_coeff_cell(c, i, j); });
        if (c.k.obc_coastal) cg_policy(c, 0);
        else if (c.k.sea_implicit) robin_picard(c, 0);
        else pcg(c, 0, 1, 1);
      } else {
        subcycle(c);
      }
      break;
    case 4: {
      const bool pol = (c.k.obc_coastal || c.k.sea_implicit) && p->core == NPOM_CORE_IMPLICIT;
      if (pol) {
        each_cell(c, [&](int i, int j) { phase_i5a_cell(c, i, j); });
        policy_lines(c, 1);
      }
      each_cell(c, [&](int i, int j) {
        if (phase_i5_cell(c, i, j)) *c.status |= NPOM_DEV_VMAX;
      });
      if (pol && c.k.obc_coastal) each_cell(c, [&](int i, int j) { cbc_coastal_cell(c, i, j); });
      if (pol && c.k.sea_implicit) {
        each_cell(c, [&](int i, int j) { sea_transport_cell(c, i, j); });
        std::vector<float> e((size_t)c.im * c.jm);
        each_cell(c, [&](int i, int j) { e[NPOM_I2(c, i, j)] = sea_etf_cell(c, i, j); });
        std::memcpy(c.F[NPOM_F_etf], e.data(), e.size() * sizeof(float));
      }
      break;
    }
    case 5: each_cell(c, [&](int i, int j) { phase_b1_column(c, i, j); }); break;
    case 6: each_cell(c, [&](int i, int j) { phase_b2a_column(c, i, j); }); break;
    case 7: each_point(c, [&](int i, int j, int k) { phase_b2b_point(c, i, j, k); }); break;
    case 8: each_cell(c, [&](int i, int j) { phase_b3_column(c, i, j); }); break;
    case 9: each_point(c, [&](int i, int j, int k) { phase_b4_point(c, i, j, k); }); break;
    case 10:
      if (c.k.nadv == 2 && c.k.mode != 4) {
        auto pass = [&](int ps, int it) {
          each_point(c, [&](int i, int j, int k) { phase_b5_mpdata_point(c, ps, it, i, j, k); });
        };
        pass(MP_FILTER, 0);
        pass(MP_INIT, 0);
        for (int it = 1; it <= c.k.nitera; ++it) {
          pass(MP_UPWIND, it);
          pass(MP_FORECAST, it);
          pass(MP_ANTIDIFF, it);
        }
        pass(MP_DIFFUSION, 0);
        pass(MP_FINISH, 0);
      } else {
        each_point(c, [&](int i, int j, int k) { phase_b5_point(c, i, j, k); });
      }
      break;
    case 11:
      each_cell(c, [&](int i, int j) { phase_b6_column(c, i, j); });
      if (c.k.obc_seamount)
        for (int j = 0; j < c.jm; ++j)
          for (int k = 0; k < c.kb; ++k) obc_seamount_ts_point(c, j, k);
      break;
    case 12: each_point(c, [&](int i, int j, int k) { phase_b7_point(c, i, j, k); }); break;
    case 13:
      each_cell(c, [&](int i, int j) { phase_b8_column(c, i, j); });
      if (c.k.obc_seamount)
        for (int j = 0; j < c.jm; ++j)
          for (int k = 0; k < c.kb; ++k) obc_seamount_u_point(c, j, k);
      break;
    case 14: each_cell(c, [&](int i, int j) { phase_b9_column(c, i, j); }); break;
  }
  wrap_x(c);
}

// the implicit free-surface phase of the recomputation: PCG without its post
// step, the solution kept in xs, then the post step (as k_imp_post)
void imp_forward(const Ctx &c, float *xs) {
  pcg(c, 0, 1, 0);
  const size_t n = (size_t)c.im * c.jm;
  std::memcpy(xs, c.F[NPOM_F_elf], n * 4);
  each_cell(c, [&](int i, int j) {
    const size_t q = NPOM_I2(c, i, j);
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
    P2(d, i, j) = F2(h, i, j) + ev;
    P2(elf, i, j) = ev;
  });
}

// its reverse: g = dJ/dx, the eta-solve adjoint (npom_pcg_adjoint restated
// on the host with the same bodies), the rhs and transports
void imp_reverse(const Ctx &c, const Adj &a, const float *xs, float *g, float *lam, float *gd) {
  const size_t n = (size_t)c.im * c.jm;
  each_cell(c, [&](int i, int j) { g[NPOM_I2(c, i, j)] = imp_post_grad(c, a, i, j); });
  float amax = 0.0f;
  each_cell(c, [&](int i, int j) {
    const size_t o = NPOM_I2(c, i, j);
    const float v = g[o] / adj_area(c, i, j);
    c.W[NPOM_W_rhs][o] = v;
    amax = std::max(amax, std::fabs(v));
  });
  const float scale = amax > 1.0f ? amax : 1.0f;
  for (size_t o = 0; o < n; ++o) {
    c.W[NPOM_W_rhs][o] = c.W[NPOM_W_rhs][o] / scale;
    lam[o] = 0.0f;
  }
  Ctx ca = c;
  ca.F[NPOM_F_elf] = lam;
  ca.k.eta_tol = c.k.eta_tol / (double)scale;
  pcg(ca, 0, 0, 0);
  each_cell(c, [&](int i, int j) { gd[NPOM_I2(c, i, j)] = adj_grad_d_cell(c, xs, lam, scale, i, j); });
  each_cell(c, [&](int i, int j) {
    const size_t o = NPOM_I2(c, i, j);
    lam[o] = (lam[o] * adj_area(c, i, j)) * scale;
  });
  each_cell(c, [&](int i, int j) { imp_rhs_cell_adj(c, a, i, j, lam, gd); });
}

void fwd_plan_phase(const Ctx &c, const AdjPhaseRec &r, float *xs) {
  switch (r.phase) {
    case AP_EI: imp_forward(c, xs); break;
    case AP_I5: each_cell(c, [&](int i, int j) { (void)phase_i5_cell(c, i, j); }); break;
    case AP_A1: a1(c); break;
    case AP_A2: each_cell(c, [&](int i, int j) { phase_a2_column(c, i, j); }); break;
    case AP_A3: each_cell(c, [&](int i, int j) { phase_a3_cell(c, i, j); }); break;
    case AP_E1: each_cell(c, [&](int i, int j) { ext_phase1_cell(c, i, j, r.adv != 0); }); break;
    case AP_E2: each_cell(c, [&](int i, int j) { (void)ext_phase2_cell(c, i, j, r.iext); }); break;
    case AP_E3: each_cell(c, [&](int i, int j) { ext_phase3_cell(c, i, j, r.iext); }); break;
    case AP_B1: each_cell(c, [&](int i, int j) { phase_b1_column(c, i, j); }); break;
    case AP_B2A: each_cell(c, [&](int i, int j) { phase_b2a_column(c, i, j); }); break;
    case AP_B2B: each_point(c, [&](int i, int j, int k) { phase_b2b_point(c, i, j, k); }); break;
    case AP_B3: each_cell(c, [&](int i, int j) { phase_b3_column(c, i, j); }); break;
    case AP_B4: each_point(c, [&](int i, int j, int k) { phase_b4_point(c, i, j, k); }); break;
    case AP_B5: each_point(c, [&](int i, int j, int k) { phase_b5_point(c, i, j, k); }); break;
    case AP_B6: each_cell(c, [&](int i, int j) { phase_b6_column(c, i, j); }); break;
    case AP_B7: each_point(c, [&](int i, int j, int k) { phase_b7_point(c, i, j, k); }); break;
    case AP_B8: each_cell(c, [&](int i, int j) { phase_b8_column(c, i, j); }); break;
    case AP_B9: each_cell(c, [&](int i, int j) { phase_b9_column(c, i, j); }); break;
    case AP_MQ:
    case AP_MINIT:
    case AP_MUP:
    case AP_MFC:
    case AP_MAD:
    case AP_MDIF:
    case AP_MFIN:
      each_point(c, [&](int i, int j, int k) { phase_b5_mpdata_point(c, mp_pass_of(r.phase), r.iext, i, j, k); });
      break;
  }
}

void adj_plan_phase(const Ctx &c, const Adj &a, const AdjPhaseRec &r, const float *xs, float *g, float *lam,
                    float *gd) {
  switch (r.phase) {
    case AP_EI: imp_reverse(c, a, xs, g, lam, gd); break;
    case AP_I5: each_cell(c, [&](int i, int j) { phase_i5_cell_adj(c, a, i, j); }); break;
    case AP_A1: each_point(c, [&](int i, int j, int k) { phase_a1_point_adj(c, a, i, j, k); }); break;
    case AP_A2: each_cell(c, [&](int i, int j) { phase_a2_column_adj<KMAX>(c, a, i, j); }); break;
    case AP_A3: each_cell(c, [&](int i, int j) { phase_a3_cell_adj(c, a, i, j); }); break;
    case AP_E1: each_cell(c, [&](int i, int j) { ext_phase1_cell_adj(c, a, i, j, r.adv != 0); }); break;
    case AP_E2: each_cell(c, [&](int i, int j) { ext_phase2_cell_adj(c, a, i, j, r.iext); }); break;
    case AP_E3: each_cell(c, [&](int i, int j) { ext_phase3_cell_adj(c, a, i, j, r.iext); }); break;
    case AP_B1: each_cell(c, [&](int i, int j) { phase_b1_column_adj<KMAX>(c, a, i, j); }); break;
    case AP_B2A: each_cell(c, [&](int i, int j) { phase_b2a_column_adj<KMAX>(c, a, i, j); }); break;
    case AP_B2B: each_point(c, [&](int i, int j, int k) { phase_b2b_point_adj(c, a, i, j, k); }); break;
    case AP_B3: each_cell(c, [&](int i, int j) { phase_b3_column_adj<KMAX>(c, a, i, j); }); break;
    case AP_B4: each_point(c, [&](int i, int j, int k) { phase_b4_point_adj(c, a, i, j, k); }); break;
    case AP_B5: each_point(c, [&](int i, int j, int k) { phase_b5_point_adj(c, a, i, j, k); }); break;
    case AP_B6: each_cell(c, [&](int i, int j) { phase_b6_column_adj<KMAX>(c, a, i, j); }); break;
    case AP_B7: each_point(c, [&](int i, int j, int k) { phase_b7_point_adj(c, a, i, j, k); }); break;
    case AP_B8: each_cell(c, [&](int i, int j) { phase_b8_column_adj<KMAX>(c, a, i, j); }); break;
    case AP_B9: each_cell(c, [&](int i, int j) { phase_b9_column_adj<KMAX>(c, a, i, j); }); break;
    case AP_MQ:
    case AP_MINIT:
    case AP_MUP:
    case AP_MFC:
    case AP_MAD:
    case AP_MDIF:
    case AP_MFIN:
      each_point(c, [&](int i, int j, int k) { mp_phase_adj(c, a, r.phase, r.iext, i, j, k); });
      break;
  }
}

}  // namespace

extern "C" {

// CPU emulation of npom_step_explicit_adjoint: same plan, same bodies.
// stop_after >= 0 ends the reverse sweep after that many phases (tests of
// single phases); -1 runs all of them.
int emul_step_adjoint(const npom_params *p, float *const *fields, const npom_workspace *ws, const npom_clock *clk,
                      float *const *grads, float *const *lam, float *save, size_t save_floats, int stop_after) {
  if (!check_args(p, fields, ws) || !clk || clk->nsteps != 1 || !adj_supported(p)) return 1;
  Ctx c = make_ctx(p, fields, ws);
  const int iint = clk->first_iint;
  const double time = p->dti * iint * 1.0 / 86400.0 + clk->time0;
  c.ramp = ramp_of(p, time);
  c.do_internal = (iint != 1 || clk->time0 != 0.0) ? 1 : 0;
  Adj a;
  for (int f = 0; f < NPOM_NFIELDS; ++f) {
    a.G[f] = grads[f];
    a.L[f] = lam[f];
  }
  std::vector<AdjPhaseRec> plan((size_t)adj_plan_capacity(p->isplit, p->nitera));
  size_t need = 0;
  const int np = adj_step_plan(c, plan.data(), (int)plan.size(), &need);
  const size_t ncell = (size_t)c.im * c.jm;
  if (need + adj_scratch_floats(c) > save_floats) return 2;
  float *scratch = save + need;
  std::memset(scratch, 0, adj_scratch_floats(c) * 4);
  adj_bind_scratch(c, a, scratch);
  float *xs = scratch + (size_t)(2 * AW_COUNT) * ncell, *g = xs + ncell, *lamw = g + ncell, *gd = lamw + ncell;
  if (p->core == NPOM_CORE_IMPLICIT) each_cell(c, [&](int i, int j) { elliptic_coeff_cell(c, i, j); });
  for (int q = 0; q < np; ++q) {
    const AdjPhaseRec &r = plan[q];
    for (int e = 0; e < r.n; ++e)
      std::memcpy(save + r.off[e], adj_fptr(c, r.fld[e]), adj_field_len(c, r.fld[e]) * 4);
    fwd_plan_phase(c, r, xs);
  }
  int done = 0;
  for (int q = np - 1; q >= 0; --q) {
    if (stop_after >= 0 && done >= stop_after) break;
    const AdjPhaseRec &r = plan[q];
    for (int e = 0; e < r.n; ++e) {
      const int f = r.fld[e];
      const size_t n = adj_field_len(c, f);
      std::memcpy(adj_fptr(c, f), save + r.off[e], n * 4);
      if (r.move[e]) {
        std::memcpy(a.L[f], a.G[f], n * 4);
        std::memset(a.G[f], 0, n * 4);
      }
    }
    adj_plan_phase(c, a, r, xs, g, lamw, gd);
    ++done;
  }
  return 0;
}

// the number of phases of one step and the save area they need
int emul_adjoint_plan(const npom_params *p, int do_internal, size_t *save_floats) {
  Ctx c;
  std::memset(&c, 0, sizeof(c));
  c.im = p->im;
  c.jm = p->jm;
  c.kb = p->kb;
  c.k = make_consts(*p);
  c.do_internal = do_internal;
  std::vector<AdjPhaseRec> plan((size_t)adj_plan_capacity(p->isplit, p->nitera));
  const int np = adj_step_plan(c, plan.data(), (int)plan.size(), save_floats);
  *save_floats += adj_scratch_floats(c);
  return np;
}

int emul_run_phase(const npom_params *p, float *const *fields, const npom_workspace *ws, int phase, double ramp) {
  if (!check_args(p, fields, ws)) return 1;
  Ctx c = make_ctx(p, fields, ws);
  c.ramp = (float)ramp;
  c.do_internal = 1;
  run_phase(c, p, phase);
  return 0;
}

int emul_steps(const npom_params *p, float *const *fields, const npom_workspace *ws, const npom_clock *clk) {
  if (!check_args(p, fields, ws) || !clk) return 1;
  Ctx c = make_ctx(p, fields, ws);
  if (p->core == NPOM_CORE_IMPLICIT) each_cell(c, [&](int i, int j) { elliptic_coeff_cell(c, i, j); });
  for (int n = 0; n < clk->nsteps; ++n) {
    int iint = clk->first_iint + n;
    double time = p->dti * iint * 1.0 / 86400.0 + clk->time0;
    c.ramp = ramp_of(p, time);
    c.do_internal = ((iint != 1 || clk->time0 != 0.0) && p->mode != 2) ? 1 : 0;
    c.tide_t0 = time * 86400.0 - (p->core == NPOM_CORE_IMPLICIT ? p->dte : p->dti);
    run_phase(c, p, 0);
    run_phase(c, p, 1);
    run_phase(c, p, 2);
    if (p->core == NPOM_CORE_IMPLICIT) {
      if (c.k.obc_coastal) cg_policy(c, n);
      else if (c.k.sea_implicit) robin_picard(c, n);
      else pcg(c, n, 1, 1);
      wrap_x(c);
      run_phase(c, p, 4);
    } else {
      subcycle(c);
      if (c.k.obc_coastal) each_cell(c, [&](int i, int j) { cbc_coastal_cell(c, i, j); });
    }
    if (c.do_internal)
      for (int ph = 5; ph <= 13; ++ph) run_phase(c, p, ph);
    run_phase(c, p, 14);
  }
  return 0;
}

}  // extern "C"
