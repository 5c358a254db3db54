// npom_adjoint.cuh -- hand-written adjoint (reverse-mode) of every phase of
// the explicit core's internal step (explicit/time_loop.py:20-709).
//
// Convention.  Ctx c holds the model state as it was BEFORE the phase ran
// (the caller restores it from the per-phase saves); Adj a holds
//   G[f]: the running cotangent of every state field, and
//   L[f]: for each field the phase overwrites, the cotangent of its new
//         value, moved out of G (G[f] is zeroed by the move).
// An adjoint body visits the element(s) its forward body computes,
// recomputes the forward intermediates it needs, and scatters
// lambda * d(output)/d(input) into G of every differentiable input.  For an
// element of an overwritten field that the forward body leaves untouched
// the body passes L straight back into G.  Scatters are atomic on the
// device (several outputs share an input); the CPU emulation adds in order.
//
// Derivatives follow torch autograd's conventions on the reference's
// operations: |x| has derivative sign(x) (0 at 0), clamp/where pass the
// gradient only on the kept branch, the Smagorinsky vector norm has a zero
// gradient at the origin (time_loop.py:8-14), sqrt(x + eps) is smooth.
// Geometry, forcing and boundary arrays are constants.
#pragma once

#include "npom_phases_int.cuh"

namespace npom {

// Workspace arrays that carry a cotangent inside an implicit step (written
// by the predictor, read by the free-surface solve and the corrector): their
// slots follow the fields in Adj.
enum AdjWs { AW_us = 0, AW_vs, AW_den_u, AW_den_v, AW_d_baro, AW_COUNT };
// The MPDATA scratch (nadv 2: per tracer xm ym zw xf yf zf, 3-D) carries a
// cotangent between the passes of B5: its slots follow the workspace's.
constexpr int kAdjMpSlots = 12;
constexpr int kAdjSlots = NPOM_NFIELDS + AW_COUNT + kAdjMpSlots;
NPOM_HD int mp_slot(int tracer, int arr) { return NPOM_NFIELDS + AW_COUNT + tracer * 6 + arr; }

NPOM_HD int aw_ws(int k) {
  return k == AW_us ? NPOM_W_us
                    : (k == AW_vs ? NPOM_W_vs : (k == AW_den_u ? NPOM_W_den_u : (k == AW_den_v ? NPOM_W_den_v : NPOM_W_d_baro)));
}

struct Adj {
  float *G[kAdjSlots];
  float *L[kAdjSlots];
};

// state array of a slot: a field, a workspace array or an MPDATA scratch array
NPOM_HD float *adj_fptr(const Ctx &c, int id) {
  if (id < NPOM_NFIELDS) return c.F[id];
  if (id < NPOM_NFIELDS + AW_COUNT) return c.W[aw_ws(id - NPOM_NFIELDS)];
  return c.mp3d + (size_t)(id - NPOM_NFIELDS - AW_COUNT) * ((size_t)c.im * c.jm * c.kb);
}

NPOM_HD void aadd(float *p, float v) {
#if defined(__CUDA_ARCH__)
  if (v != 0.0f) atomicAdd(p, v);
#else
  *p += v;
#endif
}

NPOM_HD float sgnf(float x) { return x > 0.0f ? 1.0f : (x < 0.0f ? -1.0f : 0.0f); }

#define GA3(name, i, j, k, v) ::npom::aadd(&a.G[NPOM_F_##name][NPOM_I3(c, i, j, k)], (v))
#define GA2(name, i, j, v) ::npom::aadd(&a.G[NPOM_F_##name][NPOM_I2(c, i, j)], (v))
#define LA3(name, i, j, k) (a.L[NPOM_F_##name][NPOM_I3(c, i, j, k)])
#define LA2(name, i, j) (a.L[NPOM_F_##name][NPOM_I2(c, i, j)])
#define PASS3(name, i, j, k) GA3(name, i, j, k, LA3(name, i, j, k))
#define PASS2(name, i, j) GA2(name, i, j, LA2(name, i, j))
#define GAW(k, i, j, v) ::npom::aadd(&a.G[NPOM_NFIELDS + (k)][NPOM_I2(c, i, j)], (v))
#define LAW(k, i, j) (a.L[NPOM_NFIELDS + (k)][NPOM_I2(c, i, j)])

// ===========================================================================
// A1: ADVCT (baroclinic.py:14-260) and the surface forcing
// ===========================================================================
NPOM_HD void advct_curv_adj(const Ctx &c, const Adj &a, int i, int j, int k, float lam) {
  if (lam == 0.0f || !interior(c, i, j)) return;
  const float D = F2(dx, i, j) * F2(dy, i, j) + 1e-20f;
  const float cv = 0.25f * (F2(dy, i + 1, j) - F2(dy, i - 1, j)) / D * lam;
  const float cu = -0.25f * (F2(dx, i, j + 1) - F2(dx, i, j - 1)) / D * lam;
  GA3(v, i, j + 1, k, cv);
  GA3(v, i, j, k, cv);
  GA3(u, i + 1, j, k, cu);
  GA3(u, i, j, k, cu);
}

NPOM_HD void advct_xflux_u_adj(const Ctx &c, const Adj &a, int ip, int j, int k, float lam) {
  if (lam == 0.0f || ip < 1 || ip > c.im - 2) return;
  const float dA = F2(dt, ip + 1, j), dB = F2(dt, ip, j), dC = F2(dt, ip - 1, j);
  const float u1 = F3(u, ip + 1, j, k), u0 = F3(u, ip, j, k);
  float l0 = lam;
  if (j >= 1) {
    const float dxs = F2(dx, ip, j) + 1e-20f;
    const float gu = (F3(ub, ip + 1, j, k) - F3(ub, ip, j, k)) / dxs;
    const float am = F3(aam, ip, j, k);
    l0 = lam * F2(dy, ip, j);
    const float lg = -l0 * dB * am * 2.0f;
    GA2(dt, ip, j, -l0 * am * 2.0f * gu);
    GA3(aam, ip, j, k, -l0 * dB * 2.0f * gu);
    GA3(ub, ip + 1, j, k, lg / dxs);
    GA3(ub, ip, j, k, -lg / dxs);
  }
  const float sa = dA + dB, sb = dB + dC;
  const float s = sa * u1 + sb * u0, su = u1 + u0;
  const float ls = l0 * 0.125f * su, lsu = l0 * 0.125f * s;
  GA3(u, ip + 1, j, k, ls * sa + lsu);
  GA3(u, ip, j, k, ls * sb + lsu);
  GA2(dt, ip + 1, j, ls * u1);
  GA2(dt, ip, j, ls * (u1 + u0));
  GA2(dt, ip - 1, j, ls * u0);
}

NPOM_HD void advct_shear_adj(const Ctx &c, const Adj &a, int i, int j, int k, float lam) {
  if (lam == 0.0f) return;
  const float dt_avg = 0.25f * (F2(dt, i, j) + F2(dt, i - 1, j) + F2(dt, i, j - 1) + F2(dt, i - 1, j - 1));
  const float aam_sum = F3(aam, i, j, k) + F3(aam, i - 1, j, k) + F3(aam, i, j - 1, k) + F3(aam, i - 1, j - 1, k);
  const float den_dy = F2(dy, i, j) + F2(dy, i - 1, j) + F2(dy, i, j - 1) + F2(dy, i - 1, j - 1) + 1e-20f;
  const float den_dx = F2(dx, i, j) + F2(dx, i - 1, j) + F2(dx, i, j - 1) + F2(dx, i - 1, j - 1) + 1e-20f;
  const float g = (F3(ub, i, j, k) - F3(ub, i, j - 1, k)) / den_dy + (F3(vb, i, j, k) - F3(vb, i - 1, j, k)) / den_dx;
  const float ldt = lam * g * aam_sum * 0.25f;
  GA2(dt, i, j, ldt);
  GA2(dt, i - 1, j, ldt);
  GA2(dt, i, j - 1, ldt);
  GA2(dt, i - 1, j - 1, ldt);
  const float la = lam * g * dt_avg;
  GA3(aam, i, j, k, la);
  GA3(aam, i - 1, j, k, la);
  GA3(aam, i, j - 1, k, la);
  GA3(aam, i - 1, j - 1, k, la);
  const float lg = lam * dt_avg * aam_sum;
  GA3(ub, i, j, k, lg / den_dy);
  GA3(ub, i, j - 1, k, -lg / den_dy);
  GA3(vb, i, j, k, lg / den_dx);
  GA3(vb, i - 1, j, k, -lg / den_dx);
}

NPOM_HD void advct_yflux_u_adj(const Ctx &c, const Adj &a, int i, int jp, int k, float lam) {
  if (lam == 0.0f || i < 1 || jp < 1) return;
  float l0 = lam;
  if (i <= c.im - 2) {
    const float dx_sum = F2(dx, i, jp) + F2(dx, i - 1, jp) + F2(dx, i, jp - 1) + F2(dx, i - 1, jp - 1);
    l0 = lam * 0.25f * dx_sum;
    advct_shear_adj(c, a, i, jp, k, -l0);
  }
  const float sa = F2(dt, i, jp) + F2(dt, i, jp - 1), sb = F2(dt, i - 1, jp) + F2(dt, i - 1, jp - 1);
  const float v1 = F3(v, i, jp, k), v0 = F3(v, i - 1, jp, k);
  const float s = sa * v1 + sb * v0, su = F3(u, i, jp, k) + F3(u, i, jp - 1, k);
  const float ls = l0 * 0.125f * su, lsu = l0 * 0.125f * s;
  GA3(v, i, jp, k, ls * sa);
  GA3(v, i - 1, jp, k, ls * sb);
  GA2(dt, i, jp, ls * v1);
  GA2(dt, i, jp - 1, ls * v1);
  GA2(dt, i - 1, jp, ls * v0);
  GA2(dt, i - 1, jp - 1, ls * v0);
  GA3(u, i, jp, k, lsu);
  GA3(u, i, jp - 1, k, lsu);
}

NPOM_HD void advct_xflux_v_adj(const Ctx &c, const Adj &a, int ip, int j, int k, float lam) {
  if (lam == 0.0f || ip < 1 || j < 1) return;
  float l0 = lam;
  if (j <= c.jm - 2) {
    const float dy_sum = F2(dy, ip, j) + F2(dy, ip - 1, j) + F2(dy, ip, j - 1) + F2(dy, ip - 1, j - 1);
    l0 = lam * 0.25f * dy_sum;
    advct_shear_adj(c, a, ip, j, k, -l0);
  }
  const float sa = F2(dt, ip, j) + F2(dt, ip - 1, j), sb = F2(dt, ip, j - 1) + F2(dt, ip - 1, j - 1);
  const float u1 = F3(u, ip, j, k), u0 = F3(u, ip, j - 1, k);
  const float s = sa * u1 + sb * u0, sv = F3(v, ip, j, k) + F3(v, ip - 1, j, k);
  const float ls = l0 * 0.125f * sv, lsv = l0 * 0.125f * s;
  GA3(u, ip, j, k, ls * sa);
  GA3(u, ip, j - 1, k, ls * sb);
  GA2(dt, ip, j, ls * u1);
  GA2(dt, ip - 1, j, ls * u1);
  GA2(dt, ip, j - 1, ls * u0);
  GA2(dt, ip - 1, j - 1, ls * u0);
  GA3(v, ip, j, k, lsv);
  GA3(v, ip - 1, j, k, lsv);
}

NPOM_HD void advct_yflux_v_adj(const Ctx &c, const Adj &a, int i, int jp, int k, float lam) {
  if (lam == 0.0f || jp < 1 || jp > c.jm - 2) return;
  const float dA = F2(dt, i, jp + 1), dB = F2(dt, i, jp), dC = F2(dt, i, jp - 1);
  const float v1 = F3(v, i, jp + 1, k), v0 = F3(v, i, jp, k);
  float l0 = lam;
  if (i >= 1) {
    const float dys = F2(dy, i, jp) + 1e-20f;
    const float gv = (F3(vb, i, jp + 1, k) - F3(vb, i, jp, k)) / dys;
    const float am = F3(aam, i, jp, k);
    l0 = lam * F2(dx, i, jp);
    const float lg = -l0 * dB * am * 2.0f;
    GA2(dt, i, jp, -l0 * am * 2.0f * gv);
    GA3(aam, i, jp, k, -l0 * dB * 2.0f * gv);
    GA3(vb, i, jp + 1, k, lg / dys);
    GA3(vb, i, jp, k, -lg / dys);
  }
  const float sa = dA + dB, sb = dB + dC;
  const float s = sa * v1 + sb * v0, sv = v1 + v0;
  const float ls = l0 * 0.125f * sv, lsv = l0 * 0.125f * s;
  GA3(v, i, jp + 1, k, ls * sa + lsv);
  GA3(v, i, jp, k, ls * sb + lsv);
  GA2(dt, i, jp + 1, ls * v1);
  GA2(dt, i, jp, ls * (v1 + v0));
  GA2(dt, i, jp - 1, ls * v0);
}

// one point of A1: advx/advy/curv are written everywhere (zero off the
// interior and on the ghost level); the forcing zeroes w(:, :, 0) on the
// interior, every other element of w passes through
NPOM_HD void phase_a1_point_adj(const Ctx &c, const Adj &a, int i, int j, int k) {
  if (!(k == 0 && interior(c, i, j))) PASS3(w, i, j, k);
  if (k >= c.kb - 1 || !interior(c, i, j)) return;
  const float lx = LA3(advx, i, j, k), ly = LA3(advy, i, j, k);
  float lcurv = LA3(curv, i, j, k);
  advct_xflux_u_adj(c, a, i, j, k, lx);
  advct_xflux_u_adj(c, a, i - 1, j, k, -lx);
  advct_yflux_u_adj(c, a, i, j + 1, k, lx);
  advct_yflux_u_adj(c, a, i, j, k, -lx);
  if (i >= 2 && lx != 0.0f) {
    const float mu = -F2(aru, i, j) * 0.25f * lx;
    const float cv = advct_curv(c, i, j, k), cm = advct_curv(c, i - 1, j, k);
    const float vs0 = F3(v, i, j + 1, k) + F3(v, i, j, k), vs1 = F3(v, i - 1, j + 1, k) + F3(v, i - 1, j, k);
    const float d0 = F2(dt, i, j), d1 = F2(dt, i - 1, j);
    lcurv += mu * d0 * vs0;
    GA2(dt, i, j, mu * cv * vs0);
    GA3(v, i, j + 1, k, mu * cv * d0);
    GA3(v, i, j, k, mu * cv * d0);
    advct_curv_adj(c, a, i - 1, j, k, mu * d1 * vs1);
    GA2(dt, i - 1, j, mu * cm * vs1);
    GA3(v, i - 1, j + 1, k, mu * cm * d1);
    GA3(v, i - 1, j, k, mu * cm * d1);
  }
  advct_xflux_v_adj(c, a, i + 1, j, k, ly);
  advct_xflux_v_adj(c, a, i, j, k, -ly);
  advct_yflux_v_adj(c, a, i, j, k, ly);
  advct_yflux_v_adj(c, a, i, j - 1, k, -ly);
  if (j >= 2 && ly != 0.0f) {
    const float mu = F2(arv, i, j) * 0.25f * ly;
    const float cv = advct_curv(c, i, j, k), cm = advct_curv(c, i, j - 1, k);
    const float us0 = F3(u, i + 1, j, k) + F3(u, i, j, k), us1 = F3(u, i + 1, j - 1, k) + F3(u, i, j - 1, k);
    const float d0 = F2(dt, i, j), d1 = F2(dt, i, j - 1);
    lcurv += mu * d0 * us0;
    GA2(dt, i, j, mu * cv * us0);
    GA3(u, i + 1, j, k, mu * cv * d0);
    GA3(u, i, j, k, mu * cv * d0);
    advct_curv_adj(c, a, i, j - 1, k, mu * d1 * us1);
    GA2(dt, i, j - 1, mu * cm * us1);
    GA3(u, i + 1, j - 1, k, mu * cm * d1);
    GA3(u, i, j - 1, k, mu * cm * d1);
  }
  advct_curv_adj(c, a, i, j, k, lcurv);
}

// ===========================================================================
// A2: BAROPG (momentum.py:543-700), Smagorinsky (time_loop.py:8-14,193-233),
// depth integrals (time_loop.py:240-258)
// ===========================================================================
NPOM_HD void smag_level_adj(const Ctx &c, const Adj &a, int i, int j, int k, float lam) {
  if (lam == 0.0f) return;
  const float dxs = F2(dx, i, j), dys = F2(dy, i, j);
  const float du_dx = (F3(u, i + 1, j, k) - F3(u, i, j, k)) / dxs;
  const float dv_dy = (F3(v, i, j + 1, k) - F3(v, i, j, k)) / dys;
  const float u_term =
      0.25f * (F3(u, i, j + 1, k) + F3(u, i + 1, j + 1, k) - F3(u, i, j - 1, k) - F3(u, i + 1, j - 1, k)) / dys;
  const float v_term =
      0.25f * (F3(v, i + 1, j, k) + F3(v, i + 1, j + 1, k) - F3(v, i - 1, j, k) - F3(v, i - 1, j + 1, k)) / dxs;
  float mag, gsh;  // the norm and d(norm^2)/2 per unit of (u_term + v_term), times mag
  if (is_explicit(c)) {
    const float cc = (u_term + v_term) * c.k.sqrt_half;
    mag = sqrtf(du_dx * du_dx + dv_dy * dv_dy + cc * cc);
    gsh = cc * c.k.sqrt_half;
  } else {
    const float sh = u_term + v_term;
    mag = sqrtf(du_dx * du_dx + dv_dy * dv_dy + 0.5f * (sh * sh));
    gsh = 0.5f * sh;
    if (c.k.aam_min > 0.0f && !(c.k.horcon * dxs * dys * mag >= c.k.aam_min)) return;  // clamped
  }
  // the norm's gradient is zero at the origin (explicit time_loop.py:8-14,
  // implicit autograd.py:5-29)
  if (!(mag > 0.0f)) return;
  const float lm = lam * c.k.horcon * dxs * dys / mag;
  const float ldu = lm * du_dx / dxs, ldv = lm * dv_dy / dys, lcc = lm * gsh;
  GA3(u, i + 1, j, k, ldu);
  GA3(u, i, j, k, -ldu);
  GA3(v, i, j + 1, k, ldv);
  GA3(v, i, j, k, -ldv);
  const float lut = lcc * 0.25f / dys, lvt = lcc * 0.25f / dxs;
  GA3(u, i, j + 1, k, lut);
  GA3(u, i + 1, j + 1, k, lut);
  GA3(u, i, j - 1, k, -lut);
  GA3(u, i + 1, j - 1, k, -lut);
  GA3(v, i + 1, j, k, lvt);
  GA3(v, i + 1, j + 1, k, lvt);
  GA3(v, i - 1, j, k, -lvt);
  GA3(v, i - 1, j + 1, k, -lvt);
}

template <int KM>
NPOM_HD void baropg_column_adj(const Ctx &c, const Adj &a, int i, int j, const float *lamx, const float *lamy) {
  const int kbm1 = (KM == 16 ? 16 : c.kb) - 1;
  const float ramp = c.ramp;
  for (int comp = 0; comp < 2; ++comp) {
    const float *lam = comp == 0 ? lamx : lamy;
    const int bi = comp == 0 ? i - 1 : i;
    const int bj = comp == 0 ? j : j - 1;
    const float term_dt = F2(dt, i, j) + F2(dt, bi, bj);
    const float dt_diff = F2(dt, i, j) - F2(dt, bi, bj);
    float r[KM], rb[KM], V[KM], lr[KM], lrb[KM];
    for (int k = 0; k < kbm1; ++k) {
      r[k] = F3(rho, i, j, k) - F3(rmean, i, j, k);
      rb[k] = F3(rho, bi, bj, k) - F3(rmean, bi, bj, k);
      lr[k] = 0.0f;
      lrb[k] = 0.0f;
    }
    const float val0 = c.k.half_g * (-F1(zz, 0)) * term_dt * (r[0] - rb[0]);
    const float mask = comp == 0 ? F2(dum, i, j) : F2(dvm, i, j);
    const float area = comp == 0 ? (F2(dy, i, j) + F2(dy, bi, bj)) : (F2(dx, i, j) + F2(dx, bi, bj));
    const float scale = 0.25f * term_dt * mask * area;
    V[0] = val0;
    double acc = 0.0;
    for (int k = 1; k < kbm1; ++k) {
      const float zzk = F1(zz, k), zzkm = F1(zz, k - 1);
      float term1 = c.k.quarter_g * (zzkm - zzk) * term_dt * ((r[k] - rb[k]) + (r[k - 1] - rb[k - 1]));
      float term2 = c.k.quarter_g * (zzkm + zzk) * dt_diff * ((r[k] + rb[k]) - (r[k - 1] + rb[k - 1]));
      acc += (double)(term1 + term2);
      V[k] = val0 + (float)acc;
    }
    float lscale = 0.0f, lterm_dt = 0.0f, ldt_diff = 0.0f, S = 0.0f;
    for (int k = 0; k < kbm1; ++k) lscale += lam[k] * V[k] * ramp;
    for (int k = kbm1 - 1; k >= 1; --k) {
      S += lam[k] * scale * ramp;
      const float zzk = F1(zz, k), zzkm = F1(zz, k - 1);
      const float A = c.k.quarter_g * (zzkm - zzk);
      const float X = (r[k] - rb[k]) + (r[k - 1] - rb[k - 1]);
      lterm_dt += S * A * X;
      const float lX = S * A * term_dt;
      lr[k] += lX;
      lrb[k] -= lX;
      lr[k - 1] += lX;
      lrb[k - 1] -= lX;
      const float B = c.k.quarter_g * (zzkm + zzk);
      const float Y = (r[k] + rb[k]) - (r[k - 1] + rb[k - 1]);
      ldt_diff += S * B * Y;
      const float lY = S * B * dt_diff;
      lr[k] += lY;
      lrb[k] += lY;
      lr[k - 1] -= lY;
      lrb[k - 1] -= lY;
    }
    const float lval0 = S + lam[0] * scale * ramp;
    const float c0 = c.k.half_g * (-F1(zz, 0));
    lterm_dt += lval0 * c0 * (r[0] - rb[0]);
    const float l01 = lval0 * c0 * term_dt;
    lr[0] += l01;
    lrb[0] -= l01;
    lterm_dt += lscale * 0.25f * mask * area;
    GA2(dt, i, j, lterm_dt + ldt_diff);
    GA2(dt, bi, bj, lterm_dt - ldt_diff);
    for (int k = 0; k < kbm1; ++k) {
      GA3(rho, i, j, k, lr[k]);
      GA3(rho, bi, bj, k, lrb[k]);
    }
  }
}

template <int KM>
NPOM_HD void phase_a2_column_adj(const Ctx &c, const Adj &a, int i, int j) {
  const int kb = KM == 16 ? 16 : c.kb, kbm1 = kb - 1;
  const bool inner = interior(c, i, j);
  const float lsx = LA2(adx2d, i, j), lsy = LA2(ady2d, i, j), lrx = LA2(drx2d, i, j), lry = LA2(dry2d, i, j);
  const float lsa = LA2(aam2d, i, j);
  float lrhox[KM], lrhoy[KM], laam[KM];
  for (int k = 0; k < kb; ++k) {
    lrhox[k] = LA3(drhox, i, j, k);
    lrhoy[k] = LA3(drhoy, i, j, k);
    laam[k] = LA3(aam, i, j, k);
  }
  for (int k = 0; k < kbm1; ++k) {
    const float dzk = F1(dz, k);
    GA3(advx, i, j, k, lsx * dzk);
    GA3(advy, i, j, k, lsy * dzk);
    lrhox[k] += lrx * dzk;
    lrhoy[k] += lry * dzk;
    laam[k] += lsa * dzk;
  }
  if (inner) {
    for (int k = 0; k < kbm1; ++k) smag_level_adj(c, a, i, j, k, laam[k]);
    GA3(aam, i, j, kbm1, laam[kbm1]);
    baropg_column_adj<KM>(c, a, i, j, lrhox, lrhoy);
  } else {
    for (int k = 0; k < kb; ++k) GA3(aam, i, j, k, laam[k]);
  }
}

// ===========================================================================
// ADVAVE, mode 3 (baroclinic.py:262-494)
// ===========================================================================
NPOM_HD void advave_tps_adj(const Ctx &c, const Adj &a, int i, int j, float lam) {
  if (lam == 0.0f) return;
  const float d_sum = F2(d, i, j) + F2(d, i - 1, j) + F2(d, i, j - 1) + F2(d, i - 1, j - 1);
  const float aam_sum = F2(aam2d, i, j) + F2(aam2d, i, j - 1) + F2(aam2d, i - 1, j) + F2(aam2d, i - 1, j - 1);
  const float dy_sum = F2(dy, i, j) + F2(dy, i - 1, j) + F2(dy, i, j - 1) + F2(dy, i - 1, j - 1);
  const float dx_sum = F2(dx, i, j) + F2(dx, i - 1, j) + F2(dx, i, j - 1) + F2(dx, i - 1, j - 1);
  const float g = (F2(uab, i, j) - F2(uab, i, j - 1)) / dy_sum + (F2(vab, i, j) - F2(vab, i - 1, j)) / dx_sum;
  const float ld = lam * 0.25f * aam_sum * g;
  GA2(d, i, j, ld);
  GA2(d, i - 1, j, ld);
  GA2(d, i, j - 1, ld);
  GA2(d, i - 1, j - 1, ld);
  const float la = lam * 0.25f * d_sum * g;
  GA2(aam2d, i, j, la);
  GA2(aam2d, i, j - 1, la);
  GA2(aam2d, i - 1, j, la);
  GA2(aam2d, i - 1, j - 1, la);
  const float lg = lam * 0.25f * d_sum * aam_sum;
  GA2(uab, i, j, lg / dy_sum);
  GA2(uab, i, j - 1, -lg / dy_sum);
  GA2(vab, i, j, lg / dx_sum);
  GA2(vab, i - 1, j, -lg / dx_sum);
}

NPOM_HD void advave_fluxua1_adj(const Ctx &c, const Adj &a, int i, int j, float lam) {
  if (lam == 0.0f) return;
  if (i < 1 || j < 1) {
    GA2(fluxua, i, j, lam);
    return;
  }
  const float d1 = F2(d, i + 1, j), d0 = F2(d, i, j), dm = F2(d, i - 1, j);
  const float u1 = F2(ua, i + 1, j), u0 = F2(ua, i, j);
  const float sa = d1 + d0, sb = d0 + dm;
  const float s = sa * u1 + sb * u0, su = u1 + u0;
  const float dxv = F2(dx, i, j);
  const float diff = (F2(uab, i + 1, j) - F2(uab, i, j)) / dxv;
  const float am = F2(aam2d, i, j);
  const float lf = lam * F2(dy, i, j);
  const float ls = lf * 0.125f * su, lsu = lf * 0.125f * s;
  GA2(ua, i + 1, j, ls * sa + lsu);
  GA2(ua, i, j, ls * sb + lsu);
  GA2(d, i + 1, j, ls * u1);
  GA2(d, i, j, ls * (u1 + u0) - lf * 2.0f * am * diff);
  GA2(d, i - 1, j, ls * u0);
  GA2(aam2d, i, j, -lf * d0 * 2.0f * diff);
  const float ldiff = -lf * d0 * 2.0f * am / dxv;
  GA2(uab, i + 1, j, ldiff);
  GA2(uab, i, j, -ldiff);
}

NPOM_HD void advave_fluxva1_adj(const Ctx &c, const Adj &a, int i, int j, float lam) {
  if (lam == 0.0f) return;
  if (i < 1 || j < 1) {
    GA2(fluxva, i, j, lam);
    return;
  }
  const float dA = F2(d, i, j) + F2(d, i, j - 1), dB = F2(d, i - 1, j) + F2(d, i - 1, j - 1);
  const float v1 = F2(va, i, j), v0 = F2(va, i - 1, j);
  const float s = dA * v1 + dB * v0, su = F2(ua, i, j) + F2(ua, i, j - 1);
  const float dx_sum = F2(dx, i, j) + F2(dx, i - 1, j) + F2(dx, i, j - 1) + F2(dx, i - 1, j - 1);
  const float lf = lam * 0.25f * dx_sum;
  advave_tps_adj(c, a, i, j, -lf);
  const float ls = lf * 0.125f * su, lsu = lf * 0.125f * s;
  GA2(d, i, j, ls * v1);
  GA2(d, i, j - 1, ls * v1);
  GA2(d, i - 1, j, ls * v0);
  GA2(d, i - 1, j - 1, ls * v0);
  GA2(va, i, j, ls * dA);
  GA2(va, i - 1, j, ls * dB);
  GA2(ua, i, j, lsu);
  GA2(ua, i, j - 1, lsu);
}

NPOM_HD void advave_fluxua2_adj(const Ctx &c, const Adj &a, int i, int j, float lam) {
  if (lam == 0.0f) return;
  if (i < 1 || j < 1) {
    GA2(fluxua, i, j, lam);
    return;
  }
  const float dA = F2(d, i, j) + F2(d, i - 1, j), dB = F2(d, i, j - 1) + F2(d, i - 1, j - 1);
  const float u1 = F2(ua, i, j), u0 = F2(ua, i, j - 1);
  const float s = dA * u1 + dB * u0, sv = F2(va, i - 1, j) + F2(va, i, j);
  const float dy_sum = F2(dy, i, j) + F2(dy, i - 1, j) + F2(dy, i, j - 1) + F2(dy, i - 1, j - 1);
  const float lf = lam * 0.25f * dy_sum;
  advave_tps_adj(c, a, i, j, -lf);
  const float ls = lf * 0.125f * sv, lsv = lf * 0.125f * s;
  GA2(d, i, j, ls * u1);
  GA2(d, i - 1, j, ls * u1);
  GA2(d, i, j - 1, ls * u0);
  GA2(d, i - 1, j - 1, ls * u0);
  GA2(ua, i, j, ls * dA);
  GA2(ua, i, j - 1, ls * dB);
  GA2(va, i - 1, j, lsv);
  GA2(va, i, j, lsv);
}

NPOM_HD void advave_fluxva2_adj(const Ctx &c, const Adj &a, int i, int j, float lam) {
  if (lam == 0.0f) return;
  if (i < 1 || j < 1) {
    GA2(fluxva, i, j, lam);
    return;
  }
  if (j == c.jm - 1) {
    advave_fluxva1_adj(c, a, i, j, lam * F2(dx, i, j));
    return;
  }
  const float d1 = F2(d, i, j + 1), d0 = F2(d, i, j), dm = F2(d, i, j - 1);
  const float v1 = F2(va, i, j + 1), v0 = F2(va, i, j);
  const float sa = d1 + d0, sb = d0 + dm;
  const float s = sa * v1 + sb * v0, sv = v1 + v0;
  const float dyv = F2(dy, i, j);
  const float diff = (F2(vab, i, j + 1) - F2(vab, i, j)) / dyv;
  const float am = F2(aam2d, i, j);
  const float lf = lam * F2(dx, i, j);
  const float ls = lf * 0.125f * sv, lsv = lf * 0.125f * s;
  GA2(va, i, j + 1, ls * sa + lsv);
  GA2(va, i, j, ls * sb + lsv);
  GA2(d, i, j + 1, ls * v1);
  GA2(d, i, j, ls * (v1 + v0) - lf * 2.0f * am * diff);
  GA2(d, i, j - 1, ls * v0);
  GA2(aam2d, i, j, -lf * d0 * 2.0f * diff);
  const float ldiff = -lf * d0 * 2.0f * am / dyv;
  GA2(vab, i, j + 1, ldiff);
  GA2(vab, i, j, -ldiff);
}

// ADVAVE outputs of one cell: advua/advva (all cells) and, for i, j >= 1,
// fluxua/fluxva/tps; the caller passes through the unwritten flux elements
NPOM_HD void advave_cell_adj(const Ctx &c, const Adj &a, int i, int j, float lua, float lva, float lfu, float lfv,
                             float ltps) {
  if (interior(c, i, j)) {
    advave_fluxua1_adj(c, a, i, j, lua);
    advave_fluxua1_adj(c, a, i - 1, j, -lua);
    advave_fluxva1_adj(c, a, i, j + 1, lua);
    advave_fluxva1_adj(c, a, i, j, -lua);
    advave_fluxua2_adj(c, a, i + 1, j, lva);
    advave_fluxua2_adj(c, a, i, j, -lva);
    advave_fluxva2_adj(c, a, i, j, lva);
    advave_fluxva2_adj(c, a, i, j - 1, -lva);
  }
  if (i >= 1 && j >= 1) {
    advave_fluxua2_adj(c, a, i, j, lfu);
    advave_fluxva2_adj(c, a, i, j, lfv);
    advave_tps_adj(c, a, i, j, ltps);
  }
}

// The implicit barotropic predictor at an interior cell (core.py:795-845):
// us/den_u (comp 0) or vs/den_v (comp 1).  The provisional forcing is
// evaluated from the old adx2d, whose ADVAVE round trip (adx2d - advua +
// advua) changes it by rounding only.
NPOM_HD void a3_predictor_adj(const Ctx &c, const Adj &a, int i, int j, int comp) {
  const float lus = LAW(comp == 0 ? AW_us : AW_vs, i, j), lden_in = LAW(comp == 0 ? AW_den_u : AW_den_v, i, j);
  if (lus == 0.0f && lden_in == 0.0f) return;
  const float g4 = c.k.quarter_g, al = c.k.alpha, a12 = c.k.one_m_2alpha;
  const int oi = comp == 0 ? i - 1 : i, oj = comp == 0 ? j : j - 1;
  const float ar = comp == 0 ? F2(aru, i, j) : F2(arv, i, j);
  const float msk = comp == 0 ? F2(dum, i, j) : F2(dvm, i, j);
  const float d0 = F2(d, i, j), dw = F2(d, oi, oj);
  float s0, s1;
  if (comp == 0) {
    s0 = F2(va, i, j + 1) + F2(va, i, j);
    s1 = F2(va, i - 1, j + 1) + F2(va, i - 1, j);
  } else {
    s0 = F2(ua, i + 1, j) + F2(ua, i, j);
    s1 = F2(ua, i + 1, j - 1) + F2(ua, i, j - 1);
  }
  const float cor = 0.25f * (F2(cor, i, j) * d0 * s0 + F2(cor, oi, oj) * dw * s1);
  const float G = g4 * (comp == 0 ? (F2(dy, i, j) + F2(dy, i - 1, j)) : (F2(dx, i, j) + F2(dx, i, j - 1)));
  const float E = a12 * (F2(el, i, j) - F2(el, oi, oj)) + al * (F2(elb, i, j) - F2(elb, oi, oj)) + F2(e_atmos, i, j) -
                  F2(e_atmos, oi, oj);
  const float gu = G * (d0 + dw) * E;
  float up;
  if (comp == 0)
    up = F2(adx2d, i, j) - ar * cor + gu + F2(drx2d, i, j) - ar * (-F2(wusurf, i, j) + F2(wubot, i, j));
  else
    up = F2(ady2d, i, j) + ar * cor + gu + F2(dry2d, i, j) - ar * (-F2(wvsurf, i, j) + F2(wvbot, i, j));
  const float den = (F2(h, i, j) + F2(el, i, j) + F2(h, oi, oj) + F2(el, oi, oj)) * ar;
  const float hb = F2(h, i, j) + F2(elb, i, j) + F2(h, oi, oj) + F2(elb, oi, oj);
  const float ub = comp == 0 ? F2(uab, i, j) : F2(vab, i, j);
  const float num = hb * ar * ub - c.k.four_dti * up;
  const float dd = den + 1e-20f;
  const float q = num / dd;
  const float lq = lus * msk * msk;
  const float lnum = lq / dd;
  const float lden = lden_in - lq * q / dd;
  GA2(el, i, j, lden * ar);
  GA2(el, oi, oj, lden * ar);
  const float tb = lnum * ar * ub;
  GA2(elb, i, j, tb);
  GA2(elb, oi, oj, tb);
  if (comp == 0) GA2(uab, i, j, lnum * hb * ar);
  else GA2(vab, i, j, lnum * hb * ar);
  const float lup = -lnum * c.k.four_dti;
  if (comp == 0) {
    GA2(adx2d, i, j, lup);
    GA2(drx2d, i, j, lup);
    GA2(wubot, i, j, -lup * ar);
  } else {
    GA2(ady2d, i, j, lup);
    GA2(dry2d, i, j, lup);
    GA2(wvbot, i, j, -lup * ar);
  }
  const float lc = (comp == 0 ? -lup : lup) * ar * 0.25f;
  GA2(d, i, j, lc * F2(cor, i, j) * s0);
  GA2(d, oi, oj, lc * F2(cor, oi, oj) * s1);
  const float q0 = lc * F2(cor, i, j) * d0, q1 = lc * F2(cor, oi, oj) * dw;
  if (comp == 0) {
    GA2(va, i, j + 1, q0);
    GA2(va, i, j, q0);
    GA2(va, i - 1, j + 1, q1);
    GA2(va, i - 1, j, q1);
  } else {
    GA2(ua, i + 1, j, q0);
    GA2(ua, i, j, q0);
    GA2(ua, i + 1, j - 1, q1);
    GA2(ua, i, j - 1, q1);
  }
  const float ld = lup * G * E;
  GA2(d, i, j, ld);
  GA2(d, oi, oj, ld);
  const float lE = lup * G * (d0 + dw);
  GA2(el, i, j, lE * a12);
  GA2(el, oi, oj, -lE * a12);
  GA2(elb, i, j, lE * al);
  GA2(elb, oi, oj, -lE * al);
}

// A3 (explicit core): rho round trip (derivative one, rho is not moved),
// ADVAVE, adx2d/ady2d -= advua/advva, egf, provisional utf/vtf
NPOM_HD void phase_a3_cell_adj(const Ctx &c, const Adj &a, int i, int j) {
  const float lax = LA2(adx2d, i, j), lay = LA2(ady2d, i, j);
  GA2(adx2d, i, j, lax);
  GA2(ady2d, i, j, lay);
  const float lua = LA2(advua, i, j) - lax, lva = LA2(advva, i, j) - lay;
  GA2(el, i, j, LA2(egf, i, j) * c.k.ispi);
  if (i >= 1) {
    const float l = LA2(utf, i, j) * c.k.isp2i;
    GA2(ua, i, j, l * (F2(d, i, j) + F2(d, i - 1, j)));
    const float t = l * F2(ua, i, j);
    GA2(d, i, j, t);
    GA2(d, i - 1, j, t);
  } else {
    PASS2(utf, i, j);
  }
  if (j >= 1) {
    const float l = LA2(vtf, i, j) * c.k.isp2i;
    GA2(va, i, j, l * (F2(d, i, j) + F2(d, i, j - 1)));
    const float t = l * F2(va, i, j);
    GA2(d, i, j, t);
    GA2(d, i, j - 1, t);
  } else {
    PASS2(vtf, i, j);
  }
  const bool wf = (i >= 1 && j >= 1);
  advave_cell_adj(c, a, i, j, lua, lva, wf ? LA2(fluxua, i, j) : 0.0f, wf ? LA2(fluxva, i, j) : 0.0f,
                  wf ? LA2(tps, i, j) : 0.0f);
  if (!wf) {
    PASS2(fluxua, i, j);
    PASS2(fluxva, i, j);
    PASS2(tps, i, j);
  }
  if (is_explicit(c)) return;
  GA2(elb, i, j, LAW(AW_d_baro, i, j));
  if (!interior(c, i, j)) return;  // us, vs, den_u, den_v are zero off the interior
  a3_predictor_adj(c, a, i, j, 0);
  a3_predictor_adj(c, a, i, j, 1);
}

// ===========================================================================
// E: one external substep (time_loop.py:292-431, baroclinic.py:496-571)
// ===========================================================================
NPOM_HD void ext_transport_u_adj(const Ctx &c, const Adj &a, int ii, int jj, float lam) {
  const float q = 0.25f * (F2(dy, ii, jj) + F2(dy, ii - 1, jj));
  GA2(ua, ii, jj, lam * q * (F2(d, ii, jj) + F2(d, ii - 1, jj)));
  const float t = lam * q * F2(ua, ii, jj);
  GA2(d, ii, jj, t);
  GA2(d, ii - 1, jj, t);
}
NPOM_HD void ext_transport_v_adj(const Ctx &c, const Adj &a, int ii, int jj, float lam) {
  const float q = 0.25f * (F2(dx, ii, jj) + F2(dx, ii, jj - 1));
  GA2(va, ii, jj, lam * q * (F2(d, ii, jj) + F2(d, ii, jj - 1)));
  const float t = lam * q * F2(va, ii, jj);
  GA2(d, ii, jj, t);
  GA2(d, ii, jj - 1, t);
}

NPOM_HD void ext_elf_interior_adj(const Ctx &c, const Adj &a, int i, int j, float lam) {
  if (lam == 0.0f) return;
  GA2(elb, i, j, lam);
  const float ldiv = -lam * c.k.dte2 / F2(art, i, j);
  ext_transport_u_adj(c, a, i + 1, j, ldiv);
  ext_transport_u_adj(c, a, i, j, -ldiv);
  ext_transport_v_adj(c, a, i, j + 1, ldiv);
  ext_transport_v_adj(c, a, i, j, -ldiv);
}

// phase 1: elf with bcond 1, transports or ADVAVE into fluxua/fluxva
NPOM_HD void ext_phase1_cell_adj(const Ctx &c, const Adj &a, int i, int j, bool do_advave) {
  int si = i, sj = j;
  if (si == 0) si = 1;
  if (si == c.im - 1) si = c.im - 2;
  if (sj == 0) sj = 1;
  if (sj == c.jm - 1) sj = c.jm - 2;
  ext_elf_interior_adj(c, a, si, sj, LA2(elf, i, j) * F2(fsm, i, j));
  const bool wf = (i >= 1 && j >= 1);
  if (do_advave) {
    advave_cell_adj(c, a, i, j, LA2(advua, i, j), LA2(advva, i, j), wf ? LA2(fluxua, i, j) : 0.0f,
                    wf ? LA2(fluxva, i, j) : 0.0f, wf ? LA2(tps, i, j) : 0.0f);
    if (!wf) PASS2(tps, i, j);
  } else if (wf) {
    ext_transport_u_adj(c, a, i, j, LA2(fluxua, i, j));
    ext_transport_v_adj(c, a, i, j, LA2(fluxva, i, j));
  }
  if (!wf) {
    PASS2(fluxua, i, j);
    PASS2(fluxva, i, j);
  }
}

// uaf from the interior momentum balance (time_loop.py:326-358)
NPOM_HD void ext_uaf_interior_adj(const Ctx &c, const Adj &a, int i, int j, float lu) {
  const float g4 = c.k.quarter_g, al = c.k.alpha, a12 = c.k.one_m_2alpha;
  const float d0 = F2(d, i, j), dw = F2(d, i - 1, j);
  const float vs0 = F2(va, i, j + 1) + F2(va, i, j), vs1 = F2(va, i - 1, j + 1) + F2(va, i - 1, j);
  const float cor_u = 0.25f * (F2(cor, i, j) * d0 * vs0 + F2(cor, i - 1, j) * dw * vs1);
  const float G = g4 * (F2(dy, i, j) + F2(dy, i - 1, j));
  const float E = a12 * (F2(el, i, j) - F2(el, i - 1, j)) +
                  al * (F2(elb, i, j) - F2(elb, i - 1, j) + F2(elf, i, j) - F2(elf, i - 1, j)) + F2(e_atmos, i, j) -
                  F2(e_atmos, i - 1, j);
  const float gu = G * (d0 + dw) * E;
  const float aru = F2(aru, i, j);
  const float up = F2(adx2d, i, j) + F2(advua, i, j) - aru * cor_u + gu + F2(drx2d, i, j) -
                   aru * (-F2(wusurf, i, j) + F2(wubot, i, j));
  const float hb = F2(h, i, j) + F2(elb, i, j) + F2(h, i - 1, j) + F2(elb, i - 1, j);
  const float den = (F2(h, i, j) + F2(elf, i, j) + F2(h, i - 1, j) + F2(elf, i - 1, j)) * aru + 1e-20f;
  const float num = hb * aru * F2(uab, i, j) - c.k.four_dte * up;
  const float lnum = lu / den, lden = -lu * (num / den) / den;
  GA2(elf, i, j, lden * aru);
  GA2(elf, i - 1, j, lden * aru);
  const float tb = lnum * aru * F2(uab, i, j);
  GA2(elb, i, j, tb);
  GA2(elb, i - 1, j, tb);
  GA2(uab, i, j, lnum * hb * aru);
  const float lup = -lnum * c.k.four_dte;
  GA2(adx2d, i, j, lup);
  GA2(advua, i, j, lup);
  GA2(drx2d, i, j, lup);
  GA2(wubot, i, j, -lup * aru);
  const float lc = -lup * aru * 0.25f;
  GA2(d, i, j, lc * F2(cor, i, j) * vs0);
  GA2(va, i, j + 1, lc * F2(cor, i, j) * d0);
  GA2(va, i, j, lc * F2(cor, i, j) * d0);
  GA2(d, i - 1, j, lc * F2(cor, i - 1, j) * vs1);
  GA2(va, i - 1, j + 1, lc * F2(cor, i - 1, j) * dw);
  GA2(va, i - 1, j, lc * F2(cor, i - 1, j) * dw);
  const float ld = lup * G * E;
  GA2(d, i, j, ld);
  GA2(d, i - 1, j, ld);
  const float lE = lup * G * (d0 + dw);
  GA2(el, i, j, lE * a12);
  GA2(el, i - 1, j, -lE * a12);
  GA2(elb, i, j, lE * al);
  GA2(elb, i - 1, j, -lE * al);
  GA2(elf, i, j, lE * al);
  GA2(elf, i - 1, j, -lE * al);
}

NPOM_HD void ext_vaf_interior_adj(const Ctx &c, const Adj &a, int i, int j, float lv) {
  const float g4 = c.k.quarter_g, al = c.k.alpha, a12 = c.k.one_m_2alpha;
  const float d0 = F2(d, i, j), ds = F2(d, i, j - 1);
  const float us0 = F2(ua, i + 1, j) + F2(ua, i, j), us1 = F2(ua, i + 1, j - 1) + F2(ua, i, j - 1);
  const float cor_v = 0.25f * (F2(cor, i, j) * d0 * us0 + F2(cor, i, j - 1) * ds * us1);
  const float G = g4 * (F2(dx, i, j) + F2(dx, i, j - 1));
  const float E = a12 * (F2(el, i, j) - F2(el, i, j - 1)) +
                  al * (F2(elb, i, j) - F2(elb, i, j - 1) + F2(elf, i, j) - F2(elf, i, j - 1)) + F2(e_atmos, i, j) -
                  F2(e_atmos, i, j - 1);
  const float gv = G * (d0 + ds) * E;
  const float arv = F2(arv, i, j);
  const float vp = F2(ady2d, i, j) + F2(advva, i, j) + arv * cor_v + gv + F2(dry2d, i, j) -
                   arv * (-F2(wvsurf, i, j) + F2(wvbot, i, j));
  const float hb = F2(h, i, j) + F2(elb, i, j) + F2(h, i, j - 1) + F2(elb, i, j - 1);
  const float den = (F2(h, i, j) + F2(elf, i, j) + F2(h, i, j - 1) + F2(elf, i, j - 1)) * arv + 1e-20f;
  const float num = hb * arv * F2(vab, i, j) - c.k.four_dte * vp;
  const float lnum = lv / den, lden = -lv * (num / den) / den;
  GA2(elf, i, j, lden * arv);
  GA2(elf, i, j - 1, lden * arv);
  const float tb = lnum * arv * F2(vab, i, j);
  GA2(elb, i, j, tb);
  GA2(elb, i, j - 1, tb);
  GA2(vab, i, j, lnum * hb * arv);
  const float lvp = -lnum * c.k.four_dte;
  GA2(ady2d, i, j, lvp);
  GA2(advva, i, j, lvp);
  GA2(dry2d, i, j, lvp);
  GA2(wvbot, i, j, -lvp * arv);
  const float lc = lvp * arv * 0.25f;
  GA2(d, i, j, lc * F2(cor, i, j) * us0);
  GA2(ua, i + 1, j, lc * F2(cor, i, j) * d0);
  GA2(ua, i, j, lc * F2(cor, i, j) * d0);
  GA2(d, i, j - 1, lc * F2(cor, i, j - 1) * us1);
  GA2(ua, i + 1, j - 1, lc * F2(cor, i, j - 1) * ds);
  GA2(ua, i, j - 1, lc * F2(cor, i, j - 1) * ds);
  const float ld = lvp * G * E;
  GA2(d, i, j, ld);
  GA2(d, i, j - 1, ld);
  const float lE = lvp * G * (d0 + ds);
  GA2(el, i, j, lE * a12);
  GA2(el, i, j - 1, -lE * a12);
  GA2(elb, i, j, lE * al);
  GA2(elb, i, j - 1, -lE * al);
  GA2(elf, i, j, lE * al);
  GA2(elf, i, j - 1, -lE * al);
}

// phase 2: uaf/vaf with bcond 2 (the last assignment of the forward wins)
// and the etf filter of the last three substeps
NPOM_HD void ext_phase2_cell_adj(const Ctx &c, const Adj &a, int i, int j, int iext) {
  const int im = c.im, jm = c.jm, isplit = c.k.isplit;
  if (iext >= isplit - 2) {
    const float le = LA2(etf, i, j);
    if (iext == isplit - 2) {
      GA2(elf, i, j, c.k.quarter_smoth * le);
    } else if (iext == isplit - 1) {
      GA2(etf, i, j, le);
      GA2(elf, i, j, c.k.etf_mid * le);
    } else {
      const float f = F2(fsm, i, j);
      GA2(etf, i, j, le * f);
      GA2(elf, i, j, 0.5f * f * le);
    }
  }
  const float lu = LA2(uaf, i, j) * F2(dum, i, j), lv = LA2(vaf, i, j) * F2(dvm, i, j);
  enum { BASE = 0, OPEN = 1, ZERO = 2 };
  int su = BASE, sv = BASE, side_u = -1, side_v = -1;
  if (j >= 1 && j <= jm - 2) {
    if (i == im - 1) { su = OPEN; side_u = 0; sv = ZERO; }
    if (i == 1 || i == 0) { su = OPEN; side_u = 1; }
    if (i == 0) sv = ZERO;
  }
  if (i >= 1 && i <= im - 2) {
    if (j == jm - 1) { sv = OPEN; side_v = 2; su = ZERO; }
    if (j == 1 || j == 0) { sv = OPEN; side_v = 3; }
    if (j == 0) su = ZERO;
  }
  const float ramp = c.ramp, g = c.k.grav;
  auto rad = [&](float hh) { return sqrtf(fmaxf_t(g / fmaxf_t(hh, 1e-8f), 1e-8f)); };
  if (su == OPEN) {
    if (side_u == 0) GA2(el, im - 2, j, lu * ramp * c.k.rfe * rad(F2(h, im - 2, j)));
    else GA2(el, 1, j, -lu * ramp * c.k.rfw * rad(F2(h, 1, j)));
  } else if (su == BASE) {
    if (interior(c, i, j)) {
      if (lu != 0.0f) ext_uaf_interior_adj(c, a, i, j, lu);
    } else {
      GA2(uaf, i, j, lu);
    }
  }
  if (sv == OPEN) {
    if (side_v == 2) GA2(el, i, jm - 2, lv * ramp * c.k.rfn * rad(F2(h, i, jm - 2)));
    else GA2(el, i, 1, -lv * ramp * c.k.rfs * rad(F2(h, i, 1)));
  } else if (sv == BASE) {
    if (interior(c, i, j)) {
      if (lv != 0.0f) ext_vaf_interior_adj(c, a, i, j, lv);
    } else {
      GA2(vaf, i, j, lv);
    }
  }
}

// phase 3: Robert-Asselin filter, shifts, egf/utf/vtf accumulation
NPOM_HD void ext_phase3_cell_adj(const Ctx &c, const Adj &a, int i, int j, int iext) {
  const float hs = c.k.half_smoth, ohs = 1.0f - 2.0f * hs;
  const float lelb = LA2(elb, i, j), luab = LA2(uab, i, j), lvab = LA2(vab, i, j);
  GA2(el, i, j, lelb * ohs);
  GA2(elb, i, j, lelb * hs);
  GA2(ua, i, j, luab * ohs);
  GA2(uab, i, j, luab * hs);
  GA2(va, i, j, lvab * ohs);
  GA2(vab, i, j, lvab * hs);
  float lelf = lelb * hs + LA2(el, i, j) + LA2(d, i, j);
  float luaf = luab * hs + LA2(ua, i, j);
  float lvaf = lvab * hs + LA2(va, i, j);
  if (iext != c.k.isplit) {
    const float lg = LA2(egf, i, j);
    GA2(egf, i, j, lg);
    lelf += lg * c.k.ispi;
    const float elf0 = F2(elf, i, j), dn = F2(h, i, j) + elf0;
    if (i >= 1) {
      const float lt = LA2(utf, i, j);
      GA2(utf, i, j, lt);
      const float ds = dn + (F2(h, i - 1, j) + F2(elf, i - 1, j));
      luaf += lt * ds * c.k.isp2i;
      const float t = lt * F2(uaf, i, j) * c.k.isp2i;
      lelf += t;
      GA2(elf, i - 1, j, t);
    } else {
      PASS2(utf, i, j);
    }
    if (j >= 1) {
      const float lt = LA2(vtf, i, j);
      GA2(vtf, i, j, lt);
      const float ds = dn + (F2(h, i, j - 1) + F2(elf, i, j - 1));
      lvaf += lt * ds * c.k.isp2i;
      const float t = lt * F2(vaf, i, j) * c.k.isp2i;
      lelf += t;
      GA2(elf, i, j - 1, t);
    } else {
      PASS2(vtf, i, j);
    }
  }
  GA2(elf, i, j, lelf);
  GA2(uaf, i, j, luaf);
  GA2(vaf, i, j, lvaf);
}

// ===========================================================================
// Implicit free surface (core.py:858-943, time_loop.py:269-387)
// ===========================================================================

// Shapiro filter (gamma 0) and masks of the solution: d(elf)/dx = fsm^2 on
// the interior; d = h + elf there; ring values are constants
NPOM_HD float imp_post_grad(const Ctx &c, const Adj &a, int i, int j) {
  if (!interior(c, i, j)) return 0.0f;
  const float f = F2(fsm, i, j);
  return (LA2(elf, i, j) + LA2(d, i, j)) * f * f;
}

// one face transport fed by the predictor (rhs_fluxua / rhs_fluxva)
NPOM_HD void imp_flux_adj(const Ctx &c, const Adj &a, int comp, int i, int j, float lam) {
  if (lam == 0.0f || i < 1 || j < 1) return;
  const int oi = comp == 0 ? i - 1 : i, oj = comp == 0 ? j : j - 1;
  const float q = 0.25f * (comp == 0 ? (F2(dy, i, j) + F2(dy, i - 1, j)) : (F2(dx, i, j) + F2(dx, i, j - 1)));
  const float sv = comp == 0 ? ld(c.W[NPOM_W_us] + NPOM_I2(c, i, j)) : ld(c.W[NPOM_W_vs] + NPOM_I2(c, i, j));
  GAW(comp == 0 ? AW_us : AW_vs, i, j, lam * q * (F2(d, i, j) + F2(d, oi, oj)));
  const float t = lam * q * sv;
  GA2(d, i, j, t);
  GA2(d, oi, oj, t);
}

// rhs and stored transports of one cell, given lambda = A^-T g (lam) and
// the depth gradient of the solve (gd)
NPOM_HD void imp_rhs_cell_adj(const Ctx &c, const Adj &a, int i, int j, const float *lam, const float *gd) {
  const size_t o = NPOM_I2(c, i, j);
  GA2(d, i, j, ld(gd + o));
  imp_flux_adj(c, a, 0, i, j, LA2(fluxua, i, j));
  imp_flux_adj(c, a, 1, i, j, LA2(fluxva, i, j));
  if (!interior(c, i, j)) return;
  const float l = ld(lam + o);
  GA2(elb, i, j, l);
  const float ldiv = -c.k.two_dti * l / (F2(art, i, j) + 1e-20f);
  imp_flux_adj(c, a, 0, i + 1, j, ldiv);
  imp_flux_adj(c, a, 0, i, j, -ldiv);
  imp_flux_adj(c, a, 1, i, j + 1, ldiv);
  imp_flux_adj(c, a, 1, i, j, -ldiv);
}

// The terms of the eta-solve adjoint (implicit_p0_fixed/core.py:231-252,
// 645-675): relative cell area, and the face terms of the depth adjoint.
NPOM_HD float adj_area(const Ctx &c, int i, int j) {
  return interior(c, i, j) ? F2(art, i, j) / F2(art, 1, 1) : 1.0f;
}
NPOM_HD float adj_lam(const Ctx &c, const float *sol, float scale, int i, int j) {
  const size_t o = NPOM_I2(c, i, j);
  const float lam = (ld(sol + o) * adj_area(c, i, j)) * scale;
  return (lam * c.k.implicit_coeff) * W2(inv_art, i, j);
}
NPOM_HD float adj_east(const Ctx &c, const float *x, const float *sol, float scale, int i, int j) {
  return (((0.5f * adj_lam(c, sol, scale, i, j)) * (ld(x + NPOM_I2(c, i + 1, j)) - ld(x + NPOM_I2(c, i, j)))) *
          W2(ce, i, j)) *
         F2(dum, i + 1, j);
}
NPOM_HD float adj_west(const Ctx &c, const float *x, const float *sol, float scale, int i, int j) {
  return (((0.5f * adj_lam(c, sol, scale, i, j)) * (ld(x + NPOM_I2(c, i, j)) - ld(x + NPOM_I2(c, i - 1, j)))) *
          W2(cw, i, j)) *
         F2(dum, i, j);
}
NPOM_HD float adj_north(const Ctx &c, const float *x, const float *sol, float scale, int i, int j) {
  return (((0.5f * adj_lam(c, sol, scale, i, j)) * (ld(x + NPOM_I2(c, i, j + 1)) - ld(x + NPOM_I2(c, i, j)))) *
          W2(cn, i, j)) *
         F2(dvm, i, j + 1);
}
NPOM_HD float adj_south(const Ctx &c, const float *x, const float *sol, float scale, int i, int j) {
  return (((0.5f * adj_lam(c, sol, scale, i, j)) * (ld(x + NPOM_I2(c, i, j)) - ld(x + NPOM_I2(c, i, j - 1)))) *
          W2(cs, i, j)) *
         F2(dvm, i, j);
}
// grad_d = -(depth adjoint): the reference scatters eight face terms with
// in-place adds in a fixed statement order; each cell gathers the same
// terms in that order (east of i-1, east, west, west of i+1, north of j-1,
// north, south, south of j+1)
NPOM_HD float adj_grad_d_cell(const Ctx &c, const float *x, const float *sol, float scale, int i, int j) {
  float acc = 0.0f;
  if (interior(c, i - 1, j)) acc = acc + -adj_east(c, x, sol, scale, i - 1, j);
  if (interior(c, i, j)) {
    acc = acc + -adj_east(c, x, sol, scale, i, j);
    acc = acc + adj_west(c, x, sol, scale, i, j);
  }
  if (interior(c, i + 1, j)) acc = acc + adj_west(c, x, sol, scale, i + 1, j);
  if (interior(c, i, j - 1)) acc = acc + -adj_north(c, x, sol, scale, i, j - 1);
  if (interior(c, i, j)) {
    acc = acc + -adj_north(c, x, sol, scale, i, j);
    acc = acc + adj_south(c, x, sol, scale, i, j);
  }
  if (interior(c, i, j + 1)) acc = acc + adj_south(c, x, sol, scale, i, j + 1);
  return -acc;
}

// I5: corrector with closed-basin bcond 2, etf, Robert-Asselin filter,
// shifts, egf and endpoint transports (core.py:918-943,
// time_loop.py:309-387)
NPOM_HD void phase_i5_cell_adj(const Ctx &c, const Adj &a, int i, int j) {
  const float hs = c.k.half_smoth, ohs = 1.0f - 2.0f * hs;
  const bool inner = interior(c, i, j);
  const float elf0 = F2(elf, i, j), dn = F2(h, i, j) + elf0;
  const float dum = F2(dum, i, j), dvm = F2(dvm, i, j);
  // forward values
  float uaf = 0.0f, vaf = 0.0f, Nu = 0.0f, Nv = 0.0f, dfu = 0.0f, dfv = 0.0f;
  float Gu = 0.0f, Gv = 0.0f, Su = 0.0f, Sv = 0.0f, Du = 0.0f, Dv = 0.0f;
  const float g4 = c.k.quarter_g, al = c.k.alpha;
  if (inner) {
    const float h0 = F2(h, i, j);
    Gu = g4 * (F2(dy, i, j) + F2(dy, i - 1, j));
    Gv = g4 * (F2(dx, i, j) + F2(dx, i, j - 1));
    Su = (h0 + elf0) + (F2(h, i - 1, j) + F2(elf, i - 1, j));
    Sv = (h0 + elf0) + (F2(h, i, j - 1) + F2(elf, i, j - 1));
    Du = elf0 - F2(elf, i - 1, j);
    Dv = elf0 - F2(elf, i, j - 1);
    const float gu = Gu * Su * al * Du, gv = Gv * Sv * al * Dv;
    dfu = (h0 + elf0 + F2(h, i - 1, j) + F2(elf, i - 1, j)) * F2(aru, i, j) + 1e-20f;
    dfv = (h0 + elf0 + F2(h, i, j - 1) + F2(elf, i, j - 1)) * F2(arv, i, j) + 1e-20f;
    Nu = W2(us, i, j) * W2(den_u, i, j) - c.k.four_dti * gu;
    Nv = W2(vs, i, j) * W2(den_v, i, j) - c.k.four_dti * gv;
    uaf = (Nu / dfu * dum) * dum;
    vaf = (Nv / dfv * dvm) * dvm;
  }
  const float ua = F2(ua, i, j), va = F2(va, i, j);
  const float uaf_f = ua + hs * (F2(uab, i, j) - 2.0f * ua + uaf);
  const float vaf_f = va + hs * (F2(vab, i, j) - 2.0f * va + vaf);
  // cotangents of the outputs
  float luaf = LA2(uaf, i, j) + LA2(ua, i, j), lvaf = LA2(vaf, i, j) + LA2(va, i, j);
  float luaf_f = LA2(uab, i, j), lvaf_f = LA2(vab, i, j);
  float lel_f = LA2(elb, i, j) + 0.5f * LA2(egf, i, j);
  float lelf = LA2(etf, i, j) * F2(fsm, i, j) + LA2(el, i, j) + LA2(d, i, j) + 0.5f * LA2(egf, i, j);
  if (i >= 1) {
    const float lt = 0.25f * LA2(utf, i, j);
    const float dsum_new = dn + (F2(h, i - 1, j) + F2(elf, i - 1, j));
    const float dsum_baro = W2(d_baro, i, j) + W2(d_baro, i - 1, j);
    luaf_f += lt * dsum_baro;
    luaf += lt * dsum_new;
    lelf += lt * uaf;
    GA2(elf, i - 1, j, lt * uaf);
    GAW(AW_d_baro, i, j, lt * uaf_f);
    GAW(AW_d_baro, i - 1, j, lt * uaf_f);
  } else {
    PASS2(utf, i, j);
  }
  if (j >= 1) {
    const float lt = 0.25f * LA2(vtf, i, j);
    const float dsum_new = dn + (F2(h, i, j - 1) + F2(elf, i, j - 1));
    const float dsum_baro = W2(d_baro, i, j) + W2(d_baro, i, j - 1);
    lvaf_f += lt * dsum_baro;
    lvaf += lt * dsum_new;
    lelf += lt * vaf;
    GA2(elf, i, j - 1, lt * vaf);
    GAW(AW_d_baro, i, j, lt * vaf_f);
    GAW(AW_d_baro, i, j - 1, lt * vaf_f);
  } else {
    PASS2(vtf, i, j);
  }
  // Robert-Asselin filters
  GA2(ua, i, j, luaf_f * ohs);
  GA2(uab, i, j, luaf_f * hs);
  luaf += luaf_f * hs;
  GA2(va, i, j, lvaf_f * ohs);
  GA2(vab, i, j, lvaf_f * hs);
  lvaf += lvaf_f * hs;
  GA2(el, i, j, lel_f * ohs);
  GA2(elb, i, j, lel_f * hs);
  lelf += lel_f * hs;
  // corrector (the ring is zero)
  if (inner) {
    for (int comp = 0; comp < 2; ++comp) {
      const float m = comp == 0 ? dum : dvm;
      const float lq = (comp == 0 ? luaf : lvaf) * m * m;
      if (lq == 0.0f) continue;
      const float df = comp == 0 ? dfu : dfv, N = comp == 0 ? Nu : Nv;
      const float lN = lq / df, ldf = -lq * (N / df) / df;
      if (comp == 0) {
        GAW(AW_us, i, j, lN * W2(den_u, i, j));
        GAW(AW_den_u, i, j, lN * W2(us, i, j));
      } else {
        GAW(AW_vs, i, j, lN * W2(den_v, i, j));
        GAW(AW_den_v, i, j, lN * W2(vs, i, j));
      }
      const int oi = comp == 0 ? i - 1 : i, oj = comp == 0 ? j : j - 1;
      const float ar = comp == 0 ? F2(aru, i, j) : F2(arv, i, j);
      const float Gc = comp == 0 ? Gu : Gv, S = comp == 0 ? Su : Sv, D = comp == 0 ? Du : Dv;
      const float lg = -lN * c.k.four_dti;
      const float lS = lg * Gc * al * D, lD = lg * Gc * S * al;
      lelf += lS + lD + ldf * ar;
      GA2(elf, oi, oj, lS - lD + ldf * ar);
    }
  }
  GA2(elf, i, j, lelf);
}

// ===========================================================================
// B1: barotropic fix (time_loop.py:440-477)
// ===========================================================================
template <int KM>
NPOM_HD void phase_b1_column_adj(const Ctx &c, const Adj &a, int i, int j) {
  const int kbm1 = (KM == 16 ? 16 : c.kb) - 1;
  for (int comp = 0; comp < 2; ++comp) {
    const int fld = comp == 0 ? NPOM_F_u : NPOM_F_v;
    const size_t o = NPOM_I3(c, i, j, 0);
    const float *Lf = a.L[fld] + o;
    float *Gf = a.G[fld] + o;
    aadd(Gf + kbm1, Lf[kbm1]);
    const bool solved = comp == 0 ? (i >= 1) : (j >= 1);
    if (!solved) {
      for (int k = 0; k < kbm1; ++k) aadd(Gf + k, Lf[k]);
      continue;
    }
    float ls = 0.0f;
    for (int k = 0; k < kbm1; ++k) ls += Lf[k];
    for (int k = 0; k < kbm1; ++k) aadd(Gf + k, Lf[k] - ls * F1(dz, k));
    const int oi = comp == 0 ? i - 1 : i, oj = comp == 0 ? j : j - 1;
    const float D = (F2(dt, i, j) + F2(dt, oi, oj)) + 1e-20f;
    const float num = comp == 0 ? (F2(utb, i, j) + F2(utf, i, j)) : (F2(vtb, i, j) + F2(vtf, i, j));
    if (comp == 0) {
      GA2(utb, i, j, ls / D);
      GA2(utf, i, j, ls / D);
    } else {
      GA2(vtb, i, j, ls / D);
      GA2(vtf, i, j, ls / D);
    }
    const float ldt = -ls * (num / D) / D;
    GA2(dt, i, j, ldt);
    GA2(dt, oi, oj, ldt);
  }
}

// ===========================================================================
// B2a: VERTVL (baroclinic.py:930-1040) and bcond 5
// ===========================================================================
NPOM_HD void vertvl_xflux_adj(const Ctx &c, const Adj &a, int i, int j, int k, float lam) {
  const float q = 0.25f * (F2(dy, i, j) + F2(dy, i - 1, j));
  GA3(u, i, j, k, lam * q * (F2(dt, i, j) + F2(dt, i - 1, j)));
  const float t = lam * q * F3(u, i, j, k);
  GA2(dt, i, j, t);
  GA2(dt, i - 1, j, t);
}
NPOM_HD void vertvl_yflux_adj(const Ctx &c, const Adj &a, int i, int j, int k, float lam) {
  const float q = 0.25f * (F2(dx, i, j) + F2(dx, i, j - 1));
  GA3(v, i, j, k, lam * q * (F2(dt, i, j) + F2(dt, i, j - 1)));
  const float t = lam * q * F3(v, i, j, k);
  GA2(dt, i, j, t);
  GA2(dt, i, j - 1, t);
}

template <int KM>
NPOM_HD void phase_b2a_column_adj(const Ctx &c, const Adj &a, int i, int j) {
  const int kb = KM == 16 ? 16 : c.kb, kbm1 = kb - 1;
  const float fsm = F2(fsm, i, j);
  // bcond 5: explicit masks levels < kb-1, the closed basin every level
  const int kend = is_explicit(c) ? kbm1 : kb;
  float lw[KM];
  for (int k = 0; k < kb; ++k) lw[k] = LA3(w, i, j, k) * (k < kend ? fsm : 1.0f);
  if (!interior(c, i, j)) {
    for (int k = 0; k < kb; ++k) GA3(w, i, j, k, lw[k]);
    return;
  }
  const float area = F2(dx, i, j) * F2(dy, i, j);
  float S = 0.0f, leta = 0.0f;
  for (int k = kbm1 - 1; k >= 0; --k) {
    S += lw[k + 1];
    const float dzk = F1(dz, k);
    const float ldiv = S * dzk / area;
    leta += S * dzk;
    vertvl_xflux_adj(c, a, i + 1, j, k, ldiv);
    vertvl_xflux_adj(c, a, i, j, k, -ldiv);
    vertvl_yflux_adj(c, a, i, j + 1, k, ldiv);
    vertvl_yflux_adj(c, a, i, j, k, -ldiv);
  }
  GA2(etf, i, j, leta / c.k.dti2);
  GA2(etb, i, j, -leta / c.k.dti2);
}

// ===========================================================================
// B2b: ADVQ (tracers.py:14-156) of q2 -> uf and q2l -> vf
// ===========================================================================
NPOM_HD void advq_xflux_adj(const Ctx &c, const Adj &a, int fq, int fqb, int i, int j, int k, float lam) {
  const float *q = c.F[fq], *qb = c.F[fqb];
  float *gq = a.G[fq], *gqb = a.G[fqb];
  const size_t o = NPOM_I3(c, i, j, k), om = NPOM_I3(c, i - 1, j, k);
  const float A = ld(q + o) + ld(q + om), B = F2(dt, i, j) + F2(dt, i - 1, j);
  const float Cu = F3(u, i, j, k) + F3(u, i, j, k - 1);
  const float aam_sum = F3(aam, i, j, k) + F3(aam, i - 1, j, k) + F3(aam, i, j, k - 1) + F3(aam, i - 1, j, k - 1);
  const float hsum = F2(h, i, j) + F2(h, i - 1, j), qd = ld(qb + o) - ld(qb + om);
  const float X = F2(dum, i, j) / (F2(dx, i, j) + F2(dx, i - 1, j));
  const float l = lam * 0.5f * (F2(dy, i, j) + F2(dy, i - 1, j));
  const float t = l * 0.125f;
  aadd(gq + o, t * B * Cu);
  aadd(gq + om, t * B * Cu);
  GA2(dt, i, j, t * A * Cu);
  GA2(dt, i - 1, j, t * A * Cu);
  GA3(u, i, j, k, t * A * B);
  GA3(u, i, j, k - 1, t * A * B);
  const float la = -l * 0.25f * hsum * qd * X;
  GA3(aam, i, j, k, la);
  GA3(aam, i - 1, j, k, la);
  GA3(aam, i, j, k - 1, la);
  GA3(aam, i - 1, j, k - 1, la);
  const float lq = -l * 0.25f * aam_sum * hsum * X;
  aadd(gqb + o, lq);
  aadd(gqb + om, -lq);
}
NPOM_HD void advq_yflux_adj(const Ctx &c, const Adj &a, int fq, int fqb, int i, int j, int k, float lam) {
  const float *q = c.F[fq], *qb = c.F[fqb];
  float *gq = a.G[fq], *gqb = a.G[fqb];
  const size_t o = NPOM_I3(c, i, j, k), om = NPOM_I3(c, i, j - 1, k);
  const float A = ld(q + o) + ld(q + om), B = F2(dt, i, j) + F2(dt, i, j - 1);
  const float Cv = F3(v, i, j, k) + F3(v, i, j, k - 1);
  const float aam_sum = F3(aam, i, j, k) + F3(aam, i, j - 1, k) + F3(aam, i, j, k - 1) + F3(aam, i, j - 1, k - 1);
  const float hsum = F2(h, i, j) + F2(h, i, j - 1), qd = ld(qb + o) - ld(qb + om);
  const float X = F2(dvm, i, j) / (F2(dy, i, j) + F2(dy, i, j - 1));
  const float l = lam * 0.5f * (F2(dx, i, j) + F2(dx, i, j - 1));
  const float t = l * 0.125f;
  aadd(gq + o, t * B * Cv);
  aadd(gq + om, t * B * Cv);
  GA2(dt, i, j, t * A * Cv);
  GA2(dt, i, j - 1, t * A * Cv);
  GA3(v, i, j, k, t * A * B);
  GA3(v, i, j, k - 1, t * A * B);
  const float la = -l * 0.25f * hsum * qd * X;
  GA3(aam, i, j, k, la);
  GA3(aam, i, j - 1, k, la);
  GA3(aam, i, j, k - 1, la);
  GA3(aam, i, j - 1, k - 1, la);
  const float lq = -l * 0.25f * aam_sum * hsum * X;
  aadd(gqb + o, lq);
  aadd(gqb + om, -lq);
}

NPOM_HD void advq_point_adj(const Ctx &c, const Adj &a, int fq, int fqb, int i, int j, int k, float lam) {
  const int kbm1 = c.kb - 1;
  if (lam == 0.0f || !interior(c, i, j) || k < 1 || k > kbm1 - 1) return;
  const float *q = c.F[fq], *qb = c.F[fqb];
  float *gq = a.G[fq], *gqb = a.G[fqb];
  const float art = F2(art, i, j);
  const float dzs = F1(dz, k) + F1(dz, k - 1);
  const size_t okm = NPOM_I3(c, i, j, k - 1), okp = NPOM_I3(c, i, j, k + 1), ok = NPOM_I3(c, i, j, k);
  const float wkm = F3(w, i, j, k - 1), wkp = F3(w, i, j, k + 1), qkm = ld(q + okm), qkp = ld(q + okp);
  const float vert = (wkm * qkm - wkp * qkp) * art / dzs;
  const float horiz = advq_xflux(c, q, qb, i + 1, j, k) - advq_xflux(c, q, qb, i, j, k) +
                      advq_yflux(c, q, qb, i, j + 1, k) - advq_yflux(c, q, qb, i, j, k);
  const float qf = vert + horiz;
  const float tb = (F2(h, i, j) + F2(etb, i, j)) * art;
  const float tf = (F2(h, i, j) + F2(etf, i, j)) * art + 1e-20f;
  const float qbk = ld(qb + ok);
  const float out = (tb * qbk - c.k.dti2 * qf) / tf;
  const float lnum = lam / tf;
  GA2(etf, i, j, -lam * out / tf * art);
  GA2(etb, i, j, lnum * qbk * art);
  aadd(gqb + ok, lnum * tb);
  const float lqf = -lnum * c.k.dti2;
  const float lv = lqf * art / dzs;
  GA3(w, i, j, k - 1, lv * qkm);
  aadd(gq + okm, lv * wkm);
  GA3(w, i, j, k + 1, -lv * qkp);
  aadd(gq + okp, -lv * wkp);
  advq_xflux_adj(c, a, fq, fqb, i + 1, j, k, lqf);
  advq_xflux_adj(c, a, fq, fqb, i, j, k, -lqf);
  advq_yflux_adj(c, a, fq, fqb, i, j + 1, k, lqf);
  advq_yflux_adj(c, a, fq, fqb, i, j, k, -lqf);
}

NPOM_HD void phase_b2b_point_adj(const Ctx &c, const Adj &a, int i, int j, int k) {
  advq_point_adj(c, a, NPOM_F_q2, NPOM_F_q2b, i, j, k, LA3(uf, i, j, k));
  advq_point_adj(c, a, NPOM_F_q2l, NPOM_F_q2lb, i, j, k, LA3(vf, i, j, k));
}

// ===========================================================================
// B3: PROFQ, Mellor-Yamada 2.5 (tracers.py:158-431), explicit forms
// ===========================================================================
template <int KM>
NPOM_HD void phase_b3_column_adj(const Ctx &c, const Adj &a, int i, int j) {
  // KM == 16 is instantiated for kb == 16 only: a compile-time level count
  // lets the compiler unroll the level loops and keep the column in registers
  const int im = c.im, jm = c.jm, kb = KM == 16 ? 16 : c.kb, kbm1 = kb - 1;
  const float dti2 = c.k.dti2, umol2 = c.k.two_umol, grav = c.k.grav, kappa = c.k.kappa, small = c.k.small;
  const float b1 = 16.6f, e1 = 1.8f, e2 = 1.33f;
  const float eps = 1e-20f;
  // ---- forward recomputation (phase_b3_column) ----
  float A[KM], C[KM], cc[KM], ccs_[KM], radv[KM], pp[KM], boygr[KM], lraw[KM], l[KM];
  float ghraw[KM], gh[KM], kn[KM], dtef[KM], ee1[KM], gg1[KM], den1[KM], ee2[KM], gg2[KM];
  float den2[KM], wall0[KM], wallv[KM], uo[KM], vo[KM];
  bool clampc[KM], clip[KM];
  const float dh = F2(h, i, j) + F2(etf, i, j);
  for (int k = 0; k < kb; ++k) {
    A[k] = 0.0f;
    C[k] = 0.0f;
  }
  for (int k = 1; k < kbm1; ++k) {
    const float den_a = F1(dzz, k - 1) * F1(dz, k) * dh * dh;
    const float den_c = F1(dzz, k - 1) * F1(dz, k - 1) * dh * dh;
    A[k] = c.k.neg_dti2 * (F3(kq, i, j, k + 1) + F3(kq, i, j, k) + umol2) * 0.5f / den_a;
    C[k] = c.k.neg_dti2 * (F3(kq, i, j, k - 1) + F3(kq, i, j, k) + umol2) * 0.5f / den_c;
  }
  float utau2 = 0.0f, l0 = 0.0f, magb = 0.0f, ubm = 0.0f, vbm = 0.0f;
  const bool sb_region = (i < im - 1) && (j < jm - 1);
  if (sb_region) {
    const float us_ = 0.5f * (F2(wusurf, i, j) + F2(wusurf, i + 1, j));
    const float vs_ = 0.5f * (F2(wvsurf, i, j) + F2(wvsurf, i, j + 1));
    utau2 = sqrtf(us_ * us_ + vs_ * vs_ + 1e-8f);
    l0 = c.k.surfl * utau2 / grav;
    ubm = 0.5f * (F2(wubot, i, j) + F2(wubot, i + 1, j));
    vbm = 0.5f * (F2(wvbot, i, j) + F2(wvbot, i, j + 1));
    magb = sqrtf(ubm * ubm + vbm * vbm + 1e-8f);
  }
  const float uf_bottom = magb * c.k.prof_const1;
  for (int k = 0; k < kbm1; ++k) {
    const float tp = F3(t, i, j, k) + c.k.tbias;
    const float sp = F3(s, i, j, k) + c.k.sbias;
    const float p = c.k.g_rhoref * (-F1(zz, k) * dh) * 1.0e-4f;
    float ccs = 1449.1f + 0.00821f * p + 4.55f * tp - 0.045f * (tp * tp) + 1.34f * (sp - 35.0f);
    clampc[k] = fabsf(ccs) < 1e-6f;
    if (clampc[k]) ccs = 1e-6f;
    const float rad = (1.0f - 0.01642f * p / ccs) * (1.0f - 0.40f * p / (ccs * ccs));
    ccs_[k] = ccs;
    radv[k] = rad;
    pp[k] = p;
    cc[k] = ccs / sqrtf(fmaxf_t(rad, 1e-8f));
  }
  for (int k = 0; k < kb; ++k) boygr[k] = 0.0f;
  for (int k = 1; k < kbm1; ++k) {
    const float term1 = grav * (F3(rho, i, j, k - 1) - F3(rho, i, j, k)) / (F1(dzz, k - 1) * dh);
    const float term2 = c.k.g2x2 / (cc[k - 1] * cc[k - 1] + cc[k] * cc[k]);
    boygr[k] = term1 + term2;
  }
  for (int k = 0; k < kb; ++k) {
    l[k] = 0.0f;
    lraw[k] = 0.0f;
  }
  for (int k = 1; k < kbm1; ++k) lraw[k] = l[k] = fabsf(F3(q2lb, i, j, k)) / (fabsf(F3(q2b, i, j, k)) + 1e-20f);
  const float kl0 = kappa * l0;
  for (int k = 0; k < kbm1; ++k)
    if (F1(z, k) > -0.5f) l[k] = fmaxf_t(l[k], kl0);
  for (int k = 0; k < kb; ++k) {
    gh[k] = 0.0f;
    ghraw[k] = 0.0f;
  }
  for (int k = 1; k < kbm1; ++k) {
    ghraw[k] = (l[k] * l[k]) * boygr[k] / (fabsf(F3(q2b, i, j, k)) + 1e-20f);
    gh[k] = fminf_t(ghraw[k], 0.028f);
  }
  l[0] = kl0;
  l[kb - 1] = 0.0f;
  for (int k = 0; k < kb; ++k) kn[k] = 0.0f;
  const bool inner = interior(c, i, j);
  if (inner) {
    for (int k = 1; k < kbm1; ++k) {
      const float du = F3(u, i, j, k) - F3(u, i, j, k - 1) + F3(u, i + 1, j, k) - F3(u, i + 1, j, k - 1);
      const float dv = F3(v, i, j, k) - F3(v, i, j, k - 1) + F3(v, i, j + 1, k) - F3(v, i, j + 1, k - 1);
      float den = F1(dzz, k - 1) * dh;
      den = den * den;
      const float kmk = F3(km, i, j, k);
      float knk = kmk * 0.25f * 1.0f * (du * du + dv * dv) / den;
      knk = knk - 0.0f * kmk * boygr[k] + F3(kh, i, j, k) * boygr[k];
      kn[k] = knk;
    }
  }
  for (int k = 0; k < kb; ++k) dtef[k] = sqrtf(fabsf(F3(q2b, i, j, k)) + 1e-8f) * 1.0f / (b1 * l[k] + small);
  ee1[0] = 0.0f;
  gg1[0] = sb_region ? c.k.prof_gg0 * utau2 : 0.0f;
  for (int k = 1; k < kbm1; ++k) {
    den1[k] = A[k] + C[k] * (1.0f - ee1[k - 1]) - (c.k.two_dti2 * dtef[k] + 1.0f);
    ee1[k] = A[k] / (den1[k] + eps);
    gg1[k] = (c.k.neg_two_dti2 * kn[k] + C[k] * gg1[k - 1] - F3(uf, i, j, k)) / (den1[k] + eps);
  }
  uo[kb - 1] = uf_bottom;
  for (int k = kbm1 - 1; k >= 0; --k) uo[k] = ee1[k] * uo[k + 1] + gg1[k];
  const float z0 = F1(z, 0), zb = F1(z, kb - 1);
  ee2[0] = 0.0f;
  gg2[0] = 0.0f;
  for (int k = 1; k < kbm1; ++k) {
    const float zk = F1(z, k);
    const float weps = is_explicit(c) ? 1e-20f : 1e-8f;
    wall0[k] = 1.0f / (fabsf(zk - z0) + weps) + 1.0f / (fabsf(zk - zb) + weps);
    wallv[k] = wall0[k] * l[k] / (dh * kappa);
    const float dtefk = dtef[k] * (1.0f + e2 * (wallv[k] * wallv[k]));
    den2[k] = A[k] + C[k] * (1.0f - ee2[k - 1]) - (dti2 * dtefk + 1.0f);
    ee2[k] = A[k] / (den2[k] + eps);
    gg2[k] = (dti2 * (-kn[k] * l[k] * e1) + C[k] * gg2[k - 1] - F3(vf, i, j, k)) / (den2[k] + eps);
  }
  vo[kb - 1] = 0.0f;
  for (int k = kbm1 - 1; k >= 0; --k) vo[k] = ee2[k] * vo[k + 1] + gg2[k];
  for (int k = 0; k < kb; ++k) clip[k] = false;
  for (int k = 1; k < kbm1; ++k) clip[k] = (uo[k] <= small) || (vo[k] <= small);

  // ---- reverse sweep ----
  const float coef4 = (float)(18.0 * 0.92 * 0.92 + 9.0 * 0.92 * 0.74);
  const float coef5 = (float)(9.0 * 0.92 * 0.74);
  const float coef1 = (float)(0.74 * (1.0 - 6.0 * 0.92 / 16.6));
  const float coef2 = (float)(3.0 * 0.74 * 10.1 + 18.0 * 0.92 * 0.74);
  const float coef3 = (float)(0.92 * (1.0 - 3.0 * 0.08 - 6.0 * 0.92 / 16.6));
  float lA[KM], lC[KM], ldtef[KM], lkn[KM], lgh[KM], ll[KM], lcc[KM], lboy[KM];
  float luo[KM], lvo[KM], lee[KM], lgg[KM];
  for (int k = 0; k < kb; ++k) {
    lA[k] = lC[k] = ldtef[k] = lkn[k] = lgh[k] = ll[k] = lcc[k] = lboy[k] = 0.0f;
  }
  float ldh = 0.0f;
  for (int k = 0; k < kb; ++k) {
    const float lkq = LA3(kq, i, j, k), lkm = LA3(km, i, j, k), lkh = LA3(kh, i, j, k);
    GA3(kq, i, j, k, 0.5f * lkq);
    GA3(km, i, j, k, 0.5f * lkm);
    GA3(kh, i, j, k, 0.5f * lkh);
    const float ghk = gh[k];
    const float D2 = (1.0f - coef2 * ghk) + 1e-20f;
    const float sh = coef1 / D2;
    const float D5 = (1.0f - coef5 * ghk) + 1e-20f;
    const float N5 = coef3 + sh * coef4 * ghk;
    const float sm = N5 / D5;
    const float q2v = F3(q2, i, j, k);
    const float sq = sqrtf(fabsf(q2v) + 1e-8f);
    const float knf = l[k] * sq;
    const float lknf = 0.5f * (0.41f * sh * lkq + sm * lkm + sh * lkh);
    float lsh = 0.5f * knf * (0.41f * lkq + lkh);
    const float lsm = 0.5f * knf * lkm;
    lsh += lsm * coef4 * ghk / D5;
    lgh[k] += lsm * (sh * coef4 / D5 + N5 * coef5 / (D5 * D5));
    lgh[k] += lsh * coef1 * coef2 / (D2 * D2);
    ll[k] += lknf * sq + LA3(l, i, j, k);
    GA3(q2, i, j, k, lknf * l[k] * sgnf(q2v) * 0.5f / sq);
    luo[k] = LA3(uf, i, j, k);
    lvo[k] = LA3(vf, i, j, k);
  }
  for (int k = 1; k < kbm1; ++k) {
    if (clip[k]) {
      GA2(dt, i, j, lvo[k] * 0.1f * small);
      luo[k] = 0.0f;
      lvo[k] = 0.0f;
    }
  }
  // q2l: back substitution, then the forward recursion
  for (int k = 0; k < kb; ++k) lee[k] = lgg[k] = 0.0f;
  for (int k = 0; k < kbm1; ++k) {
    lee[k] += lvo[k] * vo[k + 1];
    lgg[k] += lvo[k];
    lvo[k + 1] += lvo[k] * ee2[k];
  }
  for (int k = kbm1 - 1; k >= 1; --k) {
    const float dd = den2[k] + eps;
    const float lden = -(lee[k] * ee2[k] + lgg[k] * gg2[k]) / dd;
    lA[k] += lee[k] / dd + lden;
    const float lN = lgg[k] / dd;
    lC[k] += lden * (1.0f - ee2[k - 1]) + lN * gg2[k - 1];
    lee[k - 1] -= lden * C[k];
    lgg[k - 1] += lN * C[k];
    const float ldtefk = -lden * dti2;
    lkn[k] += lN * dti2 * (-l[k] * e1);
    ll[k] += lN * dti2 * (-kn[k] * e1);
    GA3(vf, i, j, k, -lN);
    const float wv = wallv[k];
    ldtef[k] += ldtefk * (1.0f + e2 * (wv * wv));
    const float lwall = ldtefk * dtef[k] * e2 * 2.0f * wv;
    ll[k] += lwall * wall0[k] / (dh * kappa);
    ldh += -lwall * wv / dh;
  }
  // q2: back substitution, then the forward recursion
  for (int k = 0; k < kb; ++k) lee[k] = lgg[k] = 0.0f;
  for (int k = 0; k < kbm1; ++k) {
    lee[k] += luo[k] * uo[k + 1];
    lgg[k] += luo[k];
    luo[k + 1] += luo[k] * ee1[k];
  }
  if (sb_region && luo[kb - 1] != 0.0f) {
    const float lm = luo[kb - 1] * c.k.prof_const1 / magb;
    GA2(wubot, i, j, lm * ubm * 0.5f);
    GA2(wubot, i + 1, j, lm * ubm * 0.5f);
    GA2(wvbot, i, j, lm * vbm * 0.5f);
    GA2(wvbot, i, j + 1, lm * vbm * 0.5f);
  }
  for (int k = kbm1 - 1; k >= 1; --k) {
    const float dd = den1[k] + eps;
    const float lden = -(lee[k] * ee1[k] + lgg[k] * gg1[k]) / dd;
    lA[k] += lee[k] / dd + lden;
    const float lN = lgg[k] / dd;
    lC[k] += lden * (1.0f - ee1[k - 1]) + lN * gg1[k - 1];
    lee[k - 1] -= lden * C[k];
    lgg[k - 1] += lN * C[k];
    ldtef[k] += -lden * c.k.two_dti2;
    lkn[k] += lN * c.k.neg_two_dti2;
    GA3(uf, i, j, k, -lN);
  }
  // dtef (every level)
  for (int k = 0; k < kb; ++k) {
    if (ldtef[k] == 0.0f) continue;
    const float q = F3(q2b, i, j, k);
    const float sq = sqrtf(fabsf(q) + 1e-8f);
    const float den = b1 * l[k] + small;
    GA3(q2b, i, j, k, ldtef[k] / den * sgnf(q) * 0.5f / sq);
    ll[k] += -ldtef[k] * dtef[k] * b1 / den;
  }
  // shear / buoyancy production
  if (inner) {
    for (int k = 1; k < kbm1; ++k) {
      if (lkn[k] == 0.0f) continue;
      const float du = F3(u, i, j, k) - F3(u, i, j, k - 1) + F3(u, i + 1, j, k) - F3(u, i + 1, j, k - 1);
      const float dv = F3(v, i, j, k) - F3(v, i, j, k - 1) + F3(v, i, j + 1, k) - F3(v, i, j + 1, k - 1);
      const float X = F1(dzz, k - 1) * dh;
      const float den = X * X;
      const float kmk = F3(km, i, j, k);
      const float Sq = du * du + dv * dv;
      GA3(km, i, j, k, lkn[k] * 0.25f * Sq / den);
      const float lS = lkn[k] * kmk * 0.25f / den;
      const float ldu = 2.0f * du * lS, ldv = 2.0f * dv * lS;
      ldh += -lkn[k] * kmk * 0.25f * Sq / (den * den) * 2.0f * X * F1(dzz, k - 1);
      GA3(kh, i, j, k, lkn[k] * boygr[k]);
      lboy[k] += lkn[k] * F3(kh, i, j, k);
      GA3(u, i, j, k, ldu);
      GA3(u, i, j, k - 1, -ldu);
      GA3(u, i + 1, j, k, ldu);
      GA3(u, i + 1, j, k - 1, -ldu);
      GA3(v, i, j, k, ldv);
      GA3(v, i, j, k - 1, -ldv);
      GA3(v, i, j + 1, k, ldv);
      GA3(v, i, j + 1, k - 1, -ldv);
    }
  }
  // gh = min(l^2 boygr / |q2b|, 0.028) on 1..kbm1-1 (gh, l at 0 and kb-1
  // are constants)
  for (int k = 1; k < kbm1; ++k) {
    if (lgh[k] != 0.0f && ghraw[k] <= 0.028f) {
      const float q = F3(q2b, i, j, k);
      const float qa = fabsf(q) + 1e-20f;
      ll[k] += lgh[k] * 2.0f * l[k] * boygr[k] / qa;
      lboy[k] += lgh[k] * l[k] * l[k] / qa;
      GA3(q2b, i, j, k, -lgh[k] * ghraw[k] / qa * sgnf(q));
    }
  }
  for (int k = 1; k < kbm1; ++k) {
    const bool pass = !(F1(z, k) > -0.5f) || lraw[k] > kl0;
    if (!pass || ll[k] == 0.0f) continue;
    const float qb = F3(q2b, i, j, k), qlb = F3(q2lb, i, j, k);
    const float qa = fabsf(qb) + 1e-20f;
    GA3(q2lb, i, j, k, ll[k] * sgnf(qlb) / qa);
    GA3(q2b, i, j, k, -ll[k] * lraw[k] / qa * sgnf(qb));
  }
  // buoyancy frequency
  for (int k = 1; k < kbm1; ++k) {
    if (lboy[k] == 0.0f) continue;
    const float X = F1(dzz, k - 1) * dh;
    const float term1 = grav * (F3(rho, i, j, k - 1) - F3(rho, i, j, k)) / X;
    const float Q = cc[k - 1] * cc[k - 1] + cc[k] * cc[k];
    const float term2 = c.k.g2x2 / Q;
    GA3(rho, i, j, k - 1, lboy[k] * grav / X);
    GA3(rho, i, j, k, -lboy[k] * grav / X);
    ldh += -lboy[k] * term1 / dh;
    const float lQ = -lboy[k] * term2 / Q;
    lcc[k - 1] += lQ * 2.0f * cc[k - 1];
    lcc[k] += lQ * 2.0f * cc[k];
  }
  // sound speed
  for (int k = 0; k < kbm1; ++k) {
    if (lcc[k] == 0.0f) continue;
    const float radc = fmaxf_t(radv[k], 1e-8f);
    const float sr = sqrtf(radc);
    const float ccs = ccs_[k], p = pp[k];
    float lccs = lcc[k] / sr;
    const float lrad = radv[k] >= 1e-8f ? -lcc[k] * cc[k] / (2.0f * radc) : 0.0f;
    const float P1 = 1.0f - 0.01642f * p / ccs, P2 = 1.0f - 0.40f * p / (ccs * ccs);
    const float lP1 = lrad * P2, lP2 = lrad * P1;
    lccs += lP1 * 0.01642f * p / (ccs * ccs) + lP2 * 0.80f * p / (ccs * ccs * ccs);
    float lp = -lP1 * 0.01642f / ccs - lP2 * 0.40f / (ccs * ccs);
    if (!clampc[k]) {
      const float tp = F3(t, i, j, k) + c.k.tbias;
      lp += lccs * 0.00821f;
      GA3(t, i, j, k, lccs * (4.55f - 0.09f * tp));
      GA3(s, i, j, k, lccs * 1.34f);
    }
    ldh += lp * c.k.g_rhoref * (-F1(zz, k)) * 1.0e-4f;
  }
  // tridiagonal coefficients
  for (int k = 1; k < kbm1; ++k) {
    const float den_a = F1(dzz, k - 1) * F1(dz, k) * dh * dh;
    const float den_c = F1(dzz, k - 1) * F1(dz, k - 1) * dh * dh;
    const float fa = lA[k] * c.k.neg_dti2 * 0.5f / den_a, fc = lC[k] * c.k.neg_dti2 * 0.5f / den_c;
    GA3(kq, i, j, k + 1, fa);
    GA3(kq, i, j, k, fa + fc);
    GA3(kq, i, j, k - 1, fc);
    ldh += -(lA[k] * A[k] + lC[k] * C[k]) * 2.0f / dh;
  }
  GA2(etf, i, j, ldh);
}

// ===========================================================================
// B4: km/kh edge copies and explicit bcond 6 (baroclinic.py:856-919)
// ===========================================================================
NPOM_HD void phase_b4_point_adj(const Ctx &c, const Adj &a, int i, int j, int k) {
  const int im = c.im, jm = c.jm;
  const bool edge = (i == 0 || i == im - 1 || j == 0 || j == jm - 1);
  if (!edge) {
    PASS3(km, i, j, k);
    PASS3(kh, i, j, k);
    if (is_explicit(c)) {
      PASS3(uf, i, j, k);
      PASS3(vf, i, j, k);
    }
    return;
  }
  for (int comp = 0; comp < 2; ++comp) {
    const int fld = comp == 0 ? NPOM_F_km : NPOM_F_kh;
    const float lam = a.L[fld][NPOM_I3(c, i, j, k)];
    int si, sj;
    float f = F2(fsm, i, j);
    if (j == 0 || j == jm - 1) {
      sj = (j == 0) ? 1 : jm - 2;
      if (i == 0) { si = 1; f *= F2(fsm, 0, sj); }
      else if (i == im - 1) { si = im - 2; f *= F2(fsm, im - 1, sj); }
      else si = i;
    } else {
      si = (i == 0) ? 1 : im - 2;
      sj = j;
    }
    aadd(&a.G[fld][NPOM_I3(c, si, sj, k)], lam * f);
  }
  if (!is_explicit(c)) return;  // uf/vf are not moved for the closed basin
  // bcond 6: the last side in the order east, west, north, south wins
  const float lu = LA3(uf, i, j, k), lv = LA3(vf, i, j, k);
  const float dti = c.k.dti, small = c.k.small;
  int side = -1;
  if (i == im - 1) side = 0;
  if (i == 0) side = 1;
  if (j == jm - 1) side = 2;
  if (j == 0) side = 3;
  int ei, ej, ii, ij, vi, vj;  // edge point, inner point, velocity point
  float dsum;
  if (side == 0) { ei = im - 1; ej = j; ii = im - 2; ij = j; vi = im - 1; vj = j; dsum = F2(dx, im - 1, j) + F2(dx, im - 2, j); }
  else if (side == 1) { ei = 0; ej = j; ii = 1; ij = j; vi = 1; vj = j; dsum = F2(dx, 0, j) + F2(dx, 1, j); }
  else if (side == 2) { ei = i; ej = jm - 1; ii = i; ij = jm - 2; vi = i; vj = jm - 1; dsum = F2(dy, i, jm - 1) + F2(dy, i, jm - 2); }
  else { ei = i; ej = 0; ii = i; ij = 1; vi = i; vj = 1; dsum = F2(dy, i, 0) + F2(dy, i, 1); }
  const bool xdir = side <= 1;
  const float vel = xdir ? F3(u, vi, vj, k) : F3(v, vi, vj, k);
  const float u1 = 2.0f * vel * dti / dsum;
  const float q = F3(q2, ei, ej, k), ql = F3(q2l, ei, ej, k);
  const float qi = F3(q2, ii, ij, k), qli = F3(q2l, ii, ij, k);
  float lu1;
  if (side == 0 || side == 2) {
    if (u1 <= 0.0f) {
      GA3(q2, ei, ej, k, lu * (1.0f + u1));
      GA3(q2l, ei, ej, k, lv * (1.0f + u1));
      lu1 = -lu * (small - q) - lv * (small - ql);
    } else {
      GA3(q2, ei, ej, k, lu * (1.0f - u1));
      GA3(q2, ii, ij, k, lu * u1);
      GA3(q2l, ei, ej, k, lv * (1.0f - u1));
      GA3(q2l, ii, ij, k, lv * u1);
      lu1 = -lu * (q - qi) - lv * (ql - qli);
    }
  } else {
    if (u1 >= 0.0f) {
      GA3(q2, ei, ej, k, lu * (1.0f - u1));
      GA3(q2l, ei, ej, k, lv * (1.0f - u1));
      lu1 = -lu * (q - small) - lv * (ql - small);
    } else {
      GA3(q2, ei, ej, k, lu * (1.0f + u1));
      GA3(q2, ii, ij, k, -lu * u1);
      GA3(q2l, ei, ej, k, lv * (1.0f + u1));
      GA3(q2l, ii, ij, k, -lv * u1);
      lu1 = -lu * (qi - q) - lv * (qli - ql);
    }
  }
  const float lvel = lu1 * 2.0f * dti / dsum;
  if (xdir) GA3(u, vi, vj, k, lvel);
  else GA3(v, vi, vj, k, lvel);
}

// ===========================================================================
// B5: q2/q2l filter with the bcond 6 mask, ADVT1 of T and S
// (time_loop.py:521-556, tracers.py:433-569)
// ===========================================================================
NPOM_HD void advt1_xflux_adj(const Ctx &c, const Adj &a, int ff, int ffb, int fclim, int ii, int j, int k,
                             float lam) {
  const float *f = c.F[ff], *fb = c.F[ffb], *fcl = c.F[fclim];
  float *gf = a.G[ff], *gfb = a.G[ffb];
  const size_t o = NPOM_I3(c, ii, j, k), om = NPOM_I3(c, ii - 1, j, k);
  const float l = lam * 0.5f * (F2(dy, ii, j) + F2(dy, ii - 1, j));
  const float B = F2(dt, ii, j) + F2(dt, ii - 1, j), Fs = ld(f + o) + ld(f + om), uu = F3(u, ii, j, k);
  const float t = l * 0.25f;
  GA2(dt, ii, j, t * Fs * uu);
  GA2(dt, ii - 1, j, t * Fs * uu);
  aadd(gf + o, t * B * uu);
  aadd(gf + om, t * B * uu);
  GA3(u, ii, j, k, t * B * Fs);
  const float X = (F2(h, ii, j) + F2(h, ii - 1, j)) * c.k.tprni * F2(dum, ii, j) / (F2(dx, ii, j) + F2(dx, ii - 1, j));
  const float fdiff = (ld(fb + o) - ld(fcl + o)) - (ld(fb + om) - ld(fcl + om));
  const float aam_avg = 0.5f * (F3(aam, ii, j, k) + F3(aam, ii - 1, j, k));
  const float la = -l * X * fdiff * 0.5f;
  GA3(aam, ii, j, k, la);
  GA3(aam, ii - 1, j, k, la);
  const float lfa = -l * aam_avg * X;
  aadd(gfb + o, lfa);
  aadd(gfb + om, -lfa);
}

NPOM_HD void advt1_yflux_adj(const Ctx &c, const Adj &a, int ff, int ffb, int fclim, int i, int jj, int k,
                             float lam) {
  const float *f = c.F[ff], *fb = c.F[ffb], *fcl = c.F[fclim];
  float *gf = a.G[ff], *gfb = a.G[ffb];
  const size_t o = NPOM_I3(c, i, jj, k), om = NPOM_I3(c, i, jj - 1, k);
  const float l = lam * 0.5f * (F2(dx, i, jj) + F2(dx, i, jj - 1));
  const float B = F2(dt, i, jj) + F2(dt, i, jj - 1), Fs = ld(f + o) + ld(f + om), vv = F3(v, i, jj, k);
  const float t = l * 0.25f;
  GA2(dt, i, jj, t * Fs * vv);
  GA2(dt, i, jj - 1, t * Fs * vv);
  aadd(gf + o, t * B * vv);
  aadd(gf + om, t * B * vv);
  GA3(v, i, jj, k, t * B * Fs);
  const float X = (F2(h, i, jj) + F2(h, i, jj - 1)) * c.k.tprni * F2(dvm, i, jj) / (F2(dy, i, jj) + F2(dy, i, jj - 1));
  const float fdiff = (ld(fb + o) - ld(fcl + o)) - (ld(fb + om) - ld(fcl + om));
  const float aam_avg = 0.5f * (F3(aam, i, jj, k) + F3(aam, i, jj - 1, k));
  const float la = -l * X * fdiff * 0.5f;
  GA3(aam, i, jj, k, la);
  GA3(aam, i, jj - 1, k, la);
  const float lfa = -l * aam_avg * X;
  aadd(gfb + o, lfa);
  aadd(gfb + om, -lfa);
}

NPOM_HD void advt1_point_adj(const Ctx &c, const Adj &a, int ff, int ffb, int fclim, int i, int j, int k, float lam) {
  const int kbm1 = c.kb - 1;
  if (lam == 0.0f || !interior(c, i, j) || k >= kbm1) return;
  const float *f = c.F[ff], *fb = c.F[ffb], *fcl = c.F[fclim];
  float *gf = a.G[ff], *gfb = a.G[ffb];
  const float art = F2(art, i, j);
  const float horiz = advt1_xflux(c, f, fb, fcl, i + 1, j, k) - advt1_xflux(c, f, fb, fcl, i, j, k) +
                      advt1_yflux(c, f, fb, fcl, i, j + 1, k) - advt1_yflux(c, f, fb, fcl, i, j, k);
  const float out = advt1_finish(c, f, fb, i, j, k, horiz);
  const float tb = (F2(h, i, j) + F2(etb, i, j)) * art;
  const float tf = (F2(h, i, j) + F2(etf, i, j)) * art + 1e-20f;
  const size_t ok = NPOM_I3(c, i, j, k);
  const float lnum = lam / tf;
  GA2(etf, i, j, -lam * out / tf * art);
  GA2(etb, i, j, lnum * ld(fb + ok) * art);
  aadd(gfb + ok, lnum * tb);
  const float lff = -lnum * c.k.dti2;
  const float lz = lff / F1(dz, k);
  for (int s = 0; s < 2; ++s) {
    const int kk = k + s;
    const float lzz = s == 0 ? lz : -lz;
    if (kk == 0) {
      aadd(gf + NPOM_I3(c, i, j, 0), lzz * F3(w, i, j, 0) * art);
      GA3(w, i, j, 0, lzz * ld(f + NPOM_I3(c, i, j, 0)) * art);
    } else if (kk < kbm1) {
      const float fs = ld(f + NPOM_I3(c, i, j, kk - 1)) + ld(f + NPOM_I3(c, i, j, kk));
      const float t = lzz * 0.5f * F3(w, i, j, kk) * art;
      aadd(gf + NPOM_I3(c, i, j, kk - 1), t);
      aadd(gf + NPOM_I3(c, i, j, kk), t);
      GA3(w, i, j, kk, lzz * 0.5f * fs * art);
    }
  }
  advt1_xflux_adj(c, a, ff, ffb, fclim, i + 1, j, k, lff);
  advt1_xflux_adj(c, a, ff, ffb, fclim, i, j, k, -lff);
  advt1_yflux_adj(c, a, ff, ffb, fclim, i, j + 1, k, lff);
  advt1_yflux_adj(c, a, ff, ffb, fclim, i, j, k, -lff);
}

NPOM_HD void phase_b5_point_adj(const Ctx &c, const Adj &a, int i, int j, int k) {
  const int kb = c.kb;
  if (k == kb - 1) {
    GA3(t, i, j, kb - 2, LA3(t, i, j, k));
    GA3(tb, i, j, kb - 2, LA3(tb, i, j, k));
    GA3(s, i, j, kb - 2, LA3(s, i, j, k));
    GA3(sb, i, j, kb - 2, LA3(sb, i, j, k));
  } else {
    PASS3(t, i, j, k);
    PASS3(tb, i, j, k);
    PASS3(s, i, j, k);
    PASS3(sb, i, j, k);
  }
  advt1_point_adj(c, a, NPOM_F_t, NPOM_F_tb, NPOM_F_tclim, i, j, k, LA3(uf, i, j, k));
  advt1_point_adj(c, a, NPOM_F_s, NPOM_F_sb, NPOM_F_sclim, i, j, k, LA3(vf, i, j, k));
  if (!is_explicit(c) && c.k.has_vmix) {
    // clamp(x, 0, vmix): the gradient passes where 0 <= x <= vmix
    const float vm = c.k.vmix;
    const float kh = F3(kh, i, j, k), km = F3(km, i, j, k), kq = F3(kq, i, j, k);
    GA3(kh, i, j, k, (kh >= 0.0f && kh <= vm) ? LA3(kh, i, j, k) : 0.0f);
    GA3(km, i, j, k, (km >= 0.0f && km <= vm) ? LA3(km, i, j, k) : 0.0f);
    GA3(kq, i, j, k, (kq >= 0.0f && kq <= vm) ? LA3(kq, i, j, k) : 0.0f);
  }
  const float fsm = F2(fsm, i, j), hs = c.k.half_smoth, ohs = 1.0f - 2.0f * hs;
  const float lq2b = LA3(q2b, i, j, k), lq2lb = LA3(q2lb, i, j, k);
  GA3(q2, i, j, k, lq2b * ohs);
  GA3(q2b, i, j, k, lq2b * hs);
  GA3(uf, i, j, k, (LA3(q2, i, j, k) + lq2b * hs) * fsm);
  GA3(q2l, i, j, k, lq2lb * ohs);
  GA3(q2lb, i, j, k, lq2lb * hs);
  GA3(vf, i, j, k, (LA3(q2l, i, j, k) + lq2lb * hs) * fsm);
}

// ===========================================================================
// B6: PROFT of T and S (tracers.py:890-1010, nbc 1 or 3) and explicit
// bcond 4 on the edge columns (baroclinic.py:666-846)
// ===========================================================================
template <int KM>
NPOM_HD void proft_column_adj(const Ctx &c, const Adj &a, int i, int j, int fld, int nbc, float wfsurf,
                              float fsurf, const float *lout, float &ldh) {
  const int kb = KM == 16 ? 16 : c.kb, kbm1 = kb - 1, kbm2 = kb - 2;
  const size_t o = NPOM_I3(c, i, j, 0);
  const float *fcol = c.F[fld] + o;
  const float *khc = c.F[NPOM_F_kh] + o;
  const float dh = F2(h, i, j) + F2(etf, i, j);
  const float dh2 = dh * dh;
  const float neg_dti2 = -c.k.dti2;
  float fin[KM], av[KM], cc[KM], ee[KM], gg[KM], inv[KM], outv[KM];
  for (int k = 0; k < kb; ++k) {
    fin[k] = ld(fcol + k);
    av[k] = cc[k] = ee[k] = gg[k] = inv[k] = 0.0f;
  }
  for (int k = 1; k < kbm1; ++k) {
    const float num = neg_dti2 * (ld(khc + k) + c.k.umol);
    av[k - 1] = num / (F1(dz, k - 1) * F1(dzz, k - 1) * dh2);
    cc[k] = num / (F1(dz, k) * F1(dzz, k - 1) * dh2);
  }
  float T0 = 0.0f, den0 = 0.0f;
  if (nbc == 1) {
    den0 = av[0] - 1.0f;
    ee[0] = av[0] / den0;
    T0 = neg_dti2 * wfsurf / (-F1(dz, 0) * dh);
    gg[0] = (T0 - fin[0]) / den0;
  } else {
    ee[0] = 0.0f;
    gg[0] = fsurf;  // constant surface value (nbc 3)
  }
  for (int k = 1; k < kbm2; ++k) {
    const float den = av[k] + cc[k] * (1.0f - ee[k - 1]) - 1.0f;
    inv[k] = 1.0f / (den + 1e-20f);
    ee[k] = av[k] * inv[k];
    gg[k] = (cc[k] * gg[k - 1] - fin[k] + 0.0f) * inv[k];
  }
  const int kbt = kbm1 - 1;
  const float numT = cc[kbt] * gg[kbt - 1] - fin[kbt];
  const float denT = cc[kbt] * (1.0f - ee[kbt - 1]) - 1.0f + 1e-20f;
  outv[kbt] = numT / denT;
  for (int k = kbm1 - 2; k >= 0; --k) outv[k] = ee[k] * outv[k + 1] + gg[k];
  // reverse
  float lfin[KM], la[KM], lcc[KM], lee[KM], lgg[KM], lo[KM];
  for (int k = 0; k < kb; ++k) {
    lfin[k] = la[k] = lcc[k] = lee[k] = lgg[k] = 0.0f;
    lo[k] = lout[k];
  }
  lfin[kb - 1] += lo[kb - 1];
  for (int k = 0; k <= kbm1 - 2; ++k) {
    lee[k] += lo[k] * outv[k + 1];
    lgg[k] += lo[k];
    lo[k + 1] += lo[k] * ee[k];
  }
  {
    const float lq = lo[kbt];
    const float lnum = lq / denT, lden = -lq * outv[kbt] / denT;
    lcc[kbt] += lnum * gg[kbt - 1] + lden * (1.0f - ee[kbt - 1]);
    lgg[kbt - 1] += lnum * cc[kbt];
    lfin[kbt] -= lnum;
    lee[kbt - 1] -= lden * cc[kbt];
  }
  for (int k = kbm2 - 1; k >= 1; --k) {
    const float N = cc[k] * gg[k - 1] - fin[k];
    const float linv = lee[k] * av[k] + lgg[k] * N;
    la[k] += lee[k] * inv[k];
    const float lN = lgg[k] * inv[k];
    lcc[k] += lN * gg[k - 1];
    lgg[k - 1] += lN * cc[k];
    lfin[k] -= lN;
    const float lden = -linv * inv[k] * inv[k];
    la[k] += lden;
    lcc[k] += lden * (1.0f - ee[k - 1]);
    lee[k - 1] -= lden * cc[k];
  }
  if (nbc == 1) {
    la[0] += -lee[0] / (den0 * den0);
    la[0] += -lgg[0] * gg[0] / den0;
    const float lT0 = lgg[0] / den0;
    lfin[0] -= lgg[0] / den0;
    ldh += -lT0 * T0 / dh;
  }
  float ldh2 = 0.0f;
  for (int k = 1; k < kbm1; ++k) {
    const float da = F1(dz, k - 1) * F1(dzz, k - 1) * dh2, dc = F1(dz, k) * F1(dzz, k - 1) * dh2;
    const float lnum = la[k - 1] / da + lcc[k] / dc;
    GA3(kh, i, j, k, lnum * neg_dti2);
    ldh2 += -(la[k - 1] * av[k - 1] + lcc[k] * cc[k]) / dh2;
  }
  ldh += ldh2 * 2.0f * dh;
  float *gcol = a.G[fld] + o;
  for (int k = 0; k < kb; ++k) aadd(gcol + k, lfin[k]);
}

// adjoint of bcond4_explicit_level: (lu, lv) are the cotangents of the new
// uf/vf at level k of an edge column
NPOM_HD void bcond4_explicit_level_adj(const Ctx &c, const Adj &a, int i, int j, int k, float lu, float lv) {
  const int im = c.im, jm = c.jm, kbm1 = c.kb - 1;
  const float dti = c.k.dti;
  int side = -1;
  if (i == im - 1) side = 0;
  if (i == 0) side = 1;
  if (j == jm - 1) side = 2;
  if (j == 0) side = 3;
  if (side < 0 || (lu == 0.0f && lv == 0.0f)) return;
  const bool xdir = side <= 1;
  int ei, ej, ii, ij, vi, vj;
  float dsum;
  if (side == 0) { ei = im - 1; ej = j; ii = im - 2; ij = j; vi = im - 1; vj = j; dsum = F2(dx, im - 1, j) + F2(dx, im - 2, j); }
  else if (side == 1) { ei = 0; ej = j; ii = 1; ij = j; vi = 1; vj = j; dsum = F2(dx, 0, j) + F2(dx, 1, j); }
  else if (side == 2) { ei = i; ej = jm - 1; ii = i; ij = jm - 2; vi = i; vj = jm - 1; dsum = F2(dy, i, jm - 1) + F2(dy, i, jm - 2); }
  else { ei = i; ej = 0; ii = i; ij = 1; vi = i; vj = 1; dsum = F2(dy, i, 0) + F2(dy, i, 1); }
  const float vel = xdir ? F3(u, vi, vj, k) : F3(v, vi, vj, k);
  const float u1 = 2.0f * vel * dti / dsum;
  const float tc = F3(t, ei, ej, k), sc = F3(s, ei, ej, k), ti = F3(t, ii, ij, k), si = F3(s, ii, ij, k);
  float te, se;
  if (xdir) {
    const size_t eo = (size_t)j * c.kb + k;
    te = ld((side == 0 ? c.F[NPOM_F_tbe] : c.F[NPOM_F_tbw]) + eo);
    se = ld((side == 0 ? c.F[NPOM_F_sbe] : c.F[NPOM_F_sbw]) + eo);
  } else {
    const size_t eo = (size_t)i * c.kb + k;
    te = ld((side == 2 ? c.F[NPOM_F_tbn] : c.F[NPOM_F_tbs]) + eo);
    se = ld((side == 2 ? c.F[NPOM_F_sbn] : c.F[NPOM_F_sbs]) + eo);
  }
  const bool east_like = (side == 0 || side == 2);
  float lu1;
  if (east_like) {
    if (u1 <= 0.0f) {
      GA3(t, ei, ej, k, lu * (1.0f + u1));
      GA3(s, ei, ej, k, lv * (1.0f + u1));
      lu1 = -lu * (te - tc) - lv * (se - sc);
    } else {
      GA3(t, ei, ej, k, lu * (1.0f - u1));
      GA3(t, ii, ij, k, lu * u1);
      GA3(s, ei, ej, k, lv * (1.0f - u1));
      GA3(s, ii, ij, k, lv * u1);
      lu1 = -lu * (tc - ti) - lv * (sc - si);
    }
  } else {
    if (u1 >= 0.0f) {
      GA3(t, ei, ej, k, lu * (1.0f - u1));
      GA3(s, ei, ej, k, lv * (1.0f - u1));
      lu1 = -lu * (tc - te) - lv * (sc - se);
    } else {
      GA3(t, ei, ej, k, lu * (1.0f + u1));
      GA3(t, ii, ij, k, -lu * u1);
      GA3(s, ei, ej, k, lv * (1.0f + u1));
      GA3(s, ii, ij, k, -lv * u1);
      lu1 = -lu * (ti - tc) - lv * (si - sc);
    }
  }
  if (kbm1 > 2 && k >= 1 && k <= kbm1 - 2) {
    const bool outflow = east_like ? (u1 > 0.0f) : (u1 < 0.0f);
    if (outflow) {
      const float wsum = F3(w, ii, ij, k) + F3(w, ii, ij, k + 1);
      const float dtv = F2(dt, ii, ij);
      const float dzv = F1(zz, k - 1) - F1(zz, k + 1);
      const float wm = 0.5f * wsum * dti / (dzv * dtv);
      const float tm = F3(t, ii, ij, k - 1), tp = F3(t, ii, ij, k + 1);
      const float sm = F3(s, ii, ij, k - 1), sp = F3(s, ii, ij, k + 1);
      GA3(t, ii, ij, k - 1, -lu * wm);
      GA3(t, ii, ij, k + 1, lu * wm);
      GA3(s, ii, ij, k - 1, -lv * wm);
      GA3(s, ii, ij, k + 1, lv * wm);
      const float lwm = -lu * (tm - tp) - lv * (sm - sp);
      const float lws = lwm * 0.5f * dti / (dzv * dtv);
      GA3(w, ii, ij, k, lws);
      GA3(w, ii, ij, k + 1, lws);
      GA2(dt, ii, ij, -lwm * wm / dtv);
    }
  }
  const float lvel = lu1 * 2.0f * dti / dsum;
  if (xdir) GA3(u, vi, vj, k, lvel);
  else GA3(v, vi, vj, k, lvel);
}

template <int KM>
NPOM_HD void phase_b6_column_adj(const Ctx &c, const Adj &a, int i, int j) {
  const int kb = c.kb, kbm1 = kb - 1;
  float ldh = LA2(tps, i, j);
  float lu[KM], lv[KM];
  for (int k = 0; k < kb; ++k) {
    lu[k] = LA3(uf, i, j, k);
    lv[k] = LA3(vf, i, j, k);
  }
  if (is_explicit(c) && (i == 0 || i == c.im - 1 || j == 0 || j == c.jm - 1)) {
    for (int k = 0; k < kbm1; ++k) {
      bcond4_explicit_level_adj(c, a, i, j, k, lu[k], lv[k]);
      lu[k] = 0.0f;
      lv[k] = 0.0f;
    }
  }
  proft_column_adj<KM>(c, a, i, j, NPOM_F_uf, c.k.nbct, F2(wtsurf, i, j), F2(tsurf, i, j), lu, ldh);
  proft_column_adj<KM>(c, a, i, j, NPOM_F_vf, c.k.nbcs, F2(wssurf, i, j), F2(ssurf, i, j), lv, ldh);
  GA2(etf, i, j, ldh);
}

// ===========================================================================
// B7: explicit mask, T/S Robert-Asselin filter, shift and DENS
// (time_loop.py:583-603, momentum.py:467-541)
// ===========================================================================
NPOM_HD void dens_point_adj(const Ctx &c, float t, float s, int i, int j, int k, float &dt_, float &ds_) {
  const float tr = t + c.k.tbias, sr = s + c.k.sbias;
  const float tr2 = tr * tr, tr3 = tr2 * tr, tr4 = tr3 * tr;
  const float p = c.k.g_rhoref * (-F1(zz, k) * F2(h, i, j)) * 1.0e-5f;
  const float d1 = 6.793952e-2f - 2.0f * 9.095290e-3f * tr + 3.0f * 1.001685e-4f * tr2 - 4.0f * 1.120083e-6f * tr3 +
                   5.0f * 6.536332e-9f * tr4;
  const float P2 = 0.824493f - 4.0899e-3f * tr + 7.6438e-5f * tr2 - 8.2467e-7f * tr3 + 5.3875e-9f * tr4;
  const float d2 = -4.0899e-3f + 2.0f * 7.6438e-5f * tr - 3.0f * 8.2467e-7f * tr2 + 4.0f * 5.3875e-9f * tr3;
  const float P3 = -5.72466e-3f + 1.0227e-4f * tr - 1.6546e-6f * tr2;
  const float d3 = 1.0227e-4f - 2.0f * 1.6546e-6f * tr;
  const float as = fmaxf_t(fabsf(sr), 1e-8f);
  const float S15 = powf(as, 1.5f);
  const float dS15 = fabsf(sr) >= 1e-8f ? 1.5f * sqrtf(as) * sgnf(sr) : 0.0f;
  const float cr = 1449.1f + 0.0821f * p + 4.55f * tr - 0.045f * tr2 + 1.34f * (sr - 35.0f);
  const float cr2 = cr * cr;
  const float dQ = -2.0e5f * p / (cr2 * cr) + 8.0e5f * p * p / (cr2 * cr2 * cr);
  const float f = F2(fsm, i, j) / c.k.rhoref;
  dt_ = f * (d1 + d2 * sr + d3 * S15 + dQ * (4.55f - 0.09f * tr));
  ds_ = f * (P2 + P3 * dS15 + 2.0f * 4.8314e-4f * sr + dQ * 1.34f);
}

// explicit: T/S = uf/vf * fsm; closed basin (Shapiro gamma 0): the edge
// values copy the bcond 4 source cell, then T/S = value * fsm while the
// filter sees the unmasked value
NPOM_HD void phase_b7_point_adj(const Ctx &c, const Adj &a, int i, int j, int k) {
  const int im = c.im, jm = c.jm, kb = c.kb;
  const float fsm = F2(fsm, i, j), hs = c.k.half_smoth, ohs = 1.0f - 2.0f * hs;
  int si = i, sj = j;
  float fmask = fsm;  // d(ufv)/d(uf at the source): fsm for the explicit mask
  if (!is_explicit(c)) {
    fmask = 1.0f;
    if (sj == 0) sj = 1;
    if (sj == jm - 1) sj = jm - 2;
    if (si == 0) si = 1;
    if (si == im - 1) si = im - 2;
  }
  const float ufv = F3(uf, si, sj, k) * fmask, vfv = F3(vf, si, sj, k) * fmask;
  // tn = ufv (explicit) or ufv * fsm (closed basin)
  const float tmask = is_explicit(c) ? 1.0f : fsm;
  float lt = LA3(t, i, j, k), ls = LA3(s, i, j, k);
  if (k < kb - 1) {
    const float lr = LA3(rho, i, j, k);
    if (lr != 0.0f) {
      float dtn, dsn;
      dens_point_adj(c, ufv * tmask, vfv * tmask, i, j, k, dtn, dsn);
      lt += lr * dtn;
      ls += lr * dsn;
    }
  } else {
    PASS3(rho, i, j, k);
  }
  const float ltb = LA3(tb, i, j, k), lsb = LA3(sb, i, j, k);
  GA3(t, i, j, k, ltb * ohs);
  GA3(tb, i, j, k, ltb * hs);
  GA3(uf, si, sj, k, (ltb * hs + lt * tmask) * fmask);
  GA3(s, i, j, k, lsb * ohs);
  GA3(sb, i, j, k, lsb * hs);
  GA3(vf, si, sj, k, (lsb * hs + ls * tmask) * fmask);
}

// ===========================================================================
// B8: ADVU/ADVV + PROFU/PROFV (momentum.py:14-465), explicit bcond 3
// (baroclinic.py:576-661)
// ===========================================================================
NPOM_HD void advu_point_adj(const Ctx &c, const Adj &a, int i, int j, int k, float lam) {
  if (lam == 0.0f) return;
  const int kbm1 = c.kb - 1;
  const float aru = F2(aru, i, j);
  const float out = advu_point(c, i, j, k);
  const float hs = F2(h, i, j) + F2(h, i - 1, j);
  const float den = (hs + F2(etf, i, j) + F2(etf, i - 1, j)) * aru + 1e-20f;
  const float fo = (hs + F2(etb, i, j) + F2(etb, i - 1, j)) * aru;
  const float lold = lam / den, lrhs = -lam * c.k.two_dti2 / den, lden = -lam * out / den;
  GA2(etf, i, j, lden * aru);
  GA2(etf, i - 1, j, lden * aru);
  const float ub = F3(ub, i, j, k);
  GA2(etb, i, j, lold * aru * ub);
  GA2(etb, i - 1, j, lold * aru * ub);
  GA3(ub, i, j, k, lold * fo);
  GA3(advx, i, j, k, lrhs);
  GA3(drhox, i, j, k, lrhs);
  const float lvf = lrhs * aru / F1(dz, k);
  for (int s = 0; s < 2; ++s) {
    const int kk = k + s;
    const float l = s == 0 ? lvf : -lvf;
    if (kk < 1 || kk > kbm1 - 1) continue;
    const float ws = F3(w, i, j, kk) + F3(w, i - 1, j, kk), us = F3(u, i, j, kk) + F3(u, i, j, kk - 1);
    GA3(w, i, j, kk, l * 0.25f * us);
    GA3(w, i - 1, j, kk, l * 0.25f * us);
    GA3(u, i, j, kk, l * 0.25f * ws);
    GA3(u, i, j, kk - 1, l * 0.25f * ws);
  }
  const float lc = -lrhs * aru * 0.25f;
  const float vs1 = F3(v, i, j + 1, k) + F3(v, i, j, k), vs2 = F3(v, i - 1, j + 1, k) + F3(v, i - 1, j, k);
  GA2(dt, i, j, lc * F2(cor, i, j) * vs1);
  GA3(v, i, j + 1, k, lc * F2(cor, i, j) * F2(dt, i, j));
  GA3(v, i, j, k, lc * F2(cor, i, j) * F2(dt, i, j));
  GA2(dt, i - 1, j, lc * F2(cor, i - 1, j) * vs2);
  GA3(v, i - 1, j + 1, k, lc * F2(cor, i - 1, j) * F2(dt, i - 1, j));
  GA3(v, i - 1, j, k, lc * F2(cor, i - 1, j) * F2(dt, i - 1, j));
  const float geg = (F2(egf, i, j) - F2(egf, i - 1, j)) + (F2(egb, i, j) - F2(egb, i - 1, j));
  const float gpa = 2.0f * (F2(e_atmos, i, j) - F2(e_atmos, i - 1, j));
  const float lp = lrhs * c.k.g_eighth;
  const float dys = F2(dy, i, j) + F2(dy, i - 1, j), dts = F2(dt, i, j) + F2(dt, i - 1, j);
  GA2(dt, i, j, lp * (geg + gpa) * dys);
  GA2(dt, i - 1, j, lp * (geg + gpa) * dys);
  const float lg = lp * dts * dys;
  GA2(egf, i, j, lg);
  GA2(egf, i - 1, j, -lg);
  GA2(egb, i, j, lg);
  GA2(egb, i - 1, j, -lg);
}

NPOM_HD void advv_point_adj(const Ctx &c, const Adj &a, int i, int j, int k, float lam) {
  if (lam == 0.0f) return;
  const int kbm1 = c.kb - 1;
  const float arv = F2(arv, i, j);
  const float out = advv_point(c, i, j, k);
  const float hs = F2(h, i, j) + F2(h, i, j - 1);
  const float den = (hs + F2(etf, i, j) + F2(etf, i, j - 1)) * arv + 1e-20f;
  const float fo = (hs + F2(etb, i, j) + F2(etb, i, j - 1)) * arv;
  const float lold = lam / den, lrhs = -lam * c.k.two_dti2 / den, lden = -lam * out / den;
  GA2(etf, i, j, lden * arv);
  GA2(etf, i, j - 1, lden * arv);
  const float vb = F3(vb, i, j, k);
  GA2(etb, i, j, lold * arv * vb);
  GA2(etb, i, j - 1, lold * arv * vb);
  GA3(vb, i, j, k, lold * fo);
  GA3(advy, i, j, k, lrhs);
  GA3(drhoy, i, j, k, lrhs);
  const float lvf = lrhs * arv / F1(dz, k);
  for (int s = 0; s < 2; ++s) {
    const int kk = k + s;
    const float l = s == 0 ? lvf : -lvf;
    if (kk < 1 || kk > kbm1 - 1) continue;
    const float ws = F3(w, i, j, kk) + F3(w, i, j - 1, kk), vs = F3(v, i, j, kk) + F3(v, i, j, kk - 1);
    GA3(w, i, j, kk, l * 0.25f * vs);
    GA3(w, i, j - 1, kk, l * 0.25f * vs);
    GA3(v, i, j, kk, l * 0.25f * ws);
    GA3(v, i, j, kk - 1, l * 0.25f * ws);
  }
  const float lc = lrhs * arv * 0.25f;
  const float us1 = F3(u, i + 1, j, k) + F3(u, i, j, k), us2 = F3(u, i + 1, j - 1, k) + F3(u, i, j - 1, k);
  GA2(dt, i, j, lc * F2(cor, i, j) * us1);
  GA3(u, i + 1, j, k, lc * F2(cor, i, j) * F2(dt, i, j));
  GA3(u, i, j, k, lc * F2(cor, i, j) * F2(dt, i, j));
  GA2(dt, i, j - 1, lc * F2(cor, i, j - 1) * us2);
  GA3(u, i + 1, j - 1, k, lc * F2(cor, i, j - 1) * F2(dt, i, j - 1));
  GA3(u, i, j - 1, k, lc * F2(cor, i, j - 1) * F2(dt, i, j - 1));
  const float geg = (F2(egf, i, j) - F2(egf, i, j - 1)) + (F2(egb, i, j) - F2(egb, i, j - 1));
  const float gpa = 2.0f * (F2(e_atmos, i, j) - F2(e_atmos, i, j - 1));
  const float lp = lrhs * c.k.g_eighth;
  const float dxs = F2(dx, i, j) + F2(dx, i, j - 1), dts = F2(dt, i, j) + F2(dt, i, j - 1);
  GA2(dt, i, j, lp * (geg + gpa) * dxs);
  GA2(dt, i, j - 1, lp * (geg + gpa) * dxs);
  const float lg = lp * dts * dxs;
  GA2(egf, i, j, lg);
  GA2(egf, i, j - 1, -lg);
  GA2(egb, i, j, lg);
  GA2(egb, i, j - 1, -lg);
}

// PROFU (comp 0) / PROFV (comp 1).  lout: cotangents of the column output
// (modified); lwbot, ltps: of the stored wubot/wvbot and tps; lfin: out,
// cotangents of the ADVU/ADVV forecast.
template <int KM>
NPOM_HD void profuv_column_adj(const Ctx &c, const Adj &a, int comp, int i, int j, float *lout, float lwbot,
                               float ltps, float *lfin) {
  const int kb = KM == 16 ? 16 : c.kb, kbm1 = kb - 1, kbm2 = kb - 2;
  for (int k = 0; k < kb; ++k) lfin[k] = 0.0f;
  if (i < 1 || j < 1 || !interior(c, i, j)) {
    // out = fin, wbot keeps its value
    for (int k = 0; k < kb; ++k) lfin[k] = lout[k];
    if (comp == 0) GA2(wubot, i, j, lwbot);
    else GA2(wvbot, i, j, lwbot);
    return;
  }
  const int oi = comp == 0 ? i - 1 : i, oj = comp == 0 ? j : j - 1;
  const float dti2 = c.k.dti2, eps = 1e-20f;
  float fin[KM], av[KM], cc[KM], ee[KM], gg[KM], inv[KM], outv[KM];
  for (int k = 0; k < kb; ++k) {
    fin[k] = (k < kb - 1) ? (comp == 0 ? advu_point(c, i, j, k) : advv_point(c, i, j, k)) : 0.0f;
    av[k] = cc[k] = ee[k] = gg[k] = inv[k] = 0.0f;
  }
  const float dhf = 0.5f * (F2(h, i, j) + F2(etf, i, j) + F2(h, oi, oj) + F2(etf, oi, oj));
  const float dh2 = dhf * dhf;
  for (int k = 1; k < kbm1; ++k) {
    const float kmf = 0.5f * (F3(km, i, j, k) + F3(km, oi, oj, k));
    const float num = c.k.neg_dti2 * (kmf + c.k.umol);
    av[k - 1] = num / (F1(dz, k - 1) * F1(dzz, k - 1) * dh2);
    cc[k] = num / (F1(dz, k) * F1(dzz, k - 1) * dh2);
  }
  const float dd0 = (av[0] - 1.0f) + eps;
  ee[0] = av[0] / dd0;
  const float wsurf = comp == 0 ? F2(wusurf, i, j) : F2(wvsurf, i, j);
  const float term = c.k.neg_dti2 * wsurf / (-F1(dz, 0) * dhf);
  gg[0] = (term - fin[0]) / dd0;
  for (int k = 1; k < kbm2; ++k) {
    const float den = av[k] + cc[k] * (1.0f - ee[k - 1]) - 1.0f;
    inv[k] = 1.0f / (den + eps);
    ee[k] = av[k] * inv[k];
    gg[k] = (cc[k] * gg[k - 1] - fin[k]) * inv[k];
  }
  const int kbt = kbm1 - 1;
  float cbc_avg, mag, ub0, vavg;
  if (comp == 0) {
    cbc_avg = 0.5f * (F2(cbc, i, j) + F2(cbc, i - 1, j));
    ub0 = F3(ub, i, j, kbt);
    vavg = 0.25f * (F3(vb, i, j, kbt) + F3(vb, i, j + 1, kbt) + F3(vb, i - 1, j, kbt) + F3(vb, i - 1, j + 1, kbt));
  } else {
    cbc_avg = 0.5f * (F2(cbc, i, j) + F2(cbc, i, j - 1));
    ub0 = F3(vb, i, j, kbt);
    vavg = 0.25f * (F3(ub, i, j, kbt) + F3(ub, i + 1, j, kbt) + F3(ub, i, j - 1, kbt) + F3(ub, i + 1, j - 1, kbt));
  }
  mag = sqrtf(ub0 * ub0 + vavg * vavg + 1e-8f);
  const float tps = cbc_avg * mag;
  const float fric = tps * dti2 / (-F1(dz, kbt) * dhf);
  const float den = fric - 1.0f - (ee[kbt - 1] - 1.0f) * cc[kbt] + eps;
  const float num = cc[kbt] * gg[kbt - 1] - fin[kbt];
  const float mask = comp == 0 ? F2(dum, i, j) : F2(dvm, i, j);
  const float q = num / den;
  outv[kbt] = q * mask;
  for (int k = kbt - 1; k >= 0; --k) outv[k] = (ee[k] * outv[k + 1] + gg[k]) * mask;
  // reverse
  float la[KM], lcc[KM], lee[KM], lgg[KM];
  for (int k = 0; k < kb; ++k) la[k] = lcc[k] = lee[k] = lgg[k] = 0.0f;
  lfin[kb - 1] += lout[kb - 1];
  lout[kbt] += -lwbot * tps;
  float ltp = ltps - lwbot * outv[kbt];
  for (int k = 0; k < kbt; ++k) {
    const float lp = lout[k] * mask;
    lee[k] += lp * outv[k + 1];
    lgg[k] += lp;
    lout[k + 1] += lp * ee[k];
  }
  const float lq = lout[kbt] * mask;
  const float lnum = lq / den, lden = -lq * q / den;
  lcc[kbt] += lnum * gg[kbt - 1] - lden * (ee[kbt - 1] - 1.0f);
  lgg[kbt - 1] += lnum * cc[kbt];
  lfin[kbt] -= lnum;
  lee[kbt - 1] -= lden * cc[kbt];
  float ldhf = -lden * fric / dhf;
  ltp += lden * dti2 / (-F1(dz, kbt) * dhf);
  const float lmag = ltp * cbc_avg;
  if (lmag != 0.0f) {
    const float l0 = lmag * ub0 / mag, l1 = lmag * vavg / mag * 0.25f;
    if (comp == 0) {
      GA3(ub, i, j, kbt, l0);
      GA3(vb, i, j, kbt, l1);
      GA3(vb, i, j + 1, kbt, l1);
      GA3(vb, i - 1, j, kbt, l1);
      GA3(vb, i - 1, j + 1, kbt, l1);
    } else {
      GA3(vb, i, j, kbt, l0);
      GA3(ub, i, j, kbt, l1);
      GA3(ub, i + 1, j, kbt, l1);
      GA3(ub, i, j - 1, kbt, l1);
      GA3(ub, i + 1, j - 1, kbt, l1);
    }
  }
  for (int k = kbm2 - 1; k >= 1; --k) {
    const float N = cc[k] * gg[k - 1] - fin[k];
    const float linv = lee[k] * av[k] + lgg[k] * N;
    la[k] += lee[k] * inv[k];
    const float lN = lgg[k] * inv[k];
    lcc[k] += lN * gg[k - 1];
    lgg[k - 1] += lN * cc[k];
    lfin[k] -= lN;
    const float ld_ = -linv * inv[k] * inv[k];
    la[k] += ld_;
    lcc[k] += ld_ * (1.0f - ee[k - 1]);
    lee[k - 1] -= ld_ * cc[k];
  }
  la[0] += lee[0] / dd0 - lee[0] * ee[0] / dd0 - lgg[0] * gg[0] / dd0;
  const float lterm = lgg[0] / dd0;
  lfin[0] -= lgg[0] / dd0;
  ldhf += -lterm * term / dhf;
  float ldh2 = 0.0f;
  for (int k = 1; k < kbm1; ++k) {
    const float da = F1(dz, k - 1) * F1(dzz, k - 1) * dh2, dc = F1(dz, k) * F1(dzz, k - 1) * dh2;
    const float ln = (la[k - 1] / da + lcc[k] / dc) * c.k.neg_dti2 * 0.5f;
    GA3(km, i, j, k, ln);
    GA3(km, oi, oj, k, ln);
    ldh2 += -(la[k - 1] * av[k - 1] + lcc[k] * cc[k]) / dh2;
  }
  ldhf += ldh2 * 2.0f * dhf;
  GA2(etf, i, j, 0.5f * ldhf);
  GA2(etf, oi, oj, 0.5f * ldhf);
}

// explicit bcond 3: levels overwritten by the edge formulas take their
// cotangent out of luo/lvo
// comps: 1 the u edges, 2 the v edges, 3 both (their cotangents and
// scatters are independent)
NPOM_HD void bcond3_explicit_edge_adj(const Ctx &c, const Adj &a, int i, int j, float *luo, float *lvo,
                                      int comps = 3) {
  const int im = c.im, jm = c.jm, kbm1 = c.kb - 1;
  enum { KEEP = 0, EAST, WEST, NORTH, SOUTH, ZERO };
  int su = KEEP, sv = KEEP;
  if (j >= 1 && j <= jm - 2) {
    if (i == im - 1) { su = EAST; sv = ZERO; }
    if (i == 1 || i == 0) { su = WEST; if (i == 0) sv = ZERO; }
  }
  if (i >= 1 && i <= im - 2) {
    if (j == jm - 1) { sv = NORTH; su = ZERO; }
    if (j == 1 || j == 0) { sv = SOUTH; if (j == 0) su = ZERO; }
  }
  if (!(comps & 1)) su = KEEP;
  if (!(comps & 2)) sv = KEEP;
  if (su == KEEP && sv == KEEP) return;
  const float hmax = c.k.hmax;
  auto ga_of = [&](float hh) { return sqrtf(fmaxf_t(hh / hmax, 1e-8f)); };
  for (int k = 0; k < kbm1; ++k) {
    const float lu = (comps & 1) ? luo[k] : 0.0f, lv = (comps & 2) ? lvo[k] : 0.0f;
    if (su == EAST || su == WEST) {
      const float ga = su == EAST ? ga_of(F2(h, im - 1, j)) : ga_of(F2(h, 0, j));
      const int ii = su == EAST ? im - 2 : 2, io = su == EAST ? im - 1 : 1;
      GA3(u, ii, j - 1, k, 0.25f * ga * lu);
      GA3(u, ii, j, k, 0.50f * ga * lu);
      GA3(u, ii, j + 1, k, 0.25f * ga * lu);
      const float g1 = 1.0f - ga;
      GA3(u, io, j - 1, k, 0.25f * g1 * lu);
      GA3(u, io, j, k, 0.50f * g1 * lu);
      GA3(u, io, j + 1, k, 0.25f * g1 * lu);
    }
    if (sv == NORTH || sv == SOUTH) {
      const float ga = sv == NORTH ? ga_of(F2(h, i, jm - 1)) : ga_of(F2(h, i, 0));
      const int jj = sv == NORTH ? jm - 2 : 2, jo = sv == NORTH ? jm - 1 : 1;
      GA3(v, i - 1, jj, k, 0.25f * ga * lv);
      GA3(v, i, jj, k, 0.50f * ga * lv);
      GA3(v, i + 1, jj, k, 0.25f * ga * lv);
      const float g1 = 1.0f - ga;
      GA3(v, i - 1, jo, k, 0.25f * g1 * lv);
      GA3(v, i, jo, k, 0.50f * g1 * lv);
      GA3(v, i + 1, jo, k, 0.25f * g1 * lv);
    }
    if (su != KEEP) luo[k] = 0.0f;
    if (sv != KEEP) lvo[k] = 0.0f;
  }
}

// one component of B8 (comp 0: ADVU, PROFU and the u edges of bcond 3;
// 1: the v side, which also carries the cotangent of tps): the two share
// no intermediate, so the device runs them on two threads
template <int KM>
NPOM_HD void phase_b8_comp_adj(const Ctx &c, const Adj &a, int comp, int i, int j) {
  const int kb = c.kb;
  const bool inner = interior(c, i, j);
  float lo[KM], lfin[KM];
  for (int k = 0; k < kb; ++k) lo[k] = comp == 0 ? LA3(uf, i, j, k) : LA3(vf, i, j, k);
  if (is_explicit(c)) bcond3_explicit_edge_adj(c, a, i, j, lo, lo, comp == 0 ? 1 : 2);
  if (comp == 0) {
    profuv_column_adj<KM>(c, a, 0, i, j, lo, LA2(wubot, i, j), 0.0f, lfin);
    if (inner)
      for (int k = 0; k < kb - 1; ++k) advu_point_adj(c, a, i, j, k, lfin[k]);
  } else {
    profuv_column_adj<KM>(c, a, 1, i, j, lo, LA2(wvbot, i, j), LA2(tps, i, j), lfin);
    if (inner)
      for (int k = 0; k < kb - 1; ++k) advv_point_adj(c, a, i, j, k, lfin[k]);
  }
}

template <int KM>
NPOM_HD void phase_b8_column_adj(const Ctx &c, const Adj &a, int i, int j) {
  phase_b8_comp_adj<KM>(c, a, 0, i, j);
  phase_b8_comp_adj<KM>(c, a, 1, i, j);
}

// ===========================================================================
// B9: velocity filter and shift, 2-D shifts (time_loop.py:628-696)
// ===========================================================================
template <int KM>
NPOM_HD void phase_b9_column_adj(const Ctx &c, const Adj &a, int i, int j) {
  const int kb = KM == 16 ? 16 : c.kb, kbm1 = kb - 1;
  if (c.do_internal) {
    const float hs = c.k.half_smoth;
    const bool ring = (i == 0 || i == c.im - 1 || j == 0 || j == c.jm - 1);
    for (int comp = 0; comp < 2; ++comp) {
      const float mask = comp == 0 ? F2(dum, i, j) : F2(dvm, i, j);
      // closed basin: the ring is zero and the filtered value is masked
      const float fmask = (!is_explicit(c) && ring) ? 0.0f : mask;
      const float bmask = is_explicit(c) ? 1.0f : mask;
      const int fa = comp == 0 ? NPOM_F_u : NPOM_F_v;
      const int fb = comp == 0 ? NPOM_F_ub : NPOM_F_vb;
      const int ff = comp == 0 ? NPOM_F_uf : NPOM_F_vf;
      const size_t o = NPOM_I3(c, i, j, 0);
      float lfnew[KM], lterm[KM];
      float ltps = 0.0f;
      for (int k = 0; k < kb; ++k) {
        lfnew[k] = a.L[fa][o + k] + a.L[ff][o + k];
        lterm[k] = 0.0f;
        const float lfb = a.L[fb][o + k] * bmask;
        aadd(a.G[fa] + o + k, lfb);
        if (k < kbm1) {
          lterm[k] += hs * lfb;
          ltps -= hs * lfb;
        }
      }
      for (int k = 0; k < kbm1; ++k) {
        lterm[k] += ltps * F1(dz, k);
        lfnew[k] += lterm[k];
        aadd(a.G[fb] + o + k, lterm[k]);
        aadd(a.G[fa] + o + k, -2.0f * lterm[k]);
      }
      for (int k = 0; k < kb; ++k) aadd(a.G[ff] + o + k, lfnew[k] * fmask);
    }
  }
  GA2(egf, i, j, LA2(egb, i, j));
  GA2(et, i, j, LA2(etb, i, j));
  GA2(etf, i, j, LA2(et, i, j) + LA2(dt, i, j));
  GA2(utf, i, j, LA2(utb, i, j));
  GA2(vtf, i, j, LA2(vtb, i, j));
}

#undef GA3
#undef GA2
#undef LA3
#undef LA2
#undef PASS3
#undef PASS2
#undef GAW
#undef LAW

}  // namespace npom

// ---------------------------------------------------------------------------
// The phase plan of one explicit internal step, shared by the CUDA driver
// and the CPU emulation: the phases in forward order, and for each the
// fields it overwrites (saved before the forward recomputation, restored
// before its adjoint) and whether their cotangents move (fields whose
// derivative is the identity, the rho round trip of A3, only restore).
// Geometry and the explicit core's zero forcing fields are never saved.
// ---------------------------------------------------------------------------
namespace npom {

enum AdjPhase {
  AP_A1 = 0, AP_A2, AP_A3, AP_E1, AP_E2, AP_E3, AP_B1, AP_B2A, AP_B2B, AP_B3, AP_B4, AP_B5, AP_B6, AP_B7, AP_B8, AP_B9,
  AP_EI, AP_I5,
  // B5 with MPDATA (nadv 2), pass by pass: the q2/q2l filter, mass fluxes,
  // per iteration (iext = the iteration) upstream fluxes, forecast and
  // antidiffusive fluxes, then the diffusive fluxes and the final update
  AP_MQ, AP_MINIT, AP_MUP, AP_MFC, AP_MAD, AP_MDIF, AP_MFIN
};
// phases of one step's plan at most (isplit substeps of three phases)
NPOM_HD int adj_plan_capacity(int isplit, int nitera) { return 24 + 3 * isplit + 3 * nitera; }
constexpr int kAdjMaxFields = 16;

struct AdjPhaseRec {
  int phase, iext, adv, n;
  int fld[kAdjMaxFields];
  int move[kAdjMaxFields];
  size_t off[kAdjMaxFields];
};

NPOM_HD size_t adj_field_len(const Ctx &c, int f) {
  const bool three_d = (f >= NPOM_F_u && f <= NPOM_F_curv) || f >= NPOM_NFIELDS + AW_COUNT;
  return three_d ? (size_t)c.im * c.jm * c.kb : (size_t)c.im * c.jm;
}

// The 2-D fields external-substep phase ph (1, 2, 3) of substep iext
// overwrites, in save order; returns their number (at most 10).
NPOM_HD int ext_phase_fields(int iext, int ph, int isplit, int ispadv, int *fld) {
  int n = 0;
  if (ph == 1) {
    fld[n++] = NPOM_F_elf;
    fld[n++] = NPOM_F_fluxua;
    fld[n++] = NPOM_F_fluxva;
    if ((iext % ispadv) == 0) {
      fld[n++] = NPOM_F_advua;
      fld[n++] = NPOM_F_advva;
      fld[n++] = NPOM_F_tps;
    }
  } else if (ph == 2) {
    fld[n++] = NPOM_F_uaf;
    fld[n++] = NPOM_F_vaf;
    if (iext >= isplit - 2) fld[n++] = NPOM_F_etf;
  } else {
    fld[n++] = NPOM_F_elb;
    fld[n++] = NPOM_F_el;
    fld[n++] = NPOM_F_d;
    fld[n++] = NPOM_F_uab;
    fld[n++] = NPOM_F_ua;
    fld[n++] = NPOM_F_vab;
    fld[n++] = NPOM_F_va;
    if (iext != isplit) {
      fld[n++] = NPOM_F_egf;
      fld[n++] = NPOM_F_utf;
      fld[n++] = NPOM_F_vtf;
    }
  }
  return n;
}

// Fills out (capacity cap) and returns the number of phases; *save_floats
// receives the size of the save area.
inline int adj_step_plan(const Ctx &c, AdjPhaseRec *out, int cap, size_t *save_floats) {
  int np = 0;
  size_t off = 0;
  auto begin = [&](int phase, int iext, int adv) -> AdjPhaseRec * {
    if (np >= cap) return nullptr;
    AdjPhaseRec *r = &out[np++];
    r->phase = phase;
    r->iext = iext;
    r->adv = adv;
    r->n = 0;
    return r;
  };
  auto add = [&](AdjPhaseRec *r, int f, int move) {
    if (!r || r->n >= kAdjMaxFields) return;
    r->fld[r->n] = f;
    r->move[r->n] = move;
    r->off[r->n] = off;
    off += adj_field_len(c, f);
    r->n++;
  };
  AdjPhaseRec *r = begin(AP_A1, 0, 0);
  for (int f : {NPOM_F_advx, NPOM_F_advy, NPOM_F_curv, NPOM_F_w}) add(r, f, 1);
  r = begin(AP_A2, 0, 0);
  for (int f : {NPOM_F_drhox, NPOM_F_drhoy, NPOM_F_aam, NPOM_F_adx2d, NPOM_F_ady2d, NPOM_F_drx2d, NPOM_F_dry2d,
                NPOM_F_aam2d})
    add(r, f, 1);
  r = begin(AP_A3, 0, 0);
  add(r, NPOM_F_rho, 0);
  for (int f : {NPOM_F_advua, NPOM_F_advva, NPOM_F_fluxua, NPOM_F_fluxva, NPOM_F_tps, NPOM_F_adx2d, NPOM_F_ady2d,
                NPOM_F_egf, NPOM_F_utf, NPOM_F_vtf})
    add(r, f, 1);
  const bool imp = c.k.core == NPOM_CORE_IMPLICIT;
  if (imp) {
    for (int w = 0; w < AW_COUNT; ++w) add(r, NPOM_NFIELDS + w, 1);
    r = begin(AP_EI, 0, 0);
    for (int f : {NPOM_F_fluxua, NPOM_F_fluxva, NPOM_F_elf, NPOM_F_d}) add(r, f, 1);
    r = begin(AP_I5, 0, 0);
    for (int f : {NPOM_F_uaf, NPOM_F_vaf, NPOM_F_etf, NPOM_F_elb, NPOM_F_el, NPOM_F_d, NPOM_F_uab, NPOM_F_ua,
                  NPOM_F_vab, NPOM_F_va, NPOM_F_egf, NPOM_F_utf, NPOM_F_vtf})
      add(r, f, 1);
  }
  const int isplit = imp ? 0 : c.k.isplit;
  for (int iext = 1; iext <= isplit; ++iext) {
    const int adv = (iext % c.k.ispadv) == 0;
    for (int ph = 1; ph <= 3; ++ph) {
      r = begin(ph == 1 ? AP_E1 : (ph == 2 ? AP_E2 : AP_E3), iext, adv);
      int fl[10];
      const int nf = ext_phase_fields(iext, ph, isplit, c.k.ispadv, fl);
      for (int e = 0; e < nf; ++e) add(r, fl[e], 1);
    }
  }
  if (c.do_internal) {
    r = begin(AP_B1, 0, 0);
    add(r, NPOM_F_u, 1);
    add(r, NPOM_F_v, 1);
    r = begin(AP_B2A, 0, 0);
    add(r, NPOM_F_w, 1);
    r = begin(AP_B2B, 0, 0);
    add(r, NPOM_F_uf, 1);
    add(r, NPOM_F_vf, 1);
    r = begin(AP_B3, 0, 0);
    for (int f : {NPOM_F_l, NPOM_F_kq, NPOM_F_km, NPOM_F_kh, NPOM_F_uf, NPOM_F_vf}) add(r, f, 1);
    r = begin(AP_B4, 0, 0);
    add(r, NPOM_F_km, 1);
    add(r, NPOM_F_kh, 1);
    if (!imp) {
      add(r, NPOM_F_uf, 1);
      add(r, NPOM_F_vf, 1);
    }
    if (c.k.nadv == 2 && c.k.mode != 4) {
      r = begin(AP_MQ, 0, 0);
      for (int f : {NPOM_F_q2b, NPOM_F_q2, NPOM_F_q2lb, NPOM_F_q2l}) add(r, f, 1);
      if (imp && c.k.has_vmix)
        for (int f : {NPOM_F_kh, NPOM_F_km, NPOM_F_kq}) add(r, f, 1);
      r = begin(AP_MINIT, 0, 0);
      for (int tr = 0; tr < 2; ++tr)
        for (int m = 0; m < 3; ++m) add(r, mp_slot(tr, m), 1);
      add(r, NPOM_F_tb, 1);
      add(r, NPOM_F_sb, 1);
      for (int it = 1; it <= c.k.nitera; ++it) {
        r = begin(AP_MUP, it, 0);
        for (int tr = 0; tr < 2; ++tr)
          for (int m = 3; m < 6; ++m) add(r, mp_slot(tr, m), 1);
        r = begin(AP_MFC, it, 0);
        add(r, NPOM_F_uf, 1);
        add(r, NPOM_F_vf, 1);
        r = begin(AP_MAD, it, 0);
        for (int tr = 0; tr < 2; ++tr)
          for (int m = 0; m < 3; ++m) add(r, mp_slot(tr, m), 1);
      }
      r = begin(AP_MDIF, 0, 0);
      for (int tr = 0; tr < 2; ++tr)
        for (int m = 3; m < 5; ++m) add(r, mp_slot(tr, m), 1);
      r = begin(AP_MFIN, 0, 0);
      add(r, NPOM_F_uf, 1);
      add(r, NPOM_F_vf, 1);
    } else {
      r = begin(AP_B5, 0, 0);
      for (int f : {NPOM_F_q2b, NPOM_F_q2, NPOM_F_q2lb, NPOM_F_q2l, NPOM_F_uf, NPOM_F_vf, NPOM_F_t, NPOM_F_tb,
                    NPOM_F_s, NPOM_F_sb})
        add(r, f, 1);
      if (imp && c.k.has_vmix)
        for (int f : {NPOM_F_kh, NPOM_F_km, NPOM_F_kq}) add(r, f, 1);
    }
    r = begin(AP_B6, 0, 0);
    for (int f : {NPOM_F_uf, NPOM_F_vf, NPOM_F_tps}) add(r, f, 1);
    r = begin(AP_B7, 0, 0);
    for (int f : {NPOM_F_tb, NPOM_F_sb, NPOM_F_t, NPOM_F_s, NPOM_F_rho}) add(r, f, 1);
    r = begin(AP_B8, 0, 0);
    for (int f : {NPOM_F_uf, NPOM_F_vf, NPOM_F_wubot, NPOM_F_wvbot, NPOM_F_tps}) add(r, f, 1);
  }
  r = begin(AP_B9, 0, 0);
  if (c.do_internal)
    for (int f : {NPOM_F_u, NPOM_F_ub, NPOM_F_uf, NPOM_F_v, NPOM_F_vb, NPOM_F_vf}) add(r, f, 1);
  for (int f : {NPOM_F_egb, NPOM_F_etb, NPOM_F_et, NPOM_F_dt, NPOM_F_utb, NPOM_F_vtb}) add(r, f, 1);
  if (save_floats) *save_floats = off;
  return np;
}

// Settings the adjoint covers: mode 3 with centred tracer advection and
// surface flux (nbc 1) or value (nbc 3) conditions; for the implicit core
// the production Shapiro filters (gamma 0).
inline bool adj_supported(const npom_params *p) {
  // the POM08-WAD PROFQ is forward only, as in the reference's case
  // policies (which refuse advancement with gradients)
  // (periodic x is forward only too: its halo copies have no reverse here)
  const bool base = p->mode == 3 && (p->nbct == 1 || p->nbct == 3) && (p->nbcs == 1 || p->nbcs == 3) &&
                    p->profq_form == NPOM_PROFQ_PRODUCTION && p->obc_form == NPOM_OBC_NATIVE && !p->periodic_x;
  if (p->core == NPOM_CORE_EXPLICIT) return base && (p->nadv == 1 || p->nadv == 2);
  return base && (p->nadv == 1 || p->nadv == 2) && p->core == NPOM_CORE_IMPLICIT && p->barotropic_shapiro == 0.0 &&
         p->tracer_shapiro == 0.0;
}

// The scratch of one step adjoint, after the plan's saves: G and L of the
// workspace slots, the PCG solution, g, lambda and grad d (2-D planes),
// then with MPDATA G and L of its slots (3-D arrays).
constexpr int kAdjScratchPlanes = 2 * AW_COUNT + 4;
NPOM_HD bool adj_has_mp(const Ctx &c) { return c.k.nadv == 2 && c.k.mode != 4; }
inline size_t adj_scratch_floats(const Ctx &c) {
  const size_t ncell = (size_t)c.im * c.jm;
  return (size_t)kAdjScratchPlanes * ncell + (adj_has_mp(c) ? (size_t)2 * kAdjMpSlots * ncell * c.kb : 0);
}
// the floats of the scratch that start each step at zero: G of the
// workspace slots, then (a separate range) G of the MPDATA slots
inline size_t adj_mp_offset(const Ctx &c) { return (size_t)kAdjScratchPlanes * c.im * c.jm; }
inline size_t adj_mp_zero_floats(const Ctx &c) {
  return adj_has_mp(c) ? (size_t)kAdjMpSlots * c.im * c.jm * c.kb : 0;
}
// points the workspace and MPDATA slots of a into scratch
inline void adj_bind_scratch(const Ctx &c, Adj &a, float *scratch) {
  const size_t ncell = (size_t)c.im * c.jm, n3 = ncell * c.kb;
  for (int w = 0; w < AW_COUNT; ++w) {
    a.G[NPOM_NFIELDS + w] = scratch + (size_t)w * ncell;
    a.L[NPOM_NFIELDS + w] = scratch + (size_t)(AW_COUNT + w) * ncell;
  }
  float *mp = scratch + adj_mp_offset(c);
  for (int q = 0; q < kAdjMpSlots; ++q) {
    a.G[NPOM_NFIELDS + AW_COUNT + q] = adj_has_mp(c) ? mp + (size_t)q * n3 : nullptr;
    a.L[NPOM_NFIELDS + AW_COUNT + q] = adj_has_mp(c) ? mp + (size_t)(kAdjMpSlots + q) * n3 : nullptr;
  }
}

}  // namespace npom
