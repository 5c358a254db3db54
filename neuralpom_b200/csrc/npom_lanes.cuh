// npom_lanes.cuh -- the column phases with one 16-lane segment per water
// column (kb == 16): lane k owns sigma level k.  Level-local arithmetic runs
// in parallel; the vertical recurrences (k-sums, k-cumsums, the forward and
// backward sweeps of the Thomas algorithm) keep the reference's sequential
// order by passing one value per step through warp shuffles.  Every body
// computes exactly the same floating-point expressions, in the same order,
// as the sequential column bodies of npom_phases_a/_int.cuh (which the CPU
// emulator runs); only the mapping onto threads differs.
#pragma once

#include "npom_phases_int.cuh"

namespace npom {

constexpr int KL = 16;  // levels per column on the lane path
constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ float sh(float v, int src) { return __shfl_sync(kFull, v, src, KL); }
__device__ __forceinline__ double shd(double v, int src) { return __shfl_sync(kFull, v, src, KL); }

// ((0 + v_0) + v_1) + ... + v_{n-1}, the same in every lane
__device__ __forceinline__ float seg_sum(float v, int n) {
  float s = 0.0f;
#pragma unroll
  for (int m = 0; m < KL; ++m) {
    float t = sh(v, m);
    if (m < n) s += t;
  }
  return s;
}

// sum_{m=lo..hi} (double)v_m in increasing m (hi may depend on the lane)
__device__ __forceinline__ double seg_prefix(double v, int lo, int hi) {
  double acc = 0.0;
#pragma unroll
  for (int m = 0; m < KL; ++m) {
    double t = shd(v, m);
    if (m >= lo && m <= hi) acc += t;
  }
  return acc;
}

// ---------------------------------------------------------------------------
// A2: BAROPG + Smagorinsky + depth integrals
// ---------------------------------------------------------------------------
__device__ __forceinline__ void lane_a2(const Ctx &c, int i, int j, int k, bool st) {
  const int kbm1 = KL - 1;
  const bool in = interior(c, i, j);
  float dr[2] = {0.0f, 0.0f};
  if (in) {
    const float ramp = c.ramp;
#pragma unroll
    for (int comp = 0; comp < 2; ++comp) {
      const int bi = comp == 0 ? i - 1 : i;
      const int bj = comp == 0 ? j : j - 1;
      float term_dt = F2(dt, i, j) + F2(dt, bi, bj);
      float dt_diff = F2(dt, i, j) - F2(dt, bi, bj);
      float r0 = F3(rho, i, j, 0) - F3(rmean, i, j, 0);
      float rb0 = F3(rho, bi, bj, 0) - F3(rmean, bi, bj, 0);
      float val0 = c.k.half_g * (-F1(zz, 0)) * term_dt * (r0 - rb0);
      float mask = comp == 0 ? F2(dum, i, j) : F2(dvm, i, j);
      float area = comp == 0 ? (F2(dy, i, j) + F2(dy, bi, bj)) : (F2(dx, i, j) + F2(dx, bi, bj));
      float scale = 0.25f * term_dt * mask * area;
      float inc = 0.0f;
      if (k >= 1 && k < kbm1) {
        float rk = F3(rho, i, j, k) - F3(rmean, i, j, k);
        float rbk = F3(rho, bi, bj, k) - F3(rmean, bi, bj, k);
        float rkm = F3(rho, i, j, k - 1) - F3(rmean, i, j, k - 1);
        float rbkm = F3(rho, bi, bj, k - 1) - F3(rmean, bi, bj, k - 1);
        float zzk = F1(zz, k), zzkm = F1(zz, k - 1);
        float term1 = c.k.quarter_g * (zzkm - zzk) * term_dt * ((rk - rbk) + (rkm - rbkm));
        float term2 = c.k.quarter_g * (zzkm + zzk) * dt_diff * ((rk + rbk) - (rkm + rbkm));
        inc = term1 + term2;
      }
      double acc = seg_prefix((double)inc, 1, k);
      float out;
      if (k == 0) out = val0 * scale * ramp;
      else if (k < kbm1) out = (val0 + (float)acc) * scale * ramp;
      else out = 0.0f;
      dr[comp] = out;
    }
  }
  float aam = F3(aam, i, j, k);
  if (in && k < kbm1) {
    const float dxs = F2(dx, i, j), dys = F2(dy, i, j);
    float du_dx = (F3(u, i + 1, j, k) - F3(u, i, j, k)) / dxs;
    float dv_dy = (F3(v, i, j + 1, k) - F3(v, i, j, k)) / dys;
    float u_term = 0.25f * (F3(u, i, j + 1, k) + F3(u, i + 1, j + 1, k) - F3(u, i, j - 1, k) - F3(u, i + 1, j - 1, k)) / dys;
    float v_term = 0.25f * (F3(v, i + 1, j, k) + F3(v, i + 1, j + 1, k) - F3(v, i - 1, j, k) - F3(v, i - 1, j + 1, k)) / dxs;
    float mag;
    if (c.k.core == NPOM_CORE_EXPLICIT) {
      float cc = (u_term + v_term) * c.k.sqrt_half;
      mag = sqrtf(du_dx * du_dx + dv_dy * dv_dy + cc * cc);
    } else {
      float shr = u_term + v_term;
      mag = sqrtf(du_dx * du_dx + dv_dy * dv_dy + 0.5f * (shr * shr));
    }
    aam = c.k.horcon * dxs * dys * mag;
    if (c.k.core == NPOM_CORE_IMPLICIT && c.k.aam_min > 0.0f) aam = fmaxf_t(aam, c.k.aam_min);
  }
  const float dzk = F1(dz, k);
  float sx = seg_sum(F3(advx, i, j, k) * dzk, kbm1);
  float sy = seg_sum(F3(advy, i, j, k) * dzk, kbm1);
  float rx = seg_sum(dr[0] * dzk, kbm1);
  float ry = seg_sum(dr[1] * dzk, kbm1);
  float sa = seg_sum(aam * dzk, kbm1);
  if (!st) return;
  P3(drhox, i, j, k) = dr[0];
  P3(drhoy, i, j, k) = dr[1];
  if (in && k < kbm1) P3(aam, i, j, k) = aam;
  if (k == 0) {
    P2(adx2d, i, j) = sx;
    P2(ady2d, i, j) = sy;
    P2(drx2d, i, j) = rx;
    P2(dry2d, i, j) = ry;
    P2(aam2d, i, j) = sa;
  }
}

// ---------------------------------------------------------------------------
// B1: barotropic fix of u and v
// ---------------------------------------------------------------------------
__device__ __forceinline__ void lane_b1(const Ctx &c, int i, int j, int k, bool st) {
  const int kbm1 = KL - 1;
  const float dzk = F1(dz, k);
  float uk = F3(u, i, j, k), vk = F3(v, i, j, k);
  float su = seg_sum(uk * dzk, kbm1);
  float sv = seg_sum(vk * dzk, kbm1);
  if (!st || k >= kbm1) return;
  if (i >= 1) {
    float corr = (F2(utb, i, j) + F2(utf, i, j)) / ((F2(dt, i, j) + F2(dt, i - 1, j)) + 1e-20f);
    P3(u, i, j, k) = (uk - su) + corr;
  }
  if (j >= 1) {
    float corr = (F2(vtb, i, j) + F2(vtf, i, j)) / ((F2(dt, i, j) + F2(dt, i, j - 1)) + 1e-20f);
    P3(v, i, j, k) = (vk - sv) + corr;
  }
}

// ---------------------------------------------------------------------------
// B2A: VERTVL + bcond 5
// ---------------------------------------------------------------------------
__device__ __forceinline__ void lane_b2a(const Ctx &c, int i, int j, int k, bool st) {
  const int kbm1 = KL - 1;
  float w = F3(w, i, j, k);
  if (interior(c, i, j)) {
    float w0 = 0.5f * (F2(vfluxb, i, j) + F2(vfluxf, i, j));
    float area = F2(dx, i, j) * F2(dy, i, j);
    float eta_term = (F2(etf, i, j) - F2(etb, i, j)) / c.k.dti2;
    float inc = 0.0f;
    if (k < kbm1) {
      float div = vertvl_xflux(c, i + 1, j, k) - vertvl_xflux(c, i, j, k) + vertvl_yflux(c, i, j + 1, k) -
                  vertvl_yflux(c, i, j, k);
      inc = (div / area + eta_term) * F1(dz, k);
    }
    double acc = seg_prefix((double)inc, 0, k - 1);
    w = (k == 0) ? w0 : w0 + (float)acc;
  }
  const int kend = is_explicit(c) ? kbm1 : KL;
  if (k < kend) w = w * F2(fsm, i, j);
  if (st) P3(w, i, j, k) = w;
}

// ---------------------------------------------------------------------------
// B3: PROFQ
// ---------------------------------------------------------------------------
__device__ __forceinline__ void lane_b3(const Ctx &c, int i, int j, int k, bool st) {
  const int im = c.im, jm = c.jm, kb = KL, kbm1 = KL - 1;
  const float dti2 = c.k.dti2, umol2 = c.k.two_umol, grav = c.k.grav, kappa = c.k.kappa, small = c.k.small;
  const float b1 = 16.6f, e1 = 1.8f, e2 = 1.33f;
  const float dh = F2(h, i, j) + F2(etf, i, j);
  float A = 0.0f, C = 0.0f;
  if (k >= 1 && k < kbm1) {
    float den_a = F1(dzz, k - 1) * F1(dz, k) * dh * dh;
    float den_c = F1(dzz, k - 1) * F1(dz, k - 1) * dh * dh;
    float kqk = F3(kq, i, j, k);
    A = c.k.neg_dti2 * (F3(kq, i, j, k + 1) + kqk + umol2) * 0.5f / den_a;
    C = c.k.neg_dti2 * (F3(kq, i, j, k - 1) + kqk + umol2) * 0.5f / den_c;
  }
  float utau2 = 0.0f, l0 = 0.0f, uf_bottom = 0.0f;
  const bool sb_region = (i < im - 1) && (j < jm - 1);
  if (sb_region) {
    float us_ = 0.5f * (F2(wusurf, i, j) + F2(wusurf, i + 1, j));
    float vs_ = 0.5f * (F2(wvsurf, i, j) + F2(wvsurf, i, j + 1));
    utau2 = sqrtf(us_ * us_ + vs_ * vs_ + 1e-8f);
    l0 = c.k.surfl * utau2 / grav;
    float ub_ = 0.5f * (F2(wubot, i, j) + F2(wubot, i + 1, j));
    float vb_ = 0.5f * (F2(wvbot, i, j) + F2(wvbot, i, j + 1));
    uf_bottom = sqrtf(ub_ * ub_ + vb_ * vb_ + 1e-8f) * c.k.prof_const1;
  }
  float cc = 0.0f;
  if (k < kbm1) {
    float tp = F3(t, i, j, k) + c.k.tbias;
    float sp = F3(s, i, j, k) + c.k.sbias;
    float p = c.k.g_rhoref * (-F1(zz, k) * dh) * 1.0e-4f;
    float ccs = 1449.1f + 0.00821f * p + 4.55f * tp - 0.045f * (tp * tp) + 1.34f * (sp - 35.0f);
    if (fabsf(ccs) < 1e-6f) ccs = 1e-6f;
    float rad = (1.0f - 0.01642f * p / ccs) * (1.0f - 0.40f * p / (ccs * ccs));
    cc = ccs / sqrtf(fmaxf_t(rad, 1e-8f));
  }
  float cc_m = sh(cc, k > 0 ? k - 1 : 0);
  float boygr = 0.0f;
  if (k >= 1 && k < kbm1) {
    float term1 = grav * (F3(rho, i, j, k - 1) - F3(rho, i, j, k)) / (F1(dzz, k - 1) * dh);
    float term2 = c.k.g2x2 / (cc_m * cc_m + cc * cc);
    boygr = term1 + term2;
  }
  const float q2b_abs = fabsf(F3(q2b, i, j, k));
  float l = 0.0f;
  if (k >= 1 && k < kbm1) l = fabsf(F3(q2lb, i, j, k)) / (q2b_abs + 1e-20f);
  const float kl0 = kappa * l0;
  if (k < kbm1 && F1(z, k) > -0.5f) l = fmaxf_t(l, kl0);
  float gh = 0.0f;
  if (k >= 1 && k < kbm1) gh = fminf_t((l * l) * boygr / (q2b_abs + 1e-20f), 0.028f);
  if (k == 0) l = kl0;
  if (k == kb - 1) l = 0.0f;
  float kn = 0.0f;
  if (interior(c, i, j) && k >= 1 && k < kbm1) {
    float du = F3(u, i, j, k) - F3(u, i, j, k - 1) + F3(u, i + 1, j, k) - F3(u, i + 1, j, k - 1);
    float dv = F3(v, i, j, k) - F3(v, i, j, k - 1) + F3(v, i, j + 1, k) - F3(v, i, j + 1, k - 1);
    float den = F1(dzz, k - 1) * dh;
    den = den * den;
    float kmk = F3(km, i, j, k);
    float knk = kmk * 0.25f * 1.0f * (du * du + dv * dv) / den;
    kn = knk - 0.0f * kmk * boygr + F3(kh, i, j, k) * boygr;
  }
  const float dtef = sqrtf(q2b_abs + 1e-8f) * 1.0f / (b1 * l + small);
  // q2l wall-function factor of this level
  float dtef2 = 0.0f;
  if (k >= 1 && k < kbm1) {
    const float z0 = F1(z, 0), zb = F1(z, kb - 1), zk = F1(z, k);
    float wall;
    if (is_explicit(c)) wall = 1.0f / (fabsf(zk - z0) + 1e-20f) + 1.0f / (fabsf(zk - zb) + 1e-20f);
    else wall = 1.0f / (fabsf(zk - z0) + 1e-8f) + 1.0f / (fabsf(zk - zb) + 1e-8f);
    wall = wall * l / (dh * kappa);
    dtef2 = dtef * (1.0f + e2 * (wall * wall));
  }
  const float ufin = F3(uf, i, j, k), vfin = F3(vf, i, j, k);
  // forward sweeps (q2 and q2l together)
  float ee1 = 0.0f, gg1 = (k == 0 && sb_region) ? c.k.prof_gg0 * utau2 : 0.0f;
  float ee2 = 0.0f, gg2 = 0.0f;
#pragma unroll
  for (int s = 1; s < kbm1; ++s) {
    float pe1 = sh(ee1, s - 1), pg1 = sh(gg1, s - 1);
    float pe2 = sh(ee2, s - 1), pg2 = sh(gg2, s - 1);
    if (k == s) {
      float den = A + C * (1.0f - pe1) - (c.k.two_dti2 * dtef + 1.0f);
      ee1 = A / (den + 1e-20f);
      gg1 = (c.k.neg_two_dti2 * kn + C * pg1 - ufin) / (den + 1e-20f);
      float den2 = A + C * (1.0f - pe2) - (dti2 * dtef2 + 1.0f);
      ee2 = A / (den2 + 1e-20f);
      gg2 = (dti2 * (-kn * l * e1) + C * pg2 - vfin) / (den2 + 1e-20f);
    }
  }
  // back substitution
  float q2v = (k == kb - 1) ? uf_bottom : 0.0f;
  float q2lv = 0.0f;
#pragma unroll
  for (int s = kbm1 - 1; s >= 0; --s) {
    float n1 = sh(q2v, s + 1), n2 = sh(q2lv, s + 1);
    if (k == s) {
      q2v = ee1 * n1 + gg1;
      q2lv = ee2 * n2 + gg2;
    }
  }
  if (k >= 1 && k < kbm1) {
    if ((q2v <= small) || (q2lv <= small)) {
      q2v = is_explicit(c) ? small : q2v * 0.0f + small;
      q2lv = 0.1f * F2(dt, i, j) * small;
    }
  }
  const float coef4 = (float)(18.0 * 0.92 * 0.92 + 9.0 * 0.92 * 0.74);
  const float coef5 = (float)(9.0 * 0.92 * 0.74);
  const float coef1 = (float)(0.74 * (1.0 - 6.0 * 0.92 / 16.6));
  const float coef2 = (float)(3.0 * 0.74 * 10.1 + 18.0 * 0.92 * 0.74);
  const float coef3 = (float)(0.92 * (1.0 - 3.0 * 0.08 - 6.0 * 0.92 / 16.6));
  float shv = coef1 / ((1.0f - coef2 * gh) + 1e-20f);
  float smv = (coef3 + shv * coef4 * gh) / ((1.0f - coef5 * gh) + 1e-20f);
  float knf = l * sqrtf(fabsf(F3(q2, i, j, k)) + 1e-8f);
  float kq_ = (knf * 0.41f * shv + F3(kq, i, j, k)) * 0.5f;
  float km_ = (knf * smv + F3(km, i, j, k)) * 0.5f;
  float kh_ = (knf * shv + F3(kh, i, j, k)) * 0.5f;
  if (!st) return;
  P3(l, i, j, k) = l;
  P3(kq, i, j, k) = kq_;
  P3(km, i, j, k) = km_;
  P3(kh, i, j, k) = kh_;
  P3(uf, i, j, k) = q2v;
  P3(vf, i, j, k) = q2lv;
}

// ---------------------------------------------------------------------------
// B6: PROFT for T (uf) and S (vf), tps = h + etf, explicit bcond 4 edges
// ---------------------------------------------------------------------------
__device__ __forceinline__ float lane_proft(const Ctx &c, int k, float f, float khk, float kh_next, float wfsurf,
                                            float fsurf, int nbc, float dh, float swrad) {
  const int kbm1 = KL - 1, kbm2 = KL - 2;
  const float dti2 = c.k.dti2, umol = c.k.umol, neg_dti2 = -c.k.dti2;
  const float dh2 = dh * dh;
  float a = 0.0f, cv = 0.0f;
  if (k <= kbm1 - 2) a = (neg_dti2 * (kh_next + umol)) / (F1(dz, k) * F1(dzz, k) * dh2);
  if (k >= 1 && k < kbm1) cv = (neg_dti2 * (khk + umol)) / (F1(dz, k) * F1(dzz, k - 1) * dh2);
  float rad = 0.0f;
  if ((nbc == 2 || nbc == 4) && k < kbm1) {
    const float R[5] = {0.58f, 0.62f, 0.67f, 0.77f, 0.78f};
    const float AD1[5] = {0.35f, 0.60f, 1.00f, 1.50f, 1.40f};
    const float AD2[5] = {0.23f, 20.0f, 17.0f, 14.0f, 7.90f};
    const int ix = c.k.ntp - 1;
    float zt = F1(z, k) * dh;
    rad = swrad * (R[ix] * expf(zt / AD1[ix]) + (1.0f - R[ix]) * expf(zt / AD2[ix]));
  }
  const float rad_next = sh(rad, k < KL - 1 ? k + 1 : k);
  const float rad1 = sh(rad, 1);
  float ee = 0.0f, gg = 0.0f;
  if (k == 0) {
    if (nbc == 1) {
      float den = a - 1.0f;
      ee = a / den;
      gg = (neg_dti2 * wfsurf / (-F1(dz, 0) * dh) - f) / den;
    } else if (nbc == 2) {
      float den = a - 1.0f;
      ee = a / den;
      gg = (dti2 * (wfsurf + (rad - rad1)) / (F1(dz, 0) * dh) - f) / den;
    } else {
      ee = 0.0f;
      gg = fsurf;
    }
  }
#pragma unroll
  for (int s = 1; s < kbm2; ++s) {
    float pe = sh(ee, s - 1), pg = sh(gg, s - 1);
    if (k == s) {
      float den = a + cv * (1.0f - pe) - 1.0f;
      float inv = 1.0f / (den + 1e-20f);
      ee = a * inv;
      float rt = dti2 * (rad - rad_next) / (dh * F1(dz, k));
      gg = (cv * pg - f + rt) * inv;
    }
  }
  const int kbt = kbm1 - 1;
  float pe = sh(ee, kbt - 1), pg = sh(gg, kbt - 1);
  float out = f;
  if (k == kbt) {
    float rt = dti2 * (rad - rad_next) / (dh * F1(dz, kbt));
    float num = cv * pg - f + rt;
    float den = cv * (1.0f - pe) - 1.0f;
    out = num / (den + 1e-20f);
  }
#pragma unroll
  for (int s = kbm1 - 2; s >= 0; --s) {
    float nx = sh(out, s + 1);
    if (k == s) out = ee * nx + gg;
  }
  return out;
}

__device__ __forceinline__ void lane_b6(const Ctx &c, int i, int j, int k, bool st) {
  const float dh = F2(h, i, j) + F2(etf, i, j);
  const float khk = F3(kh, i, j, k);
  const float kh_next = (k + 1 < KL) ? F3(kh, i, j, k + 1) : 0.0f;
  const float swrad = F2(swrad, i, j);
  float tf = lane_proft(c, k, F3(uf, i, j, k), khk, kh_next, F2(wtsurf, i, j), F2(tsurf, i, j), c.k.nbct, dh, swrad);
  float sf = lane_proft(c, k, F3(vf, i, j, k), khk, kh_next, F2(wssurf, i, j), F2(ssurf, i, j), c.k.nbcs, dh, swrad);
  // explicit bcond 4 (upstream T/S at the edges) replaces levels
  // 0..kbm1-1 of an edge column; each lane evaluates its own level
  if (explicit_bc(c) && !c.k.obc_seamount && k < KL - 1 && (i == 0 || i == c.im - 1 || j == 0 || j == c.jm - 1)) {
    float ub, vb;
    if (bcond4_explicit_level(c, i, j, k, ub, vb)) {
      tf = ub;
      sf = vb;
    }
  }
  if (!st) return;
  P3(uf, i, j, k) = tf;
  P3(vf, i, j, k) = sf;
  if (k == 0) P2(tps, i, j) = dh;
}

// ---------------------------------------------------------------------------
// B8: ADVU+PROFU and ADVV+PROFV, explicit bcond 3 edges
// ---------------------------------------------------------------------------
__device__ __forceinline__ void lane_profuv(const Ctx &c, int comp, int i, int j, int k, float fin, float &out,
                                            float &wbot, float &tps) {
  const int kbm1 = KL - 1, kbm2 = KL - 2;
  out = fin;
  wbot = comp == 0 ? F2(wubot, i, j) : F2(wvbot, i, j);
  tps = 0.0f;
  if (i < 1 || j < 1) return;
  const int oi = comp == 0 ? i - 1 : i, oj = comp == 0 ? j : j - 1;
  const float dti2 = c.k.dti2;
  float dhf = 0.5f * (F2(h, i, j) + F2(etf, i, j) + F2(h, oi, oj) + F2(etf, oi, oj));
  float dh2 = dhf * dhf;
  float a = 0.0f, cv = 0.0f;
  if (k <= kbm1 - 2) {
    float kmf = 0.5f * (F3(km, i, j, k + 1) + F3(km, oi, oj, k + 1));
    a = (c.k.neg_dti2 * (kmf + c.k.umol)) / (F1(dz, k) * F1(dzz, k) * dh2);
  }
  if (k >= 1 && k < kbm1) {
    float kmf = 0.5f * (F3(km, i, j, k) + F3(km, oi, oj, k));
    cv = (c.k.neg_dti2 * (kmf + c.k.umol)) / (F1(dz, k) * F1(dzz, k - 1) * dh2);
  }
  float ee = 0.0f, gg = 0.0f;
  if (k == 0) {
    float den0 = a - 1.0f;
    ee = a / (den0 + 1e-20f);
    float wsurf = comp == 0 ? F2(wusurf, i, j) : F2(wvsurf, i, j);
    float term = c.k.neg_dti2 * wsurf / (-F1(dz, 0) * dhf);
    gg = (term - fin) / (den0 + 1e-20f);
  }
#pragma unroll
  for (int s = 1; s < kbm2; ++s) {
    float pe = sh(ee, s - 1), pg = sh(gg, s - 1);
    if (k == s) {
      float den = a + cv * (1.0f - pe) - 1.0f;
      float inv = 1.0f / (den + 1e-20f);
      ee = a * inv;
      gg = (cv * pg - fin) * inv;
    }
  }
  if (!interior(c, i, j)) return;
  const int kbt = kbm1 - 1;
  float cbc_avg, mag;
  // the coastal tide policy's step copy drops the 1e-8 of the bottom speed
  // (coastal_explicit_momentum.py:327,435)
  const float eps8 = c.k.obc_coastal ? 0.0f : 1e-8f;
  if (comp == 0) {
    cbc_avg = 0.5f * (F2(cbc, i, j) + F2(cbc, i - 1, j));
    float usq = F3(ub, i, j, kbt);
    usq = usq * usq;
    float vsum = F3(vb, i, j, kbt) + F3(vb, i, j + 1, kbt) + F3(vb, i - 1, j, kbt) + F3(vb, i - 1, j + 1, kbt);
    float va = 0.25f * vsum;
    mag = sqrtf(usq + va * va + eps8);
  } else {
    cbc_avg = 0.5f * (F2(cbc, i, j) + F2(cbc, i, j - 1));
    float vsq = F3(vb, i, j, kbt);
    vsq = vsq * vsq;
    float usum = F3(ub, i, j, kbt) + F3(ub, i + 1, j, kbt) + F3(ub, i, j - 1, kbt) + F3(ub, i + 1, j - 1, kbt);
    float ua = 0.25f * usum;
    mag = sqrtf(ua * ua + vsq + eps8);
  }
  tps = cbc_avg * mag;
  const float mask = comp == 0 ? F2(dum, i, j) : F2(dvm, i, j);
  float pe = sh(ee, kbt - 1), pg = sh(gg, kbt - 1);
  float nxt = 0.0f;
  if (k == kbt) {
    float fric = tps * dti2 / (-F1(dz, kbt) * dhf);
    float den = fric - 1.0f - (pe - 1.0f) * cv;
    float num = cv * pg - fin;
    nxt = num / (den + 1e-20f) * mask;
    out = nxt;
  }
#pragma unroll
  for (int s = kbt - 1; s >= 0; --s) {
    float nx = sh(out, s + 1);
    if (k == s) out = (ee * nx + gg) * mask;
  }
  float obot = sh(out, kbt);
  wbot = -tps * obot;
}

__device__ __forceinline__ void lane_bcond3_explicit(const Ctx &c, int i, int j, int k, float &uo, float &vo) {
  const int im = c.im, jm = c.jm, kbm1 = KL - 1;
  if (k >= kbm1) return;
  const float hmax = c.k.hmax;
  auto ga_of = [&](float hh) { return sqrtf(fmaxf_t(hh / hmax, 1e-8f)); };
  const int gf = c.k.obc_coastal ? NPOM_F_d : NPOM_F_h;  // coastal policy: total depth
  if (j >= 1 && j <= jm - 2) {
    if (i == im - 1) {
      float ga = ga_of(ld(c.F[gf] + NPOM_I2(c, im - 1, j)));
      float ui = 0.25f * F3(u, im - 2, j - 1, k) + 0.50f * F3(u, im - 2, j, k) + 0.25f * F3(u, im - 2, j + 1, k);
      float uo2 = 0.25f * F3(u, im - 1, j - 1, k) + 0.50f * F3(u, im - 1, j, k) + 0.25f * F3(u, im - 1, j + 1, k);
      uo = ga * ui + (1.0f - ga) * uo2;
      vo = 0.0f;
    }
    if (i == 1 || i == 0) {
      float ga = ga_of(ld(c.F[gf] + NPOM_I2(c, 0, j)));
      float ui = 0.25f * F3(u, 2, j - 1, k) + 0.50f * F3(u, 2, j, k) + 0.25f * F3(u, 2, j + 1, k);
      float uo2 = 0.25f * F3(u, 1, j - 1, k) + 0.50f * F3(u, 1, j, k) + 0.25f * F3(u, 1, j + 1, k);
      uo = ga * ui + (1.0f - ga) * uo2;
      if (i == 0) vo = 0.0f;
    }
  }
  if (i >= 1 && i <= im - 2) {
    if (j == jm - 1) {
      float ga = ga_of(ld(c.F[gf] + NPOM_I2(c, i, jm - 1)));
      float vi = 0.25f * F3(v, i - 1, jm - 2, k) + 0.50f * F3(v, i, jm - 2, k) + 0.25f * F3(v, i + 1, jm - 2, k);
      float vo2 = 0.25f * F3(v, i - 1, jm - 1, k) + 0.50f * F3(v, i, jm - 1, k) + 0.25f * F3(v, i + 1, jm - 1, k);
      vo = ga * vi + (1.0f - ga) * vo2;
      uo = 0.0f;
    }
    if (j == 1 || j == 0) {
      float ga = ga_of(ld(c.F[gf] + NPOM_I2(c, i, 0)));
      float vi = 0.25f * F3(v, i - 1, 2, k) + 0.50f * F3(v, i, 2, k) + 0.25f * F3(v, i + 1, 2, k);
      float vo2 = 0.25f * F3(v, i - 1, 1, k) + 0.50f * F3(v, i, 1, k) + 0.25f * F3(v, i + 1, 1, k);
      vo = ga * vi + (1.0f - ga) * vo2;
      if (j == 0) uo = 0.0f;
    }
  }
}

__device__ __forceinline__ void lane_b8(const Ctx &c, int i, int j, int k, bool st) {
  const bool inner = interior(c, i, j);
  float fu = (inner && k < KL - 1) ? advu_point(c, i, j, k) : 0.0f;
  float fv = (inner && k < KL - 1) ? advv_point(c, i, j, k) : 0.0f;
  float uo, vo, wub, wvb, tpsu, tpsv;
  lane_profuv(c, 0, i, j, k, fu, uo, wub, tpsu);
  lane_profuv(c, 1, i, j, k, fv, vo, wvb, tpsv);
  if (c.k.obc_jzb) jzb_bcond3_level(c, i, j, k, uo, vo);
  else if (explicit_bc(c) && !c.k.obc_seamount) lane_bcond3_explicit(c, i, j, k, uo, vo);
  if (!st) return;
  P3(uf, i, j, k) = uo;
  P3(vf, i, j, k) = vo;
  if (k == 0) {
    P2(wubot, i, j) = wub;
    P2(wvbot, i, j) = wvb;
    P2(tps, i, j) = tpsv;
  }
}

// ---------------------------------------------------------------------------
// B9: bcond 3 masks, internal velocity filter, shifts
// ---------------------------------------------------------------------------
__device__ __forceinline__ void lane_b9(const Ctx &c, int i, int j, int k, bool st) {
  const int im = c.im, jm = c.jm, kbm1 = KL - 1;
  if (c.do_internal) {
    const bool ring = (i == 0 || i == im - 1 || j == 0 || j == jm - 1);
    const float hs = c.k.half_smoth;
    const float dzk = F1(dz, k);
#pragma unroll
    for (int comp = 0; comp < 2; ++comp) {
      const float mask = comp == 0 ? F2(dum, i, j) : F2(dvm, i, j);
      float *fa = comp == 0 ? c.F[NPOM_F_u] : c.F[NPOM_F_v];
      float *fb = comp == 0 ? c.F[NPOM_F_ub] : c.F[NPOM_F_vb];
      float *ff = comp == 0 ? c.F[NPOM_F_uf] : c.F[NPOM_F_vf];
      const size_t o = NPOM_I3(c, i, j, k);
      float x = ff[o] * mask;
      if (!explicit_bc(c) && ring) x = 0.0f;
      const float cur = fa[o];
      const float term = x + fb[o] - 2.0f * cur;
      const float tps = seg_sum(term * dzk, kbm1);
      float filt = (k < kbm1) ? cur + hs * (term - tps) : cur;
      if (!is_explicit(c)) filt = filt * mask;
      if (st) {
        fb[o] = filt;
        fa[o] = x;
        ff[o] = x;
      }
    }
  }
  if (!st || k != 0) return;
  P2(egb, i, j) = F2(egf, i, j);
  P2(etb, i, j) = F2(et, i, j);
  float etf = F2(etf, i, j);
  P2(et, i, j) = etf;
  P2(dt, i, j) = F2(h, i, j) + etf;
  P2(utb, i, j) = F2(utf, i, j);
  P2(vtb, i, j) = F2(vtf, i, j);
  P2(vfluxb, i, j) = F2(vfluxf, i, j);
}

}  // namespace npom
