// npom_phases_int.cuh -- internal (3-D) mode shared by both cores:
// barotropic velocity fix, VERTVL, ADVQ, PROFQ (Mellor-Yamada 2.5), ADVT1,
// PROFT, DENS, ADVU/ADVV, PROFU/PROFV, the boundary conditions of each core
// and the Robert-Asselin filters (explicit/time_loop.py:437-696,
// implicit_p0_fixed/time_loop.py:393-668).
#pragma once

#include "npom_phases_ext.cuh"

namespace npom {

constexpr int KMAX = 64;  // largest kb the column bodies accept

NPOM_HD bool is_explicit(const Ctx &c) { return c.k.core == NPOM_CORE_EXPLICIT; }

// bcond 3-6 in the explicit core's form: the explicit core, and the
// semi-implicit core under a case policy -- the tide policies hand indices
// 3-6 to the explicit step copy's bcond (case_adapters/coastal_boundary.py:
// 29, jzb_boundary.py:142), the seamount policy applies its own
// (seamount_boundary.py:20-43)
NPOM_HD bool explicit_bc(const Ctx &c) { return is_explicit(c) || c.k.obc_coastal || c.k.obc_seamount; }

// ---------------------------------------------------------------------------
// B1 (column): u/v barotropic fix (explicit time_loop.py:440-477).
// ---------------------------------------------------------------------------
NPOM_HD void phase_b1_column(const Ctx &c, int i, int j) {
  const int kbm1 = c.kb - 1;
  if (i >= 1) {
    float tps = 0.0f;
    for (int k = 0; k < kbm1; ++k) tps += F3(u, i, j, k) * F1(dz, k);
    float corr = (F2(utb, i, j) + F2(utf, i, j)) / ((F2(dt, i, j) + F2(dt, i - 1, j)) + 1e-20f);
    for (int k = 0; k < kbm1; ++k) P3(u, i, j, k) = (F3(u, i, j, k) - tps) + corr;
  }
  if (j >= 1) {
    float tps = 0.0f;
    for (int k = 0; k < kbm1; ++k) tps += F3(v, i, j, k) * F1(dz, k);
    float corr = (F2(vtb, i, j) + F2(vtf, i, j)) / ((F2(dt, i, j) + F2(dt, i, j - 1)) + 1e-20f);
    for (int k = 0; k < kbm1; ++k) P3(v, i, j, k) = (F3(v, i, j, k) - tps) + corr;
  }
}

// ---------------------------------------------------------------------------
// B2a (column): VERTVL (baroclinic.py:930-1040) then bcond 5.
// ---------------------------------------------------------------------------
NPOM_HD float vertvl_xflux(const Ctx &c, int i, int j, int k) {
  return 0.25f * (F2(dy, i, j) + F2(dy, i - 1, j)) * (F2(dt, i, j) + F2(dt, i - 1, j)) * F3(u, i, j, k);
}
NPOM_HD float vertvl_yflux(const Ctx &c, int i, int j, int k) {
  return 0.25f * (F2(dx, i, j) + F2(dx, i, j - 1)) * (F2(dt, i, j) + F2(dt, i, j - 1)) * F3(v, i, j, k);
}

NPOM_HD void phase_b2a_column(const Ctx &c, int i, int j) {
  const int kb = c.kb, kbm1 = kb - 1;
  const float fsm = F2(fsm, i, j);
  if (interior(c, i, j)) {
    float w0 = 0.5f * (F2(vfluxb, i, j) + F2(vfluxf, i, j));
    float area = F2(dx, i, j) * F2(dy, i, j);
    float eta_term = (F2(etf, i, j) - F2(etb, i, j)) / c.k.dti2;
    P3(w, i, j, 0) = w0;
    double acc = 0.0;
    for (int k = 0; k < kbm1; ++k) {
      float div = vertvl_xflux(c, i + 1, j, k) - vertvl_xflux(c, i, j, k) + vertvl_yflux(c, i, j + 1, k) -
                  vertvl_yflux(c, i, j, k);
      float inc = (div / area + eta_term) * F1(dz, k);
      acc += (double)inc;
      P3(w, i, j, k + 1) = w0 + (float)acc;
    }
  }
  // bcond 5: explicit masks levels < kb-1 (baroclinic.py:849-851); the
  // closed basin masks every level (closed_basin.py:300-302)
  const int kend = is_explicit(c) ? kbm1 : kb;
  for (int k = 0; k < kend; ++k) P3(w, i, j, k) = F3(w, i, j, k) * fsm;
}

// ---------------------------------------------------------------------------
// B2b (point): ADVQ for q2 and q2l (tracers.py:14-156) -> uf, vf.
// ---------------------------------------------------------------------------
NPOM_HD float advq_xflux(const Ctx &c, const float *q, const float *qb, int i, int j, int k) {
  // i >= 1, j >= 1, 1 <= k <= kbm1-1
  const size_t o = NPOM_I3(c, i, j, k), om = NPOM_I3(c, i - 1, j, k);
  const size_t stride_k = 1;
  float xf = 0.125f * (ld(q + o) + ld(q + om)) * (F2(dt, i, j) + F2(dt, i - 1, j)) *
             (F3(u, i, j, k) + F3(u, i, j, k - 1));
  float aam_sum = F3(aam, i, j, k) + F3(aam, i - 1, j, k) + F3(aam, i, j, k - 1) + F3(aam, i - 1, j, k - 1);
  xf -= 0.25f * aam_sum * (F2(h, i, j) + F2(h, i - 1, j)) * (ld(qb + o) - ld(qb + om)) * F2(dum, i, j) /
        (F2(dx, i, j) + F2(dx, i - 1, j));
  xf *= 0.5f * (F2(dy, i, j) + F2(dy, i - 1, j));
  (void)stride_k;
  return xf;
}
NPOM_HD float advq_yflux(const Ctx &c, const float *q, const float *qb, int i, int j, int k) {
  const size_t o = NPOM_I3(c, i, j, k), om = NPOM_I3(c, i, j - 1, k);
  float yf = 0.125f * (ld(q + o) + ld(q + om)) * (F2(dt, i, j) + F2(dt, i, j - 1)) *
             (F3(v, i, j, k) + F3(v, i, j, k - 1));
  float aam_sum = F3(aam, i, j, k) + F3(aam, i, j - 1, k) + F3(aam, i, j, k - 1) + F3(aam, i, j - 1, k - 1);
  yf -= 0.25f * aam_sum * (F2(h, i, j) + F2(h, i, j - 1)) * (ld(qb + o) - ld(qb + om)) * F2(dvm, i, j) /
        (F2(dy, i, j) + F2(dy, i, j - 1));
  yf *= 0.5f * (F2(dx, i, j) + F2(dx, i, j - 1));
  return yf;
}

NPOM_HD float advq_point(const Ctx &c, const float *q, const float *qb, int i, int j, int k) {
  const int kbm1 = c.kb - 1;
  if (!interior(c, i, j) || k < 1 || k > kbm1 - 1) return 0.0f;
  float art = F2(art, i, j);
  float vert = (F3(w, i, j, k - 1) * ld(q + NPOM_I3(c, i, j, k - 1)) - F3(w, i, j, k + 1) * ld(q + NPOM_I3(c, i, j, k + 1))) *
               art / (F1(dz, k) + F1(dz, k - 1));
  float horiz = advq_xflux(c, q, qb, i + 1, j, k) - advq_xflux(c, q, qb, i, j, k) + advq_yflux(c, q, qb, i, j + 1, k) -
                advq_yflux(c, q, qb, i, j, k);
  float qf = vert + horiz;
  float tb = (F2(h, i, j) + F2(etb, i, j)) * art;
  float tf = (F2(h, i, j) + F2(etf, i, j)) * art;
  return (tb * ld(qb + NPOM_I3(c, i, j, k)) - c.k.dti2 * qf) / (tf + 1e-20f);
}

NPOM_HD void phase_b2b_point(const Ctx &c, int i, int j, int k) {
  P3(uf, i, j, k) = advq_point(c, c.F[NPOM_F_q2], c.F[NPOM_F_q2b], i, j, k);
  P3(vf, i, j, k) = advq_point(c, c.F[NPOM_F_q2l], c.F[NPOM_F_q2lb], i, j, k);
}

// ---------------------------------------------------------------------------
// B3 (column): PROFQ (tracers.py:158-431; implicit epsilon forms
// implicit_p0_fixed/tracers.py:156-430).  Writes l, kq and the raw km/kh
// (edge copies follow in B4), and the q2/q2l forecasts into uf/vf.
// ---------------------------------------------------------------------------
NPOM_HD void phase_b3_pom08_column(const Ctx &c, int i, int j);

NPOM_HD void phase_b3_column(const Ctx &c, int i, int j) {
  if (c.k.profq_pom08) {
    phase_b3_pom08_column(c, i, j);
    return;
  }
  const int im = c.im, jm = c.jm, kb = c.kb, kbm1 = kb - 1;
  const float dti2 = c.k.dti2, umol2 = c.k.two_umol, grav = c.k.grav, kappa = c.k.kappa;
  const float small = c.k.small;
  const float a1 = 0.92f, b1 = 16.6f, a2 = 0.74f, b2 = 10.1f, c1 = 0.08f;
  (void)a1; (void)a2; (void)b2; (void)c1;
  const float e1 = 1.8f, e2 = 1.33f;
  float A[KMAX], C[KMAX], dtef[KMAX], kn[KMAX], gh[KMAX], l[KMAX], cc[KMAX], ee[KMAX], gg[KMAX];
  const float dh = F2(h, i, j) + F2(etf, i, j);
  for (int k = 0; k < kb; ++k) {
    A[k] = 0.0f;
    C[k] = 0.0f;
  }
  for (int k = 1; k < kbm1; ++k) {
    float den_a = F1(dzz, k - 1) * F1(dz, k) * dh * dh;
    float den_c = F1(dzz, k - 1) * F1(dz, k - 1) * dh * dh;
    A[k] = c.k.neg_dti2 * (F3(kq, i, j, k + 1) + F3(kq, i, j, k) + umol2) * 0.5f / den_a;
    C[k] = c.k.neg_dti2 * (F3(kq, i, j, k - 1) + F3(kq, i, j, k) + umol2) * 0.5f / den_c;
  }
  // surface / bottom values on [0, im-1) x [0, jm-1)
  float utau2 = 0.0f, l0 = 0.0f, uf_bottom = 0.0f;
  bool sb_region = (i < im - 1) && (j < jm - 1);
  if (sb_region) {
    float us_ = 0.5f * (F2(wusurf, i, j) + F2(wusurf, i + 1, j));
    float vs_ = 0.5f * (F2(wvsurf, i, j) + F2(wvsurf, i, j + 1));
    utau2 = sqrtf(us_ * us_ + vs_ * vs_ + 1e-8f);
    l0 = c.k.surfl * utau2 / grav;
    float ub_ = 0.5f * (F2(wubot, i, j) + F2(wubot, i + 1, j));
    float vb_ = 0.5f * (F2(wvbot, i, j) + F2(wvbot, i, j + 1));
    uf_bottom = sqrtf(ub_ * ub_ + vb_ * vb_ + 1e-8f) * c.k.prof_const1;
  }
  // buoyancy (sound speed from the pressure-corrected EOS)
  for (int k = 0; k < kbm1; ++k) {
    float tp = F3(t, i, j, k) + c.k.tbias;
    float sp = F3(s, i, j, k) + c.k.sbias;
    float p = c.k.g_rhoref * (-F1(zz, k) * dh) * 1.0e-4f;
    float ccs = 1449.1f + 0.00821f * p + 4.55f * tp - 0.045f * (tp * tp) + 1.34f * (sp - 35.0f);
    if (fabsf(ccs) < 1e-6f) ccs = 1e-6f;
    float rad = (1.0f - 0.01642f * p / ccs) * (1.0f - 0.40f * p / (ccs * ccs));
    cc[k] = ccs / sqrtf(fmaxf_t(rad, 1e-8f));
  }
  float boygr[KMAX];
  boygr[0] = 0.0f;
  for (int k = 1; k < kb; ++k) boygr[k] = 0.0f;
  for (int k = 1; k < kbm1; ++k) {
    float term1 = grav * (F3(rho, i, j, k - 1) - F3(rho, i, j, k)) / (F1(dzz, k - 1) * dh);
    float term2 = c.k.g2x2 / (cc[k - 1] * cc[k - 1] + cc[k] * cc[k]);
    boygr[k] = term1 + term2;
  }
  // length scale and gh
  for (int k = 0; k < kb; ++k) l[k] = 0.0f;
  for (int k = 1; k < kbm1; ++k) l[k] = fabsf(F3(q2lb, i, j, k)) / (fabsf(F3(q2b, i, j, k)) + 1e-20f);
  const float kl0 = kappa * l0;
  for (int k = 0; k < kbm1; ++k)
    if (F1(z, k) > -0.5f) l[k] = fmaxf_t(l[k], kl0);
  for (int k = 0; k < kb; ++k) gh[k] = 0.0f;
  for (int k = 1; k < kbm1; ++k) {
    float lk = l[k];
    gh[k] = fminf_t((lk * lk) * boygr[k] / (fabsf(F3(q2b, i, j, k)) + 1e-20f), 0.028f);
  }
  l[0] = kl0;
  l[kb - 1] = 0.0f;
  gh[0] = 0.0f;
  gh[kb - 1] = 0.0f;
  // shear production (interior only)
  for (int k = 0; k < kb; ++k) kn[k] = 0.0f;
  if (interior(c, i, j)) {
    for (int k = 1; k < kbm1; ++k) {
      float du = F3(u, i, j, k) - F3(u, i, j, k - 1) + F3(u, i + 1, j, k) - F3(u, i + 1, j, k - 1);
      float dv = F3(v, i, j, k) - F3(v, i, j, k - 1) + F3(v, i, j + 1, k) - F3(v, i, j + 1, k - 1);
      float den = F1(dzz, k - 1) * dh;
      den = den * den;
      float kmk = F3(km, i, j, k);
      float knk = kmk * 0.25f * 1.0f * (du * du + dv * dv) / den;
      knk = knk - 0.0f * kmk * boygr[k] + F3(kh, i, j, k) * boygr[k];
      kn[k] = knk;
    }
  }
  for (int k = 0; k < kb; ++k) dtef[k] = sqrtf(fabsf(F3(q2b, i, j, k)) + 1e-8f) * 1.0f / (b1 * l[k] + small);

  // q2 sweep
  float uf_out[KMAX], vf_out[KMAX];
  ee[0] = 0.0f;
  gg[0] = sb_region ? c.k.prof_gg0 * utau2 : 0.0f;
  for (int k = 1; k < kbm1; ++k) {
    float den = A[k] + C[k] * (1.0f - ee[k - 1]) - (c.k.two_dti2 * dtef[k] + 1.0f);
    ee[k] = A[k] / (den + 1e-20f);
    gg[k] = (c.k.neg_two_dti2 * kn[k] + C[k] * gg[k - 1] - F3(uf, i, j, k)) / (den + 1e-20f);
  }
  uf_out[kb - 1] = uf_bottom;
  for (int k = kbm1 - 1; k >= 0; --k) uf_out[k] = ee[k] * uf_out[k + 1] + gg[k];
  // q2l sweep
  const float z0 = F1(z, 0), zb = F1(z, kb - 1);
  ee[0] = 0.0f;
  gg[0] = 0.0f;
  for (int k = 1; k < kbm1; ++k) {
    float zk = F1(z, k);
    float wall;
    if (is_explicit(c)) {
      wall = 1.0f / (fabsf(zk - z0) + 1e-20f) + 1.0f / (fabsf(zk - zb) + 1e-20f);
    } else {
      wall = 1.0f / (fabsf(zk - z0) + 1e-8f) + 1.0f / (fabsf(zk - zb) + 1e-8f);
    }
    wall = wall * l[k] / (dh * kappa);
    float dtefk = dtef[k] * (1.0f + e2 * (wall * wall));
    float den = A[k] + C[k] * (1.0f - ee[k - 1]) - (dti2 * dtefk + 1.0f);
    ee[k] = A[k] / (den + 1e-20f);
    gg[k] = (dti2 * (-kn[k] * l[k] * e1) + C[k] * gg[k - 1] - F3(vf, i, j, k)) / (den + 1e-20f);
  }
  vf_out[kb - 1] = 0.0f;
  for (int k = kbm1 - 1; k >= 0; --k) vf_out[k] = ee[k] * vf_out[k + 1] + gg[k];
  // clipping
  const float dtij = F2(dt, i, j);
  for (int k = 1; k < kbm1; ++k) {
    bool m = (uf_out[k] <= small) || (vf_out[k] <= small);
    if (m) {
      uf_out[k] = is_explicit(c) ? small : uf_out[k] * 0.0f + small;
      vf_out[k] = 0.1f * dtij * small;
    }
  }
  // stability functions and mixing coefficients (raw; edges in B4)
  const float coef4 = (float)(18.0 * 0.92 * 0.92 + 9.0 * 0.92 * 0.74);
  const float coef5 = (float)(9.0 * 0.92 * 0.74);
  const float coef1 = (float)(0.74 * (1.0 - 6.0 * 0.92 / 16.6));
  const float coef2 = (float)(3.0 * 0.74 * 10.1 + 18.0 * 0.92 * 0.74);
  const float coef3 = (float)(0.92 * (1.0 - 3.0 * 0.08 - 6.0 * 0.92 / 16.6));
  for (int k = 0; k < kb; ++k) {
    float sh = coef1 / ((1.0f - coef2 * gh[k]) + 1e-20f);
    float sm = (coef3 + sh * coef4 * gh[k]) / ((1.0f - coef5 * gh[k]) + 1e-20f);
    float knf = l[k] * sqrtf(fabsf(F3(q2, i, j, k)) + 1e-8f);
    float kq_ = (knf * 0.41f * sh + F3(kq, i, j, k)) * 0.5f;
    float km_ = (knf * sm + F3(km, i, j, k)) * 0.5f;
    float kh_ = (knf * sh + F3(kh, i, j, k)) * 0.5f;
    P3(l, i, j, k) = l[k];
    P3(kq, i, j, k) = kq_;
    P3(km, i, j, k) = km_;
    P3(kh, i, j, k) = kh_;
    P3(uf, i, j, k) = uf_out[k];
    P3(vf, i, j, k) = vf_out[k];
  }
}

// ---------------------------------------------------------------------------
// B3 in the POM08-WAD form of the reference's case policies
// (cores/case_adapters/fortran_compat.py:26-147, after pom08.f with nwad=0):
// sound speed from the fixed reference pressure of (-zz * max(h, 0)),
// buoyancy over h + et, exact stress norms and square roots (no epsilon),
// |q2b| and |q2lb| on the interior levels (written back: the time loop keeps
// them as q2b/q2lb), the q2 sweep with reciprocal pivots, the q2l sweep with
// Dirichlet values on the second and the penultimate level, |q2| and |q2l|
// forecasts instead of clipping, kn = (kappa zsh + l) sqrt|q2| and
// kq = (0.20 kn + kq) / 2.  km/kh edges follow in B4 (north/south first).
// ---------------------------------------------------------------------------
NPOM_HD void phase_b3_pom08_column(const Ctx &c, int i, int j) {
  const int im = c.im, jm = c.jm, kb = c.kb, kbm1 = kb - 1;
  const float dti2 = c.k.dti2, umol2 = c.k.two_umol, grav = c.k.grav, kappa = c.k.kappa;
  const float small = c.k.small;
  float A[KMAX], C[KMAX], diss[KMAX], prod[KMAX], gh[KMAX], l[KMAX], snd[KMAX], boy[KMAX];
  float qb[KMAX], ee[KMAX], gg[KMAX], usol[KMAX], vsol[KMAX];
  const float dh = F2(h, i, j) + F2(etf, i, j);
  for (int k = 0; k < kb; ++k) {
    A[k] = 0.0f;
    C[k] = 0.0f;
  }
  for (int k = 1; k < kbm1; ++k) {
    float den_a = F1(dzz, k - 1) * F1(dz, k) * dh * dh;
    float den_c = F1(dzz, k - 1) * F1(dz, k - 1) * dh * dh;
    A[k] = c.k.neg_dti2 * (F3(kq, i, j, k + 1) + F3(kq, i, j, k) + umol2) * 0.5f / den_a;
    C[k] = c.k.neg_dti2 * (F3(kq, i, j, k - 1) + F3(kq, i, j, k) + umol2) * 0.5f / den_c;
  }
  // stresses on [0, im-1) x [0, jm-1) (fortran_compat.py:42-53)
  const bool sb = (i < im - 1) && (j < jm - 1);
  float l0 = 0.0f, surface_q = 0.0f, bottom = F3(uf, i, j, kb - 1);
  if (sb) {
    float us_ = 0.5f * (F2(wusurf, i, j) + F2(wusurf, i + 1, j));
    float vs_ = 0.5f * (F2(wvsurf, i, j) + F2(wvsurf, i, j + 1));
    float ub_ = 0.5f * (F2(wubot, i, j) + F2(wubot, i + 1, j));
    float vb_ = 0.5f * (F2(wvbot, i, j) + F2(wvbot, i, j + 1));
    float utau2 = sqrtf(us_ * us_ + vs_ * vs_);
    float btau2 = sqrtf(ub_ * ub_ + vb_ * vb_);
    l0 = c.k.surfl * utau2 / grav;
    surface_q = c.k.prof_gg0 * utau2;
    bottom = btau2 * c.k.prof_const1;
  }
  // sound speed from the fixed reference pressure (:56-60)
  const float hpos = fmaxf_t(F2(h, i, j), 0.0f);
  for (int k = 0; k < kbm1; ++k) {
    float pd = c.k.g_rhoref * (-F1(zz, k) * hpos);
    pd = pd * 1.0e-5f;
    float p = pd * 10.0f;
    float tp = F3(t, i, j, k) + c.k.tbias;
    float sp = F3(s, i, j, k) + c.k.sbias;
    float snd0 = 1449.1f + 0.00821f * p + 4.55f * tp - 0.045f * (tp * tp) + 1.34f * (sp - 35.0f);
    snd[k] = snd0 / sqrtf((1.0f - 0.01642f * p / snd0) * (1.0f - 0.40f * p / (snd0 * snd0)));
  }
  for (int k = 0; k < kb; ++k) {
    float q = F3(q2b, i, j, k), ql = F3(q2lb, i, j, k);
    if (k >= 1 && k < kbm1) {
      q = fabsf(q);
      ql = fabsf(ql);
      P3(q2b, i, j, k) = q;
      P3(q2lb, i, j, k) = ql;
    }
    qb[k] = q;
    if (k >= 1 && k < kbm1) l[k] = fabsf(ql / q);
  }
  // buoyancy, length scale, stability (:68-84)
  const float ddep = F2(h, i, j) + F2(et, i, j);
  const float kl0 = kappa * l0;
  for (int k = 0; k < kb; ++k) {
    boy[k] = 0.0f;
    gh[k] = 0.0f;
  }
  l[0] = kl0;
  l[kb - 1] = 0.0f;
  for (int k = 1; k < kbm1; ++k) {
    float b = grav * (F3(rho, i, j, k - 1) - F3(rho, i, j, k)) / (F1(dzz, k - 1) * ddep);
    b = b + c.k.g2x2 / (snd[k - 1] * snd[k - 1] + snd[k] * snd[k]);
    float ll = l[k];
    if (F1(z, k) > -0.5f) ll = fmaxf_t(ll, kl0);
    boy[k] = b;
    l[k] = ll;
    gh[k] = fminf_t((ll * ll) * b / qb[k], 0.028f);
  }
  // production on the interior (:86-94)
  for (int k = 0; k < kb; ++k) prod[k] = 0.0f;
  if (interior(c, i, j)) {
    for (int k = 1; k < kbm1; ++k) {
      float du = F3(u, i, j, k) - F3(u, i, j, k - 1) + F3(u, i + 1, j, k) - F3(u, i + 1, j, k - 1);
      float dv = F3(v, i, j, k) - F3(v, i, j, k - 1) + F3(v, i, j + 1, k) - F3(v, i, j + 1, k - 1);
      float den = F1(dzz, k - 1) * dh;
      den = den * den;
      float pr = F3(km, i, j, k) * 0.25f * (du * du + dv * dv) / den;
      prod[k] = pr + F3(kh, i, j, k) * boy[k];
    }
  }
  for (int k = 0; k < kb; ++k) diss[k] = sqrtf(fabsf(qb[k])) / (16.6f * l[k] + small);
  // q2: the sweep with reciprocal pivots (:97-105)
  ee[0] = 0.0f;
  gg[0] = surface_q;
  for (int k = 1; k < kbm1; ++k) {
    float inv = 1.0f / (A[k] + C[k] * (1.0f - ee[k - 1]) - (c.k.two_dti2 * diss[k] + 1.0f));
    ee[k] = A[k] * inv;
    gg[k] = (c.k.neg_two_dti2 * prod[k] + C[k] * gg[k - 1] - F3(uf, i, j, k)) * inv;
  }
  usol[kb - 1] = bottom;
  for (int k = kbm1 - 1; k >= 0; --k) usol[k] = ee[k] * usol[k + 1] + gg[k];
  // q2l: Dirichlet values on the second and the penultimate level (:107-130)
  const float z0 = F1(z, 0), zb = F1(z, kb - 1);
  const float q21 = F3(q2, i, j, 1), q2p = F3(q2, i, j, kbm1 - 1);
  ee[0] = 0.0f;
  gg[0] = 0.0f;
  ee[1] = 0.0f;
  gg[1] = ((-kappa) * F1(z, 1)) * dh * q21;
  for (int k = 2; k < kbm1; ++k) {
    float zk = F1(z, k);
    float wall = (1.0f / fabsf(zk - z0) + 1.0f / fabsf(zk - zb)) * l[k] / (dh * kappa);
    float ds = diss[k] * (1.0f + 1.33f * (wall * wall));
    float inv = 1.0f / (A[k] + C[k] * (1.0f - ee[k - 1]) - (dti2 * ds + 1.0f));
    ee[k] = A[k] * inv;
    float rhs = (k == kbm1 - 1) ? (kappa * (1.0f + F1(z, kbm1 - 1))) * dh * q2p : F3(vf, i, j, k);
    gg[k] = (dti2 * (-prod[k] * l[k] * 1.8f) + C[k] * gg[k - 1] - rhs) * inv;
  }
  vsol[0] = 0.0f;
  vsol[kb - 1] = 0.0f;
  for (int k = kbm1 - 1; k >= 1; --k) vsol[k] = ee[k] * vsol[k + 1] + gg[k];
  for (int k = 1; k < kbm1; ++k) {
    usol[k] = fabsf(usol[k]);
    vsol[k] = fabsf(vsol[k]);
  }
  // stability functions and mixing (:134-144); km/kh edges in B4
  const float coef4 = (float)(18.0 * 0.92 * 0.92 + 9.0 * 0.92 * 0.74);
  const float coef5 = (float)(9.0 * 0.92 * 0.74);
  const float coef1 = (float)(0.74 * (1.0 - 6.0 * 0.92 / 16.6));
  const float coef2 = (float)(3.0 * 0.74 * 10.1 + 18.0 * 0.92 * 0.74);
  const float coef3 = (float)(0.92 * (1.0 - 3.0 * 0.08 - 6.0 * 0.92 / 16.6));
  for (int k = 0; k < kb; ++k) {
    float sh = coef1 / (1.0f - coef2 * gh[k]);
    float sm = (coef3 + sh * coef4 * gh[k]) / (1.0f - coef5 * gh[k]);
    float kn = (c.k.kappa_zsh + l[k]) * sqrtf(fabsf(F3(q2, i, j, k)));
    P3(l, i, j, k) = l[k];
    P3(kq, i, j, k) = (kn * 0.20f + F3(kq, i, j, k)) * 0.5f;
    P3(km, i, j, k) = (kn * sm + F3(km, i, j, k)) * 0.5f;
    P3(kh, i, j, k) = (kn * sh + F3(kh, i, j, k)) * 0.5f;
    P3(uf, i, j, k) = usol[k];
    P3(vf, i, j, k) = vsol[k];
  }
}

// ---------------------------------------------------------------------------
// B4 (edge point): km/kh edge copies of PROFQ (tracers.py:425-429) and, for
// the explicit core, bcond 6 upstream values of the q2/q2l forecasts
// (baroclinic.py:856-919).  Runs over every (i, j, k); non-edge points exit.
// ---------------------------------------------------------------------------
NPOM_HD void phase_b4_point(const Ctx &c, int i, int j, int k) {
  const int im = c.im, jm = c.jm;
  bool edge = (i == 0 || i == im - 1 || j == 0 || j == jm - 1);
  if (!edge) return;
  // raw value source after "rows then columns" copies
  for (int comp = 0; comp < 2; ++comp) {
    float *arr = comp == 0 ? c.F[NPOM_F_km] : c.F[NPOM_F_kh];
    float val;
    if (j == 0 || j == jm - 1) {
      int sj = (j == 0) ? 1 : jm - 2;
      // column pass copies from the row-pass result at (i, sj)
      // corners: the production operator copies along i first (the source
      // row's own mask, fsm(i, sj)); the POM08-WAD form copies along j first
      // (fortran_compat.py:19-24: the source's mask at the corner row, fsm(si, j))
      float src;
      const bool jfirst = c.k.profq_pom08 != 0;
      if (i == 0) src = ld(arr + NPOM_I3(c, 1, sj, k)) * (jfirst ? F2(fsm, 1, j) : F2(fsm, 0, sj));
      else if (i == im - 1) src = ld(arr + NPOM_I3(c, im - 2, sj, k)) * (jfirst ? F2(fsm, im - 2, j) : F2(fsm, im - 1, sj));
      else src = ld(arr + NPOM_I3(c, i, sj, k));
      val = src * F2(fsm, i, j);
    } else {
      int si = (i == 0) ? 1 : im - 2;
      val = ld(arr + NPOM_I3(c, si, j, k)) * F2(fsm, i, j);
    }
    // written to uf/vf scratch first? no: B4 writes into a side buffer is
    // unnecessary because sources are never edges (si, sj are interior rows
    // /columns, and the corner sources are edge-free by construction).
    arr[NPOM_I3(c, i, j, k)] = val;
  }
  if (!explicit_bc(c)) return;
  if (c.k.obc_seamount) {
    // the seamount policy's bcond 6 (seamount_boundary.py:40-42): 1e-10 on
    // the east and west edges (B5 then applies uf * fsm + 1e-10)
    if (i == 0 || i == im - 1) {
      P3(uf, i, j, k) = 1e-10f;
      P3(vf, i, j, k) = 1e-10f;
    }
    return;
  }
  // explicit bcond 6 on the edges (east, west, north, south order)
  const float dti = c.k.dti, small = c.k.small;
  float ufv = F3(uf, i, j, k), vfv = F3(vf, i, j, k);
  if (i == im - 1) {
    float u1 = 2.0f * F3(u, im - 1, j, k) * dti / (F2(dx, im - 1, j) + F2(dx, im - 2, j));
    float q = F3(q2, im - 1, j, k), ql = F3(q2l, im - 1, j, k);
    if (u1 <= 0.0f) {
      ufv = q - u1 * (small - q);
      vfv = ql - u1 * (small - ql);
    } else {
      ufv = q - u1 * (q - F3(q2, im - 2, j, k));
      vfv = ql - u1 * (ql - F3(q2l, im - 2, j, k));
    }
  }
  if (i == 0) {
    float u1 = 2.0f * F3(u, 1, j, k) * dti / (F2(dx, 0, j) + F2(dx, 1, j));
    float q = F3(q2, 0, j, k), ql = F3(q2l, 0, j, k);
    if (u1 >= 0.0f) {
      ufv = q - u1 * (q - small);
      vfv = ql - u1 * (ql - small);
    } else {
      ufv = q - u1 * (F3(q2, 1, j, k) - q);
      vfv = ql - u1 * (F3(q2l, 1, j, k) - ql);
    }
  }
  if (j == jm - 1) {
    float u1 = 2.0f * F3(v, i, jm - 1, k) * dti / (F2(dy, i, jm - 1) + F2(dy, i, jm - 2));
    float q = F3(q2, i, jm - 1, k), ql = F3(q2l, i, jm - 1, k);
    if (u1 <= 0.0f) {
      ufv = q - u1 * (small - q);
      vfv = ql - u1 * (small - ql);
    } else {
      ufv = q - u1 * (q - F3(q2, i, jm - 2, k));
      vfv = ql - u1 * (ql - F3(q2l, i, jm - 2, k));
    }
  }
  if (j == 0) {
    float u1 = 2.0f * F3(v, i, 1, k) * dti / (F2(dy, i, 0) + F2(dy, i, 1));
    float q = F3(q2, i, 0, k), ql = F3(q2l, i, 0, k);
    if (u1 >= 0.0f) {
      ufv = q - u1 * (q - small);
      vfv = ql - u1 * (ql - small);
    } else {
      ufv = q - u1 * (F3(q2, i, 1, k) - q);
      vfv = ql - u1 * (F3(q2l, i, 1, k) - ql);
    }
  }
  P3(uf, i, j, k) = ufv;
  P3(vf, i, j, k) = vfv;
}

// ---------------------------------------------------------------------------
// B5 (point): bcond 6 mask, turbulence Robert-Asselin filter and shift
// (time_loop.py:521-540), optional mixing clamp, then ADVT1 for T and S
// (tracers.py:433-569) into uf/vf with the ghost-level copies of t/tb/s/sb.
// ---------------------------------------------------------------------------
// ADVT1 face fluxes of field f (tracers.py:433-569): x-face at (ii, j) for
// ii >= 1 and y-face at (i, jj) for jj >= 1, level k < kb-1
NPOM_HD float advt1_xflux(const Ctx &c, const float *f, const float *fb, const float *fclim, int ii, int j, int k) {
  const size_t o = NPOM_I3(c, ii, j, k), om = NPOM_I3(c, ii - 1, j, k);
  float xf = 0.25f * (F2(dt, ii, j) + F2(dt, ii - 1, j)) * (ld(f + o) + ld(f + om)) * F3(u, ii, j, k);
  float aam_avg = 0.5f * (F3(aam, ii, j, k) + F3(aam, ii - 1, j, k));
  float fa = ld(fb + o) - ld(fclim + o), fam = ld(fb + om) - ld(fclim + om);
  xf -= aam_avg * (F2(h, ii, j) + F2(h, ii - 1, j)) * c.k.tprni * (fa - fam) * F2(dum, ii, j) /
        (F2(dx, ii, j) + F2(dx, ii - 1, j));
  xf *= 0.5f * (F2(dy, ii, j) + F2(dy, ii - 1, j));
  return xf;
}

NPOM_HD float advt1_yflux(const Ctx &c, const float *f, const float *fb, const float *fclim, int i, int jj, int k) {
  const size_t o = NPOM_I3(c, i, jj, k), om = NPOM_I3(c, i, jj - 1, k);
  float yf = 0.25f * (F2(dt, i, jj) + F2(dt, i, jj - 1)) * (ld(f + o) + ld(f + om)) * F3(v, i, jj, k);
  float aam_avg = 0.5f * (F3(aam, i, jj, k) + F3(aam, i, jj - 1, k));
  float fa = ld(fb + o) - ld(fclim + o), fam = ld(fb + om) - ld(fclim + om);
  yf -= aam_avg * (F2(h, i, jj) + F2(h, i, jj - 1)) * c.k.tprni * (fa - fam) * F2(dvm, i, jj) /
        (F2(dy, i, jj) + F2(dy, i, jj - 1));
  yf *= 0.5f * (F2(dx, i, jj) + F2(dx, i, jj - 1));
  return yf;
}

// the ADVT1 forecast at an interior (i, j, k < kb-1) from its horizontal
// flux divergence (the ghost level of f/fb is never read here)
NPOM_HD float advt1_finish(const Ctx &c, const float *f, const float *fb, int i, int j, int k, float horiz) {
  const int kbm1 = c.kb - 1;
  const float art = F2(art, i, j);
  auto zflux = [&](int kk) {
    if (kk == 0) return ld(f + NPOM_I3(c, i, j, 0)) * F3(w, i, j, 0) * art;
    if (kk >= kbm1) return 0.0f;
    return 0.5f * (ld(f + NPOM_I3(c, i, j, kk - 1)) + ld(f + NPOM_I3(c, i, j, kk))) * F3(w, i, j, kk) * art;
  };
  float vert = (zflux(k) - zflux(k + 1)) / F1(dz, k);
  float ff = horiz + vert;
  float tb = (F2(h, i, j) + F2(etb, i, j)) * art;
  float tf = (F2(h, i, j) + F2(etf, i, j)) * art;
  return (tb * ld(fb + NPOM_I3(c, i, j, k)) - c.k.dti2 * ff) / (tf + 1e-20f);
}

NPOM_HD float advt1_point(const Ctx &c, const float *f, const float *fb, const float *fclim, int i, int j, int k) {
  if (!interior(c, i, j) || k >= c.kb - 1) return 0.0f;
  float horiz = advt1_xflux(c, f, fb, fclim, i + 1, j, k) - advt1_xflux(c, f, fb, fclim, i, j, k) +
                advt1_yflux(c, f, fb, fclim, i, j + 1, k) - advt1_yflux(c, f, fb, fclim, i, j, k);
  return advt1_finish(c, f, fb, i, j, k, horiz);
}

// B5 at one point, part 1: q2/q2l Robert-Asselin filter with the bcond 6
// mask and the optional mixing clamp
NPOM_HD void phase_b5_filter(const Ctx &c, int i, int j, int k) {
  const float fsm = F2(fsm, i, j);
  // bcond 6 mask (explicit adds 1e-10)
  float uf6 = F3(uf, i, j, k) * fsm;
  float vf6 = F3(vf, i, j, k) * fsm;
  if (explicit_bc(c)) {
    uf6 = uf6 + 1.0e-10f;
    vf6 = vf6 + 1.0e-10f;
  }
  const float hs = c.k.half_smoth;
  float q2 = F3(q2, i, j, k), q2l = F3(q2l, i, j, k);
  float q2f = q2 + hs * (uf6 + F3(q2b, i, j, k) - 2.0f * q2);
  float q2lf = q2l + hs * (vf6 + F3(q2lb, i, j, k) - 2.0f * q2l);
  P3(q2b, i, j, k) = q2f;
  P3(q2, i, j, k) = uf6;
  P3(q2lb, i, j, k) = q2lf;
  P3(q2l, i, j, k) = vf6;
  if (!is_explicit(c) && c.k.has_vmix) {
    P3(kh, i, j, k) = fminf_t(fmaxf_t(F3(kh, i, j, k), 0.0f), c.k.vmix);
    P3(km, i, j, k) = fminf_t(fmaxf_t(F3(km, i, j, k), 0.0f), c.k.vmix);
    P3(kq, i, j, k) = fminf_t(fmaxf_t(F3(kq, i, j, k), 0.0f), c.k.vmix);
  }
}

// B5 part 2: store the ADVT1 forecasts; the ghost copy f[..., kb-1] =
// f[..., kb-2] is part of the stored t/tb/s/sb state (advt1 returns the
// modified copies)
NPOM_HD void phase_b5_store(const Ctx &c, int i, int j, int k, float tf_, float sf_) {
  const int kb = c.kb;
  P3(uf, i, j, k) = tf_;
  P3(vf, i, j, k) = sf_;
  if (k == kb - 1) {
    P3(t, i, j, k) = F3(t, i, j, kb - 2);
    P3(tb, i, j, k) = F3(tb, i, j, kb - 2);
    P3(s, i, j, k) = F3(s, i, j, kb - 2);
    P3(sb, i, j, k) = F3(sb, i, j, kb - 2);
  }
}

NPOM_HD void phase_b5_point(const Ctx &c, int i, int j, int k) {
  phase_b5_filter(c, i, j, k);
  if (c.k.mode == 4) return;
  float tf_ = advt1_point(c, c.F[NPOM_F_t], c.F[NPOM_F_tb], c.F[NPOM_F_tclim], i, j, k);
  float sf_ = advt1_point(c, c.F[NPOM_F_s], c.F[NPOM_F_sb], c.F[NPOM_F_sclim], i, j, k);
  phase_b5_store(c, i, j, k, tf_, sf_);
}

// ---------------------------------------------------------------------------
// PROFT column solve (tracers.py:890-1010) for any kb <= KMAX.
// ---------------------------------------------------------------------------
struct ProftCol {
  const float *f;      // column input, stride 1
  float *out;          // column output (may alias f)
  float wfsurf, fsurf, h, etf, swrad;
  const float *kh;     // column
  const float *dz, *dzz, *z;
  int kb, nbc, ntp;
  float dti2, umol;
};

// KM: the level arrays; KM == 16 is used for kb == 16 only, whose
// compile-time level count lets the loops unroll into registers
template <int KM = KMAX>
NPOM_HD float proft_column(const ProftCol &q) {
  const int kb = KM == 16 ? 16 : q.kb, kbm1 = kb - 1, kbm2 = kb - 2;
  float a[KM], cc[KM], ee[KM], gg[KM], rad[KM], fin[KM];
  for (int k = 0; k < kb; ++k) {
    a[k] = 0.0f;
    cc[k] = 0.0f;
    ee[k] = 0.0f;
    gg[k] = 0.0f;
    rad[k] = 0.0f;
    fin[k] = ld(q.f + k);
  }
  const float dh = q.h + q.etf;
  const float dh2 = dh * dh;
  const float neg_dti2 = -q.dti2;
  for (int k = 1; k < kbm1; ++k) {
    float num = neg_dti2 * (ld(q.kh + k) + q.umol);
    a[k - 1] = num / (ld(q.dz + k - 1) * ld(q.dzz + k - 1) * dh2);
    cc[k] = num / (ld(q.dz + k) * ld(q.dzz + k - 1) * dh2);
  }
  if (q.nbc == 2 || q.nbc == 4) {
    const float R[5] = {0.58f, 0.62f, 0.67f, 0.77f, 0.78f};
    const float AD1[5] = {0.35f, 0.60f, 1.00f, 1.50f, 1.40f};
    const float AD2[5] = {0.23f, 20.0f, 17.0f, 14.0f, 7.90f};
    const int ix = q.ntp - 1;
    for (int k = 0; k < kbm1; ++k) {
      float zt = ld(q.z + k) * dh;
      rad[k] = q.swrad * (R[ix] * expf(zt / AD1[ix]) + (1.0f - R[ix]) * expf(zt / AD2[ix]));
    }
  }
  float gprev;
  if (q.nbc == 1) {
    float den = a[0] - 1.0f;
    ee[0] = a[0] / den;
    gprev = (neg_dti2 * q.wfsurf / (-ld(q.dz) * dh) - fin[0]) / den;
  } else if (q.nbc == 2) {
    float den = a[0] - 1.0f;
    ee[0] = a[0] / den;
    gprev = (q.dti2 * (q.wfsurf + (rad[0] - rad[1])) / (ld(q.dz) * dh) - fin[0]) / den;
  } else {
    ee[0] = 0.0f;
    gprev = q.fsurf;
  }
  gg[0] = gprev;
  for (int k = 1; k < kbm2; ++k) {
    float den = a[k] + cc[k] * (1.0f - ee[k - 1]) - 1.0f;
    float inv = 1.0f / (den + 1e-20f);
    ee[k] = a[k] * inv;
    float rt = q.dti2 * (rad[k] - rad[k + 1]) / (dh * ld(q.dz + k));
    gprev = (cc[k] * gprev - fin[k] + rt) * inv;
    gg[k] = gprev;
  }
  const int kbt = kbm1 - 1;
  float rt = q.dti2 * (rad[kbt] - rad[kbt + 1]) / (dh * ld(q.dz + kbt));
  float num = cc[kbt] * gg[kbt - 1] - fin[kbt] + rt;
  float den = cc[kbt] * (1.0f - ee[kbt - 1]) - 1.0f;
  float nxt = num / (den + 1e-20f);
  float outv[KM];
  for (int k = 0; k < kb; ++k) outv[k] = fin[k];
  outv[kbt] = nxt;
  for (int k = kbm1 - 2; k >= 0; --k) {
    nxt = ee[k] * nxt + gg[k];
    outv[k] = nxt;
  }
  for (int k = 0; k < kb; ++k) q.out[k] = outv[k];
  return dh;
}

// ---------------------------------------------------------------------------
// B6 (column): PROFT for T (uf) and S (vf); tps = h + etf; explicit bcond 4
// upstream edge values (baroclinic.py:666-844).
// ---------------------------------------------------------------------------
NPOM_HD void bcond4_explicit_edge(const Ctx &c, int i, int j, float *ufc, float *vfc);
NPOM_HD bool bcond4_explicit_level(const Ctx &c, int i, int j, int k, float &uo, float &vo);

template <int KM = KMAX>
NPOM_HD void phase_b6_column(const Ctx &c, int i, int j) {
  const int kb = c.kb;
  ProftCol q;
  q.kh = &c.F[NPOM_F_kh][NPOM_I3(c, i, j, 0)];
  q.dz = c.F[NPOM_F_dz];
  q.dzz = c.F[NPOM_F_dzz];
  q.z = c.F[NPOM_F_z];
  q.kb = kb;
  q.ntp = c.k.ntp;
  q.dti2 = c.k.dti2;
  q.umol = c.k.umol;
  q.h = F2(h, i, j);
  q.etf = F2(etf, i, j);
  q.swrad = F2(swrad, i, j);
  float *ufc = &c.F[NPOM_F_uf][NPOM_I3(c, i, j, 0)];
  float *vfc = &c.F[NPOM_F_vf][NPOM_I3(c, i, j, 0)];
  q.f = ufc;
  q.out = ufc;
  q.nbc = c.k.nbct;
  q.wfsurf = F2(wtsurf, i, j);
  q.fsurf = F2(tsurf, i, j);
  proft_column<KM>(q);
  q.f = vfc;
  q.out = vfc;
  q.nbc = c.k.nbcs;
  q.wfsurf = F2(wssurf, i, j);
  q.fsurf = F2(ssurf, i, j);
  float dh = proft_column<KM>(q);
  P2(tps, i, j) = dh;
  if (explicit_bc(c) && !c.k.obc_seamount && (i == 0 || i == c.im - 1 || j == 0 || j == c.jm - 1))
    bcond4_explicit_edge(c, i, j, ufc, vfc);
}

// Explicit bcond 4 at level k (< kbm1) of an edge column: upstream T/S on
// the east, west, north and south edges, in the reference order
// (explicit/baroclinic.py:666-846; later sides win at corners).  Returns
// false when (i, j) lies on no edge; uo/vo are the new uf/vf values.
NPOM_HD bool bcond4_explicit_level(const Ctx &c, int i, int j, int k, float &uo, float &vo) {
  const int im = c.im, jm = c.jm, kbm1 = c.kb - 1;
  const float dti = c.k.dti;
  bool any = false;
  for (int side = 0; side < 4; ++side) {
    int ie, ii;  // edge index and inner index along the normal
    bool xdir;
    if (side == 0) { if (i != im - 1) continue; ie = im - 1; ii = im - 2; xdir = true; }
    else if (side == 1) { if (i != 0) continue; ie = 0; ii = 1; xdir = true; }
    else if (side == 2) { if (j != jm - 1) continue; ie = jm - 1; ii = jm - 2; xdir = false; }
    else { if (j != 0) continue; ie = 0; ii = 1; xdir = false; }
    any = true;
    float u1;
    float tc, sc, ti, si, te, se;
    if (xdir) {
      float vel = (side == 0) ? F3(u, im - 1, j, k) : F3(u, 1, j, k);
      float dsum = (side == 0) ? (F2(dx, im - 1, j) + F2(dx, im - 2, j)) : (F2(dx, 0, j) + F2(dx, 1, j));
      u1 = 2.0f * vel * dti / dsum;
      tc = F3(t, ie, j, k); sc = F3(s, ie, j, k); ti = F3(t, ii, j, k); si = F3(s, ii, j, k);
      size_t eo = (size_t)j * c.kb + k;
      te = ::npom::ld((side == 0 ? c.F[NPOM_F_tbe] : c.F[NPOM_F_tbw]) + eo);
      se = ::npom::ld((side == 0 ? c.F[NPOM_F_sbe] : c.F[NPOM_F_sbw]) + eo);
    } else {
      float vel = (side == 2) ? F3(v, i, jm - 1, k) : F3(v, i, 1, k);
      float dsum = (side == 2) ? (F2(dy, i, jm - 1) + F2(dy, i, jm - 2)) : (F2(dy, i, 0) + F2(dy, i, 1));
      u1 = 2.0f * vel * dti / dsum;
      tc = F3(t, i, ie, k); sc = F3(s, i, ie, k); ti = F3(t, i, ii, k); si = F3(s, i, ii, k);
      size_t eo = (size_t)i * c.kb + k;
      te = ::npom::ld((side == 2 ? c.F[NPOM_F_tbn] : c.F[NPOM_F_tbs]) + eo);
      se = ::npom::ld((side == 2 ? c.F[NPOM_F_sbn] : c.F[NPOM_F_sbs]) + eo);
    }
    bool east_like = (side == 0 || side == 2);
    if (east_like) {
      if (u1 <= 0.0f) { uo = tc - u1 * (te - tc); vo = sc - u1 * (se - sc); }
      else { uo = tc - u1 * (tc - ti); vo = sc - u1 * (sc - si); }
    } else {
      if (u1 >= 0.0f) { uo = tc - u1 * (tc - te); vo = sc - u1 * (sc - se); }
      else { uo = tc - u1 * (ti - tc); vo = sc - u1 * (si - sc); }
    }
    // vertical correction for outflow on 1 <= k <= kbm1-2
    if (kbm1 > 2 && k >= 1 && k <= kbm1 - 2) {
      bool outflow = east_like ? (u1 > 0.0f) : (u1 < 0.0f);
      if (outflow) {
        float wsum, dtv, tm, tp, sm, sp;
        if (xdir) {
          wsum = F3(w, ii, j, k) + F3(w, ii, j, k + 1);
          dtv = F2(dt, ii, j);
          tm = F3(t, ii, j, k - 1); tp = F3(t, ii, j, k + 1); sm = F3(s, ii, j, k - 1); sp = F3(s, ii, j, k + 1);
        } else {
          wsum = F3(w, i, ii, k) + F3(w, i, ii, k + 1);
          dtv = F2(dt, i, ii);
          tm = F3(t, i, ii, k - 1); tp = F3(t, i, ii, k + 1); sm = F3(s, i, ii, k - 1); sp = F3(s, i, ii, k + 1);
        }
        float wm = 0.5f * wsum * dti / ((F1(zz, k - 1) - F1(zz, k + 1)) * dtv);
        uo = uo - wm * (tm - tp);
        vo = vo - wm * (sm - sp);
      }
    }
  }
  return any;
}

NPOM_HD void bcond4_explicit_edge(const Ctx &c, int i, int j, float *ufc, float *vfc) {
  const int kbm1 = c.kb - 1;
  for (int k = 0; k < kbm1; ++k) {
    float uo, vo;
    if (bcond4_explicit_level(c, i, j, k, uo, vo)) {
      ufc[k] = uo;
      vfc[k] = vo;
    }
  }
}

// ---------------------------------------------------------------------------
// B7 (point): closed-basin bcond 4 (implicit) or the explicit mask, T/S
// Robert-Asselin filter, tracer Shapiro filter, shifts and DENS
// (momentum.py:467-541).
// ---------------------------------------------------------------------------
NPOM_HD float bc4_implicit_value(const Ctx &c, const float *arr, int i, int j, int k) {
  // closed_basin.py:287-298: rows 0/im-1 copy rows 1/im-2, then columns
  // 0/jm-1 copy columns 1/jm-2 (corners see the row-copied values)
  const int im = c.im, jm = c.jm;
  int si = i, sj = j;
  if (j == 0) sj = 1;
  if (j == jm - 1) sj = jm - 2;
  if (si == 0) si = 1;
  if (si == im - 1) si = im - 2;
  return ld(arr + NPOM_I3(c, si, sj, k));
}

NPOM_HD float dens_point(const Ctx &c, float t, float s, int i, int j, int k) {
  float tr = t + c.k.tbias;
  float sr = s + c.k.sbias;
  float tr2 = tr * tr;
  float tr3 = tr2 * tr;
  float tr4 = tr3 * tr;
  float p = c.k.g_rhoref * (-F1(zz, k) * F2(h, i, j)) * 1.0e-5f;
  float rhor = -0.157406f + 6.793952e-2f * tr - 9.095290e-3f * tr2 + 1.001685e-4f * tr3 - 1.120083e-6f * tr4 +
               6.536332e-9f * tr4 * tr;
  rhor = rhor + (0.824493f - 4.0899e-3f * tr + 7.6438e-5f * tr2 - 8.2467e-7f * tr3 + 5.3875e-9f * tr4) * sr;
  rhor = rhor + (-5.72466e-3f + 1.0227e-4f * tr - 1.6546e-6f * tr2) * powf(fmaxf_t(fabsf(sr), 1e-8f), 1.5f);
  rhor = rhor + 4.8314e-4f * sr * sr;
  float cr = 1449.1f + 0.0821f * p + 4.55f * tr - 0.045f * tr2 + 1.34f * (sr - 35.0f);
  float cr2 = cr * cr;
  float tp = 1.0e5f * p / cr2;
  rhor = rhor + tp * (1.0f - 2.0f * p / cr2);
  return (rhor / c.k.rhoref) * F2(fsm, i, j);
}

NPOM_HD void phase_b7_point(const Ctx &c, int i, int j, int k) {
  if (c.k.mode == 4) return;
  const int im = c.im, jm = c.jm, kb = c.kb;
  const float fsm = F2(fsm, i, j);
  const float *ufa = c.F[NPOM_F_uf];
  const float *vfa = c.F[NPOM_F_vf];
  float ufv, vfv;
  bool edge = (i == 0 || i == im - 1 || j == 0 || j == jm - 1);
  if (explicit_bc(c)) {
    ufv = F3(uf, i, j, k) * fsm;
    vfv = F3(vf, i, j, k) * fsm;
  } else {
    ufv = edge ? bc4_implicit_value(c, ufa, i, j, k) : F3(uf, i, j, k);
    vfv = edge ? bc4_implicit_value(c, vfa, i, j, k) : F3(vf, i, j, k);
  }
  const float hs = c.k.half_smoth;
  float t = F3(t, i, j, k), s = F3(s, i, j, k);
  float tf = t + hs * (ufv + F3(tb, i, j, k) - 2.0f * t);
  float sf = s + hs * (vfv + F3(sb, i, j, k) - 2.0f * s);
  float tn = ufv, sn = vfv;
  if (!is_explicit(c)) {
    // numerics/double_gyre.py:78-111: Shapiro (gamma > 0) then fsm mask
    if (c.k.tshap > 0.0 && interior(c, i, j) && k < kb - 1) {
      auto val = [&](const float *arr, int ii, int jj) {
        bool e2 = (ii == 0 || ii == im - 1 || jj == 0 || jj == jm - 1);
        return e2 ? bc4_implicit_value(c, arr, ii, jj, k) : ld(arr + NPOM_I3(c, ii, jj, k));
      };
      tn = ufv + c.k.tshap_q * (val(ufa, i + 1, j) + val(ufa, i - 1, j) + val(ufa, i, j + 1) + val(ufa, i, j - 1) - 4.0f * ufv);
      sn = vfv + c.k.tshap_q * (val(vfa, i + 1, j) + val(vfa, i - 1, j) + val(vfa, i, j + 1) + val(vfa, i, j - 1) - 4.0f * vfv);
    }
    tn = tn * fsm;
    sn = sn * fsm;
  }
  P3(tb, i, j, k) = tf;
  P3(sb, i, j, k) = sf;
  P3(t, i, j, k) = tn;
  P3(s, i, j, k) = sn;
  if (k < kb - 1) P3(rho, i, j, k) = dens_point(c, tn, sn, i, j, k);
}

// ---------------------------------------------------------------------------
// B8 (column): ADVU + PROFU and ADVV + PROFV (momentum.py:14-465); explicit
// bcond 3 edge values (baroclinic.py:576-661).
// ---------------------------------------------------------------------------
NPOM_HD float advu_point(const Ctx &c, int i, int j, int k) {
  // interior i, j; k < kbm1
  const int kbm1 = c.kb - 1;
  auto vflux = [&](int kk) {
    if (kk < 1 || kk > kbm1 - 1) return 0.0f;
    return 0.25f * (F3(w, i, j, kk) + F3(w, i - 1, j, kk)) * (F3(u, i, j, kk) + F3(u, i, j, kk - 1));
  };
  float aru = F2(aru, i, j);
  float vdiv = (vflux(k) - vflux(k + 1)) * aru / F1(dz, k);
  float ct1 = F2(cor, i, j) * F2(dt, i, j) * (F3(v, i, j + 1, k) + F3(v, i, j, k));
  float ct2 = F2(cor, i - 1, j) * F2(dt, i - 1, j) * (F3(v, i - 1, j + 1, k) + F3(v, i - 1, j, k));
  float corio = -aru * 0.25f * (ct1 + ct2);
  float geg = (F2(egf, i, j) - F2(egf, i - 1, j)) + (F2(egb, i, j) - F2(egb, i - 1, j));
  float gpa = 2.0f * (F2(e_atmos, i, j) - F2(e_atmos, i - 1, j));
  float press = c.k.g_eighth * ((F2(dt, i, j) + F2(dt, i - 1, j)) * (geg + gpa) * (F2(dy, i, j) + F2(dy, i - 1, j)));
  float rhs = F3(advx, i, j, k) + vdiv + corio + press + F3(drhox, i, j, k);
  float hs = F2(h, i, j) + F2(h, i - 1, j);
  float den = (hs + F2(etf, i, j) + F2(etf, i - 1, j)) * aru;
  float old = ((hs + F2(etb, i, j) + F2(etb, i - 1, j)) * aru) * F3(ub, i, j, k);
  return (old - c.k.two_dti2 * rhs) / (den + 1e-20f);
}

NPOM_HD float advv_point(const Ctx &c, int i, int j, int k) {
  const int kbm1 = c.kb - 1;
  auto vflux = [&](int kk) {
    if (kk < 1 || kk > kbm1 - 1) return 0.0f;
    return 0.25f * (F3(w, i, j, kk) + F3(w, i, j - 1, kk)) * (F3(v, i, j, kk) + F3(v, i, j, kk - 1));
  };
  float arv = F2(arv, i, j);
  float vdiv = (vflux(k) - vflux(k + 1)) * arv / F1(dz, k);
  float ct1 = F2(cor, i, j) * F2(dt, i, j) * (F3(u, i + 1, j, k) + F3(u, i, j, k));
  float ct2 = F2(cor, i, j - 1) * F2(dt, i, j - 1) * (F3(u, i + 1, j - 1, k) + F3(u, i, j - 1, k));
  float corio = arv * 0.25f * (ct1 + ct2);
  float geg = (F2(egf, i, j) - F2(egf, i, j - 1)) + (F2(egb, i, j) - F2(egb, i, j - 1));
  float gpa = 2.0f * (F2(e_atmos, i, j) - F2(e_atmos, i, j - 1));
  float press = c.k.g_eighth * ((F2(dt, i, j) + F2(dt, i, j - 1)) * (geg + gpa) * (F2(dx, i, j) + F2(dx, i, j - 1)));
  float rhs = F3(advy, i, j, k) + vdiv + corio + press + F3(drhoy, i, j, k);
  float hs = F2(h, i, j) + F2(h, i, j - 1);
  float den = (hs + F2(etf, i, j) + F2(etf, i, j - 1)) * arv;
  float old = ((hs + F2(etb, i, j) + F2(etb, i, j - 1)) * arv) * F3(vb, i, j, k);
  return (old - c.k.two_dti2 * rhs) / (den + 1e-20f);
}

// PROFU (comp 0) / PROFV (comp 1) for one column, given the ADVU/ADVV
// forecast fin[] of that column.  Returns wbot; writes out[] and tps.
NPOM_HD void profuv_column(const Ctx &c, int comp, int i, int j, const float *fin, float *out, float &wbot,
                           float &tps) {
  const int kb = c.kb, kbm1 = kb - 1, kbm2 = kb - 2;
  for (int k = 0; k < kb; ++k) out[k] = fin[k];
  wbot = comp == 0 ? F2(wubot, i, j) : F2(wvbot, i, j);
  tps = 0.0f;
  if (i < 1 || j < 1) return;  // outside [1:im, 1:jm] nothing is solved
  const int oi = comp == 0 ? i - 1 : i, oj = comp == 0 ? j : j - 1;
  const float dti2 = c.k.dti2;
  float dhf = 0.5f * (F2(h, i, j) + F2(etf, i, j) + F2(h, oi, oj) + F2(etf, oi, oj));
  float dh2 = dhf * dhf;
  float a[KMAX], cc[KMAX], ee[KMAX], gg[KMAX];
  for (int k = 0; k < kb; ++k) {
    a[k] = 0.0f;
    cc[k] = 0.0f;
    ee[k] = 0.0f;
    gg[k] = 0.0f;
  }
  for (int k = 1; k < kbm1; ++k) {
    float kmf = 0.5f * (F3(km, i, j, k) + F3(km, oi, oj, k));
    float num = c.k.neg_dti2 * (kmf + c.k.umol);
    a[k - 1] = num / (F1(dz, k - 1) * F1(dzz, k - 1) * dh2);
    cc[k] = num / (F1(dz, k) * F1(dzz, k - 1) * dh2);
  }
  float den0 = a[0] - 1.0f;
  ee[0] = a[0] / (den0 + 1e-20f);
  float wsurf = comp == 0 ? F2(wusurf, i, j) : F2(wvsurf, i, j);
  float term = c.k.neg_dti2 * wsurf / (-F1(dz, 0) * dhf);
  float gprev = (term - fin[0]) / (den0 + 1e-20f);
  gg[0] = gprev;
  for (int k = 1; k < kbm2; ++k) {
    float den = a[k] + cc[k] * (1.0f - ee[k - 1]) - 1.0f;
    float inv = 1.0f / (den + 1e-20f);
    ee[k] = a[k] * inv;
    gprev = (cc[k] * gprev - fin[k]) * inv;
    gg[k] = gprev;
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
  float fric = tps * dti2 / (-F1(dz, kbt) * dhf);
  float den = fric - 1.0f - (ee[kbt - 1] - 1.0f) * cc[kbt];
  float num = cc[kbt] * gg[kbt - 1] - fin[kbt];
  float mask = comp == 0 ? F2(dum, i, j) : F2(dvm, i, j);
  float nxt = num / (den + 1e-20f) * mask;
  out[kbt] = nxt;
  for (int k = kbt - 1; k >= 0; --k) {
    nxt = (ee[k] * nxt + gg[k]) * mask;
    out[k] = nxt;
  }
  wbot = -tps * out[kbt];
}

NPOM_HD void bcond3_explicit_edge(const Ctx &c, int i, int j, float *ufo, float *vfo) {
  const int im = c.im, jm = c.jm, kbm1 = c.kb - 1;
  const float hmax = c.k.hmax;
  auto ga_of = [&](float hh) { return sqrtf(fmaxf_t(hh / hmax, 1e-8f)); };
  // the coastal tide policy weighs by the total depth d (its step copy,
  // coastal_explicit_baroclinic.py:586-641), the native bcond by h
  const int gf = c.k.obc_coastal ? NPOM_F_d : NPOM_F_h;
  if (j >= 1 && j <= jm - 2) {
    if (i == im - 1) {
      float ga = ga_of(ld(c.F[gf] + NPOM_I2(c, im - 1, j)));
      for (int k = 0; k < kbm1; ++k) {
        float ui = 0.25f * F3(u, im - 2, j - 1, k) + 0.50f * F3(u, im - 2, j, k) + 0.25f * F3(u, im - 2, j + 1, k);
        float uo = 0.25f * F3(u, im - 1, j - 1, k) + 0.50f * F3(u, im - 1, j, k) + 0.25f * F3(u, im - 1, j + 1, k);
        ufo[k] = ga * ui + (1.0f - ga) * uo;
        vfo[k] = 0.0f;
      }
    }
    if (i == 1 || i == 0) {
      float ga = ga_of(ld(c.F[gf] + NPOM_I2(c, 0, j)));
      for (int k = 0; k < kbm1; ++k) {
        float ui = 0.25f * F3(u, 2, j - 1, k) + 0.50f * F3(u, 2, j, k) + 0.25f * F3(u, 2, j + 1, k);
        float uo = 0.25f * F3(u, 1, j - 1, k) + 0.50f * F3(u, 1, j, k) + 0.25f * F3(u, 1, j + 1, k);
        ufo[k] = ga * ui + (1.0f - ga) * uo;
        if (i == 0) vfo[k] = 0.0f;
      }
    }
  }
  if (i >= 1 && i <= im - 2) {
    if (j == jm - 1) {
      float ga = ga_of(ld(c.F[gf] + NPOM_I2(c, i, jm - 1)));
      for (int k = 0; k < kbm1; ++k) {
        float vi = 0.25f * F3(v, i - 1, jm - 2, k) + 0.50f * F3(v, i, jm - 2, k) + 0.25f * F3(v, i + 1, jm - 2, k);
        float vo = 0.25f * F3(v, i - 1, jm - 1, k) + 0.50f * F3(v, i, jm - 1, k) + 0.25f * F3(v, i + 1, jm - 1, k);
        vfo[k] = ga * vi + (1.0f - ga) * vo;
        ufo[k] = 0.0f;
      }
    }
    if (j == 1 || j == 0) {
      float ga = ga_of(ld(c.F[gf] + NPOM_I2(c, i, 0)));
      for (int k = 0; k < kbm1; ++k) {
        float vi = 0.25f * F3(v, i - 1, 2, k) + 0.50f * F3(v, i, 2, k) + 0.25f * F3(v, i + 1, 2, k);
        float vo = 0.25f * F3(v, i - 1, 1, k) + 0.50f * F3(v, i, 1, k) + 0.25f * F3(v, i + 1, 1, k);
        vfo[k] = ga * vi + (1.0f - ga) * vo;
        if (j == 0) ufo[k] = 0.0f;
      }
    }
  }
}

// The Jiaozhou Bay policy's bcond 3 (jzb_boundary.py:88-140) at one level
// k < kbm1: u on the east edge and at column 1 (its ghost column 0 a copy),
// v on the north edge and at row 1 (its ghost row 0 a copy), each the blend
// ga * (1-2-1 average across the edge one cell inside) + (1 - ga) * (the
// same at the edge) with ga = sqrt(max(d / hmax, 0)) at the depth cell the
// policy names (east and north edges, column 0, row 1), times ramp except
// on the north edge, wherever that d > 0; there the tangential component
// on the outer ring is zero.  Reads u, v and d only; the edge sets touch
// different values, so their order does not matter.  The masks follow in
// B9.
NPOM_HD void jzb_bcond3_level(const Ctx &c, int i, int j, int k, float &uo, float &vo) {
  const int im = c.im, jm = c.jm;
  if (k >= c.kb - 1) return;
  const float hmax = c.k.hmax, ramp = c.ramp;
  auto ga_of = [&](int ii, int jj) { return sqrtf(fmaxf_t(F2(d, ii, jj) / hmax, 0.0f)); };
  auto avg_u = [&](int ii) {
    return 0.25f * F3(u, ii, j - 1, k) + 0.50f * F3(u, ii, j, k) + 0.25f * F3(u, ii, j + 1, k);
  };
  auto avg_v = [&](int jj) {
    return 0.25f * F3(v, i - 1, jj, k) + 0.50f * F3(v, i, jj, k) + 0.25f * F3(v, i + 1, jj, k);
  };
  if (j >= 1 && j <= jm - 2) {
    if (i == im - 1 && F2(d, im - 1, j) > 0.0f) {
      const float ga = ga_of(im - 1, j);
      uo = (ga * avg_u(im - 2) + (1.0f - ga) * avg_u(im - 1)) * ramp;
      vo = 0.0f;
    }
    if ((i == 1 || i == 0) && F2(d, 0, j) > 0.0f) {
      const float ga = ga_of(0, j);
      uo = (ga * avg_u(2) + (1.0f - ga) * avg_u(1)) * ramp;
      if (i == 0) vo = 0.0f;
    }
  }
  if (i >= 1 && i <= im - 2) {
    if (j == jm - 1 && F2(d, i, jm - 1) > 0.0f) {
      const float ga = ga_of(i, jm - 1);
      vo = ga * avg_v(jm - 2) + (1.0f - ga) * avg_v(jm - 1);
      uo = 0.0f;
    }
    if ((j == 1 || j == 0) && F2(d, i, 1) > 0.0f) {
      const float ga = ga_of(i, 1);
      vo = (ga * avg_v(2) + (1.0f - ga) * avg_v(1)) * ramp;
      if (j == 0) uo = 0.0f;
    }
  }
}

NPOM_HD void phase_b8_column(const Ctx &c, int i, int j) {
  const int kb = c.kb;
  float fin[KMAX], uo[KMAX], vo[KMAX];
  bool inner = interior(c, i, j);
  // ADVU: zero outside the interior (fresh tensor)
  for (int k = 0; k < kb; ++k) fin[k] = (inner && k < kb - 1) ? advu_point(c, i, j, k) : 0.0f;
  float wub, wvb, tpsu, tpsv;
  profuv_column(c, 0, i, j, fin, uo, wub, tpsu);
  for (int k = 0; k < kb; ++k) fin[k] = (inner && k < kb - 1) ? advv_point(c, i, j, k) : 0.0f;
  profuv_column(c, 1, i, j, fin, vo, wvb, tpsv);
  if (c.k.obc_jzb) {
    for (int k = 0; k < kb; ++k) jzb_bcond3_level(c, i, j, k, uo[k], vo[k]);
  } else if (explicit_bc(c) && !c.k.obc_seamount) {
    bcond3_explicit_edge(c, i, j, uo, vo);
  }
  for (int k = 0; k < kb; ++k) {
    P3(uf, i, j, k) = uo[k];
    P3(vf, i, j, k) = vo[k];
  }
  P2(wubot, i, j) = wub;
  P2(wvbot, i, j) = wvb;
  P2(tps, i, j) = tpsv;
}

// ---------------------------------------------------------------------------
// B9 (column): bcond 3 masks, internal velocity filter and shift
// (time_loop.py:628-678; implicit numerics/double_gyre.py:147-184), then the
// 2-D shifts that close every step (time_loop.py:680-696).
// ---------------------------------------------------------------------------
NPOM_HD void phase_b9_column(const Ctx &c, int i, int j) {
  const int im = c.im, jm = c.jm, kb = c.kb, kbm1 = kb - 1;
  if (c.do_internal) {
    const float dum = F2(dum, i, j), dvm = F2(dvm, i, j);
    bool ring = (i == 0 || i == im - 1 || j == 0 || j == jm - 1);
    const float hs = c.k.half_smoth;
    for (int comp = 0; comp < 2; ++comp) {
      const float mask = comp == 0 ? dum : dvm;
      float *fa = comp == 0 ? c.F[NPOM_F_u] : c.F[NPOM_F_v];
      float *fb = comp == 0 ? c.F[NPOM_F_ub] : c.F[NPOM_F_vb];
      float *ff = comp == 0 ? c.F[NPOM_F_uf] : c.F[NPOM_F_vf];
      float fnew[KMAX], term[KMAX];
      for (int k = 0; k < kb; ++k) {
        float x = ld(ff + NPOM_I3(c, i, j, k)) * mask;
        if (!explicit_bc(c) && ring) x = 0.0f;
        fnew[k] = x;
      }
      float tps = 0.0f;
      for (int k = 0; k < kbm1; ++k) {
        term[k] = fnew[k] + ld(fb + NPOM_I3(c, i, j, k)) - 2.0f * ld(fa + NPOM_I3(c, i, j, k));
        tps += term[k] * F1(dz, k);
      }
      for (int k = 0; k < kb; ++k) {
        float cur = ld(fa + NPOM_I3(c, i, j, k));
        float filt = (k < kbm1) ? cur + hs * (term[k] - tps) : cur;
        if (!is_explicit(c)) filt = filt * mask;  // Shapiro (gamma 0) + mask
        fb[NPOM_I3(c, i, j, k)] = filt;
        fa[NPOM_I3(c, i, j, k)] = fnew[k];
        ff[NPOM_I3(c, i, j, k)] = fnew[k];
      }
    }
  }
  P2(egb, i, j) = F2(egf, i, j);
  P2(etb, i, j) = F2(et, i, j);
  float etf = F2(etf, i, j);
  P2(et, i, j) = etf;
  P2(dt, i, j) = F2(h, i, j) + etf;
  P2(utb, i, j) = F2(utf, i, j);
  P2(vtb, i, j) = F2(vtf, i, j);
  P2(vfluxb, i, j) = F2(vfluxf, i, j);
}

// ---------------------------------------------------------------------------
// The seamount case policy's Orlanski edges (seamount_boundary.py:20-38), one
// thread per (j, k): after B8 for u (bcond 3), after B6 for T and S (bcond
// 4).  They read the new values of the columns next to the edges, which
// other threads of those phases compute, so they run as a pass of their
// own; the masks follow in B9 and B7, after the edges, as in the reference.
// A zero denominator becomes 0.01, the Orlanski ratio is clamped to [0, 1].
// ---------------------------------------------------------------------------
NPOM_HD float orlanski_ratio(float past_near, float out_near, float cur_next) {
  float den = out_near + past_near - 2.0f * cur_next;
  if (den == 0.0f) den = 0.01f;
  return fminf_t(fmaxf_t((past_near - out_near) / den, 0.0f), 1.0f);
}

// bcond 3: u on the west (column 1, from 2 and 3) and east (im-1, from
// im-2 and im-3) edges, no v through them, the west ghost column a copy
NPOM_HD void obc_seamount_u_point(const Ctx &c, int j, int k) {
  const int im = c.im;
  if (j < 1 || j > c.jm - 2 || k >= c.kb - 1) return;
  float *uf = c.F[NPOM_F_uf], *vf = c.F[NPOM_F_vf];
  for (int side = 0; side < 2; ++side) {
    const int edge = side == 0 ? 1 : im - 1, near = side == 0 ? 2 : im - 2, nexti = side == 0 ? 3 : im - 3;
    const float cl = orlanski_ratio(F3(ub, near, j, k), uf[NPOM_I3(c, near, j, k)], F3(u, nexti, j, k));
    uf[NPOM_I3(c, edge, j, k)] = (F3(ub, edge, j, k) * (1.0f - cl) + 2.0f * cl * F3(u, near, j, k)) / (1.0f + cl);
    vf[NPOM_I3(c, side == 0 ? 0 : im - 1, j, k)] = 0.0f;
  }
  uf[NPOM_I3(c, 0, j, k)] = uf[NPOM_I3(c, 1, j, k)];
}

// bcond 4: T (uf) and S (vf) on the west (column 0) and east (im-1) edges;
// where the ratio is 0 and the flow at the edge enters, the exterior
// profile (tbw/sbw, tbe/sbe) instead
NPOM_HD void obc_seamount_ts_point(const Ctx &c, int j, int k) {
  const int im = c.im;
  if (k >= c.kb - 1) return;
  const size_t eo = (size_t)j * c.kb + k;
  for (int side = 0; side < 2; ++side) {
    const int edge = side == 0 ? 0 : im - 1, near = side == 0 ? 1 : im - 2, nexti = side == 0 ? 2 : im - 3;
    const float vel = F3(ub, side == 0 ? 1 : im - 1, j, k);
    const float sign = side == 0 ? 1.0f : -1.0f;
    for (int tr = 0; tr < 2; ++tr) {
      float *out = c.F[tr == 0 ? NPOM_F_uf : NPOM_F_vf];
      const float *past = c.F[tr == 0 ? NPOM_F_tb : NPOM_F_sb];
      const float *cur = c.F[tr == 0 ? NPOM_F_t : NPOM_F_s];
      const float *ext = c.F[side == 0 ? (tr == 0 ? NPOM_F_tbw : NPOM_F_sbw) : (tr == 0 ? NPOM_F_tbe : NPOM_F_sbe)];
      const float cl =
          orlanski_ratio(ld(past + NPOM_I3(c, near, j, k)), out[NPOM_I3(c, near, j, k)], ld(cur + NPOM_I3(c, nexti, j, k)));
      const float value =
          (ld(past + NPOM_I3(c, edge, j, k)) * (1.0f - cl) + 2.0f * cl * ld(cur + NPOM_I3(c, near, j, k))) / (1.0f + cl);
      out[NPOM_I3(c, edge, j, k)] = (cl == 0.0f && sign * vel >= 0.0f) ? ld(ext + eo) : value;
    }
  }
}

}  // namespace npom
