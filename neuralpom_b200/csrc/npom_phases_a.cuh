// npom_phases_a.cuh -- phases that open an internal step: surface forcing,
// momentum advection (ADVCT), baroclinic pressure gradient (BAROPG),
// Smagorinsky viscosity, depth integrals and the 2-D advection (ADVAVE).
//
// Every body evaluates the reference's expression for one output element
// with the reference's operation order (no FMA contraction: the library is
// built with --fmad=false) so that results agree with the PyTorch core to
// float32 rounding.
#pragma once

#include "npom_ctx.cuh"

namespace npom {

// ---------------------------------------------------------------------------
// ADVCT (src/neuralpom/cores/explicit/baroclinic.py:14-260)
// ---------------------------------------------------------------------------

// curv(i,j,k), interior only (baroclinic.py:58-69)
NPOM_HD float advct_curv(const Ctx &c, int i, int j, int k) {
  if (!interior(c, i, j)) return 0.0f;
  float t1 = (F3(v, i, j + 1, k) + F3(v, i, j, k)) * (F2(dy, i + 1, j) - F2(dy, i - 1, j));
  float t2 = (F3(u, i + 1, j, k) + F3(u, i, j, k)) * (F2(dx, i, j + 1) - F2(dx, i, j - 1));
  return 0.25f * (t1 - t2) / (F2(dx, i, j) * F2(dy, i, j) + 1e-20f);
}

// x-momentum x-flux at (ip, j), ip in 1..im-2 (baroclinic.py:76-139)
NPOM_HD float advct_xflux_u(const Ctx &c, int ip, int j, int k) {
  if (ip < 1 || ip > c.im - 2) return 0.0f;
  float t1 = (F2(dt, ip + 1, j) + F2(dt, ip, j)) * F3(u, ip + 1, j, k);
  float t2 = (F2(dt, ip, j) + F2(dt, ip - 1, j)) * F3(u, ip, j, k);
  float xf = 0.125f * (t1 + t2) * (F3(u, ip + 1, j, k) + F3(u, ip, j, k));
  if (j >= 1) {
    float grad_u = (F3(ub, ip + 1, j, k) - F3(ub, ip, j, k)) / (F2(dx, ip, j) + 1e-20f);
    xf = xf - F2(dt, ip, j) * F3(aam, ip, j, k) * 2.0f * grad_u;
    xf *= F2(dy, ip, j);
  }
  return xf;
}

// shear diffusion term dtaam*(du/dy + dv/dx) at a corner point (i, j)
NPOM_HD float advct_shear(const Ctx &c, int i, int j, int k) {
  float dt_avg = 0.25f * (F2(dt, i, j) + F2(dt, i - 1, j) + F2(dt, i, j - 1) + F2(dt, i - 1, j - 1));
  float aam_sum = F3(aam, i, j, k) + F3(aam, i - 1, j, k) + F3(aam, i, j - 1, k) + F3(aam, i - 1, j - 1, k);
  float dtaam = dt_avg * aam_sum;
  float den_dy = F2(dy, i, j) + F2(dy, i - 1, j) + F2(dy, i, j - 1) + F2(dy, i - 1, j - 1);
  float den_dx = F2(dx, i, j) + F2(dx, i - 1, j) + F2(dx, i, j - 1) + F2(dx, i - 1, j - 1);
  float du_dy = (F3(ub, i, j, k) - F3(ub, i, j - 1, k)) / (den_dy + 1e-20f);
  float dv_dx = (F3(vb, i, j, k) - F3(vb, i - 1, j, k)) / (den_dx + 1e-20f);
  return dtaam * (du_dy + dv_dx);
}

// x-momentum y-flux at (i, jp), i in 1..im-1, jp in 1..jm-1
NPOM_HD float advct_yflux_u(const Ctx &c, int i, int jp, int k) {
  if (i < 1 || jp < 1) return 0.0f;
  float t1 = (F2(dt, i, jp) + F2(dt, i, jp - 1)) * F3(v, i, jp, k);
  float t2 = (F2(dt, i - 1, jp) + F2(dt, i - 1, jp - 1)) * F3(v, i - 1, jp, k);
  float yf = 0.125f * (t1 + t2) * (F3(u, i, jp, k) + F3(u, i, jp - 1, k));
  if (i <= c.im - 2) {
    yf = yf - advct_shear(c, i, jp, k);
    float dx_sum = F2(dx, i, jp) + F2(dx, i - 1, jp) + F2(dx, i, jp - 1) + F2(dx, i - 1, jp - 1);
    yf *= 0.25f * dx_sum;
  }
  return yf;
}

// y-momentum x-flux at (ip, j), ip in 1..im-1, j in 1..jm-1
NPOM_HD float advct_xflux_v(const Ctx &c, int ip, int j, int k) {
  if (ip < 1 || j < 1) return 0.0f;
  float t1 = (F2(dt, ip, j) + F2(dt, ip - 1, j)) * F3(u, ip, j, k);
  float t2 = (F2(dt, ip, j - 1) + F2(dt, ip - 1, j - 1)) * F3(u, ip, j - 1, k);
  float xf = 0.125f * (t1 + t2) * (F3(v, ip, j, k) + F3(v, ip - 1, j, k));
  if (j <= c.jm - 2) {
    xf = xf - advct_shear(c, ip, j, k);
    float dy_sum = F2(dy, ip, j) + F2(dy, ip - 1, j) + F2(dy, ip, j - 1) + F2(dy, ip - 1, j - 1);
    xf *= 0.25f * dy_sum;
  }
  return xf;
}

// y-momentum y-flux at (i, jp), jp in 1..jm-2
NPOM_HD float advct_yflux_v(const Ctx &c, int i, int jp, int k) {
  if (jp < 1 || jp > c.jm - 2) return 0.0f;
  float t1 = (F2(dt, i, jp + 1) + F2(dt, i, jp)) * F3(v, i, jp + 1, k);
  float t2 = (F2(dt, i, jp) + F2(dt, i, jp - 1)) * F3(v, i, jp, k);
  float yf = 0.125f * (t1 + t2) * (F3(v, i, jp + 1, k) + F3(v, i, jp, k));
  if (i >= 1) {
    float grad_v = (F3(vb, i, jp + 1, k) - F3(vb, i, jp, k)) / (F2(dy, i, jp) + 1e-20f);
    yf = yf - F2(dt, i, jp) * F3(aam, i, jp, k) * 2.0f * grad_v;
    yf *= F2(dx, i, jp);
  }
  return yf;
}

NPOM_HD void advct_point(const Ctx &c, int i, int j, int k, float &advx, float &advy, float &curv) {
  advx = 0.0f;
  advy = 0.0f;
  curv = 0.0f;
  if (k >= c.kb - 1 || !interior(c, i, j)) return;
  curv = advct_curv(c, i, j, k);
  float ax = advct_xflux_u(c, i, j, k) - advct_xflux_u(c, i - 1, j, k) + advct_yflux_u(c, i, j + 1, k) -
             advct_yflux_u(c, i, j, k);
  if (i >= 2) {
    float tc1 = curv * F2(dt, i, j) * (F3(v, i, j + 1, k) + F3(v, i, j, k));
    float tc2 = advct_curv(c, i - 1, j, k) * F2(dt, i - 1, j) * (F3(v, i - 1, j + 1, k) + F3(v, i - 1, j, k));
    ax -= F2(aru, i, j) * 0.25f * (tc1 + tc2);
  }
  float ay = advct_xflux_v(c, i + 1, j, k) - advct_xflux_v(c, i, j, k) + advct_yflux_v(c, i, j, k) -
             advct_yflux_v(c, i, j - 1, k);
  if (j >= 2) {
    float tc1 = curv * F2(dt, i, j) * (F3(u, i + 1, j, k) + F3(u, i, j, k));
    float tc2 = advct_curv(c, i, j - 1, k) * F2(dt, i, j - 1) * (F3(u, i + 1, j - 1, k) + F3(u, i, j - 1, k));
    ay += F2(arv, i, j) * 0.25f * (tc1 + tc2);
  }
  advx = ax;
  advy = ay;
}

// ---------------------------------------------------------------------------
// Surface forcing (explicit/time_loop.py:118-164,
// implicit_p0_fixed/forcing/surface.py:20-84) -- 2-D, one cell.
// ---------------------------------------------------------------------------
NPOM_HD void forcing_cell(const Ctx &c, int i, int j) {
  if (c.k.core == NPOM_CORE_IMPLICIT && c.k.wind_forcing) {
    float arg = c.k.two_pi * (F2(north_e, i, j) - 30.0f) / 20.0f;
    P2(wusurf, i, j) = c.k.wind_kf * (1.0f - cosf(arg)) * F2(dum, i, j);
    P2(wvsurf, i, j) = 0.0f;
  }
  if (!interior(c, i, j)) return;
  P2(e_atmos, i, j) = 0.0f;
  P2(vfluxf, i, j) = 0.0f;
  P2(swrad, i, j) = 0.0f;
  const float vf = 0.0f;
  P3(w, i, j, 0) = vf;
  float ts = F3(t, i, j, 0);
  float tatm = ts + c.k.tbias;
  P2(wtsurf, i, j) = F2(wtsurf, i, j) + vf * (tatm - ts - c.k.tbias);
  float ss = F3(s, i, j, 0);
  P2(wssurf, i, j) = vf * (0.0f - ss - c.k.sbias);
}

// ---------------------------------------------------------------------------
// BAROPG (explicit/momentum.py:543-700) for one column; writes drhox/drhoy.
// The k-cumsum accumulates in double like torch's CPU cumsum.
// ---------------------------------------------------------------------------
NPOM_HD void baropg_column(const Ctx &c, int i, int j) {
  const int kb = c.kb, kbm1 = kb - 1;
  if (!interior(c, i, j)) {
    for (int k = 0; k < kb; ++k) {
      P3(drhox, i, j, k) = 0.0f;
      P3(drhoy, i, j, k) = 0.0f;
    }
    return;
  }
  const float ramp = c.ramp;
  for (int comp = 0; comp < 2; ++comp) {
    const int bi = comp == 0 ? i - 1 : i;
    const int bj = comp == 0 ? j : j - 1;
    float *out = comp == 0 ? &P3(drhox, i, j, 0) : &P3(drhoy, i, j, 0);
    float term_dt = F2(dt, i, j) + F2(dt, bi, bj);
    float dt_diff = F2(dt, i, j) - F2(dt, bi, bj);
    float r0 = F3(rho, i, j, 0) - F3(rmean, i, j, 0);
    float rb0 = F3(rho, bi, bj, 0) - F3(rmean, bi, bj, 0);
    float val0 = c.k.half_g * (-F1(zz, 0)) * term_dt * (r0 - rb0);
    float mask = comp == 0 ? F2(dum, i, j) : F2(dvm, i, j);
    float area = comp == 0 ? (F2(dy, i, j) + F2(dy, bi, bj)) : (F2(dx, i, j) + F2(dx, bi, bj));
    float scale = 0.25f * term_dt * mask * area;
    out[0] = val0 * scale * ramp;
    double acc = 0.0;
    float rkm = r0, rbkm = rb0;
    for (int k = 1; k < kbm1; ++k) {
      float rk = F3(rho, i, j, k) - F3(rmean, i, j, k);
      float rbk = F3(rho, bi, bj, k) - F3(rmean, bi, bj, k);
      float zzk = F1(zz, k), zzkm = F1(zz, k - 1);
      float term1 = c.k.quarter_g * (zzkm - zzk) * term_dt * ((rk - rbk) + (rkm - rbkm));
      float term2 = c.k.quarter_g * (zzkm + zzk) * dt_diff * ((rk + rbk) - (rkm + rbkm));
      acc += (double)(term1 + term2);
      float v = val0 + (float)acc;
      out[k] = v * scale * ramp;
      rkm = rk;
      rbkm = rbk;
    }
    for (int k = kbm1; k < kb; ++k) out[k] = 0.0f;
  }
}

// ---------------------------------------------------------------------------
// Smagorinsky viscosity for one column (explicit time_loop.py:10-16,193-233;
// implicit time_loop.py:153-199 with autograd.py strain_magnitude).
// ---------------------------------------------------------------------------
NPOM_HD void smag_column(const Ctx &c, int i, int j) {
  if (!interior(c, i, j)) return;
  const float dxs = F2(dx, i, j), dys = F2(dy, i, j);
  for (int k = 0; k < c.kb - 1; ++k) {
    float du_dx = (F3(u, i + 1, j, k) - F3(u, i, j, k)) / dxs;
    float dv_dy = (F3(v, i, j + 1, k) - F3(v, i, j, k)) / dys;
    float u_term = 0.25f * (F3(u, i, j + 1, k) + F3(u, i + 1, j + 1, k) - F3(u, i, j - 1, k) - F3(u, i + 1, j - 1, k)) / dys;
    float v_term = 0.25f * (F3(v, i + 1, j, k) + F3(v, i + 1, j + 1, k) - F3(v, i - 1, j, k) - F3(v, i - 1, j + 1, k)) / dxs;
    float mag;
    if (c.k.core == NPOM_CORE_EXPLICIT) {
      float cc = (u_term + v_term) * c.k.sqrt_half;
      mag = sqrtf(du_dx * du_dx + dv_dy * dv_dy + cc * cc);
    } else {
      float sh = u_term + v_term;
      mag = sqrtf(du_dx * du_dx + dv_dy * dv_dy + 0.5f * (sh * sh));
    }
    float a = c.k.horcon * dxs * dys * mag;
    if (c.k.core == NPOM_CORE_IMPLICIT && c.k.aam_min > 0.0f) a = fmaxf_t(a, c.k.aam_min);
    P3(aam, i, j, k) = a;
  }
}

// Column phase: BAROPG, Smagorinsky, then the depth integrals of
// advx/advy/drhox/drhoy/aam (time_loop.py:240-258).
NPOM_HD void phase_a2_column(const Ctx &c, int i, int j) {
  baropg_column(c, i, j);
  smag_column(c, i, j);
  float sx = 0.0f, sy = 0.0f, rx = 0.0f, ry = 0.0f, sa = 0.0f;
  for (int k = 0; k < c.kb - 1; ++k) {
    float dzk = F1(dz, k);
    sx += F3(advx, i, j, k) * dzk;
    sy += F3(advy, i, j, k) * dzk;
    rx += F3(drhox, i, j, k) * dzk;
    ry += F3(drhoy, i, j, k) * dzk;
    sa += F3(aam, i, j, k) * dzk;
  }
  P2(adx2d, i, j) = sx;
  P2(ady2d, i, j) = sy;
  P2(drx2d, i, j) = rx;
  P2(dry2d, i, j) = ry;
  P2(aam2d, i, j) = sa;
}

// ---------------------------------------------------------------------------
// ADVAVE, mode 3 (explicit/baroclinic.py:262-494).  Section-1 fluxes feed
// advua, section-2 fluxes feed advva and are what remains stored in
// fluxua/fluxva.  Row 0 / column 0 of fluxua/fluxva are never written by
// the reference and are read back from memory.
// ---------------------------------------------------------------------------
NPOM_HD float advave_tps(const Ctx &c, int i, int j) {
  float d_sum = F2(d, i, j) + F2(d, i - 1, j) + F2(d, i, j - 1) + F2(d, i - 1, j - 1);
  float aam_sum = F2(aam2d, i, j) + F2(aam2d, i, j - 1) + F2(aam2d, i - 1, j) + F2(aam2d, i - 1, j - 1);
  float dy_sum = F2(dy, i, j) + F2(dy, i - 1, j) + F2(dy, i, j - 1) + F2(dy, i - 1, j - 1);
  float dx_sum = F2(dx, i, j) + F2(dx, i - 1, j) + F2(dx, i, j - 1) + F2(dx, i - 1, j - 1);
  float du_dy = (F2(uab, i, j) - F2(uab, i, j - 1)) / dy_sum;
  float dv_dx = (F2(vab, i, j) - F2(vab, i - 1, j)) / dx_sum;
  return 0.25f * d_sum * aam_sum * (du_dy + dv_dx);
}

// section 1 fluxua (i in 1..im-2, j >= 1), stale value elsewhere
NPOM_HD float advave_fluxua1(const Ctx &c, int i, int j) {
  if (i < 1 || j < 1) return F2(fluxua, i, j);
  float t1 = (F2(d, i + 1, j) + F2(d, i, j)) * F2(ua, i + 1, j);
  float t2 = (F2(d, i, j) + F2(d, i - 1, j)) * F2(ua, i, j);
  float f = 0.125f * (t1 + t2) * (F2(ua, i + 1, j) + F2(ua, i, j));
  float diff_u = (F2(uab, i + 1, j) - F2(uab, i, j)) / F2(dx, i, j);
  f -= F2(d, i, j) * 2.0f * F2(aam2d, i, j) * diff_u;
  return f * F2(dy, i, j);
}

// section 1 fluxva (i >= 1, j >= 1)
NPOM_HD float advave_fluxva1(const Ctx &c, int i, int j) {
  if (i < 1 || j < 1) return F2(fluxva, i, j);
  float t1 = (F2(d, i, j) + F2(d, i, j - 1)) * F2(va, i, j);
  float t2 = (F2(d, i - 1, j) + F2(d, i - 1, j - 1)) * F2(va, i - 1, j);
  float f = 0.125f * (t1 + t2) * (F2(ua, i, j) + F2(ua, i, j - 1));
  float dx_sum = F2(dx, i, j) + F2(dx, i - 1, j) + F2(dx, i, j - 1) + F2(dx, i - 1, j - 1);
  return (f - advave_tps(c, i, j)) * 0.25f * dx_sum;
}

// section 2 fluxua (i >= 1, j >= 1)
NPOM_HD float advave_fluxua2(const Ctx &c, int i, int j) {
  if (i < 1 || j < 1) return F2(fluxua, i, j);
  float t1 = (F2(d, i, j) + F2(d, i - 1, j)) * F2(ua, i, j);
  float t2 = (F2(d, i, j - 1) + F2(d, i - 1, j - 1)) * F2(ua, i, j - 1);
  float f = 0.125f * (t1 + t2) * (F2(va, i - 1, j) + F2(va, i, j));
  float dy_sum = F2(dy, i, j) + F2(dy, i - 1, j) + F2(dy, i, j - 1) + F2(dy, i - 1, j - 1);
  return (f - advave_tps(c, i, j)) * 0.25f * dy_sum;
}

// section 2 fluxva (i >= 1, 1 <= j <= jm-2; column jm-1 keeps section 1 * dx)
NPOM_HD float advave_fluxva2(const Ctx &c, int i, int j) {
  if (i < 1 || j < 1) return F2(fluxva, i, j);
  if (j == c.jm - 1) return advave_fluxva1(c, i, j) * F2(dx, i, j);
  float t1 = (F2(d, i, j + 1) + F2(d, i, j)) * F2(va, i, j + 1);
  float t2 = (F2(d, i, j) + F2(d, i, j - 1)) * F2(va, i, j);
  float f = 0.125f * (t1 + t2) * (F2(va, i, j + 1) + F2(va, i, j));
  float diff_v = (F2(vab, i, j + 1) - F2(vab, i, j)) / F2(dy, i, j);
  f -= F2(d, i, j) * 2.0f * F2(aam2d, i, j) * diff_v;
  return f * F2(dx, i, j);
}

struct AdvaveOut {
  float advua, advva, fluxua, fluxva, tps;
  bool write_flux, write_tps;
};

NPOM_HD AdvaveOut advave_cell(const Ctx &c, int i, int j) {
  AdvaveOut o;
  o.advua = 0.0f;
  o.advva = 0.0f;
  if (interior(c, i, j)) {
    o.advua = advave_fluxua1(c, i, j) - advave_fluxua1(c, i - 1, j) + advave_fluxva1(c, i, j + 1) -
              advave_fluxva1(c, i, j);
    o.advva = advave_fluxua2(c, i + 1, j) - advave_fluxua2(c, i, j) + advave_fluxva2(c, i, j) -
              advave_fluxva2(c, i, j - 1);
  }
  o.write_flux = (i >= 1 && j >= 1);
  o.write_tps = o.write_flux;
  if (o.write_flux) {
    o.fluxua = advave_fluxua2(c, i, j);
    o.fluxva = advave_fluxva2(c, i, j);
    o.tps = advave_tps(c, i, j);
  }
  return o;
}

}  // namespace npom
