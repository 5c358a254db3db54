// npom_mpdata.cuh -- MPDATA tracer advection (nadv = 2): the Smolarkiewicz
// iterative upstream scheme ADVT2 with its antidiffusive velocities SMOL_ADIF
// (explicit/tracers.py:571-888), for T (into uf) and S (into vf).
//
// One pass per body, over points (i, j, k).  The passes of one tracer:
//   mp_init      mass fluxes xm/ym from u/v, zw = w, the ghost level of fb
//   mp_upwind    (nitera times) upstream fluxes xf/yf/zf of fbmem
//   mp_forecast  the forecast into ff, then ff *= fsm everywhere (SMOL_ADIF's
//                first statement)
//   mp_antidiff  antidiffusive mass fluxes from ff (in place in xm/ym/zw)
//   mp_diffusion horizontal diffusive fluxes of fb - fclim into xf/yf
//   mp_finish    ff -= dti2 * div / volume on the interior
// fbmem is fb on the first iteration and ff afterwards.  Every expression
// keeps the reference's evaluation order.
#pragma once

#include "npom_phases_int.cuh"

namespace npom {

// per-tracer scratch, each (im, jm, kb)
struct MpScratch {
  float *xm, *ym, *zw, *xf, *yf, *zf;
};

NPOM_HD void mp_init(const Ctx &c, const MpScratch &m, float *fb, int i, int j, int k) {
  const int kb = c.kb, kbm1 = kb - 1;
  const size_t o = NPOM_I3(c, i, j, k);
  float xm = 0.0f, ym = 0.0f;
  if (i >= 1 && j >= 1 && k < kbm1) {
    xm = 0.25f * (F2(dy, i - 1, j) + F2(dy, i, j)) * (F2(dt, i - 1, j) + F2(dt, i, j)) * F3(u, i, j, k);
    ym = 0.25f * (F2(dx, i, j - 1) + F2(dx, i, j)) * (F2(dt, i, j - 1) + F2(dt, i, j)) * F3(v, i, j, k);
  }
  m.xm[o] = xm;
  m.ym[o] = ym;
  m.zw[o] = F3(w, i, j, k);
  if (k == kb - 1) fb[o] = ld(fb + NPOM_I3(c, i, j, kbm1 - 1));
}

NPOM_HD float mp_up(float flux, float in, float out) {
  const float af = fabsf(flux);
  return 0.5f * ((flux + af) * in + (flux - af) * out);
}

// upstream fluxes of fbmem; first: the first iteration (surface flux w f art)
NPOM_HD void mp_upwind(const Ctx &c, const MpScratch &m, const float *fbmem, const float *f, bool first, int i,
                       int j, int k) {
  const int kb = c.kb, kbm1 = kb - 1, im = c.im, jm = c.jm;
  const size_t o = NPOM_I3(c, i, j, k);
  if (i >= 1 && j >= 1 && k < kbm1) {
    m.xf[o] = mp_up(ld(m.xm + o), ld(fbmem + NPOM_I3(c, i - 1, j, k)), ld(fbmem + o));
    m.yf[o] = mp_up(ld(m.ym + o), ld(fbmem + NPOM_I3(c, i, j - 1, k)), ld(fbmem + o));
  }
  const bool in_xy = i >= 1 && i <= im - 2 && j >= 1 && j <= jm - 2;
  if (k == 0) {
    m.zf[o] = (first && in_xy) ? F3(w, i, j, 0) * ld(f + o) * F2(art, i, j) : 0.0f;
  } else if (k == kb - 1) {
    m.zf[o] = 0.0f;
  } else if (in_xy) {
    const float z = mp_up(ld(m.zw + o), ld(fbmem + o), ld(fbmem + NPOM_I3(c, i, j, k - 1)));
    m.zf[o] = z * F2(art, i, j);
  }
}

// forecast on the interior, then the mask of every point; ff may alias
// fbmem (both are read and written at this point only)
NPOM_HD void mp_forecast(const Ctx &c, const MpScratch &m, const float *fbmem, float *ff, const float *eta, int i,
                         int j, int k) {
  const int kbm1 = c.kb - 1;
  const size_t o = NPOM_I3(c, i, j, k);
  float v = ld(ff + o);
  if (interior(c, i, j) && k < kbm1) {
    const float horiz = ld(m.xf + NPOM_I3(c, i + 1, j, k)) - ld(m.xf + o) + ld(m.yf + NPOM_I3(c, i, j + 1, k)) -
                        ld(m.yf + o);
    const float vert = (ld(m.zf + o) - ld(m.zf + o + 1)) / F1(dz, k);
    const float div = horiz + vert;
    const float art = F2(art, i, j);
    const float told = (F2(h, i, j) + ld(eta + NPOM_I2(c, i, j))) * art;
    const float tnew = (F2(h, i, j) + F2(etf, i, j)) * art;
    v = (told * ld(fbmem + o) - c.k.dti2 * div) / (tnew + 1e-20f);
  }
  ff[o] = v * F2(fsm, i, j);
}

// antidiffusive mass fluxes from the masked forecast (SMOL_ADIF)
NPOM_HD void mp_antidiff(const Ctx &c, const MpScratch &m, const float *ff, int i, int j, int k) {
  const int kbm1 = c.kb - 1, im = c.im, jm = c.jm;
  const float vmin = 1.0e-9f, eps = 1.0e-14f, sw = c.k.sw, dti2 = c.k.dti2;
  const size_t o = NPOM_I3(c, i, j, k);
  if (k >= kbm1) return;
  const float fc = ld(ff + o);
  if (i >= 1 && j >= 1 && j <= jm - 2) {
    const float fp = ld(ff + NPOM_I3(c, i - 1, j, k));
    const float flux = ld(m.xm + o);
    const float udx = fabsf(flux);
    const float u2dt = dti2 * (flux * flux) * 2.0f / (F2(aru, i, j) * (F2(dt, i - 1, j) + F2(dt, i, j)) + eps);
    const float mol = (fc - fp) / (fp + fc + eps);
    const float fn = (udx - u2dt) * mol * sw;
    m.xm[o] = ((fc < vmin) || (fp < vmin) || (fabsf(udx) < fabsf(u2dt))) ? 0.0f : fn;
  }
  if (i >= 1 && i <= im - 2 && j >= 1) {
    const float fp = ld(ff + NPOM_I3(c, i, j - 1, k));
    const float flux = ld(m.ym + o);
    const float vdy = fabsf(flux);
    const float v2dt = dti2 * (flux * flux) * 2.0f / (F2(arv, i, j) * (F2(dt, i, j - 1) + F2(dt, i, j)) + eps);
    const float mol = (fc - fp) / (fp + fc + eps);
    const float fn = (vdy - v2dt) * mol * sw;
    m.ym[o] = ((fc < vmin) || (fp < vmin) || (fabsf(vdy) < fabsf(v2dt))) ? 0.0f : fn;
  }
  if (interior(c, i, j) && k >= 1) {
    const float fp = ld(ff + o - 1);
    const float flux = ld(m.zw + o);
    const float wdz = fabsf(flux);
    const float w2dt = dti2 * (flux * flux) / (F1(dzz, k - 1) * F2(dt, i, j) + eps);
    const float mol = (fp - fc) / (fc + fp + eps);
    const float fn = (wdz - w2dt) * mol * sw;
    m.zw[o] = ((fc < vmin) || (fp < vmin) || (fabsf(wdz) < fabsf(w2dt))) ? 0.0f : fn;
  }
}

// horizontal diffusive fluxes of the anomaly fb - fclim
NPOM_HD void mp_diffusion(const Ctx &c, const MpScratch &m, const float *fb, const float *fclim, int i, int j,
                          int k) {
  if (i < 1 || j < 1 || k >= c.kb - 1) return;
  const size_t o = NPOM_I3(c, i, j, k), ox = NPOM_I3(c, i - 1, j, k), oy = NPOM_I3(c, i, j - 1, k);
  const float an = ld(fb + o) - ld(fclim + o);
  {
    const float xm = 0.5f * (F3(aam, i, j, k) + F3(aam, i - 1, j, k));
    const float fd = an - (ld(fb + ox) - ld(fclim + ox));
    m.xf[o] = -xm * (F2(h, i, j) + F2(h, i - 1, j)) * c.k.tprni * fd * F2(dum, i, j) *
              (F2(dy, i, j) + F2(dy, i - 1, j)) * 0.5f / (F2(dx, i, j) + F2(dx, i - 1, j));
  }
  {
    const float ym = 0.5f * (F3(aam, i, j, k) + F3(aam, i, j - 1, k));
    const float fd = an - (ld(fb + oy) - ld(fclim + oy));
    m.yf[o] = -ym * (F2(h, i, j) + F2(h, i, j - 1)) * c.k.tprni * fd * F2(dvm, i, j) *
              (F2(dx, i, j) + F2(dx, i, j - 1)) * 0.5f / (F2(dy, i, j) + F2(dy, i, j - 1));
  }
}

// the passes of B5 with nadv 2 at one point: the q2/q2l filter, then ADVT2
// for T into uf and S into vf (pass < 0: the filter)
enum MpPass { MP_FILTER = 0, MP_INIT, MP_UPWIND, MP_FORECAST, MP_ANTIDIFF, MP_DIFFUSION, MP_FINISH };

NPOM_HD MpScratch mp_scratch(const Ctx &c, int tracer) {
  const size_t n3 = (size_t)c.im * c.jm * c.kb;
  float *b = c.mp3d + (size_t)tracer * 6 * n3;
  MpScratch m;
  m.xm = b;
  m.ym = b + n3;
  m.zw = b + 2 * n3;
  m.xf = b + 3 * n3;
  m.yf = b + 4 * n3;
  m.zf = b + 5 * n3;
  return m;
}

NPOM_HD void mp_finish(const Ctx &c, const MpScratch &m, float *ff, int i, int j, int k);

NPOM_HD void phase_b5_mpdata_point(const Ctx &c, int pass, int itera, int i, int j, int k) {
  if (pass == MP_FILTER) {
    phase_b5_filter(c, i, j, k);
    return;
  }
  for (int tr = 0; tr < 2; ++tr) {
    const MpScratch m = mp_scratch(c, tr);
    float *f = c.F[tr == 0 ? NPOM_F_t : NPOM_F_s];
    float *fb = c.F[tr == 0 ? NPOM_F_tb : NPOM_F_sb];
    const float *fclim = c.F[tr == 0 ? NPOM_F_tclim : NPOM_F_sclim];
    float *ff = c.F[tr == 0 ? NPOM_F_uf : NPOM_F_vf];
    const float *fbmem = itera == 1 ? fb : ff;
    switch (pass) {
      case MP_INIT: mp_init(c, m, fb, i, j, k); break;
      case MP_UPWIND: mp_upwind(c, m, fbmem, f, itera == 1, i, j, k); break;
      case MP_FORECAST: mp_forecast(c, m, fbmem, ff, c.F[itera == 1 ? NPOM_F_etb : NPOM_F_etf], i, j, k); break;
      case MP_ANTIDIFF: mp_antidiff(c, m, ff, i, j, k); break;
      case MP_DIFFUSION: mp_diffusion(c, m, fb, fclim, i, j, k); break;
      case MP_FINISH: mp_finish(c, m, ff, i, j, k); break;
    }
  }
}

NPOM_HD void mp_finish(const Ctx &c, const MpScratch &m, float *ff, int i, int j, int k) {
  if (!interior(c, i, j) || k >= c.kb - 1) return;
  const size_t o = NPOM_I3(c, i, j, k);
  const float tnew = (F2(h, i, j) + F2(etf, i, j)) * F2(art, i, j);
  const float hd = ld(m.xf + NPOM_I3(c, i + 1, j, k)) - ld(m.xf + o) + ld(m.yf + NPOM_I3(c, i, j + 1, k)) -
                   ld(m.yf + o);
  ff[o] = ld(ff + o) - c.k.dti2 * hd / (tnew + 1e-20f);
}

}  // namespace npom
