// npom_mpdata_adjoint.cuh -- reverse mode of B5 with MPDATA tracer advection
// (nadv = 2: ADVT2 and SMOL_ADIF, explicit/tracers.py:571-888), pass by pass.
//
// The step adjoint's plan runs B5 as its forward passes (npom_mpdata.cuh):
// the q2/q2l filter, mass fluxes, per iteration upstream fluxes, forecast
// and antidiffusive fluxes, then the diffusive fluxes and the final update.
// Each pass saves what it overwrites -- state fields or the MPDATA scratch
// arrays, which have cotangent slots of their own (mp_slot) -- and its
// reverse body below sees the pass's inputs restored, the cotangents of its
// outputs in L and scatters into G, with the conventions of
// npom_adjoint.cuh: |x| -> sign(x) (0 at 0), a where() passes the gradient
// only to its kept branch (the antidiffusive flux is 0 where the limiter
// trips), tclim/sclim and the geometry are constants.
#pragma once

#include "npom_adjoint.cuh"
#include "npom_mpdata.cuh"

namespace npom {

#define MPG(tr, arr, o, v) ::npom::aadd(&a.G[mp_slot((tr), (arr))][(o)], (v))
#define MPL(tr, arr, o) (a.L[mp_slot((tr), (arr))][(o)])
#define GA3(name, i, j, k, v) ::npom::aadd(&a.G[NPOM_F_##name][NPOM_I3(c, i, j, k)], (v))
#define GA2(name, i, j, v) ::npom::aadd(&a.G[NPOM_F_##name][NPOM_I2(c, i, j)], (v))
#define LA3(name, i, j, k) (a.L[NPOM_F_##name][NPOM_I3(c, i, j, k)])

NPOM_HD int mp_fld_f(int tr) { return tr == 0 ? NPOM_F_t : NPOM_F_s; }
NPOM_HD int mp_fld_fb(int tr) { return tr == 0 ? NPOM_F_tb : NPOM_F_sb; }
NPOM_HD int mp_fld_ff(int tr) { return tr == 0 ? NPOM_F_uf : NPOM_F_vf; }

// lam * d up(F, in, out) scattered: F into slot (tr, arr) at o, in and out
// into field fbm at oi / oo
NPOM_HD void mp_up_adj(const Adj &a, int tr, int arr, size_t o, float F, float in, float out, float lam, int fbm,
                       size_t oi, size_t oo) {
  if (lam == 0.0f) return;
  const float af = fabsf(F), s = sgnf(F);
  MPG(tr, arr, o, lam * 0.5f * ((1.0f + s) * in + (1.0f - s) * out));
  aadd(&a.G[fbm][oi], lam * 0.5f * (F + af));
  aadd(&a.G[fbm][oo], lam * 0.5f * (F - af));
}

// the q2/q2l filter (phase_b5_filter) of B5, and on the semi-implicit core
// the clamp of kh, km, kq to [0, vmix]: the gradient passes where
// 0 <= x <= vmix
NPOM_HD void mp_filter_adj(const Ctx &c, const Adj &a, int i, int j, int k) {
  if (!is_explicit(c) && c.k.has_vmix) {
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

// mp_init: mass fluxes xm, ym from u, v and dt; zw = w; the ghost level of fb
NPOM_HD void mp_init_adj(const Ctx &c, const Adj &a, int tr, int i, int j, int k) {
  const int kb = c.kb, kbm1 = kb - 1;
  const size_t o = NPOM_I3(c, i, j, k);
  const int fb = mp_fld_fb(tr);
  if (k == kb - 1) aadd(&a.G[fb][NPOM_I3(c, i, j, kbm1 - 1)], a.L[fb][o]);
  else aadd(&a.G[fb][o], a.L[fb][o]);
  const float lx = MPL(tr, 0, o), ly = MPL(tr, 1, o);
  if (i >= 1 && j >= 1 && k < kbm1) {
    const float DY = F2(dy, i - 1, j) + F2(dy, i, j), DT = F2(dt, i - 1, j) + F2(dt, i, j);
    const float U = F3(u, i, j, k);
    GA3(u, i, j, k, lx * (0.25f * DY) * DT);
    GA2(dt, i - 1, j, lx * (0.25f * DY) * U);
    GA2(dt, i, j, lx * (0.25f * DY) * U);
    const float DX = F2(dx, i, j - 1) + F2(dx, i, j), DTy = F2(dt, i, j - 1) + F2(dt, i, j);
    const float V = F3(v, i, j, k);
    GA3(v, i, j, k, ly * (0.25f * DX) * DTy);
    GA2(dt, i, j - 1, ly * (0.25f * DX) * V);
    GA2(dt, i, j, ly * (0.25f * DX) * V);
  }
  GA3(w, i, j, k, MPL(tr, 2, o));
}

// mp_upwind: upstream fluxes of fbmem (fb on the first iteration, ff after)
NPOM_HD void mp_upwind_adj(const Ctx &c, const Adj &a, int tr, int it, int i, int j, int k) {
  const int kb = c.kb, kbm1 = kb - 1, im = c.im, jm = c.jm;
  const size_t o = NPOM_I3(c, i, j, k);
  const MpScratch m = mp_scratch(c, tr);
  const int fbm = it == 1 ? mp_fld_fb(tr) : mp_fld_ff(tr);
  const float *fbmem = c.F[fbm];
  const float lx = MPL(tr, 3, o), ly = MPL(tr, 4, o), lz = MPL(tr, 5, o);
  if (i >= 1 && j >= 1 && k < kbm1) {
    const size_t ox = NPOM_I3(c, i - 1, j, k), oy = NPOM_I3(c, i, j - 1, k);
    mp_up_adj(a, tr, 0, o, m.xm[o], fbmem[ox], fbmem[o], lx, fbm, ox, o);
    mp_up_adj(a, tr, 1, o, m.ym[o], fbmem[oy], fbmem[o], ly, fbm, oy, o);
  } else {
    // not written: the old values pass through
    MPG(tr, 3, o, lx);
    MPG(tr, 4, o, ly);
  }
  const bool in_xy = i >= 1 && i <= im - 2 && j >= 1 && j <= jm - 2;
  if (k == 0) {
    if (it == 1 && in_xy && lz != 0.0f) {
      const int ff = mp_fld_f(tr);
      const float art = F2(art, i, j);
      GA3(w, i, j, 0, lz * c.F[ff][o] * art);
      aadd(&a.G[ff][o], lz * F3(w, i, j, 0) * art);
    }
  } else if (k == kb - 1) {
    // zf = 0 there
  } else if (in_xy) {
    const float art = F2(art, i, j);
    const size_t ob = NPOM_I3(c, i, j, k - 1);
    mp_up_adj(a, tr, 2, o, m.zw[o], fbmem[o], fbmem[ob], lz * art, fbm, o, ob);
  } else {
    MPG(tr, 5, o, lz);
  }
}

// mp_forecast: ff = ((told fbmem - dti2 div) / tnew) * fsm on the interior,
// ff * fsm elsewhere; told uses etb on the first iteration, etf after
NPOM_HD void mp_forecast_adj(const Ctx &c, const Adj &a, int tr, int it, int i, int j, int k) {
  const int kbm1 = c.kb - 1;
  const size_t o = NPOM_I3(c, i, j, k);
  const MpScratch m = mp_scratch(c, tr);
  const int ff = mp_fld_ff(tr), fbm = it == 1 ? mp_fld_fb(tr) : ff;
  const float lam = a.L[ff][o];
  if (lam == 0.0f) return;
  const float lv = lam * F2(fsm, i, j);
  if (interior(c, i, j) && k < kbm1) {
    const int eta = it == 1 ? NPOM_F_etb : NPOM_F_etf;
    const float horiz = m.xf[NPOM_I3(c, i + 1, j, k)] - m.xf[o] + m.yf[NPOM_I3(c, i, j + 1, k)] - m.yf[o];
    const float vert = (m.zf[o] - m.zf[o + 1]) / F1(dz, k);
    const float div = horiz + vert;
    const float art = F2(art, i, j);
    const float told = (F2(h, i, j) + c.F[eta][NPOM_I2(c, i, j)]) * art;
    const float tnew = (F2(h, i, j) + F2(etf, i, j)) * art;
    const float den = tnew + 1e-20f;
    const float fbv = c.F[fbm][o];
    const float v = (told * fbv - c.k.dti2 * div) / den;
    aadd(&a.G[fbm][o], lv * told / den);
    aadd(&a.G[eta][NPOM_I2(c, i, j)], lv * fbv * art / den);
    GA2(etf, i, j, -lv * v / den * art);
    const float ld = -lv * c.k.dti2 / den;
    MPG(tr, 3, NPOM_I3(c, i + 1, j, k), ld);
    MPG(tr, 3, o, -ld);
    MPG(tr, 4, NPOM_I3(c, i, j + 1, k), ld);
    MPG(tr, 4, o, -ld);
    const float lz = ld / F1(dz, k);
    MPG(tr, 5, o, lz);
    MPG(tr, 5, o + 1, -lz);
  } else {
    aadd(&a.G[ff][o], lv);
  }
}

// one antidiffusive flux: fn = (|F| - F2) * mol * sw with F2 = dti2 F^2 2 / D
// (horizontal, two) or dti2 F^2 / D (vertical), as the forward evaluates
// them, mol = (p - q) / (p + q + eps), 0 where fc or fp < vmin or
// |F| < |F2|; lam * d fn scattered to F (slot), the dt terms of D (weight wd
// each), p and q
NPOM_HD void mp_antiflux_adj(const Ctx &c, const Adj &a, int tr, int arr, size_t o, float F, float D, bool two,
                             float p, float q, float fc, float fp, float lam, int ff, size_t op, size_t oq,
                             size_t odt1, size_t odt2, float wd) {
  const float vmin = 1.0e-9f, eps = 1.0e-14f, sw = c.k.sw, dti2 = c.k.dti2;
  if (lam == 0.0f) return;
  const float mag = fabsf(F);
  const float F2 = two ? dti2 * (F * F) * 2.0f / D : dti2 * (F * F) / D;
  const float c2 = two ? 2.0f * dti2 : dti2;
  if ((fc < vmin) || (fp < vmin) || (fabsf(mag) < fabsf(F2))) return;
  const float S = p + q + eps;
  const float mol = (p - q) / S;
  const float lm = lam * mol * sw;
  MPG(tr, arr, o, lm * sgnf(F) - lm * (2.0f * c2 * F / D));
  const float ld = lm * F2 / D * wd;  // d fn / d D = mol sw F2 / D
  aadd(&a.G[NPOM_F_dt][odt1], ld);
  if (odt2 != odt1) aadd(&a.G[NPOM_F_dt][odt2], ld);
  const float lr = lam * (mag - F2) * sw / (S * S);
  aadd(&a.G[ff][op], lr * (2.0f * q + eps));
  aadd(&a.G[ff][oq], lr * (-2.0f * p - eps));
}

// mp_antidiff: antidiffusive mass fluxes from the masked forecast
NPOM_HD void mp_antidiff_adj(const Ctx &c, const Adj &a, int tr, int i, int j, int k) {
  const int kbm1 = c.kb - 1, im = c.im, jm = c.jm;
  const size_t o = NPOM_I3(c, i, j, k);
  const MpScratch m = mp_scratch(c, tr);
  const int ff = mp_fld_ff(tr);
  const float *f = c.F[ff];
  const float eps = 1.0e-14f;
  const float lx = MPL(tr, 0, o), ly = MPL(tr, 1, o), lz = MPL(tr, 2, o);
  if (k >= kbm1) {
    MPG(tr, 0, o, lx);
    MPG(tr, 1, o, ly);
    MPG(tr, 2, o, lz);
    return;
  }
  const float fc = f[o];
  if (i >= 1 && j >= 1 && j <= jm - 2) {
    const size_t ox = NPOM_I3(c, i - 1, j, k);
    const float D = F2(aru, i, j) * (F2(dt, i - 1, j) + F2(dt, i, j)) + eps;
    mp_antiflux_adj(c, a, tr, 0, o, m.xm[o], D, true, fc, f[ox], fc, f[ox], lx, ff, o, ox, NPOM_I2(c, i - 1, j),
                    NPOM_I2(c, i, j), F2(aru, i, j));
  } else {
    MPG(tr, 0, o, lx);
  }
  if (i >= 1 && i <= im - 2 && j >= 1) {
    const size_t oy = NPOM_I3(c, i, j - 1, k);
    const float D = F2(arv, i, j) * (F2(dt, i, j - 1) + F2(dt, i, j)) + eps;
    mp_antiflux_adj(c, a, tr, 1, o, m.ym[o], D, true, fc, f[oy], fc, f[oy], ly, ff, o, oy, NPOM_I2(c, i, j - 1),
                    NPOM_I2(c, i, j), F2(arv, i, j));
  } else {
    MPG(tr, 1, o, ly);
  }
  if (interior(c, i, j) && k >= 1) {
    // mol = (fp - fc) / (fc + fp + eps); dD/ddt = dzz(k-1)
    const float fp = f[o - 1];
    const float D = F1(dzz, k - 1) * F2(dt, i, j) + eps;
    mp_antiflux_adj(c, a, tr, 2, o, m.zw[o], D, false, fp, fc, fc, fp, lz, ff, o - 1, o, NPOM_I2(c, i, j),
                    NPOM_I2(c, i, j), F1(dzz, k - 1));
  } else {
    MPG(tr, 2, o, lz);
  }
}

// mp_diffusion: horizontal diffusive fluxes of fb - fclim
NPOM_HD void mp_diffusion_adj(const Ctx &c, const Adj &a, int tr, int i, int j, int k) {
  const size_t o = NPOM_I3(c, i, j, k);
  const float lx = MPL(tr, 3, o), ly = MPL(tr, 4, o);
  if (i < 1 || j < 1 || k >= c.kb - 1) {
    MPG(tr, 3, o, lx);
    MPG(tr, 4, o, ly);
    return;
  }
  const int fbi = mp_fld_fb(tr);
  const float *fb = c.F[fbi], *fcl = c.F[tr == 0 ? NPOM_F_tclim : NPOM_F_sclim];
  const size_t ox = NPOM_I3(c, i - 1, j, k), oy = NPOM_I3(c, i, j - 1, k);
  const float an = fb[o] - fcl[o];
  if (lx != 0.0f) {
    const float xm = 0.5f * (F3(aam, i, j, k) + F3(aam, i - 1, j, k));
    const float fd = an - (fb[ox] - fcl[ox]);
    const float K = (F2(h, i, j) + F2(h, i - 1, j)) * c.k.tprni * F2(dum, i, j) * (F2(dy, i, j) + F2(dy, i - 1, j)) *
                    0.5f / (F2(dx, i, j) + F2(dx, i - 1, j));
    const float la = -lx * fd * K * 0.5f;
    GA3(aam, i, j, k, la);
    GA3(aam, i - 1, j, k, la);
    const float lf = -lx * xm * K;
    aadd(&a.G[fbi][o], lf);
    aadd(&a.G[fbi][ox], -lf);
  }
  if (ly != 0.0f) {
    const float ym = 0.5f * (F3(aam, i, j, k) + F3(aam, i, j - 1, k));
    const float fd = an - (fb[oy] - fcl[oy]);
    const float K = (F2(h, i, j) + F2(h, i, j - 1)) * c.k.tprni * F2(dvm, i, j) * (F2(dx, i, j) + F2(dx, i, j - 1)) *
                    0.5f / (F2(dy, i, j) + F2(dy, i, j - 1));
    const float la = -ly * fd * K * 0.5f;
    GA3(aam, i, j, k, la);
    GA3(aam, i, j - 1, k, la);
    const float lf = -ly * ym * K;
    aadd(&a.G[fbi][o], lf);
    aadd(&a.G[fbi][oy], -lf);
  }
}

// mp_finish: ff -= dti2 * div(diffusive fluxes) / tnew on the interior
NPOM_HD void mp_finish_adj(const Ctx &c, const Adj &a, int tr, int i, int j, int k) {
  const size_t o = NPOM_I3(c, i, j, k);
  const int ff = mp_fld_ff(tr);
  const float lam = a.L[ff][o];
  if (lam == 0.0f) return;
  aadd(&a.G[ff][o], lam);
  if (!interior(c, i, j) || k >= c.kb - 1) return;
  const MpScratch m = mp_scratch(c, tr);
  const float art = F2(art, i, j);
  const float tnew = (F2(h, i, j) + F2(etf, i, j)) * art;
  const float den = tnew + 1e-20f;
  const float hd = m.xf[NPOM_I3(c, i + 1, j, k)] - m.xf[o] + m.yf[NPOM_I3(c, i, j + 1, k)] - m.yf[o];
  const float l2 = -lam * c.k.dti2 / den;
  MPG(tr, 3, NPOM_I3(c, i + 1, j, k), l2);
  MPG(tr, 3, o, -l2);
  MPG(tr, 4, NPOM_I3(c, i, j + 1, k), l2);
  MPG(tr, 4, o, -l2);
  GA2(etf, i, j, lam * c.k.dti2 * hd / (den * den) * art);
}

// the reverse of plan phase ph (AP_MQ .. AP_MFIN) at point (i, j, k);
// it: the iteration of AP_MUP / AP_MFC / AP_MAD
NPOM_HD void mp_phase_adj(const Ctx &c, const Adj &a, int ph, int it, int i, int j, int k) {
  if (ph == AP_MQ) {
    mp_filter_adj(c, a, i, j, k);
    return;
  }
  for (int tr = 0; tr < 2; ++tr) {
    switch (ph) {
      case AP_MINIT: mp_init_adj(c, a, tr, i, j, k); break;
      case AP_MUP: mp_upwind_adj(c, a, tr, it, i, j, k); break;
      case AP_MFC: mp_forecast_adj(c, a, tr, it, i, j, k); break;
      case AP_MAD: mp_antidiff_adj(c, a, tr, i, j, k); break;
      case AP_MDIF: mp_diffusion_adj(c, a, tr, i, j, k); break;
      case AP_MFIN: mp_finish_adj(c, a, tr, i, j, k); break;
    }
  }
}

// the forward pass of plan phase ph (npom_mpdata.cuh)
NPOM_HD int mp_pass_of(int ph) {
  switch (ph) {
    case AP_MQ: return MP_FILTER;
    case AP_MINIT: return MP_INIT;
    case AP_MUP: return MP_UPWIND;
    case AP_MFC: return MP_FORECAST;
    case AP_MAD: return MP_ANTIDIFF;
    case AP_MDIF: return MP_DIFFUSION;
    default: return MP_FINISH;
  }
}

#undef MPG
#undef MPL
#undef GA3
#undef GA2
#undef LA3

}  // namespace npom
