// npom_host.cuh -- host-side construction of the step context from the C
// ABI structs (shared by the CUDA library and the CPU phase emulator used by
// the tests).
#pragma once

#include <cmath>
#include <cstring>

#include "npom_phases_int.cuh"

namespace npom {

inline Consts make_consts(const npom_params &p) {
  Consts k;
  std::memset(&k, 0, sizeof(k));
  k.dti2 = (float)p.dti2;
  k.dte2 = (float)p.dte2;
  k.two_dti2 = (float)(2.0 * p.dti2);
  k.neg_dti2 = (float)(-p.dti2);
  k.neg_two_dti2 = (float)(-2.0 * p.dti2);
  k.four_dte = (float)(4.0 * p.dte);
  k.four_dti = (float)(4.0 * p.dti);
  k.two_dti = (float)(2.0 * p.dti);
  k.dti = (float)p.dti;
  k.ispi = (float)p.ispi;
  k.isp2i = (float)p.isp2i;
  k.smoth = (float)p.smoth;
  k.half_smoth = (float)(0.5 * p.smoth);
  k.quarter_smoth = (float)(0.25 * p.smoth);
  k.etf_mid = (float)(0.5 * (1.0 - 0.5 * p.smoth));
  k.horcon = (float)p.horcon;
  k.umol = (float)p.umol;
  k.two_umol = (float)(2.0 * p.umol);
  k.tprni = (float)p.tprni;
  k.small = (float)p.small;
  k.kappa = (float)p.kappa;
  k.rhoref = (float)p.rhoref;
  k.tbias = (float)p.tbias;
  k.sbias = (float)p.sbias;
  k.aam_min = (float)p.aam_min;
  k.alpha = (float)p.alpha;
  k.one_m_2alpha = (float)(1.0 - 2.0 * p.alpha);
  k.half_g = (float)(0.5 * p.grav);
  k.quarter_g = (float)(0.25 * p.grav);
  k.g_eighth = (float)(p.grav * 0.125);
  k.grav = (float)p.grav;
  k.g_rhoref = (float)(p.grav * p.rhoref);
  k.g2x2 = (float)((p.grav * p.grav) * 2.0);
  k.sqrt_half = (float)std::sqrt(0.5);
  k.prof_const1 = (float)std::pow(16.6, 2.0 / 3.0);
  k.prof_gg0 = (float)std::pow(15.8 * 100.0, 2.0 / 3.0);
  k.surfl = 2.0e5f;
  k.profq_pom08 = p.profq_form == NPOM_PROFQ_POM08 ? 1 : 0;
  k.kappa_zsh = (float)(p.kappa * p.zsh);
  k.obc_seamount = p.obc_form == NPOM_OBC_SEAMOUNT ? 1 : 0;
  k.obc_coastal = (p.obc_form == NPOM_OBC_COASTAL || p.obc_form == NPOM_OBC_JZB) ? 1 : 0;
  k.obc_jzb = p.obc_form == NPOM_OBC_JZB ? 1 : 0;
  k.sea_implicit = (p.obc_form == NPOM_OBC_SEAMOUNT && p.core == NPOM_CORE_IMPLICIT) ? 1 : 0;
  k.periodic_x = p.periodic_x ? 1 : 0;
  // coastal_boundary.py:9-10: (29.03225806451612*3.1416/180) in double
  // the policies' M2 angular speeds (rad/h) as they write them
  k.tide_w = k.obc_jzb ? 28.98410424 * 3.1416 / 180.0 : 29.03225806451612 * 3.1416 / 180.0;
  k.dte_d = p.dte;
  // coastal_compat.py:4-16
  k.zsh_cbc = 0.01f;
  k.z0b_cbc = k.obc_jzb ? 0.01f : 0.005f;
  k.hc_cbc = 0.05f;
  k.cbcmin = 0.0025f;
  k.cbcmax = 1.0f;
  k.wind_kf = (float)(-(p.wind_tau0 / p.rhoref));
  k.two_pi = (float)(2.0 * p.pi);
  k.hmax = (float)p.hmax;
  k.rfe = (float)p.rfe;
  k.rfw = (float)p.rfw;
  k.rfn = (float)p.rfn;
  k.rfs = (float)p.rfs;
  k.vmaxl = (float)p.vmaxl;
  k.vmix = (float)p.vmix;
  k.bshap = p.barotropic_shapiro;
  k.tshap = p.tracer_shapiro;
  k.vshap = p.velocity_shapiro;
  k.bshap_q = (float)(p.barotropic_shapiro / 4.0);
  k.tshap_q = (float)(p.tracer_shapiro / 4.0);
  k.vshap_q = (float)(p.velocity_shapiro / 4.0);
  k.implicit_coeff = (float)(4.0 * (p.dti * p.dti) * p.grav * p.alpha);
  k.inverse_scale = (float)p.inverse_scale;
  k.isplit = p.isplit;
  k.ispadv = p.ispadv;
  k.nbct = p.nbct;
  k.nbcs = p.nbcs;
  k.ntp = p.ntp;
  k.mode = p.mode;
  k.core = p.core;
  k.wind_forcing = p.wind_forcing;
  k.has_vmix = p.has_vmix;
  k.nadv = p.nadv;
  k.nitera = p.nitera;
  k.sw = (float)p.sw;
  k.eta_max_iter = p.eta_max_iter;
  k.eta_precond = p.eta_precond;
  k.eta_tol = p.eta_tol;
  k.eta_rel_tol = p.eta_rel_tol;
  return k;
}

inline bool check_args(const npom_params *p, float *const *fields, const npom_workspace *ws) {
  if (!p || !fields || !ws) return false;
  if (p->im < 3 || p->jm < 3 || p->kb < 3 || p->kb > KMAX) return false;
  if (p->core == NPOM_CORE_EXPLICIT && (p->isplit < 3 || p->ispadv < 1)) return false;
  if (p->velocity_shapiro != 0.0) return false;  // not supported (production value is 0)
  if (p->nbct < 1 || p->nbct > 4 || p->nbcs < 1 || p->nbcs > 4 || p->ntp < 1 || p->ntp > 5) return false;
  for (int f = 0; f < NPOM_NFIELDS; ++f)
    if (!fields[f]) return false;
  if (!ws->partials || !ws->sync || !ws->status || !ws->cg_iters) return false;
  if (p->nadv != 1 && (p->nadv != 2 || !ws->mp3d || p->nitera < 1)) return false;
  // the seamount policy on the explicit core; the tide policies on either
  // core (the semi-implicit one with its Shapiro filter at 0, as their
  // installers set it)
  const bool tide_policy = p->obc_form == NPOM_OBC_COASTAL || p->obc_form == NPOM_OBC_JZB;
  if (p->obc_form != NPOM_OBC_NATIVE &&
      ((p->obc_form != NPOM_OBC_SEAMOUNT && !tide_policy) || p->im < 6 || p->jm < 6 ||
       (tide_policy && !ws->tide) ||
       (p->obc_form == NPOM_OBC_SEAMOUNT && p->core == NPOM_CORE_IMPLICIT && !ws->robin) ||
       (p->core == NPOM_CORE_IMPLICIT && p->barotropic_shapiro != 0.0)))
    return false;
  if (p->periodic_x &&
      (p->periodic_x != 1 || p->core != NPOM_CORE_IMPLICIT || p->obc_form != NPOM_OBC_NATIVE || p->nadv != 1 ||
       p->im < 8))
    return false;
  for (int w = 0; w < NPOM_NWS; ++w)
    if (!ws->buf[w]) return false;
  return true;
}

inline Ctx make_ctx(const npom_params *p, float *const *fields, const npom_workspace *ws) {
  Ctx c;
  std::memset(&c, 0, sizeof(c));
  c.im = p->im;
  c.jm = p->jm;
  c.kb = p->kb;
  for (int f = 0; f < NPOM_NFIELDS; ++f) c.F[f] = fields[f];
  for (int w = 0; w < NPOM_NWS; ++w) c.W[w] = ws->buf[w];
  c.partials = ws->partials;
  c.sync = ws->sync;
  c.status = ws->status;
  c.cg_iters = ws->cg_iters;
  c.mp3d = ws->mp3d;
  c.tide = ws->tide;
  c.robin = ws->robin;
  c.k = make_consts(*p);
  c.ramp = 1.0f;
  c.do_internal = 1;
  c.tune = p->tuning;
  return c;
}

inline float ramp_of(const npom_params *p, double time) {
  if (!p->lramp) return 1.0f;
  float r = (float)time / (float)p->period;
  return r > 1.0f ? 1.0f : r;
}

}  // namespace npom
