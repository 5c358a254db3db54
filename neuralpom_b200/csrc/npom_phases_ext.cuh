// npom_phases_ext.cuh -- external (2-D) mode of both cores.
//
//  * implicit: barotropic predictor, transport/RHS, elliptic operator and
//    preconditioners of the PCG free-surface solve, corrector, time filter
//    (implicit_p0_fixed/core.py:121-943, time_loop.py:243-387,
//    boundary/closed_basin.py:27-98);
//  * explicit: one external substep split into the phases of the fused
//    subcycle kernel (explicit/time_loop.py:275-431, baroclinic.py:496-571).
#pragma once

#include "npom_phases_a.cuh"

namespace npom {

// ---------------------------------------------------------------------------
// Phase A3 (2-D cell, both cores): rho round trip of BAROPG, ADVAVE,
// adx2d/ady2d -= advua/advva, egf and provisional utf/vtf; implicit core
// also stores d_baro and the predictor (u*, v*) with bcond 2.
// ---------------------------------------------------------------------------
NPOM_HD void bcond2_jzb(const Ctx &c, int i, int j, float &uaf, float &vaf);

NPOM_HD void phase_a3_cell(const Ctx &c, int i, int j) {
  const int im = c.im, jm = c.jm;
  // rho = (rho - rmean) + rmean (momentum.py:554,698)
  for (int k = 0; k < c.kb; ++k) {
    float rm = F3(rmean, i, j, k);
    P3(rho, i, j, k) = (F3(rho, i, j, k) - rm) + rm;
  }
  AdvaveOut o = advave_cell(c, i, j);
  P2(advua, i, j) = o.advua;
  P2(advva, i, j) = o.advva;
  if (o.write_flux) {
    P2(fluxua, i, j) = o.fluxua;
    P2(fluxva, i, j) = o.fluxva;
  }
  if (o.write_tps) P2(tps, i, j) = o.tps;
  float adx = F2(adx2d, i, j) - o.advua;
  float ady = F2(ady2d, i, j) - o.advva;
  P2(adx2d, i, j) = adx;
  P2(ady2d, i, j) = ady;
  P2(egf, i, j) = F2(el, i, j) * c.k.ispi;
  if (i >= 1) P2(utf, i, j) = F2(ua, i, j) * (F2(d, i, j) + F2(d, i - 1, j)) * c.k.isp2i;
  if (j >= 1) P2(vtf, i, j) = F2(va, i, j) * (F2(d, i, j) + F2(d, i, j - 1)) * c.k.isp2i;
  if (c.k.core != NPOM_CORE_IMPLICIT) return;

  PW2(d_baro, i, j) = F2(h, i, j) + F2(elb, i, j);
  // predictor (core.py:795-845) then closed-basin bcond 2 (closed_basin.py:261-272)
  float us = 0.0f, vs = 0.0f, den_u = 0.0f, den_v = 0.0f;
  if (interior(c, i, j)) {
    const float g4 = c.k.quarter_g, al = c.k.alpha, a12 = c.k.one_m_2alpha;
    float cor_u = 0.25f * (F2(cor, i, j) * F2(d, i, j) * (F2(va, i, j + 1) + F2(va, i, j)) +
                           F2(cor, i - 1, j) * F2(d, i - 1, j) * (F2(va, i - 1, j + 1) + F2(va, i - 1, j)));
    float cor_v = 0.25f * (F2(cor, i, j) * F2(d, i, j) * (F2(ua, i + 1, j) + F2(ua, i, j)) +
                           F2(cor, i, j - 1) * F2(d, i, j - 1) * (F2(ua, i + 1, j - 1) + F2(ua, i, j - 1)));
    float gu = g4 * (F2(dy, i, j) + F2(dy, i - 1, j)) * (F2(d, i, j) + F2(d, i - 1, j)) *
               (a12 * (F2(el, i, j) - F2(el, i - 1, j)) + al * (F2(elb, i, j) - F2(elb, i - 1, j)) +
                F2(e_atmos, i, j) - F2(e_atmos, i - 1, j));
    float gv = g4 * (F2(dx, i, j) + F2(dx, i, j - 1)) * (F2(d, i, j) + F2(d, i, j - 1)) *
               (a12 * (F2(el, i, j) - F2(el, i, j - 1)) + al * (F2(elb, i, j) - F2(elb, i, j - 1)) +
                F2(e_atmos, i, j) - F2(e_atmos, i, j - 1));
    float aru = F2(aru, i, j), arv = F2(arv, i, j);
    float uprov = adx + o.advua - aru * cor_u + gu + F2(drx2d, i, j) - aru * (-F2(wusurf, i, j) + F2(wubot, i, j));
    float vprov = ady + o.advva + arv * cor_v + gv + F2(dry2d, i, j) - arv * (-F2(wvsurf, i, j) + F2(wvbot, i, j));
    den_u = (F2(h, i, j) + F2(el, i, j) + F2(h, i - 1, j) + F2(el, i - 1, j)) * aru;
    float num_u = (F2(h, i, j) + F2(elb, i, j) + F2(h, i - 1, j) + F2(elb, i - 1, j)) * aru * F2(uab, i, j) -
                  c.k.four_dti * uprov;
    den_v = (F2(h, i, j) + F2(el, i, j) + F2(h, i, j - 1) + F2(el, i, j - 1)) * arv;
    float num_v = (F2(h, i, j) + F2(elb, i, j) + F2(h, i, j - 1) + F2(elb, i, j - 1)) * arv * F2(vab, i, j) -
                  c.k.four_dti * vprov;
    us = (num_u / (den_u + 1e-20f)) * F2(dum, i, j);
    vs = (num_v / (den_v + 1e-20f)) * F2(dvm, i, j);
    us = us * F2(dum, i, j);
    vs = vs * F2(dvm, i, j);
  }
  const bool ring = i == 0 || i == im - 1 || j == 0 || j == jm - 1;
  if (c.k.obc_seamount) {
    // the seamount policy's predictor (seamount_boundary.py:86-92): the
    // ring keeps the raw values (ua, va); the incident transport on the
    // west edge (column 1 and its ghost 0) and the east edge, no v through
    // them; then the masks
    if (ring) {
      us = F2(ua, i, j);
      vs = F2(va, i, j);
    }
    if (j >= 1 && j <= jm - 2) {
      if (i == 1 || i == 0) us = c.ramp * F1(uabw, j);
      if (i == im - 1) us = c.ramp * F1(uabe, j);
    }
    if (i == 0 || i == im - 1) vs = 0.0f;
    us = us * F2(dum, i, j);
    vs = vs * F2(dvm, i, j);
  } else if (c.k.obc_coastal) {
    // the tide policies' bcond 2 on u*, v* (coastal_boundary.py:23-29,
    // jzb_boundary.py:51-86): the ring keeps the predictor's raw values (ua,
    // va); the bay's Sommerfeld edges read only ua, va and d; the coastal
    // radiation reads the neighbours' new u*, v* (policy_bc2_line, next
    // launch); then the masks
    if (ring) {
      us = F2(ua, i, j);
      vs = F2(va, i, j);
    }
    if (c.k.obc_jzb) bcond2_jzb(c, i, j, us, vs);
    us = us * F2(dum, i, j);
    vs = vs * F2(dvm, i, j);
  } else if (ring) {
    us = 0.0f;
    vs = 0.0f;
  }
  PW2(us, i, j) = us;
  PW2(vs, i, j) = vs;
  PW2(den_u, i, j) = den_u;
  PW2(den_v, i, j) = den_v;
}

// ---------------------------------------------------------------------------
// Implicit free-surface solve pieces.
// ---------------------------------------------------------------------------

// Barotropic transports fed by the predictor (core.py:858-891): stored as
// fluxua/fluxva (zero on row 0 / column 0).
NPOM_HD float rhs_fluxua(const Ctx &c, int i, int j) {
  if (i < 1 || j < 1) return 0.0f;
  return 0.25f * (F2(d, i, j) + F2(d, i - 1, j)) * (F2(dy, i, j) + F2(dy, i - 1, j)) * W2(us, i, j);
}
NPOM_HD float rhs_fluxva(const Ctx &c, int i, int j) {
  if (i < 1 || j < 1) return 0.0f;
  return 0.25f * (F2(d, i, j) + F2(d, i, j - 1)) * (F2(dx, i, j) + F2(dx, i, j - 1)) * W2(vs, i, j);
}

// RHS of the elliptic problem with the Dirichlet ring zeroed
// (core.py:879-880 and 480-485).
NPOM_HD float rhs_cell(const Ctx &c, int i, int j) {
  if (!interior(c, i, j)) return 0.0f;
  float div = rhs_fluxua(c, i + 1, j) - rhs_fluxua(c, i, j) + rhs_fluxva(c, i, j + 1) - rhs_fluxva(c, i, j);
  return F2(elb, i, j) - c.k.two_dti * (div / (F2(art, i, j) + 1e-20f) + F2(vfluxf, i, j));
}

// Geometry coefficients of the operator (core.py:129-185), stored in the
// workspace once per core (they depend on the grid only).
NPOM_HD void elliptic_coeff_cell(const Ctx &c, int i, int j) {
  if (!interior(c, i, j)) {
    PW2(ce, i, j) = 0.0f;
    PW2(cw, i, j) = 0.0f;
    PW2(cn, i, j) = 0.0f;
    PW2(cs, i, j) = 0.0f;
    PW2(inv_art, i, j) = 0.0f;
    return;
  }
  float dx_e = 0.5f * (F2(dx, i + 1, j) + F2(dx, i, j));
  float dx_w = 0.5f * (F2(dx, i, j) + F2(dx, i - 1, j));
  float dy_e = 0.5f * (F2(dy, i + 1, j) + F2(dy, i, j));
  float dy_w = 0.5f * (F2(dy, i, j) + F2(dy, i - 1, j));
  float dy_n = 0.5f * (F2(dy, i, j + 1) + F2(dy, i, j));
  float dy_s = 0.5f * (F2(dy, i, j) + F2(dy, i, j - 1));
  float dx_n = 0.5f * (F2(dx, i, j + 1) + F2(dx, i, j));
  float dx_s = 0.5f * (F2(dx, i, j) + F2(dx, i, j - 1));
  PW2(ce, i, j) = dy_e / (dx_e + 1e-20f);
  PW2(cw, i, j) = dy_w / (dx_w + 1e-20f);
  PW2(cn, i, j) = dx_n / (dy_n + 1e-20f);
  PW2(cs, i, j) = dx_s / (dy_s + 1e-20f);
  PW2(inv_art, i, j) = 1.0f / (F2(art, i, j) + 1e-20f);
}

// The unknowns of the free-surface solve: rows pcg_i0 .. im-1-pcg_i0 of
// the interior columns 1..jm-2 -- the interior (Dirichlet ring), or with
// periodic x the unique columns 2..im-3 (the halo columns 1 and im-2 are
// copies, not unknowns).
NPOM_HD int pcg_i0(const Ctx &c) { return c.k.periodic_x ? 2 : 1; }

// Row of the x neighbour of unknown row i seen by the solve's vectors (the
// geometry's halo columns are copies already): i -/+ 1, wrapped across
// the period with periodic x.
NPOM_HD int pcg_west(const Ctx &c, int i) { return (c.k.periodic_x && i == 2) ? c.im - 3 : i - 1; }
NPOM_HD int pcg_east(const Ctx &c, int i) { return (c.k.periodic_x && i == c.im - 3) ? 2 : i + 1; }

// out = eta - coeff * div(D grad eta) / art on the interior (core.py:591-639);
// eta is a workspace or field vector with a zero Dirichlet ring (with
// periodic x its x neighbours are read across the period).
NPOM_HD float elliptic_apply_cell(const Ctx &c, const float *eta, int i, int j) {
  const size_t o = NPOM_I2(c, i, j);
  float e = ldc(c, eta + o);
  if (!interior(c, i, j)) return e;
  const float *dd = c.F[NPOM_F_d];
  const int jm = c.jm;
  float d0 = ldc(c, dd + o);
  float he = 0.5f * (ldc(c, dd + o + jm) + d0);
  float hw = 0.5f * (d0 + ldc(c, dd + o - jm));
  float hn = 0.5f * (ldc(c, dd + o + 1) + d0);
  float hs = 0.5f * (d0 + ldc(c, dd + o - 1));
  const float ee = ldc(c, eta + NPOM_I2(c, pcg_east(c, i), j));
  const float ew = ldc(c, eta + NPOM_I2(c, pcg_west(c, i), j));
  float fe = he * (ee - e) * W2(ce, i, j) * F2(dum, i + 1, j);
  float fw = hw * (e - ew) * W2(cw, i, j) * F2(dum, i, j);
  float fn = hn * (ldc(c, eta + o + 1) - e) * W2(cn, i, j) * F2(dvm, i, j + 1);
  float fs = hs * (e - ldc(c, eta + o - 1)) * W2(cs, i, j) * F2(dvm, i, j);
  float div = (fe - fw + fn - fs) * W2(inv_art, i, j);
  return e - c.k.implicit_coeff * div;
}

// The same operator applied to p' = p * beta + z (p on the ring cells),
// from the unchanged p and z: every value p' takes is computed with the
// expression the PCG's direction update stores, so the result is the
// operator applied to the stored p'.  *centre receives p' at (i, j).
NPOM_HD float elliptic_apply_cell_pz(const Ctx &c, const float *p, const float *z, float beta, int i, int j,
                                     float *centre) {
  const int jm = c.jm;
  auto pv = [&](int ii, int jj) {
    const size_t q = NPOM_I2(c, ii, jj);
    const float v = ldc(c, p + q);
    return interior(c, ii, jj) ? v * beta + ldc(c, z + q) : v;
  };
  const size_t o = NPOM_I2(c, i, j);
  float e = pv(i, j);
  *centre = e;
  if (!interior(c, i, j)) return e;
  const float *dd = c.F[NPOM_F_d];
  float d0 = ldc(c, dd + o);
  float he = 0.5f * (ldc(c, dd + o + jm) + d0);
  float hw = 0.5f * (d0 + ldc(c, dd + o - jm));
  float hn = 0.5f * (ldc(c, dd + o + 1) + d0);
  float hs = 0.5f * (d0 + ldc(c, dd + o - 1));
  float fe = he * (pv(pcg_east(c, i), j) - e) * W2(ce, i, j) * F2(dum, i + 1, j);
  float fw = hw * (e - pv(pcg_west(c, i), j)) * W2(cw, i, j) * F2(dum, i, j);
  float fn = hn * (pv(i, j + 1) - e) * W2(cn, i, j) * F2(dvm, i, j + 1);
  float fs = hs * (e - pv(i, j - 1)) * W2(cs, i, j) * F2(dvm, i, j);
  float div = (fe - fw + fn - fs) * W2(inv_art, i, j);
  return e - c.k.implicit_coeff * div;
}

// Jacobi diagonal (core.py:677-700)
NPOM_HD float jacobi_diag_cell(const Ctx &c, int i, int j) {
  if (!interior(c, i, j)) return 1.0f;
  float d0 = F2(d, i, j);
  float he = 0.5f * (F2(d, i + 1, j) + d0);
  float hw = 0.5f * (d0 + F2(d, i - 1, j));
  float hn = 0.5f * (F2(d, i, j + 1) + d0);
  float hs = 0.5f * (d0 + F2(d, i, j - 1));
  return 1.0f + c.k.implicit_coeff * W2(inv_art, i, j) *
                    (he * W2(ce, i, j) * F2(dum, i + 1, j) + hw * W2(cw, i, j) * F2(dum, i, j) +
                     hn * W2(cn, i, j) * F2(dvm, i, j + 1) + hs * W2(cs, i, j) * F2(dvm, i, j));
}

// Spectral preconditioner stages (core.py:762-773): DST-I along i, along j,
// scale by the inverse eigenvalues, DST-I along i, along j, / inverse_scale.
// Index (a, b) runs over the ni x nj interior.
// With periodic x the rows are the unique columns (ni = im-4, grid row
// a + 2) and Sx is the Hartley matrix of the period (see spectral_setup).
NPOM_HD float dst_stage_i(const Ctx &c, const float *src, bool src_is_grid, int a, int b) {
  const int i0 = pcg_i0(c), ni = c.im - 2 * i0, nj = c.jm - 2;
  const float *sx = c.W[NPOM_W_sx];
  double acc = 0.0;
  for (int m = 0; m < ni; ++m) {
    float v = src_is_grid ? ldc(c, src + NPOM_I2(c, m + i0, b + 1)) : ldc(c, src + (size_t)m * nj + b);
    acc += (double)ldc(c, sx + (size_t)a * ni + m) * (double)v;
  }
  return (float)acc;
}
NPOM_HD float dst_stage_j(const Ctx &c, const float *src, int a, int b) {
  const int nj = c.jm - 2;
  const float *sy = c.W[NPOM_W_sy];
  double acc = 0.0;
  for (int m = 0; m < nj; ++m) acc += (double)ldc(c, src + (size_t)a * nj + m) * (double)ldc(c, sy + (size_t)m * nj + b);
  return (float)acc;
}

// Corrector, closed-basin bcond 2, etf, Robert-Asselin filter, state shifts,
// egf and endpoint transports (core.py:918-943, time_loop.py:309-387).
// Returns true when |vaf| exceeds vmaxl at this cell.
// The corrector and its bcond 2 (core.py:918-943).  The tide policies'
// step copy leaves d at its old value for the pressure-gradient transport
// (coastal_implicit_time_loop.py:301-303), keeps the raw ring (the old uaf)
// and applies the policy's bcond 2, like the predictor's.
NPOM_HD void i5_uvaf(const Ctx &c, int i, int j, float &uaf, float &vaf) {
  const int im = c.im, jm = c.jm;
  const float elf0 = F2(elf, i, j);
  uaf = F2(uaf, i, j);
  vaf = F2(vaf, i, j);
  if (interior(c, i, j)) {
    const float g4 = c.k.quarter_g, al = c.k.alpha;
    float h0 = F2(h, i, j);
    float dnew = h0 + elf0;
    float dnew_w = F2(h, i - 1, j) + F2(elf, i - 1, j);
    float dnew_s = F2(h, i, j - 1) + F2(elf, i, j - 1);
    if (c.k.obc_coastal) {
      dnew = F2(d, i, j);
      dnew_w = F2(d, i - 1, j);
      dnew_s = F2(d, i, j - 1);
    }
    float gu = g4 * (F2(dy, i, j) + F2(dy, i - 1, j)) * (dnew + dnew_w) * al * (elf0 - F2(elf, i - 1, j));
    float gv = g4 * (F2(dx, i, j) + F2(dx, i, j - 1)) * (dnew + dnew_s) * al * (elf0 - F2(elf, i, j - 1));
    float dfu = (h0 + elf0 + F2(h, i - 1, j) + F2(elf, i - 1, j)) * F2(aru, i, j);
    float dfv = (h0 + elf0 + F2(h, i, j - 1) + F2(elf, i, j - 1)) * F2(arv, i, j);
    uaf = (W2(us, i, j) * W2(den_u, i, j) - c.k.four_dti * gu) / (dfu + 1e-20f) * F2(dum, i, j);
    vaf = (W2(vs, i, j) * W2(den_v, i, j) - c.k.four_dti * gv) / (dfv + 1e-20f) * F2(dvm, i, j);
  }
  if (c.k.obc_coastal && c.k.obc_jzb) bcond2_jzb(c, i, j, uaf, vaf);
  uaf = uaf * F2(dum, i, j);
  vaf = vaf * F2(dvm, i, j);
  if (!c.k.obc_coastal && (i == 0 || i == im - 1 || j == 0 || j == jm - 1)) {
    uaf = 0.0f;
    vaf = 0.0f;
  }
}

// The seamount policy's corrector (seamount_boundary.py:120-134): the
// transport of the predictor's u*, v* at the old face depth plus the
// implicit pressure gradient, divided by the new face depth (h + elf); row
// and column 0 zero; the west edge (column 1 and its ghost 0) and the east
// edge from the characteristic radiation about the exterior elevation;
// then the masks.  The old depth is d, which the solve leaves alone.
NPOM_HD void sea_corrector(const Ctx &c, int i, int j, float &uaf, float &vaf) {
  const int im = c.im, jm = c.jm;
  const float k2 = (float)(2.0 * (double)c.k.dti * (double)c.k.grav * (double)c.k.alpha);
  uaf = 0.0f;
  vaf = 0.0f;
  if (i >= 1) {
    const float hu = 0.5f * (F2(d, i, j) + F2(d, i - 1, j));
    const float hun = 0.5f * ((F2(h, i, j) + F2(elf, i, j)) + (F2(h, i - 1, j) + F2(elf, i - 1, j)));
    const float dxu = 0.5f * (F2(dx, i, j) + F2(dx, i - 1, j));
    uaf = (hu * W2(us, i, j) - k2 * hu * (F2(elf, i, j) - F2(elf, i - 1, j)) / dxu) / hun;
  }
  if (j >= 1) {
    const float hv = 0.5f * (F2(d, i, j) + F2(d, i, j - 1));
    const float hvn = 0.5f * ((F2(h, i, j) + F2(elf, i, j)) + (F2(h, i, j - 1) + F2(elf, i, j - 1)));
    const float dyv = 0.5f * (F2(dy, i, j) + F2(dy, i, j - 1));
    vaf = (hv * W2(vs, i, j) - k2 * hv * (F2(elf, i, j) - F2(elf, i, j - 1)) / dyv) / hvn;
  }
  if (j >= 1 && j <= jm - 2) {
    const float g = c.k.grav;
    if (i == 1 || i == 0)
      uaf = c.ramp * F1(uabw, j) - sqrtf(g / F2(h, 1, j)) * (F2(elf, 1, j) - F1(elw, j));
    if (i == im - 1)
      uaf = c.ramp * F1(uabe, j) + sqrtf(g / F2(h, im - 2, j)) * (F2(elf, im - 2, j) - F1(ele, j));
  }
  uaf = uaf * F2(dum, i, j);
  vaf = vaf * F2(dvm, i, j);
}

// Phase I5a of the policies on the semi-implicit core: the corrector with
// bcond 2 into uaf/vaf (the coastal radiation's edges follow in
// policy_bc2_line); I5 then reads them.  Reads ua, va, d and uaf, none of
// which it writes elsewhere.
NPOM_HD void phase_i5a_cell(const Ctx &c, int i, int j) {
  float uaf, vaf;
  if (c.k.obc_seamount) sea_corrector(c, i, j, uaf, vaf);
  else i5_uvaf(c, i, j, uaf, vaf);
  P2(uaf, i, j) = uaf;
  P2(vaf, i, j) = vaf;
}

NPOM_HD bool phase_i5_cell(const Ctx &c, int i, int j) {
  const int im = c.im, jm = c.jm;
  const float elf0 = F2(elf, i, j);
  float uaf, vaf;
  if (c.k.obc_coastal || c.k.obc_seamount) {
    uaf = F2(uaf, i, j);
    vaf = F2(vaf, i, j);
  } else {
    i5_uvaf(c, i, j, uaf, vaf);
  }
  P2(uaf, i, j) = uaf;
  P2(vaf, i, j) = vaf;
  P2(etf, i, j) = elf0 * F2(fsm, i, j);
  bool exceed = !(fabsf(vaf) <= c.k.vmaxl);
  // Robert-Asselin filter and shifts (speculatively applied; a VMAX status
  // aborts the step on the host)
  const float hs = c.k.half_smoth;
  float ua = F2(ua, i, j), va = F2(va, i, j), el = F2(el, i, j);
  float uaf_f = ua + hs * (F2(uab, i, j) - 2.0f * ua + uaf);
  float vaf_f = va + hs * (F2(vab, i, j) - 2.0f * va + vaf);
  float el_f = el + hs * (F2(elb, i, j) - 2.0f * el + elf0);
  P2(elb, i, j) = el_f;
  P2(el, i, j) = elf0;
  float dn = F2(h, i, j) + elf0;
  P2(d, i, j) = dn;
  P2(uab, i, j) = uaf_f;
  P2(ua, i, j) = uaf;
  P2(vab, i, j) = vaf_f;
  P2(va, i, j) = vaf;
  P2(egf, i, j) = (el_f + elf0) * 0.5f;
  if (i >= 1) {
    float dsum_new = dn + (F2(h, i - 1, j) + F2(elf, i - 1, j));
    float dsum_baro = W2(d_baro, i, j) + W2(d_baro, i - 1, j);
    P2(utf, i, j) = 0.25f * (uaf_f * dsum_baro + uaf * dsum_new);
  }
  if (j >= 1) {
    float dsum_new = dn + (F2(h, i, j - 1) + F2(elf, i, j - 1));
    float dsum_baro = W2(d_baro, i, j) + W2(d_baro, i, j - 1);
    P2(vtf, i, j) = 0.25f * (vaf_f * dsum_baro + vaf * dsum_new);
  }
  return exceed;
}

// ---------------------------------------------------------------------------
// Explicit external substep (explicit/time_loop.py:292-431).
// ---------------------------------------------------------------------------

// Interior elf before bcond 1 (time_loop.py:299-312)
NPOM_HD float ext_elf_interior(const Ctx &c, int i, int j) {
  auto fu = [&](int ii, int jj) {
    return 0.25f * (F2(d, ii, jj) + F2(d, ii - 1, jj)) * (F2(dy, ii, jj) + F2(dy, ii - 1, jj)) * F2(ua, ii, jj);
  };
  auto fv = [&](int ii, int jj) {
    return 0.25f * (F2(d, ii, jj) + F2(d, ii, jj - 1)) * (F2(dx, ii, jj) + F2(dx, ii, jj - 1)) * F2(va, ii, jj);
  };
  float div = fu(i + 1, j) - fu(i, j) + fv(i, j + 1) - fv(i, j);
  float term = -(div / F2(art, i, j)) - F2(vfluxf, i, j);
  return F2(elb, i, j) + c.k.dte2 * term;
}

// elf after the explicit bcond 1 (baroclinic.py:510-524): edges copy the
// adjacent cell (rows first, then columns, so corners take the diagonal
// interior value), then the whole field is masked by fsm.
NPOM_HD float ext_elf_cell_seamount(const Ctx &c, int i, int j);
NPOM_HD float ext_elf_cell_coastal(const Ctx &c, int i, int j, int iext);
NPOM_HD float ext_elf_cell_jzb(const Ctx &c, int i, int j, int iext);

NPOM_HD float ext_elf_cell(const Ctx &c, int i, int j, int iext) {
  if (c.k.obc_seamount) return ext_elf_cell_seamount(c, i, j);
  if (c.k.obc_jzb) return ext_elf_cell_jzb(c, i, j, iext);
  if (c.k.obc_coastal) return ext_elf_cell_coastal(c, i, j, iext);
  int si = i, sj = j;
  if (si == 0) si = 1;
  if (si == c.im - 1) si = c.im - 2;
  if (sj == 0) sj = 1;
  if (sj == c.jm - 1) sj = c.jm - 2;
  return ext_elf_interior(c, si, sj) * F2(fsm, i, j);
}

// elf after the seamount policy's bcond 1 (seamount_boundary.py:9-12,15):
// only the east and west edges copy the adjacent column, then the mask.
// The north and south rows keep the value they hold (the interior update
// does not reach them).  A corner reads that value of its neighbour in the
// row, which the neighbour's own thread rewrites as value * fsm in this
// phase; the two agree wherever they matter: a corner outside the sea is 0
// without the read, and a sea corner's neighbour is sea as well.
NPOM_HD float ext_elf_cell_seamount(const Ctx &c, int i, int j) {
  const float fsm = F2(fsm, i, j);
  const int si = i == 0 ? 1 : (i == c.im - 1 ? c.im - 2 : i);
  if (si != i && (j == 0 || j == c.jm - 1) && fsm == 0.0f) return 0.0f;
  const float raw = interior(c, si, j) ? ext_elf_interior(c, si, j) : F2(elf, si, j);
  return raw * fsm;
}

// elf after the coastal tide policy's bcond 1 (coastal_boundary.py:9-22):
// at the flagged cells the tide amp cos(w t - phase) at the substep's time
// t = (time * 86400 - dti) + dte * (iext - 1) s, the argument w t / 3600
// formed in double and rounded once, as the policy's Python floats are; no
// edge copies; then the mask.
NPOM_HD float ext_elf_cell_coastal(const Ctx &c, int i, int j, int iext) {
  const size_t o = NPOM_I2(c, i, j), n2 = (size_t)c.im * c.jm;
  float raw;
  if (c.tide[o] != 0.0f) {
    const double sec = c.tide_t0 + c.k.dte_d * (double)(iext - 1);
    const float arg = (float)(c.k.tide_w * sec / 3600.0);
    raw = c.tide[n2 + o] * cosf(arg - c.tide[2 * n2 + o] * 3.1416f / 180.0f);
  } else {
    raw = interior(c, i, j) ? ext_elf_interior(c, i, j) : F2(elf, i, j);
  }
  return raw * F2(fsm, i, j);
}

// elf after the Jiaozhou Bay policy's bcond 1 (jzb_boundary.py:17-49): at
// the flagged cells the tide amp cos(w (t / 3600) - phase) times fsm there
// (t as in the coastal policy, the argument's product formed in double from
// t / 3600); then the edges copy the adjacent cell (west and east, then
// south and north, so a corner takes the diagonal interior value) and the
// whole field is masked.  A tide cell on the ring is overwritten by the
// copy, so every value comes from the interior cell (si, sj).
NPOM_HD float ext_elf_cell_jzb(const Ctx &c, int i, int j, int iext) {
  const int si = i == 0 ? 1 : (i == c.im - 1 ? c.im - 2 : i);
  const int sj = j == 0 ? 1 : (j == c.jm - 1 ? c.jm - 2 : j);
  const size_t o = NPOM_I2(c, si, sj), n2 = (size_t)c.im * c.jm;
  float raw;
  if (c.tide[o] != 0.0f) {
    const double sec = c.tide_t0 + c.k.dte_d * (double)(iext - 1);
    const float arg = (float)(c.k.tide_w * (sec / 3600.0));
    raw = c.tide[n2 + o] * cosf(arg - c.tide[2 * n2 + o] * 3.1416f / 180.0f) * F2(fsm, si, sj);
  } else {
    raw = ext_elf_interior(c, si, sj);
  }
  return raw * F2(fsm, i, j);
}

// Phase 1 of a substep: elf with bcond 1, and the stored fluxua/fluxva:
// the transports (time_loop.py:299-305), or on ADVAVE substeps
// (iext % ispadv == 0) the ADVAVE outputs that overwrite them.  ADVAVE reads
// fluxua/fluxva only on row 0 / column 0, which no phase writes, so both
// fit in one phase.
NPOM_HD void ext_phase1_cell(const Ctx &c, int i, int j, bool do_advave, int iext = 1) {
  P2(elf, i, j) = ext_elf_cell(c, i, j, iext);
  if (do_advave) {
    AdvaveOut o = advave_cell(c, i, j);
    P2(advua, i, j) = o.advua;
    P2(advva, i, j) = o.advva;
    if (o.write_flux) {
      P2(fluxua, i, j) = o.fluxua;
      P2(fluxva, i, j) = o.fluxva;
    }
    if (o.write_tps) P2(tps, i, j) = o.tps;
  } else if (i >= 1 && j >= 1) {
    P2(fluxua, i, j) = 0.25f * (F2(d, i, j) + F2(d, i - 1, j)) * (F2(dy, i, j) + F2(dy, i - 1, j)) * F2(ua, i, j);
    P2(fluxva, i, j) = 0.25f * (F2(d, i, j) + F2(d, i, j - 1)) * (F2(dx, i, j) + F2(dx, i, j - 1)) * F2(va, i, j);
  }
}

// uaf/vaf of phase 2 before bcond 2 (time_loop.py:326-383): the momentum
// update on the interior, the values the fields hold elsewhere
NPOM_HD void ext_uvaf_raw(const Ctx &c, int i, int j, float &uaf, float &vaf) {
  uaf = F2(uaf, i, j);
  vaf = F2(vaf, i, j);
  if (interior(c, i, j)) {
    const float g4 = c.k.quarter_g, al = c.k.alpha, a12 = c.k.one_m_2alpha;
    float d0 = F2(d, i, j);
    float cor_u = 0.25f * (F2(cor, i, j) * d0 * (F2(va, i, j + 1) + F2(va, i, j)) +
                           F2(cor, i - 1, j) * F2(d, i - 1, j) * (F2(va, i - 1, j + 1) + F2(va, i - 1, j)));
    float gu = g4 * (F2(dy, i, j) + F2(dy, i - 1, j)) * (d0 + F2(d, i - 1, j)) *
               (a12 * (F2(el, i, j) - F2(el, i - 1, j)) +
                al * (F2(elb, i, j) - F2(elb, i - 1, j) + F2(elf, i, j) - F2(elf, i - 1, j)) + F2(e_atmos, i, j) -
                F2(e_atmos, i - 1, j));
    float aru = F2(aru, i, j), arv = F2(arv, i, j);
    float up = F2(adx2d, i, j) + F2(advua, i, j) - aru * cor_u + gu + F2(drx2d, i, j) -
               aru * (-F2(wusurf, i, j) + F2(wubot, i, j));
    float den = (F2(h, i, j) + F2(elf, i, j) + F2(h, i - 1, j) + F2(elf, i - 1, j)) * aru;
    float num = (F2(h, i, j) + F2(elb, i, j) + F2(h, i - 1, j) + F2(elb, i - 1, j)) * aru * F2(uab, i, j) -
                c.k.four_dte * up;
    uaf = num / (den + 1e-20f);
    float cor_v = 0.25f * (F2(cor, i, j) * d0 * (F2(ua, i + 1, j) + F2(ua, i, j)) +
                           F2(cor, i, j - 1) * F2(d, i, j - 1) * (F2(ua, i + 1, j - 1) + F2(ua, i, j - 1)));
    float gv = g4 * (F2(dx, i, j) + F2(dx, i, j - 1)) * (d0 + F2(d, i, j - 1)) *
               (a12 * (F2(el, i, j) - F2(el, i, j - 1)) +
                al * (F2(elb, i, j) - F2(elb, i, j - 1) + F2(elf, i, j) - F2(elf, i, j - 1)) + F2(e_atmos, i, j) -
                F2(e_atmos, i, j - 1));
    float vp = F2(ady2d, i, j) + F2(advva, i, j) + arv * cor_v + gv + F2(dry2d, i, j) -
               arv * (-F2(wvsurf, i, j) + F2(wvbot, i, j));
    float denv = (F2(h, i, j) + F2(elf, i, j) + F2(h, i, j - 1) + F2(elf, i, j - 1)) * arv;
    float numv = (F2(h, i, j) + F2(elb, i, j) + F2(h, i, j - 1) + F2(elb, i, j - 1)) * arv * F2(vab, i, j) -
                 c.k.four_dte * vp;
    vaf = numv / (denv + 1e-20f);
  }
}

// The coastal tide policy's bcond 2 (coastal_boundary.py:23-29):
// characteristic radiation with the total depth d on the east, west, north
// and south edges in that order, the west and south ghosts copies.  A value
// that reads a neighbour's new uaf/vaf recomputes that neighbour's interior
// update (the same expression on the same inputs, so the same bits).
NPOM_HD void bcond2_coastal(const Ctx &c, int i, int j, float &uaf, float &vaf) {
  const int im = c.im, jm = c.jm;
  const float g = c.k.grav;
  auto rad = [&](int ii, int jj) { return sqrtf(g / F2(d, ii, jj)); };
  float un, vn;
  if (j >= 1 && j <= jm - 2) {
    if (i == im - 1) {
      ext_uvaf_raw(c, im - 2, j, un, vn);
      uaf = un + c.k.rfe * rad(im - 2, j) * (F2(el, im - 2, j) - F2(el, im - 1, j));
      vaf = 0.0f;
    }
    if (i == 1 || i == 0) {
      if (i == 0) ext_uvaf_raw(c, 1, j, un, vn);
      else un = uaf;
      uaf = un - c.k.rfw * rad(1, j) * (F2(el, 1, j) - F2(el, 0, j));
      if (i == 0) vaf = 0.0f;
    }
  }
  if (i >= 1 && i <= im - 2) {
    if (j == jm - 1) {
      ext_uvaf_raw(c, i, jm - 2, un, vn);
      vaf = vn + c.k.rfn * rad(i, jm - 2) * (F2(el, i, jm - 2) - F2(el, i, jm - 1));
      uaf = 0.0f;
    }
    if (j == 1 || j == 0) {
      if (j == 0) ext_uvaf_raw(c, i, 1, un, vn);
      else vn = vaf;
      vaf = vn - c.k.rfs * rad(i, 1) * (F2(el, i, 1) - F2(el, i, 0));
      if (j == 0) uaf = 0.0f;
    }
  }
}

// The Jiaozhou Bay policy's bcond 2 (jzb_boundary.py:51-86): Sommerfeld
// radiation of the transports, uaf on the east edge (from ua at im-2) and at
// column 1 (from ua at 2), vaf on the north edge (from va at jm-2) and at
// row 1 (from va at 2), with the weight dte sqrt(max(g d, 0)) / dx (dy)
// at the depth cell the policy names, times ramp, wherever that d > 0;
// there the tangential component on the outer ring is zero.  Reads only
// ua, va and d, none of which the phase writes; the edge sets do not
// overlap, so their order does not matter.
NPOM_HD void bcond2_jzb(const Ctx &c, int i, int j, float &uaf, float &vaf) {
  const int im = c.im, jm = c.jm;
  const float g = c.k.grav, dte = (float)c.k.dte_d, ramp = c.ramp;
  auto gae = [&](int ii, int jj, float len) { return dte * sqrtf(fmaxf_t(g * F2(d, ii, jj), 0.0f)) / len; };
  if (j >= 1 && j <= jm - 2) {
    if (i == im - 1 && F2(d, im - 1, j) > 0.0f) {
      const float w = gae(im - 1, j, F2(dx, im - 1, j));
      uaf = (w * F2(ua, im - 2, j) + (1.0f - w) * F2(ua, im - 1, j)) * ramp;
      vaf = 0.0f;
    }
    if ((i == 1 || i == 0) && F2(d, 1, j) > 0.0f) {
      const float w = gae(1, j, F2(dx, 1, j));
      if (i == 1) uaf = ramp * (w * F2(ua, 2, j) + (1.0f - w) * F2(ua, 1, j));
      else vaf = 0.0f;
    }
  }
  if (i >= 1 && i <= im - 2) {
    if (j == jm - 1 && F2(d, i, jm - 1) > 0.0f) {
      const float w = gae(i, jm - 1, F2(dy, i, jm - 1));
      vaf = (w * F2(va, i, jm - 2) + (1.0f - w) * F2(va, i, jm - 1)) * ramp;
      uaf = 0.0f;
    }
    if ((j == 1 || j == 0) && F2(d, i, 1) > 0.0f) {
      const float w = gae(i, 1, F2(dy, i, 1));
      if (j == 1) vaf = (w * F2(va, i, 2) + (1.0f - w) * F2(va, i, 1)) * ramp;
      else uaf = 0.0f;
    }
  }
}

// Phase 2: uaf/vaf with bcond 2 and the etf time filter
// (time_loop.py:326-391).  Returns |vaf| > vmaxl.
NPOM_HD bool ext_phase2_cell(const Ctx &c, int i, int j, int iext) {
  const int im = c.im, jm = c.jm;
  float uaf, vaf;
  ext_uvaf_raw(c, i, j, uaf, vaf);
  // bcond 2 (baroclinic.py:529-571): open-boundary (Flather) values, zero
  // normal/tangential components on the ring, then masks.
  const float ramp = c.ramp, g = c.k.grav;
  auto rad = [&](float hh) { return sqrtf(fmaxf_t(g / fmaxf_t(hh, 1e-8f), 1e-8f)); };
  if (c.k.obc_jzb) {
    bcond2_jzb(c, i, j, uaf, vaf);
  } else if (c.k.obc_coastal) {
    bcond2_coastal(c, i, j, uaf, vaf);
  } else if (c.k.obc_seamount) {
    // the seamount policy (seamount_boundary.py:16-19): characteristic
    // radiation about the exterior elevation on the west and east edges
    // only, the west ghost column a copy, no normal flow through them
    if (j >= 1 && j <= jm - 2) {
      if (i == 1 || i == 0) uaf = ramp * F1(uabw, j) - sqrtf(g / F2(h, 1, j)) * (F2(el, 1, j) - F1(elw, j));
      if (i == 0) vaf = 0.0f;
      if (i == im - 1) {
        uaf = ramp * F1(uabe, j) + sqrtf(g / F2(h, im - 2, j)) * (F2(el, im - 2, j) - F1(ele, j));
        vaf = 0.0f;
      }
    }
  } else if (j >= 1 && j <= jm - 2) {
    if (i == im - 1) {
      float te = c.k.rfe * rad(F2(h, im - 2, j)) * (F2(el, im - 2, j) - F1(ele, j));
      uaf = (F1(uabe, j) + te) * ramp;
      vaf = 0.0f;
    }
    if (i == 1 || i == 0) {
      float tw = c.k.rfw * rad(F2(h, 1, j)) * (F2(el, 1, j) - F1(elw, j));
      uaf = (F1(uabw, j) - tw) * ramp;
    }
    if (i == 0) vaf = 0.0f;
  }
  if (!c.k.obc_seamount && !c.k.obc_coastal && i >= 1 && i <= im - 2) {
    if (j == jm - 1) {
      float tn = c.k.rfn * rad(F2(h, i, jm - 2)) * (F2(el, i, jm - 2) - F1(eln, i));
      vaf = (F1(vabn, i) + tn) * ramp;
      uaf = 0.0f;
    }
    if (j == 1 || j == 0) {
      float ts = c.k.rfs * rad(F2(h, i, 1)) * (F2(el, i, 1) - F1(els, i));
      vaf = (F1(vabs, i) - ts) * ramp;
    }
    if (j == 0) uaf = 0.0f;
  }
  uaf = uaf * F2(dum, i, j);
  vaf = vaf * F2(dvm, i, j);
  P2(uaf, i, j) = uaf;
  P2(vaf, i, j) = vaf;
  // etf filter (time_loop.py:386-391)
  const int isplit = c.k.isplit;
  float elf0 = F2(elf, i, j);
  if (iext == isplit - 2) {
    P2(etf, i, j) = c.k.quarter_smoth * elf0;
  } else if (iext == isplit - 1) {
    P2(etf, i, j) = F2(etf, i, j) + c.k.etf_mid * elf0;
  } else if (iext == isplit) {
    P2(etf, i, j) = (F2(etf, i, j) + 0.5f * elf0) * F2(fsm, i, j);
  }
  return !(fabsf(vaf) <= c.k.vmaxl);
}

// Phase 3: Robert-Asselin filter, shifts, egf/utf/vtf accumulation
// (time_loop.py:395-431).  Reads only this cell plus elf/h of the west and
// south neighbours (d at the end of the substep is h + elf).
NPOM_HD void ext_phase3_cell(const Ctx &c, int i, int j, int iext) {
  const float hs = c.k.half_smoth;
  float ua = F2(ua, i, j), va = F2(va, i, j), el = F2(el, i, j);
  float uaf = F2(uaf, i, j), vaf = F2(vaf, i, j), elf0 = F2(elf, i, j);
  float ua_f = ua + hs * (F2(uab, i, j) - 2.0f * ua + uaf);
  float va_f = va + hs * (F2(vab, i, j) - 2.0f * va + vaf);
  float el_f = el + hs * (F2(elb, i, j) - 2.0f * el + elf0);
  P2(elb, i, j) = el_f;
  P2(el, i, j) = elf0;
  float dn = F2(h, i, j) + elf0;
  P2(d, i, j) = dn;
  P2(uab, i, j) = ua_f;
  P2(ua, i, j) = uaf;
  P2(vab, i, j) = va_f;
  P2(va, i, j) = vaf;
  if (iext != c.k.isplit) {
    P2(egf, i, j) = F2(egf, i, j) + elf0 * c.k.ispi;
    if (i >= 1) {
      float ds = dn + (F2(h, i - 1, j) + F2(elf, i - 1, j));
      P2(utf, i, j) = F2(utf, i, j) + uaf * ds * c.k.isp2i;
    }
    if (j >= 1) {
      float ds = dn + (F2(h, i, j - 1) + F2(elf, i, j - 1));
      P2(vtf, i, j) = F2(vtf, i, j) + vaf * ds * c.k.isp2i;
    }
  }
}

// ---------------------------------------------------------------------------
// The semi-implicit core under the coastal or Jiaozhou Bay tide policy.
// ---------------------------------------------------------------------------

// The coastal policy's bcond 2 on the semi-implicit core's u*, v* (after
// A3, which = 0, on the us/vs planes) or uaf, vaf (after I5a, which = 1):
// line t < jm handles row j = t (east edge, then column 1 and its ghost
// column 0), line jm + i column i (north edge, then row 1 and its ghost row
// 0), in coastal_boundary.py:23-29's formulas with el and the depth d the
// step holds (the old depth: the step copy updates d after the corrector).
// Each line writes values no other line reads or writes; the masks apply.
NPOM_HD void policy_bc2_line(const Ctx &c, int t, int which) {
  const int im = c.im, jm = c.jm;
  float *ua = which == 0 ? c.W[NPOM_W_us] : c.F[NPOM_F_uaf];
  float *va = which == 0 ? c.W[NPOM_W_vs] : c.F[NPOM_F_vaf];
  const float g = c.k.grav;
  auto rad = [&](int ii, int jj) { return sqrtf(g / F2(d, ii, jj)); };
  if (t < jm) {
    const int j = t;
    if (j < 1 || j > jm - 2) return;
    const float ue = ld(ua + NPOM_I2(c, im - 2, j)) + c.k.rfe * rad(im - 2, j) * (F2(el, im - 2, j) - F2(el, im - 1, j));
    ua[NPOM_I2(c, im - 1, j)] = ue * F2(dum, im - 1, j);
    va[NPOM_I2(c, im - 1, j)] = 0.0f * F2(dvm, im - 1, j);
    const float uw = ld(ua + NPOM_I2(c, 1, j)) - c.k.rfw * rad(1, j) * (F2(el, 1, j) - F2(el, 0, j));
    ua[NPOM_I2(c, 1, j)] = uw * F2(dum, 1, j);
    ua[NPOM_I2(c, 0, j)] = uw * F2(dum, 0, j);
    va[NPOM_I2(c, 0, j)] = 0.0f * F2(dvm, 0, j);
  } else if (t < jm + im) {
    const int i = t - jm;
    if (i < 1 || i > im - 2) return;
    const float vn = ld(va + NPOM_I2(c, i, jm - 2)) + c.k.rfn * rad(i, jm - 2) * (F2(el, i, jm - 2) - F2(el, i, jm - 1));
    va[NPOM_I2(c, i, jm - 1)] = vn * F2(dvm, i, jm - 1);
    ua[NPOM_I2(c, i, jm - 1)] = 0.0f * F2(dum, i, jm - 1);
    const float vs = ld(va + NPOM_I2(c, i, 1)) - c.k.rfs * rad(i, 1) * (F2(el, i, 1) - F2(el, i, 0));
    va[NPOM_I2(c, i, 1)] = vs * F2(dvm, i, 1);
    va[NPOM_I2(c, i, 0)] = vs * F2(dvm, i, 0);
    ua[NPOM_I2(c, i, 0)] = 0.0f * F2(dum, i, 0);
  }
}

// The tide policies' elevation at a tide-table cell at the step's solve
// time t = time * 86400 - dte (c.tide_t0): the coastal policy's
// amp cos(w t / 3600 - phase), the bay's amp cos(w (t / 3600) - phase)
// (coastal_boundary.py:9-10, jzb_boundary.py:17-21); the caller applies the
// bay's fsm.
NPOM_HD float policy_tide(const Ctx &c, size_t o) {
  const size_t n2 = (size_t)c.im * c.jm;
  const double sec = c.tide_t0;
  const float arg = c.k.obc_jzb ? (float)(c.k.tide_w * (sec / 3600.0)) : (float)(c.k.tide_w * sec / 3600.0);
  return c.tide[n2 + o] * cosf(arg - c.tide[2 * n2 + o] * 3.1416f / 180.0f);
}

// The policy solve's fixed nodes (not unknowns): the ring, land and the
// tide cells (coastal_boundary.py:62-64, jzb_boundary.py:208-211).
NPOM_HD bool policy_fixed(const Ctx &c, int i, int j) {
  return !interior(c, i, j) || F2(fsm, i, j) == 0.0f || c.tide[NPOM_I2(c, i, j)] != 0.0f;
}

// The solve's lift: the tide at the tide cells, zero elsewhere; the bay's
// times fsm there, then its edges copying the adjacent cell and the mask
// (jzb_boundary.py:152-157).
NPOM_HD float policy_lift(const Ctx &c, int i, int j) {
  if (c.k.obc_jzb) {
    const int si = i == 0 ? 1 : (i == c.im - 1 ? c.im - 2 : i);
    const int sj = j == 0 ? 1 : (j == c.jm - 1 ? c.jm - 2 : j);
    const size_t o = NPOM_I2(c, si, sj);
    const float v = c.tide[o] != 0.0f ? policy_tide(c, o) * F2(fsm, si, sj) : 0.0f;
    return v * F2(fsm, i, j);
  }
  const size_t o = NPOM_I2(c, i, j);
  return c.tide[o] != 0.0f ? policy_tide(c, o) : 0.0f;
}

// elf after the policy solve and the step's bcond 1 (core.py:913-916 with
// the Shapiro filter at gamma 0): from x + lift (x holds the solution, zero
// on the fixed nodes), the interior masked, the tide cells set to the tide
// and the mask; the bay's edges copy the adjacent cell first (the solve's
// own copy, then bcond 1's, both of the same interior cell).
NPOM_HD float policy_elf(const Ctx &c, const float *x, int i, int j) {
  auto inner = [&](int ii, int jj) {
    const size_t o = NPOM_I2(c, ii, jj);
    const float fsm = F2(fsm, ii, jj);
    if (c.tide[o] != 0.0f) return c.k.obc_jzb ? policy_tide(c, o) * fsm : policy_tide(c, o);
    float v = ld(x + o) + policy_lift(c, ii, jj);
    if (c.k.obc_jzb) v = v * fsm;
    return interior(c, ii, jj) ? v * fsm : v;
  };
  if (c.k.obc_jzb) {
    const int si = i == 0 ? 1 : (i == c.im - 1 ? c.im - 2 : i);
    const int sj = j == 0 ? 1 : (j == c.jm - 1 ? c.jm - 2 : j);
    return inner(si, sj) * F2(fsm, i, j);
  }
  return inner(i, j) * F2(fsm, i, j);
}

// ---------------------------------------------------------------------------
// The seamount policy on the semi-implicit core (seamount_boundary.py:
// 45-147).  Its solve runs in FP64 on the npom_workspace.robin planes.
// ---------------------------------------------------------------------------

// eta_ghost (seamount_boundary.py:9-11): the east and west edge columns
// copy the adjacent column, then the mask
NPOM_HD int sea_gi(const Ctx &c, int i) { return i == 0 ? 1 : (i == c.im - 1 ? c.im - 2 : i); }
NPOM_HD double sea_ghost(const Ctx &c, const double *v, int i, int j) {
  return v[NPOM_I2(c, sea_gi(c, i), j)] * (double)F2(fsm, i, j);
}
// the unknowns: interior sea cells
NPOM_HD bool sea_free(const Ctx &c, int i, int j) { return interior(c, i, j) && F2(fsm, i, j) > 0.0f; }

// The Robin terms of row j (1..jm-2) from the Picard guess G = ghost(x):
// face depths of the new depth h + G at the west (columns 0, 1) and east
// (im-2, im-1) edges, and the characteristic flux coefficients
// 2 dti H dy sqrt(g / h) / art of columns 1 and im-2.
struct SeaRobin {
  double hw, he, dyw, dye, bw, be, rw, re;
};
NPOM_HD SeaRobin sea_robin(const Ctx &c, const double *G, int j) {
  const int im = c.im;
  const double dti = c.k.dti, g = c.k.grav;
  SeaRobin r;
  r.hw = 0.5 * (((double)F2(h, 1, j) + G[NPOM_I2(c, 1, j)]) + ((double)F2(h, 0, j) + G[NPOM_I2(c, 0, j)]));
  r.he = 0.5 * (((double)F2(h, im - 1, j) + G[NPOM_I2(c, im - 1, j)]) +
                ((double)F2(h, im - 2, j) + G[NPOM_I2(c, im - 2, j)]));
  r.dyw = 0.5 * ((double)F2(dy, 1, j) + (double)F2(dy, 0, j));
  r.dye = 0.5 * ((double)F2(dy, im - 1, j) + (double)F2(dy, im - 2, j));
  r.bw = sqrt(g / (double)F2(h, 1, j));
  r.be = sqrt(g / (double)F2(h, im - 2, j));
  r.rw = 2.0 * dti * r.hw * r.dyw * r.bw / (double)F2(art, 1, j);
  r.re = 2.0 * dti * r.he * r.dye * r.be / (double)F2(art, im - 2, j);
  return r;
}

// op(v) = the elliptic operator (old depth d) on ghost(v), plus the Robin
// terms on columns 1 and im-2, zero off the unknowns (seamount_boundary.py:
// 73-76), in FP64
NPOM_HD double sea_robin_op(const Ctx &c, const double *v, const double *G, int i, int j) {
  if (!sea_free(c, i, j)) return 0.0;
  auto z = [&](int ii, int jj) { return sea_ghost(c, v, ii, jj); };
  const double e = z(i, j);
  const double d0 = F2(d, i, j);
  const double he = 0.5 * ((double)F2(d, i + 1, j) + d0), hw = 0.5 * (d0 + (double)F2(d, i - 1, j));
  const double hn = 0.5 * ((double)F2(d, i, j + 1) + d0), hs = 0.5 * (d0 + (double)F2(d, i, j - 1));
  const double fe = he * (z(i + 1, j) - e) * (double)W2(ce, i, j) * (double)F2(dum, i + 1, j);
  const double fw = hw * (e - z(i - 1, j)) * (double)W2(cw, i, j) * (double)F2(dum, i, j);
  const double fn = hn * (z(i, j + 1) - e) * (double)W2(cn, i, j) * (double)F2(dvm, i, j + 1);
  const double fs = hs * (e - z(i, j - 1)) * (double)W2(cs, i, j) * (double)F2(dvm, i, j);
  double out = e - (double)c.k.implicit_coeff * ((fe - fw + fn - fs) * (double)W2(inv_art, i, j));
  if (j >= 1 && j <= c.jm - 2 && (i == 1 || i == c.im - 2)) {
    const SeaRobin r = sea_robin(c, G, j);
    if (i == 1) out += r.rw * e;
    if (i == c.im - 2) out += r.re * e;
  }
  return out;
}

// The right-hand side b of one Picard iteration (seamount_boundary.py:
// 77-86): the step's RHS on the unknowns, plus on columns 1 and im-2 the
// new-depth incident and exterior-elevation fluxes, minus the old-depth
// incident flux the predictor already holds
NPOM_HD double sea_rhs(const Ctx &c, const float *rhs, const double *G, int i, int j) {
  double b = sea_free(c, i, j) ? (double)rhs[NPOM_I2(c, i, j)] : 0.0;
  if (j >= 1 && j <= c.jm - 2 && (i == 1 || i == c.im - 2)) {
    const int im = c.im;
    const SeaRobin r = sea_robin(c, G, j);
    const double dti = c.k.dti, ramp = c.ramp;
    if (i == 1) {
      b += 2.0 * dti * r.hw * r.dyw * (ramp * (double)F1(uabw, j) + r.bw * (double)F1(elw, j)) / (double)F2(art, 1, j);
      b -= 2.0 * dti * 0.5 * ((double)F2(d, 1, j) + (double)F2(d, 0, j)) * r.dyw * ramp * (double)F1(uabw, j) /
           (double)F2(art, 1, j);
    }
    if (i == im - 2) {
      b -= 2.0 * dti * r.he * r.dye * (ramp * (double)F1(uabe, j) - r.be * (double)F1(ele, j)) /
           (double)F2(art, im - 2, j);
      b += 2.0 * dti * 0.5 * ((double)F2(d, im - 1, j) + (double)F2(d, im - 2, j)) * r.dye * ramp *
           (double)F1(uabe, j) / (double)F2(art, im - 2, j);
    }
  }
  return b;
}

// elf after the solve (ghost(x)), the Shapiro filter at gamma 0 (the
// interior masked) and bcond 1 (ghost again)
NPOM_HD float sea_elf(const Ctx &c, const double *x, int i, int j) {
  const int si = sea_gi(c, i);
  double e = sea_ghost(c, x, si, j);
  if (interior(c, si, j)) e = e * (double)F2(fsm, si, j);
  return (float)(e * (double)F2(fsm, i, j));
}

// The body continuity after the filter (seamount_boundary.py:28-42): the
// transports from the filtered and new velocities and depths (hb = h + elb,
// hn = h + el, both after the filter and shift) ...
NPOM_HD void sea_transport_cell(const Ctx &c, int i, int j) {
  if (i >= 1) {
    const float hb = (F2(h, i, j) + F2(elb, i, j)) + (F2(h, i - 1, j) + F2(elb, i - 1, j));
    const float hn = (F2(h, i, j) + F2(el, i, j)) + (F2(h, i - 1, j) + F2(el, i - 1, j));
    P2(utf, i, j) = 0.25f * (F2(uab, i, j) * hb + F2(ua, i, j) * hn);
  }
  if (j >= 1) {
    const float hb = (F2(h, i, j) + F2(elb, i, j)) + (F2(h, i, j - 1) + F2(elb, i, j - 1));
    const float hn = (F2(h, i, j) + F2(el, i, j)) + (F2(h, i, j - 1) + F2(el, i, j - 1));
    P2(vtf, i, j) = 0.25f * (F2(vab, i, j) * hb + F2(va, i, j) * hn);
  }
}

// ... then etf on the interior from the continuity of the interval-mean
// transports, 0.5 (utb + utf) and 0.5 (vtb + vtf), and the mean surface
// volume flux; the east and west edges copy the adjacent column, then the
// mask.  A cell off the interior rows keeps the etf I5 stored.
NPOM_HD float sea_etf_interior(const Ctx &c, int i, int j) {
  auto fx = [&](int ii) {
    return (0.5f * (F2(utb, ii, j) + F2(utf, ii, j))) * 0.5f * (F2(dy, ii, j) + F2(dy, ii - 1, j));
  };
  auto fy = [&](int jj) {
    return (0.5f * (F2(vtb, i, jj) + F2(vtf, i, jj))) * 0.5f * (F2(dx, i, jj) + F2(dx, i, jj - 1));
  };
  const float div = (fx(i + 1) - fx(i) + fy(j + 1) - fy(j)) / (F2(dx, i, j) * F2(dy, i, j));
  const float flux = 0.5f * (F2(vfluxb, i, j) + F2(vfluxf, i, j));
  return F2(etb, i, j) - c.k.dti2 * (div + flux);
}
NPOM_HD float sea_etf_cell(const Ctx &c, int i, int j) {
  const int si = sea_gi(c, i);
  const float v = interior(c, si, j) ? sea_etf_interior(c, si, j) : F2(etf, si, j);
  return v * F2(fsm, i, j);
}

// The coastal tide policy's drag coefficient (coastal_compat.py:4-11):
// (kappa / log((zsh + (1 + zz[kbm1-1]) d) / z0b))^2 on sea cells, cbcmin on
// land, clipped to [cbcmin, cbcmax].  The policy updates it after every
// external substep from the new depth; only the last update reaches a
// reader (the bottom stress of B8), so it runs once after the subcycle.
// The Jiaozhou Bay policy's law (jzb_compat.py:8-27) also needs d >= 0.05 m
// and takes z0b = 0.01 m.
NPOM_HD void cbc_coastal_cell(const Ctx &c, int i, int j) {
  const float dd = F2(d, i, j);
  const bool valid = F2(fsm, i, j) > 0.0f && (!c.k.obc_jzb || dd >= c.k.hc_cbc);
  const float ratio = (c.k.zsh_cbc + (1.0f + F1(zz, c.kb - 2)) * (valid ? dd : 1.0f)) / c.k.z0b_cbc;
  const float q = c.k.kappa / logf(ratio);
  const float v = valid ? q * q : c.k.cbcmin;
  P2(cbc, i, j) = fminf_t(fmaxf_t(v, c.k.cbcmin), c.k.cbcmax);
}

}  // namespace npom
