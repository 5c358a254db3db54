// npom_ctx.cuh -- execution context shared by every phase of the step.
//
// A phase body is a __host__ __device__ function of one grid point, one
// water column or one 2-D cell.  The CUDA kernels map threads onto those
// bodies; the CPU emulator used by the tests runs the very same bodies in
// loops, which checks the index logic of every phase against the oracle
// without a GPU.
#pragma once

#include <math.h>
#include <stddef.h>
#include <stdint.h>

#include "../../include/npom.h"

#if defined(__CUDACC__)
#define NPOM_HD __host__ __device__ __forceinline__
#else
#define NPOM_HD inline
#endif

namespace npom {

// Plain loads are L1-cached and coherent within a thread block, which is all
// the one-phase kernels need (a phase never reads what another block writes
// in the same launch).  The persistent cooperative kernels read values that
// other blocks wrote before a grid barrier, so they load through L2
// (ld.global.cg); Ctx::coh selects that path.
NPOM_HD float ld(const float *p) { return *p; }

// Scalars of the step, pre-folded the way the reference folds its Python
// float constants (in double, rounded once to float when they meet a
// float32 tensor).
struct Consts {
  float dti2, dte2, two_dti2, neg_dti2, neg_two_dti2, four_dte, four_dti, two_dti;
  float ispi, isp2i, half_smoth, quarter_smoth, etf_mid, smoth;
  float horcon, umol, two_umol, tprni, small, kappa, rhoref, tbias, sbias, aam_min;
  float alpha, one_m_2alpha, half_g, quarter_g, g_eighth, grav, g_rhoref, g2x2;
  float sqrt_half, prof_const1, prof_gg0, surfl, wind_kf, two_pi, dti, hmax;
  float rfe, rfw, rfn, rfs, vmaxl, vmix;
  float bshap_q, tshap_q, vshap_q;  // gamma / 4 of the three Shapiro filters
  double bshap, tshap, vshap;
  float implicit_coeff, inverse_scale;
  int isplit, ispadv, nbct, nbcs, ntp, mode, core, wind_forcing, has_vmix, nadv, nitera;
  float sw;
  int eta_max_iter, eta_precond;
  double eta_tol, eta_rel_tol;
  int profq_pom08;     // PROFQ in the POM08-WAD form
  float kappa_zsh;     // POM08-WAD: kappa * zsh (folded in double)
  int obc_seamount;    // the seamount case policy's boundary (explicit core)
  int obc_coastal;     // the coastal tide policy's machinery (also set for JZB)
  int obc_jzb;         // the Jiaozhou Bay tide policy
  int sea_implicit;    // the seamount policy on the semi-implicit core
  int periodic_x;      // periodic x: two halo columns each side, unique columns 2..im-3
  double tide_w;       // tide angular speed, rad/h, as the policy writes it
  double dte_d;        // dte in double (tide time of a substep)
  float zsh_cbc, z0b_cbc, cbcmin, cbcmax;  // coastal policy's drag coefficient
  float hc_cbc;                           // JZB: the drag law from this depth on
};

struct Ctx {
  int im, jm, kb;
  float *F[NPOM_NFIELDS];
  float *W[NPOM_NWS];
  double *partials;
  unsigned int *sync;
  unsigned int *status;
  int *cg_iters;
  float *mp3d;  // MPDATA scratch (nadv 2)
  const float *tide;  // coastal policy: tide flag, amplitude, phase planes
  double *robin;      // semi-implicit seamount policy: the FP64 Robin solve's planes
  double tide_t0;     // coastal policy: seconds at the start of the step
  Consts k;
  int coh;         // 1: loads bypass L1 (persistent cooperative kernels)
  // the blocks of a cooperative launch that work on this context: blocks
  // [grid_base, grid_base + grid_blocks) (grid_blocks 0: the whole grid);
  // several members share one launch, each with its own grid barrier
  int grid_base, grid_blocks;
  // when set: the PCG's absolute tolerance is eta_tol / max(f, 1) with f
  // the float whose bits are stored here (the adjoint solve's rhs scale,
  // kept on the device)
  const unsigned int *tol_scale_bits;
  float ramp;      // per step
  int do_internal; // per step: 0 on the first step from time0 == 0
  npom_tuning tune;  // launch shapes (host-side decisions only)
};

NPOM_HD float ldc(const Ctx &c, const float *p) {
#if defined(__CUDA_ARCH__)
  return c.coh ? __ldcg(p) : *p;
#else
  (void)c;
  return *p;
#endif
}

// ---- indexing ----------------------------------------------------------
#define NPOM_I2(c, i, j) ((size_t)(i) * (c).jm + (size_t)(j))
#define NPOM_I3(c, i, j, k) (((size_t)(i) * (c).jm + (size_t)(j)) * (c).kb + (size_t)(k))

#define F3(name, i, j, k) ::npom::ldc(c, &c.F[NPOM_F_##name][NPOM_I3(c, i, j, k)])
#define F2(name, i, j) ::npom::ldc(c, &c.F[NPOM_F_##name][NPOM_I2(c, i, j)])
#define F1(name, k) ::npom::ldc(c, &c.F[NPOM_F_##name][(k)])
#define P3(name, i, j, k) (c.F[NPOM_F_##name][NPOM_I3(c, i, j, k)])
#define P2(name, i, j) (c.F[NPOM_F_##name][NPOM_I2(c, i, j)])
#define W2(name, i, j) ::npom::ldc(c, &c.W[NPOM_W_##name][NPOM_I2(c, i, j)])
#define PW2(name, i, j) (c.W[NPOM_W_##name][NPOM_I2(c, i, j)])

NPOM_HD bool interior(const Ctx &c, int i, int j) {
  return i >= 1 && i <= c.im - 2 && j >= 1 && j <= c.jm - 2;
}

NPOM_HD float fmaxf_t(float a, float b) {
  // torch.maximum / clamp semantics: NaN propagates
  return (a != a) ? a : ((b != b) ? b : (a > b ? a : b));
}
NPOM_HD float fminf_t(float a, float b) {
  return (a != a) ? a : ((b != b) ? b : (a < b ? a : b));
}

}  // namespace npom
