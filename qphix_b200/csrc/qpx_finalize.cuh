// Scalar recurrences of the Krylov solvers, executed on the device by the
// last block of the reduction that produces their inputs (see qpx_reduce.cuh).
// Each follows the host-side scalar arithmetic of the reference solver cited
// beside it; a right-hand side that has converged (or broken down) gets zero
// update coefficients so that later iterations leave its x and r untouched.
#pragma once

#include "qpx_reduce.cuh"

namespace qpx {

__device__ __forceinline__ void cdiv(double &rr, double &ri, double ar, double ai, double br, double bi)
{
  double d = br * br + bi * bi;
  double re = (ar * br + ai * bi) / d;
  double im = (ai * br - ar * bi) / d;
  rr = re;
  ri = im;
}

__device__ __forceinline__ void end_iteration(SolverState *st, int nrhs)
{
  st->iter++;
  bool all = true;
  for (int r = 0; r < nrhs; r++) all = all && (st->rhs_done[r] != 0);
  if (all) {
    st->done = 1;
  } else if (st->iter >= st->max_iter) {
    st->done = 1;
    st->status = 1;
  }
}

__device__ __forceinline__ void stop_rhs(SolverState *st, int r, int how)
{
  st->rhs_done[r] = how;
  st->rhs_iter[r] = st->iter + 1;
  st->v[S_A][r] = 0;
  st->v[S_B][r] = 0;
  st->v[S_ALPHA_RE][r] = 0;
  st->v[S_ALPHA_IM][r] = 0;
  st->v[S_OMEGA_RE][r] = 0;
  st->v[S_OMEGA_IM][r] = 0;
  st->v[S_BETA_RE][r] = 0;
  st->v[S_BETA_IM][r] = 0;
  if (how == 2) st->status = 2;
}

__device__ inline void finalize(int fin, SolverState *st, const double *res, int nrhs, int nval)
{
  double(*v)[QPX_MAX_RHS] = st->v;
  switch (fin) {
  case FIN_STORE:
    break;
  // ---- CG (include/qphix/invcg.h:281-417) --------------------------------
  case FIN_CG_A:
    for (int r = 0; r < nrhs; r++) {
      if (st->rhs_done[r]) continue;
      v[S_D][r] = res[r * nval];
      v[S_A][r] = v[S_C][r] / v[S_D][r];
    }
    break;
  case FIN_CG_R:
    for (int r = 0; r < nrhs; r++) {
      if (st->rhs_done[r]) continue;
      double cp = res[r * nval];
      v[S_RNORM][r] = cp;
      if (cp < v[S_RSD][r]) {
        stop_rhs(st, r, 1);
        st->rhs_iter[r] = st->iter;  // the reference reports k, the 0-based index
        continue;
      }
      v[S_B][r] = cp / v[S_C][r];
      v[S_C][r] = cp;
    }
    end_iteration(st, nrhs);
    break;
  // ---- BiCGStab (include/qphix/invbicgstab.h:156-254) --------------------
  case FIN_BICG_ALPHA:
    for (int r = 0; r < nrhs; r++) {
      if (st->rhs_done[r]) continue;
      double ar = res[r * nval], ai = res[r * nval + 1];
      if (ar == 0.0 && ai == 0.0) {
        stop_rhs(st, r, 2);
        continue;
      }
      cdiv(v[S_ALPHA_RE][r], v[S_ALPHA_IM][r], v[S_RHO_RE][r], v[S_RHO_IM][r], ar, ai);
      v[S_RHOP_RE][r] = v[S_RHO_RE][r];
      v[S_RHOP_IM][r] = v[S_RHO_IM][r];
    }
    {
      bool all = true;
      for (int r = 0; r < nrhs; r++) all = all && st->rhs_done[r];
      if (all) st->done = 1;
    }
    break;
  case FIN_BICG_OMEGA:
    for (int r = 0; r < nrhs; r++) {
      if (st->rhs_done[r]) continue;
      double tn = res[r * nval];
      v[S_TNORM][r] = tn;
      if (tn == 0.0) {
        stop_rhs(st, r, 2);
        continue;
      }
      v[S_OMEGA_RE][r] = res[r * nval + 1] / tn;
      v[S_OMEGA_IM][r] = res[r * nval + 2] / tn;
    }
    {
      bool all = true;
      for (int r = 0; r < nrhs; r++) all = all && st->rhs_done[r];
      if (all) st->done = 1;
    }
    break;
  case FIN_BICG_RX:
    for (int r = 0; r < nrhs; r++) {
      if (st->rhs_done[r]) continue;
      double rn = res[r * nval];
      v[S_RNORM][r] = rn;
      if (rn < v[S_RSD][r]) {
        stop_rhs(st, r, 1);
        continue;
      }
      double rr = res[r * nval + 1], ri = res[r * nval + 2];
      if (rr == 0.0 && ri == 0.0) {
        stop_rhs(st, r, 2);
        continue;
      }
      v[S_RHO_RE][r] = rr;
      v[S_RHO_IM][r] = ri;
      double t1r, t1i, t2r, t2i;
      cdiv(t1r, t1i, rr, ri, v[S_RHOP_RE][r], v[S_RHOP_IM][r]);
      cdiv(t2r, t2i, v[S_ALPHA_RE][r], v[S_ALPHA_IM][r], v[S_OMEGA_RE][r], v[S_OMEGA_IM][r]);
      v[S_BETA_RE][r] = t1r * t2r - t1i * t2i;
      v[S_BETA_IM][r] = t1r * t2i + t1i * t2r;
    }
    end_iteration(st, nrhs);
    break;
  // ---- MR (include/qphix/invmr.h:143-190) ---------------------------------
  case FIN_MR_A:
    for (int r = 0; r < nrhs; r++) {
      if (st->rhs_done[r]) continue;
      double d = res[r * nval];
      v[S_ALPHA_RE][r] = v[S_AUX0][r] * res[r * nval + 1] / d;
      v[S_ALPHA_IM][r] = v[S_AUX0][r] * res[r * nval + 2] / d;
    }
    break;
  case FIN_MR_R:
    for (int r = 0; r < nrhs; r++) {
      if (st->rhs_done[r]) continue;
      double cp = res[r * nval];
      v[S_RNORM][r] = cp;
      if (!(cp > v[S_RSD][r])) stop_rhs(st, r, 1);
    }
    end_iteration(st, nrhs);
    break;
  default:
    break;
  }
}

}  // namespace qpx
