// Scalar recurrences of the Krylov solvers, executed on the device by one
// warp of the fold kernel of the reduction that produces their inputs
// (fold_kernel in blas.cu, on a shared-memory copy of the solver state).
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

__device__ __forceinline__ bool all_done(const SolverState *st, int nrhs, int lane)
{
  return __all_sync(0xffffffffu, lane >= nrhs || st->rhs_done[lane] != 0);
}

// Executed by all 32 lanes of one warp on the state (a shared-memory copy in
// the fold kernel): lane r carries right-hand side (or shift) r, nrhs <= 32,
// so the per-rhs recurrences run side by side.  A lane writes only its own
// rhs's slots; the scalars every lane shares (iteration counter, done and
// status flags, multishift CG's slot-0 scalars) are read by all lanes before
// the __syncwarp() that precedes lane 0's update of them.  The arithmetic of
// each rhs is the serial recurrence's, operation for operation.
template <int FIN>
__device__ void finalize_warp(SolverState *st, const double *res, int nrhs, int nval, int lane)
{
  double(*v)[QPX_MAX_RHS] = st->v;
  const int r = lane;
  const bool live = r < nrhs && !st->rhs_done[r];
  // ---- CG (include/qphix/invcg.h:281-417) --------------------------------
  // shifted CG (M^+M + s, s = v[S_AUX3], 0 for plain CG): <p, (M^+M + s) p> =
  // |Mp|^2 + s |p|^2, with |p|^2 from the p update's fold (FIN_CG_P, v[S_AUX4])
  if constexpr (FIN == FIN_CG_A) {
    if (live) {
      double d = res[r * nval];
      if (v[S_AUX3][r] != 0.0) d += v[S_AUX3][r] * v[S_AUX4][r];
      v[S_D][r] = d;
      v[S_A][r] = v[S_C][r] / v[S_D][r];
    }
  } else if constexpr (FIN == FIN_CG_P) {
    if (live) v[S_AUX4][r] = res[r * nval];
  } else if constexpr (FIN == FIN_CG_R) {
    if (live) {
      double cp = res[r * nval];
      v[S_RNORM][r] = cp;
      if (cp < v[S_RSD][r]) {
        stop_rhs(st, r, 1);
        st->rhs_iter[r] = st->iter;  // the reference reports k, the 0-based index
      } else {
        v[S_B][r] = cp / v[S_C][r];
        v[S_C][r] = cp;
      }
    }
    __syncwarp();
    if (lane == 0) end_iteration(st, nrhs);
  }
  // ---- BiCGStab (include/qphix/invbicgstab.h:156-254) --------------------
  else if constexpr (FIN == FIN_BICG_ALPHA) {
    if (live) {
      double ar = res[r * nval], ai = res[r * nval + 1];
      if (ar == 0.0 && ai == 0.0) {
        stop_rhs(st, r, 2);
      } else {
        cdiv(v[S_ALPHA_RE][r], v[S_ALPHA_IM][r], v[S_RHO_RE][r], v[S_RHO_IM][r], ar, ai);
        v[S_RHOP_RE][r] = v[S_RHO_RE][r];
        v[S_RHOP_IM][r] = v[S_RHO_IM][r];
      }
    }
    if (all_done(st, nrhs, lane) && lane == 0) st->done = 1;
  } else if constexpr (FIN == FIN_BICG_OMEGA) {
    if (live) {
      double tn = res[r * nval];
      v[S_TNORM][r] = tn;
      if (tn == 0.0) {
        stop_rhs(st, r, 2);
      } else {
        v[S_OMEGA_RE][r] = res[r * nval + 1] / tn;
        v[S_OMEGA_IM][r] = res[r * nval + 2] / tn;
      }
    }
    if (all_done(st, nrhs, lane) && lane == 0) st->done = 1;
  } else if constexpr (FIN == FIN_BICG_RX) {
    if (live) {
      double rn = res[r * nval];
      v[S_RNORM][r] = rn;
      double rr = res[r * nval + 1], ri = res[r * nval + 2];
      if (rn < v[S_RSD][r]) {
        stop_rhs(st, r, 1);
      } else if (rr == 0.0 && ri == 0.0) {
        stop_rhs(st, r, 2);
      } else {
        v[S_RHO_RE][r] = rr;
        v[S_RHO_IM][r] = ri;
        double t1r, t1i, t2r, t2i;
        cdiv(t1r, t1i, rr, ri, v[S_RHOP_RE][r], v[S_RHOP_IM][r]);
        cdiv(t2r, t2i, v[S_ALPHA_RE][r], v[S_ALPHA_IM][r], v[S_OMEGA_RE][r], v[S_OMEGA_IM][r]);
        v[S_BETA_RE][r] = t1r * t2r - t1i * t2i;
        v[S_BETA_IM][r] = t1r * t2i + t1i * t2r;
      }
    }
    __syncwarp();
    if (lane == 0) end_iteration(st, nrhs);
  }
  // ---- BiCGStab with reliable updates ---------------------------------------
  // As FIN_BICG_RX, but instead of stopping, right-hand sides whose iterated
  // residual fell below their update threshold (S_AUX1, delta^2 |r_true|^2 at
  // the last update) or their target ask the host for a reliable update:
  // st->status = 3 and the iteration graph stops (done) until the host has
  // replaced r by the recomputed true residual.  One update serves every
  // right-hand side of the batch, so it is asked for once half of the active
  // ones have crossed, or as soon as one has fallen ten times below its
  // threshold (before the low-precision recurrence drifts from the true
  // residual); with one or two right-hand sides that is any crossing.
  else if constexpr (FIN == FIN_BICG_RU) {
    bool crossed = false, request = false;
    if (live) {
      double rn = res[r * nval];
      v[S_RNORM][r] = rn;
      crossed = rn < v[S_AUX1][r] || rn < v[S_RSD][r];
      request = rn < 0.1 * v[S_AUX1][r];
      double rr = res[r * nval + 1], ri = res[r * nval + 2];
      if (rr == 0.0 && ri == 0.0) {
        request = true;  // let the true residual decide
      } else {
        v[S_RHO_RE][r] = rr;
        v[S_RHO_IM][r] = ri;
        double t1r, t1i, t2r, t2i;
        cdiv(t1r, t1i, rr, ri, v[S_RHOP_RE][r], v[S_RHOP_IM][r]);
        cdiv(t2r, t2i, v[S_ALPHA_RE][r], v[S_ALPHA_IM][r], v[S_OMEGA_RE][r], v[S_OMEGA_IM][r]);
        v[S_BETA_RE][r] = t1r * t2r - t1i * t2i;
        v[S_BETA_IM][r] = t1r * t2i + t1i * t2r;
      }
    }
    const int active = __popc(__ballot_sync(0xffffffffu, live));
    const int ncrossed = __popc(__ballot_sync(0xffffffffu, crossed));
    request = __any_sync(0xffffffffu, request);
    __syncwarp();
    if (lane == 0) {
      end_iteration(st, nrhs);
      if (2 * ncrossed >= active && ncrossed > 0) request = true;
      if (request) {
        st->done = 1;
        st->status = 3;
      }
    }
  }
  // ---- MR (include/qphix/invmr.h:143-190) ---------------------------------
  else if constexpr (FIN == FIN_MR_A) {
    if (live) {
      double d = res[r * nval];
      v[S_ALPHA_RE][r] = v[S_AUX0][r] * res[r * nval + 1] / d;
      v[S_ALPHA_IM][r] = v[S_AUX0][r] * res[r * nval + 2] / d;
    }
  } else if constexpr (FIN == FIN_MR_R) {
    if (live) {
      double cp = res[r * nval];
      v[S_RNORM][r] = cp;
      if (!(cp > v[S_RSD][r])) stop_rhs(st, r, 1);
    }
    __syncwarp();
    if (lane == 0) end_iteration(st, nrhs);
  }
  // ---- multishift CG (include/qphix/minvcg.h:279-384) -------------------
  // scalars in slot [0]: a S_A, b S_B, c S_C, d S_D, cp S_AUX4, bp S_AUX5;
  // per shift s: zeta S_AUX0, zeta_prev S_AUX1, beta S_BETA_RE, as S_AUX2,
  // shift S_AUX3, pending x coefficient S_AUX6, target S_RSD, final S_RNORM
  else if constexpr (FIN == FIN_MCG_D) {
    if (lane == 0) {
      v[S_AUX4][0] = v[S_C][0];  // cp = c
      v[S_AUX5][0] = v[S_B][0];  // bp = b
      v[S_D][0] = res[0];
      v[S_B][0] = -v[S_AUX4][0] / v[S_D][0];
    }
  } else if constexpr (FIN == FIN_MCG_R) {
    // one base system (nrhs = 1); the shifts are the state's st->nrhs entries
    const int nsh = st->nrhs;
    const double c = res[0], b = v[S_B][0], bp = v[S_AUX5][0], a = v[S_A][0];
    const double an = c / v[S_AUX4][0];  // the next iteration's a
    const int sh = lane;
    if (sh < nsh) {
      if (st->rhs_done[sh]) {
        v[S_AUX6][sh] = 0.0;
      } else {
        double z0 = v[S_AUX0][sh], z1 = v[S_AUX1][sh];
        v[S_AUX1][sh] = z0;
        double z = z0 * z1 * bp;
        z /= (b * a * (z1 - z0) + z1 * bp * (1.0 - v[S_AUX3][sh] * b));
        v[S_AUX0][sh] = z;
        v[S_BETA_RE][sh] = b * z / z0;
        v[S_AUX6][sh] = v[S_BETA_RE][sh];
        double css = c * z * z;
        if (css < v[S_RSD][sh]) {
          st->rhs_done[sh] = 1;
          st->rhs_iter[sh] = st->iter + 1;
          v[S_RNORM][sh] = css;
        }
        // coefficient of the next iteration's p update
        if (!st->rhs_done[sh]) v[S_AUX2][sh] = an * v[S_AUX0][sh] * v[S_BETA_RE][sh] / (v[S_AUX1][sh] * b);
      }
    }
    const bool all = all_done(st, nsh, lane);
    __syncwarp();
    if (lane == 0) {
      v[S_C][0] = c;
      v[S_A][0] = an;
      st->iter++;
      if (all) {
        st->done = 1;
      } else if (st->iter + 1 >= st->max_iter) {  // the reference loop runs k = 1 .. MaxIters - 1
        st->done = 1;
        st->status = 1;
      }
    }
  }
}

}  // namespace qpx
