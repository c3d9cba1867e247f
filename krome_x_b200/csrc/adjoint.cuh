// The discrete adjoint of the lane integrator: the reverse sweep over a
// cell's tape (bdf_lane.cuh, TP_*), one lane per cell.
//
// The differentiated map is the forward solve's own discrete map: the step
// sizes, orders, Newton and error-test decisions are the forward's
// (constants), every Nordsieck operation is linear (rescale, order change,
// Pascal predictor and its undo, the interpolation at tout), and each
// accepted step's corrector is differentiated at its root,
//   acor = gamma f(zn0 + acor) - rl1 zn1
//   (I - gamma J) d acor = gamma J d zn0 - rl1 d zn1 + gamma dF/dm dm,
// with J = dF/dy at the accepted y_n. The forward's Newton matrix is not
// reused for the transposed solves: it is built from a Jacobian up to 20
// steps old at another gamma, which would make the gradient approximate;
// J(y_n) is re-evaluated here instead (the stoichiometric block, central
// differences for the Tgas column and forward differences for the Tgas row,
// or central differences on every column when a rate depends on the
// densities) and I - gamma J factored.
// The per-reaction ln-multiplier terms come from the emitted lnk_vjp.
//
// The same sweep, record for record, is the oracle's adjoint_sweep_
// (oracle/bdf_oracle.cpp); the tests compare the two and check both against
// central finite differences of tight-tolerance solves.
#pragma once

namespace kba {

using namespace kbnet;
using namespace kbw;

// dF/dy at yin, column-major N x N (J[i + j N] = dF_i / dy_j), and the
// rates k at yin; mrow: the rate factors exp(m) (null: none). One
// out-of-line copy: the state is loaded into registers here and every
// perturbed state is built by compile-time selects, so that each full_rhs
// works on registers. With density-independent rates the Tgas row's species
// columns need only the thermal term at the rates of y (the values of the
// oracle's full-rhs differences, whose rates do not move with n), as
// forward differences: their error, ~1e-7 of the row, leaves the gradients
// unchanged at the tests' precision and halves the work.
template <int N, bool EVT>
__device__ __noinline__ void adj_jac(const double* yin, const Params& p,
                                     double Tfix, const double* mrow,
                                     double* J, double* kout) {
  double y[N], f0[N], k[NREA + 1];
  KB_UNROLL for (int i = 0; i < N; ++i) y[i] = yin[i];
  KBL_LOOP for (int i = 0; i < N * N; ++i) J[i] = 0.0;
  full_rhs<N, EVT>(y, f0, p, Tfix, k, mrow);
  KBL_LOOP for (int i = 0; i <= NREA; ++i) kout[i] = k[i];
  double sumabs = 0.0;
  KB_UNROLL for (int i = 0; i < NSPEC; ++i) sumabs += fabs(y[i]);
  if (!RATES_DEPEND_ON_N) {
    jac_stoich(y, k, J, 1, N);
    if (!EVT) return;
    // the Tgas column: the full rhs at T +/- h (the rates move with T)
    {
      const double h = fmax(1e-6 * fabs(y[N - 1]), 1e-8);
      double yp[N], fp[N], fq[N], kk[NREA + 1];
      KB_UNROLL for (int i = 0; i < N; ++i) yp[i] = y[i];
      yp[N - 1] = y[N - 1] + h;
      full_rhs<N, EVT>(yp, fp, p, Tfix, kk, mrow);
      yp[N - 1] = y[N - 1] - h;
      full_rhs<N, EVT>(yp, fq, p, Tfix, kk, mrow);
      KB_UNROLL for (int i = 0; i < N; ++i)
        J[i + (N - 1) * N] = (fp[i] - fq[i]) / (2.0 * h);
    }
    // the Tgas row's species columns: forward differences of the thermal
    // term at the rates of y, from its value at y (the integrator's
    // fd_step_n steps); the cooling's temperature-only parts are evaluated
    // once for the row (thermal_pre: the same values as per column)
    const double Tth = fmin(fmax(y[N - 1], 2.73), 1e9);
    ThermalPre tq;
    thermal_pre(Tth, y, p, tq);
    KBL_LOOP for (int j = 0; j < NSPEC; ++j) {
      double yj = 0.0;
      KB_UNROLL for (int i = 0; i < N; ++i) yj = i == j ? y[i] : yj;
      const double h = fmax(fmax(1e-7 * fabs(yj), 1e-9 * sumabs), 1e-30);
      double yp[N];
      KB_UNROLL for (int i = 0; i < N; ++i) yp[i] = i == j ? yj + h : y[i];
      J[(N - 1) + j * N] =
          (thermal_dTdt_with(tq, Tth, yp, k, p) - f0[N - 1]) / h;
    }
    return;
  }
  // rates that move with the densities: central differences on every column
  KBL_LOOP for (int j = 0; j < N; ++j) {
    const bool tcol = EVT && j == N - 1;
    double yj = 0.0;
    KB_UNROLL for (int i = 0; i < N; ++i) yj = i == j ? y[i] : yj;
    const double h = tcol ? fmax(1e-6 * fabs(yj), 1e-8)
                          : fmax(fmax(1e-7 * fabs(yj), 1e-9 * sumabs), 1e-30);
    double yp[N], fp[N], fq[N], kk[NREA + 1];
    KB_UNROLL for (int i = 0; i < N; ++i) yp[i] = i == j ? yj + h : y[i];
    full_rhs<N, EVT>(yp, fp, p, Tfix, kk, mrow);
    KB_UNROLL for (int i = 0; i < N; ++i) yp[i] = i == j ? yj - h : y[i];
    full_rhs<N, EVT>(yp, fq, p, Tfix, kk, mrow);
    KB_UNROLL for (int i = 0; i < N; ++i) J[i + j * N] = (fp[i] - fq[i]) / (2.0 * h);
  }
}

// the adjoint state of one cell: lam over the Nordsieck array, the
// ln-multiplier gradient, scratch
template <int N>
struct AdjCell {
  double lam[L_MAX][N];
  double gm[NREA + 1];
  double J[N * N];  // dF/dy, overwritten by (I - gamma J)^T and its LU
  double mu[N], la[N], yv[N];
  double k[NREA + 1];
  int piv[N];
};

// the length a record of kind op has, -1 for an unknown kind
template <int N>
__device__ __forceinline__ long record_len(int op) {
  return op == kbl::TP_INIT || op == kbl::TP_RESET1 ? 3 + N
       : op == kbl::TP_RESCALE || op == kbl::TP_DKY ? 4
       : op == kbl::TP_INCREASE ? 4 + L_MAX
       : op == kbl::TP_DECREASE ? 3 + L_MAX
       : op == kbl::TP_PREDICT || op == kbl::TP_RESTORE ? 3
       : op == kbl::TP_CORRECT ? 6 + L_MAX + N : -1;
}

// the gradients of a finished cell
template <int N, bool EVT>
__device__ void adj_write(const AdjCell<N>& a, int c, double* dn0,
                          double* dT0, double* dm) {
  KBL_LOOP for (int i = 0; i < NSPEC; ++i) dn0[(long)c * NSPEC + i] = a.lam[0][i];
  if (EVT && dT0 != nullptr) dT0[c] = a.lam[0][N - 1];
  KBL_LOOP for (int r = 0; r < NREA; ++r) dm[(long)c * NREA + r] = a.gm[r];
}

// The reverse sweep, one cell per lane at a time: cell c's tape, seeded with
// gn[c][:], gT[c] (components clipped to 0 by the forward get no seed);
// out: dn0[c][NSPEC], dT0[c] (evolve_T), dm[c][NREA]. Cells that failed or
// recorded nothing get zero gradients. Lanes take their cells from the work
// queue `cursor` (reset by the caller), so that a lane whose tape ends takes
// the next cell instead of idling until the longest tape of its warp ends.
//
// The sweep runs in rounds so that the expensive records (a corrector, an
// initial or restarted zn[1] = h f: each needs dF/dy) are processed by the
// lanes of a warp together: in a round every lane first consumes its cheap
// records (linear Nordsieck maps) up to its next expensive one, then the
// lanes holding one evaluate their Jacobians and apply them in step.
// Bounded: every pass of the inner loop consumes a record or a cell index;
// every record is validated (its length is its kind's, its order in
// 1..QMAX) and a damaged record ends its cell's sweep.
#ifndef KBA_MINB
#define KBA_MINB 2  // resident 128-thread blocks per SM the sweep is built for
#endif
template <bool EVT>
__global__ void __launch_bounds__(128, KBA_MINB)
kb_adjoint_cells(int ncell, const double* T0, const double* par, int pstride,
                 const double* mult, int mstride, const double* gn,
                 const double* gT, const int* flags, const double* tape,
                 long cap, const long* tlen, const double* yfin, int clip,
                 double* dn0, double* dT0, double* dm, unsigned* cursor) {
  constexpr int N = NSPEC + (EVT ? 1 : 0);
  constexpr unsigned FULLM = 0xffffffffu;
  int c = -1;          // the cell being swept by this lane
  bool more = true;    // the queue may hold more cells
  long pos = 0;
  Params p;
  double Tfix = 0.0;
  const double* mrow = nullptr;
  const double* tp = tape;
  AdjCell<N> a;
  double lamy[N];
  for (;;) {
    // ---- this lane's cheap records, up to its next expensive one ----
    int pend = 0;
    const double* pr = nullptr;
    for (;;) {
      if (c < 0) {
        if (!more) break;
        const int nc = (int)atomicAdd(cursor, 1u);
        if (nc >= ncell) {
          more = false;
          break;
        }
        c = nc;
        KBL_LOOP for (int r = 0; r < NREA; ++r) dm[(long)c * NREA + r] = 0.0;
        KBL_LOOP for (int i = 0; i < NSPEC; ++i) dn0[(long)c * NSPEC + i] = 0.0;
        if (dT0 != nullptr) dT0[c] = 0.0;
        const long total = tlen[c];
        if (flags[c] != 0 || total <= 0 || total > cap) {
          c = -1;
          continue;
        }
        pos = total;
        params_from_row(par + (long)c * pstride, p);
        Tfix = T0[c];
        mrow = mult != nullptr ? mult + (long)c * mstride : nullptr;
        tp = tape + (long)c * cap;
        KBL_LOOP for (int j = 0; j < L_MAX; ++j)
          KBL_LOOP for (int i = 0; i < N; ++i) a.lam[j][i] = 0.0;
        KBL_LOOP for (int r = 0; r <= NREA; ++r) a.gm[r] = 0.0;
        KBL_LOOP for (int i = 0; i < NSPEC; ++i) {
          const bool clipped = clip && yfin[(long)c * N + i] < 0.0;
          lamy[i] = clipped ? 0.0 : gn[(long)c * NSPEC + i];
        }
        if (EVT) lamy[N - 1] = gT != nullptr ? gT[c] : 0.0;
      }
      bool end = pos <= 0;
      long len = 0;
      const double* r = nullptr;
      int op = 0;
      if (!end) {
        len = (long)tp[pos - 1];
        end = len < 2 || len > pos;
      }
      if (!end) {
        r = tp + (pos - len);
        op = (int)r[0];
        end = len != record_len<N>(op);
      }
      if (!end && op != kbl::TP_INIT && op != kbl::TP_RESET1) {
        const double qd = r[op == kbl::TP_RESCALE || op == kbl::TP_DKY ? 2 : 1];
        end = !(qd >= 1.0 && qd <= QMAX);
      }
      if (end) {  // the tape is consumed (or damaged): the cell is done
        adj_write<N, EVT>(a, c, dn0, dT0, dm);
        c = -1;
        continue;
      }
      pos -= len;
      if (op == kbl::TP_CORRECT || op == kbl::TP_INIT || op == kbl::TP_RESET1) {
        pend = op;
        pr = r;
        break;
      }
      if (op == kbl::TP_DKY) {
        const double sv = r[1];
        const int q = (int)r[2];
        KBL_LOOP for (int j = 0; j <= q; j++) {
          double cj = 1.0;
          KBL_LOOP for (int i = 0; i < j; i++) cj *= sv;
          KBL_LOOP for (int i = 0; i < N; i++) a.lam[j][i] += cj * lamy[i];
        }
      } else if (op == kbl::TP_PREDICT || op == kbl::TP_RESTORE) {
        const int q = (int)r[1];
        const double sg = op == kbl::TP_PREDICT ? 1.0 : -1.0;
        KBL_LOOP for (int k = q; k >= 1; k--)
          KBL_LOOP for (int j = k; j <= q; j++)
            KBL_LOOP for (int i = 0; i < N; i++) a.lam[j][i] += sg * a.lam[j - 1][i];
      } else if (op == kbl::TP_RESCALE) {
        const double eta = r[1];
        const int q = (int)r[2];
        double cj = eta;
        KBL_LOOP for (int j = 1; j <= q; j++) {
          KBL_LOOP for (int i = 0; i < N; i++) a.lam[j][i] *= cj;
          cj = eta * cj;
        }
      } else if (op == kbl::TP_INCREASE) {
        const int q = (int)r[1];
        const double A1 = r[2];
        const double* l = r + 3;
        const int L = q + 1;
        KBL_LOOP for (int j = 2; j <= q; j++)
          KBL_LOOP for (int i = 0; i < N; i++) a.lam[L][i] += l[j] * a.lam[j][i];
        if (L == QMAX) {
          KBL_LOOP for (int i = 0; i < N; i++) a.lam[QMAX][i] *= A1;
        } else {
          KBL_LOOP for (int i = 0; i < N; i++) {
            a.lam[QMAX][i] += A1 * a.lam[L][i];
            a.lam[L][i] = 0.0;
          }
        }
      } else if (op == kbl::TP_DECREASE) {
        const int q = (int)r[1];
        const double* l = r + 2;
        KBL_LOOP for (int j = 2; j < q; j++)
          KBL_LOOP for (int i = 0; i < N; i++) a.lam[q][i] -= l[j] * a.lam[j][i];
      }
    }
    // a lane leaves the loop above without an expensive record only when
    // the queue is exhausted and its last cell is written
    if (__all_sync(FULLM, pend == 0)) break;
    if (pend == 0) continue;
    // ---- the expensive records, the warp's lanes together ----
    const double* r = pr;
    const bool corr = pend == kbl::TP_CORRECT;
    const double* yrec = corr ? r + 5 + L_MAX : r + 2;
    KBL_LOOP for (int i = 0; i < N; i++) a.yv[i] = yrec[i];
    adj_jac<N, EVT>(a.yv, p, Tfix, mrow, a.J, a.k);
    const double Tth = EVT ? fmin(fmax(a.yv[N - 1], 2.73), 1e9)
                           : fmin(fmax(Tfix, 2.73), 1e9);
    if (corr) {
      // (I - gamma J)^T mu = lam_acor; lam0 += gamma J^T mu = mu - lam_acor,
      // lam1 -= rl1 mu, gm += gamma dF/dm^T mu
      const int q = (int)r[1];
      const double gam = r[2], rl1 = r[3];
      const double* l = r + 4;
      const bool save = r[4 + L_MAX] != 0.0;
      KBL_LOOP for (int i = 0; i < N; i++) {
        double t = save ? a.lam[QMAX][i] : 0.0;
        KBL_LOOP for (int j = 0; j <= q; j++) t += l[j] * a.lam[j][i];
        a.la[i] = t;
      }
      if (save) KBL_LOOP for (int i = 0; i < N; i++) a.lam[QMAX][i] = 0.0;
      // J := (I - gamma J)^T in place
      KBL_LOOP for (int j = 0; j < N; j++) {
        KBL_LOOP for (int i = 0; i < j; i++) {
          const double x = a.J[i + j * N], y = a.J[j + i * N];
          a.J[i + j * N] = -gam * y;
          a.J[j + i * N] = -gam * x;
        }
        a.J[j + j * N] = 1.0 - gam * a.J[j + j * N];
      }
      kbl::getrf_<N, double>(a.J, a.piv);
      KBL_LOOP for (int i = 0; i < N; i++) a.mu[i] = a.la[i];
      kbl::getrs_<N, double>(a.J, a.piv, a.mu);
      KBL_LOOP for (int i = 0; i < N; i++) {
        a.lam[0][i] += a.mu[i] - a.la[i];
        a.lam[1][i] -= rl1 * a.mu[i];
        a.mu[i] *= gam;
      }
    } else {
      // TP_INIT, TP_RESET1: zn[1] = h f(y): lam0 += h J^T lam1,
      // gm += h dF/dm^T lam1, lam1 = 0
      const double h = r[1];
      KBL_LOOP for (int i = 0; i < N; ++i) a.mu[i] = h * a.lam[1][i];
      KBL_LOOP for (int j = 0; j < N; ++j) {
        double t = 0.0;
        KBL_LOOP for (int i = 0; i < N; ++i) t += a.J[i + j * N] * a.mu[i];
        a.lam[0][j] += t;
      }
      KBL_LOOP for (int i = 0; i < N; ++i) a.lam[1][i] = 0.0;
      if (pend == kbl::TP_INIT)
        KBL_LOOP for (int j = 1; j < L_MAX; j++)
          KBL_LOOP for (int i = 0; i < N; i++) a.lam[j][i] = 0.0;
    }
    lnk_vjp(a.yv, a.k, Tth, p, a.mu, EVT ? a.mu[N - 1] : 0.0, a.gm);
  }
}

}  // namespace kba
