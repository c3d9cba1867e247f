// Lane-per-cell CVODE BDF integrator for sm_100a: each lane of a warp
// integrates its own cell, and the warp serves the lanes' right-hand-side
// and Jacobian requests together.
//
// Why this layout. The network math (rate coefficients with their exp /
// log / pow, the thermal terms) dominates the solve and is scalar per
// cell. With one warp per cell (bdf_warp.cuh) every lane evaluates the
// same state, so a warp instruction does one cell's work; here a warp
// instruction evaluates 32 cells. The integrator's control flow differs
// between cells (Newton iteration counts, Jacobian refreshes, failed
// attempts, cells that finish early), so each lane keeps its place in
// CVODE as a phase and stops at every rhs or Jacobian request:
//
//   loop:  1. one sweep runs the phase handlers in a fixed order, each a
//             structured block over the lanes in that phase (cheap O(N) and
//             O(N^2) vector work in the lane's private memory); a lane
//             passes through as many handlers as its cell needs, and the
//             order follows CVODE's flow, so every lane reaches its next
//             request within the sweep. Lanes in the same phase execute a
//             handler together and reconverge after it. A lane whose cell
//             is done writes it back and takes the next cell (a fixed one,
//             or the next one of the device work queue in the persistent
//             kernel), so lanes never wait for the slowest cell of their
//             warp;
//          2. Jacobian requests are served by the whole warp: lane j of a
//             request's group evaluates the rhs perturbed in component j
//             (the difference-quotient columns, or the hybrid analytic
//             Jacobian's thermal-row and Tgas-column terms), the columns
//             meet in shared memory;
//          3. all lanes with an rhs request evaluate it in one SIMT pass.
//
// The algorithm and every decision are CVODE's as the reference ports it
// (runtime/core/cvode/bdf_cell.hpp:490-1547: cvHin, cvStep, the modified
// Newton iteration, cvLsSetup's reuse heuristics, the dense LU with
// partial pivoting, the error test, the step and order selection, the
// restart wrapper) around the reference's per-cell problem
// (runtime/core/solve_cell.hpp:750-813, 883-1118, 1631-1642, 2094-2203).
// Every loop is bounded as in bdf_warp.cuh (max_steps, the per-step
// failure limits, max_restarts; the queue loop by the number of cells).
#pragma once

namespace kbl {

using namespace kbnet;
using kbw::SolveOpts;
using kbw::NSTAT;
using namespace kbw;  // flags and CVODE constants

// what a lane waits for at the end of a sweep
enum : int { WAIT_NONE = 0, WAIT_RHS = 1, WAIT_JAC = 2 };

// the phases, in the order one sweep runs their handlers
enum : int {
  PH_RES_OUTER = 0,  // consume the rhs of a Newton pass's first residual
  PH_RES_INNER,      // consume the rhs of a later Newton residual
  PH_SETUP,          // cvLsSetup: reuse J or ask the warp for it
  PH_LSFINISH,       // A = I - gamma J, its LU, cvNlsLSetup's bookkeeping
  PH_NEWTON,         // one Newton iteration and its convergence test
  PH_NLS_AFTER,      // a failed Newton pass: retry with a fresh J?
  PH_NLS_END,        // cvNls' tail, cvHandleNFlag, cvDoErrorTest
  PH_ERRTEST_RHS,    // consume the rhs of the order-1 restart of a step
  PH_STEP_OK,        // cvCompleteStep, cvPrepareNextStep, tout reached?
  PH_SOLVE_END,      // the restart wrapper
  PH_SOLVE,          // CVode's first-call block
  PH_FIRST_RHS,      // consume f(t0, y0)
  PH_HIN_START,      // cvHin's bounds
  PH_HIN_RHS,        // consume cvYddNorm's rhs
  PH_HIN_REQ,        // cvYddNorm: request the rhs at t0 + hg
  PH_AFTER_HIN,      // the first step size is known
  PH_STEP,           // the CVode loop top and cvStep's prologue
  PH_ATTEMPT,        // predict, cvSet, cvNls' set-up
  PH_NLS_OUTER,      // request the rhs of a Newton pass's first residual
  PH_DONE,           // the cell is finished (flag set): take the next one
  PH_IDLE            // no cell left for this lane
};

// the discrete adjoint's tape: every operation of the forward solve that
// changes the Nordsieck array zn, in order, one record each
// [op, payload..., record length]; the records and their payloads are the
// oracle's (oracle/bdf_oracle.cpp, TapeOp)
enum : int {
  TP_INIT = 1,   // zn[0] = y0, zn[1] = h f(y0):            h, y0[N]
  TP_RESCALE,    // zn[j] *= eta^j, j = 1..q:                eta, q
  TP_INCREASE,   // zn[L] = A1 zn[QMAX]; zn[j] += l_j zn[L]:  q, A1, l[0..5]
  TP_DECREASE,   // zn[j] -= l_j zn[q], j = 2..q-1:          q, l[0..5]
  TP_PREDICT,    // zn[j-1] += zn[j] (Pascal):               q
  TP_RESTORE,    // zn[j-1] -= zn[j] (Pascal):               q
  TP_RESET1,     // zn[1] = h f(zn[0]):                      h, y[N]
  TP_CORRECT,    // zn[j] += l_j acor (+ zn[QMAX] = acor) with
                 // acor = gamma f(zn0 + acor) - rl1 zn1:   q, gamma, rl1,
                 //                                           l[0..5], save, y_n[N]
  TP_DKY         // y = sum_j s^j zn[j]:                     s, q
};

template <int N>
struct LaneCell {
  // ---- the cell ----
  int cell;        // the cell being integrated, -1 when none
  int ph, wait;    // the phase, and the request the lane waits on
  int retval;      // the result carried into the next phase
  int flag;        // the finished cell's flag (PH_DONE)
  double dt;
  double Tfix;
  double xin;      // mass-fraction input: the fractions' input sum
  Params p;
  bool hitT0;
  int restarts;
  long tot[NSTAT];
  // ---- vectors ----
  double zn[L_MAX][N];
  double ewt[N], y[N], acor[N], tempv[N], ftemp[N], delta[N];
  double yreq[N], freq[N];   // the pending rhs request and its result
  int rhs_ret;
  double savedJ[N * N];      // column-major (element (i, j) at i + j N)
  union {                    // the Newton matrix's factors
    double A[N * N];
    float A32[N * N];        // the FP32 form (SolveOpts::lu32)
  };
  int piv[N];
  bool lu64;                 // lu32: factor in FP64 until the next step
  bool fact32;               // the current factors are A32's
  double atol[N];
  // ---- CVodeMem ----
  long st[NSTAT];
  long mxstep, nstloc;
  bool atolmin0;
  double tn, h, hin, hprime, hscale, next_h, hu, eta, etamax, etaq;
  double etaqm1, etaqp1, tolsf, saved_tq5;
  double tau[L_MAX + 1], tq[6], l[L_MAX];
  double rl1, gamma, gammap, gamrat, crate, delp, delnrm, acnrm;
  int q, qprime, next_q, qu, L, qwait;
  long nscon, nstlp, nstlj;
  int convfail;
  bool acnrmcur, jcur, nls_jcur;
  // ---- loop state kept across requests ----
  double tret;
  // cvHin
  int hin_count1, hin_count2, hin_sign;
  double hin_hg, hin_hs, hin_hnew, hin_hlb, hin_hub, hin_hgs;
  // cvStep
  int ncf, nef, nflag;
  double saved_t, dsm;
  // Newton
  bool callSetup, jbad;
  long niters, nconvfails;
  int curiter;
  double tol;
  // ls_setup
  int ls_retval;
  // the adjoint's tape (recording kernels): this cell's region, its
  // capacity and length in doubles (-1: the capacity was exceeded)
  double* tp;
  long tcap, tlen;
  bool qmax_saved;
};

// Code size. Every instruction of the sweep's control code competes with
// the rhs for the instruction cache; these switches keep it compact: the
// control loops rolled (KBL_LOOP, on by default: the primordial3 hydro calls
// run 12% faster than with the loops unrolled), the vector and step helpers
// out of line (KBL_HELPER, KBL_VEC) and the sweep one function (KBL_SWEEP),
// both off by default (the calls cost more than the code they save).
#ifndef KBL_LOOP
#define KBL_LOOP _Pragma("unroll 1")
#endif
// the N-vector helpers' loops unrolled (each helper's loads issue together:
// one memory latency per helper instead of one per element; 3 % on the
// primordial3 hydro calls), the dense LU's loops as the other control loops
// (measured on the B200: the LU unrolled, or restructured to load whole
// columns at a time, ran the hydro calls 5-15 % slower -- its code crowds
// the rhs out of the instruction cache -- and staging the Nordsieck rows of
// the step helpers in registers spilled 15 KB per lane)
#ifndef KBL_VLOOP
#define KBL_VLOOP _Pragma("unroll")
#endif
#ifndef KBL_LULOOP
#define KBL_LULOOP KBL_LOOP
#endif
#ifndef KBL_VEC
#define KBL_VEC __forceinline__
#endif
#ifndef KBL_HELPER
#define KBL_HELPER
#endif
#ifndef KBL_SWEEP
#define KBL_SWEEP
#endif

// ---- vector operations (bdf_cell.hpp:296-400), private arrays ----
template <int N>
__device__ KBL_VEC void axpy_(double a, const double* x, double* y) {
  if (a == 1.0) {
    KBL_VLOOP for (int i = 0; i < N; i++) y[i] += x[i];
  } else if (a == -1.0) {
    KBL_VLOOP for (int i = 0; i < N; i++) y[i] -= x[i];
  } else {
    KBL_VLOOP for (int i = 0; i < N; i++) y[i] += a * x[i];
  }
}
template <int N>
__device__ KBL_VEC void lin_sum_(double a, const double* x, double b,
                                         const double* y, double* z) {
  if (b == 1.0 && z == y) { axpy_<N>(a, x, z); return; }
  if (a == 1.0 && z == x) { axpy_<N>(b, y, z); return; }
  if (a == 1.0 && b == 1.0) {
    KBL_VLOOP for (int i = 0; i < N; i++) z[i] = x[i] + y[i];
    return;
  }
  bool test;
  if ((test = (a == 1.0 && b == -1.0)) || (a == -1.0 && b == 1.0)) {
    const double* v1 = test ? y : x;
    const double* v2 = test ? x : y;
    KBL_VLOOP for (int i = 0; i < N; i++) z[i] = v2[i] - v1[i];
    return;
  }
  if ((test = (a == 1.0)) || b == 1.0) {
    const double c = test ? b : a;
    const double* v1 = test ? y : x;
    const double* v2 = test ? x : y;
    KBL_VLOOP for (int i = 0; i < N; i++) z[i] = (c * v1[i]) + v2[i];
    return;
  }
  if ((test = (a == -1.0)) || b == -1.0) {
    const double c = test ? b : a;
    const double* v1 = test ? y : x;
    const double* v2 = test ? x : y;
    KBL_VLOOP for (int i = 0; i < N; i++) z[i] = (c * v1[i]) - v2[i];
    return;
  }
  if (a == b) {
    KBL_VLOOP for (int i = 0; i < N; i++) z[i] = a * (x[i] + y[i]);
    return;
  }
  if (a == -b) {
    KBL_VLOOP for (int i = 0; i < N; i++) z[i] = a * (x[i] - y[i]);
    return;
  }
  KBL_VLOOP for (int i = 0; i < N; i++) z[i] = (a * x[i]) + (b * y[i]);
}
template <int N>
__device__ KBL_VEC void scale_(double c, const double* x, double* z) {
  KBL_VLOOP for (int i = 0; i < N; i++) z[i] = c * x[i];
}
template <int N>
__device__ KBL_VEC double wrms_(const double* x, const double* w) {
  double sum = 0.0;
  KBL_VLOOP for (int i = 0; i < N; i++) {
    const double pv = x[i] * w[i];
    sum += pv * pv;
  }
  return ssqrt_(sum / N);
}

// dense LU with partial pivoting, column-major (bdf_cell.hpp:405-457). R is
// the factors' type: double, or float for the FP32 Newton-matrix form (the
// factorisation's arithmetic in float; the solve's right-hand side and its
// accumulation stay double)
template <int N, class R>
__device__ KBL_HELPER int getrf_(R* a, int* p) {
  KBL_LULOOP for (int k = 0; k < N; k++) {
    R* col_k = a + k * N;
    int l = k;
    KBL_LULOOP for (int i = k + 1; i < N; i++)
      if (fabs(col_k[i]) > fabs(col_k[l])) l = i;
    p[k] = l;
    if (col_k[l] == R(0)) return k + 1;
    if (l != k) {
      KBL_LULOOP for (int i = 0; i < N; i++) {
        R* ci = a + i * N;
        const R t = ci[l];
        ci[l] = ci[k];
        ci[k] = t;
      }
    }
    const R mult = R(1) / col_k[k];
    KBL_LULOOP for (int i = k + 1; i < N; i++) col_k[i] *= mult;
    KBL_LULOOP for (int j = k + 1; j < N; j++) {
      R* col_j = a + j * N;
      const R a_kj = col_j[k];
      if (a_kj != R(0)) {
        KBL_LULOOP for (int i = k + 1; i < N; i++) col_j[i] -= a_kj * col_k[i];
      }
    }
  }
  return 0;
}
template <int N, class R>
__device__ KBL_HELPER void getrs_(const R* a, const int* p, double* b) {
  KBL_LULOOP for (int k = 0; k < N; k++) {
    const int pk = p[k];
    if (pk != k) { const double t = b[k]; b[k] = b[pk]; b[pk] = t; }
  }
  KBL_LULOOP for (int k = 0; k < N - 1; k++) {
    const R* col_k = a + k * N;
    const double bk = b[k];
    KBL_LULOOP for (int i = k + 1; i < N; i++) b[i] -= (double)col_k[i] * bk;
  }
  KBL_LULOOP for (int k = N - 1; k > 0; k--) {
    const R* col_k = a + k * N;
    b[k] /= (double)col_k[k];
    const double bk = b[k];
    KBL_LULOOP for (int i = 0; i < k; i++) b[i] -= (double)col_k[i] * bk;
  }
  b[0] /= (double)a[0];
}

template <int N, bool EVT, bool REC = false>
struct Machine {
  LaneCell<N>& s;
  const SolveOpts& o;
  __device__ Machine(LaneCell<N>& s_, const SolveOpts& o_) : s(s_), o(o_) {}

  // one tape record (REC only): [op, a (na >= 1), b (na == 2), l[] (with_l),
  // v[N] (v non-null), length]; with no tape (tp null) only its length is
  // counted
  __device__ void rec_(int op, int na, double a, double b, bool with_l,
                       const double* v) {
    if constexpr (REC) {
      if (s.tlen < 0) return;
      const long len = 2 + na + (with_l ? L_MAX : 0) + (v != nullptr ? N : 0);
      if (s.tlen + len > s.tcap) {
        s.tlen = -1;
        return;
      }
      if (s.tp == nullptr) {
        s.tlen += len;
        return;
      }
      double* t = s.tp + s.tlen;
      int w = 0;
      t[w++] = op;
      if (na >= 1) t[w++] = a;
      if (na >= 2) t[w++] = b;
      if (with_l) KBL_LOOP for (int i = 0; i < L_MAX; i++) t[w++] = s.l[i];
      if (v != nullptr) KBL_LOOP for (int i = 0; i < N; i++) t[w++] = v[i];
      t[w++] = (double)len;
      s.tlen += len;
    }
  }
  // the accepted step's corrector record
  __device__ void rec_correct_(int q) {
    if constexpr (REC) {
      if (s.tlen < 0) return;
      const long len = 6 + L_MAX + N;
      if (s.tlen + len > s.tcap) {
        s.tlen = -1;
        return;
      }
      if (s.tp == nullptr) {
        s.tlen += len;
        return;
      }
      double* t = s.tp + s.tlen;
      int w = 0;
      t[w++] = TP_CORRECT;
      t[w++] = q;
      t[w++] = s.gamma;
      t[w++] = s.rl1;
      KBL_LOOP for (int i = 0; i < L_MAX; i++) t[w++] = s.l[i];
      t[w++] = s.qmax_saved ? 1.0 : 0.0;
      KBL_LOOP for (int i = 0; i < N; i++) t[w++] = s.y[i];
      t[w++] = (double)len;
      s.tlen += len;
    }
  }

  __device__ KBL_HELPER int ewt_set(const double* ycur, double* w) {
    if (o.rtol_v) {  // per-species rtol: KROME's per-slot weights
      KBL_VLOOP for (int i = 0; i < N; i++) {
        const double rt = i < NSPEC ? o.rtol_sp[i < KB_NSP_TOL ? i : 0] : o.rtol;
        const double d = fma(rt, fabs(ycur[i]), s.atol[i]);
        if (!(d > 0.0)) return -1;
        w[i] = 1.0 / d;
      }
      return 0;
    }
    // (in registers: ycur and w may be the same array)
    double v[N];
    KB_UNROLL for (int i = 0; i < N; i++) v[i] = (o.rtol * fabs(ycur[i])) + s.atol[i];
    if (s.atolmin0) {
      double mn = v[0];
      KB_UNROLL for (int i = 1; i < N; i++) if (v[i] < mn) mn = v[i];
      if (mn <= 0.0) {
        KB_UNROLL for (int i = 0; i < N; i++) w[i] = v[i];
        return -1;
      }
    }
    KB_UNROLL for (int i = 0; i < N; i++) w[i] = 1.0 / v[i];
    return 0;
  }

  __device__ KBL_HELPER void reinit(double t0, const double* y0, double h_init) {
    s.tn = t0;
    KBL_LOOP for (int i = 0; i < N; i++) s.zn[0][i] = y0[i];
    s.q = 1; s.L = 2; s.qwait = s.L;
    s.etamax = ETA_MAX_FS;
    s.qu = 0; s.hu = 0.0; s.tolsf = 1.0;
    KBL_LOOP for (int i = 0; i < NSTAT; ++i) s.st[i] = 0;
    s.nstlp = 0; s.nscon = 0; s.next_h = 0.0; s.next_q = 0;
    s.hin = h_init;
    s.nstlj = 0;
    s.acnrmcur = false; s.nls_jcur = false; s.jcur = false;
    s.lu64 = false; s.fact32 = false;
    s.saved_tq5 = 0.0;
    KBL_LOOP for (int i = 0; i <= L_MAX; i++) s.tau[i] = 0.0;
    s.eta = 1.0;
  }

  __device__ __forceinline__ void request_rhs(const double* yv, int ph) {
    KBL_LOOP for (int i = 0; i < N; i++) s.yreq[i] = yv[i];
    s.ph = ph;
    s.wait = WAIT_RHS;
  }
  // a failed CVode call: to the restart wrapper at the current time
  __device__ __forceinline__ void fail_solve(int retval) {
    s.tret = s.tn;
    s.retval = retval;
    s.ph = PH_SOLVE_END;
  }

  // ---- step helpers (bdf_cell.hpp:825-954, 1386-1500) ----
  __device__ KBL_HELPER void rescale_() {
    rec_(TP_RESCALE, 2, s.eta, s.q, false, nullptr);
    double c = s.eta;
    KBL_LOOP for (int j = 1; j <= s.q; j++) {
      scale_<N>(c, s.zn[j], s.zn[j]);
      c = s.eta * c;
    }
    s.h = s.hscale * s.eta;
    s.next_h = s.h;
    s.hscale = s.h;
    s.nscon = 0;
  }
  __device__ KBL_HELPER void increase_bdf_() {
    KBL_LOOP for (int i = 0; i <= QMAX; i++) s.l[i] = 0.0;
    double alpha1, prod, xiold, alpha0;
    s.l[2] = alpha1 = prod = xiold = 1.0;
    alpha0 = -1.0;
    double hsum = s.hscale;
    if (s.q > 1)
      for (int j = 1; j < s.q; j++) {
        hsum += s.tau[j + 1];
        const double xi = hsum / s.hscale;
        prod *= xi;
        alpha0 -= 1.0 / (j + 1);
        alpha1 += 1.0 / xi;
        KBL_LOOP for (int i = j + 2; i >= 2; i--) s.l[i] = s.l[i] * xiold + s.l[i - 1];
        xiold = xi;
      }
    const double A1 = (-alpha0 - alpha1) / prod;
    scale_<N>(A1, s.zn[QMAX], s.zn[s.L]);
    if (s.q > 1) {
      KBL_LOOP for (int j = 2; j <= s.q; j++) axpy_<N>(s.l[j], s.zn[s.L], s.zn[j]);
    }
    rec_(TP_INCREASE, 2, s.q, A1, true, nullptr);
  }
  __device__ KBL_HELPER void decrease_bdf_() {
    KBL_LOOP for (int i = 0; i <= QMAX; i++) s.l[i] = 0.0;
    s.l[2] = 1.0;
    double hsum = 0.0;
    KBL_LOOP for (int j = 1; j <= s.q - 2; j++) {
      hsum += s.tau[j];
      const double xi = hsum / s.hscale;
      KBL_LOOP for (int i = j + 2; i >= 2; i--) s.l[i] = s.l[i] * xi + s.l[i - 1];
    }
    if (s.q > 2) {
      KBL_LOOP for (int j = 2; j < s.q; j++) axpy_<N>(-s.l[j], s.zn[s.q], s.zn[j]);
      rec_(TP_DECREASE, 1, s.q, 0.0, true, nullptr);
    }
  }
  __device__ KBL_HELPER void adjust_order_(int deltaq) {
    if ((s.q == 2) && (deltaq != 1)) return;
    if (deltaq == 1) increase_bdf_();
    else if (deltaq == -1) decrease_bdf_();
  }
  __device__ KBL_HELPER void predict_() {
    rec_(TP_PREDICT, 1, s.q, 0.0, false, nullptr);
    s.tn += s.h;
    KBL_LOOP for (int k = 1; k <= s.q; k++)
      for (int j = s.q; j >= k; j--) axpy_<N>(1.0, s.zn[j], s.zn[j - 1]);
  }
  __device__ KBL_HELPER void restore_(double saved_t) {
    rec_(TP_RESTORE, 1, s.q, 0.0, false, nullptr);
    s.tn = saved_t;
    KBL_LOOP for (int k = 1; k <= s.q; k++)
      for (int j = s.q; j >= k; j--) axpy_<N>(-1.0, s.zn[j], s.zn[j - 1]);
  }
  __device__ KBL_HELPER void set_() {
    double xi_inv, xistar_inv, alpha0, alpha0_hat;
    s.l[0] = s.l[1] = xi_inv = xistar_inv = 1.0;
    KBL_LOOP for (int i = 2; i <= s.q; i++) s.l[i] = 0.0;
    alpha0 = alpha0_hat = -1.0;
    double hsum = s.h;
    const int q = s.q;
    if (q > 1) {
      KBL_LOOP for (int j = 2; j < q; j++) {
        hsum += s.tau[j - 1];
        xi_inv = s.h / hsum;
        alpha0 -= 1.0 / j;
        KBL_LOOP for (int i = j; i >= 1; i--) s.l[i] += s.l[i - 1] * xi_inv;
      }
      alpha0 -= 1.0 / q;
      xistar_inv = -s.l[1] - alpha0;
      hsum += s.tau[q - 1];
      xi_inv = s.h / hsum;
      alpha0_hat = -s.l[1] - xi_inv;
      KBL_LOOP for (int i = q; i >= 1; i--) s.l[i] += s.l[i - 1] * xistar_inv;
    }
    const double A1 = 1.0 - alpha0_hat + alpha0;
    const double A2 = 1.0 + q * A1;
    s.tq[2] = fabs(A1 / (alpha0 * A2));
    s.tq[5] = fabs(A2 * xistar_inv / (s.l[q] * xi_inv));
    if (s.qwait == 1) {
      if (q > 1) {
        const double C = xistar_inv / s.l[q];
        const double A3 = alpha0 + 1.0 / q;
        const double A4 = alpha0_hat + xi_inv;
        const double Cpinv = (1.0 - A4 + A3) / A3;
        s.tq[1] = fabs(C * Cpinv);
      } else {
        s.tq[1] = 1.0;
      }
      hsum += s.tau[q];
      const double xi2 = s.h / hsum;
      const double A5 = alpha0 - (1.0 / (q + 1));
      const double A6 = alpha0_hat - xi2;
      const double Cppinv = (1.0 - A6 + A5) / A2;
      s.tq[3] = fabs(Cppinv / (xi2 * (q + 2) * A5));
    }
    s.tq[4] = CORTES / s.tq[2];
    s.rl1 = 1.0 / s.l[1];
    s.gamma = s.h * s.rl1;
    if (s.st[ST_NST] == 0) s.gammap = s.gamma;
    s.gamrat = (s.st[ST_NST] > 0) ? s.gamma / s.gammap : 1.0;
  }
  __device__ KBL_HELPER void complete_step_() {
    s.lu64 = false;
    s.st[ST_NST]++;
    s.nscon++;
    s.hu = s.h;
    s.qu = s.q;
    KBL_LOOP for (int i = s.q; i >= 2; i--) s.tau[i] = s.tau[i - 1];
    if ((s.q == 1) && (s.st[ST_NST] > 1)) s.tau[2] = s.tau[1];
    s.tau[1] = s.h;
    KBL_LOOP for (int j = 0; j <= s.q; j++) axpy_<N>(s.l[j], s.acor, s.zn[j]);
    s.qwait--;
    if ((s.qwait == 1) && (s.q != QMAX)) {
      KBL_LOOP for (int i = 0; i < N; i++) s.zn[QMAX][i] = s.acor[i];
      if constexpr (REC) s.qmax_saved = true;
      s.saved_tq5 = s.tq[5];
    }
  }
  __device__ KBL_HELPER void set_eta_() {
    if ((s.eta > ETA_MIN_FX) && (s.eta < ETA_MAX_FX)) {
      s.eta = 1.0;
      s.hprime = s.h;
      return;
    }
    if (s.eta >= ETA_MAX_FX) s.eta = smin_(s.eta, s.etamax);
    else s.eta = smax_(s.eta, ETA_MIN);
    s.hprime = s.h * s.eta;
    if (s.qprime < s.q) s.nscon = 0;
  }
  __device__ KBL_HELPER void prepare_next_step_(double dsm) {
    if (s.etamax == 1.0) {
      s.qwait = s.qwait > 2 ? s.qwait : 2;
      s.qprime = s.q;
      s.hprime = s.h;
      s.eta = 1.0;
      return;
    }
    s.etaq = 1.0 / (pow(BIAS2 * dsm, 1.0 / s.L) + ADDON);
    if (s.qwait != 0) {
      s.eta = s.etaq;
      s.qprime = s.q;
      set_eta_();
      return;
    }
    s.qwait = 2;
    s.etaqm1 = 0.0;
    if (s.q > 1) {
      const double ddn = wrms_<N>(s.zn[s.q], s.ewt) * s.tq[1];
      s.etaqm1 = 1.0 / (pow(BIAS1 * ddn, 1.0 / s.q) + ADDON);
    }
    s.etaqp1 = 0.0;
    if (s.q != QMAX && s.saved_tq5 != 0.0) {
      const double rr = s.h / s.tau[2];
      double prod = 1.0;
      KBL_LOOP for (int i = 1; i <= s.L; i++) prod *= rr;
      const double cquot = (s.tq[5] / s.saved_tq5) * prod;
      lin_sum_<N>(-cquot, s.zn[QMAX], 1.0, s.acor, s.tempv);
      const double dup = wrms_<N>(s.tempv, s.ewt) * s.tq[3];
      s.etaqp1 = 1.0 / (pow(BIAS3 * dup, 1.0 / (s.L + 1)) + ADDON);
    }
    const double etam = smax_(s.etaqm1, smax_(s.etaq, s.etaqp1));
    if ((etam > ETA_MIN_FX) && (etam < ETA_MAX_FX)) {
      s.eta = 1.0;
      s.qprime = s.q;
    } else if (etam == s.etaq) {
      s.eta = s.etaq;
      s.qprime = s.q;
    } else if (etam == s.etaqm1) {
      s.eta = s.etaqm1;
      s.qprime = s.q - 1;
    } else {
      s.eta = s.etaqp1;
      s.qprime = s.q + 1;
      KBL_LOOP for (int i = 0; i < N; i++) s.zn[QMAX][i] = s.acor[i];
      if constexpr (REC) s.qmax_saved = true;
    }
    set_eta_();
  }
  __device__ KBL_HELPER void get_dky_(double t, double* dky) {
    const double sv = (t - s.tn) / s.h;
    KBL_LOOP for (int j = s.q; j >= 0; j--) {
      double c = 1.0;
      KBL_LOOP for (int i = 0; i < j; i++) c *= sv;
      if (j == s.q) scale_<N>(c, s.zn[j], dky);
      else axpy_<N>(c, s.zn[j], dky);
    }
  }
  // the charge invariant of a DQ-Jacobian Newton correction
  // (bdf_cell.hpp:1266-1287); the species loops are unrolled so that the
  // charges are constants
  __device__ double inv_dot_(const double* x) const {
    double sum = 0.0;
    KB_UNROLL for (int i = 0; i < NSPEC; i++)
      if (species_charge(i) != 0) sum += species_charge(i) * x[i];
    return sum;
  }
  __device__ void inv_set_(double* x, double target) const {
    const int r = IDX_ELECTRON < 0 ? 0 : IDX_ELECTRON;
    double sum = 0.0, sa = 0.0;
    KB_UNROLL for (int i = 0; i < NSPEC; i++)
      if (i != r && species_charge(i) != 0) {
        sum += species_charge(i) * x[i];
        sa += fabs(species_charge(i) * (s.zn[0][i] + s.acor[i]));
      }
    const double yr = s.zn[0][r] + s.acor[r];
    const double cr = (double)species_charge(r);
    const double xr = (target - sum) / cr;
    if (fabs(cr * yr) >= 1e-6 * sa && yr + xr >= 0.0) x[r] = xr;
  }
  // the Newton matrix after a (re)evaluated or reused J: A = I - gamma J
  // and its LU (the tail of cvLsSetup, bdf_cell.hpp:1097-1130)
  __device__ KBL_HELPER int ls_finish_() {
    const int retval = s.ls_retval;
    if (s.jcur) {
      s.st[ST_NJE]++;
      s.nstlj = s.st[ST_NST];
    }
    if (retval != 0) return retval;
    const double c = -s.gamma;
    s.fact32 = o.lu32 && !s.lu64;
    if (s.fact32) {
      KBL_LOOP for (int j = 0; j < N; j++)
        KB_UNROLL for (int i = 0; i < N; i++) {
          const int k = i + j * N;
          double a = s.savedJ[k] * c;
          if (i == j) a += 1.0;
          s.A32[k] = (float)a;
        }
      return getrf_<N, float>(s.A32, s.piv) > 0 ? LS_LUFACT_FAIL : 0;
    }
    KBL_LOOP for (int j = 0; j < N; j++) {
      KB_UNROLL for (int i = 0; i < N; i++) {
        const int k = i + j * N;
        // the product rounded on its own, as the reference's two passes
        // (A = -gamma J, then the diagonal's + 1) round it
        double v = __dmul_rn(s.savedJ[k], c);
        if (i == j) v += 1.0;
        s.A[k] = v;
      }
    }
    if (o.lu32) s.st[ST_NLU64]++;
    return getrf_<N, double>(s.A, s.piv) > 0 ? LS_LUFACT_FAIL : 0;
  }
  // cvNlsLSetup's bookkeeping around ls_setup (bdf_cell.hpp:1051-1065)
  __device__ int lsetup_done_(int retval) {
    s.st[ST_NSETUPS]++;
    s.nls_jcur = s.jcur;
    s.gamrat = 1.0;
    s.gammap = s.gamma;
    s.crate = 1.0;
    s.delnrm = 0.0;
    s.nstlp = s.st[ST_NST];
    if (retval < 0) return LSETUP_FAIL;
    if (retval > 0) return NLS_CONV_RECVR;
    return SUCCESS;
  }

  // ---- one sweep of the phase handlers ----
  // Each handler acts on the lanes in its phase and may move them on to a
  // later handler; a lane leaves the sweep waiting for an rhs or a
  // Jacobian, in PH_DONE, or (after an early failure of a CVode call,
  // rare) in PH_SOLVE_END, which the next sweep takes up.
  __device__ KBL_SWEEP void sweep() {
    if (s.wait != WAIT_NONE) return;
    // ---- cvNlsResidual's tail (bdf_cell.hpp:1022-1032) ----
    // (a failure of a pass's first residual or of its lsetup ends the
    // Newton solve without the retry, bdf_cell.hpp:972-977)
    if (s.ph == PH_RES_OUTER) {
      const int r = residual_done_();
      if (r != SUCCESS) { s.retval = r; s.ph = PH_NLS_END; }
      else s.ph = s.callSetup ? PH_SETUP : PH_NEWTON;
    }
    if (s.ph == PH_RES_INNER) {
      const int r = residual_done_();
      if (r != SUCCESS) { s.retval = r; s.ph = PH_NLS_AFTER; }
      else s.ph = PH_NEWTON;
    }
    // ---- cvNlsLSetup -> cvLsSetup (bdf_cell.hpp:1051-1096) ----
    if (s.ph == PH_SETUP) {
      if (s.jbad) s.convfail = FAIL_BAD_J;
      const double dgamma = fabs((s.gamma / s.gammap) - 1.0);
      const bool jbad_ls = (s.st[ST_NST] == 0) || (s.st[ST_NST] >= s.nstlj + MSBJ)
          || ((s.convfail == FAIL_BAD_J) && (dgamma < DGMAX_JBAD))
          || (s.convfail == FAIL_OTHER);
      s.ls_retval = 0;
      s.jcur = jbad_ls;
      s.ph = PH_LSFINISH;
      if (jbad_ls) {
        s.wait = WAIT_JAC;  // savedJ and ls_retval come from the warp
        return;
      }
    }
    if (s.ph == PH_LSFINISH) {
      const int r = lsetup_done_(ls_finish_());
      if (r != SUCCESS) { s.retval = r; s.ph = PH_NLS_END; }
      else s.ph = PH_NEWTON;
    }
    // ---- one Newton iteration (bdf_cell.hpp:978-1000) and
    //      cvNlsConvTest (bdf_cell.hpp:1035-1048) ----
    if (s.ph == PH_NEWTON) {
      s.niters++;
      const bool inv = (o.jac == 2) && IDX_ELECTRON >= 0 && KB_NFREEZE == 0;
      const double cg = inv ? inv_dot_(s.delta) : 0.0;
      scale_<N>(-1.0, s.delta, s.delta);
      if (s.fact32) getrs_<N, float>(s.A32, s.piv, s.delta);
      else getrs_<N, double>(s.A, s.piv, s.delta);
      if (s.gamrat != 1.0) scale_<N>(2.0 / (1.0 + s.gamrat), s.delta, s.delta);
      if (inv) inv_set_(s.delta, -cg);
      lin_sum_<N>(1.0, s.acor, 1.0, s.delta, s.acor);
      const int m = s.curiter;
      s.delnrm = wrms_<N>(s.delta, s.ewt);
      if (m > 0) s.crate = smax_(CRDOWN * s.crate, s.delnrm / s.delp);
      const double dcon = s.delnrm * smin_(1.0, s.crate) / s.tol;
      int r;
      if (dcon <= 1.0) {
        s.acnrm = (m == 0) ? s.delnrm : wrms_<N>(s.acor, s.ewt);
        s.acnrmcur = true;
        r = SUCCESS;
      } else if ((m >= 1) && (s.delnrm > RDIV * s.delp)) {
        r = NLS_CONV_RECVR;
      } else {
        s.delp = s.delnrm;
        r = NLS_CONTINUE;
      }
      s.curiter++;
      if (r == SUCCESS) s.nls_jcur = false;
      if (r == NLS_CONTINUE && s.curiter >= NLS_MAXCOR) r = NLS_CONV_RECVR;
      if (r != NLS_CONTINUE) {
        s.retval = r;
        s.ph = PH_NLS_AFTER;
      } else {
        lin_sum_<N>(1.0, s.zn[0], 1.0, s.acor, s.y);
        request_rhs(s.y, PH_RES_INNER);
        return;
      }
    }
    // ---- a failed pass retries once with a fresh Jacobian
    //      (bdf_cell.hpp:1002-1010) ----
    if (s.ph == PH_NLS_AFTER) {
      const int r = s.retval;
      // a Newton failure with FP32 factors: FP64 from the next setup on
      if (r > 0 && s.fact32) s.lu64 = true;
      if (r > 0 && !s.nls_jcur) {
        s.nconvfails++;
        s.callSetup = true;
        s.jbad = true;
        KBL_LOOP for (int i = 0; i < N; i++) s.acor[i] = 0.0;
        s.ph = PH_NLS_OUTER;
      } else {
        s.ph = PH_NLS_END;
      }
    }
    // ---- cvNls' tail (bdf_cell.hpp:1011-1018), cvHandleNFlag
    //      (1315-1337), cvDoErrorTest (1339-1381) ----
    if (s.ph == PH_NLS_END) {
      const int r = s.retval;
      if (r > 0 && s.fact32) s.lu64 = true;
      if (r != SUCCESS) s.nconvfails++;
      s.st[ST_NNI] += s.niters;
      s.st[ST_NNF] += s.nconvfails;
      if (r == SUCCESS) {
        lin_sum_<N>(1.0, s.zn[0], 1.0, s.acor, s.y);
        if (!s.acnrmcur) s.acnrm = wrms_<N>(s.acor, s.ewt);
        s.jcur = false;
      }
      s.nflag = r;
      if (r != SUCCESS) {
        restore_(s.saved_t);
        if (r < 0) {
          fail_solve((r == LSETUP_FAIL || r == LSOLVE_FAIL || r == RHSFUNC_FAIL)
                         ? r : NLS_FAIL);
        } else {
          s.ncf++;
          s.etamax = 1.0;
          if (((fabs(s.h) <= 0.0) || (s.ncf == o.max_conv_fails))
              && (r == NLS_CONV_RECVR || r == RHSFUNC_RECVR)) {
            fail_solve(r == NLS_CONV_RECVR ? CONV_FAILURE : REPTD_RHSFUNC_ERR);
          } else {
            s.eta = smax_(ETA_CF, 0.0 / fabs(s.h));
            s.nflag = PREV_CONV_FAIL;
            rescale_();
            s.ph = PH_ATTEMPT;
          }
        }
      } else {
        const double dsm = s.acnrm * s.tq[2];
        s.dsm = dsm;
        if (dsm <= 1.0) {
          s.ph = PH_STEP_OK;
        } else {
          s.nef++;
          s.st[ST_NETF]++;
          s.nflag = PREV_ERR_FAIL;
          restore_(s.saved_t);
          if ((fabs(s.h) <= 0.0) || (s.nef == o.max_err_fails)) {
            fail_solve(ERR_FAILURE);
          } else {
            s.etamax = 1.0;
            if (s.nef <= MXNEF1) {
              s.eta = 1.0 / (pow(BIAS2 * dsm, 1.0 / s.L) + ADDON);
              s.eta = smax_(ETA_MIN_EF, smax_(s.eta, 0.0 / fabs(s.h)));
              if (s.nef >= SMALL_NEF) s.eta = smin_(s.eta, ETA_MAX_EF);
              rescale_();
              s.ph = PH_ATTEMPT;
            } else if (s.q > 1) {
              s.eta = smax_(ETA_MIN_EF, 0.0 / fabs(s.h));
              adjust_order_(-1);
              s.L = s.q;
              s.q--;
              s.qwait = s.L;
              rescale_();
              s.ph = PH_ATTEMPT;
            } else {
              // order 1: restart the history from y' = f(tn, y)
              s.eta = smax_(ETA_MIN_EF, 0.0 / fabs(s.h));
              s.h *= s.eta;
              s.next_h = s.h;
              s.hscale = s.h;
              s.qwait = LONG_WAIT;
              s.nscon = 0;
              request_rhs(s.zn[0], PH_ERRTEST_RHS);
              return;
            }
          }
        }
      }
    }
    if (s.ph == PH_ERRTEST_RHS) {
      KBL_LOOP for (int i = 0; i < N; i++) s.tempv[i] = s.freq[i];
      s.st[ST_NFE]++;
      if (s.rhs_ret > 0) {
        fail_solve(UNREC_RHSFUNC_ERR);
      } else {
        scale_<N>(s.h, s.tempv, s.zn[1]);
        rec_(TP_RESET1, 1, s.h, 0.0, false, s.zn[0]);
        s.ph = PH_ATTEMPT;
      }
    }
    // ---- the accepted step and CVode's tout test (bdf_cell.hpp:620-636,
    //      1386-1500) ----
    if (s.ph == PH_STEP_OK) {
      if constexpr (REC) s.qmax_saved = false;
      const int q_step = s.q;
      complete_step_();
      prepare_next_step_(s.dsm);
      rec_correct_(q_step);  // y holds zn[0] + acor of the accepted attempt
      s.etamax = (s.st[ST_NST] <= SMALL_NST) ? ETA_MAX_ES : ETA_MAX_GS;
      scale_<N>(s.tq[2], s.acor, s.acor);
      s.nstloc++;
      if ((s.tn - s.dt) * s.h >= 0.0) {
        s.tret = s.dt;
        get_dky_(s.dt, s.y);  // y(tout) into y
        rec_(TP_DKY, 2, (s.dt - s.tn) / s.h, s.q, false, nullptr);
        s.next_q = s.qprime;
        s.next_h = s.hprime;
        s.retval = SUCCESS;
        s.ph = PH_SOLVE_END;
      } else {
        s.ph = PH_STEP;
      }
    }
    // ---- the restart wrapper (bdf_cell.hpp:1536-1546). y holds y(tout)
    //      on success; on failure the last accepted state, which is zn[0]
    //      (also when the failure precedes the first step: zn[0] is then
    //      the state of the last reinit, the reference's untouched
    //      yout) ----
    if (s.ph == PH_SOLVE_END) {
      const int r = s.retval;
      if (r < 0)
        for (int i = 0; i < N; i++) s.y[i] = s.zn[0][i];
      KBL_LOOP for (int i = 0; i < NSTAT; ++i) s.tot[i] += s.st[i];
      const bool restartable = r == ERR_FAILURE || r == CONV_FAILURE
                               || r == REPTD_RHSFUNC_ERR;
      if (r >= 0 || !restartable || s.restarts >= o.max_restarts) {
        s.flag = r >= 0 ? 0 : r;
        s.ph = PH_DONE;
        return;
      }
      ++s.restarts;
      const double hcur = s.next_h;
      reinit(s.tret, s.y, hcur > 0.0 ? 0.1 * hcur : 0.0);
      s.ph = PH_SOLVE;
    }
    // ---- CVode(dt)'s first-call block (bdf_cell.hpp:570-593) ----
    if (s.ph == PH_SOLVE) {
      s.tret = s.tn;
      const double tout = s.dt;
      const double tdist = fabs(tout - s.tn);
      const double tround = UROUND * smax_(fabs(s.tn), fabs(tout));
      if (tdist == 0.0 || tdist < 2.0 * tround) {
        fail_solve(TOO_CLOSE);
        return;
      }
      if (ewt_set(s.zn[0], s.ewt) != 0) {
        fail_solve(ILL_INPUT);
        return;
      }
      request_rhs(s.zn[0], PH_FIRST_RHS);
      return;
    }
    if (s.ph == PH_FIRST_RHS) {
      KBL_LOOP for (int i = 0; i < N; i++) s.zn[1][i] = s.freq[i];
      s.st[ST_NFE]++;
      if (s.rhs_ret > 0) {
        fail_solve(FIRST_RHSFUNC_ERR);
        return;
      }
      s.h = s.hin;
      if (s.h != 0.0 && (s.dt - s.tn) * s.h < 0.0) {
        fail_solve(ILL_INPUT);
        return;
      }
      s.ph = (s.h != 0.0) ? PH_AFTER_HIN : PH_HIN_START;
    }
    // ---- cvHin (bdf_cell.hpp:717-794) ----
    if (s.ph == PH_HIN_START) {
      const double tout = s.dt;
      const double tdiff = tout - s.tn;
      s.hin_sign = (tdiff > 0.0) ? 1 : -1;
      const double tdist = fabs(tdiff);
      const double tround = UROUND * smax_(fabs(s.tn), fabs(tout));
      s.hin_hlb = HLB_FACTOR * tround;
      {  // cvUpperBoundH0
        double* temp1 = s.tempv;
        double* temp2 = s.acor;
        KBL_LOOP for (int i = 0; i < N; i++) temp2[i] = fabs(s.zn[0][i]);
        ewt_set(s.zn[0], temp1);
        KBL_LOOP for (int i = 0; i < N; i++) temp1[i] = 1.0 / temp1[i];
        lin_sum_<N>(HUB_FACTOR, temp2, 1.0, temp1, temp1);
        KBL_LOOP for (int i = 0; i < N; i++) temp2[i] = fabs(s.zn[1][i]);
        KBL_LOOP for (int i = 0; i < N; i++) temp1[i] = temp2[i] / temp1[i];
        double hub_inv = 0.0;
        KBL_LOOP for (int i = 0; i < N; i++)
          if (fabs(temp1[i]) > hub_inv) hub_inv = fabs(temp1[i]);
        double hub = HUB_FACTOR * tdist;
        if (hub * hub_inv > 1.0) hub = 1.0 / hub_inv;
        s.hin_hub = hub;
      }
      s.hin_hg = ssqrt_(s.hin_hlb * s.hin_hub);
      if (s.hin_hub < s.hin_hlb) {
        s.h = s.hin_sign == -1 ? -s.hin_hg : s.hin_hg;
        s.ph = PH_AFTER_HIN;
      } else {
        s.hin_hs = s.hin_hg;
        s.hin_hnew = s.hin_hg;
        s.hin_count1 = 1;
        s.hin_count2 = 1;
        s.ph = PH_HIN_REQ;
      }
    }
    if (s.ph == PH_HIN_RHS) {
      KBL_LOOP for (int i = 0; i < N; i++) s.tempv[i] = s.freq[i];
      s.st[ST_NFE]++;
      bool done = false;
      if (s.rhs_ret == 0) {
        lin_sum_<N>(1.0 / s.hin_hgs, s.tempv, -1.0 / s.hin_hgs, s.zn[1], s.tempv);
        const double yddnrm = wrms_<N>(s.tempv, s.ewt);
        s.hin_hs = s.hin_hg;
        const double hub = s.hin_hub;
        s.hin_hnew = (yddnrm * hub * hub > 2.0) ? ssqrt_(2.0 / yddnrm)
                                                : ssqrt_(s.hin_hg * hub);
        const double hrat = s.hin_hnew / s.hin_hg;
        if (s.hin_count1 == MAX_ITERS || ((hrat > 0.5) && (hrat < 2.0))) {
          done = true;
        } else if ((s.hin_count1 > 1) && (hrat > 2.0)) {
          s.hin_hnew = s.hin_hg;
          done = true;
        } else {
          s.hin_hg = s.hin_hnew;
          s.hin_count1++;
          s.hin_count2 = 1;
          s.ph = PH_HIN_REQ;
        }
      } else {
        s.hin_hg *= 0.2;
        if (++s.hin_count2 <= MAX_ITERS) {
          s.ph = PH_HIN_REQ;
        } else if (s.hin_count1 <= 2) {
          fail_solve(REPTD_RHSFUNC_ERR);
          return;
        } else {
          s.hin_hnew = s.hin_hs;
          done = true;
        }
      }
      if (done) {
        double h0 = H_BIAS * s.hin_hnew;
        if (h0 < s.hin_hlb) h0 = s.hin_hlb;
        if (h0 > s.hin_hub) h0 = s.hin_hub;
        if (s.hin_sign == -1) h0 = -h0;
        s.h = h0;
        s.ph = PH_AFTER_HIN;
      }
    }
    if (s.ph == PH_HIN_REQ) {
      s.hin_hgs = s.hin_hg * s.hin_sign;
      lin_sum_<N>(s.hin_hgs, s.zn[1], 1.0, s.zn[0], s.y);
      request_rhs(s.y, PH_HIN_RHS);
      return;
    }
    if (s.ph == PH_AFTER_HIN) {
      s.hscale = s.h;
      s.hprime = s.h;
      scale_<N>(s.h, s.zn[1], s.zn[1]);
      rec_(TP_INIT, 1, s.h, 0.0, false, s.zn[0]);
      s.nstloc = 0;
      s.ph = PH_STEP;
    }
    // ---- the CVode main loop's top (bdf_cell.hpp:595-619) and cvStep's
    //      prologue (798-805) ----
    if (s.ph == PH_STEP) {
      s.next_h = s.h;
      s.next_q = s.q;
      if (s.st[ST_NST] > 0 && ewt_set(s.zn[0], s.ewt) != 0) {
        fail_solve(ILL_INPUT);
        return;
      }
      if (s.mxstep > 0 && s.nstloc >= s.mxstep) {
        fail_solve(TOO_MUCH_WORK);
        return;
      }
      const double nrm = wrms_<N>(s.zn[0], s.ewt);
      s.tolsf = UROUND * nrm;
      if (s.tolsf > 1.0) {
        s.tolsf *= 2.0;
        fail_solve(TOO_MUCH_ACC);
        return;
      }
      s.tolsf = 1.0;
      s.ncf = 0;
      s.nef = 0;
      s.dsm = 0.0;
      if (s.st[ST_NST] > 0 && s.hprime != s.h) {
        if (s.qprime != s.q) {
          adjust_order_(s.qprime - s.q);
          s.q = s.qprime;
          s.L = s.q + 1;
          s.qwait = s.L;
        }
        rescale_();
      }
      s.saved_t = s.tn;
      s.nflag = FIRST_CALL;
      s.ph = PH_ATTEMPT;
    }
    // ---- an attempt: predict, cvSet, cvNls' set-up
    //      (bdf_cell.hpp:806-808, 958-977) ----
    if (s.ph == PH_ATTEMPT) {
      predict_();
      set_();
      s.convfail = ((s.nflag == FIRST_CALL) || (s.nflag == PREV_ERR_FAIL))
                       ? NO_FAILURES : FAIL_OTHER;
      s.callSetup = (s.nflag == PREV_CONV_FAIL) || (s.nflag == PREV_ERR_FAIL)
                    || (s.st[ST_NST] == 0) || (s.st[ST_NST] >= s.nstlp + MSBP)
                    || (fabs(s.gamrat - 1.0) > DGMAX_LSETUP);
      KBL_LOOP for (int i = 0; i < N; i++) s.acor[i] = 0.0;
      s.tol = s.tq[4];
      s.jbad = false;
      s.niters = 0;
      s.nconvfails = 0;
      s.ph = PH_NLS_OUTER;
    }
    if (s.ph == PH_NLS_OUTER) {
      s.curiter = 0;
      lin_sum_<N>(1.0, s.zn[0], 1.0, s.acor, s.y);
      request_rhs(s.y, PH_RES_OUTER);
    }
  }

  // cvNlsResidual's tail after its rhs (bdf_cell.hpp:1022-1032)
  __device__ KBL_HELPER int residual_done_() {
    KBL_LOOP for (int i = 0; i < N; i++) s.ftemp[i] = s.freq[i];
    s.st[ST_NFE]++;
    if (s.rhs_ret > 0) return RHSFUNC_RECVR;
    lin_sum_<N>(s.rl1, s.zn[1], 1.0, s.acor, s.delta);
    lin_sum_<N>(-s.gamma, s.ftemp, 1.0, s.delta, s.delta);
    return SUCCESS;
  }
};

}  // namespace kbl
