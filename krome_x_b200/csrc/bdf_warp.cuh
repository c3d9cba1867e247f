// Warp-per-cell CVODE BDF integrator for sm_100a.
//
// One warp integrates one cell (NEQ <= 32 equations). The algorithm is the
// reference's per-cell integrator -- CVODE 7.9's fixed-leading-coefficient
// BDF in Nordsieck form with cvHin, step/order selection, the local error
// test, the modified Newton iteration with its convergence test, the
// Jacobian / Newton-matrix reuse heuristics, the gamma-ratio scaling of the
// correction, the dense DQ Jacobian, partial-pivot LU and the interpolated
// output (reference: runtime/core/cvode/bdf_cell.hpp:490-1547) -- with the
// same constants and decisions; the data layout is the warp's:
//
//   * lane i holds component i of every N-vector (zn[0..5], ewt, y, acor,
//     tempv, ftemp, delta) in registers; norms are warp-shuffle reductions;
//     all control flow and every scalar of the integrator is warp-uniform;
//   * the Newton matrix A = I - gamma J and its LU factors are row-per-lane
//     registers (lane i: row i); the pivot search is a shuffle arg-max, the
//     row exchange and the eliminations are shuffles of the pivot row;
//   * the saved Jacobian is a per-warp N x N block of shared memory;
//   * the network's scalar math (rates, rhs, thermal equation) is
//     SIMT-uniform: each lane evaluates it on its own full state vector.
//     One rhs call evaluates the same state on every lane; the Jacobians
//     give every lane a different state (lane j: column j of the
//     difference-quotient Jacobian, or species j of the thermal row), so
//     their N rhs evaluations run in parallel.
//
// The per-cell problem around it (the state layout [n | Tgas], the thermal
// equation, the hybrid analytic Jacobian, the charge invariant of the
// Newton correction, the restart wrapper and the post-solve rules) follows
// runtime/core/solve_cell.hpp:438-1132, 1631-1705, 2094-2203.
//
// Every loop is bounded: steps by max_steps (a negative value, "no limit"
// in the reference, is capped at KB_MAX_STEPS_CAP), the attempts of one
// step by max_err_fails + max_conv_fails, restarts by max_restarts.
#pragma once
#include <cfloat>
#include <cstdint>

#ifndef KB_MAX_STEPS_CAP
#define KB_MAX_STEPS_CAP 100000000L
#endif

namespace kbw {

using namespace kbnet;

constexpr unsigned FULL = 0xffffffffu;

// flags (reference runtime/krome.hpp:95-145)
enum : int {
  SUCCESS = 0, TOO_MUCH_WORK = -1, TOO_MUCH_ACC = -2, ERR_FAILURE = -3,
  CONV_FAILURE = -4, LSETUP_FAIL = -6, LSOLVE_FAIL = -7, RHSFUNC_FAIL = -8,
  FIRST_RHSFUNC_ERR = -9, REPTD_RHSFUNC_ERR = -10, UNREC_RHSFUNC_ERR = -11,
  NLS_FAIL = -16, ILL_INPUT = -22, TOO_CLOSE = -27,
  FLAG_PARAM_UNSET = -105, FLAG_NONPOSITIVE_T = -110,
  FLAG_TAPE_FULL = -120  // the adjoint's tape outgrew its capacity
};
enum : int {
  DO_ERROR_TEST = 2, PREDICT_AGAIN = 3, TRY_AGAIN = 5, FIRST_CALL = 6,
  PREV_CONV_FAIL = 7, PREV_ERR_FAIL = 9, RHSFUNC_RECVR = 10,
  NLS_CONTINUE = 901, NLS_CONV_RECVR = 902, LS_LUFACT_FAIL = 1
};
enum : int { NO_FAILURES = 0, FAIL_BAD_J = 1, FAIL_OTHER = 2 };

constexpr int QMAX = 5, L_MAX = 6;
constexpr double HLB_FACTOR = 100.0, HUB_FACTOR = 0.1, H_BIAS = 0.5;
constexpr int MAX_ITERS = 4;
constexpr double CORTES = 0.1, ETA_MIN_FX = 0.0, ETA_MAX_FX = 1.5,
                 ETA_MAX_FS = 10000.0, ETA_MAX_ES = 10.0, ETA_MAX_GS = 10.0,
                 ETA_MIN = 0.1, ETA_MAX_EF = 0.2, ETA_MIN_EF = 0.1,
                 ETA_CF = 0.25;
constexpr long SMALL_NST = 10;
constexpr int SMALL_NEF = 2;
constexpr double ADDON = 1e-6, BIAS1 = 6.0, BIAS2 = 6.0, BIAS3 = 10.0;
constexpr int LONG_WAIT = 10, MXNEF1 = 3;
constexpr long MSBP = 20, MSBJ = 51;
constexpr double DGMAX_LSETUP = 0.3, DGMAX_JBAD = 0.2, MIN_INC_MULT = 1000.0;
constexpr int NLS_MAXCOR = 3;
constexpr double CRDOWN = 0.3, RDIV = 2.0;
constexpr double UROUND = DBL_EPSILON;

// per-cell counters written by the kernels (the CVODE counters of the
// reference's SolveStats, runtime/krome.hpp:257-268)
enum : int {
  ST_NST, ST_NFE, ST_NFEDQ, ST_NJE, ST_NSETUPS, ST_NNI, ST_NNF, ST_NETF,
  ST_RESTARTS, ST_NLU64, NSTAT
};

// per-species tolerances are carried for networks of up to 64 species
constexpr int KB_NSP_TOL = kbnet::NSPEC <= 64 ? kbnet::NSPEC : 1;

// the options of one solve (the krome_opts keys the hot path reads)
struct SolveOpts {
  int evolve_T;
  int jac;  // resolved: 1 analytic (hybrid), 2 difference quotients
  double rtol, atol_n, atol_T;
  long max_steps;
  int max_err_fails, max_conv_fails, max_restarts;
  int clip_negative;
  int fail_every;  // fault injection: cells c with (c + 1) % fail_every == 0
                   // report TOO_MUCH_WORK without integrating (0: off)
  int lu32;        // the Newton matrix factored in FP32 (lane layout only)
  int conserve;    // post-solve conservation mode (kb_conserve.h), 0 none
  // the species' absolute tolerances (atol_n where the caller set none) and,
  // when some species' relative tolerance differs from rtol (rtol_v = 1),
  // the relative ones (krome_opts_set_atol_species / rtol_species)
  double atol_sp[KB_NSP_TOL];
  double rtol_sp[KB_NSP_TOL];
  int rtol_v;
  // photon bins (krome_opts_set_photo): the bin-averaged cross sections
  // sigma[NPHOTO][ph_B] and the cells' fields Phi[ncell][ph_B] on the
  // device; ph_B = 0: no field
  const double* ph_sigma;
  const double* ph_phi;
  int ph_B;
};

// a cell's photo rates from its photon field, k_r = sum_b sigma_rb Phi_b,
// into its parameters (the field is fixed during the solve)
template <class P>
__device__ __forceinline__ void photo_rates_of_row(P& p, const double* sigma,
                                                   const double* phi, int B) {
  if constexpr (NPHOTO > 0) {
    for (int r = 0; r < NPHOTO; ++r) {
      double acc = 0.0;
      for (int b = 0; b < B; ++b) acc += sigma[(long)r * B + b] * phi[b];
      p.kph[r] = acc;
    }
  } else {
    (void)p; (void)sigma; (void)phi; (void)B;
  }
}
template <class P>
__device__ __forceinline__ void photo_rates_of_cell(P& p, long c,
                                                    const SolveOpts& so) {
  if (so.ph_B > 0) photo_rates_of_row(p, so.ph_sigma, so.ph_phi + c * so.ph_B, so.ph_B);
}

__device__ __forceinline__ double smax_(double a, double b) { return a > b ? a : b; }
__device__ __forceinline__ double smin_(double a, double b) { return a < b ? a : b; }
__device__ __forceinline__ double ssqrt_(double x) { return x <= 0.0 ? 0.0 : sqrt(x); }

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(FULL, v, o));
  return v;
}
__device__ __forceinline__ bool warp_any(bool b) { return __any_sync(FULL, b); }

// the network's rhs of one full state (every lane its own), the
// reference's full_rhs_ (solve_cell.hpp:750-789) with eval_rates_ and the
// thermal row aux_ (rates at state_T_ = clamp(T, Tcmb, 1e9), thermal
// terms at thermal_T_ = clamp(T, 2.73, 1e9)); k: NREA scratch; mrow: the
// per-reaction rate factors exp(m_r) of the adjoint's ln-multipliers, null
// for none
// the network's freeze directives (the reference's freeze_rows_ and the
// frozen rows of jac_cell_, solve_cell.hpp:711-720, 1118-1131): the rows of
// the species a directive holds for these parameters are zero in the rhs
// and in the analytic Jacobian
template <int N>
KB_HD inline void freeze_rows(const Params& p, double (&f)[N]) {
#if KB_NFREEZE > 0
  static_assert(NSPEC <= 64, "frozen-row masks hold 64 species");
  int idx[KB_NFREEZE];
  const int m = frozen_species(p, idx);
  unsigned long long mask = 0;
  for (int q = 0; q < m; ++q) mask |= 1ull << idx[q];
  KB_UNROLL for (int i = 0; i < NSPEC; ++i)
    if ((mask >> i) & 1ull) f[i] = 0.0;
#else
  (void)p; (void)f;
#endif
}
#ifndef KB_LARGE_NETWORK
// the analytic Jacobian's rate-derivative part (jac_dk, then the
// aggregates' coupling U W^T) added to J (element (i, j) at i rs + j cs),
// at the rate temperature T. Out of line: its scratch (U, the perturbed
// state of the difference quotients) would otherwise raise the register
// and stack budget of every kernel that can call it
__device__ __noinline__ void jac_rate_terms(double T, const double* y,
                                            const Params& p, const double* k,
                                            double* J, long rs, long cs) {
  double U[NSPEC * NAGG];
  jac_dk(T, y, p, k, J, U, rs, cs);
  jac_agg_(J, U, rs, cs);
}
#endif

// J's element (i, j) at i rs + j cs
template <int N>
KB_HD inline void freeze_jac_rows(const Params& p, double* J, int rs, int cs) {
#if KB_NFREEZE > 0
  int idx[KB_NFREEZE];
  const int m = frozen_species(p, idx);
  for (int q = 0; q < m; ++q)
    for (int j = 0; j < N; ++j) J[idx[q] * rs + j * cs] = 0.0;
#else
  (void)p; (void)J; (void)rs; (void)cs;
#endif
}

template <int N, bool EVT>
__device__ __forceinline__ void full_rhs(const double (&yf)[N], double (&f)[N],
                                         const Params& p, double Tfix,
                                         double (&k)[NREA + 1],
                                         const double* mrow = nullptr) {
  const double T0 = EVT ? yf[N - 1] : Tfix;
  const double T = fmin(fmax(T0, p.Tcmb), 1e9);
  KB_UNROLL
  for (int i = 0; i <= NREA; ++i) k[i] = 0.0;
  rates_fixed(T, yf, p, k);
  rates_var(T, yf, p, k);
  if (mrow != nullptr) {
    KB_UNROLL
    for (int i = 0; i < NREA; ++i) k[i] *= mrow[i];
  }
  rhs(yf, k, f);
  if (EVT) {
    const double Tth = fmin(fmax(yf[N - 1], 2.73), 1e9);
    f[N - 1] = thermal_dTdt(Tth, yf, k, p);
  }
  freeze_rows(p, f);
}

// the integrator's view of the rhs (rhs_host_, solve_cell.hpp:794-813):
// a trial state with Tgas <= 0 or a non-finite f is recoverable (1)
template <int N, bool EVT>
__device__ __forceinline__ int rhs_check(const double (&yf)[N], double (&f)[N],
                                         const Params& p, double Tfix,
                                         double (&k)[NREA + 1], bool& hitT0) {
  if (EVT && !(yf[N - 1] > 0.0)) {
    hitT0 = true;
    return 1;
  }
  full_rhs<N, EVT>(yf, f, p, Tfix, k);
  bool ok = true;
  KB_UNROLL
  for (int i = 0; i < N; ++i) ok = ok && isfinite(f[i]);
  return ok ? 0 : 1;
}

// lane i's component of a full vector
template <int N>
__device__ __forceinline__ double pick(const double (&v)[N], int lane) {
  double r = 0.0;
  KB_UNROLL
  for (int i = 0; i < N; ++i) r = (i == lane) ? v[i] : r;
  return r;
}
// the full vector from the lane components
template <int N>
__device__ __forceinline__ void gather(double x, double (&v)[N]) {
  KB_UNROLL
  for (int i = 0; i < N; ++i) v[i] = __shfl_sync(FULL, x, i);
}

template <int N, bool EVT>
struct Cell {
  // ---- lane-held vectors (component `lane`) ----
  double zn[L_MAX];
  double ewt, y, acor, tempv, ftemp, delta;
  double arow[N];  // the LU factors of I - gamma J, row `lane`
  int piv;         // lane k: the pivot row of step k
  double atol;     // this component's absolute tolerance
  // ---- per-warp shared memory ----
  double* sJ;      // N x N saved Jacobian, row-major
  double* sv;      // 2 N scratch (Jacobian columns)
  // ---- the problem ----
  Params p;
  double Tfix;
  bool hitT0;
  int lane;
  const SolveOpts* o;
  long mxstep;
  bool atolmin0;
  // ---- CVodeMem (uniform) ----
  long st[NSTAT];
  double tn, h, hin, hprime, hscale, next_h, hu, eta, etamax, etaq;
  double etaqm1, etaqp1, tolsf, saved_tq5;
  double tau[L_MAX + 1], tq[6], l[L_MAX];
  double rl1, gamma, gammap, gamrat, crate, delp, delnrm, acnrm;
  int q, qprime, next_q, qu, L, qwait;
  long nscon, nstlp, nstlj;
  int convfail;
  bool acnrmcur, jcur, nls_jcur;

  __device__ __forceinline__ bool act() const { return lane < N; }

  __device__ __forceinline__ double wrms(double x) const {
    const double pv = act() ? x * ewt : 0.0;
    return ssqrt_(warp_sum(pv * pv) / N);
  }

  // ---- rhs calls (every lane evaluates the same state) ----
  __device__ int rhs_state(double ylane, double& flane) {
    double yf[N], f[N], k[NREA + 1];
    gather<N>(ylane, yf);
    const int r = rhs_check<N, EVT>(yf, f, p, Tfix, k, hitT0);
    flane = pick<N>(f, lane);
    return r;
  }

  __device__ int ewt_set(double ycur, double& w) {
    if (o->rtol_v) {  // per-species rtol: KROME's per-slot weights
      const double rt = lane < NSPEC ? o->rtol_sp[lane < KB_NSP_TOL ? lane : 0]
                                     : o->rtol;
      const double d = act() ? fma(rt, fabs(ycur), atol) : 1.0;
      if (__any_sync(FULL, !(d > 0.0))) return -1;
      w = 1.0 / d;
      return 0;
    }
    double wv = act() ? (o->rtol * fabs(ycur)) + atol : 1.0;
    if (atolmin0) {
      const double mn = -warp_max(act() ? -wv : -1e300);
      if (mn <= 0.0) return -1;
    }
    w = 1.0 / wv;
    return 0;
  }

  __device__ void reinit(double t0, double y0, double h_init) {
    tn = t0;
    zn[0] = y0;
    q = 1; L = 2; qwait = L;
    etamax = ETA_MAX_FS;
    qu = 0; hu = 0.0; tolsf = 1.0;
    for (int i = 0; i < NSTAT; ++i) st[i] = 0;
    nstlp = 0; nscon = 0; next_h = 0.0; next_q = 0;
    hin = h_init;
    nstlj = 0;
    acnrmcur = false; nls_jcur = false; jcur = false;
    saved_tq5 = 0.0;
    for (int i = 0; i <= L_MAX; i++) tau[i] = 0.0;
    eta = 1.0;
  }

  // CVode(tout, CV_NORMAL) (bdf_cell.hpp:566-638)
  __device__ int solve(double tout, double& yout, double& tret) {
    tret = tn;
    {
      const double tdist = fabs(tout - tn);
      const double tround = UROUND * smax_(fabs(tn), fabs(tout));
      if (tdist == 0.0 || tdist < 2.0 * tround) return TOO_CLOSE;
      if (ewt_set(zn[0], ewt) != 0) return ILL_INPUT;
      const int retval = rhs_state(zn[0], zn[1]);
      st[ST_NFE]++;
      if (retval > 0) return FIRST_RHSFUNC_ERR;
      h = hin;
      if (h != 0.0 && (tout - tn) * h < 0.0) return ILL_INPUT;
      if (h == 0.0) {
        const int hflag = hin_(tout);
        if (hflag != SUCCESS) return hflag;
      }
      hscale = h;
      hprime = h;
      zn[1] = h * zn[1];
    }
    long nstloc = 0;
    int istate;
    for (;;) {
      next_h = h;
      next_q = q;
      if (st[ST_NST] > 0 && ewt_set(zn[0], ewt) != 0) {
        istate = ILL_INPUT; tret = tn; yout = zn[0]; break;
      }
      if (mxstep > 0 && nstloc >= mxstep) {
        istate = TOO_MUCH_WORK; tret = tn; yout = zn[0]; break;
      }
      const double nrm = wrms(zn[0]);
      tolsf = UROUND * nrm;
      if (tolsf > 1.0) {
        istate = TOO_MUCH_ACC; tret = tn; yout = zn[0];
        tolsf *= 2.0;
        break;
      }
      tolsf = 1.0;
      const int kflag = step_();
      if (kflag != SUCCESS) {
        istate = kflag; tret = tn; yout = zn[0]; break;
      }
      nstloc++;
      if ((tn - tout) * h >= 0.0) {
        istate = SUCCESS;
        tret = tout;
        get_dky_(tout, yout);
        next_q = qprime;
        next_h = hprime;
        break;
      }
    }
    return istate;
  }

  // cvHin (bdf_cell.hpp:717-794)
  __device__ int hin_(double tout) {
    const double tdiff = tout - tn;
    const int sign = (tdiff > 0.0) ? 1 : -1;
    const double tdist = fabs(tdiff);
    const double tround = UROUND * smax_(fabs(tn), fabs(tout));
    const double hlb = HLB_FACTOR * tround;
    // upper bound: temp1 = 1/ewt, then hub_FACTOR |y0| + temp1, then
    // |y0'| / that; the max norm
    double t1;
    {
      const double t2 = fabs(zn[0]);
      double w;
      ewt_set(zn[0], w);
      t1 = 1.0 / w;
      t1 = (HUB_FACTOR * t2) + t1;  // lin_sum_(HUB, temp2, 1, temp1, temp1)
      const double t2b = fabs(zn[1]);
      t1 = t2b / t1;
    }
    const double hub_inv = warp_max(act() ? fabs(t1) : 0.0);
    double hub = HUB_FACTOR * tdist;
    if (hub * hub_inv > 1.0) hub = 1.0 / hub_inv;
    double hg = ssqrt_(hlb * hub);
    if (hub < hlb) {
      h = sign == -1 ? -hg : hg;
      return SUCCESS;
    }
    double hs = hg, hnew = hg, yddnrm = 0.0;
    for (int count1 = 1; count1 <= MAX_ITERS; count1++) {
      bool hgOK = false;
      for (int count2 = 1; count2 <= MAX_ITERS; count2++) {
        const double hgs = hg * sign;
        // cvYddNorm
        const double yv = (hgs * zn[1]) + zn[0];
        double fv;
        const int retval = rhs_state(yv, fv);
        st[ST_NFE]++;
        if (retval == 0) {
          const double a = 1.0 / hgs, b = -1.0 / hgs;
          const double t = (a == -b) ? a * (fv - zn[1]) : (a * fv) + (b * zn[1]);
          yddnrm = wrms(t);
          hgOK = true;
          break;
        }
        hg *= 0.2;
      }
      if (!hgOK) {
        if (count1 <= 2) return REPTD_RHSFUNC_ERR;
        hnew = hs;
        break;
      }
      hs = hg;
      hnew = (yddnrm * hub * hub > 2.0) ? ssqrt_(2.0 / yddnrm)
                                         : ssqrt_(hg * hub);
      if (count1 == MAX_ITERS) break;
      const double hrat = hnew / hg;
      if ((hrat > 0.5) && (hrat < 2.0)) break;
      if ((count1 > 1) && (hrat > 2.0)) { hnew = hg; break; }
      hg = hnew;
    }
    double h0 = H_BIAS * hnew;
    if (h0 < hlb) h0 = hlb;
    if (h0 > hub) h0 = hub;
    if (sign == -1) h0 = -h0;
    h = h0;
    return SUCCESS;
  }

  // cvStep (bdf_cell.hpp:798-822)
  __device__ int step_() {
    int ncf = 0, nef = 0;
    double dsm = 0.0;
    if (st[ST_NST] > 0 && hprime != h) adjust_params_();
    const double saved_t = tn;
    int nflag = FIRST_CALL;
    for (;;) {
      predict_();
      set_();
      nflag = nls_(nflag);
      const int kflag = handle_nflag_(nflag, saved_t, ncf);
      if (kflag == PREDICT_AGAIN) continue;
      if (kflag != DO_ERROR_TEST) return kflag;
      const int eflag = do_error_test_(nflag, saved_t, nef, dsm);
      if (eflag == TRY_AGAIN) continue;
      if (eflag != SUCCESS) return eflag;
      break;
    }
    complete_step_();
    prepare_next_step_(dsm);
    etamax = (st[ST_NST] <= SMALL_NST) ? ETA_MAX_ES : ETA_MAX_GS;
    acor = tq[2] * acor;
    return SUCCESS;
  }

  __device__ void adjust_params_() {
    if (qprime != q) {
      adjust_order_(qprime - q);
      q = qprime;
      L = q + 1;
      qwait = L;
    }
    rescale_();
  }
  __device__ void adjust_order_(int deltaq) {
    if ((q == 2) && (deltaq != 1)) return;
    if (deltaq == 1) increase_bdf_();
    else if (deltaq == -1) decrease_bdf_();
  }
  __device__ __forceinline__ double znq(int j) const {
    double r = zn[0];
    KB_UNROLL
    for (int i = 1; i < L_MAX; ++i) r = (i == j) ? zn[i] : r;
    return r;
  }
  __device__ __forceinline__ void set_zn(int j, double v) {
    KB_UNROLL
    for (int i = 0; i < L_MAX; ++i) zn[i] = (i == j) ? v : zn[i];
  }
  __device__ __forceinline__ void axpy_zn(int j, double a, double x) {
    // axpy_ special cases (bdf_cell.hpp:296-307)
    KB_UNROLL
    for (int i = 0; i < L_MAX; ++i)
      if (i == j) {
        if (a == 1.0) zn[i] += x;
        else if (a == -1.0) zn[i] -= x;
        else zn[i] += a * x;
      }
  }
  __device__ void increase_bdf_() {
    for (int i = 0; i <= QMAX; i++) l[i] = 0.0;
    double alpha1, prod, xiold, alpha0;
    l[2] = alpha1 = prod = xiold = 1.0;
    alpha0 = -1.0;
    double hsum = hscale;
    if (q > 1)
      for (int j = 1; j < q; j++) {
        hsum += tau[j + 1];
        const double xi = hsum / hscale;
        prod *= xi;
        alpha0 -= 1.0 / (j + 1);
        alpha1 += 1.0 / xi;
        for (int i = j + 2; i >= 2; i--) l[i] = l[i] * xiold + l[i - 1];
        xiold = xi;
      }
    const double A1 = (-alpha0 - alpha1) / prod;
    const double zl = A1 * zn[QMAX];
    set_zn(L, zl);
    if (q > 1)
      for (int j = 2; j <= q; j++) axpy_zn(j, l[j], zl);
  }
  __device__ void decrease_bdf_() {
    for (int i = 0; i <= QMAX; i++) l[i] = 0.0;
    l[2] = 1.0;
    double hsum = 0.0;
    for (int j = 1; j <= q - 2; j++) {
      hsum += tau[j];
      const double xi = hsum / hscale;
      for (int i = j + 2; i >= 2; i--) l[i] = l[i] * xi + l[i - 1];
    }
    if (q > 2) {
      const double zq = znq(q);
      for (int j = 2; j < q; j++) axpy_zn(j, -l[j], zq);
    }
  }
  __device__ void rescale_() {
    double c = eta;
    KB_UNROLL
    for (int j = 1; j < L_MAX; j++)
      if (j <= q) {
        zn[j] = c * zn[j];
        c = eta * c;
      }
    h = hscale * eta;
    next_h = h;
    hscale = h;
    nscon = 0;
  }
  __device__ void predict_() {
    tn += h;
    KB_UNROLL
    for (int k = 1; k < L_MAX; k++)
      KB_UNROLL
      for (int j = L_MAX - 1; j >= 1; j--)
        if (k <= q && j <= q && j >= k) zn[j - 1] += zn[j];
  }
  __device__ void restore_(double saved_t) {
    tn = saved_t;
    KB_UNROLL
    for (int k = 1; k < L_MAX; k++)
      KB_UNROLL
      for (int j = L_MAX - 1; j >= 1; j--)
        if (k <= q && j <= q && j >= k) zn[j - 1] -= zn[j];
  }
  // cvSet, cvSetTqBDF (bdf_cell.hpp:903-954)
  __device__ void set_() {
    double xi_inv, xistar_inv, alpha0, alpha0_hat;
    l[0] = l[1] = xi_inv = xistar_inv = 1.0;
    for (int i = 2; i <= q; i++) l[i] = 0.0;
    alpha0 = alpha0_hat = -1.0;
    double hsum = h;
    if (q > 1) {
      for (int j = 2; j < q; j++) {
        hsum += tau[j - 1];
        xi_inv = h / hsum;
        alpha0 -= 1.0 / j;
        for (int i = j; i >= 1; i--) l[i] += l[i - 1] * xi_inv;
      }
      alpha0 -= 1.0 / q;
      xistar_inv = -l[1] - alpha0;
      hsum += tau[q - 1];
      xi_inv = h / hsum;
      alpha0_hat = -l[1] - xi_inv;
      for (int i = q; i >= 1; i--) l[i] += l[i - 1] * xistar_inv;
    }
    {
      const double A1 = 1.0 - alpha0_hat + alpha0;
      const double A2 = 1.0 + q * A1;
      tq[2] = fabs(A1 / (alpha0 * A2));
      tq[5] = fabs(A2 * xistar_inv / (l[q] * xi_inv));
      if (qwait == 1) {
        if (q > 1) {
          const double C = xistar_inv / l[q];
          const double A3 = alpha0 + 1.0 / q;
          const double A4 = alpha0_hat + xi_inv;
          const double Cpinv = (1.0 - A4 + A3) / A3;
          tq[1] = fabs(C * Cpinv);
        } else {
          tq[1] = 1.0;
        }
        hsum += tau[q];
        const double xi2 = h / hsum;
        const double A5 = alpha0 - (1.0 / (q + 1));
        const double A6 = alpha0_hat - xi2;
        const double Cppinv = (1.0 - A6 + A5) / A2;
        tq[3] = fabs(Cppinv / (xi2 * (q + 2) * A5));
      }
      tq[4] = CORTES / tq[2];
    }
    rl1 = 1.0 / l[1];
    gamma = h * rl1;
    if (st[ST_NST] == 0) gammap = gamma;
    gamrat = (st[ST_NST] > 0) ? gamma / gammap : 1.0;
  }

  // the charge invariant of a DQ-Jacobian Newton correction
  // (bdf_cell.hpp:1266-1287, solve_cell.hpp:1631-1642)
  __device__ __forceinline__ double charge_of_lane() const {
    return (lane < NSPEC) ? (double)species_charge(lane < NSPEC ? lane : 0) : 0.0;
  }
  __device__ void inv_set_(double& x, double target) const {
    const int r = IDX_ELECTRON;
    const double cl = charge_of_lane();
    const bool other = act() && lane < NSPEC && lane != r && cl != 0.0;
    const double s = warp_sum(other ? cl * x : 0.0);
    const double sa = warp_sum(other ? fabs(cl * (zn[0] + acor)) : 0.0);
    const double yr = __shfl_sync(FULL, zn[0] + acor, r);
    const double cr = (double)species_charge(r);
    const double xr = (target - s) / cr;
    if (fabs(cr * yr) >= 1e-6 * sa && yr + xr >= 0.0)
      if (lane == r) x = xr;
  }

  // cvNls + Newton (bdf_cell.hpp:958-1048)
  __device__ int nls_(int nflag) {
    convfail = ((nflag == FIRST_CALL) || (nflag == PREV_ERR_FAIL))
                   ? NO_FAILURES : FAIL_OTHER;
    bool callSetup = (nflag == PREV_CONV_FAIL) || (nflag == PREV_ERR_FAIL)
                     || (st[ST_NST] == 0) || (st[ST_NST] >= nstlp + MSBP)
                     || (fabs(gamrat - 1.0) > DGMAX_LSETUP);
    acor = 0.0;
    const double tol = tq[4];
    bool jbad = false;
    long niters = 0, nconvfails = 0;
    int retval;
    const bool inv = (o->jac == 2) && IDX_ELECTRON >= 0 && KB_NFREEZE == 0;
    for (;;) {
      int curiter = 0;
      retval = residual_();
      if (retval != SUCCESS) break;
      if (callSetup) {
        retval = nls_lsetup_(jbad);
        if (retval != SUCCESS) break;
      }
      for (;;) {
        niters++;
        double cg = 0.0;
        if (inv) {
          const double cl = charge_of_lane();
          cg = warp_sum((act() && lane < NSPEC && cl != 0.0) ? cl * delta : 0.0);
        }
        delta = -1.0 * delta;
        lsolve_(delta);
        if (inv) inv_set_(delta, -cg);
        acor = acor + delta;
        retval = conv_test_(curiter, tol);
        curiter++;
        if (retval == SUCCESS) { nls_jcur = false; break; }
        if (retval != NLS_CONTINUE) break;
        if (curiter >= NLS_MAXCOR) { retval = NLS_CONV_RECVR; break; }
        retval = residual_();
        if (retval != SUCCESS) break;
      }
      if (retval == SUCCESS) break;
      if ((retval > 0) && !nls_jcur) {
        nconvfails++;
        callSetup = true;
        jbad = true;
        acor = 0.0;
        continue;
      }
      break;
    }
    if (retval != SUCCESS) nconvfails++;
    st[ST_NNI] += niters;
    st[ST_NNF] += nconvfails;
    if (retval != SUCCESS) return retval;
    y = zn[0] + acor;
    if (!acnrmcur) acnrm = wrms(acor);
    jcur = false;
    return SUCCESS;
  }
  __device__ int residual_() {
    y = zn[0] + acor;
    const int retval = rhs_state(y, ftemp);
    st[ST_NFE]++;
    if (retval > 0) return RHSFUNC_RECVR;
    // lin_sum_(rl1, zn1, 1, acor, delta): (rl1 zn1) + acor
    delta = (rl1 == 1.0) ? zn[1] + acor : (rl1 * zn[1]) + acor;
    // lin_sum_(-gamma, ftemp, 1, delta, delta): axpy
    const double a = -gamma;
    if (a == 1.0) delta += ftemp;
    else if (a == -1.0) delta -= ftemp;
    else delta += a * ftemp;
    return SUCCESS;
  }
  __device__ int conv_test_(int m, double tol) {
    delnrm = wrms(delta);
    if (m > 0) crate = smax_(CRDOWN * crate, delnrm / delp);
    const double dcon = delnrm * smin_(1.0, crate) / tol;
    if (dcon <= 1.0) {
      acnrm = (m == 0) ? delnrm : wrms(acor);
      acnrmcur = true;
      return SUCCESS;
    }
    if ((m >= 1) && (delnrm > RDIV * delp)) return NLS_CONV_RECVR;
    delp = delnrm;
    return NLS_CONTINUE;
  }
  __device__ int nls_lsetup_(bool jbad) {
    if (jbad) convfail = FAIL_BAD_J;
    const int retval = ls_setup_();
    st[ST_NSETUPS]++;
    nls_jcur = jcur;
    gamrat = 1.0;
    gammap = gamma;
    crate = 1.0;
    delnrm = 0.0;
    nstlp = st[ST_NST];
    if (retval < 0) return LSETUP_FAIL;
    if (retval > 0) return NLS_CONV_RECVR;
    return SUCCESS;
  }

  // ---- the Jacobians (written into sJ, row-major) ----
  // CVODE's dense DQ Jacobian (bdf_cell.hpp:1290-1311): lane j evaluates
  // column j; the first failing column (in column order) fails the setup
  __device__ int dq_jac_() {
    const double srur = ssqrt_(UROUND);
    const double fnorm = wrms(ftemp);
    const double minInc = (fnorm != 0.0)
        ? (MIN_INC_MULT * fabs(h) * UROUND * (double)N * fnorm) : 1.0;
    double yf[N], fy[N], f[N], k[NREA + 1];
    gather<N>(y, yf);
    gather<N>(ftemp, fy);
    const double ewtj = act() ? ewt : 1.0;
    const double yj = pick<N>(yf, lane);
    const double inc = smax_(srur * fabs(yj), minInc / ewtj);
    KB_UNROLL
    for (int i = 0; i < N; ++i) yf[i] = (i == lane) ? yf[i] + inc : yf[i];
    int r = rhs_check<N, EVT>(yf, f, p, Tfix, k, hitT0);
    if (!act()) r = 0;
    const unsigned bad = __ballot_sync(FULL, r != 0);
    const int first_bad = bad ? __ffs(bad) - 1 : N;
    st[ST_NFEDQ] += bad ? first_bad + 1 : N;
    if (act() && lane < first_bad) {
      const double inc_inv = 1.0 / inc;
      KB_UNROLL
      for (int i = 0; i < N; ++i)
        sJ[i * N + lane] = inc_inv * (f[i] - fy[i]);
    }
    __syncwarp();
    return bad ? 1 : 0;
  }

  // JAC_ANALYTIC with Tgas evolved (jac_assemble_, solve_cell.hpp:883-1118):
  // the stoichiometric species block, the Tgas column by central
  // differences of the full rhs, the thermal row by difference quotients
  // with the rates re-evaluated at each perturbed density. Lane j < NSPEC
  // perturbs species j, lane NSPEC evaluates the base state, lanes
  // NSPEC+1 / NSPEC+2 the Tgas column at T + h / T - h: one rhs per lane.
  __device__ int analytic_jac_() {
    double yf[N], f[N], k[NREA + 1];
    gather<N>(y, yf);
    const double T = EVT ? fmin(fmax(yf[N - 1], p.Tcmb), 1e9)
                         : fmin(fmax(Tfix, p.Tcmb), 1e9);
    if (lane == 0) {
      double k0[NREA + 1];
      KB_UNROLL
      for (int i = 0; i <= NREA; ++i) k0[i] = 0.0;
      rates_fixed(T, yf, p, k0);
      rates_var(T, yf, p, k0);
      jac_stoich(yf, k0, sJ, N, 1);
#ifndef KB_LARGE_NETWORK
      if constexpr (KB_RATE_NDEP > 0)  // the rate-derivative terms
        jac_rate_terms(T, yf, p, k0, sJ, N, 1);
#endif
    }
    if (!EVT) {
      __syncwarp();
      return 0;
    }
    constexpr int iT = N - 1;
    double sumabs = 0.0;
    KB_UNROLL
    for (int i = 0; i < NSPEC; ++i) sumabs += fabs(yf[i]);
    const double hT = fmax(1e-6 * fabs(yf[iT]), 1e-8);
    double hj = 0.0;
    // this lane's state
    const double yjl = pick<N>(yf, lane);
    if (lane < NSPEC) hj = fmax(fmax(1e-7 * fabs(yjl), 1e-9 * sumabs), 1e-30);
    KB_UNROLL
    for (int i = 0; i < N; ++i) {
      double v = yf[i];
      if (lane < NSPEC && i == lane) v = yf[i] + hj;
      if (lane == NSPEC + 1 && i == iT) v = yf[iT] + hT;
      if (lane == NSPEC + 2 && i == iT) v = yf[iT] - hT;
      yf[i] = v;
    }
    // species lanes keep the rate temperature of the base state: their
    // perturbation does not move Tgas, so state_T is T
    const double Tl = (lane == NSPEC + 1 || lane == NSPEC + 2)
                          ? fmin(fmax(yf[iT], p.Tcmb), 1e9) : T;
    KB_UNROLL
    for (int i = 0; i <= NREA; ++i) k[i] = 0.0;
    rates_fixed(Tl, yf, p, k);
    rates_var(Tl, yf, p, k);
    rhs(yf, k, f);
    const double Tth = fmin(fmax(yf[iT], 2.73), 1e9);
    f[iT] = thermal_dTdt(Tth, yf, k, p);
    // Tgas column: lanes NSPEC+1/+2 hold f(T+h), f(T-h)
    if (lane == NSPEC + 1) {
      KB_UNROLL
      for (int i = 0; i < N; ++i) sv[i] = f[i];
    }
    if (lane == NSPEC + 2) {
      KB_UNROLL
      for (int i = 0; i < N; ++i) sv[N + i] = f[i];
    }
    __syncwarp();
    if (act()) sJ[lane * N + iT] = (sv[lane] - sv[N + lane]) / (2.0 * hT);
    // thermal row: (aux(y + h e_j) - aux(y)) / h
    const double f0 = __shfl_sync(FULL, f[iT], NSPEC);
    if (lane < NSPEC) sJ[iT * N + lane] = (f[iT] - f0) / hj;
    __syncwarp();
    return 0;
  }

  // cvLsSetup (bdf_cell.hpp:1069-1130): J reused or re-evaluated, then
  // A = I - gamma J and its LU factorization
  __device__ int ls_setup_() {
    const double dgamma = fabs((gamma / gammap) - 1.0);
    const bool jbad_ls = (st[ST_NST] == 0) || (st[ST_NST] >= nstlj + MSBJ)
                         || ((convfail == FAIL_BAD_J) && (dgamma < DGMAX_JBAD))
                         || (convfail == FAIL_OTHER);
    int retval = 0;
    if (!jbad_ls) {
      jcur = false;
    } else {
      jcur = true;
      if (o->jac != 2) {
        for (int k = lane; k < N * N; k += 32) sJ[k] = 0.0;
        __syncwarp();
      }
      const int jr = (o->jac == 2) ? dq_jac_() : analytic_jac_();
      if (o->jac != 2) {  // the frozen species' rows of the analytic J
        if (lane == 0) freeze_jac_rows<N>(p, sJ, N, 1);
        __syncwarp();
      }
      if (jr > 0) retval = 1;
    }
    if (retval == 0) {
      const double c = -gamma;
      KB_UNROLL
      for (int j = 0; j < N; ++j) {
        const double a = act() ? sJ[lane * N + j] * c : 0.0;
        arow[j] = (j == lane) ? a + 1.0 : a;
      }
    }
    if (jcur) {
      st[ST_NJE]++;
      nstlj = st[ST_NST];
    }
    if (retval != 0) return retval;
    return getrf_() > 0 ? LS_LUFACT_FAIL : 0;
  }

  // partial-pivot LU, row `lane` in arow (bdf_cell.hpp:405-433): pivot =
  // the largest |a_ik|, i >= k, the first one on ties
  __device__ int getrf_() {
    KB_UNROLL
    for (int k = 0; k < N; ++k) {
      double v = (act() && lane >= k) ? fabs(arow[k]) : -1.0;
      int ix = lane;
      KB_UNROLL
      for (int off = 16; off > 0; off >>= 1) {
        const double ov = __shfl_xor_sync(FULL, v, off);
        const int oi = __shfl_xor_sync(FULL, ix, off);
        if (ov > v || (ov == v && oi < ix)) { v = ov; ix = oi; }
      }
      const int lp = __shfl_sync(FULL, ix, 0);
      if (lane == k) piv = lp;
      const double pv = __shfl_sync(FULL, arow[k], lp);
      if (pv == 0.0) return k + 1;
      if (lp != k) {
        const int src = (lane == k) ? lp : (lane == lp ? k : lane);
        KB_UNROLL
        for (int j = 0; j < N; ++j) arow[j] = __shfl_sync(FULL, arow[j], src);
      }
      const double mult = 1.0 / pv;
      if (lane > k) arow[k] *= mult;
      KB_UNROLL
      for (int j = k + 1; j < N; ++j) {
        const double a_kj = __shfl_sync(FULL, arow[j], k);
        if (a_kj != 0.0 && lane > k) arow[j] -= a_kj * arow[k];
      }
    }
    return 0;
  }
  // x = A^-1 b with the factors (bdf_cell.hpp:435-457), b lane-held
  __device__ void getrs_(double& b) const {
    KB_UNROLL
    for (int k = 0; k < N; ++k) {
      const int pk = __shfl_sync(FULL, piv, k);
      if (pk != k) {
        const double bk = __shfl_sync(FULL, b, k);
        const double bp = __shfl_sync(FULL, b, pk);
        if (lane == k) b = bp;
        if (lane == pk) b = bk;
      }
    }
    KB_UNROLL
    for (int k = 0; k < N - 1; ++k) {
      const double bk = __shfl_sync(FULL, b, k);
      if (lane > k) b -= arow[k] * bk;
    }
    KB_UNROLL
    for (int k = N - 1; k > 0; --k) {
      if (lane == k) b /= arow[k];
      const double bk = __shfl_sync(FULL, b, k);
      if (lane < k) b -= arow[k] * bk;
    }
    if (lane == 0) b /= arow[0];
  }
  __device__ void lsolve_(double& b) const {
    getrs_(b);
    if (gamrat != 1.0) b = (2.0 / (1.0 + gamrat)) * b;
  }

  // cvHandleNFlag, cvDoErrorTest (bdf_cell.hpp:1315-1381)
  __device__ int handle_nflag_(int& nflag_io, double saved_t, int& ncf) {
    const int nflag = nflag_io;
    if (nflag == SUCCESS) return DO_ERROR_TEST;
    st[ST_NNF] += 0;
    ncfn_++;
    restore_(saved_t);
    if (nflag < 0) {
      if (nflag == LSETUP_FAIL) return LSETUP_FAIL;
      if (nflag == LSOLVE_FAIL) return LSOLVE_FAIL;
      if (nflag == RHSFUNC_FAIL) return RHSFUNC_FAIL;
      return NLS_FAIL;
    }
    ncf++;
    etamax = 1.0;
    if ((fabs(h) <= 0.0) || (ncf == o->max_conv_fails)) {
      if (nflag == NLS_CONV_RECVR) return CONV_FAILURE;
      if (nflag == RHSFUNC_RECVR) return REPTD_RHSFUNC_ERR;
    }
    eta = smax_(ETA_CF, 0.0 / fabs(h));
    nflag_io = PREV_CONV_FAIL;
    rescale_();
    return PREDICT_AGAIN;
  }
  long ncfn_;
  __device__ int do_error_test_(int& nflag_io, double saved_t, int& nef,
                                double& dsm_out) {
    const double dsm = acnrm * tq[2];
    dsm_out = dsm;
    if (dsm <= 1.0) return SUCCESS;
    nef++;
    st[ST_NETF]++;
    nflag_io = PREV_ERR_FAIL;
    restore_(saved_t);
    if ((fabs(h) <= 0.0) || (nef == o->max_err_fails)) return ERR_FAILURE;
    etamax = 1.0;
    if (nef <= MXNEF1) {
      eta = 1.0 / (pow(BIAS2 * dsm, 1.0 / L) + ADDON);
      eta = smax_(ETA_MIN_EF, smax_(eta, 0.0 / fabs(h)));
      if (nef >= SMALL_NEF) eta = smin_(eta, ETA_MAX_EF);
      rescale_();
      return TRY_AGAIN;
    }
    if (q > 1) {
      eta = smax_(ETA_MIN_EF, 0.0 / fabs(h));
      adjust_order_(-1);
      L = q;
      q--;
      qwait = L;
      rescale_();
      return TRY_AGAIN;
    }
    eta = smax_(ETA_MIN_EF, 0.0 / fabs(h));
    h *= eta;
    next_h = h;
    hscale = h;
    qwait = LONG_WAIT;
    nscon = 0;
    const int retval = rhs_state(zn[0], tempv);
    st[ST_NFE]++;
    if (retval > 0) return UNREC_RHSFUNC_ERR;
    zn[1] = h * tempv;
    return TRY_AGAIN;
  }
  // cvCompleteStep, cvPrepareNextStep and friends (bdf_cell.hpp:1386-1488)
  __device__ void complete_step_() {
    st[ST_NST]++;
    nscon++;
    hu = h;
    qu = q;
    for (int i = q; i >= 2; i--) tau[i] = tau[i - 1];
    if ((q == 1) && (st[ST_NST] > 1)) tau[2] = tau[1];
    tau[1] = h;
    KB_UNROLL
    for (int j = 0; j < L_MAX; j++)
      if (j <= q) {
        const double a = l[j];
        if (a == 1.0) zn[j] += acor;
        else if (a == -1.0) zn[j] -= acor;
        else zn[j] += a * acor;
      }
    qwait--;
    if ((qwait == 1) && (q != QMAX)) {
      zn[QMAX] = acor;
      saved_tq5 = tq[5];
    }
  }
  __device__ void prepare_next_step_(double dsm) {
    if (etamax == 1.0) {
      qwait = qwait > 2 ? qwait : 2;
      qprime = q;
      hprime = h;
      eta = 1.0;
      return;
    }
    etaq = 1.0 / (pow(BIAS2 * dsm, 1.0 / L) + ADDON);
    if (qwait != 0) {
      eta = etaq;
      qprime = q;
      set_eta_();
    } else {
      qwait = 2;
      etaqm1 = 0.0;
      if (q > 1) {
        const double ddn = wrms(znq(q)) * tq[1];
        etaqm1 = 1.0 / (pow(BIAS1 * ddn, 1.0 / q) + ADDON);
      }
      etaqp1 = 0.0;
      if (q != QMAX && saved_tq5 != 0.0) {
        double rr = h / tau[2], prod = 1.0;
        for (int i = 1; i <= L; i++) prod *= rr;
        const double cquot = (tq[5] / saved_tq5) * prod;
        const double a = -cquot;
        const double t = (a == -1.0) ? acor - zn[QMAX] : (a * zn[QMAX]) + acor;
        const double dup = wrms(t) * tq[3];
        etaqp1 = 1.0 / (pow(BIAS3 * dup, 1.0 / (L + 1)) + ADDON);
      }
      const double etam = smax_(etaqm1, smax_(etaq, etaqp1));
      if ((etam > ETA_MIN_FX) && (etam < ETA_MAX_FX)) {
        eta = 1.0;
        qprime = q;
      } else if (etam == etaq) {
        eta = etaq;
        qprime = q;
      } else if (etam == etaqm1) {
        eta = etaqm1;
        qprime = q - 1;
      } else {
        eta = etaqp1;
        qprime = q + 1;
        zn[QMAX] = acor;
      }
      set_eta_();
    }
  }
  __device__ void set_eta_() {
    if ((eta > ETA_MIN_FX) && (eta < ETA_MAX_FX)) {
      eta = 1.0;
      hprime = h;
      return;
    }
    if (eta >= ETA_MAX_FX) {
      eta = smin_(eta, etamax);
    } else {
      eta = smax_(eta, ETA_MIN);
    }
    hprime = h * eta;
    if (qprime < q) nscon = 0;
  }
  // CVodeGetDky(t, 0) (bdf_cell.hpp:1492-1500)
  __device__ void get_dky_(double t, double& dky) const {
    const double s = (t - tn) / h;
    KB_UNROLL
    for (int j = L_MAX - 1; j >= 0; j--) {
      if (j > q) continue;
      double c = 1.0;
      for (int i = 0; i < j; i++) c *= s;
      if (j == q) dky = c * zn[j];
      else if (c == 1.0) dky += zn[j];
      else if (c == -1.0) dky -= zn[j];
      else dky += c * zn[j];
    }
  }
};

// integrate one cell over [0, dt] with the reference's restart wrapper
// (bdf_cell.hpp:1513-1547) and the post-solve rules of solve()
// (solve_cell.hpp:2094-2203). All 32 lanes of the warp call it; n / T are
// the cell's rows (lane i reads and writes species i), st_out the cell's
// counters (or nullptr). Returns the flag (uniform).
template <int N, bool EVT>
__device__ int solve_cell(double* __restrict__ n, double* __restrict__ Tg,
                          const double* __restrict__ prow, double dt,
                          const SolveOpts& so, double* smem, long* st_out,
                          long cell) {
  const int lane = threadIdx.x & 31;
  Cell<N, EVT> c;
  c.lane = lane;
  c.o = &so;
  c.sJ = smem;
  c.sv = smem + N * N;
  c.hitT0 = false;
  c.ncfn_ = 0;
  params_from_row(prow, c.p);
  if (params_missing(c.p) >= 0) return FLAG_PARAM_UNSET;
  photo_rates_of_cell(c.p, cell, so);
  const double T0 = *Tg;
  c.Tfix = T0;
  double y0 = 0.0;
  if (lane < NSPEC) y0 = n[lane];
  if (EVT && lane == N - 1) y0 = T0;
  c.atol = (lane < NSPEC) ? so.atol_sp[lane < KB_NSP_TOL ? lane : 0] : so.atol_T;
  c.mxstep = so.max_steps == 0 ? 500
             : (so.max_steps < 0 ? KB_MAX_STEPS_CAP : so.max_steps);
  c.atolmin0 = -warp_max(lane < N ? -c.atol : -1e300) == 0.0;
  long tot[NSTAT];
  for (int i = 0; i < NSTAT; ++i) tot[i] = 0;
  double yv = y0;
  c.reinit(0.0, yv, 0.0);
  double t = 0.0;
  int restarts = 0, flag;
  for (;;) {
    const int f = c.solve(dt, yv, t);
    for (int i = 0; i < NSTAT; ++i) tot[i] += c.st[i];
    if (f >= 0) { flag = 0; break; }
    const bool restartable = f == ERR_FAILURE || f == CONV_FAILURE
                             || f == REPTD_RHSFUNC_ERR;
    if (!restartable || restarts >= so.max_restarts) { flag = f; break; }
    ++restarts;
    const double hcur = c.next_h;
    c.reinit(t, yv, hcur > 0.0 ? 0.1 * hcur : 0.0);
  }
  tot[ST_RESTARTS] = restarts;
  if (st_out != nullptr && lane < NSTAT) {
    long v = 0;
    for (int i = 0; i < NSTAT; ++i) v = (i == lane) ? tot[i] : v;
    st_out[lane] = v;
  }
  const double Tend = __shfl_sync(FULL, yv, N - 1);
  if (flag == 0 && EVT && !(Tend > 0.0 && isfinite(Tend)))
    flag = FLAG_NONPOSITIVE_T;
  const bool hit = __any_sync(FULL, c.hitT0);
  if (hit && (flag == REPTD_RHSFUNC_ERR || flag == RHSFUNC_FAIL
              || flag == UNREC_RHSFUNC_ERR || flag == FIRST_RHSFUNC_ERR))
    flag = FLAG_NONPOSITIVE_T;
  if (flag == 0) {
    double v = lane < NSPEC ? yv : 0.0;
    if (so.clip_negative && v < 0.0) v = 0.0;
    if (so.conserve > 0) {  // lane 0 conserves the cell against its input
      const double v0 = lane < NSPEC ? n[lane] : 0.0;
      double cn[NSPEC], c0[NSPEC];
      KB_UNROLL for (int i = 0; i < NSPEC; ++i) {
        cn[i] = __shfl_sync(FULL, v, i);
        c0[i] = __shfl_sync(FULL, v0, i);
      }
      if (lane == 0) kbnet::conserve_cell(c0, cn, so.conserve, c.p);
      KB_UNROLL for (int i = 0; i < NSPEC; ++i) {
        const double ci = __shfl_sync(FULL, cn[i], 0);
        if (lane == i) v = ci;
      }
    }
    if (lane < NSPEC) n[lane] = v;
    if (EVT && lane == 0) *Tg = Tend;
  }
  return flag;
}

}  // namespace kbw
