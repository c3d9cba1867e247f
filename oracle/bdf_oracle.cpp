// CPU ORACLE -- test infrastructure only (the checker, never the product).
//
// A serial restatement, in plain C++, of the reference's per-cell stiff
// solve: the CVODE 7.9 BDF port (reference runtime/core/cvode/
// bdf_cell.hpp) driven by the per-cell problem of runtime/core/
// solve_cell.hpp (state layout, rhs with the thermal equation, the JAC_FD
// and hybrid JAC_ANALYTIC Jacobians, the restart wrapper, the post-solve
// rules) and the batch rules of runtime/core/solve_cells.hpp. The network
// math comes from the generated header selected by KB_NET_HEADER (the same
// scalar form the GPU kernels compile). Every function keeps the
// reference's operation order, so on the same inputs this file reproduces
// the reference's strict build (oracle/_ref/libkrome_<net>_strict.so) bit
// for bit; tests/test_oracle_pin.py checks exactly that.
//
// Built by oracle/build.py into oracle/_build/liboracle_<net>.so; only
// tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load it.
#include <cfloat>
#include <cmath>
#include <cstring>
#include <vector>
#include KB_NET_HEADER
#include "krome_x_b200/csrc/kb_photo.h"
#ifndef KB_NFREEZE
#define KB_NFREEZE 0  // a network header from before freeze directives
#endif

using namespace kbnet;

namespace {

// ---- flags (reference runtime/krome.hpp:95-145, bdf_cell.hpp:108-123) ----
enum : int {
  SUCCESS = 0, TOO_MUCH_WORK = -1, TOO_MUCH_ACC = -2, ERR_FAILURE = -3,
  CONV_FAILURE = -4, LSETUP_FAIL = -6, LSOLVE_FAIL = -7, RHSFUNC_FAIL = -8,
  FIRST_RHSFUNC_ERR = -9, REPTD_RHSFUNC_ERR = -10, UNREC_RHSFUNC_ERR = -11,
  NLS_FAIL = -16, ILL_INPUT = -22, TOO_CLOSE = -27,
  FLAG_PARAM_UNSET = -105, FLAG_NONPOSITIVE_T = -110
};
// internal flags (bdf_cell.hpp:227-239)
enum : int {
  DO_ERROR_TEST = 2, PREDICT_AGAIN = 3, TRY_AGAIN = 5, FIRST_CALL = 6,
  PREV_CONV_FAIL = 7, PREV_ERR_FAIL = 9, RHSFUNC_RECVR = 10,
  NLS_CONTINUE = 901, NLS_CONV_RECVR = 902, LS_LUFACT_FAIL = 1
};
enum : int { NO_FAILURES = 0, FAIL_BAD_J = 1, FAIL_OTHER = 2 };

// CVODE constants (bdf_cell.hpp:242-272)
constexpr int QMAX = 5, L_MAX = 6;
constexpr double HLB_FACTOR = 100.0, HUB_FACTOR = 0.1, H_BIAS = 0.5;
constexpr int MAX_ITERS = 4;
constexpr double CORTES = 0.1, ETA_MIN_FX = 0.0, ETA_MAX_FX = 1.5,
                 ETA_MAX_FS = 10000.0, ETA_MAX_ES = 10.0, ETA_MAX_GS = 10.0,
                 ETA_MIN = 0.1, ETA_MAX_EF = 0.2, ETA_MIN_EF = 0.1,
                 ETA_CF = 0.25;
constexpr long SMALL_NST = 10;
constexpr int SMALL_NEF = 2;
constexpr double ONEPSM = 1.000001, ADDON = 1e-6, BIAS1 = 6.0, BIAS2 = 6.0,
                 BIAS3 = 10.0;
constexpr int LONG_WAIT = 10, MXNEF1 = 3;
constexpr long MSBP = 20, MSBJ = 51;
constexpr double DGMAX_LSETUP = 0.3, DGMAX_JBAD = 0.2, MIN_INC_MULT = 1000.0;
constexpr int NLS_MAXCOR = 3;
constexpr double CRDOWN = 0.3, RDIV = 2.0;
constexpr double UROUND = DBL_EPSILON;

inline double smax_(double a, double b) { return a > b ? a : b; }
inline double smin_(double a, double b) { return a < b ? a : b; }
inline double ssqrt_(double x) { return x <= 0.0 ? 0.0 : std::sqrt(x); }
inline double spowi_(double base, int e) {
  double prod = 1.0;
  const int ex = e < 0 ? -e : e;
  for (int i = 1; i <= ex; i++) prod *= base;
  if (e < 0) prod = 1.0 / prod;
  return prod;
}

// ---- serial N_Vector operations with N_VLinearSum's special cases -------
// (bdf_cell.hpp:296-400)
void axpy_(int N, double a, const double* x, double* y) {
  if (a == 1.0) { for (int i = 0; i < N; i++) y[i] += x[i]; return; }
  if (a == -1.0) { for (int i = 0; i < N; i++) y[i] -= x[i]; return; }
  for (int i = 0; i < N; i++) y[i] += a * x[i];
}
void lin_sum_(int N, double a, const double* x, double b, const double* y,
              double* z) {
  if (b == 1.0 && z == y) { axpy_(N, a, x, z); return; }
  if (a == 1.0 && z == x) { axpy_(N, b, y, z); return; }
  if (a == 1.0 && b == 1.0) {
    for (int i = 0; i < N; i++) z[i] = x[i] + y[i];
    return;
  }
  bool test;
  if ((test = (a == 1.0 && b == -1.0)) || (a == -1.0 && b == 1.0)) {
    const double* v1 = test ? y : x;
    const double* v2 = test ? x : y;
    for (int i = 0; i < N; i++) z[i] = v2[i] - v1[i];
    return;
  }
  if ((test = (a == 1.0)) || b == 1.0) {
    const double c = test ? b : a;
    const double* v1 = test ? y : x;
    const double* v2 = test ? x : y;
    for (int i = 0; i < N; i++) z[i] = (c * v1[i]) + v2[i];
    return;
  }
  if ((test = (a == -1.0)) || b == -1.0) {
    const double c = test ? b : a;
    const double* v1 = test ? y : x;
    const double* v2 = test ? x : y;
    for (int i = 0; i < N; i++) z[i] = (c * v1[i]) - v2[i];
    return;
  }
  if (a == b) { for (int i = 0; i < N; i++) z[i] = a * (x[i] + y[i]); return; }
  if (a == -b) { for (int i = 0; i < N; i++) z[i] = a * (x[i] - y[i]); return; }
  for (int i = 0; i < N; i++) z[i] = (a * x[i]) + (b * y[i]);
}
void scale_(int N, double c, const double* x, double* z) {
  for (int i = 0; i < N; i++) z[i] = c * x[i];
}
double wrms_(int N, const double* x, const double* w) {
  double sum = 0.0;
  for (int i = 0; i < N; i++) {
    const double p = x[i] * w[i];
    sum += p * p;
  }
  return ssqrt_(sum / N);
}
double max_norm_(int N, const double* x) {
  double mx = 0.0;
  for (int i = 0; i < N; i++)
    if (std::fabs(x[i]) > mx) mx = std::fabs(x[i]);
  return mx;
}

// dense LU with partial pivoting, column-major (bdf_cell.hpp:405-457). R is
// the factors' type: double, or float for the FP32 Newton-matrix form (the
// factorisation's arithmetic in float; the solve's right-hand side and its
// accumulation stay double)
template <class R>
int getrf_(R* a, int n, int* p) {
  for (int k = 0; k < n; k++) {
    R* col_k = a + (long)k * n;
    int l = k;
    for (int i = k + 1; i < n; i++)
      if (std::fabs(col_k[i]) > std::fabs(col_k[l])) l = i;
    p[k] = l;
    if (col_k[l] == R(0)) return k + 1;
    if (l != k)
      for (int i = 0; i < n; i++) {
        R* ci = a + (long)i * n;
        const R t = ci[l];
        ci[l] = ci[k];
        ci[k] = t;
      }
    const R mult = R(1) / col_k[k];
    for (int i = k + 1; i < n; i++) col_k[i] *= mult;
    for (int j = k + 1; j < n; j++) {
      R* col_j = a + (long)j * n;
      const R a_kj = col_j[k];
      if (a_kj != R(0))
        for (int i = k + 1; i < n; i++) col_j[i] -= a_kj * col_k[i];
    }
  }
  return 0;
}
template <class R>
void getrs_(const R* a, int n, const int* p, double* b) {
  for (int k = 0; k < n; k++) {
    const int pk = p[k];
    if (pk != k) { const double t = b[k]; b[k] = b[pk]; b[pk] = t; }
  }
  for (int k = 0; k < n - 1; k++) {
    const R* col_k = a + (long)k * n;
    for (int i = k + 1; i < n; i++) b[i] -= (double)col_k[i] * b[k];
  }
  for (int k = n - 1; k > 0; k--) {
    const R* col_k = a + (long)k * n;
    b[k] /= (double)col_k[k];
    for (int i = 0; i < k; i++) b[i] -= (double)col_k[i] * b[k];
  }
  b[0] /= (double)a[0];
}

#ifdef KB_LARGE_NETWORK
// ---- the static-pivot sparse LU of the large networks ----
// The reference's sparse path (bdf_cell.hpp:1163-1264: a row-form IKJ LU
// over a pattern fixed when the network is generated, static pivots in the
// pattern's order, failure on a zero or non-finite pivot) restated over this
// build's generation-time structure (net_<net>.h: sp_rp / sp_ci / sp_di in
// the elimination order sp_perm). a: the values in the pattern; w: a zeroed
// dense row of N doubles (left zeroed). Returns 0, or the failing row + 1.
int sp_getrf_(double* a, double* w) {
  for (int i = 0; i < NSPEC; i++) {
    const int p0 = sp_rp[i], p1 = sp_rp[i + 1], pd = sp_di[i];
    for (int p = p0; p < p1; p++) w[sp_ci[p]] = a[p];
    for (int p = p0; p < pd; p++) {
      const int k = sp_ci[p];
      const double l = w[k] / a[sp_di[k]];
      w[k] = l;
      for (int q = sp_di[k] + 1; q < sp_rp[k + 1]; q++) w[sp_ci[q]] -= l * a[q];
    }
    const double piv = w[i];
    for (int p = p0; p < p1; p++) {
      a[p] = w[sp_ci[p]];
      w[sp_ci[p]] = 0.0;
    }
    if (piv == 0.0 || !std::isfinite(piv)) return i + 1;
  }
  return 0;
}
// x = A^-1 b with the factors of sp_getrf_ (b in the species order; t: N
// doubles of scratch); x may alias b
void sp_getrs_(const double* a, const double* b, double* t, double* x) {
  for (int i = 0; i < NSPEC; i++) t[i] = b[sp_perm[i]];
  for (int i = 0; i < NSPEC; i++) {
    double s = t[i];
    for (int p = sp_rp[i]; p < sp_di[i]; p++) s -= a[p] * t[sp_ci[p]];
    t[i] = s;
  }
  for (int i = NSPEC - 1; i >= 0; i--) {
    double s = t[i];
    for (int p = sp_di[i] + 1; p < sp_rp[i + 1]; p++) s -= a[p] * t[sp_ci[p]];
    t[i] = s / a[sp_di[i]];
  }
  for (int i = 0; i < NSPEC; i++) x[sp_perm[i]] = t[i];
}
// The Tgas border of an evolved-Tgas solve (bdf_cell.hpp:1192-1219 with
// m = 1, the reference's layout of one border equation): with the species
// factors of sp_getrf_, B' = L^-1 (c B), C' = (c C) U^-1 and the Schur
// complement Z = c D + 1 - C' B' (its 1 x 1 LU: a zero Z fails). B, C:
// the saved Tgas column and row over the species (species order), D the
// saved corner.
struct SpBorder {
  double *B = nullptr, *C = nullptr, D = 0.0;  // saved Jacobian
  double *Bt = nullptr, *Ct = nullptr, Z = 0.0;  // factors (pivot order)
};
int sp_border_factor_(const double* a, double c, SpBorder& br) {
  double* x = br.Bt;
  for (int k = 0; k < NSPEC; k++) x[k] = br.B[sp_perm[k]] * c;
  for (int i = 0; i < NSPEC; i++) {  // x = L^-1 x (unit lower)
    double s = x[i];
    for (int p = sp_rp[i]; p < sp_di[i]; p++) s -= a[p] * x[sp_ci[p]];
    x[i] = s;
  }
  x = br.Ct;  // x U = the row: a forward sweep over U's rows
  for (int k = 0; k < NSPEC; k++) x[k] = br.C[sp_perm[k]] * c;
  for (int k = 0; k < NSPEC; k++) {
    const double xk = x[k] / a[sp_di[k]];
    x[k] = xk;
    if (xk != 0.0)
      for (int q = sp_di[k] + 1; q < sp_rp[k + 1]; q++) x[sp_ci[q]] -= xk * a[q];
  }
  double z = br.D * c;
  z += 1.0;
  for (int k = 0; k < NSPEC; k++) z -= br.Ct[k] * br.Bt[k];
  br.Z = z;
  return z == 0.0 ? 1 : 0;
}
// x = A^-1 b for the bordered matrix (bdf_cell.hpp:1233-1264): b, x of
// NSPEC + 1 entries (Tgas last), may alias; t: NSPEC doubles of scratch
void sp_getrs_border_(const double* a, const SpBorder& br, const double* b,
                      double* t, double* x) {
  for (int i = 0; i < NSPEC; i++) t[i] = b[sp_perm[i]];
  for (int i = 0; i < NSPEC; i++) {
    double s = t[i];
    for (int p = sp_rp[i]; p < sp_di[i]; p++) s -= a[p] * t[sp_ci[p]];
    t[i] = s;
  }
  double v = b[NSPEC];
  for (int k = 0; k < NSPEC; k++) v -= br.Ct[k] * t[k];
  v /= br.Z;
  if (v != 0.0)
    for (int k = 0; k < NSPEC; k++) t[k] -= br.Bt[k] * v;
  for (int i = NSPEC - 1; i >= 0; i--) {
    double s = t[i];
    for (int p = sp_di[i] + 1; p < sp_rp[i + 1]; p++) s -= a[p] * t[sp_ci[p]];
    t[i] = s / a[sp_di[i]];
  }
  for (int i = 0; i < NSPEC; i++) x[sp_perm[i]] = t[i];
  x[NSPEC] = v;
}
#endif

// ---- the per-cell problem (solve_cell.hpp:438-813, 883-1132) ------------
struct Problem {
  Params p;
  double Tfix = 0.0;
  int NEQ = NSPEC;
  int iT = -1;
  bool hit_T0 = false;
  bool kfix_on = false;   // fixed Tgas: rates_fixed once per solve
  double kfix[NREA + 1];
  bool kT_on = false;     // evolved Tgas: rates_fixed cached per Tgas
  bool kT_ok = false;
  double kT_T = 0.0;
  double kT[NREA + 1];
  double k[NREA + 1];
  double k0[NREA + 1], kp[NREA + 1];
  double fm[NSPEC + 1];
  const double* mult = nullptr;  // per-reaction factors exp(m_r) (adjoint)

  double state_T(const double* y) const {
    const double T = iT >= 0 ? y[iT] : Tfix;
    return std::fmin(std::fmax(T, p.Tcmb), 1e9);
  }
  static double thermal_T(double T) { return std::fmin(std::fmax(T, 2.73), 1e9); }

  void eval_rates(double T, const double* y, double* kk) {
    if (kfix_on) {
      for (int i = 0; i < NREA; ++i) kk[i] = kfix[i];
      rates_var(T, y, p, kk);
    } else if (kT_on) {
      if (!kT_ok || T != kT_T) {
        for (int i = 0; i < NREA; ++i) kT[i] = 0.0;
        rates_fixed(T, y, p, kT);
        kT_T = T;
        kT_ok = true;
      }
      for (int i = 0; i < NREA; ++i) kk[i] = kT[i];
      rates_var(T, y, p, kk);
    } else {
      for (int i = 0; i < NREA; ++i) kk[i] = 0.0;
      rates_fixed(T, y, p, kk);
      rates_var(T, y, p, kk);
    }
    if (mult != nullptr)
      for (int i = 0; i < NREA; ++i) kk[i] *= mult[i];
  }
#ifdef KB_LARGE_NETWORK
  // the sparse Jacobian of the species at fixed k (the emitted gather
  // form, entry e at sp_jpos[e] of the LU pattern)
  int jac_sparse_cb(const double* y, double* Jc) {
    eval_rates(state_T(y), y, k0);
    for (int part = 0; part < NPART; ++part) jac_gather_part(part, y, k0, Jc);
    return 0;
  }
  // the Tgas border of the evolved-Tgas Jacobian (jac_assemble_,
  // solve_cell.hpp:1053-1090): the Tgas column by central differences of
  // the full rhs (B over the species, D its Tgas entry), the Tgas row by
  // difference quotients over the densities with the rates re-evaluated (C)
  void jac_border(const double* y, double* B, double* C, double* D,
                  double* yp, double* fp) {
    const int N = NEQ;
    const double T = state_T(y);
    for (int i = 0; i < N; ++i) yp[i] = y[i];
    const double h = std::fmax(1e-6 * std::fabs(y[iT]), 1e-8);
    yp[iT] = y[iT] + h;
    full_rhs(yp, fp);
    yp[iT] = y[iT] - h;
    full_rhs(yp, fm);
    yp[iT] = y[iT];
    for (int i = 0; i < NSPEC; ++i) B[i] = (fp[i] - fm[i]) / (2.0 * h);
    *D = (fp[iT] - fm[iT]) / (2.0 * h);
    eval_rates(T, y, k0);
    const double f0 = aux(y, k0);
    for (int j = 0; j < NSPEC; ++j) {
      const double hj = fd_step_n(y, j);
      yp[j] = y[j] + hj;
      eval_rates(T, yp, kp);
      const double f1 = aux(yp, kp);
      yp[j] = y[j];
      C[j] = (f1 - f0) / hj;
    }
  }
#endif
  // g[r] += sum_i mu_i d f_i / d ln k_r at y (the emitted lnk_vjp)
  void lnk_vjp_at(const double* y, const double* mu, double* g) {
    eval_rates(state_T(y), y, k0);
    const double Tth = thermal_T(iT >= 0 ? y[iT] : Tfix);
    lnk_vjp(y, k0, Tth, p, mu, iT >= 0 ? mu[iT] : 0.0, g);
  }
  double aux(const double* y, const double* kk) {
    const double T = thermal_T(iT >= 0 ? y[iT] : Tfix);
    return thermal_dTdt(T, y, kk, p);
  }
  // the species a freeze directive holds for this cell (none: 0)
  int frozen(int* idx) const {
#if KB_NFREEZE > 0
    return frozen_species(p, idx);
#else
    (void)idx;
    return 0;
#endif
  }
  void full_rhs(const double* y, double* f) {
    const double T = state_T(y);
    eval_rates(T, y, k);
    rhs(y, k, f);
    if (iT >= 0) f[iT] = aux(y, k);
    // freeze_rows_ (solve_cell.hpp:711-720)
    int idx[KB_NFREEZE > 0 ? KB_NFREEZE : 1];
    const int m = frozen(idx);
    for (int q = 0; q < m; ++q) f[idx[q]] = 0.0;
  }
  // the integrator's view: T <= 0 or a non-finite f is recoverable
  int rhs_cb(const double* y, double* f) {
    if (iT >= 0 && !(y[iT] > 0.0)) { hit_T0 = true; return 1; }
    full_rhs(y, f);
    for (int i = 0; i < NEQ; ++i)
      if (!std::isfinite(f[i])) return 1;
    return 0;
  }
  // fd_step_n_ (solve_cell.hpp:729-733)
  static double fd_step_n(const double* y, int j) {
    double s = 0.0;
    for (int i = 0; i < NSPEC; ++i) s += std::fabs(y[i]);
    return std::fmax(std::fmax(1e-7 * std::fabs(y[j]), 1e-9 * s), 1e-30);
  }
  // JAC_ANALYTIC: stoichiometric block + central-difference Tgas column +
  // difference-quotient thermal row (jac_assemble_, solve_cell.hpp:883-1118);
  // J column-major NEQ x NEQ, zeroed by the caller
  int jac_cb(const double* y, double* J, double* yp, double* fp) {
    jac_assemble(y, J, yp, fp);
    // jac_cell_: the frozen species' rows zeroed (solve_cell.hpp:1118-1131)
    int idx[KB_NFREEZE > 0 ? KB_NFREEZE : 1];
    const int m = frozen(idx);
    for (int q = 0; q < m; ++q)
      for (int j = 0; j < NEQ; ++j) J[idx[q] + (long)j * NEQ] = 0.0;
    return 0;
  }
  int jac_assemble(const double* y, double* J, double* yp, double* fp) {
    const int N = NEQ;
    const double T = state_T(y);
    eval_rates(T, y, k0);
    jac_stoich(y, k0, J, 1, N);
#ifndef KB_LARGE_NETWORK
    if (KB_RATE_NDEP > 0) {  // jacobian_split's rate-derivative part, U W^T
      double U[NSPEC * NAGG];
      jac_dk(T, y, p, k0, J, U, 1, N);
      jac_agg_(J, U, 1, N);
    }
#endif
    if (iT < 0) return 0;
    for (int i = 0; i < N; ++i) yp[i] = y[i];
    {
      const int col = iT;
      const double h = std::fmax(1e-6 * std::fabs(y[col]), 1e-8);
      yp[col] = y[col] + h;
      full_rhs(yp, fp);
      yp[col] = y[col] - h;
      full_rhs(yp, fm);
      yp[col] = y[col];
      for (int i = 0; i < N; ++i)
        J[i + (long)col * N] = (fp[i] - fm[i]) / (2.0 * h);
    }
    eval_rates(T, y, k0);
    const double f0 = aux(y, k0);
    for (int j = 0; j < NSPEC; ++j) {
      const double h = fd_step_n(y, j);
      yp[j] = y[j] + h;
      eval_rates(T, yp, kp);
      const double f1 = aux(yp, kp);
      yp[j] = y[j];
      J[iT + (long)j * N] = (f1 - f0) / h;
    }
    return 0;
  }
};

struct Stats {
  long nst = 0, nfe = 0, nfeDQ = 0, nje = 0, nsetups = 0, nni = 0, nnf = 0,
       ncfn = 0, netf = 0, nlu64 = 0;
  void add(const Stats& s) {
    nst += s.nst; nfe += s.nfe; nfeDQ += s.nfeDQ; nje += s.nje;
    nsetups += s.nsetups; nni += s.nni; nnf += s.nnf; ncfn += s.ncfn;
    netf += s.netf; nlu64 += s.nlu64;
  }
};

struct BdfOpts {
  double rtol = 1e-4;
  const double* atol = nullptr;
  const double* rtol_v = nullptr;  // per-slot rtol (KROME's ewt_cb_), or null
  long max_steps = 500;
  int max_err_fails = 7, max_conv_fails = 10;
  double h0 = 0.0;
  bool dq_jac = false;
  int inv_row = -1, inv_n = 0;
  // the Newton matrix factored in FP32 (residuals, rhs, history and error
  // test stay FP64), refactored in FP64 after a Newton failure until the
  // next accepted step
  bool lu32 = false;
};

// ---- the discrete adjoint's tape ----
// The forward solve records every operation that changes the Nordsieck
// array zn, in order; the step sizes, orders and Newton / error-test
// decisions are the forward's (constants of the discrete map). Each record
// is [op, payload..., record length].
enum TapeOp {
  TP_INIT = 1,   // zn[0] = y0, zn[1] = h f(y0):           h, y0[N]
  TP_RESCALE,    // zn[j] *= eta^j, j = 1..q:               eta, q
  TP_INCREASE,   // zn[L] = A1 zn[QMAX]; zn[j] += l_j zn[L]: q, A1, l[0..5]
  TP_DECREASE,   // zn[j] -= l_j zn[q], j = 2..q-1:         q, l[0..5]
  TP_PREDICT,    // zn[j-1] += zn[j] (Pascal):              q
  TP_RESTORE,    // zn[j-1] -= zn[j] (Pascal):              q
  TP_RESET1,     // zn[1] = h f(zn[0]):                     h, y[N]
  TP_CORRECT,    // zn[j] += l_j acor (+ zn[QMAX] = acor),
                 // acor = gamma f(zn0 + acor) - rl1 zn1:  q, gamma, rl1,
                 //                                          l[0..5], save, y_n[N]
  TP_DKY         // y = sum_j s^j zn[j]:                    s, q
};

// one cell's CVODE BDF (bdf_cell.hpp:490-1501), unit stride, dense LU
class Cvode {
 public:
  Stats st;
  std::vector<double>* tape = nullptr;  // recording for the adjoint
  Cvode(Problem& prob, int n, const BdfOpts& opts)
      : P(prob), N(n), o(opts),
#ifdef KB_LARGE_NETWORK
        work((L_MAX + 10) * n + NNZ_LU + NNZ_J + 4 * NSPEC),
#else
        work((L_MAX + 9) * n + 2 * n * n),
#endif
        A32(opts.lu32 ? (long)n * n : 0), piv(n) {
    double* w = work.data();
    for (int j = 0; j < L_MAX; j++, w += N) zn[j] = w;
    ewt = w; w += N;
    y = w; w += N;
    acor = w; w += N;
    tempv = w; w += N;
    ftemp = w; w += N;
    delta = w; w += N;
    vtemp1 = w; w += N;
    vtemp2 = w; w += N;
    vtemp3 = w; w += N;
#ifdef KB_LARGE_NETWORK
    A = w; w += NNZ_LU;       // the LU values in the sparse pattern
    savedJ = w; w += NNZ_J;   // the Jacobian's entries
    spw = w;                  // the LU's dense work row (kept zeroed)
    for (int i = 0; i < N; i++) spw[i] = 0.0;
    w += N;
    border.B = w; w += NSPEC;  // the Tgas border (evolved Tgas)
    border.C = w; w += NSPEC;
    border.Bt = w; w += NSPEC;
    border.Ct = w;
#else
    A = w; w += (long)N * N;
    savedJ = w;
#endif
    mxstep = o.max_steps == 0 ? 500 : o.max_steps;
    double mn = o.atol[0];
    for (int i = 1; i < N; i++)
      if (o.atol[i] < mn) mn = o.atol[i];
    atolmin0 = mn == 0.0;
  }

  void reinit(double t0, const double* y0, double h_init) {
    tn = t0;
    for (int i = 0; i < N; i++) zn[0][i] = y0[i];
    q = 1; L = 2; qwait = L;
    etamax = ETA_MAX_FS;
    qu = 0; hu = 0.0; tolsf = 1.0;
    st = Stats();
    nstlp = 0; nscon = 0; h0u = 0.0; next_h = 0.0; next_q = 0;
    hin = h_init;
    nstlj = 0;
    acnrmcur = false; nls_jcur = false; jcur = false;
    lu64 = false; fact32 = false;
    saved_tq5 = 0.0;
    for (int i = 0; i <= L_MAX; i++) tau[i] = 0.0;
    eta = 1.0;
  }

  int solve(double tout, double* yout, double* tret) {
    int istate = SUCCESS;
    *tret = tn;
    {
      const double tdist = std::fabs(tout - tn);
      const double tround = UROUND * smax_(std::fabs(tn), std::fabs(tout));
      if (tdist == 0.0 || tdist < 2.0 * tround) return TOO_CLOSE;
      if (ewt_set(zn[0], ewt) != 0) return ILL_INPUT;
      const int retval = P.rhs_cb(zn[0], zn[1]);
      st.nfe++;
      if (retval < 0) return RHSFUNC_FAIL;
      if (retval > 0) return FIRST_RHSFUNC_ERR;
      h = hin;
      if (h != 0.0 && (tout - tn) * h < 0.0) return ILL_INPUT;
      if (h == 0.0) {
        const int hflag = hin_(tout);
        if (hflag != SUCCESS) return hflag;
      }
      // hmax_inv = 0, hmin = 0 (CVODE defaults)
      hscale = h;
      h0u = h;
      hprime = h;
      scale_(N, h, zn[1], zn[1]);
      rec_(TP_INIT, {h}, zn[0]);
    }
    long nstloc = 0;
    for (;;) {
      next_h = h;
      next_q = q;
      if (st.nst > 0 && ewt_set(zn[0], ewt) != 0) {
        istate = ILL_INPUT; *tret = tn; copy_(zn[0], yout); break;
      }
      if (mxstep > 0 && nstloc >= mxstep) {
        istate = TOO_MUCH_WORK; *tret = tn; copy_(zn[0], yout); break;
      }
      const double nrm = wrms_(N, zn[0], ewt);
      tolsf = UROUND * nrm;
      if (tolsf > 1.0) {
        istate = TOO_MUCH_ACC; *tret = tn; copy_(zn[0], yout);
        tolsf *= 2.0;
        break;
      }
      tolsf = 1.0;
      const int kflag = step_();
      if (kflag != SUCCESS) {
        istate = kflag; *tret = tn; copy_(zn[0], yout); break;
      }
      nstloc++;
      if ((tn - tout) * h >= 0.0) {
        istate = SUCCESS;
        *tret = tout;
        get_dky_(tout, yout);
        rec_(TP_DKY, {(tout - tn) / h, (double)q});
        next_q = qprime;
        next_h = hprime;
        break;
      }
    }
    return istate;
  }
  double current_step() const { return next_h; }

 private:
  Problem& P;
  const int N;
  const BdfOpts o;
  std::vector<double> work;
  std::vector<float> A32;  // the FP32 factors (lu32)
  std::vector<int> piv;
  bool lu64 = false;       // lu32: factor in FP64 until the next accepted step
  bool fact32 = false;     // the current factors are A32's
  long mxstep;
  bool atolmin0;
  double* zn[L_MAX];
  double *ewt, *y, *acor, *tempv, *ftemp, *delta, *vtemp1, *vtemp2, *vtemp3;
  double *A, *savedJ;
  double* spw = nullptr;
#ifdef KB_LARGE_NETWORK
  SpBorder border;
#endif
  double tn = 0.0, h = 0.0, hin = 0.0, hprime = 0.0, hscale = 0.0, h0u = 0.0;
  double next_h = 0.0, hu = 0.0, eta = 1.0, etamax = 0.0, etaq = 0.0;
  double etaqm1 = 0.0, etaqp1 = 0.0, tolsf = 1.0, saved_tq5 = 0.0;
  double tau[L_MAX + 1] = {}, tq[6] = {}, l[L_MAX] = {};
  double rl1 = 0.0, gamma = 0.0, gammap = 0.0, gamrat = 0.0;
  double crate = 0.0, delp = 0.0, delnrm = 0.0, acnrm = 0.0;
  int q = 1, qprime = 1, next_q = 0, qu = 0, L = 2, qwait = 2;
  long nscon = 0, nstlp = 0, nstlj = 0;
  int convfail = 0;
  bool acnrmcur = false, jcur = false, nls_jcur = false;

  void copy_(const double* x, double* z) const {
    for (int i = 0; i < N; i++) z[i] = x[i];
  }
  bool qmax_saved = false;
  void rec_(int op, std::initializer_list<double> vals, const double* v = nullptr) {
    if (tape == nullptr) return;
    const size_t start = tape->size();
    tape->push_back(op);
    for (double x : vals) tape->push_back(x);
    if (v != nullptr)
      for (int i = 0; i < N; i++) tape->push_back(v[i]);
    tape->push_back((double)(tape->size() - start + 1));
  }
  void rec_l_(int op, std::initializer_list<double> head) {
    if (tape == nullptr) return;
    const size_t start = tape->size();
    tape->push_back(op);
    for (double x : head) tape->push_back(x);
    for (int i = 0; i < L_MAX; i++) tape->push_back(l[i]);
    tape->push_back((double)(tape->size() - start + 1));
  }
  // cvEwtSetSV, or KROME's per-slot weights with rtol_v (bdf_cell.hpp:
  // 689-713)
  int ewt_set(const double* ycur, double* weight) {
    if (o.rtol_v != nullptr) {
      for (int i = 0; i < N; i++) {
        const double d = std::fma(o.rtol_v[i], std::fabs(ycur[i]), o.atol[i]);
        if (!(d > 0.0)) return -1;
        weight[i] = 1.0 / d;
      }
      return 0;
    }
    for (int i = 0; i < N; i++) weight[i] = std::fabs(ycur[i]);
    for (int i = 0; i < N; i++) weight[i] = (o.rtol * weight[i]) + o.atol[i];
    if (atolmin0) {
      double mn = weight[0];
      for (int i = 1; i < N; i++)
        if (weight[i] < mn) mn = weight[i];
      if (mn <= 0.0) return -1;
    }
    for (int i = 0; i < N; i++) weight[i] = 1.0 / weight[i];
    return 0;
  }
  // cvHin, cvUpperBoundH0, cvYddNorm (bdf_cell.hpp:717-794)
  int hin_(double tout) {
    const double tdiff = tout - tn;
    const int sign = (tdiff > 0.0) ? 1 : -1;
    const double tdist = std::fabs(tdiff);
    const double tround = UROUND * smax_(std::fabs(tn), std::fabs(tout));
    const double hlb = HLB_FACTOR * tround;
    const double hub = upper_bound_h0_(tdist);
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
        const int retval = ydd_norm_(hgs, &yddnrm);
        if (retval < 0) return RHSFUNC_FAIL;
        if (retval == SUCCESS) { hgOK = true; break; }
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
  double upper_bound_h0_(double tdist) {
    double* temp1 = tempv;
    double* temp2 = acor;
    for (int i = 0; i < N; i++) temp2[i] = std::fabs(zn[0][i]);
    ewt_set(zn[0], temp1);
    for (int i = 0; i < N; i++) temp1[i] = 1.0 / temp1[i];
    lin_sum_(N, HUB_FACTOR, temp2, 1.0, temp1, temp1);
    for (int i = 0; i < N; i++) temp2[i] = std::fabs(zn[1][i]);
    for (int i = 0; i < N; i++) temp1[i] = temp2[i] / temp1[i];
    const double hub_inv = max_norm_(N, temp1);
    double hub = HUB_FACTOR * tdist;
    if (hub * hub_inv > 1.0) hub = 1.0 / hub_inv;
    return hub;
  }
  int ydd_norm_(double hg, double* yddnrm) {
    lin_sum_(N, hg, zn[1], 1.0, zn[0], y);
    const int retval = P.rhs_cb(y, tempv);
    st.nfe++;
    if (retval < 0) return RHSFUNC_FAIL;
    if (retval > 0) return RHSFUNC_RECVR;
    lin_sum_(N, 1.0 / hg, tempv, -1.0 / hg, zn[1], tempv);
    *yddnrm = wrms_(N, tempv, ewt);
    return SUCCESS;
  }
  // cvStep (bdf_cell.hpp:798-822)
  int step_() {
    int ncf = 0, nef = 0;
    double dsm = 0.0;
    if (st.nst > 0 && hprime != h) adjust_params_();
    const double saved_t = tn;
    int nflag = FIRST_CALL;
    for (;;) {
      predict_();
      set_();
      nflag = nls_(nflag);
      const int kflag = handle_nflag_(&nflag, saved_t, &ncf);
      if (kflag == PREDICT_AGAIN) continue;
      if (kflag != DO_ERROR_TEST) return kflag;
      const int eflag = do_error_test_(&nflag, saved_t, &nef, &dsm);
      if (eflag == TRY_AGAIN) continue;
      if (eflag != SUCCESS) return eflag;
      break;
    }
    qmax_saved = false;
    const int q_step = q;
    complete_step_();
    prepare_next_step_(dsm);
    if (tape != nullptr) {  // y holds zn[0] + acor of the accepted attempt
      const size_t start = tape->size();
      tape->push_back(TP_CORRECT);
      tape->push_back(q_step);
      tape->push_back(gamma);
      tape->push_back(rl1);
      for (int i = 0; i < L_MAX; i++) tape->push_back(l[i]);
      tape->push_back(qmax_saved ? 1.0 : 0.0);
      for (int i = 0; i < N; i++) tape->push_back(y[i]);
      tape->push_back((double)(tape->size() - start + 1));
    }
    etamax = (st.nst <= SMALL_NST) ? ETA_MAX_ES : ETA_MAX_GS;
    scale_(N, tq[2], acor, acor);
    return SUCCESS;
  }
  void adjust_params_() {
    if (qprime != q) {
      adjust_order_(qprime - q);
      q = qprime;
      L = q + 1;
      qwait = L;
    }
    rescale_();
  }
  void adjust_order_(int deltaq) {
    if ((q == 2) && (deltaq != 1)) return;
    if (deltaq == 1) increase_bdf_();
    else if (deltaq == -1) decrease_bdf_();
  }
  void increase_bdf_() {
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
    scale_(N, A1, zn[QMAX], zn[L]);
    if (q > 1)
      for (int j = 2; j <= q; j++) axpy_(N, l[j], zn[L], zn[j]);
    rec_l_(TP_INCREASE, {(double)q, A1});
  }
  void decrease_bdf_() {
    for (int i = 0; i <= QMAX; i++) l[i] = 0.0;
    l[2] = 1.0;
    double hsum = 0.0;
    for (int j = 1; j <= q - 2; j++) {
      hsum += tau[j];
      const double xi = hsum / hscale;
      for (int i = j + 2; i >= 2; i--) l[i] = l[i] * xi + l[i - 1];
    }
    if (q > 2) {
      for (int j = 2; j < q; j++) axpy_(N, -l[j], zn[q], zn[j]);
      rec_l_(TP_DECREASE, {(double)q});
    }
  }
  void rescale_() {
    rec_(TP_RESCALE, {eta, (double)q});
    double c = eta;
    for (int j = 1; j <= q; j++) {
      scale_(N, c, zn[j], zn[j]);
      c = eta * c;
    }
    h = hscale * eta;
    next_h = h;
    hscale = h;
    nscon = 0;
  }
  void predict_() {
    rec_(TP_PREDICT, {(double)q});
    tn += h;
    for (int k = 1; k <= q; k++)
      for (int j = q; j >= k; j--) axpy_(N, 1.0, zn[j], zn[j - 1]);
  }
  void restore_(double saved_t) {
    rec_(TP_RESTORE, {(double)q});
    tn = saved_t;
    for (int k = 1; k <= q; k++)
      for (int j = q; j >= k; j--) axpy_(N, -1.0, zn[j], zn[j - 1]);
  }
  // cvSet, cvSetBDF, cvSetTqBDF (bdf_cell.hpp:903-954)
  void set_() {
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
    set_tq_bdf_(hsum, alpha0, alpha0_hat, xi_inv, xistar_inv);
    rl1 = 1.0 / l[1];
    gamma = h * rl1;
    if (st.nst == 0) gammap = gamma;
    gamrat = (st.nst > 0) ? gamma / gammap : 1.0;
  }
  void set_tq_bdf_(double hsum, double alpha0, double alpha0_hat,
                   double xi_inv, double xistar_inv) {
    const double A1 = 1.0 - alpha0_hat + alpha0;
    const double A2 = 1.0 + q * A1;
    tq[2] = std::fabs(A1 / (alpha0 * A2));
    tq[5] = std::fabs(A2 * xistar_inv / (l[q] * xi_inv));
    if (qwait == 1) {
      if (q > 1) {
        const double C = xistar_inv / l[q];
        const double A3 = alpha0 + 1.0 / q;
        const double A4 = alpha0_hat + xi_inv;
        const double Cpinv = (1.0 - A4 + A3) / A3;
        tq[1] = std::fabs(C * Cpinv);
      } else {
        tq[1] = 1.0;
      }
      hsum += tau[q];
      xi_inv = h / hsum;
      const double A5 = alpha0 - (1.0 / (q + 1));
      const double A6 = alpha0_hat - xi_inv;
      const double Cppinv = (1.0 - A6 + A5) / A2;
      tq[3] = std::fabs(Cppinv / (xi_inv * (q + 2) * A5));
    }
    tq[4] = CORTES / tq[2];
  }
  // the charge invariant of the Newton correction (bdf_cell.hpp:1266-1287)
  double inv_dot_(const double* x) const {
    double s = 0.0;
    for (int i = 0; i < o.inv_n; i++)
      if (species_charge(i) != 0) s += species_charge(i) * x[i];
    return s;
  }
  void inv_set_(double* x, double target) const {
    const int r = o.inv_row;
    double s = 0.0, sa = 0.0;
    for (int i = 0; i < o.inv_n; i++)
      if (i != r && species_charge(i) != 0) {
        s += species_charge(i) * x[i];
        sa += std::fabs(species_charge(i) * (zn[0][i] + acor[i]));
      }
    const double yr = zn[0][r] + acor[r];
    const double xr = (target - s) / species_charge(r);
    if (std::fabs(species_charge(r) * yr) >= 1e-6 * sa && yr + xr >= 0.0)
      x[r] = xr;
  }
  // cvNls + the Newton module (bdf_cell.hpp:958-1048)
  int nls_(int nflag) {
    convfail = ((nflag == FIRST_CALL) || (nflag == PREV_ERR_FAIL))
                   ? NO_FAILURES : FAIL_OTHER;
    bool callSetup = (nflag == PREV_CONV_FAIL) || (nflag == PREV_ERR_FAIL)
                     || (st.nst == 0) || (st.nst >= nstlp + MSBP)
                     || (std::fabs(gamrat - 1.0) > DGMAX_LSETUP);
    for (int i = 0; i < N; i++) acor[i] = 0.0;
    const double tol = tq[4];
    bool jbad = false;
    long niters = 0, nconvfails = 0;
    int retval;
    for (;;) {
      int curiter = 0;
      retval = residual_();
      if (retval != SUCCESS) break;
      if (callSetup) {
        retval = nls_lsetup_(jbad, &nls_jcur);
        if (retval != SUCCESS) break;
      }
      for (;;) {
        niters++;
        const bool inv = o.dq_jac && o.inv_row >= 0;
        const double cg = inv ? inv_dot_(delta) : 0.0;
        scale_(N, -1.0, delta, delta);
        retval = lsolve_(delta);
        if (retval != SUCCESS) break;
        if (inv) inv_set_(delta, -cg);
        lin_sum_(N, 1.0, acor, 1.0, delta, acor);
        retval = conv_test_(curiter, tol);
        curiter++;
        if (retval == SUCCESS) { nls_jcur = false; break; }
        if (retval != NLS_CONTINUE) break;
        if (curiter >= NLS_MAXCOR) { retval = NLS_CONV_RECVR; break; }
        retval = residual_();
        if (retval != SUCCESS) break;
      }
      if (retval == SUCCESS) break;
      // a Newton failure with FP32 factors: FP64 from the next setup on
      if (retval > 0 && fact32) lu64 = true;
      if ((retval > 0) && !nls_jcur) {
        nconvfails++;
        callSetup = true;
        jbad = true;
        for (int i = 0; i < N; i++) acor[i] = 0.0;
        continue;
      }
      break;
    }
    if (retval > 0 && fact32) lu64 = true;
    if (retval != SUCCESS) nconvfails++;
    st.nni += niters;
    st.nnf += nconvfails;
    if (retval != SUCCESS) return retval;
    lin_sum_(N, 1.0, zn[0], 1.0, acor, y);
    if (!acnrmcur) acnrm = wrms_(N, acor, ewt);
    jcur = false;
    return SUCCESS;
  }
  int residual_() {
    lin_sum_(N, 1.0, zn[0], 1.0, acor, y);
    const int retval = P.rhs_cb(y, ftemp);
    st.nfe++;
    if (retval < 0) return RHSFUNC_FAIL;
    if (retval > 0) return RHSFUNC_RECVR;
    lin_sum_(N, rl1, zn[1], 1.0, acor, delta);
    lin_sum_(N, -gamma, ftemp, 1.0, delta, delta);
    return SUCCESS;
  }
  int conv_test_(int m, double tol) {
    delnrm = wrms_(N, delta, ewt);
    if (m > 0) crate = smax_(CRDOWN * crate, delnrm / delp);
    const double dcon = delnrm * smin_(1.0, crate) / tol;
    if (dcon <= 1.0) {
      acnrm = (m == 0) ? delnrm : wrms_(N, acor, ewt);
      acnrmcur = true;
      return SUCCESS;
    }
    if ((m >= 1) && (delnrm > RDIV * delp)) return NLS_CONV_RECVR;
    delp = delnrm;
    return NLS_CONTINUE;
  }
  int nls_lsetup_(bool jbad, bool* jcur_out) {
    if (jbad) convfail = FAIL_BAD_J;
    const int retval = ls_setup_();
    st.nsetups++;
    *jcur_out = jcur;
    gamrat = 1.0;
    gammap = gamma;
    crate = 1.0;
    delnrm = 0.0;
    nstlp = st.nst;
    if (retval < 0) return LSETUP_FAIL;
    if (retval > 0) return NLS_CONV_RECVR;
    return SUCCESS;
  }
  // cvLsSetup + A = I - gamma J + dense LU (bdf_cell.hpp:1069-1130)
  int ls_setup_() {
#ifdef KB_LARGE_NETWORK
    {
      const double dgamma = std::fabs((gamma / gammap) - 1.0);
      const bool jbad_ls = (st.nst == 0) || (st.nst >= nstlj + MSBJ)
                           || ((convfail == FAIL_BAD_J) && (dgamma < DGMAX_JBAD))
                           || (convfail == FAIL_OTHER);
      jcur = jbad_ls;
      if (jbad_ls) {
        P.jac_sparse_cb(y, savedJ);
        if (N > NSPEC)
          P.jac_border(y, border.B, border.C, &border.D, vtemp1, vtemp2);
      }
      const double c = -gamma;
      for (int k = 0; k < NNZ_LU; k++) A[k] = 0.0;
      for (int e = 0; e < NNZ_J; e++) A[sp_jpos[e]] = savedJ[e] * c;
      for (int i = 0; i < NSPEC; i++) A[sp_di[i]] += 1.0;
      if (jcur) {
        st.nje++;
        nstlj = st.nst;
      }
      fact32 = false;
      if (sp_getrf_(A, spw) > 0) return LS_LUFACT_FAIL;
      if (N > NSPEC && sp_border_factor_(A, c, border) > 0)
        return LS_LUFACT_FAIL;
      return 0;
    }
#endif
    const long NN = (long)N * N;
    const double dgamma = std::fabs((gamma / gammap) - 1.0);
    const bool jbad_ls = (st.nst == 0) || (st.nst >= nstlj + MSBJ)
                         || ((convfail == FAIL_BAD_J) && (dgamma < DGMAX_JBAD))
                         || (convfail == FAIL_OTHER);
    int retval = 0;
    if (!jbad_ls) {
      jcur = false;
    } else {
      jcur = true;
      if (!o.dq_jac)
        for (long k = 0; k < NN; k++) savedJ[k] = 0.0;
      const int jr = o.dq_jac ? dq_jac_(tn, y, ftemp, savedJ, vtemp1)
                              : P.jac_cb(y, savedJ, vtemp1, vtemp2);
      if (jr < 0) retval = -1;
      else if (jr > 0) retval = 1;
    }
    if (retval == 0) {
      const double c = -gamma;
      for (int j = 0; j < N; j++) {
        for (int i = 0; i < N; i++) {
          const long k = i + (long)j * N;
          A[k] = savedJ[k] * c;
        }
        A[j + (long)j * N] += 1.0;
      }
    }
    if (jcur) {
      st.nje++;
      nstlj = st.nst;
    }
    if (retval != 0) return retval;
    fact32 = o.lu32 && !lu64;
    if (fact32) {
      for (long k = 0; k < NN; k++) A32[k] = (float)A[k];
      return getrf_(A32.data(), N, piv.data()) > 0 ? LS_LUFACT_FAIL : 0;
    }
    if (o.lu32) st.nlu64++;
    return getrf_(A, N, piv.data()) > 0 ? LS_LUFACT_FAIL : 0;
  }
  int lsolve_(double* b) {
#ifdef KB_LARGE_NETWORK
    if (N > NSPEC) sp_getrs_border_(A, border, b, vtemp3, b);
    else sp_getrs_(A, b, vtemp3, b);
#else
    if (fact32) getrs_(A32.data(), N, piv.data(), b);
    else getrs_(A, N, piv.data(), b);
#endif
    if (gamrat != 1.0) scale_(N, 2.0 / (1.0 + gamrat), b, b);
    return SUCCESS;
  }
  // cvLsDenseDQJac (bdf_cell.hpp:1290-1311)
  int dq_jac_(double t, double* yv, const double* fy, double* Jac,
              double* tmp1) {
    (void)t;
    double* ftmp = tmp1;
    const double srur = ssqrt_(UROUND);
    const double fnorm = wrms_(N, fy, ewt);
    const double minInc = (fnorm != 0.0)
        ? (MIN_INC_MULT * std::fabs(h) * UROUND * (double)N * fnorm) : 1.0;
    int retval = 0;
    for (int j = 0; j < N; j++) {
      const double yjsaved = yv[j];
      const double inc = smax_(srur * std::fabs(yjsaved), minInc / ewt[j]);
      yv[j] += inc;
      retval = P.rhs_cb(yv, ftmp);
      st.nfeDQ++;
      if (retval != 0) break;
      yv[j] = yjsaved;
      const double inc_inv = 1.0 / inc;
      lin_sum_(N, inc_inv, ftmp, -inc_inv, fy, Jac + (long)j * N);
    }
    return retval;
  }
  int handle_nflag_(int* nflagPtr, double saved_t, int* ncfPtr) {
    const int nflag = *nflagPtr;
    if (nflag == SUCCESS) return DO_ERROR_TEST;
    st.ncfn++;
    restore_(saved_t);
    if (nflag < 0) {
      if (nflag == LSETUP_FAIL) return LSETUP_FAIL;
      if (nflag == LSOLVE_FAIL) return LSOLVE_FAIL;
      if (nflag == RHSFUNC_FAIL) return RHSFUNC_FAIL;
      return NLS_FAIL;
    }
    (*ncfPtr)++;
    etamax = 1.0;
    if ((std::fabs(h) <= 0.0 * ONEPSM) || (*ncfPtr == o.max_conv_fails)) {
      if (nflag == NLS_CONV_RECVR) return CONV_FAILURE;
      if (nflag == RHSFUNC_RECVR) return REPTD_RHSFUNC_ERR;
    }
    eta = smax_(ETA_CF, 0.0 / std::fabs(h));
    *nflagPtr = PREV_CONV_FAIL;
    rescale_();
    return PREDICT_AGAIN;
  }
  int do_error_test_(int* nflagPtr, double saved_t, int* nefPtr,
                     double* dsmPtr) {
    const double dsm = acnrm * tq[2];
    *dsmPtr = dsm;
    if (dsm <= 1.0) return SUCCESS;
    (*nefPtr)++;
    st.netf++;
    *nflagPtr = PREV_ERR_FAIL;
    restore_(saved_t);
    if ((std::fabs(h) <= 0.0 * ONEPSM) || (*nefPtr == o.max_err_fails))
      return ERR_FAILURE;
    etamax = 1.0;
    if (*nefPtr <= MXNEF1) {
      eta = 1.0 / (std::pow(BIAS2 * dsm, 1.0 / L) + ADDON);
      eta = smax_(ETA_MIN_EF, smax_(eta, 0.0 / std::fabs(h)));
      if (*nefPtr >= SMALL_NEF) eta = smin_(eta, ETA_MAX_EF);
      rescale_();
      return TRY_AGAIN;
    }
    if (q > 1) {
      eta = smax_(ETA_MIN_EF, 0.0 / std::fabs(h));
      adjust_order_(-1);
      L = q;
      q--;
      qwait = L;
      rescale_();
      return TRY_AGAIN;
    }
    eta = smax_(ETA_MIN_EF, 0.0 / std::fabs(h));
    h *= eta;
    next_h = h;
    hscale = h;
    qwait = LONG_WAIT;
    nscon = 0;
    const int retval = P.rhs_cb(zn[0], tempv);
    st.nfe++;
    if (retval < 0) return RHSFUNC_FAIL;
    if (retval > 0) return UNREC_RHSFUNC_ERR;
    scale_(N, h, tempv, zn[1]);
    rec_(TP_RESET1, {h}, zn[0]);
    return TRY_AGAIN;
  }
  void complete_step_() {
    lu64 = false;
    st.nst++;
    nscon++;
    hu = h;
    qu = q;
    for (int i = q; i >= 2; i--) tau[i] = tau[i - 1];
    if ((q == 1) && (st.nst > 1)) tau[2] = tau[1];
    tau[1] = h;
    for (int j = 0; j <= q; j++) axpy_(N, l[j], acor, zn[j]);
    qwait--;
    if ((qwait == 1) && (q != QMAX)) {
      copy_(acor, zn[QMAX]);
      qmax_saved = true;
      saved_tq5 = tq[5];
    }
  }
  void prepare_next_step_(double dsm) {
    if (etamax == 1.0) {
      qwait = qwait > 2 ? qwait : 2;
      qprime = q;
      hprime = h;
      eta = 1.0;
      return;
    }
    etaq = 1.0 / (std::pow(BIAS2 * dsm, 1.0 / L) + ADDON);
    if (qwait != 0) {
      eta = etaq;
      qprime = q;
      set_eta_();
    } else {
      qwait = 2;
      etaqm1 = compute_etaqm1_();
      etaqp1 = compute_etaqp1_();
      choose_eta_();
      set_eta_();
    }
  }
  void set_eta_() {
    if ((eta > ETA_MIN_FX) && (eta < ETA_MAX_FX)) {
      eta = 1.0;
      hprime = h;
      return;
    }
    if (eta >= ETA_MAX_FX) {
      eta = smin_(eta, etamax);
      eta /= smax_(1.0, std::fabs(h) * 0.0 * eta);
    } else {
      eta = smax_(eta, ETA_MIN);
      eta = smax_(eta, 0.0 / std::fabs(h));
    }
    hprime = h * eta;
    if (qprime < q) nscon = 0;
  }
  double compute_etaqm1_() {
    etaqm1 = 0.0;
    if (q > 1) {
      const double ddn = wrms_(N, zn[q], ewt) * tq[1];
      etaqm1 = 1.0 / (std::pow(BIAS1 * ddn, 1.0 / q) + ADDON);
    }
    return etaqm1;
  }
  double compute_etaqp1_() {
    etaqp1 = 0.0;
    if (q != QMAX) {
      if (saved_tq5 == 0.0) return etaqp1;
      const double cquot = (tq[5] / saved_tq5) * spowi_(h / tau[2], L);
      lin_sum_(N, -cquot, zn[QMAX], 1.0, acor, tempv);
      const double dup = wrms_(N, tempv, ewt) * tq[3];
      etaqp1 = 1.0 / (std::pow(BIAS3 * dup, 1.0 / (L + 1)) + ADDON);
    }
    return etaqp1;
  }
  void choose_eta_() {
    const double etam = smax_(etaqm1, smax_(etaq, etaqp1));
    if ((etam > ETA_MIN_FX) && (etam < ETA_MAX_FX)) {
      eta = 1.0;
      qprime = q;
      return;
    }
    if (etam == etaq) {
      eta = etaq;
      qprime = q;
    } else if (etam == etaqm1) {
      eta = etaqm1;
      qprime = q - 1;
    } else {
      eta = etaqp1;
      qprime = q + 1;
      copy_(acor, zn[QMAX]);
      qmax_saved = true;
    }
  }
  void get_dky_(double t, double* dky) {
    const double s = (t - tn) / h;
    for (int j = q; j >= 0; j--) {
      double c = 1.0;
      for (int i = 0; i < j; i++) c *= s;
      if (j == q) scale_(N, c, zn[j], dky);
      else axpy_(N, c, zn[j], dky);
    }
  }
};

}  // namespace

// the solve options of one call (the krome_opts keys the hot path reads;
// reference runtime/krome.hpp:187-254)
struct oracle_opts {
  int evolve_T;
  int jac;      // 0 auto, 1 analytic, 2 difference quotients
  double rtol, atol_n, atol_T;
  long max_steps;
  int max_err_fails, max_conv_fails, max_restarts;
  int clip_negative;
  int lu32;     // the Newton matrix factored in FP32 (FP64 fallback)
  int conserve;  // post-solve conservation mode (solve_cell.hpp:1458-1500)
  // per-species tolerances [NSPEC] (negative entry: the scalar), or null
  const double* atol_sp;
  const double* rtol_sp;
  // photon bins: sigma[NPHOTO][ph_B] and the cells' fields Phi[ncell][ph_B]
  // (ph_B = 0: none); each cell's photo rates k_r = sum_b sigma_rb Phi_b
  // (solve_cell.hpp:609-614 with photo.hpp photo_rates)
  const double* ph_sigma;
  const double* ph_phi;
  int ph_B;
};

// per-cell counters: nst, nfe, nfeDQ, nje, nsetups, nni, nnf, netf,
// restarts, nlu64 (FP64 refactors of the lu32 form)
constexpr int ORACLE_NSTAT = 10;

#define ORACLE_API __attribute__((visibility("default")))

extern "C" {

// the rate coefficients at (T, n) with the parameter row par: the
// reference's rates() (zero, rates_fixed, rates_var)
ORACLE_API void oracle_rates(double T, const double* n, const double* par,
                             double* k) {
  Params p;
  params_from_row(par, p);
  for (int i = 0; i < NREA; ++i) k[i] = 0.0;
  rates_fixed(T, n, p, k);
  rates_var(T, n, p, k);
}
#ifdef KB_LARGE_NETWORK
// the large path's forms of the rate coefficients, beside the direct
// evaluation of oracle_rates: kp from the generated parts (hnuc =
// Hnuclei_(n)), ka with the density-dependent rates from their three points
// (fi = 0, fi = 1, hnuc = 1) as e0 (1 - fi) + e1 fi + eh hnuc. Returns
// BK_VAR_AFFINE.
ORACLE_API int oracle_rates_forms(double T, const double* n,
                                  const double* par, double* kp, double* ka) {
  Params p;
  params_from_row(par, p);
  const double h = Hnuclei_(n);
  for (int i = 0; i < NREA; ++i) kp[i] = 0.0;
  for (int part = 0; part < RPART; ++part) {
    rates_fixed_part(part, T, n, p, h, kp);
    rates_var_part(part, T, n, p, h, kp);
  }
  std::vector<double> y(n, n + NSPEC);
  y.push_back(1.0);
  std::vector<double> k(NREA, 0.0), e0(BK_NVAR), e1(BK_NVAR), eh(BK_NVAR);
  for (int pt = 0; pt < 3; ++pt) {
    bk_set_ice(y.data(), p, pt == 1);
    for (int part = 0; part < RPART; ++part)
      rates_var_part(part, T, y.data(), p, pt == 2 ? 1.0 : 0.0, k.data());
    for (int j = 0; j < BK_NVAR; ++j) {
      const double v = k[bk_var[j]];
      if (pt == 0) e0[j] = v;
      else if (pt == 1) e1[j] = v;
      else eh[j] = v - e0[j];
    }
  }
  const double fi = bk_ice_cover(n, p);
  for (int i = 0; i < NREA; ++i) ka[i] = kp[i];
  for (int j = 0; j < BK_NVAR; ++j)
    ka[bk_var[j]] = e0[j] * (1.0 - fi) + e1[j] * fi + eh[j] * h;
  return BK_VAR_AFFINE;
}
#endif
// the thermal term directly and from its temperature-only parts evaluated
// at the state y (the adjoint's Tgas row): out[0] thermal_dTdt(T, n, k, p),
// out[1] thermal_dTdt_with(thermal_pre(T, y, p), T, n, k, p)
ORACLE_API void oracle_thermal_forms(double T, const double* y,
                                     const double* n, const double* k,
                                     const double* par, double* out) {
  Params p;
  params_from_row(par, p);
  ThermalPre q;
  thermal_pre(T, y, p, q);
  out[0] = thermal_dTdt(T, n, k, p);
  out[1] = thermal_dTdt_with(q, T, n, k, p);
}
ORACLE_API int oracle_nrea(void) { return NREA; }
ORACLE_API int oracle_nspec(void) { return NSPEC; }
ORACLE_API int oracle_npar(void) { return NPAR; }
ORACLE_API const char* oracle_network(void) { return NETWORK_KEY; }

// one cell (solve_cell.hpp:2094-2203 with integrate_ 1662-1705 and the
// restart wrapper bdf_cell.hpp:1513-1547); n, Tgas in/out
namespace {
// one cell; mult (exp of the rate ln-multipliers) and tape (the adjoint's
// recording) may be null; yfin receives the integrator's final y before the
// post-solve rules (may be null)
// a cell's photo rates from its field row (none without photo reactions)
extern "C++" template <class P>
void photo_rates_(P& p, const oracle_opts* so, const double* phirow) {
  if constexpr (NPHOTO > 0) {
    if (phirow != nullptr && so->ph_B > 0)
      kbphoto::rates_of_field(so->ph_sigma, so->ph_B, phirow, p.kph);
  } else {
    (void)p; (void)so; (void)phirow;
  }
}

int solve_one_(double* n, double* Tgas, const double* par, double dt,
               const oracle_opts* so, long* stats, const double* mult,
               std::vector<double>* tape, double* yfin,
               const double* phirow = nullptr) {
  Problem c;
  c.mult = mult;
  params_from_row(par, c.p);
  if (params_missing(c.p) >= 0) return FLAG_PARAM_UNSET;
  photo_rates_(c.p, so, phirow);
#if KB_NFREEZE > 0
  // the adjoint does not differentiate frozen rows: refused there
  if (tape != nullptr && freeze_active(c.p)) return -104;
#endif
  c.Tfix = *Tgas;
  c.NEQ = NSPEC;
  if (so->evolve_T) c.iT = c.NEQ++;
  const int N = c.NEQ;
  std::vector<double> y(N), avec(N);
  for (int i = 0; i < NSPEC; ++i) y[i] = n[i];
  if (c.iT >= 0) y[c.iT] = *Tgas;
  if (NREA_FIXED > 0) {
    if (c.iT < 0) {
      for (int i = 0; i <= NREA; ++i) c.kfix[i] = 0.0;
      rates_fixed(c.state_T(n), n, c.p, c.kfix);
      c.kfix_on = true;
    } else {
      c.kT_on = true;
      c.kT_ok = false;
    }
  }
  // the species' tolerances (solve_cell.hpp:2129-2139)
  auto tol = [](const double* v, int i, double s) {
    return v != nullptr && !(v[i] < 0.0) ? v[i] : s;
  };
  for (int i = 0; i < NSPEC; ++i) avec[i] = tol(so->atol_sp, i, so->atol_n);
  if (c.iT >= 0) avec[c.iT] = so->atol_T;
  std::vector<double> rvec;
  bool rvar = false;
  for (int i = 0; i < NSPEC; ++i)
    rvar = rvar || tol(so->rtol_sp, i, so->rtol) != so->rtol;
  if (rvar) {
    rvec.assign(N, so->rtol);
    for (int i = 0; i < NSPEC; ++i) rvec[i] = tol(so->rtol_sp, i, so->rtol);
  }
  // JAC_AUTO (solve_cell.hpp:2141-2142): analytic at fixed Tgas, the
  // difference quotients when Tgas evolves
  const int jac = so->jac != 0 ? so->jac : (so->evolve_T ? 2 : 1);
#ifdef KB_LARGE_NETWORK
  // the large path's Jacobian is the analytic one (the difference
  // quotients over every column are not restated there)
  if (jac == 2) return -104;
#endif
  BdfOpts bo;
  bo.rtol = so->rtol;
  bo.atol = avec.data();
  bo.rtol_v = rvar ? rvec.data() : nullptr;
  bo.max_steps = so->max_steps;
  bo.max_err_fails = so->max_err_fails;
  bo.max_conv_fails = so->max_conv_fails;
  bo.dq_jac = jac == 2;
  bo.lu32 = so->lu32 != 0;
  if (IDX_ELECTRON >= 0 && KB_NFREEZE == 0) {  // charge_newton_ (solve_cell.hpp:1631-1642)
    bo.inv_row = IDX_ELECTRON;
    bo.inv_n = NSPEC;
  }
  Stats bs;
  int restarts = 0;
  int flag;
  {
    Cvode cv(c, N, bo);
    cv.tape = tape;
    cv.reinit(0.0, y.data(), bo.h0);
    double t = 0.0;
    for (;;) {
      const int f = cv.solve(dt, y.data(), &t);
      bs.add(cv.st);
      if (f >= 0) { flag = 0; break; }
      const bool restartable = f == ERR_FAILURE || f == CONV_FAILURE
                               || f == REPTD_RHSFUNC_ERR;
      if (!restartable || restarts >= so->max_restarts) { flag = f; break; }
      ++restarts;
      const double hcur = cv.current_step();
      cv.reinit(t, y.data(), hcur > 0.0 ? 0.1 * hcur : 0.0);
    }
  }
  if (stats != nullptr) {
    const long s[ORACLE_NSTAT] = {bs.nst, bs.nfe, bs.nfeDQ, bs.nje,
                                  bs.nsetups, bs.nni, bs.nnf, bs.netf,
                                  (long)restarts, bs.nlu64};
    for (int i = 0; i < ORACLE_NSTAT; ++i) stats[i] = s[i];
  }
  if (flag == 0 && c.iT >= 0 && !(y[c.iT] > 0.0 && std::isfinite(y[c.iT])))
    flag = FLAG_NONPOSITIVE_T;
  if (c.hit_T0 && (flag == REPTD_RHSFUNC_ERR || flag == RHSFUNC_FAIL
                   || flag == UNREC_RHSFUNC_ERR || flag == FIRST_RHSFUNC_ERR))
    flag = FLAG_NONPOSITIVE_T;
  if (yfin != nullptr)
    for (int i = 0; i < N; ++i) yfin[i] = y[i];
  if (flag == 0) {
    double n0[NSPEC];
    for (int i = 0; i < NSPEC; ++i) {
      n0[i] = n[i];
      n[i] = y[i];
      if (so->clip_negative && n[i] < 0.0) n[i] = 0.0;
    }
    conserve_cell(n0, n, so->conserve, c.p);  // solve_cell.hpp:2169-2175
    if (c.iT >= 0) *Tgas = y[c.iT];
  }
  return flag;
}

// dF/dy at y for the adjoint, column-major: the stoichiometric block where
// it is exact (rates independent of the densities: the block at fixed k is
// dF/dn), a central difference for the Tgas column and forward differences
// (fd_step_n) for the Tgas row; else central differences on every column
void adjoint_jac_(Problem& P, const double* y, double* J, double* yp,
                  double* fp, double* fq) {
  const int N = P.NEQ;
  for (long k = 0; k < (long)N * N; ++k) J[k] = 0.0;
  for (int i = 0; i < N; ++i) yp[i] = y[i];
  if (!RATES_DEPEND_ON_N) {
    P.eval_rates(P.state_T(y), y, P.k0);
    jac_stoich(y, P.k0, J, 1, N);
    if (P.iT < 0) return;
    const int t = P.iT;
    {
      const double h = std::fmax(1e-6 * std::fabs(y[t]), 1e-8);
      yp[t] = y[t] + h;
      P.full_rhs(yp, fp);
      yp[t] = y[t] - h;
      P.full_rhs(yp, fq);
      yp[t] = y[t];
      for (int i = 0; i < N; ++i) J[i + (long)t * N] = (fp[i] - fq[i]) / (2.0 * h);
    }
    P.full_rhs(y, fq);
    const double f0 = fq[t];
    for (int j = 0; j < NSPEC; ++j) {
      const double h = Problem::fd_step_n(y, j);
      yp[j] = y[j] + h;
      P.full_rhs(yp, fp);
      yp[j] = y[j];
      J[t + (long)j * N] = (fp[t] - f0) / h;
    }
    return;
  }
  for (int j = 0; j < N; ++j) {
    const double h = j == P.iT ? std::fmax(1e-6 * std::fabs(y[j]), 1e-8)
                               : Problem::fd_step_n(y, j);
    yp[j] = y[j] + h;
    P.full_rhs(yp, fp);
    yp[j] = y[j] - h;
    P.full_rhs(yp, fq);
    yp[j] = y[j];
    for (int i = 0; i < N; ++i) J[i + (long)j * N] = (fp[i] - fq[i]) / (2.0 * h);
  }
}

// the reverse sweep over one cell's tape. lam_y: the adjoint of the final
// y; out: lam_y0 (the adjoint of the initial y), gm += the ln-multiplier
// gradient. The corrector's map is differentiated at its root:
// (I - gamma J) d acor = gamma J d zn0 - rl1 d zn1 + gamma dF/dm dm.
void adjoint_sweep_(Problem& P, const std::vector<double>& tape,
                    const double* lam_y, double* lam_y0, double* gm) {
  const int N = P.NEQ;
  std::vector<double> Lam((long)L_MAX * N, 0.0), J((long)N * N), AT((long)N * N);
  std::vector<double> mu(N), la(N), yp(N), fp(N), fq(N);
  std::vector<int> piv(N);
  auto lam = [&](int j) { return Lam.data() + (long)j * N; };
  // the terms of zn1 = h f(y): lam0 += h J^T lam1, gm += h dF/dm^T lam1
  auto f_terms = [&](const double* yv, double h) {
    for (int i = 0; i < N; ++i) mu[i] = h * lam(1)[i];
    adjoint_jac_(P, yv, J.data(), yp.data(), fp.data(), fq.data());
    for (int j = 0; j < N; ++j) {
      double t = 0.0;
      for (int i = 0; i < N; ++i) t += J[i + (long)j * N] * mu[i];
      lam(0)[j] += t;
    }
    P.lnk_vjp_at(yv, mu.data(), gm);
    for (int i = 0; i < N; ++i) lam(1)[i] = 0.0;
  };
  long pos = (long)tape.size();
  while (pos > 0) {
    const long len = (long)tape[pos - 1];
    const long start = pos - len;
    const double* r = tape.data() + start;
    switch ((int)r[0]) {
      case TP_DKY: {
        const double sv = r[1];
        const int q = (int)r[2];
        for (int j = 0; j <= q; j++) {
          double c = 1.0;
          for (int i = 0; i < j; i++) c *= sv;
          for (int i = 0; i < N; i++) lam(j)[i] += c * lam_y[i];
        }
        break;
      }
      case TP_CORRECT: {
        const int q = (int)r[1];
        const double gam = r[2], rl1 = r[3];
        const double* l = r + 4;
        const bool save = r[4 + L_MAX] != 0.0;
        const double* yn = r + 5 + L_MAX;
        for (int i = 0; i < N; i++) {
          double t = save ? lam(QMAX)[i] : 0.0;
          for (int j = 0; j <= q; j++) t += l[j] * lam(j)[i];
          la[i] = t;
        }
        if (save)
          for (int i = 0; i < N; i++) lam(QMAX)[i] = 0.0;
        adjoint_jac_(P, yn, J.data(), yp.data(), fp.data(), fq.data());
        for (int j = 0; j < N; j++)
          for (int i = 0; i < N; i++)
            AT[i + (long)j * N] = (i == j ? 1.0 : 0.0) - gam * J[j + (long)i * N];
        getrf_(AT.data(), N, piv.data());
        for (int i = 0; i < N; i++) mu[i] = la[i];
        getrs_(AT.data(), N, piv.data(), mu.data());
        for (int j = 0; j < N; j++) {
          double t = 0.0;
          for (int i = 0; i < N; i++) t += J[i + (long)j * N] * mu[i];
          lam(0)[j] += gam * t;
        }
        for (int i = 0; i < N; i++) lam(1)[i] -= rl1 * mu[i];
        for (int i = 0; i < N; i++) mu[i] *= gam;
        P.lnk_vjp_at(yn, mu.data(), gm);
        break;
      }
      case TP_PREDICT:
      case TP_RESTORE: {
        const int q = (int)r[1];
        const double sg = (int)r[0] == TP_PREDICT ? 1.0 : -1.0;
        for (int k = q; k >= 1; k--)
          for (int j = k; j <= q; j++)
            for (int i = 0; i < N; i++) lam(j)[i] += sg * lam(j - 1)[i];
        break;
      }
      case TP_RESCALE: {
        const double eta = r[1];
        const int q = (int)r[2];
        double c = eta;
        for (int j = 1; j <= q; j++) {
          for (int i = 0; i < N; i++) lam(j)[i] *= c;
          c = eta * c;
        }
        break;
      }
      case TP_INCREASE: {
        const int q = (int)r[1];
        const double A1 = r[2];
        const double* l = r + 3;
        const int L = q + 1;
        for (int j = 2; j <= q; j++)
          for (int i = 0; i < N; i++) lam(L)[i] += l[j] * lam(j)[i];
        if (L == QMAX) {
          for (int i = 0; i < N; i++) lam(QMAX)[i] *= A1;
        } else {
          for (int i = 0; i < N; i++) {
            lam(QMAX)[i] += A1 * lam(L)[i];
            lam(L)[i] = 0.0;
          }
        }
        break;
      }
      case TP_DECREASE: {
        const int q = (int)r[1];
        const double* l = r + 2;
        for (int j = 2; j < q; j++)
          for (int i = 0; i < N; i++) lam(q)[i] -= l[j] * lam(j)[i];
        break;
      }
      case TP_RESET1:
        f_terms(r + 2, r[1]);
        break;
      case TP_INIT:
        f_terms(r + 2, r[1]);
        for (int j = 1; j < L_MAX; j++)
          for (int i = 0; i < N; i++) lam(j)[i] = 0.0;
        break;
      default:
        break;
    }
    pos = start;
  }
  for (int i = 0; i < N; i++) lam_y0[i] = lam(0)[i];
}
// the tangent (forward-mode) sweep over the same tape: dy0 -> dy_final
// for the perturbation dy0 of the initial state and dm of the ln-multipliers
// (the transpose of adjoint_sweep_; the tests check <lam, dy_final> =
// <lam_y0, dy0> + <gm, dm>)
void tangent_sweep_(Problem& P, const std::vector<double>& tape,
                    const double* dy0, const double* dmv, double* dyf) {
  const int N = P.NEQ;
  std::vector<double> D((long)L_MAX * N, 0.0), J((long)N * N), A((long)N * N);
  std::vector<double> b(N), yp(N), fp(N), fq(N), fm(N);
  std::vector<int> piv(N);
  bool first = true;
  auto dz = [&](int j) { return D.data() + (long)j * N; };
  // dF/dm dm at y: the change of f when ln k moves by dm (f linear in k)
  auto fm_dm = [&](const double* yv, double* out) {
    for (int i = 0; i < N; ++i) out[i] = 0.0;
    if (dmv == nullptr) return;
    for (int i = 0; i < N; ++i) yp[i] = yv[i];
    const double* save = P.mult;
    std::vector<double> mp(NREA), mm(NREA);
    for (int r = 0; r < NREA; ++r) {
      const double m0 = save != nullptr ? save[r] : 1.0;
      mp[r] = m0 * std::exp(1e-6 * dmv[r]);
      mm[r] = m0 * std::exp(-1e-6 * dmv[r]);
    }
    P.mult = mp.data();
    P.full_rhs(yp.data(), fp.data());
    P.mult = mm.data();
    P.full_rhs(yp.data(), fq.data());
    P.mult = save;
    for (int i = 0; i < N; ++i) out[i] = (fp[i] - fq[i]) / 2e-6;
  };
  for (size_t pos = 0; pos < tape.size();) {
    const double* r = tape.data() + pos;
    int len = 0;
    switch ((int)r[0]) {
      case TP_INIT: len = 3 + N; break;
      case TP_RESCALE: len = 4; break;
      case TP_INCREASE: len = 4 + L_MAX; break;
      case TP_DECREASE: len = 3 + L_MAX; break;
      case TP_PREDICT: case TP_RESTORE: len = 3; break;
      case TP_RESET1: len = 3 + N; break;
      case TP_CORRECT: len = 6 + L_MAX + N; break;
      case TP_DKY: len = 4; break;
      default: return;
    }
    switch ((int)r[0]) {
      case TP_INIT:
      case TP_RESET1: {
        const double h = r[1];
        const double* yv = r + 2;
        if ((int)r[0] == TP_INIT) {
          // the first segment starts from dy0; a restart from its zn[0]
          for (int j = 1; j < L_MAX; ++j)
            for (int i = 0; i < N; ++i) dz(j)[i] = 0.0;
          if (first)
            for (int i = 0; i < N; ++i) dz(0)[i] = dy0[i];
          first = false;
        }
        adjoint_jac_(P, yv, J.data(), yp.data(), fp.data(), fq.data());
        fm_dm(yv, fm.data());
        for (int i = 0; i < N; ++i) {
          double t = fm[i];
          for (int j = 0; j < N; ++j) t += J[i + (long)j * N] * dz(0)[j];
          dz(1)[i] = h * t;
        }
        break;
      }
      case TP_RESCALE: {
        const double eta = r[1];
        const int q = (int)r[2];
        double c = eta;
        for (int j = 1; j <= q; j++) {
          for (int i = 0; i < N; i++) dz(j)[i] *= c;
          c *= eta;
        }
        break;
      }
      case TP_INCREASE: {
        const int q = (int)r[1];
        const double A1 = r[2];
        const double* l = r + 3;
        const int L = q + 1;
        for (int i = 0; i < N; i++) dz(L)[i] = A1 * dz(QMAX)[i];
        for (int j = 2; j <= q; j++)
          for (int i = 0; i < N; i++) dz(j)[i] += l[j] * dz(L)[i];
        break;
      }
      case TP_DECREASE: {
        const int q = (int)r[1];
        const double* l = r + 2;
        for (int j = 2; j < q; j++)
          for (int i = 0; i < N; i++) dz(j)[i] -= l[j] * dz(q)[i];
        break;
      }
      case TP_PREDICT:
      case TP_RESTORE: {
        const int q = (int)r[1];
        const double sg = (int)r[0] == TP_PREDICT ? 1.0 : -1.0;
        for (int k = 1; k <= q; k++)
          for (int j = q; j >= k; j--)
            for (int i = 0; i < N; i++) dz(j - 1)[i] += sg * dz(j)[i];
        break;
      }
      case TP_CORRECT: {
        const int q = (int)r[1];
        const double gam = r[2], rl1 = r[3];
        const double* l = r + 4;
        const bool save = r[4 + L_MAX] != 0.0;
        const double* yn = r + 5 + L_MAX;
        adjoint_jac_(P, yn, J.data(), yp.data(), fp.data(), fq.data());
        fm_dm(yn, fm.data());
        for (int i = 0; i < N; i++) {
          double t = gam * fm[i] - rl1 * dz(1)[i];
          for (int j = 0; j < N; j++) t += gam * J[i + (long)j * N] * dz(0)[j];
          b[i] = t;
        }
        for (int j = 0; j < N; j++)
          for (int i = 0; i < N; i++)
            A[i + (long)j * N] = (i == j ? 1.0 : 0.0) - gam * J[i + (long)j * N];
        getrf_(A.data(), N, piv.data());
        getrs_(A.data(), N, piv.data(), b.data());
        for (int j = 0; j <= q; j++)
          for (int i = 0; i < N; i++) dz(j)[i] += l[j] * b[i];
        if (save)
          for (int i = 0; i < N; i++) dz(QMAX)[i] = b[i];
        break;
      }
      case TP_DKY: {
        const double sv = r[1];
        const int q = (int)r[2];
        for (int i = 0; i < N; i++) dyf[i] = 0.0;
        for (int j = 0; j <= q; j++) {
          double c = 1.0;
          for (int i = 0; i < j; i++) c *= sv;
          for (int i = 0; i < N; i++) dyf[i] += c * dz(j)[i];
        }
        break;
      }
    }
    pos += len;
  }
}
}  // namespace

// one cell's tangent dy_final for the perturbation (dy0, dm), from the tape
// of its forward solve (lnm one row as in oracle_adjoint_cells): the test of
// the reverse sweep's transposition, <lam, dy_final> = <lam_y0, dy0> +
// <gm, dm>
ORACLE_API int oracle_tangent_one(double* n, double* Tgas, const double* dt,
                                  const double* par, const double* lnm,
                                  const double* dy0, const double* dm,
                                  double* dyf, const oracle_opts* so) {
  double mult[NREA + 1];
  for (int r = 0; r < NREA; ++r) mult[r] = lnm != nullptr ? std::exp(lnm[r]) : 1.0;
  const int N = NSPEC + (so->evolve_T ? 1 : 0);
  std::vector<double> tape, yfin(N);
  const double T0 = *Tgas;
  const int fl = solve_one_(n, Tgas, par, *dt, so, nullptr, mult, &tape, yfin.data());
  if (fl != 0) return fl;
  Problem P;
  P.mult = mult;
  params_from_row(par, P.p);
  P.Tfix = T0;
  P.NEQ = NSPEC;
  if (so->evolve_T) P.iT = P.NEQ++;
  tangent_sweep_(P, tape, dy0, dm, dyf);
  return 0;
}

ORACLE_API int oracle_solve_one(double* n, double* Tgas, const double* par, double dt,
                     const oracle_opts* so, long* stats) {
  return solve_one_(n, Tgas, par, dt, so, stats, nullptr, nullptr, nullptr);
}

// the discrete adjoint, cell by cell: the forward solve with the rate
// multipliers exp(lnm) (lnm one row of NREA broadcast, lnm_stride 0, or
// rows; null: all 0) recording its tape, then the reverse sweep seeded with
// gn[ncell][nspec], gT[ncell]: the gradient of
// sum(gn * n_out) + sum(gT * Tgas_out) with respect to the initial n
// (dn0), Tgas (dT0, evolve_T) and the ln-multipliers (dm[ncell][nrea]).
// n, Tgas are updated as by oracle_solve_cells; a failed cell's gradients
// are 0. Returns the lowest-index failing cell's flag.
ORACLE_API int oracle_adjoint_cells(int ncell, double* n, double* Tgas,
                                    const double* dt, const double* par,
                                    int par_stride, const double* lnm,
                                    int lnm_stride, const double* gn,
                                    const double* gT, int* flags,
                                    const oracle_opts* so, double* dn0,
                                    double* dT0, double* dm, long* stats,
                                    int nthreads) {
  if (ncell < 0 || n == nullptr || Tgas == nullptr || dt == nullptr
      || so == nullptr || gn == nullptr || dn0 == nullptr || dm == nullptr
      || (par_stride != 0 && par_stride != NPAR)
      || (lnm_stride != 0 && lnm_stride != NREA))
    return -1;
  std::vector<int> fl(ncell, 0);
#pragma omp parallel for schedule(dynamic) num_threads(nthreads > 0 ? nthreads : 1)
  for (int c = 0; c < ncell; ++c) {
    const double* row = par + (long)c * par_stride;
    double mult[NREA + 1];
    for (int r = 0; r < NREA; ++r)
      mult[r] = lnm != nullptr ? std::exp(lnm[(long)c * lnm_stride + r]) : 1.0;
    const int N = NSPEC + (so->evolve_T ? 1 : 0);
    double* gmc = dm + (long)c * NREA;
    for (int r = 0; r < NREA; ++r) gmc[r] = 0.0;
    for (int i = 0; i < NSPEC; ++i) dn0[(long)c * NSPEC + i] = 0.0;
    if (dT0 != nullptr) dT0[c] = 0.0;
    if (!(dt[c] > 0.0)) continue;
    std::vector<double> tape, yfin(N), lam_y(N), lam0(N);
    long* sc = stats != nullptr ? stats + (long)c * ORACLE_NSTAT : nullptr;
    const double T0 = Tgas[c];
    fl[c] = solve_one_(n + (long)c * NSPEC, Tgas + c, row, dt[c], so, sc, mult,
                       &tape, yfin.data());
    if (fl[c] != 0) continue;
    Problem P;
    P.mult = mult;
    params_from_row(row, P.p);
    P.Tfix = T0;
    P.NEQ = NSPEC;
    if (so->evolve_T) P.iT = P.NEQ++;
    for (int i = 0; i < NSPEC; ++i) {
      const bool clipped = so->clip_negative && yfin[i] < 0.0;
      lam_y[i] = clipped ? 0.0 : gn[(long)c * NSPEC + i];
    }
    if (P.iT >= 0) lam_y[P.iT] = gT != nullptr ? gT[c] : 0.0;
    adjoint_sweep_(P, tape, lam_y.data(), lam0.data(), gmc);
    for (int i = 0; i < NSPEC; ++i) dn0[(long)c * NSPEC + i] = lam0[i];
    if (dT0 != nullptr && P.iT >= 0) dT0[c] = lam0[P.iT];
  }
  int ret = 0;
  for (int c = 0; c < ncell; ++c) {
    if (flags != nullptr) flags[c] = fl[c];
    if (ret == 0 && fl[c] != 0) ret = fl[c];
  }
  return ret;
}

// many cells (solve_cells.hpp:47-161): the required-parameter rule over
// every cell first, then each cell with dt > 0; the returned flag is the
// lowest-index failing cell's. par: one row (par_stride 0) or rows.
ORACLE_API int oracle_solve_cells(int ncell, double* n, double* Tgas, const double* dt,
                       const double* par, int par_stride, int* flags,
                       const oracle_opts* so, long* stats, int nthreads) {
  if (ncell < 0 || n == nullptr || Tgas == nullptr || dt == nullptr
      || so == nullptr)
    return -1;
  if (par_stride != 0 && par_stride != NPAR) return -1;
  std::vector<double> dflt(NPAR);
  for (int i = 0; i < NPAR; ++i) dflt[i] = param_default(i);
  const double* P = par != nullptr ? par : dflt.data();
  const int ps = par != nullptr ? par_stride : 0;
  bool missing = false;
  for (int c = 0; c < ncell; ++c) {
    Params pc;
    params_from_row(P + (long)c * ps, pc);
    const bool m = params_missing(pc) >= 0;
    if (flags != nullptr) flags[c] = m ? FLAG_PARAM_UNSET : 0;
    missing |= m;
  }
  if (missing) return FLAG_PARAM_UNSET;
  std::vector<int> fl(ncell > 0 ? ncell : 1, 0);
  (void)nthreads;
#pragma omp parallel for schedule(dynamic) num_threads(nthreads > 0 ? nthreads : 1)
  for (int c = 0; c < ncell; ++c) {
    long* sc = stats != nullptr ? stats + (long)c * ORACLE_NSTAT : nullptr;
    if (dt[c] > 0.0) {
      const double* phirow = so->ph_B > 0 ? so->ph_phi + (long)c * so->ph_B
                                          : nullptr;
      fl[c] = solve_one_(n + (long)c * NSPEC, Tgas + c, P + (long)c * ps,
                         dt[c], so, sc, nullptr, nullptr, nullptr, phirow);
    } else {
      fl[c] = 0;
      if (sc != nullptr)
        for (int i = 0; i < ORACLE_NSTAT; ++i) sc[i] = 0;
    }
  }
  int first = 0;
  for (int c = 0; c < ncell; ++c) {
    if (flags != nullptr) flags[c] = fl[c];
    if (first == 0) first = fl[c];
  }
  return first;
}

}  // extern "C"
