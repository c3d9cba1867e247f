// Warp-per-cell CVODE BDF for the large networks: the sparse path.
//
// A network of hundreds of species (Semenov: 655 species, 5,639 reactions)
// cannot keep a cell's state in registers or shared memory: the Nordsieck
// array, the vectors, the rate coefficients and fluxes, the saved Jacobian
// (NNZ_J entries) and the LU factors of I - gamma J in their generation-time
// pattern (NNZ_LU values) take ~570 KB per cell. One warp integrates one
// cell with that state in an HBM workspace slot of its own; the 32 lanes
// split every vector operation (component i on lane i mod 32) and evaluate
// the table-driven forms the emitter writes for this path:
//
//   fluxes     fl[r] = k[r] n[a_r] n[b_r] n[c_r], one lane per reaction
//   rhs        f_i = the reaction-ordered sum of its flux terms, one lane per
//              species (the order of the generated rhs)
//   Jacobian   Jc[e] = the reaction-ordered sum of entry e's terms, one lane
//              per entry, at fixed rates
//   LU         the static-pivot row-form (IKJ) sparse LU: a row at a time,
//              each eliminated row's update split over the lanes, through a
//              dense work row of N doubles
//   solves     the unit-lower and upper triangular sweeps, a row at a time,
//              each row's dot product split over the lanes
//
// The rate coefficients are generated code: the Tgas/parameter-only rates
// (rates_fixed) once per solve, the density-dependent ones (rates_var, the
// grain-surface processes among them) at every rhs, on lane 0.
//
// The CVODE algorithm and every decision are the reference's per-cell
// integrator (runtime/core/cvode/bdf_cell.hpp:490-1547) with its sparse
// linear solver (bdf_cell.hpp:1163-1264) -- the same sequence of operations
// as the CPU restatement (oracle/bdf_oracle.cpp), whose sparse path this
// follows line for line. Fixed Tgas only (the large networks' benchmark
// configuration). Every loop is bounded (max_steps, the per-step failure
// limits, max_restarts, the work queue by the number of cells).
#pragma once

#ifdef KB_LARGE_NETWORK

namespace kbg {

using namespace kbnet;
using namespace kbw;

constexpr int N = NSPEC;
constexpr unsigned FULLM = 0xffffffffu;
// a vector's stride in the workspace: N + the n[N] = 1 slot of the flux
// products, a multiple of 4 doubles
constexpr long NV = ((NSPEC + 1 + 3) / 4) * 4;
constexpr long rnd4(long x) { return ((x + 3) / 4) * 4; }

// one warp's workspace (doubles)
struct WS {
  static constexpr long ZN = 0;                       // zn[L_MAX]
  static constexpr long EWT = ZN + L_MAX * NV;
  static constexpr long Y = EWT + NV;
  static constexpr long ACOR = Y + NV;
  static constexpr long TEMPV = ACOR + NV;
  static constexpr long FTEMP = TEMPV + NV;
  static constexpr long DELTA = FTEMP + NV;
  static constexpr long YR = DELTA + NV;              // the rhs's input (+1 slot)
  static constexpr long TS = YR + NV;                 // the solves' scratch
  static constexpr long WROW = TS + NV;               // the LU's work row
  static constexpr long YOUT = WROW + NV;             // a solve's output
  static constexpr long K = YOUT + NV;                // k[NREA + 1]
  static constexpr long FL = K + rnd4(NREA + 1);      // fl[NREA]
  static constexpr long SJ = FL + rnd4(NREA);         // saved Jacobian
  static constexpr long A = SJ + rnd4(NNZ_J);         // LU values
  static constexpr long SIZE = A + rnd4(NNZ_LU);
};

__device__ __forceinline__ int lane_id() { return threadIdx.x & 31; }

// ---- warp-split vector operations (each ends with the warp's writes
//      visible to all its lanes) ----
__device__ __forceinline__ void v_copy(const double* x, double* z) {
  for (int i = lane_id(); i < N; i += 32) z[i] = x[i];
  __syncwarp();
}
__device__ __forceinline__ void v_scale(double c, const double* x, double* z) {
  for (int i = lane_id(); i < N; i += 32) z[i] = c * x[i];
  __syncwarp();
}
__device__ __forceinline__ void v_const(double c, double* z) {
  for (int i = lane_id(); i < N; i += 32) z[i] = c;
  __syncwarp();
}
__device__ __forceinline__ void v_axpy(double a, const double* x, double* y) {
  const int l = lane_id();
  if (a == 1.0) {
    for (int i = l; i < N; i += 32) y[i] += x[i];
  } else if (a == -1.0) {
    for (int i = l; i < N; i += 32) y[i] -= x[i];
  } else {
    for (int i = l; i < N; i += 32) y[i] += a * x[i];
  }
  __syncwarp();
}
// N_VLinearSum with its special cases (bdf_cell.hpp:296-400)
__device__ void v_lin_sum(double a, const double* x, double b, const double* y,
                          double* z) {
  const int l = lane_id();
  if (b == 1.0 && z == y) { v_axpy(a, x, z); return; }
  if (a == 1.0 && z == x) { v_axpy(b, y, z); return; }
  if (a == 1.0 && b == 1.0) {
    for (int i = l; i < N; i += 32) z[i] = x[i] + y[i];
  } else if ((a == 1.0 && b == -1.0) || (a == -1.0 && b == 1.0)) {
    const bool test = a == 1.0 && b == -1.0;
    const double* v1 = test ? y : x;
    const double* v2 = test ? x : y;
    for (int i = l; i < N; i += 32) z[i] = v2[i] - v1[i];
  } else if (a == 1.0 || b == 1.0) {
    const bool test = a == 1.0;
    const double c = test ? b : a;
    const double* v1 = test ? y : x;
    const double* v2 = test ? x : y;
    for (int i = l; i < N; i += 32) z[i] = (c * v1[i]) + v2[i];
  } else if (a == -1.0 || b == -1.0) {
    const bool test = a == -1.0;
    const double c = test ? b : a;
    const double* v1 = test ? y : x;
    const double* v2 = test ? x : y;
    for (int i = l; i < N; i += 32) z[i] = (c * v1[i]) - v2[i];
  } else if (a == b) {
    for (int i = l; i < N; i += 32) z[i] = a * (x[i] + y[i]);
  } else if (a == -b) {
    for (int i = l; i < N; i += 32) z[i] = a * (x[i] - y[i]);
  } else {
    for (int i = l; i < N; i += 32) z[i] = (a * x[i]) + (b * y[i]);
  }
  __syncwarp();
}
__device__ __forceinline__ double v_wrms(const double* x, const double* w) {
  double s = 0.0;
  for (int i = lane_id(); i < N; i += 32) {
    const double pv = x[i] * w[i];
    s += pv * pv;
  }
  return ssqrt_(warp_sum(s) / N);
}
__device__ __forceinline__ double v_max_norm(const double* x) {
  double m = 0.0;
  for (int i = lane_id(); i < N; i += 32) m = fmax(m, fabs(x[i]));
  return warp_max(m);
}

// ---- the network on the warp ----
struct Net {
  double* ws;
  Params p;
  double T;           // the fixed gas temperature
  const double* atolp;

  // f = F(yv): rates_var on lane 0, then the fluxes and the gather over
  // the lanes; 0, or 1 for a non-finite f (rhs_host_, solve_cell.hpp:
  // 794-813)
  __device__ int rhs(const double* yv, double* f) {
    double* yr = ws + WS::YR;
    double* k = ws + WS::K;
    double* fl = ws + WS::FL;
    const int l = lane_id();
    for (int i = l; i < N; i += 32) yr[i] = yv[i];
    if (l == 0) yr[N] = 1.0;
    __syncwarp();
    if (l == 0) rates_var(T, yr, p, k);
    __syncwarp();
    for (int r = l; r < NREA; r += 32)
      fl[r] = k[r] * yr[d_fx_a[r]] * yr[d_fx_b[r]] * yr[d_fx_c[r]];
    __syncwarp();
    bool ok = true;
    for (int i = l; i < N; i += 32) {
      double a = 0.0;
      for (int t = d_rs_rp[i]; t < d_rs_rp[i + 1]; ++t) {
        if (d_rs_s[t] < 0) a -= fl[d_rs_r[t]];
        else a += fl[d_rs_r[t]];
      }
      f[i] = a;
      ok = ok && isfinite(a);
    }
    __syncwarp();
    return __all_sync(FULLM, ok) ? 0 : 1;
  }
  // the saved Jacobian's entries at yv (the rates at yv)
  __device__ void jac(const double* yv, double* Jc) {
    double* yr = ws + WS::YR;
    double* k = ws + WS::K;
    const int l = lane_id();
    for (int i = l; i < N; i += 32) yr[i] = yv[i];
    if (l == 0) yr[N] = 1.0;
    __syncwarp();
    if (l == 0) rates_var(T, yr, p, k);
    __syncwarp();
    for (int e = l; e < NNZ_J; e += 32) {
      double a = 0.0;
      for (int t = d_jt_rp[e]; t < d_jt_rp[e + 1]; ++t)
        a += d_jt_c[t] * k[d_jt_r[t]] * yr[d_jt_o0[t]] * yr[d_jt_o1[t]];
      Jc[e] = a;
    }
    __syncwarp();
  }
};

// the static-pivot sparse LU of the values a in place (w: a zeroed row of N
// doubles, left zeroed); 0, or the failing row + 1 (a zero or non-finite
// pivot)
__device__ int sp_getrf(double* a, double* w) {
  const int l = lane_id();
  for (int i = 0; i < N; ++i) {
    const int p0 = d_sp_rp[i], p1 = d_sp_rp[i + 1], pd = d_sp_di[i];
    for (int p = p0 + l; p < p1; p += 32) w[d_sp_ci[p]] = a[p];
    __syncwarp();
    for (int p = p0; p < pd; ++p) {
      const int k = d_sp_ci[p];
      const double lk = w[k] / a[d_sp_di[k]];
      const int q1 = d_sp_rp[k + 1];
      for (int q = d_sp_di[k] + 1 + l; q < q1; q += 32) w[d_sp_ci[q]] -= lk * a[q];
      __syncwarp();
      if (l == 0) w[k] = lk;
      __syncwarp();
    }
    const double piv = w[i];
    __syncwarp();
    for (int p = p0 + l; p < p1; p += 32) {
      a[p] = w[d_sp_ci[p]];
      w[d_sp_ci[p]] = 0.0;
    }
    __syncwarp();
    if (piv == 0.0 || !isfinite(piv)) return i + 1;
  }
  return 0;
}
// x = A^-1 b with the factors (b in the species order; t: N doubles of
// scratch); x may be b
__device__ void sp_getrs(const double* a, const double* b, double* t,
                         double* x) {
  const int l = lane_id();
  for (int i = l; i < N; i += 32) t[i] = b[d_sp_perm[i]];
  __syncwarp();
  for (int i = 0; i < N; ++i) {
    double s = 0.0;
    for (int p = d_sp_rp[i] + l; p < d_sp_di[i]; p += 32) s += a[p] * t[d_sp_ci[p]];
    s = warp_sum(s);
    if (l == 0) t[i] -= s;
    __syncwarp();
  }
  for (int i = N - 1; i >= 0; --i) {
    double s = 0.0;
    for (int p = d_sp_di[i] + 1 + l; p < d_sp_rp[i + 1]; p += 32) s += a[p] * t[d_sp_ci[p]];
    s = warp_sum(s);
    if (l == 0) t[i] = (t[i] - s) / a[d_sp_di[i]];
    __syncwarp();
  }
  for (int i = l; i < N; i += 32) x[d_sp_perm[i]] = t[i];
  __syncwarp();
}

struct Stats9 {
  long nst, nfe, nje, nsetups, nni, nnf, netf;
};

// one cell's CVODE (the oracle's Cvode, sparse path, one warp)
struct BigCvode {
  Net& P;
  const SolveOpts& o;
  double* zn[L_MAX];
  double *ewt, *y, *acor, *tempv, *ftemp, *delta, *A, *savedJ, *ts, *wrow;
  Stats9 st;
  long mxstep;
  double tn, h, hin, hprime, hscale, next_h, hu, eta, etamax, etaq;
  double etaqm1, etaqp1, tolsf, saved_tq5;
  double tau[L_MAX + 1], tq[6], l[L_MAX];
  double rl1, gamma, gammap, gamrat, crate, delp, delnrm, acnrm;
  int q, qprime, next_q, qu, L, qwait;
  long nscon, nstlp, nstlj;
  int convfail;
  bool acnrmcur, jcur, nls_jcur;

  __device__ BigCvode(Net& prob, const SolveOpts& opts) : P(prob), o(opts) {
    double* w = prob.ws;
    for (int j = 0; j < L_MAX; j++) zn[j] = w + WS::ZN + j * NV;
    ewt = w + WS::EWT;
    y = w + WS::Y;
    acor = w + WS::ACOR;
    tempv = w + WS::TEMPV;
    ftemp = w + WS::FTEMP;
    delta = w + WS::DELTA;
    ts = w + WS::TS;
    wrow = w + WS::WROW;
    savedJ = w + WS::SJ;
    A = w + WS::A;
    mxstep = o.max_steps == 0 ? 500
             : (o.max_steps < 0 ? KB_MAX_STEPS_CAP : o.max_steps);
    v_const(0.0, wrow);
  }

  __device__ void reinit(double t0, const double* y0, double h_init) {
    tn = t0;
    v_copy(y0, zn[0]);
    q = 1; L = 2; qwait = L;
    etamax = ETA_MAX_FS;
    qu = 0; hu = 0.0; tolsf = 1.0;
    st = Stats9{0, 0, 0, 0, 0, 0, 0};
    nstlp = 0; nscon = 0; next_h = 0.0; next_q = 0;
    hin = h_init;
    nstlj = 0;
    acnrmcur = false; nls_jcur = false; jcur = false;
    saved_tq5 = 0.0;
    for (int i = 0; i <= L_MAX; i++) tau[i] = 0.0;
    eta = 1.0;
  }

  // cvEwtSetSV with one atol for the species (bdf_cell.hpp:689-713)
  __device__ int ewt_set(const double* ycur, double* wt) {
    const double at = o.atol_n;
    bool bad = false;
    for (int i = lane_id(); i < N; i += 32) {
      const double v = (o.rtol * fabs(ycur[i])) + at;
      bad = bad || !(v > 0.0);
      wt[i] = 1.0 / v;
    }
    __syncwarp();
    return __any_sync(FULLM, bad) ? -1 : 0;
  }

  // CVode(tout, NORMAL) (bdf_cell.hpp:566-638); y(tout) into yout
  __device__ int solve(double tout, double* yout, double* tret) {
    int istate = SUCCESS;
    *tret = tn;
    {
      const double tdist = fabs(tout - tn);
      const double tround = UROUND * smax_(fabs(tn), fabs(tout));
      if (tdist == 0.0 || tdist < 2.0 * tround) return TOO_CLOSE;
      if (ewt_set(zn[0], ewt) != 0) return ILL_INPUT;
      const int retval = P.rhs(zn[0], zn[1]);
      st.nfe++;
      if (retval > 0) return FIRST_RHSFUNC_ERR;
      h = hin;
      if (h != 0.0 && (tout - tn) * h < 0.0) return ILL_INPUT;
      if (h == 0.0) {
        const int hflag = hin_(tout);
        if (hflag != SUCCESS) return hflag;
      }
      hscale = h;
      hprime = h;
      v_scale(h, zn[1], zn[1]);
    }
    long nstloc = 0;
    for (;;) {
      next_h = h;
      next_q = q;
      if (st.nst > 0 && ewt_set(zn[0], ewt) != 0) {
        istate = ILL_INPUT; *tret = tn; v_copy(zn[0], yout); break;
      }
      if (mxstep > 0 && nstloc >= mxstep) {
        istate = TOO_MUCH_WORK; *tret = tn; v_copy(zn[0], yout); break;
      }
      const double nrm = v_wrms(zn[0], ewt);
      tolsf = UROUND * nrm;
      if (tolsf > 1.0) {
        istate = TOO_MUCH_ACC; *tret = tn; v_copy(zn[0], yout);
        tolsf *= 2.0;
        break;
      }
      tolsf = 1.0;
      const int kflag = step_();
      if (kflag != SUCCESS) {
        istate = kflag; *tret = tn; v_copy(zn[0], yout); break;
      }
      nstloc++;
      if ((tn - tout) * h >= 0.0) {
        istate = SUCCESS;
        *tret = tout;
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
  __device__ double upper_bound_h0_(double tdist) {
    double* temp1 = tempv;
    double* temp2 = acor;
    for (int i = lane_id(); i < N; i += 32) temp2[i] = fabs(zn[0][i]);
    __syncwarp();
    ewt_set(zn[0], temp1);
    for (int i = lane_id(); i < N; i += 32) temp1[i] = 1.0 / temp1[i];
    __syncwarp();
    v_lin_sum(HUB_FACTOR, temp2, 1.0, temp1, temp1);
    for (int i = lane_id(); i < N; i += 32) temp2[i] = fabs(zn[1][i]);
    __syncwarp();
    for (int i = lane_id(); i < N; i += 32) temp1[i] = temp2[i] / temp1[i];
    __syncwarp();
    const double hub_inv = v_max_norm(temp1);
    double hub = HUB_FACTOR * tdist;
    if (hub * hub_inv > 1.0) hub = 1.0 / hub_inv;
    return hub;
  }
  __device__ int ydd_norm_(double hg, double* yddnrm) {
    v_lin_sum(hg, zn[1], 1.0, zn[0], y);
    const int retval = P.rhs(y, tempv);
    st.nfe++;
    if (retval > 0) return RHSFUNC_RECVR;
    v_lin_sum(1.0 / hg, tempv, -1.0 / hg, zn[1], tempv);
    *yddnrm = v_wrms(tempv, ewt);
    return SUCCESS;
  }

  // cvStep (bdf_cell.hpp:798-822)
  __device__ int step_() {
    int ncf = 0, nef = 0;
    double dsm = 0.0;
    if (st.nst > 0 && hprime != h) {
      if (qprime != q) {
        adjust_order_(qprime - q);
        q = qprime;
        L = q + 1;
        qwait = L;
      }
      rescale_();
    }
    const double saved_t = tn;
    int nflag = FIRST_CALL;
    // bounded: each pass either returns or counts a convergence or an
    // error-test failure, limited by max_conv_fails / max_err_fails
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
    complete_step_();
    prepare_next_step_(dsm);
    etamax = (st.nst <= SMALL_NST) ? ETA_MAX_ES : ETA_MAX_GS;
    v_scale(tq[2], acor, acor);
    return SUCCESS;
  }
  __device__ void adjust_order_(int deltaq) {
    if ((q == 2) && (deltaq != 1)) return;
    if (deltaq == 1) increase_bdf_();
    else if (deltaq == -1) decrease_bdf_();
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
    v_scale(A1, zn[QMAX], zn[L]);
    if (q > 1)
      for (int j = 2; j <= q; j++) v_axpy(l[j], zn[L], zn[j]);
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
    if (q > 2)
      for (int j = 2; j < q; j++) v_axpy(-l[j], zn[q], zn[j]);
  }
  __device__ void rescale_() {
    double c = eta;
    for (int j = 1; j <= q; j++) {
      v_scale(c, zn[j], zn[j]);
      c = eta * c;
    }
    h = hscale * eta;
    next_h = h;
    hscale = h;
    nscon = 0;
  }
  __device__ void predict_() {
    tn += h;
    for (int k = 1; k <= q; k++)
      for (int j = q; j >= k; j--) v_axpy(1.0, zn[j], zn[j - 1]);
  }
  __device__ void restore_(double saved_t) {
    tn = saved_t;
    for (int k = 1; k <= q; k++)
      for (int j = q; j >= k; j--) v_axpy(-1.0, zn[j], zn[j - 1]);
  }
  // cvSet, cvSetBDF, cvSetTqBDF (bdf_cell.hpp:903-954)
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
      xi_inv = h / hsum;
      const double A5 = alpha0 - (1.0 / (q + 1));
      const double A6 = alpha0_hat - xi_inv;
      const double Cppinv = (1.0 - A6 + A5) / A2;
      tq[3] = fabs(Cppinv / (xi_inv * (q + 2) * A5));
    }
    tq[4] = CORTES / tq[2];
    rl1 = 1.0 / l[1];
    gamma = h * rl1;
    if (st.nst == 0) gammap = gamma;
    gamrat = (st.nst > 0) ? gamma / gammap : 1.0;
  }
  // cvNls + the Newton module (bdf_cell.hpp:958-1048)
  __device__ int nls_(int nflag) {
    convfail = ((nflag == FIRST_CALL) || (nflag == PREV_ERR_FAIL))
                   ? NO_FAILURES : FAIL_OTHER;
    bool callSetup = (nflag == PREV_CONV_FAIL) || (nflag == PREV_ERR_FAIL)
                     || (st.nst == 0) || (st.nst >= nstlp + MSBP)
                     || (fabs(gamrat - 1.0) > DGMAX_LSETUP);
    v_const(0.0, acor);
    const double tol = tq[4];
    bool jbad = false;
    long niters = 0, nconvfails = 0;
    int retval;
    // bounded: at most two passes (the retry needs a Jacobian that was not
    // current), each of at most NLS_MAXCOR iterations
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
        v_scale(-1.0, delta, delta);
        sp_getrs(A, delta, ts, delta);
        if (gamrat != 1.0) v_scale(2.0 / (1.0 + gamrat), delta, delta);
        v_lin_sum(1.0, acor, 1.0, delta, acor);
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
        v_const(0.0, acor);
        continue;
      }
      break;
    }
    if (retval != SUCCESS) nconvfails++;
    st.nni += niters;
    st.nnf += nconvfails;
    if (retval != SUCCESS) return retval;
    v_lin_sum(1.0, zn[0], 1.0, acor, y);
    if (!acnrmcur) acnrm = v_wrms(acor, ewt);
    jcur = false;
    return SUCCESS;
  }
  __device__ int residual_() {
    v_lin_sum(1.0, zn[0], 1.0, acor, y);
    const int retval = P.rhs(y, ftemp);
    st.nfe++;
    if (retval > 0) return RHSFUNC_RECVR;
    v_lin_sum(rl1, zn[1], 1.0, acor, delta);
    v_lin_sum(-gamma, ftemp, 1.0, delta, delta);
    return SUCCESS;
  }
  __device__ int conv_test_(int m, double tol) {
    delnrm = v_wrms(delta, ewt);
    if (m > 0) crate = smax_(CRDOWN * crate, delnrm / delp);
    const double dcon = delnrm * smin_(1.0, crate) / tol;
    if (dcon <= 1.0) {
      acnrm = (m == 0) ? delnrm : v_wrms(acor, ewt);
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
    st.nsetups++;
    nls_jcur = jcur;
    gamrat = 1.0;
    gammap = gamma;
    crate = 1.0;
    delnrm = 0.0;
    nstlp = st.nst;
    if (retval < 0) return LSETUP_FAIL;
    if (retval > 0) return NLS_CONV_RECVR;
    return SUCCESS;
  }
  // cvLsSetup with the sparse Newton matrix (bdf_cell.hpp:1069-1130,
  // 1163-1264)
  __device__ int ls_setup_() {
    const double dgamma = fabs((gamma / gammap) - 1.0);
    const bool jbad_ls = (st.nst == 0) || (st.nst >= nstlj + MSBJ)
                         || ((convfail == FAIL_BAD_J) && (dgamma < DGMAX_JBAD))
                         || (convfail == FAIL_OTHER);
    jcur = jbad_ls;
    if (jbad_ls) P.jac(y, savedJ);
    const double c = -gamma;
    const int l0 = lane_id();
    for (int k = l0; k < NNZ_LU; k += 32) A[k] = 0.0;
    __syncwarp();
    for (int e = l0; e < NNZ_J; e += 32) A[d_sp_jpos[e]] = savedJ[e] * c;
    __syncwarp();
    for (int i = l0; i < N; i += 32) A[d_sp_di[i]] += 1.0;
    __syncwarp();
    if (jcur) {
      st.nje++;
      nstlj = st.nst;
    }
    return sp_getrf(A, wrow) > 0 ? LS_LUFACT_FAIL : 0;
  }
  __device__ int handle_nflag_(int* nflagPtr, double saved_t, int* ncfPtr) {
    const int nflag = *nflagPtr;
    if (nflag == SUCCESS) return DO_ERROR_TEST;
    restore_(saved_t);
    if (nflag < 0) {
      if (nflag == LSETUP_FAIL) return LSETUP_FAIL;
      if (nflag == LSOLVE_FAIL) return LSOLVE_FAIL;
      if (nflag == RHSFUNC_FAIL) return RHSFUNC_FAIL;
      return NLS_FAIL;
    }
    (*ncfPtr)++;
    etamax = 1.0;
    if ((fabs(h) <= 0.0) || (*ncfPtr == o.max_conv_fails)) {
      if (nflag == NLS_CONV_RECVR) return CONV_FAILURE;
      if (nflag == RHSFUNC_RECVR) return REPTD_RHSFUNC_ERR;
    }
    eta = smax_(ETA_CF, 0.0 / fabs(h));
    *nflagPtr = PREV_CONV_FAIL;
    rescale_();
    return PREDICT_AGAIN;
  }
  __device__ int do_error_test_(int* nflagPtr, double saved_t, int* nefPtr,
                                double* dsmPtr) {
    const double dsm = acnrm * tq[2];
    *dsmPtr = dsm;
    if (dsm <= 1.0) return SUCCESS;
    (*nefPtr)++;
    st.netf++;
    *nflagPtr = PREV_ERR_FAIL;
    restore_(saved_t);
    if ((fabs(h) <= 0.0) || (*nefPtr == o.max_err_fails)) return ERR_FAILURE;
    etamax = 1.0;
    if (*nefPtr <= MXNEF1) {
      eta = 1.0 / (pow(BIAS2 * dsm, 1.0 / L) + ADDON);
      eta = smax_(ETA_MIN_EF, smax_(eta, 0.0 / fabs(h)));
      if (*nefPtr >= SMALL_NEF) eta = smin_(eta, ETA_MAX_EF);
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
    const int retval = P.rhs(zn[0], tempv);
    st.nfe++;
    if (retval > 0) return UNREC_RHSFUNC_ERR;
    v_scale(h, tempv, zn[1]);
    return TRY_AGAIN;
  }
  __device__ void complete_step_() {
    st.nst++;
    nscon++;
    hu = h;
    qu = q;
    for (int i = q; i >= 2; i--) tau[i] = tau[i - 1];
    if ((q == 1) && (st.nst > 1)) tau[2] = tau[1];
    tau[1] = h;
    for (int j = 0; j <= q; j++) v_axpy(l[j], acor, zn[j]);
    qwait--;
    if ((qwait == 1) && (q != QMAX)) {
      v_copy(acor, zn[QMAX]);
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
      return;
    }
    qwait = 2;
    etaqm1 = 0.0;
    if (q > 1) {
      const double ddn = v_wrms(zn[q], ewt) * tq[1];
      etaqm1 = 1.0 / (pow(BIAS1 * ddn, 1.0 / q) + ADDON);
    }
    etaqp1 = 0.0;
    if (q != QMAX && saved_tq5 != 0.0) {
      const double rr = h / tau[2];
      double prod = 1.0;
      for (int i = 1; i <= L; i++) prod *= rr;
      const double cquot = (tq[5] / saved_tq5) * prod;
      v_lin_sum(-cquot, zn[QMAX], 1.0, acor, tempv);
      const double dup = v_wrms(tempv, ewt) * tq[3];
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
      v_copy(acor, zn[QMAX]);
    }
    set_eta_();
  }
  __device__ void set_eta_() {
    if ((eta > ETA_MIN_FX) && (eta < ETA_MAX_FX)) {
      eta = 1.0;
      hprime = h;
      return;
    }
    if (eta >= ETA_MAX_FX) eta = smin_(eta, etamax);
    else eta = smax_(eta, ETA_MIN);
    hprime = h * eta;
    if (qprime < q) nscon = 0;
  }
  __device__ void get_dky_(double t, double* dky) {
    const double sv = (t - tn) / h;
    for (int j = q; j >= 0; j--) {
      double c = 1.0;
      for (int i = 0; i < j; i++) c *= sv;
      if (j == q) v_scale(c, zn[j], dky);
      else v_axpy(c, zn[j], dky);
    }
  }
};

}  // namespace kbg

#endif  // KB_LARGE_NETWORK
