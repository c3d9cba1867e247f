// Block-per-cell CVODE BDF for the large networks: the sparse path.
//
// A network of hundreds of species (Semenov: 655 species, 5,639 reactions)
// cannot keep a cell's state in registers: the Nordsieck array, the vectors,
// the rate coefficients and fluxes, the saved Jacobian (NNZ_J entries) and
// the LU factors of I - gamma J in their generation-time pattern (NNZ_LU
// values) take ~600 KB per cell. One thread block of NT threads integrates
// one cell, one block per SM over a persistent work queue; the cell's state
// lives in a global-memory workspace slot of its block (148 slots, ~90 MB,
// mostly L2-resident), and the hot part of the Newton matrix in shared
// memory:
//
//   vectors    component i on thread i mod NT; element-wise operations need
//              no barrier (each thread touches its own components), every
//              operation that reads other threads' components (rhs, Jacobian,
//              setup, solve, reductions) is bracketed by block barriers
//   rates      the Tgas/parameter-only rates once per solve (one generated
//              part per thread, RPART parts); the density-dependent ones (the
//              grain-surface processes) depend on the state only through the
//              water-ice coverage fi (affinely) and the H-nuclei density
//              hnuc (linearly), so with Tgas and Tdust fixed the generated
//              code runs at three points per solve (fi = 0, fi = 1, hnuc = 1)
//              and every rhs forms k = e0 (1 - fi) + e1 fi + eh hnuc, a
//              thread per rate (networks whose rates read the densities
//              otherwise, BK_VAR_AFFINE = 0, run the generated parts at every
//              rhs)
//   fluxes     fl[r] = k[r] n[a_r] n[b_r] n[c_r], a thread per reaction
//   rhs        f_i = the sum of its flux terms in reaction order, in chunks
//              of at most 16 terms (a thread per chunk, then per species the
//              sum of its chunks in order: the hub species' hundreds of terms
//              spread over the block)
//   Jacobian   Jc[e] = the reaction-ordered sum of entry e's terms, a thread
//              per entry, at fixed rates
//   LU         the static-pivot LU of the generation-time order, split where
//              the minimum-degree order leaves a dense trailing block: the
//              first BK_M rows sparse (factored level by level -- the rows of
//              a level eliminate only with rows of lower levels -- a thread
//              per row on wide levels, a warp per row through a shared-memory
//              work row on narrow ones), then the last BK_D rows' sparse
//              columns pivot by pivot (the Schur complement into S, every
//              row and U entry of a pivot in parallel), then the dense block
//              S (BK_D x BK_D,
//              shared memory) by a right-looking LU in panels of 16 columns
//              with register-tiled rank-16 updates
//   solves     the same split: sparse rows by level, the dense block by
//              32-row diagonal blocks (a warp with shuffles) and block
//              updates, sparse rows back by backward level
//
// The CVODE algorithm and every decision are the reference's per-cell
// integrator (runtime/core/cvode/bdf_cell.hpp:490-1547) with its sparse
// linear solver (bdf_cell.hpp:1163-1264): the sequence of operations of the
// CPU restatement (oracle/bdf_oracle.cpp, sparse path), whose IKJ row LU
// this factorization equals up to the order of its roundings (same pivots,
// same pattern, static pivoting). Tgas fixed (the large networks'
// benchmark configuration) or evolved: then the state's last component
// (the vectors' lengths from neq()), the Newton matrix bordered by its
// Tgas row and column (bdf_cell.hpp:1192-1264 with one border equation),
// on networks without thermal processes, whose dT/dt, Tgas row and corner
// are identically zero. Every loop is bounded (max_steps, the per-step
// failure limits, max_restarts, the work queue by the number of cells).
#pragma once

#ifdef KB_LARGE_NETWORK

namespace kbg {

using namespace kbnet;
using namespace kbw;

constexpr int N = NSPEC;
constexpr int NT = 256;  // threads of a cell's block
constexpr int NWARP = NT / 32;
constexpr unsigned FULLM = 0xffffffffu;
static_assert(RPART <= NT, "one rate part per thread");
static_assert(BK_D <= NT, "a thread per dense row in the Schur steps");
// a vector's stride: N + the n[N] = 1 slot of the flux products, a
// multiple of 4 doubles
constexpr long NV = ((NSPEC + 1 + 3) / 4) * 4;
constexpr long rnd4(long x) { return ((x + 3) / 4) * 4; }

// a cell's workspace in global memory (doubles)
struct WS {
  static constexpr long ZN = 0;                       // zn[L_MAX]
  static constexpr long EWT = ZN + L_MAX * NV;
  static constexpr long Y = EWT + NV;
  static constexpr long ACOR = Y + NV;
  static constexpr long TEMPV = ACOR + NV;
  static constexpr long FTEMP = TEMPV + NV;
  static constexpr long DELTA = FTEMP + NV;
  static constexpr long YOUT = DELTA + NV;            // a solve's output
  static constexpr long K = YOUT + NV;                // k[NREA + 1]
  static constexpr long FL = K + rnd4(NREA + 1);      // fl[NREA]
  static constexpr long SJ = FL + rnd4(NREA);         // saved Jacobian
  static constexpr long CP = SJ + rnd4(NNZ_J);        // rhs chunk sums
  static constexpr long VE = CP + rnd4(NCHUNK);       // e0, e1, eh [BK_NVAR]
  static constexpr long A = VE + 3 * rnd4(BK_NVAR);   // LU values
  // an evolved Tgas: the Jacobian's Tgas column over the species (B), and
  // the full rhs at Tgas +- h for its central differences
  static constexpr long BT = A + rnd4(NNZ_LU);
  static constexpr long FP = BT + NV;
  static constexpr long FM = FP + NV;
  static constexpr long SIZE = FM + NV;
};

// the block's shared memory (doubles)
struct SM {
  static constexpr int S = 0;                         // dense block [D][LD]
  static constexpr int T = S + BK_D * BK_LD;          // the solves' vector
  static constexpr int RPIV = T + (int)NV;            // 1 / pivot, per row
  static constexpr int YR = RPIV + (int)NV;           // the rhs input (+1)
  static constexpr int RED = YR + (int)NV;            // reductions
  static constexpr int MISC = RED + NWARP;            // the work queue's cell,
                                                      // the state's length
  static constexpr int SIZE = MISC + 2;
};
constexpr size_t SMEM_BYTES = SM::SIZE * sizeof(double);
static_assert(SMEM_BYTES <= 227 * 1024, "the dense block must fit shared memory");

__device__ __forceinline__ double* smem() {
  extern __shared__ double kbg_smem[];
  return kbg_smem;
}

// block reductions: every thread gets the same value (the warps' partial
// results summed in warp order)
__device__ __forceinline__ double blk_sum(double v) {
  double* red = smem() + SM::RED;
  v = warp_sum(v);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double s = 0.0;
  for (int w = 0; w < NWARP; ++w) s += red[w];
  __syncthreads();
  return s;
}
__device__ __forceinline__ double blk_max(double v) {
  double* red = smem() + SM::RED;
  v = warp_max(v);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double s = red[0];
  for (int w = 1; w < NWARP; ++w) s = fmax(s, red[w]);
  __syncthreads();
  return s;
}

// the integrator's state length: the species, and Tgas (component N) when
// it is evolved (set by the cell's first thread, then a barrier)
__device__ __forceinline__ int neq() { return (int)smem()[SM::MISC + 1]; }
__device__ __forceinline__ void set_neq(int n) {
  if (threadIdx.x == 0) smem()[SM::MISC + 1] = (double)n;
}

// ---- element-wise vector operations (component i on thread i mod NT) ----
// KBG_FOR: the species; KBG_VFOR: the integrator's state
#define KBG_FOR(i) for (int i = threadIdx.x; i < N; i += NT)
#define KBG_VFOR(i) for (int i = threadIdx.x, kbg_n_ = neq(); i < kbg_n_; i += NT)
__device__ __forceinline__ void v_copy(const double* x, double* z) {
  KBG_VFOR(i) z[i] = x[i];
}
__device__ __forceinline__ void v_scale(double c, const double* x, double* z) {
  KBG_VFOR(i) z[i] = c * x[i];
}
__device__ __forceinline__ void v_const(double c, double* z) {
  KBG_VFOR(i) z[i] = c;
}
__device__ __forceinline__ void v_axpy(double a, const double* x, double* y) {
  if (a == 1.0) {
    KBG_VFOR(i) y[i] += x[i];
  } else if (a == -1.0) {
    KBG_VFOR(i) y[i] -= x[i];
  } else {
    KBG_VFOR(i) y[i] += a * x[i];
  }
}
// N_VLinearSum with its special cases (bdf_cell.hpp:296-400)
__device__ void v_lin_sum(double a, const double* x, double b, const double* y,
                          double* z) {
  if (b == 1.0 && z == y) { v_axpy(a, x, z); return; }
  if (a == 1.0 && z == x) { v_axpy(b, y, z); return; }
  if (a == 1.0 && b == 1.0) {
    KBG_VFOR(i) z[i] = x[i] + y[i];
  } else if ((a == 1.0 && b == -1.0) || (a == -1.0 && b == 1.0)) {
    const bool test = a == 1.0 && b == -1.0;
    const double* v1 = test ? y : x;
    const double* v2 = test ? x : y;
    KBG_VFOR(i) z[i] = v2[i] - v1[i];
  } else if (a == 1.0 || b == 1.0) {
    const bool test = a == 1.0;
    const double c = test ? b : a;
    const double* v1 = test ? y : x;
    const double* v2 = test ? x : y;
    KBG_VFOR(i) z[i] = (c * v1[i]) + v2[i];
  } else if (a == -1.0 || b == -1.0) {
    const bool test = a == -1.0;
    const double c = test ? b : a;
    const double* v1 = test ? y : x;
    const double* v2 = test ? x : y;
    KBG_VFOR(i) z[i] = (c * v1[i]) - v2[i];
  } else if (a == b) {
    KBG_VFOR(i) z[i] = a * (x[i] + y[i]);
  } else if (a == -b) {
    KBG_VFOR(i) z[i] = a * (x[i] - y[i]);
  } else {
    KBG_VFOR(i) z[i] = (a * x[i]) + (b * y[i]);
  }
}
__device__ __forceinline__ double v_wrms(const double* x, const double* w) {
  double s = 0.0;
  KBG_VFOR(i) {
    const double pv = x[i] * w[i];
    s += pv * pv;
  }
  return ssqrt_(blk_sum(s) / neq());
}
__device__ __forceinline__ double v_max_norm(const double* x) {
  double m = 0.0;
  KBG_VFOR(i) m = fmax(m, fabs(x[i]));
  return blk_max(m);
}

// ---- the network on the block ----
struct Net {
  double* ws;
  Params p;
  double T;  // the fixed gas temperature

  static constexpr long VSTR = rnd4(BK_NVAR);

  // yr (shared memory) = yv with the slot yr[N] = 1, and the H-nuclei
  // density of yv (a reduction, so it ends with yr visible to the block)
  __device__ double load_state(const double* yv) {
    double* yr = smem() + SM::YR;
    double h = 0.0;
    KBG_FOR(i) {
      const double v = yv[i];
      yr[i] = v;
      h += v * d_bk_hnuc[i];
    }
    if (threadIdx.x == 0) yr[N] = 1.0;
    return blk_sum(h);
  }
  // the density-dependent rates at the state in yr (hnuc its H-nuclei
  // density)
  __device__ void rates_at(double hnuc) {
    double* k = ws + WS::K;
    if (BK_VAR_AFFINE) {
      const double fi = bk_ice_cover(smem() + SM::YR, p);
      const double* e0 = ws + WS::VE;
      const double* e1 = e0 + VSTR;
      const double* eh = e1 + VSTR;
      for (int j = threadIdx.x; j < BK_NVAR; j += NT)
        k[d_bk_var[j]] = e0[j] * (1.0 - fi) + e1[j] * fi + eh[j] * hnuc;
    } else if (threadIdx.x < RPART) {
      rates_var_part(threadIdx.x, T, smem() + SM::YR, p, hnuc, k);
    }
    __syncthreads();
  }
  // the density-dependent rates' three points of this solve (e0: fi = 0,
  // e1: fi = 1, eh: the change at hnuc = 1), from the generated code at the
  // state y0 with its ice density replaced. Starts and ends with a barrier.
  __device__ void prepare_var(const double* y0) {
    if (!BK_VAR_AFFINE) return;
    double* yr = smem() + SM::YR;
    double* k = ws + WS::K;
    double* e0 = ws + WS::VE;
    double* e1 = e0 + VSTR;
    double* eh = e1 + VSTR;
    __syncthreads();
    KBG_FOR(i) yr[i] = y0[i];
    for (int pt = 0; pt < 3; ++pt) {
      __syncthreads();
      if (threadIdx.x == 0) {
        yr[N] = 1.0;
        bk_set_ice(yr, p, pt == 1);
      }
      __syncthreads();
      if (threadIdx.x < RPART)
        rates_var_part(threadIdx.x, T, yr, p, pt == 2 ? 1.0 : 0.0, k);
      __syncthreads();
      double* e = pt == 0 ? e0 : (pt == 1 ? e1 : eh);
      for (int j = threadIdx.x; j < BK_NVAR; j += NT) {
        const double v = k[d_bk_var[j]];
        e[j] = pt == 2 ? v - e0[j] : v;
      }
    }
    __syncthreads();
  }
  // f = F(yv); 0, or 1 for a non-finite f (rhs_host_, solve_cell.hpp:
  // 794-813). Starts and ends with a block barrier.
  __device__ int rhs(const double* yv, double* f) {
    __syncthreads();
    rates_at(load_state(yv));
    return sums(f);
  }
  // f over the species from the rates in k and the state in yr, and, with
  // an evolved Tgas, f[N] = dT/dt: identically zero on the networks whose
  // large path evolves Tgas (no thermal processes: the generated
  // thermal_dTdt is (gamma - 1) (0 - 0) / (k_B n_tot)). Ends with a barrier.
  __device__ int sums(double* f) {
    const double* yr = smem() + SM::YR;
    const double* k = ws + WS::K;
    double* fl = ws + WS::FL;
    for (int r = threadIdx.x; r < NREA; r += NT)
      fl[r] = k[r] * yr[d_fx_a[r]] * yr[d_fx_b[r]] * yr[d_fx_c[r]];
    __syncthreads();
    double* cp = ws + WS::CP;
    for (int c = threadIdx.x; c < NCHUNK; c += NT) {
      const int t0 = d_ck_t[c], t1 = d_ck_t[c + 1];
      double v[16];
#pragma unroll
      for (int x = 0; x < 16; ++x) v[x] = t0 + x < t1 ? fl[d_rs_r[t0 + x]] : 0.0;
      double a = 0.0;
#pragma unroll
      for (int x = 0; x < 16; ++x)
        if (t0 + x < t1) {
          if (d_rs_s[t0 + x] < 0) a -= v[x];
          else a += v[x];
        }
      cp[c] = a;
    }
    __syncthreads();
    bool ok = true;
    KBG_FOR(i) {
      double a = 0.0;
      for (int c = d_ck_rp[i]; c < d_ck_rp[i + 1]; ++c) a += cp[c];
      f[i] = a;
      ok = ok && isfinite(a);
    }
    if (neq() > N && threadIdx.x == N % NT) f[N] = 0.0;
    return __syncthreads_and(ok) ? 0 : 1;
  }
  // the Tgas column of the evolved-Tgas Jacobian over the species
  // (jac_assemble_, solve_cell.hpp:1053-1066): central differences of the
  // full rhs at Tgas +- h, h = max(1e-6 |Tgas|, 1e-8), every rate
  // re-evaluated there (the generated parts; the affine forms of the
  // density-dependent rates hold at this solve's Tgas only), into B. The
  // Tgas row and corner are the difference quotients of a dT/dt that is
  // identically zero: zero. The rates at this solve's Tgas are restored.
  // Starts and ends with a block barrier.
  __device__ void jac_tgas(const double* yv, double* B) {
    double* fp = ws + WS::FP;
    double* fm = ws + WS::FM;
    double* k = ws + WS::K;
    __syncthreads();
    const double Ty = yv[N];
    const double h = fmax(1e-6 * fabs(Ty), 1e-8);
    for (int side = 0; side < 2; ++side) {
      const double Ts = fmin(fmax(side == 0 ? Ty + h : Ty - h, p.Tcmb), 1e9);
      const double hn = load_state(yv);
      if (threadIdx.x < RPART) {
        rates_fixed_part(threadIdx.x, Ts, smem() + SM::YR, p, hn, k);
        rates_var_part(threadIdx.x, Ts, smem() + SM::YR, p, hn, k);
      }
      __syncthreads();
      sums(side == 0 ? fp : fm);
    }
    KBG_FOR(i) B[i] = (fp[i] - fm[i]) / (2.0 * h);
    const double hn = load_state(yv);
    if (threadIdx.x < RPART)
      rates_fixed_part(threadIdx.x, T, smem() + SM::YR, p, hn, k);
    __syncthreads();
  }
  // the saved Jacobian's entries at yv (the rates at yv)
  __device__ void jac(const double* yv, double* Jc) {
    __syncthreads();
    const double* yr = smem() + SM::YR;
    const double* k = ws + WS::K;
    rates_at(load_state(yv));
    for (int e = threadIdx.x; e < NNZ_J; e += NT) {
      double a = 0.0;
      for (int t = d_jt_rp[e]; t < d_jt_rp[e + 1]; ++t)
        a += d_jt_c[t] * k[d_jt_r[t]] * yr[d_jt_o0[t]] * yr[d_jt_o1[t]];
      Jc[e] = a;
    }
    __syncthreads();
  }
};

// ---- the factorization ----
// row i's elimination with the (final) rows k of its L entries [p0, p1):
// l = a(i, k) / a(k, k), then a(i, j) -= l a(k, j) over row k's U entries
// (bk_tgt: the places of the (i, j)); by one thread. The updates of one L
// entry go in batches of 8, every load of a batch before its stores, so a
// batch costs one memory round trip.
__device__ __forceinline__ void elim_thread(int p0, int p1, double* A,
                                            double* S, const double* rpiv) {
  for (int p = p0; p < p1; ++p) {
    const int k = d_sp_ci[p];
    const double l = A[p] * rpiv[k];
    A[p] = l;
    const int q0 = d_sp_di[k] + 1, q1 = d_sp_rp[k + 1];
    const int* tg = d_bk_tgt + d_bk_uoff[p] - q0;
    for (int qb = q0; qb < q1; qb += 8) {
      int t[8];
      double u[8], a[8];
#pragma unroll
      for (int x = 0; x < 8; ++x) {
        const bool in = qb + x < q1;
        t[x] = in ? tg[qb + x] : 0;
        u[x] = in ? A[qb + x] : 0.0;
      }
#pragma unroll
      for (int x = 0; x < 8; ++x)
        a[x] = qb + x < q1 ? (t[x] >= 0 ? A[t[x]] : S[-1 - t[x]]) : 0.0;
#pragma unroll
      for (int x = 0; x < 8; ++x) {
        if (qb + x < q1) {
          const double v = a[x] - l * u[x];
          if (t[x] >= 0) A[t[x]] = v;
          else S[-1 - t[x]] = v;
        }
      }
    }
  }
}
// sparse row i's elimination by a warp through a dense work row w (shared
// memory, zero on entry and on exit): the row scattered into w by column,
// each L entry's update applied to w over the lanes, then the row gathered
// back; returns the pivot. The L entries run as a software pipeline: while
// entry p is applied, the U row of entry p + 1 is loaded into registers and
// the place of entry p + 2's U row (two dependent table loads: its pivot
// row, then the row's range) is looked up, so the chain of L entries waits
// for one L2 round trip per entry at most, not three
__device__ double elim_warp(int i, double* A, const double* rpiv, double* w) {
  const int lane = threadIdx.x & 31;
  const int p0 = d_sp_rp[i], pd = d_sp_di[i], p1 = d_sp_rp[i + 1];
  for (int p = p0 + lane; p < p1; p += 32) w[d_sp_ci[p]] = A[p];
  __syncwarp();
  constexpr int UW = 6;  // U-row entries in registers per lane
  double u[UW];
  int c[UW];
  auto where = [&](int p, int& k, int& q0, int& q1) {
    k = d_sp_ci[p];
    q0 = d_sp_di[k] + 1;
    q1 = d_sp_rp[k + 1];
  };
  auto fetch = [&](int q0, int q1) {
#pragma unroll
    for (int s = 0; s < UW; ++s) {
      const int q = q0 + lane + 32 * s;
      c[s] = q < q1 ? d_sp_ci[q] : -1;
      u[s] = q < q1 ? A[q] : 0.0;
    }
  };
  int kc = 0, qc0 = 0, qc1 = 0;  // the current entry's pivot row, U range
  int kn = 0, qn0 = 0, qn1 = 0;  // the next entry's
  if (p0 < pd) {
    where(p0, kc, qc0, qc1);
    fetch(qc0, qc1);
  }
  if (p0 + 1 < pd) where(p0 + 1, kn, qn0, qn1);
  for (int p = p0; p < pd; ++p) {
    const int k = kc, q0 = qc0, q1 = qc1;
    const double l = w[k] * rpiv[k];
    double uc[UW];
    int cc[UW];
#pragma unroll
    for (int s = 0; s < UW; ++s) {
      uc[s] = u[s];
      cc[s] = c[s];
    }
    if (p + 1 < pd) {
      fetch(qn0, qn1);
      kc = kn;
      qc0 = qn0;
      qc1 = qn1;
    }
    if (p + 2 < pd) where(p + 2, kn, qn0, qn1);
#pragma unroll
    for (int s = 0; s < UW; ++s)
      if (cc[s] >= 0) w[cc[s]] -= l * uc[s];
    for (int q = q0 + 32 * UW + lane; q < q1; q += 32) w[d_sp_ci[q]] -= l * A[q];
    __syncwarp();
    if (lane == 0) w[k] = l;
    __syncwarp();
  }
  const double piv = w[i];
  __syncwarp();
  for (int p = p0 + lane; p < p1; p += 32) {
    const int j = d_sp_ci[p];
    A[p] = w[j];
    w[j] = 0.0;
  }
  __syncwarp();
  return piv;
}

// the dense rows' sparse columns (the Schur complement into S), by levels
// of the right-looking pivot steps: a level's steps need no result of each
// other (a step follows every step that writes one of its L entries), so
// level L first turns all its L entries into multipliers l = a(i, k) /
// a(k, k) (a thread per entry), then updates all its targets (a thread per
// target, a(i, j) -= l a(k, j) over the target's contributions in step
// order): two barriers per level instead of two per pivot step. Per target
// the operations are the row-wise (IKJ) elimination's, in its order except
// where two levels' steps write the same target
__device__ void schur(double* A, double* S, const double* rpiv) {
  const int tid = threadIdx.x;
  for (int L = 0; L < BK_NSL; ++L) {
    const int e1 = d_bkl_lp[L + 1];
    for (int e = d_bkl_lp[L] + tid; e < e1; e += NT) {
      const int p = d_bkl_lpl[e];
      A[p] = A[p] * rpiv[d_bkl_lk[e]];
    }
    __syncthreads();
    const int t1 = d_bkl_tp[L + 1];
    for (int t = d_bkl_tp[L] + tid; t < t1; t += NT) {
      const int code = d_bkl_tgt[t];
      double v = code >= 0 ? A[code] : S[-1 - code];
      const int c1 = d_bkl_cp[t + 1];
      for (int c = d_bkl_cp[t]; c < c1; ++c) {
        const double w = A[d_bkl_cl[c]] * A[d_bkl_cu[c]];
        v -= w;
      }
      if (code >= 0) A[code] = v;
      else S[-1 - code] = v;
    }
    __syncthreads();
  }
}

constexpr int PB = 16;  // the dense LU's panel width

// the right-looking LU of the dense block S (no pivoting); rpd[c] = 1 /
// its pivot c; true for a zero or non-finite pivot
__device__ bool dense_lu(double* S, double* rpd) {
  constexpr int D = BK_D, LD = BK_LD;
  const int tid = threadIdx.x;
  bool bad = false;
  for (int c0 = 0; c0 < D; c0 += PB) {
    const int pe = c0 + PB < D ? c0 + PB : D;
    // the panel's columns [c0, pe): a thread per row below each pivot
    for (int c = c0; c < pe; ++c) {
      const double piv = S[c * LD + c];
      const double rc = 1.0 / piv;
      if (tid == 0) {
        rpd[c] = rc;
        bad = bad || piv == 0.0 || !isfinite(piv);
      }
      for (int i = c + 1 + tid; i < D; i += NT) {
        double* Si = S + i * LD;
        const double l = Si[c] * rc;
        Si[c] = l;
        for (int j = c + 1; j < pe; ++j) Si[j] -= l * S[c * LD + j];
      }
      __syncthreads();
    }
    if (pe == D) break;
    const int w = pe - c0;
    // the panel's rows beyond it: U12 = L11^-1 A12, a thread per column
    for (int j = pe + tid; j < D; j += NT) {
      double u[PB];
#pragma unroll
      for (int r = 0; r < PB; ++r) u[r] = r < w ? S[(c0 + r) * LD + j] : 0.0;
#pragma unroll
      for (int r = 1; r < PB; ++r) {
        if (r < w) {
          double s = u[r];
#pragma unroll
          for (int rr = 0; rr < r; ++rr) s -= S[(c0 + r) * LD + c0 + rr] * u[rr];
          u[r] = s;
        }
      }
#pragma unroll
      for (int r = 1; r < PB; ++r)
        if (r < w) S[(c0 + r) * LD + j] = u[r];
    }
    __syncthreads();
    // the trailing block [pe, D)^2 -= L21 U12, 4 x 4 tiles per thread
    const int R = D - pe, MT = (R + 3) / 4;
    for (int t = tid; t < MT * MT; t += NT) {
      const int i0 = pe + (t / MT) * 4, j0 = pe + (t % MT) * 4;
      double acc[4][4];
#pragma unroll
      for (int x = 0; x < 4; ++x)
#pragma unroll
        for (int y = 0; y < 4; ++y) acc[x][y] = 0.0;
      for (int kk = c0; kk < pe; ++kk) {
        double a[4], b[4];
#pragma unroll
        for (int x = 0; x < 4; ++x) a[x] = i0 + x < D ? S[(i0 + x) * LD + kk] : 0.0;
#pragma unroll
        for (int y = 0; y < 4; ++y) b[y] = j0 + y < D ? S[kk * LD + j0 + y] : 0.0;
#pragma unroll
        for (int x = 0; x < 4; ++x)
#pragma unroll
          for (int y = 0; y < 4; ++y) acc[x][y] += a[x] * b[y];
      }
#pragma unroll
      for (int x = 0; x < 4; ++x)
#pragma unroll
        for (int y = 0; y < 4; ++y)
          if (i0 + x < D && j0 + y < D) S[(i0 + x) * LD + j0 + y] -= acc[x][y];
    }
    __syncthreads();
  }
  return bad;
}

// the LU of the Newton matrix: A (sparse rows and the dense rows' sparse
// columns) and S (the dense block); rpiv[i] = 1 / pivot i. 0, or 1 for a
// zero or non-finite pivot. Starts and ends with a block barrier.
__device__ int block_lu(double* A) {
  double* S = smem() + SM::S;
  double* rpiv = smem() + SM::RPIV;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  bool bad = false;
  // the narrow levels' two work rows: the solve vector and the rhs input,
  // both free during the factorization
  double* wrow = smem() + (warp == 0 ? SM::T : SM::YR);
  __syncthreads();
  for (int i = tid; i < (int)NV; i += NT) {
    smem()[SM::T + i] = 0.0;
    smem()[SM::YR + i] = 0.0;
  }
  __syncthreads();
  for (int L = 0; L < BK_NLF; ++L) {
    const int r0 = d_bk_flp[L], r1 = d_bk_flp[L + 1];
    if (r1 - r0 >= 16) {  // wide: a thread per row
      for (int r = r0 + tid; r < r1; r += NT) {
        const int i = d_bk_frow[r];
        elim_thread(d_sp_rp[i], d_sp_di[i], A, S, rpiv);
        const double piv = A[d_sp_di[i]];
        rpiv[i] = 1.0 / piv;
        bad = bad || piv == 0.0 || !isfinite(piv);
      }
    } else if (warp < 2) {  // narrow: warps 0 and 1, a row at a time each
      for (int r = r0 + warp; r < r1; r += 2) {
        const int i = d_bk_frow[r];
        const double piv = elim_warp(i, A, rpiv, wrow);
        if (lane == 0) {
          rpiv[i] = 1.0 / piv;
          bad = bad || piv == 0.0 || !isfinite(piv);
        }
        __syncwarp();
      }
    }
    __syncthreads();
  }
  schur(A, S, rpiv);
  bad = dense_lu(S, rpiv + BK_M) || bad;
  return __syncthreads_or(bad) ? 1 : 0;
}

// ---- the solves ----
// x = L22^-1 x, L22 the dense block's unit lower factor
__device__ void dense_fwd(const double* S, double* x) {
  constexpr int D = BK_D, LD = BK_LD;
  const int tid = threadIdx.x, lane = tid & 31;
  for (int b0 = 0; b0 < D; b0 += 32) {
    const int be = b0 + 32 < D ? b0 + 32 : D;
    if (tid < 32) {
      const int i = b0 + lane;
      double v = i < be ? x[i] : 0.0;
      for (int j = b0; j < be - 1; ++j) {
        const double xj = __shfl_sync(FULLM, v, j - b0);
        if (i > j && i < be) v -= S[i * LD + j] * xj;
      }
      if (i < be) x[i] = v;
    }
    __syncthreads();
    if (be < D) {
      for (int i = be + tid; i < D; i += NT) {
        double s = 0.0;
        for (int j = b0; j < be; ++j) s += S[i * LD + j] * x[j];
        x[i] -= s;
      }
      __syncthreads();
    }
  }
}
// x = U22^-1 x, U22 the dense block's upper factor (rpd: 1 / its diagonal)
__device__ void dense_bwd(const double* S, const double* rpd, double* x) {
  constexpr int D = BK_D, LD = BK_LD;
  const int tid = threadIdx.x, lane = tid & 31;
  for (int be = D; be > 0; be -= 32) {
    const int b0 = be - 32 > 0 ? be - 32 : 0;
    if (tid < 32) {
      const int i = b0 + lane;
      double v = i < be ? x[i] : 0.0;
      for (int j = be - 1; j >= b0; --j) {
        if (i == j) v *= rpd[j];
        const double xj = __shfl_sync(FULLM, v, j - b0);
        if (i < j) v -= S[i * LD + j] * xj;
      }
      if (i < be) x[i] = v;
    }
    __syncthreads();
    if (b0 > 0) {
      for (int i = tid; i < b0; i += NT) {
        double s = 0.0;
        for (int j = b0; j < be; ++j) s += S[i * LD + j] * x[j];
        x[i] -= s;
      }
      __syncthreads();
    }
  }
}
// the rows of a solve phase summed by a warp
enum { RW_FWD, RW_BWD, RW_L21 };
// t[i] = (t[i] - sum_p a[p] t[ci[p]]) * sc over the entries [p0, p1) of
// each row i = rows[r] (rows == nullptr: i = r), r = r0, r0 + rs, ... < r1,
// one row after another by one warp (lanes over the entries, a warp sum),
// the next row's entries loaded while the current one is summed. MODE:
// RW_FWD the L entries (sc = 1, unit diagonal), RW_BWD the U entries (sc =
// 1 / the pivot), RW_L21 a dense row's sparse-column L entries (sc = 1).
// a row's range of entries in MODE's part of the factors
template <int MODE>
__device__ __forceinline__ void row_range(int i, int& p0, int& p1) {
  if (MODE == RW_FWD) { p0 = d_sp_rp[i]; p1 = d_sp_di[i]; }
  else if (MODE == RW_BWD) { p0 = d_sp_di[i] + 1; p1 = d_sp_rp[i + 1]; }
  else { p0 = d_sp_rp[i]; p1 = d_bk_l21e[i - BK_M]; }
}
// the first 128 entries of a warp's row (4 a lane): values and columns.
// The factors and the tables do not change during a solve, so a warp loads
// the row of its next call before the barrier that ends the current one
// (only t, read after it, does).
struct RowAhead {
  double a[4];
  int c[4];
  bool ok;
};
template <int MODE>
__device__ __forceinline__ void row_ahead(const int* rows, int r, int r1,
                                          const double* A, RowAhead& q) {
  q.ok = r < r1;
  if (!q.ok) return;
  const int lane = threadIdx.x & 31;
  int p0, p1;
  row_range<MODE>(rows != nullptr ? rows[r] : r, p0, p1);
#pragma unroll
  for (int s = 0; s < 4; ++s) {
    const int p = p0 + lane + 32 * s;
    q.c[s] = p < p1 ? d_sp_ci[p] : -1;
    q.a[s] = p < p1 ? A[p] : 0.0;
  }
}

// rows r0, r0 + rs, ... < r1 of `rows` (nullptr: the rows themselves), a
// warp per row, each row's first 128 entries loaded while the previous
// row is summed (the first row's from q when it holds them)
template <int MODE>
__device__ void rows_by_warp(const int* rows, int r0, int r1, int rs,
                             const double* A, const double* rpiv, double* t,
                             const RowAhead* q = nullptr) {
  const int lane = threadIdx.x & 31;
  auto row = [&](int r) { return rows != nullptr ? rows[r] : r; };
  RowAhead cur;
  if (q != nullptr && q->ok) cur = *q;
  else row_ahead<MODE>(rows, r0, r1, A, cur);
  for (int r = r0; r < r1; r += rs) {
    const int i = row(r);
    const RowAhead now = cur;
    if (r + rs < r1) row_ahead<MODE>(rows, r + rs, r1, A, cur);
    double sum = 0.0;
#pragma unroll
    for (int s = 0; s < 4; ++s)
      if (now.c[s] >= 0) sum += now.a[s] * t[now.c[s]];
    int p0, p1;
    row_range<MODE>(i, p0, p1);
    for (int p = p0 + 128 + lane; p < p1; p += 32) sum += A[p] * t[d_sp_ci[p]];
    sum = warp_sum(sum);
    if (lane == 0) t[i] = MODE == RW_BWD ? (t[i] - sum) * rpiv[i] : t[i] - sum;
    __syncwarp();
  }
}

// the rows r0.. < r1 of a level wider than the block's warps, G lanes a
// row (32 / G rows a warp at a time): a level of many short rows (the
// backward sweep's first levels: 50-80 rows of ~12 entries) would leave a
// warp per row mostly idle and its rows one after another
template <int MODE, int G>
__device__ void rows_by_group(const int* rows, int r0, int r1,
                              const double* A, const double* rpiv, double* t) {
  constexpr int PW = 32 / G;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int sub = lane % G;
  // bounded: each pass advances every lane's row by NWARP * PW
  for (int r = r0 + warp * PW + lane / G;; r += NWARP * PW) {
    const bool has = r < r1;
    if (!__any_sync(FULLM, has)) break;
    double sum = 0.0;
    int i = 0;
    if (has) {
      i = rows != nullptr ? rows[r] : r;
      int p0, p1;
      row_range<MODE>(i, p0, p1);
      for (int p = p0 + sub; p < p1; p += G) sum += A[p] * t[d_sp_ci[p]];
    }
#pragma unroll
    for (int o = G / 2; o > 0; o >>= 1) sum += __shfl_xor_sync(FULLM, sum, o);
    if (has && sub == 0)
      t[i] = MODE == RW_BWD ? (t[i] - sum) * rpiv[i] : t[i] - sum;
    __syncwarp();
  }
}

// x = A^-1 b with the factors (b and x in the species order; x may be b).
// Starts and ends with a block barrier; one barrier per level.
__device__ void block_solve(const double* A, const double* b, double* x) {
  const double* S = smem() + SM::S;
  const double* rpiv = smem() + SM::RPIV;
  double* t = smem() + SM::T;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  __syncthreads();
  KBG_FOR(i) t[i] = b[d_sp_perm[i]];
  __syncthreads();
  // q: this warp's first row of the next narrow level, loaded ahead
  RowAhead q;
  q.ok = false;
  // (a run of single-row levels -- the chain before the dense block --
  // goes to warp 0 in one call: its rows in order, no block barrier
  // between them, each row's factors loaded while the previous is summed)
  for (int L = 1, Ln; L < BK_NLF; L = Ln) {  // level 0 rows have no L entries
    const int r0 = d_bk_flp[L], r1 = d_bk_flp[L + 1];
    Ln = L + 1;
    if (r1 - r0 == 1) {
      while (Ln < BK_NLF && d_bk_flp[Ln + 1] - d_bk_flp[Ln] == 1) ++Ln;
      if (warp == 0)
        rows_by_warp<RW_FWD>(d_bk_frow, r0, d_bk_flp[Ln], 1, A, rpiv, t, &q);
    } else if (r1 - r0 >= 16) {  // wide levels' rows have a few L entries each
      for (int r = r0 + tid; r < r1; r += NT) {
        const int i = d_bk_frow[r];
        double s = 0.0;
        for (int p = d_sp_rp[i]; p < d_sp_di[i]; ++p) s += A[p] * t[d_sp_ci[p]];
        t[i] -= s;
      }
    } else if (r1 - r0 > NWARP) {
      rows_by_group<RW_FWD, 8>(d_bk_frow, r0, r1, A, rpiv, t);
    } else {
      rows_by_warp<RW_FWD>(d_bk_frow, r0 + warp, r1, NWARP, A, rpiv, t, &q);
    }
    if (Ln < BK_NLF) {
      const int n0 = d_bk_flp[Ln], n1 = d_bk_flp[Ln + 1];
      if (n1 - n0 <= NWARP) row_ahead<RW_FWD>(d_bk_frow, n0 + warp, n1, A, q);
      else q.ok = false;
    } else {
      row_ahead<RW_L21>(nullptr, BK_M + warp, N, A, q);
    }
    __syncthreads();
  }
  // the dense rows' sparse columns: a warp per row (a hub row has hundreds)
  rows_by_warp<RW_L21>(nullptr, BK_M + warp, N, NWARP, A, rpiv, t, &q);
  if (d_bk_blp[1] - d_bk_blp[0] <= NWARP)
    row_ahead<RW_BWD>(d_bk_brow, d_bk_blp[0] + warp, d_bk_blp[1], A, q);
  else
    q.ok = false;
  __syncthreads();
  dense_fwd(S, t + BK_M);
  dense_bwd(S, rpiv + BK_M, t + BK_M);
  for (int L = 0, Ln; L < BK_NLB; L = Ln) {  // a warp per row (U rows reach
                                             // into the dense columns)
    const int r0 = d_bk_blp[L], r1 = d_bk_blp[L + 1];
    Ln = L + 1;
    if (r1 - r0 == 1) {  // a run of single-row levels: warp 0, in order
      while (Ln < BK_NLB && d_bk_blp[Ln + 1] - d_bk_blp[Ln] == 1) ++Ln;
      if (warp == 0)
        rows_by_warp<RW_BWD>(d_bk_brow, r0, d_bk_blp[Ln], 1, A, rpiv, t, &q);
    } else if (r1 - r0 > NWARP) {
      rows_by_group<RW_BWD, 8>(d_bk_brow, r0, r1, A, rpiv, t);
    } else {
      rows_by_warp<RW_BWD>(d_bk_brow, r0 + warp, r1, NWARP, A, rpiv, t, &q);
    }
    q.ok = false;
    if (Ln < BK_NLB && d_bk_blp[Ln + 1] - d_bk_blp[Ln] <= NWARP)
      row_ahead<RW_BWD>(d_bk_brow, d_bk_blp[Ln] + warp, d_bk_blp[Ln + 1], A, q);
    __syncthreads();
  }
  KBG_FOR(i) x[d_sp_perm[i]] = t[i];
  __syncthreads();
}

struct Stats9 {
  long nst, nfe, nje, nsetups, nni, nnf, netf;
};

// one cell's CVODE (the oracle's Cvode, sparse path, one block)
struct BigCvode {
  Net& P;
  const SolveOpts& o;
  double* zn[L_MAX];
  double *ewt, *y, *acor, *tempv, *ftemp, *delta, *A, *savedJ, *bcol;
  double zb;  // an evolved Tgas: the 1 x 1 Schur complement of the border
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
    savedJ = w + WS::SJ;
    A = w + WS::A;
    bcol = w + WS::BT;
    zb = 1.0;
    mxstep = o.max_steps == 0 ? 500
             : (o.max_steps < 0 ? KB_MAX_STEPS_CAP : o.max_steps);
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

  // cvEwtSetSV with one atol for the species and atol_T for an evolved
  // Tgas (bdf_cell.hpp:689-713)
  __device__ int ewt_set(const double* ycur, double* wt) {
    bool bad = false;
    KBG_VFOR(i) {
      const double at = i < N ? o.atol_n : o.atol_T;
      const double v = (o.rtol * fabs(ycur[i])) + at;
      bad = bad || !(v > 0.0);
      wt[i] = 1.0 / v;
    }
    return __syncthreads_or(bad) ? -1 : 0;
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
    KBG_VFOR(i) temp2[i] = fabs(zn[0][i]);
    ewt_set(zn[0], temp1);
    KBG_VFOR(i) temp1[i] = 1.0 / temp1[i];
    v_lin_sum(HUB_FACTOR, temp2, 1.0, temp1, temp1);
    KBG_VFOR(i) temp2[i] = fabs(zn[1][i]);
    KBG_VFOR(i) temp1[i] = temp2[i] / temp1[i];
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
        lsolve_(delta);
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
    const bool evt = neq() > N;
    if (jbad_ls) {
      P.jac(y, savedJ);
      if (evt) P.jac_tgas(y, bcol);
    }
    const double c = -gamma;
    double* S = smem() + SM::S;
    for (int k = threadIdx.x; k < NNZ_LU; k += NT) A[k] = 0.0;
    for (int k = threadIdx.x; k < BK_D * BK_LD; k += NT) S[k] = 0.0;
    __syncthreads();
    for (int e = threadIdx.x; e < NNZ_J; e += NT) {
      const int t = d_bk_jt[e];
      const double v = savedJ[e] * c;
      if (t >= 0) A[t] = v;
      else S[-1 - t] = v;
    }
    __syncthreads();
    KBG_FOR(i) {
      if (i < BK_M) A[d_sp_di[i]] += 1.0;
      else S[(i - BK_M) * (BK_LD + 1)] += 1.0;
    }
    if (jcur) {
      st.nje++;
      nstlj = st.nst;
    }
    if (block_lu(A) > 0) return LS_LUFACT_FAIL;
    if (evt) {
      // the border (bdf_cell.hpp:1192-1219, m = 1) with a zero Tgas row:
      // C' = 0, so Z = c D + 1 - C' B' = 1 with D = 0, unless a non-finite
      // entry of B' makes the products C' B' NaN (then Z is NaN, as there)
      bool bad = false;
      KBG_FOR(i) bad = bad || !isfinite(bcol[i] * c);
      const double dc = 0.0 * c;
      zb = __syncthreads_or(bad) ? NAN : dc + 1.0;
      if (zb == 0.0) return LS_LUFACT_FAIL;
    }
    return 0;
  }
  // x = M^-1 x for the Newton matrix M (the species' block factors, and an
  // evolved Tgas's border as the reference's solve, bdf_cell.hpp:1233-
  // 1264: with a zero Tgas row the Tgas component is its right-hand side
  // over Z, and the species' part takes c B times it off before the
  // species solve, which the reference skips when it is zero)
  __device__ void lsolve_(double* x) {
    if (neq() == N) { block_solve(A, x, x); return; }
    __syncthreads();
    const double v = x[N] / zb;
    if (v != 0.0) {
      const double c = -gamma;
      KBG_FOR(i) x[i] -= (bcol[i] * c) * v;
    }
    block_solve(A, x, x);
    if (threadIdx.x == N % NT) x[N] = v;
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
