// libkrome_b200_<net>.so: the reference's generated C ABI for the per-cell
// solve (runtime/interfaces/C/krome.h), served by sm_100a kernels.
//
// Compiled once per network (-DKB_NET_HEADER="...net_<key>.h"), as the
// reference compiles krome.cpp once per generated project. The entry points
// keep the reference's names, arguments, array layouts and flags (declared,
// with the reference lines each one replaces, in include/krome_b200.h);
// the krome_b200_* entry points are this library's additions: the
// device-resident solve, the persistent work-queue kernel, per-cell
// counters and the captured hydro loop.
//
// Kernels (one warp per cell, bdf_warp.cuh):
//   kb_cells_plain       cell c = blockIdx.x * warps + warp: a fixed
//                        assignment, one cell per warp
//   kb_cells_persistent  a resident grid whose warps pull chunks of cells
//                        from a device work queue (an atomic cursor), so a
//                        warp that finishes an easy cell takes the next one
//                        instead of idling while stiff cells finish
// There is no CPU fallback: a cell that fails on the device returns its
// flag, and a missing or unusable GPU makes the solve return -104.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include KB_NET_HEADER
#ifndef KB_NFREEZE
#define KB_NFREEZE 0  // a network header from before freeze directives
#endif
#include "bdf_warp.cuh"
#include "bdf_lane.cuh"
#include "adjoint.cuh"
#include "bdf_big.cuh"
#include "kb_photo.h"

#define KB_API extern "C" __attribute__((visibility("default")))

// the reference's optional per-cell arrays of a call (krome.h:258-294)
typedef struct {
  double* Phi;
  double* Td;
  double* adust;
} krome_cells;

using kbw::SolveOpts;
using kbw::NSTAT;

namespace {

constexpr int kWarpsPerBlock = 4;

template <bool EVT>
struct Geo {
  static constexpr int N = kbnet::NSPEC + (EVT ? 1 : 0);
  // per-warp shared memory: the saved Jacobian and two columns
  static constexpr int SMEM_DOUBLES = N * N + 2 * N;
};
#ifndef KB_LARGE_NETWORK
static_assert(kbnet::NSPEC + 3 <= 32,
              "warp-per-cell kernels need NEQ + 2 <= 32 lanes");
#endif

template <bool EVT>
__device__ __forceinline__ void one_cell(int c, double* n, double* T,
                                         const double* dt, const double* par,
                                         int pstride, int* flags, long* stats,
                                         const SolveOpts& so, double* ws) {
  const int lane = threadIdx.x & 31;
  constexpr int N = Geo<EVT>::N;
  long* sc = stats != nullptr ? stats + (long)c * NSTAT : nullptr;
  int flag = 0;
  const double dtc = dt[c];
  if (so.fail_every > 0 && (c + 1) % so.fail_every == 0) {
    flag = kbw::TOO_MUCH_WORK;  // injected failure: the cell is untouched
    if (sc != nullptr && lane < NSTAT) sc[lane] = 0;
  } else if (dtc > 0.0) {
    flag = kbw::solve_cell<N, EVT>(n + (long)c * kbnet::NSPEC, T + c,
                                   par + (long)c * pstride, dtc, so, ws, sc, c);
  } else if (sc != nullptr && lane < NSTAT) {
    sc[lane] = 0;
  }
  if (lane == 0 && flags != nullptr) flags[c] = flag;
}

template <bool EVT>
__global__ void __launch_bounds__(kWarpsPerBlock * 32)
kb_cells_plain(int ncell, double* n, double* T, const double* dt,
               const double* par, int pstride, int* flags, long* stats,
               SolveOpts so) {
  extern __shared__ double smem[];
  const int warp = threadIdx.x >> 5;
  const int c = blockIdx.x * kWarpsPerBlock + warp;
  if (c >= ncell) return;
  one_cell<EVT>(c, n, T, dt, par, pstride, flags, stats, so,
                smem + warp * Geo<EVT>::SMEM_DOUBLES);
}

template <bool EVT>
__global__ void __launch_bounds__(kWarpsPerBlock * 32)
kb_cells_persistent(int ncell, double* n, double* T, const double* dt,
                    const double* par, int pstride, int* flags, long* stats,
                    SolveOpts so, unsigned* cursor, int chunk) {
  extern __shared__ double smem[];
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  double* ws = smem + warp * Geo<EVT>::SMEM_DOUBLES;
  // at most ncell / chunk + 1 pops per warp: the cursor only grows
  for (;;) {
    unsigned base = 0;
    if (lane == 0) base = atomicAdd(cursor, (unsigned)chunk);
    base = __shfl_sync(0xffffffffu, base, 0);
    if (base >= (unsigned)ncell) break;
    const int end = min((int)base + chunk, ncell);
    for (int c = (int)base; c < end; ++c)
      one_cell<EVT>(c, n, T, dt, par, pstride, flags, stats, so, ws);
  }
}

// ---- lane-per-cell kernels (bdf_lane.cuh) ----

template <bool EVT>
struct LaneGeo {
  static constexpr int N = kbnet::NSPEC + (EVT ? 1 : 0);
  // lanes one Jacobian request occupies: the N difference-quotient
  // columns, or the hybrid analytic Jacobian's NSPEC species + base +
  // Tgas +/- h states
  static constexpr int JLANES_DQ = N;
  static constexpr int JLANES_AN = EVT ? kbnet::NSPEC + 3 : 1;
  static constexpr int ROLE_BASE = EVT ? kbnet::NSPEC : 0;
  // per-warp shared memory: the Jacobians being assembled (column-major,
  // one N x N block per request of a pass) and the Tgas +/- h rhs
  // vectors of the hybrid Jacobian. Requests per pass: as many as the
  // lanes hold, within 1,536 doubles a warp (the block's four warps stay
  // under the 48 KB that needs no opt-in), at least one
  static constexpr int JBLK = N * N + 2 * N;
  static constexpr int MAXJ_LANES =
      32 / (JLANES_DQ < JLANES_AN ? JLANES_DQ : JLANES_AN);
  static constexpr int MAXJ_SMEM = 1536 / JBLK > 0 ? 1536 / JBLK : 1;
  static constexpr int MAXJ = MAXJ_LANES < MAXJ_SMEM ? MAXJ_LANES : MAXJ_SMEM;
  static constexpr int SMEM_DOUBLES = MAXJ * JBLK;
};

// the adjoint's forward solve (kb_lane_cells with REC): the rate factors
// exp(m) and where each cell's tape goes
struct RecIO {
  const double* mult;  // [ncell][NREA] (mstride NREA) or one row (0); null: 1
  int mstride;
  double* tape;        // [ncell][cap] doubles
  long cap;
  long* tlen;          // per cell: its tape's length; 0 not integrated
  double* yfin;        // [ncell][N]: the final y before the post-solve rules
};

// where the lane kernel reads and writes each cell's species: the caller's
// layout (krome.h:311-314: species-major n[i * ld + c], or cell-major
// n[c * nspec + i]) and, with rho, mass fractions x = m n / rho converted
// on the way in and out (solve_cell.hpp:2210-2233), so that the device-
// resident entry points need no staging passes around the solve
struct CellIO {
  int layout = 1;               // 0 species-major, 1 cell-major
  long ld = 0;                  // the species-major leading dimension
  const double* rho = nullptr;  // [ncell] g cm^-3: the species are x
  int renormalize = 0;          // x rescaled to its input sum on the way out
  __device__ __forceinline__ long at(int c, int i) const {
    return layout == 0 ? (long)i * ld + c : (long)c * kbnet::NSPEC + i;
  }
};

// x_to_n_ / x_sum_ / n_to_x_out_ (solve_cell.hpp:2210-2233): n = rho x / m
// (0 for a species without mass), x = m n / rho, rescaled to the input sum
// of the fractions with renormalize_x
KB_HD inline void x_to_n(const double* x, double rho, double* n) {
  for (int i = 0; i < kbnet::NSPEC; ++i) {
    const double m = kbnet::species_mass_g(i);
    n[i] = m > 0.0 ? rho * x[i] / m : 0.0;
  }
}
KB_HD inline double x_sum(const double* x) {
  double s = 0.0;
  for (int i = 0; i < kbnet::NSPEC; ++i)
    if (kbnet::species_mass_g(i) > 0.0) s += x[i];
  return s;
}
KB_HD inline void n_to_x_out(const double* n, double rho, double xin,
                             int renormalize, double* x) {
  for (int i = 0; i < kbnet::NSPEC; ++i)
    x[i] = kbnet::species_mass_g(i) * n[i] / rho;
  if (!renormalize) return;
  const double s = x_sum(x);
  if (s > 0.0)
    for (int i = 0; i < kbnet::NSPEC; ++i) x[i] *= xin / s;
}

// cell c's input densities from the caller's arrays (xin: the input sum of
// the mass fractions)
__device__ __forceinline__ void cell_densities(const double* n, const CellIO& io,
                                               int c, double* nc, double* xin) {
  using namespace kbnet;
  double v[NSPEC];
  KB_UNROLL for (int i = 0; i < NSPEC; ++i) v[i] = n[io.at(c, i)];
  if (io.rho == nullptr) {
    KB_UNROLL for (int i = 0; i < NSPEC; ++i) nc[i] = v[i];
    *xin = 0.0;
    return;
  }
  *xin = x_sum(v);
  x_to_n(v, io.rho[c], nc);
}

// start cell c on this lane: false when the cell needs no integration
// (its flag is written here)
template <bool EVT, bool REC>
__device__ bool lane_start(kbl::LaneCell<LaneGeo<EVT>::N>& s,
                           kbl::Machine<LaneGeo<EVT>::N, EVT, REC>& m, int c,
                           const double* n, const double* T, const double* dt,
                           const double* par, int pstride, int* flags,
                           long* stats, const SolveOpts& so,
                           const RecIO& rio, const CellIO& io) {
  constexpr int N = LaneGeo<EVT>::N;
  using namespace kbnet;
  const double dtc = dt[c];
  int skip_flag = 1;
  if (so.fail_every > 0 && (c + 1) % so.fail_every == 0) skip_flag = kbw::TOO_MUCH_WORK;
  else if (!(dtc > 0.0)) skip_flag = 0;
  if constexpr (REC) rio.tlen[c] = 0;
  if (skip_flag != 1) {
    if (flags != nullptr) flags[c] = skip_flag;
    if (stats != nullptr)
      for (int i = 0; i < NSTAT; ++i) stats[(long)c * NSTAT + i] = 0;
    return false;
  }
  params_from_row(par + (long)c * pstride, s.p);
  if (params_missing(s.p) >= 0) {
    if (flags != nullptr) flags[c] = kbw::FLAG_PARAM_UNSET;
    return false;
  }
  kbw::photo_rates_of_cell(s.p, c, so);
#if KB_NFREEZE > 0
  // the adjoint does not differentiate frozen rows: refused there
  if (REC && freeze_active(s.p)) {
    if (flags != nullptr) flags[c] = -104;
    return false;
  }
#endif
  if constexpr (REC) {
    // no tape: the lengths only (tape_len gets what the cell would need)
    s.tp = rio.tape != nullptr ? rio.tape + (long)c * rio.cap : nullptr;
    s.tcap = rio.tape != nullptr ? rio.cap : (1L << 62);
    s.tlen = 0;
  }
  s.cell = c;
  s.dt = dtc;
  s.Tfix = T[c];
  s.hitT0 = false;
  s.restarts = 0;
  for (int i = 0; i < NSTAT; ++i) s.tot[i] = 0;
  double y0[N];
  cell_densities(n, io, c, y0, &s.xin);
  if (EVT) y0[N - 1] = T[c];
  double amin = 1e300;
  KB_UNROLL for (int i = 0; i < N; ++i) {
    s.atol[i] = i < NSPEC ? so.atol_sp[i < kbw::KB_NSP_TOL ? i : 0] : so.atol_T;
    amin = fmin(amin, s.atol[i]);
  }
  s.atolmin0 = amin == 0.0;  // CVodeSVtolerances: N_VMin(abstol) == 0
  s.mxstep = so.max_steps == 0 ? 500
             : (so.max_steps < 0 ? KB_MAX_STEPS_CAP : so.max_steps);
  m.reinit(0.0, y0, 0.0);
  s.ph = kbl::PH_SOLVE;
  s.wait = kbl::WAIT_NONE;
  return true;
}

// the post-solve rules of solve() (solve_cell.hpp:2156-2176) and the
// write-back of a finished cell
template <bool EVT, bool REC>
__device__ void lane_finish(kbl::LaneCell<LaneGeo<EVT>::N>& s, int flag,
                            double* n, double* T, int* flags, long* stats,
                            const SolveOpts& so, const RecIO& rio,
                            const CellIO& io) {
  constexpr int N = LaneGeo<EVT>::N;
  using namespace kbnet;
  const int c = s.cell;
  if constexpr (REC) {
    // a tape that outgrew its capacity: no gradient, the cell untouched
    if (flag == 0 && s.tlen < 0) flag = kbw::FLAG_TAPE_FULL;
    rio.tlen[c] = s.tlen;
    KBL_LOOP for (int i = 0; i < N; ++i) rio.yfin[(long)c * N + i] = s.y[i];
  }
  s.tot[kbw::ST_RESTARTS] = s.restarts;
  if (stats != nullptr)
    for (int i = 0; i < NSTAT; ++i) stats[(long)c * NSTAT + i] = s.tot[i];
  const double Tend = s.y[N - 1];
  if (flag == 0 && EVT && !(Tend > 0.0 && isfinite(Tend)))
    flag = kbw::FLAG_NONPOSITIVE_T;
  if (s.hitT0 && (flag == kbw::REPTD_RHSFUNC_ERR || flag == kbw::RHSFUNC_FAIL
                  || flag == kbw::UNREC_RHSFUNC_ERR
                  || flag == kbw::FIRST_RHSFUNC_ERR))
    flag = kbw::FLAG_NONPOSITIVE_T;
  if (flag == 0) {
    double nv[NSPEC];
    KB_UNROLL for (int i = 0; i < NSPEC; ++i) {
      double v = s.y[i];
      if (so.clip_negative && v < 0.0) v = 0.0;
      nv[i] = v;
    }
    if (so.conserve > 0) {  // against the cell's input, still in n
      double n0[NSPEC], x0;
      cell_densities(n, io, c, n0, &x0);
      kbnet::conserve_cell(n0, nv, so.conserve, s.p);
    }
    if (io.rho != nullptr) {
      double xv[NSPEC];
      n_to_x_out(nv, io.rho[c], s.xin, io.renormalize, xv);
      KB_UNROLL for (int i = 0; i < NSPEC; ++i) n[io.at(c, i)] = xv[i];
    } else {
      KB_UNROLL for (int i = 0; i < NSPEC; ++i) n[io.at(c, i)] = nv[i];
    }
    if (EVT) T[c] = Tend;
  }
  if (flags != nullptr) flags[c] = flag;
  s.cell = -1;
}

// one warp = 32 cells in flight. persistent == 0: each lane integrates the
// cell of its global thread index; persistent == 1: lanes pull cells from
// the device work queue (`cursor`) until it is exhausted.
//
// Each round: (1) one sweep of the phase handlers takes every lane to its
// next request (lanes whose cell finished write it back, take their next
// cell and sweep once more); (2) the warp evaluates the requests with ONE
// rhs call site: pass 0 the
// lanes' own rhs requests, then one pass per group of Jacobian requests,
// where request r of the pass occupies lanes [r*JL, (r+1)*JL) (JL the lanes
// one Jacobian needs) and lane r*JL + j evaluates its column / term j; the
// assembled Jacobians go through shared memory to the requesting lanes.
//
// REC (the adjoint's forward solve): the rates multiplied by the cells'
// factors exp(m) and every zn operation recorded on the cell's tape.
template <bool EVT, int MINB, bool REC>
__global__ void __launch_bounds__(kWarpsPerBlock * 32, MINB)
kb_lane_cells(int ncell, double* n, double* T, const double* dt,
              const double* par, int pstride, int* flags, long* stats,
              SolveOpts so, unsigned* cursor, int persistent, RecIO rio,
              CellIO io) {
  constexpr int N = LaneGeo<EVT>::N;
  using namespace kbnet;
  constexpr unsigned FULLM = 0xffffffffu;
  extern __shared__ double smem[];
  const int warp = threadIdx.x >> 5;
  const int lane = threadIdx.x & 31;
  double* sw = smem + warp * LaneGeo<EVT>::SMEM_DOUBLES;
  kbl::LaneCell<N> s;
  kbl::Machine<N, EVT, REC> m(s, so);
  s.tp = nullptr;
  s.cell = -1;
  s.ph = kbl::PH_DONE;  // take a first cell
  s.wait = kbl::WAIT_NONE;
  bool static_taken = false;
  const int gtid = blockIdx.x * blockDim.x + threadIdx.x;
  const bool dq = so.jac == 2;
  const int JL = dq ? LaneGeo<EVT>::JLANES_DQ : LaneGeo<EVT>::JLANES_AN;
  const int per_pass = 32 / JL < LaneGeo<EVT>::MAXJ ? 32 / JL : LaneGeo<EVT>::MAXJ;
  for (;;) {
    // a lane whose cell finished in the first sweep takes its next cell
    // and sweeps again in the same round
    for (int sweep = 0; sweep < 2; ++sweep) {
      // bounded: every iteration consumes a cell index (at most ncell)
      while (s.ph == kbl::PH_DONE) {
        if (s.cell >= 0) lane_finish<EVT, REC>(s, s.flag, n, T, flags, stats, so, rio, io);
        int c;
        if (persistent) {
          c = (int)atomicAdd(cursor, 1u);
        } else {
          c = static_taken ? ncell : gtid;
          static_taken = true;
        }
        if (c >= ncell) s.ph = kbl::PH_IDLE;
        else lane_start<EVT, REC>(s, m, c, n, T, dt, par, pstride, flags, stats, so, rio, io);
      }
      if (s.ph != kbl::PH_IDLE) m.sweep();
      if (!__any_sync(FULLM, s.ph == kbl::PH_DONE)) break;
    }
    if (__all_sync(FULLM, s.ph == kbl::PH_IDLE)) break;
    const int req = s.wait;
    const unsigned jm = __ballot_sync(FULLM, req == kbl::WAIT_JAC);
    const int nj = __popc(jm);
    const int npass = 1 + (nj + per_pass - 1) / per_pass;
    unsigned jrest = jm;
    for (int pass = 0; pass < npass; ++pass) {
      // ---- this lane's task ----
      bool active;
      int src = lane, role = 0;
      unsigned passm = 0;  // the requesting lanes served in this pass
      if (pass == 0) {
        active = req == kbl::WAIT_RHS;
      } else {
        for (int r = 0; r < per_pass && jrest; ++r) {
          const unsigned b = jrest & (~jrest + 1u);
          passm |= b;
          jrest &= jrest - 1u;
        }
        const int grp = lane / JL;
        role = lane - grp * JL;
        // the grp-th set bit of passm
        unsigned t = passm;
        for (int r = 0; r < grp && t; ++r) t &= t - 1u;
        active = grp < per_pass && t != 0u;
        src = active ? __ffs(t) - 1 : lane;
      }
      // ---- the state to evaluate ----
      double yf[N], f[N], k[NREA + 1];
      Params p;
      double Tfix, inc = 1.0, hT = 1.0;
      const double* mrow = nullptr;  // REC: the evaluated cell's exp(m)
      if constexpr (REC) {
        const int ec = __shfl_sync(FULLM, s.cell, src);
        if (rio.mult != nullptr && ec >= 0) mrow = rio.mult + (long)ec * rio.mstride;
      }
      if (pass == 0) {
        KB_UNROLL for (int i = 0; i < N; ++i) yf[i] = s.yreq[i];
        p = s.p;
        Tfix = s.Tfix;
      } else {
        KB_UNROLL for (int i = 0; i < N; ++i) yf[i] = __shfl_sync(FULLM, s.y[i], src);
        {
          // the evaluated cell's parameters, the photo rates included
          constexpr int PW = sizeof(Params) / sizeof(double);
          static_assert(sizeof(Params) == PW * sizeof(double), "Params of doubles");
          const double* ps = reinterpret_cast<const double*>(&s.p);
          double* pd = reinterpret_cast<double*>(&p);
          KB_UNROLL for (int i = 0; i < PW; ++i) pd[i] = __shfl_sync(FULLM, ps[i], src);
        }
        Tfix = __shfl_sync(FULLM, s.Tfix, src);
        if (dq) {
          // CVODE's increment of column `role` (bdf_cell.hpp:1294-1301)
          double sum = 0.0, yj = 0.0, ewj = 1.0;
          KB_UNROLL for (int i = 0; i < N; ++i) {
            const double fyi = __shfl_sync(FULLM, s.ftemp[i], src);
            const double ewi = __shfl_sync(FULLM, s.ewt[i], src);
            const double pv = fyi * ewi;
            sum += pv * pv;
            if (i == role) { yj = yf[i]; ewj = ewi; }
          }
          const double h = __shfl_sync(FULLM, s.h, src);
          const double fnorm = kbw::ssqrt_(sum / N);
          const double minInc = (fnorm != 0.0)
              ? (kbw::MIN_INC_MULT * fabs(h) * kbw::UROUND * (double)N * fnorm) : 1.0;
          inc = kbw::smax_(kbw::ssqrt_(kbw::UROUND) * fabs(yj), minInc / ewj);
          KB_UNROLL for (int i = 0; i < N; ++i) if (i == role) yf[i] += inc;
        } else if (EVT) {
          // hybrid analytic Jacobian terms (solve_cell.hpp:1053-1099)
          constexpr int iT = N - 1;
          double sumabs = 0.0, yj = 0.0;
          KB_UNROLL for (int i = 0; i < NSPEC; ++i) {
            sumabs += fabs(yf[i]);
            if (i == role) yj = yf[i];
          }
          hT = fmax(1e-6 * fabs(yf[iT]), 1e-8);
          inc = role < NSPEC ? fmax(fmax(1e-7 * fabs(yj), 1e-9 * sumabs), 1e-30) : 1.0;
          KB_UNROLL for (int i = 0; i < NSPEC; ++i) if (i == role) yf[i] += inc;
          if (role == NSPEC + 1) yf[iT] += hT;
          if (role == NSPEC + 2) yf[iT] -= hT;
        }
      }
      // ---- the one rhs evaluation of this round and pass ----
      // (the hybrid Jacobian's species terms keep the base rate
      // temperature: their perturbation leaves Tgas alone)
      bool hit = false;
      int r = 0;
      if (active) {
        kbw::full_rhs<N, EVT>(yf, f, p, Tfix, k, mrow);
        // the integrator's checks (rhs_host_, solve_cell.hpp:794-813): a
        // trial Tgas <= 0 or a non-finite f is a recoverable failure; the
        // hybrid Jacobian's terms are plain full_rhs_ evaluations
        if (pass == 0 || dq) {
          if (EVT && !(yf[N - 1] > 0.0)) {
            hit = true;
            r = 1;
          } else {
            bool ok = true;
            KB_UNROLL for (int i = 0; i < N; ++i) ok = ok && isfinite(f[i]);
            r = ok ? 0 : 1;
          }
        }
        // the hybrid Jacobian's base-state lane: the stoichiometric block
        // with the rates of the base state (jacobian_split)
        if (pass > 0 && !dq && role == LaneGeo<EVT>::ROLE_BASE) {
          double* J = sw + (lane / JL) * (N * N + 2 * N);
          jac_stoich(yf, k, J, 1, N);
#ifndef KB_LARGE_NETWORK
          if constexpr (KB_RATE_NDEP > 0) {
            // the rate-derivative terms at the base state's rate
            // temperature, then the aggregates' coupling U W^T
            const double Tr = fmin(fmax(EVT ? yf[N - 1] : Tfix, p.Tcmb), 1e9);
            kbw::jac_rate_terms(Tr, yf, p, k, J, 1, N);
          }
#endif
        }
      }
      // ---- results ----
      if (pass == 0) {
        if (active) {
          KB_UNROLL for (int i = 0; i < N; ++i) s.freq[i] = f[i];
          s.rhs_ret = r;
          s.wait = kbl::WAIT_NONE;
          if (hit) s.hitT0 = true;
        }
        continue;
      }
      const int grp = lane / JL;
      double* blk = sw + (active ? grp : 0) * (N * N + 2 * N);
      const unsigned bad = __ballot_sync(FULLM, active && r != 0);
      const unsigned gmask = (JL >= 32) ? FULLM
          : (((1u << JL) - 1u) << (active ? grp * JL : 0));
      const unsigned gbad = active ? (bad & gmask) : 0u;
      const int first_bad = gbad ? (__ffs(gbad) - 1 - grp * JL) : N;
      (void)gmask;
      const unsigned hitm = __ballot_sync(FULLM, active && hit && role <= first_bad);
      if (dq) {
        const bool store = active && role < N && role < first_bad;
        const double inc_inv = 1.0 / inc;
        KB_UNROLL for (int i = 0; i < N; ++i) {
          const double fyi = __shfl_sync(FULLM, s.ftemp[i], src);
          if (store) blk[i + role * N] = inc_inv * (f[i] - fyi);
        }
      } else if (EVT) {
        constexpr int iT = N - 1;
        double* sv = blk + N * N;
        if (active && role == NSPEC + 1) { KB_UNROLL for (int i = 0; i < N; ++i) sv[i] = f[i]; }
        if (active && role == NSPEC + 2) { KB_UNROLL for (int i = 0; i < N; ++i) sv[N + i] = f[i]; }
        // the base state's thermal row value (role NSPEC of the group)
        const double f0 = __shfl_sync(FULLM, f[iT], (active ? grp * JL : 0)
                                                     + LaneGeo<EVT>::ROLE_BASE);
        if (active && role < NSPEC) blk[iT + role * N] = (f[iT] - f0) / inc;
        __syncwarp();
        if (active && role < N) blk[role + iT * N] = (sv[role] - sv[N + role]) / (2.0 * hT);
      }
      __syncwarp();
      // the requesting lane: its stoichiometric block (analytic), then the
      // assembled Jacobian into its savedJ
      if ((passm >> lane) & 1u) {
        int g = 0;
        for (unsigned t = passm & ((1u << lane) - 1u); t; t &= t - 1u) ++g;
        double* myblk = sw + g * (N * N + 2 * N);
        const int base = g * JL;
        const unsigned mbad = bad & (((JL >= 32) ? FULLM : ((1u << JL) - 1u)) << base);
        const int fb = mbad ? (__ffs(mbad) - 1 - base) : N;
        if (!dq) {
          KBL_LOOP for (int i = 0; i < N * N; ++i) s.savedJ[i] = myblk[i];
          kbw::freeze_jac_rows<N>(s.p, s.savedJ, 1, N);
          s.ls_retval = 0;
        } else {
          KBL_LOOP for (int i = 0; i < N * N; ++i) s.savedJ[i] = myblk[i];
          s.ls_retval = mbad ? 1 : 0;
          s.st[kbw::ST_NFEDQ] += mbad ? fb + 1 : N;
        }
        if (hitm & (((JL >= 32) ? FULLM : ((1u << JL) - 1u)) << base))
          s.hitT0 = true;
        s.wait = kbl::WAIT_NONE;
      }
      __syncwarp();
    }
  }
}

#ifdef KB_LARGE_NETWORK
// ---- the large networks: one thread block per cell (bdf_big.cuh) ----

// cell c on this block: the pre-solve rules, the restart wrapper
// (bdf_cell.hpp:1513-1547) and the post-solve rules (solve_cell.hpp:
// 2094-2203) around the sparse-path CVODE, fixed or evolved Tgas (the
// latter on networks without thermal processes). Every thread runs
// the same control flow (the CVODE scalars are the same in every thread).
__device__ void big_one_cell(int c, double* n, double* T, const double* dt,
                             const double* par, int pstride, int* flags,
                             long* stats, const SolveOpts& so, double* ws) {
  using namespace kbnet;
  int flag = 1;
  if (so.fail_every > 0 && (c + 1) % so.fail_every == 0) flag = kbw::TOO_MUCH_WORK;
  else if (!(dt[c] > 0.0)) flag = 0;
  kbg::Net P;
  P.ws = ws;
  params_from_row(par + (long)c * pstride, P.p);
  if (flag == 1 && params_missing(P.p) >= 0) flag = kbw::FLAG_PARAM_UNSET;
  long tot[kbw::NSTAT];
  for (int i = 0; i < kbw::NSTAT; ++i) tot[i] = 0;
  // an evolved Tgas is the state's last component (rhs_cb_: the rhs
  // refuses Tgas <= 0, which the large path's Tgas, constant without
  // thermal processes, fails at its first evaluation)
  const bool evt = so.evolve_T != 0;
  if (flag == 1 && evt && !(T[c] > 0.0)) flag = kbw::FLAG_NONPOSITIVE_T;
  if (flag == 1) {
    P.T = fmin(fmax(T[c], P.p.Tcmb), 1e9);
    double* nrow = n + (long)c * NSPEC;
    double* k = ws + kbg::WS::K;
    for (int r = threadIdx.x; r <= NREA; r += kbg::NT) k[r] = 0.0;
    kbg::set_neq(evt ? NSPEC + 1 : NSPEC);
    __syncthreads();
    // the Tgas/parameter-only rates once per solve, and the three points
    // of the density-dependent ones
    const double hnuc = P.load_state(nrow);
    if (threadIdx.x < RPART)
      rates_fixed_part(threadIdx.x, P.T, kbg::smem() + kbg::SM::YR, P.p, hnuc, k);
    P.prepare_var(nrow);
    kbg::BigCvode cv(P, so);
    double* yout = ws + kbg::WS::YOUT;  // the initial state, then the result
    for (int i = threadIdx.x; i < NSPEC; i += kbg::NT) yout[i] = nrow[i];
    if (evt && threadIdx.x == NSPEC % kbg::NT) yout[NSPEC] = T[c];
    __syncthreads();
    cv.reinit(0.0, yout, 0.0);
    double t = 0.0;
    int restarts = 0;
    for (;;) {  // bounded by max_restarts
      const int f = cv.solve(dt[c], yout, &t);
      tot[kbw::ST_NST] += cv.st.nst;
      tot[kbw::ST_NFE] += cv.st.nfe;
      tot[kbw::ST_NJE] += cv.st.nje;
      tot[kbw::ST_NSETUPS] += cv.st.nsetups;
      tot[kbw::ST_NNI] += cv.st.nni;
      tot[kbw::ST_NNF] += cv.st.nnf;
      tot[kbw::ST_NETF] += cv.st.netf;
      if (f >= 0) { flag = 0; break; }
      const bool restartable = f == kbw::ERR_FAILURE || f == kbw::CONV_FAILURE
                               || f == kbw::REPTD_RHSFUNC_ERR;
      if (!restartable || restarts >= so.max_restarts) { flag = f; break; }
      ++restarts;
      const double hcur = cv.next_h;
      cv.reinit(t, yout, hcur > 0.0 ? 0.1 * hcur : 0.0);
    }
    tot[kbw::ST_RESTARTS] = restarts;
    __syncthreads();
    const double Tend = evt ? yout[NSPEC] : 1.0;
    if (flag == 0 && !(Tend > 0.0 && isfinite(Tend)))
      flag = kbw::FLAG_NONPOSITIVE_T;
    if (flag == 0) {
      if (evt && threadIdx.x == 0) T[c] = Tend;
      for (int i = threadIdx.x; i < NSPEC; i += kbg::NT) {
        double v = yout[i];
        if (so.clip_negative && v < 0.0) v = 0.0;
        yout[i] = v;
      }
      if (so.conserve > 0) {  // thread 0, against the input still in nrow
        __syncthreads();
        if (threadIdx.x == 0) conserve_cell(nrow, yout, so.conserve, P.p);
        __syncthreads();
      }
      for (int i = threadIdx.x; i < NSPEC; i += kbg::NT) nrow[i] = yout[i];
    }
  }
  if (threadIdx.x == 0) {
    if (flags != nullptr) flags[c] = flag;
    if (stats != nullptr)
      for (int i = 0; i < kbw::NSTAT; ++i) stats[(long)c * kbw::NSTAT + i] = tot[i];
  }
  __syncthreads();  // the workspace and shared memory are free again
}

// blocks take cells from the work queue `cursor`; each resident block owns
// the workspace slot of its block index (kbg::WS::SIZE doubles)
__global__ void __launch_bounds__(kbg::NT, 1)
kb_big_cells(int ncell, double* n, double* T, const double* dt,
             const double* par, int pstride, int* flags, long* stats,
             SolveOpts so, unsigned* cursor, double* ws_base) {
  double* ws = ws_base + (long)blockIdx.x * kbg::WS::SIZE;
  double* slot = kbg::smem() + kbg::SM::MISC;
  for (;;) {  // at most ncell + 1 pops per block: the cursor only grows
    if (threadIdx.x == 0) slot[0] = (double)atomicAdd(cursor, 1u);
    __syncthreads();
    const double cd = slot[0];
    __syncthreads();
    if (cd >= (double)ncell) break;
    big_one_cell((int)cd, n, T, dt, par, pstride, flags, stats, so, ws);
  }
}
#endif

// ---- options (krome_opts keys, reference krome.cpp:198-300) ----
}  // namespace

struct krome_opts {
  int evolve_T = 0;
  int jac = 0;       // 0 auto, 1 analytic, 2 fd
  int linsol = 0;    // 0 auto, 1 dense, 2 lapack, 3 sparse
  double rtol = 1e-8, atol_n = 1e-20, atol_T = 1e-6, atol_u = 1e-10;
  long max_steps = 100000;
  int max_err_fails = 7, max_conv_fails = 10, max_restarts = 5;
  int clip_negative = 1, error_report = 0, renormalize_x = 0, conserve = 0;
  int path = 0, device_cache = 1, min_device = 10000, min_interleave = -1;
  long long device_memory = 0;
  // this library's keys
  int kernel = 1;          // 0 plain, 1 persistent work queue
  int layout = 1;          // 0 one warp per cell, 1 one lane per cell
  int lane_minb = 2;       // lane kernel: resident blocks per SM it is
                           // compiled for (2, 3, 4: the register budget)
  int queue_chunk = 1;     // cells per queue pop
  int blocks_per_sm = 0;   // persistent grid: 0 = occupancy limit
  int fail_every = 0;      // fault injection (tests)
  int lu32 = 0;            // Newton-matrix LU in FP32, FP64 after a Newton
                           // failure (lane layout)
  // per-species tolerances (krome_opts_set_atol_species / rtol_species):
  // empty, or NSPEC entries (negative: the scalar)
  std::vector<double> atol_sp, rtol_sp;
  // the reference's other keys: the equilibrium driver (first output time,
  // last time, output factor, convergence tolerances) and the reduced speed
  // of light of an evolved field
  double eq_t0 = 100.0 * kbc::seconds_per_year;
  double eq_tmax = 5e8 * kbc::seconds_per_year;
  double eq_factor = 3.0, eq_rtol = 1e-5, eq_atol = 1e-12;
  double c_red = kbc::clight;
  std::string error_file = "KROME_ERROR_REPORT";
  // photon bins: the broadening of tabulated cross sections and the
  // in-bin spectrum dN/dE ~ E^-alpha
  double broad_T = 0.0, broad_vturb = 0.0, photo_alpha = 1.0;
  kbphoto::Bins photo;  // B = 0: no photon bins
};

namespace {

std::mutex g_mu;  // the device buffers of the host-array entry points

struct DevBuf {
  void* p = nullptr;
  size_t cap = 0;
  int dev = -1;
  cudaError_t ensure(size_t bytes) {
    int d = 0;
    cudaGetDevice(&d);
    if (p != nullptr && cap >= bytes && d == dev) return cudaSuccess;
    if (p != nullptr && d == dev) cudaFree(p);
    p = nullptr;
    cap = 0;
    const cudaError_t e = cudaMalloc(&p, bytes);
    if (e == cudaSuccess) {
      cap = bytes;
      dev = d;
    }
    return e;
  }
};
DevBuf g_buf;

// A host-array call's device staging: a buffer and a stream of its own.
// Concurrent host callers each take an idle slot -- the reference's
// private-buffer fallback for a busy device cache (solve_kokkos.hpp:
// 1223-1241) --, so their copies and kernels overlap on the GPU instead of
// queueing behind one lock. A slot is made on first need (per device) and
// kept for later calls; the pool holds as many slots as calls ever ran at
// once.
struct Slot {
  DevBuf buf;
  cudaStream_t stream = nullptr;
  int dev = -1;
  // pinned staging for the caller's pageable host arrays: a copy from or to
  // pageable memory goes through the driver's shared staging and blocks
  // other threads' copies (and with them their kernels); from pinned memory
  // each slot's copies run on its own stream
  void* pin = nullptr;
  size_t pin_cap = 0;
  cudaError_t ensure_pin(size_t bytes) {
    if (pin != nullptr && pin_cap >= bytes) return cudaSuccess;
    if (pin != nullptr) cudaFreeHost(pin);
    pin = nullptr;
    pin_cap = 0;
    const cudaError_t e = cudaHostAlloc(&pin, bytes, cudaHostAllocDefault);
    if (e == cudaSuccess) pin_cap = bytes;
    return e;
  }
};

// whether a host pointer is page-locked (pinned or registered) memory
bool host_pinned(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();  // clear the error of an unknown pointer
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

// a call's host<->device copies on its slot's stream: arrays in pinned
// memory directly, pageable ones through the slot's pinned staging (in on
// the way, out after the stream's synchronization: finish())
struct Xfer {
  Slot* slot;
  cudaStream_t s;
  size_t off = 0;
  struct Out { void* dst; size_t at, bytes; };
  std::vector<Out> outs;
  char* pin(size_t at) { return static_cast<char*>(slot->pin) + at; }
  size_t take(size_t bytes) {
    const size_t at = off;
    off += (bytes + 255) & ~(size_t)255;
    return at;
  }
  cudaError_t in(void* d, const void* h, size_t bytes) {
    if (bytes == 0) return cudaSuccess;
    if (host_pinned(h)) return cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, s);
    const size_t at = take(bytes);
    std::memcpy(pin(at), h, bytes);
    return cudaMemcpyAsync(d, pin(at), bytes, cudaMemcpyHostToDevice, s);
  }
  cudaError_t out(void* h, const void* d, size_t bytes) {
    if (bytes == 0) return cudaSuccess;
    if (host_pinned(h)) return cudaMemcpyAsync(h, d, bytes, cudaMemcpyDeviceToHost, s);
    const size_t at = take(bytes);
    outs.push_back(Out{h, at, bytes});
    return cudaMemcpyAsync(pin(at), d, bytes, cudaMemcpyDeviceToHost, s);
  }
  void finish() {  // after the stream's synchronization succeeded
    for (const Out& o : outs) std::memcpy(o.dst, pin(o.at), o.bytes);
  }
};
std::mutex g_slot_mu;
std::vector<Slot*> g_idle;
Slot* take_slot() {
  int d = 0;
  if (cudaGetDevice(&d) != cudaSuccess) return nullptr;
  {
    std::lock_guard<std::mutex> lk(g_slot_mu);
    for (size_t i = 0; i < g_idle.size(); ++i)
      if (g_idle[i]->dev == d) {
        Slot* s = g_idle[i];
        g_idle.erase(g_idle.begin() + i);
        return s;
      }
  }
  Slot* s = new Slot;
  s->dev = d;
  if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking)
      != cudaSuccess) {
    delete s;
    return nullptr;
  }
  return s;
}
struct SlotLease {
  Slot* s;
  SlotLease() : s(take_slot()) {}
  ~SlotLease() {
    if (s == nullptr) return;
    std::lock_guard<std::mutex> lk(g_slot_mu);
    g_idle.push_back(s);
  }
};

int resolved_jac(const krome_opts& h) {
  if (h.jac == 1) return 1;
  if (h.jac == 2) return 2;
  // JAC_AUTO (solve_cell.hpp:2141-2142): analytic at fixed Tgas, the
  // difference quotients when Tgas evolves
  return h.evolve_T ? 2 : 1;
}

SolveOpts to_solve_opts(const krome_opts& h) {
  SolveOpts so;
  so.evolve_T = h.evolve_T;
  so.jac = resolved_jac(h);
  so.rtol = h.rtol;
  so.atol_n = h.atol_n;
  so.atol_T = h.atol_T;
  so.max_steps = h.max_steps;
  so.max_err_fails = h.max_err_fails;
  so.max_conv_fails = h.max_conv_fails;
  so.max_restarts = h.max_restarts;
  so.clip_negative = h.clip_negative;
  so.fail_every = h.fail_every;
  so.lu32 = h.lu32;
  so.conserve = h.conserve;
  // a species' tolerance: its entry, or the scalar (solve_cell.hpp:868-879)
  auto tol = [](const std::vector<double>& v, int i, double s) {
    return !v.empty() && !(v[i] < 0.0) ? v[i] : s;
  };
  so.rtol_v = 0;
  for (int i = 0; i < kbw::KB_NSP_TOL; ++i) {
    so.atol_sp[i] = tol(h.atol_sp, i, h.atol_n);
    so.rtol_sp[i] = tol(h.rtol_sp, i, h.rtol);
    if (so.rtol_sp[i] != h.rtol) so.rtol_v = 1;
  }
  so.ph_sigma = nullptr;
  so.ph_phi = nullptr;
  so.ph_B = 0;
  return so;
}

// the photon field of a launch: the bins' cross sections and the cells'
// Phi rows, both on the device (B = 0: none)
struct PhotoArgs {
  const double* sigma = nullptr;
  const double* phi = nullptr;
  int B = 0;
};

int g_num_sms = 0;
int num_sms() {
  if (g_num_sms == 0) {
    int d = 0;
    cudaGetDevice(&d);
    cudaDeviceGetAttribute(&g_num_sms, cudaDevAttrMultiProcessorCount, d);
    if (g_num_sms <= 0) g_num_sms = 148;
  }
  return g_num_sms;
}

#ifdef KB_LARGE_NETWORK
// the large networks' per-block workspace: one device buffer, grown to
// `slots` slots when it is smaller (a cudaMalloc: not inside a stream
// capture, so graph_new grows it before capturing)
std::mutex g_ws_mu;
DevBuf g_ws;
double* big_workspace(long slots) {
  std::lock_guard<std::mutex> lk(g_ws_mu);
  const size_t bytes = (size_t)slots * kbg::WS::SIZE * sizeof(double);
  if (g_ws.p != nullptr && g_ws.cap >= bytes) return (double*)g_ws.p;
  if (g_ws.ensure(bytes) != cudaSuccess) return nullptr;
  return (double*)g_ws.p;
}
#endif

template <bool EVT>
cudaError_t launch(const krome_opts& h, int ncell, double* n, double* T,
                   const double* dt, const double* par, int pstride,
                   int* flags, long* stats, unsigned* cursor,
                   cudaStream_t stream, const RecIO* rio = nullptr,
                   const PhotoArgs& ph = PhotoArgs(),
                   const CellIO& io = CellIO()) {
  SolveOpts so = to_solve_opts(h);
  so.ph_sigma = ph.sigma;
  so.ph_phi = ph.phi;
  so.ph_B = ph.B;
#ifdef KB_LARGE_NETWORK
  // the sparse path: one block per cell over a persistent grid (one block
  // per SM: the dense block of the LU fills shared memory), each block with
  // its workspace slot (the library's device buffer, grown before a launch
  // when needed; never during a graph capture: big_workspace)
  (void)rio;
  if (cursor == nullptr) return cudaErrorInvalidValue;  // always the queue
  {
    static bool attr[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) return cudaErrorInvalidDevice;
    if (!attr[dev]) {
      const cudaError_t e = cudaFuncSetAttribute(
          kb_big_cells, cudaFuncAttributeMaxDynamicSharedMemorySize,
          (int)kbg::SMEM_BYTES);
      if (e != cudaSuccess) return e;
      attr[dev] = true;
    }
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kb_big_cells,
                                                  kbg::NT, kbg::SMEM_BYTES);
    if (per_sm <= 0) per_sm = 1;
    long blocks = (long)num_sms() * per_sm;
    if (h.blocks_per_sm > 0 && h.blocks_per_sm < per_sm)
      blocks = (long)num_sms() * h.blocks_per_sm;
    if (blocks > ncell) blocks = ncell > 0 ? ncell : 1;
    double* ws = big_workspace(blocks);
    if (ws == nullptr) return cudaErrorMemoryAllocation;
    cudaError_t e = cudaMemsetAsync(cursor, 0, sizeof(unsigned), stream);
    if (e != cudaSuccess) return e;
    kb_big_cells<<<(int)blocks, kbg::NT, kbg::SMEM_BYTES, stream>>>(
        ncell, n, T, dt, par, pstride, flags, stats, so, cursor, ws);
    return cudaGetLastError();
  }
#else
  if (h.layout == 1 || rio != nullptr) {  // lane per cell
    // a persistent grid of a small batch spreads its warps over the SMs
    // (blocks of as many warps as the batch fills on every SM, at least
    // one): each SM then holds few lanes, whose state stays in its L1, and
    // every SM takes part (4,096 cells in 4-warp blocks would run on 32 of
    // the 148 SMs)
    int warps = kWarpsPerBlock;
    if (h.kernel != 0 && ncell > 0) {
      const long fill = (long)ncell / (32L * num_sms());
      warps = fill < 1 ? 1 : (fill < kWarpsPerBlock ? (int)fill : kWarpsPerBlock);
    }
    const size_t lsmem = sizeof(double) * warps * LaneGeo<EVT>::SMEM_DOUBLES;
    const int threads = warps * 32;
    // register budget of the kernel: 2, 3 or 4 resident blocks per SM; the
    // adjoint's recording forward solve runs the 2-block build
    auto kern = rio != nullptr ? kb_lane_cells<EVT, 2, true>
              : h.lane_minb == 3 ? kb_lane_cells<EVT, 3, false>
              : h.lane_minb == 4 ? kb_lane_cells<EVT, 4, false>
                                 : kb_lane_cells<EVT, 2, false>;
    long blocks;
    if (h.kernel == 0) {
      blocks = ((long)ncell + threads - 1) / threads;
      if (blocks < 1) blocks = 1;  // ncell 0: an empty launch (warm-up)
    } else {
      int per_sm = h.blocks_per_sm;
      if (per_sm <= 0) {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads,
                                                      lsmem);
        if (per_sm <= 0) per_sm = 1;
      }
      blocks = (long)num_sms() * per_sm;
      const long need = ((long)ncell + threads - 1) / threads;
      if (blocks > need) blocks = need > 0 ? need : 1;
      cudaError_t e = cudaMemsetAsync(cursor, 0, sizeof(unsigned), stream);
      if (e != cudaSuccess) return e;
    }
    const RecIO none{nullptr, 0, nullptr, 0, nullptr, nullptr};
    kern<<<(int)blocks, threads, lsmem, stream>>>(
        ncell, n, T, dt, par, pstride, flags, stats, so, cursor, h.kernel,
        rio != nullptr ? *rio : none, io);
    return cudaGetLastError();
  }
  const size_t smem = sizeof(double) * kWarpsPerBlock * Geo<EVT>::SMEM_DOUBLES;
  if (h.kernel == 0) {
    int blocks = (ncell + kWarpsPerBlock - 1) / kWarpsPerBlock;
    if (blocks < 1) blocks = 1;  // ncell 0: an empty launch (warm-up)
    kb_cells_plain<EVT><<<blocks, kWarpsPerBlock * 32, smem, stream>>>(
        ncell, n, T, dt, par, pstride, flags, stats, so);
    return cudaGetLastError();
  }
  int per_sm = h.blocks_per_sm;
  if (per_sm <= 0) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(
        &per_sm, kb_cells_persistent<EVT>, kWarpsPerBlock * 32, smem);
    if (per_sm <= 0) per_sm = 1;
  }
  const int chunk = h.queue_chunk > 0 ? h.queue_chunk : 1;
  long blocks = (long)num_sms() * per_sm;
  const long need = ((long)ncell + (long)kWarpsPerBlock * chunk - 1)
                    / ((long)kWarpsPerBlock * chunk);
  if (blocks > need) blocks = need > 0 ? need : 1;
  cudaError_t e = cudaMemsetAsync(cursor, 0, sizeof(unsigned), stream);
  if (e != cudaSuccess) return e;
  kb_cells_persistent<EVT><<<(int)blocks, kWarpsPerBlock * 32, smem, stream>>>(
      ncell, n, T, dt, par, pstride, flags, stats, so, cursor, chunk);
  return cudaGetLastError();
#endif
}

cudaError_t launch_any(const krome_opts& h, int ncell, double* n, double* T,
                       const double* dt, const double* par, int pstride,
                       int* flags, long* stats, unsigned* cursor,
                       cudaStream_t stream,
                       const PhotoArgs& ph = PhotoArgs(),
                       const CellIO& io = CellIO()) {
  return h.evolve_T
      ? launch<true>(h, ncell, n, T, dt, par, pstride, flags, stats, cursor,
                     stream, nullptr, ph, io)
      : launch<false>(h, ncell, n, T, dt, par, pstride, flags, stats, cursor,
                      stream, nullptr, ph, io);
}

// whether a launch of these options reads and writes the caller's layout
// itself (the lane-per-cell kernel); the other kernels take cell-major
// densities
bool fuses_io(const krome_opts& h) {
#ifdef KB_LARGE_NETWORK
  (void)h;
  return false;
#else
  return h.layout == 1;
#endif
}

bool row_missing(const double* row) {
  kbnet::Params p;
  kbnet::params_from_row(row, p);
  return kbnet::params_missing(p) >= 0;
}

// the required-parameter rule (solve_cells.hpp:133-140): any cell whose
// row misses a REQUIRED parameter rejects the whole call
int check_params(int ncell, const double* par, int stride, int* flags) {
  bool missing = false;
  for (int c = 0; c < ncell; ++c) {
    const bool m = row_missing(par + (long)c * stride);
    if (flags != nullptr) flags[c] = m ? -105 : 0;
    missing |= m;
  }
  return missing ? -105 : 0;
}

}  // namespace

// ---------------------------------------------------------------------------
// network description

KB_API const char* krome_version(void) { return "krome-b200 0.1 (sm_100a)"; }
KB_API const char* krome_network_name(void) { return kbnet::NETWORK_NAME; }
KB_API int krome_nspec(void) { return kbnet::NSPEC; }
KB_API int krome_nrea(void) { return kbnet::NREA; }
KB_API int krome_npar(void) { return kbnet::NPAR; }
KB_API const char* krome_species_name(int i) {
  return (i >= 0 && i < kbnet::NSPEC) ? kbnet::species_names[i] : nullptr;
}
KB_API int krome_species_index(const char* name) {
  if (name == nullptr) return -1;
  for (int i = 0; i < kbnet::NSPEC; ++i)
    if (!std::strcmp(kbnet::species_names[i], name)) return i;
  return -1;
}
KB_API const char* krome_param_name(int i) {
  return (i >= 0 && i < kbnet::NPAR) ? kbnet::param_names[i] : nullptr;
}
KB_API int krome_param_index(const char* name) {
  if (name == nullptr) return -1;
  for (int i = 0; i < kbnet::NPAR; ++i)
    if (!std::strcmp(kbnet::param_names[i], name)) return i;
  return -1;
}
KB_API void krome_params_default(double* par) {
  for (int i = 0; i < kbnet::NPAR; ++i) par[i] = kbnet::param_default(i);
}
KB_API const char* krome_param_required_by(int i) {
  return (i >= 0 && i < kbnet::NPAR) ? kbnet::param_required_by[i] : nullptr;
}

KB_API const char* krome_flag_message(int flag) {
  switch (flag) {
    case 0: return "success";
    case -1: return "max_steps exhausted before t_end (FLAG_TOO_MUCH_WORK)";
    case -2: return "tolerances too small for machine precision (FLAG_TOO_MUCH_ACC)";
    case -3: return "repeated error-test failures (FLAG_ERR_FAILURE)";
    case -4: return "repeated Newton convergence failures (FLAG_CONV_FAILURE)";
    case -6: return "Newton matrix setup / factorization failed (FLAG_LSETUP_FAIL)";
    case -7: return "linear solve failed (FLAG_LSOLVE_FAIL)";
    case -8: return "right-hand side failed (FLAG_RHSFUNC_FAIL)";
    case -9: return "right-hand side failed at the initial state (FLAG_FIRST_RHSFUNC_ERR)";
    case -10: return "repeated recoverable right-hand side errors (FLAG_REPTD_RHSFUNC_ERR)";
    case -11: return "right-hand side failed unrecoverably (FLAG_UNREC_RHSFUNC_ERR)";
    case -16: return "nonlinear solver failure (FLAG_NLS_FAIL)";
    case -22: return "illegal input (FLAG_ILL_INPUT)";
    case -27: return "t_end too close to the start (FLAG_TOO_CLOSE)";
    case -104: return "configuration not supported by this library, or no usable GPU (FLAG_UNSUPPORTED)";
    case -105: return "a required parameter is unset (NaN)";
    case -110: return "the integration ended at a non-positive or non-finite Tgas (input untouched)";
    case -111: return "device path: the cells do not fit in the device memory (FLAG_DEVICE_MEMORY)";
    case -120: return "adjoint: the cell's tape outgrew its capacity (no gradient; input untouched)";
    default: break;
  }
  return flag <= -100 ? "unknown KROME flag" : "integrator failure";
}

// ---------------------------------------------------------------------------
// options

KB_API krome_opts* krome_opts_new(void) { return new krome_opts(); }
KB_API void krome_opts_free(krome_opts* h) { delete h; }

namespace {
int* int_key(krome_opts* h, const char* k) {
  static const struct { const char* name; size_t off; } keys[] = {
      {"evolve_T", offsetof(krome_opts, evolve_T)},
      {"clip_negative", offsetof(krome_opts, clip_negative)},
      {"error_report", offsetof(krome_opts, error_report)},
      {"renormalize_x", offsetof(krome_opts, renormalize_x)},
      {"max_err_fails", offsetof(krome_opts, max_err_fails)},
      {"max_conv_fails", offsetof(krome_opts, max_conv_fails)},
      {"max_restarts", offsetof(krome_opts, max_restarts)},
      {"conserve", offsetof(krome_opts, conserve)},
      {"path", offsetof(krome_opts, path)},
      {"device_cache", offsetof(krome_opts, device_cache)},
      {"min_device", offsetof(krome_opts, min_device)},
      {"min_interleave", offsetof(krome_opts, min_interleave)},
      {"jac", offsetof(krome_opts, jac)},
      {"linsol", offsetof(krome_opts, linsol)},
      {"kernel", offsetof(krome_opts, kernel)},
      {"layout", offsetof(krome_opts, layout)},
      {"lane_minb", offsetof(krome_opts, lane_minb)},
      {"queue_chunk", offsetof(krome_opts, queue_chunk)},
      {"blocks_per_sm", offsetof(krome_opts, blocks_per_sm)},
      {"fail_every", offsetof(krome_opts, fail_every)},
      {"lu32", offsetof(krome_opts, lu32)},
  };
  for (const auto& e : keys)
    if (!std::strcmp(e.name, k))
      return reinterpret_cast<int*>(reinterpret_cast<char*>(h) + e.off);
  return nullptr;
}
double* dbl_key(krome_opts* h, const char* k) {
  if (!std::strcmp(k, "eq_t0")) return &h->eq_t0;
  if (!std::strcmp(k, "eq_tmax")) return &h->eq_tmax;
  if (!std::strcmp(k, "eq_factor")) return &h->eq_factor;
  if (!std::strcmp(k, "eq_rtol")) return &h->eq_rtol;
  if (!std::strcmp(k, "eq_atol")) return &h->eq_atol;
  if (!std::strcmp(k, "c_red")) return &h->c_red;
  if (!std::strcmp(k, "rtol")) return &h->rtol;
  if (!std::strcmp(k, "atol_n")) return &h->atol_n;
  if (!std::strcmp(k, "atol_T")) return &h->atol_T;
  if (!std::strcmp(k, "atol_u")) return &h->atol_u;
  return nullptr;
}
bool bool_key(const char* k) {
  return !std::strcmp(k, "evolve_T") || !std::strcmp(k, "clip_negative")
         || !std::strcmp(k, "error_report") || !std::strcmp(k, "renormalize_x")
         || !std::strcmp(k, "device_cache") || !std::strcmp(k, "lu32");
}
}  // namespace

KB_API int krome_opts_set(krome_opts* h, const char* key, double v) {
  if (h == nullptr || key == nullptr) return -1;
  if (double* d = dbl_key(h, key)) {
    *d = v;
    return 0;
  }
  if (!std::strcmp(key, "max_steps")) {
    h->max_steps = (long)v;
    return 0;
  }
  if (!std::strcmp(key, "device_memory")) {
    h->device_memory = (long long)v;
    return 0;
  }
  int* iv = int_key(h, key);
  if (iv == nullptr) return -1;
  if (bool_key(key)) {
    *iv = v != 0.0;
    return 0;
  }
  const int x = (int)v;
  if (!std::strcmp(key, "jac") && (x < 0 || x > 2)) return -1;
  if (!std::strcmp(key, "linsol") && (x < 0 || x > 3)) return -1;
  if (!std::strcmp(key, "path") && (x < 0 || x > 2)) return -1;
  if (!std::strcmp(key, "conserve") && (x < 0 || x > 3)) return -1;
  if (!std::strcmp(key, "kernel") && (x < 0 || x > 1)) return -1;
  if (!std::strcmp(key, "layout") && (x < 0 || x > 1)) return -1;
  if (!std::strcmp(key, "lane_minb") && (x < 2 || x > 4)) return -1;
  if ((!std::strcmp(key, "max_err_fails") || !std::strcmp(key, "max_conv_fails")
       || !std::strcmp(key, "max_restarts") || !std::strcmp(key, "queue_chunk")
       || !std::strcmp(key, "fail_every") || !std::strcmp(key, "blocks_per_sm"))
      && v < 0.0)
    return -1;
  *iv = x;
  return 0;
}

// per-species tolerances (reference krome.h:175-185, krome.cpp:494-538):
// v[NSPEC] copied into the handle (a negative entry: the scalar; NULL: the
// scalar for every species); NaN, and a zero atol, are rejected. get writes
// the tolerance each species gets.
namespace {
int set_species_tol(krome_opts* h, const double* v, bool atol) {
  if (h == nullptr) return -1;
  std::vector<double>& buf = atol ? h->atol_sp : h->rtol_sp;
  if (v == nullptr) {
    buf.clear();
    return 0;
  }
  for (int i = 0; i < kbnet::NSPEC; ++i)
    if (std::isnan(v[i]) || (atol && v[i] == 0.0)) return -1;
  buf.assign(v, v + kbnet::NSPEC);
  return 0;
}
int get_species_tol(const krome_opts* h, double* v, bool atol) {
  if (h == nullptr || v == nullptr) return -1;
  const std::vector<double>& buf = atol ? h->atol_sp : h->rtol_sp;
  const double s = atol ? h->atol_n : h->rtol;
  for (int i = 0; i < kbnet::NSPEC; ++i)
    v[i] = !buf.empty() && !(buf[i] < 0.0) ? buf[i] : s;
  return 0;
}
}  // namespace
KB_API int krome_opts_set_atol_species(krome_opts* h, const double* atol) {
  return set_species_tol(h, atol, true);
}
KB_API int krome_opts_set_rtol_species(krome_opts* h, const double* rtol) {
  return set_species_tol(h, rtol, false);
}
KB_API int krome_opts_get_atol_species(const krome_opts* h, double* atol) {
  return get_species_tol(h, atol, true);
}
KB_API int krome_opts_get_rtol_species(const krome_opts* h, double* rtol) {
  return get_species_tol(h, rtol, false);
}

KB_API int krome_opts_get(const krome_opts* hc, const char* key, double* v) {
  if (hc == nullptr || key == nullptr || v == nullptr) return -1;
  auto* h = const_cast<krome_opts*>(hc);
  if (double* d = dbl_key(h, key)) {
    *v = *d;
    return 0;
  }
  if (!std::strcmp(key, "max_steps")) {
    *v = (double)h->max_steps;
    return 0;
  }
  if (!std::strcmp(key, "device_memory")) {
    *v = (double)h->device_memory;
    return 0;
  }
  if (int* iv = int_key(h, key)) {
    *v = (double)*iv;
    return 0;
  }
  return -1;
}

#include "kb_queries.h"

// ---------------------------------------------------------------------------
// the solves

namespace {
// what this library does not implement returns FLAG_UNSUPPORTED before any
// work: LAPACK and the sparse LU (small networks use the dense LU), photon
// bins; the FP32 Newton-matrix form exists in the lane layout only
int unsupported(const krome_opts& h) {
#ifdef KB_LARGE_NETWORK
  // the large networks: the sparse LU (linsol auto or sparse), FP64, the
  // scalar tolerances; an evolved Tgas (the Newton matrix's Tgas border)
  // with the analytic (hybrid) Jacobian on networks without thermal
  // processes (dT/dt identically zero): the difference quotients over every
  // column (JAC_AUTO's choice with evolve_T) are not built for them
  if (h.linsol == 1 || h.linsol == 2) return -104;
  if (!h.atol_sp.empty() || !h.rtol_sp.empty()) return -104;
  if (h.lu32 != 0) return -104;
  if (h.evolve_T != 0 && (kbnet::HAS_THERMAL_TERMS || resolved_jac(h) != 1))
    return -104;
#else
  if (h.linsol == 2 || h.linsol == 3) return -104;
  if (h.lu32 != 0 && h.layout != 1) return -104;
#endif
  return 0;
}
}  // namespace

KB_API int krome_b200_solve_device(int ncell, double* n, double* Tgas,
                                   const double* dt, const double* par,
                                   int par_stride, int* flags, long* stats,
                                   unsigned* cursor, const krome_opts* h,
                                   void* stream) {
  if (h == nullptr || ncell < 0) return -1;
  if (ncell == 0) return 0;
  if (n == nullptr || Tgas == nullptr || dt == nullptr || par == nullptr
      || flags == nullptr)
    return -1;
  if (par_stride != 0 && par_stride != kbnet::NPAR) return -1;
#ifdef KB_LARGE_NETWORK
  if (cursor == nullptr) return -1;  // the large path always takes the queue
#endif
  if (cursor == nullptr && (h->kernel == 1)) return -1;
  if (const int u = unsupported(*h)) return u;
  // photon bins need each cell's field: krome_solve_cells(_device) take it
  if (h->photo.B > 0) return -103;
  const cudaError_t e = launch_any(*h, ncell, n, Tgas, dt, par, par_stride,
                                   flags, stats, cursor,
                                   static_cast<cudaStream_t>(stream));
  return e == cudaSuccess ? 0 : -104;
}

// ---- the discrete adjoint (adjoint.cuh) ----

KB_API int krome_has_device(void);

KB_API int krome_b200_adjoint_record_device(
    int ncell, double* n, double* Tgas, const double* dt, const double* par,
    int par_stride, const double* mult, int mult_stride, int* flags,
    long* stats, unsigned* cursor, double* tape, long tape_cap,
    long* tape_len, double* yfin, const krome_opts* h, void* stream) {
  if (h == nullptr || ncell < 0) return -1;
#ifdef KB_LARGE_NETWORK
  (void)n; (void)Tgas; (void)dt; (void)par; (void)par_stride; (void)mult;
  (void)mult_stride; (void)flags; (void)stats; (void)cursor; (void)tape;
  (void)tape_cap; (void)tape_len; (void)yfin; (void)stream;
  return -104;  // the adjoint is built for the small (dense) networks
#else
  if (ncell == 0) return 0;
  // tape NULL: a counting solve (tape_len the tape each cell needs)
  if (n == nullptr || Tgas == nullptr || dt == nullptr || par == nullptr
      || flags == nullptr || tape_len == nullptr || yfin == nullptr
      || (tape != nullptr && tape_cap <= 0))
    return -1;
  if (par_stride != 0 && par_stride != kbnet::NPAR) return -1;
  if (mult_stride != 0 && mult_stride != kbnet::NREA) return -1;
  if (cursor == nullptr && h->kernel == 1) return -1;
  if (h->linsol == 2 || h->linsol == 3 || h->conserve != 0) return -104;
  if (h->photo.B > 0) return -104;  // no adjoint of the photo rates
  const RecIO rio{mult, mult_stride, tape, tape_cap, tape_len, yfin};
  const cudaStream_t st = static_cast<cudaStream_t>(stream);
  const cudaError_t e =
      h->evolve_T ? launch<true>(*h, ncell, n, Tgas, dt, par, par_stride, flags,
                                 stats, cursor, st, &rio)
                  : launch<false>(*h, ncell, n, Tgas, dt, par, par_stride,
                                  flags, stats, cursor, st, &rio);
  return e == cudaSuccess ? 0 : -104;
#endif
}

KB_API int krome_b200_adjoint_device(
    int ncell, const double* T0, const double* par, int par_stride,
    const double* mult, int mult_stride, const double* gn, const double* gT,
    const int* flags, const double* tape, long tape_cap,
    const long* tape_len, const double* yfin, double* dn0, double* dT0,
    double* dm, unsigned* cursor, const krome_opts* h, void* stream) {
  if (h == nullptr || ncell < 0) return -1;
#ifdef KB_LARGE_NETWORK
  (void)T0; (void)par; (void)par_stride; (void)mult; (void)mult_stride;
  (void)gn; (void)gT; (void)flags; (void)tape; (void)tape_cap;
  (void)tape_len; (void)yfin; (void)dn0; (void)dT0; (void)dm; (void)cursor;
  (void)stream;
  return -104;  // the adjoint is built for the small (dense) networks
#else
  if (ncell == 0) return 0;
  if (T0 == nullptr || par == nullptr || gn == nullptr || flags == nullptr
      || tape == nullptr || tape_len == nullptr || yfin == nullptr
      || dn0 == nullptr || dm == nullptr || cursor == nullptr || tape_cap <= 0)
    return -1;
  if (par_stride != 0 && par_stride != kbnet::NPAR) return -1;
  if (mult_stride != 0 && mult_stride != kbnet::NREA) return -1;
  const cudaStream_t st = static_cast<cudaStream_t>(stream);
  auto kern = h->evolve_T ? kba::kb_adjoint_cells<true>
                          : kba::kb_adjoint_cells<false>;
  // a persistent grid over the work queue
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 128, 0);
  if (per_sm <= 0) per_sm = 1;
  long blocks = (long)num_sms() * per_sm;
  const long need = ((long)ncell + 127) / 128;
  if (blocks > need) blocks = need;
  if (cudaMemsetAsync(cursor, 0, sizeof(unsigned), st) != cudaSuccess)
    return -104;
  kern<<<(int)blocks, 128, 0, st>>>(ncell, T0, par, par_stride, mult,
                                    mult_stride, gn, gT, flags, tape, tape_cap,
                                    tape_len, yfin, h->clip_negative, dn0, dT0,
                                    dm, cursor);
  return cudaGetLastError() == cudaSuccess ? 0 : -104;
#endif
}

KB_API int krome_b200_adjoint(int ncell, double* n, double* Tgas,
                              const double* dt, const double* par,
                              int par_stride, const double* lnm,
                              int lnm_stride, const double* gn,
                              const double* gT, int* flags, double* dn0,
                              double* dT0, double* dm, long tape_cap,
                              const krome_opts* h) {
  using namespace kbnet;
  if (h == nullptr || ncell < 0 || n == nullptr || Tgas == nullptr
      || dt == nullptr || gn == nullptr || dn0 == nullptr || dm == nullptr)
    return -1;
  if (par != nullptr && par_stride != 0 && par_stride != NPAR) return -1;
  if (lnm != nullptr && lnm_stride != 0 && lnm_stride != NREA) return -1;
  if (ncell == 0) return 0;
  std::vector<double> dflt(NPAR);
  krome_params_default(dflt.data());
  const double* P = par != nullptr ? par : dflt.data();
  const int ps = par != nullptr ? par_stride : 0;
  std::vector<int> fl(ncell, 0);
  int* fo = flags != nullptr ? flags : fl.data();
  if (check_params(ncell, P, ps, fo) != 0) return -105;
  if (h->linsol == 2 || h->linsol == 3 || h->conserve != 0 || h->photo.B > 0) {
    for (int c = 0; c < ncell; ++c) fo[c] = -104;
    return -104;
  }
  if (!krome_has_device()) {
    for (int c = 0; c < ncell; ++c) fo[c] = -104;
    return -104;
  }
  const long cap = tape_cap > 0 ? tape_cap : 32768;
  const int N = NSPEC + (h->evolve_T ? 1 : 0);
  const long prow = ps == 0 ? 1 : ncell;
  const long mrows = lnm == nullptr ? 0 : (lnm_stride == 0 ? 1 : ncell);
  std::vector<double> mult(mrows * NREA);
  for (long i = 0; i < mrows * NREA; ++i) mult[i] = std::exp(lnm[i]);
  // device buffers: n T T0 dt par mult gn gT yfin dn0 dT0 dm tape (+ ints)
  const size_t nd = (size_t)ncell * NSPEC;
  const size_t dbl = 2 * nd + 3 * (size_t)ncell + prow * NPAR + mrows * NREA
                     + nd + ncell + (size_t)ncell * N + nd + ncell
                     + (size_t)ncell * NREA;
  double* d = nullptr;
  long* dlen = nullptr;
  int* dfl = nullptr;
  unsigned* dcur = nullptr;
  double* dtape = nullptr;
  auto release = [&]() {
    cudaFree(d);
    cudaFree(dlen);
    cudaFree(dfl);
    cudaFree(dcur);
    cudaFree(dtape);
  };
  if (cudaMalloc(&d, dbl * sizeof(double)) != cudaSuccess
      || cudaMalloc(&dlen, (size_t)ncell * sizeof(long)) != cudaSuccess
      || cudaMalloc(&dfl, (size_t)ncell * sizeof(int)) != cudaSuccess
      || cudaMalloc(&dcur, sizeof(unsigned)) != cudaSuccess
      || cudaMalloc(&dtape, (size_t)ncell * cap * sizeof(double))
             != cudaSuccess) {
    release();
    cudaGetLastError();
    for (int c = 0; c < ncell; ++c) fo[c] = -111;
    return -111;
  }
  double* dn = d;
  double* dT = dn + nd;
  double* dT0v = dT + ncell;
  double* ddt = dT0v + ncell;
  double* dpar = ddt + ncell;
  double* dmult = dpar + prow * NPAR;
  double* dgn = dmult + mrows * NREA;
  double* dgT = dgn + nd;
  double* dyf = dgT + ncell;
  double* ddn0 = dyf + (size_t)ncell * N;
  double* ddT0 = ddn0 + nd;
  double* ddm = ddT0 + ncell;
  std::vector<double> zero(ncell, 0.0);
  cudaMemcpy(dn, n, nd * sizeof(double), cudaMemcpyHostToDevice);
  cudaMemcpy(dT, Tgas, ncell * sizeof(double), cudaMemcpyHostToDevice);
  cudaMemcpy(dT0v, Tgas, ncell * sizeof(double), cudaMemcpyHostToDevice);
  cudaMemcpy(ddt, dt, ncell * sizeof(double), cudaMemcpyHostToDevice);
  cudaMemcpy(dpar, P, prow * NPAR * sizeof(double), cudaMemcpyHostToDevice);
  if (mrows > 0)
    cudaMemcpy(dmult, mult.data(), mrows * NREA * sizeof(double),
               cudaMemcpyHostToDevice);
  cudaMemcpy(dgn, gn, nd * sizeof(double), cudaMemcpyHostToDevice);
  cudaMemcpy(dgT, gT != nullptr ? gT : zero.data(), ncell * sizeof(double),
             cudaMemcpyHostToDevice);
  int r = krome_b200_adjoint_record_device(
      ncell, dn, dT, ddt, dpar, ps, mrows > 0 ? dmult : nullptr,
      mrows > 1 ? NREA : 0, dfl, nullptr, dcur, dtape, cap, dlen, dyf, h,
      nullptr);
  if (r == 0)
    r = krome_b200_adjoint_device(ncell, dT0v, dpar, ps,
                                  mrows > 0 ? dmult : nullptr,
                                  mrows > 1 ? NREA : 0, dgn, dgT, dfl, dtape,
                                  cap, dlen, dyf, ddn0, ddT0, ddm, dcur, h,
                                  nullptr);
  if (r == 0 && cudaDeviceSynchronize() != cudaSuccess) r = -104;
  if (r == 0) {
    cudaMemcpy(n, dn, nd * sizeof(double), cudaMemcpyDeviceToHost);
    cudaMemcpy(Tgas, dT, ncell * sizeof(double), cudaMemcpyDeviceToHost);
    cudaMemcpy(fo, dfl, ncell * sizeof(int), cudaMemcpyDeviceToHost);
    cudaMemcpy(dn0, ddn0, nd * sizeof(double), cudaMemcpyDeviceToHost);
    if (dT0 != nullptr)
      cudaMemcpy(dT0, ddT0, ncell * sizeof(double), cudaMemcpyDeviceToHost);
    cudaMemcpy(dm, ddm, (size_t)ncell * NREA * sizeof(double),
               cudaMemcpyDeviceToHost);
    if (cudaGetLastError() != cudaSuccess) r = -104;
  }
  release();
  if (r != 0) {
    for (int c = 0; c < ncell; ++c) fo[c] = r;
    return r;
  }
  for (int c = 0; c < ncell; ++c)
    if (fo[c] != 0) return fo[c];
  return 0;
}

namespace {
// the host-array solve: krome_b200_solve_batch, and krome_solve_cells with
// the photon field phi[ncell][nbins] of its extra rows (required with photon
// bins on the handle: -103 without)
int solve_host(int ncell, double* n, double* Tgas, const double* dt,
               const double* par, int par_stride, const double* phi,
               int* flags, long* stats, const krome_opts* h) {
  if (h == nullptr || ncell < 0 || n == nullptr || Tgas == nullptr
      || dt == nullptr)
    return -1;
  if (par != nullptr && par_stride != 0 && par_stride != kbnet::NPAR)
    return -1;
  if (ncell == 0) return 0;
  std::vector<double> dflt(kbnet::NPAR);
  krome_params_default(dflt.data());
  const double* P = par != nullptr ? par : dflt.data();
  const int ps = par != nullptr ? par_stride : 0;
  std::vector<int> fl(ncell, 0);
  if (check_params(ncell, P, ps, flags != nullptr ? flags : fl.data()) != 0)
    return -105;
  int u = unsupported(*h);
  const int B = h->photo.B;
  if (u == 0 && B > 0 && phi == nullptr) u = -103;  // bins without a field
  if (u != 0) {
    if (flags != nullptr)
      for (int c = 0; c < ncell; ++c) flags[c] = u;
    return u;
  }
  const size_t nb = sizeof(double) * (size_t)ncell * kbnet::NSPEC;
  const size_t tb = sizeof(double) * (size_t)ncell;
  const size_t pb = sizeof(double) * (size_t)(ps ? (size_t)ncell * ps : kbnet::NPAR);
  const size_t fb = sizeof(int) * (size_t)ncell;
  const size_t sb = stats != nullptr ? sizeof(long) * (size_t)ncell * NSTAT : 0;
  const size_t xb = B > 0 ? sizeof(double) * (size_t)kbnet::NPHOTO * B : 0;
  const size_t hb = B > 0 ? sizeof(double) * (size_t)ncell * B : 0;
  auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
  const size_t total = al(nb) + 2 * al(tb) + al(pb) + al(fb) + al(sb)
                       + al(xb) + al(hb) + 256;
  SlotLease lease;
  // the staging the pageable arrays may need: in (n, Tgas, dt, par, Phi),
  // out (n, Tgas, flags, stats)
  const size_t stage = al(nb) + 2 * al(tb) + al(pb) + al(xb) + al(hb)
                       + al(nb) + al(tb) + al(fb) + al(sb);
  if (lease.s == nullptr || lease.s->buf.ensure(total) != cudaSuccess
      || lease.s->ensure_pin(stage) != cudaSuccess) {
    if (flags != nullptr)
      for (int c = 0; c < ncell; ++c) flags[c] = -111;
    return -111;
  }
  char* b = static_cast<char*>(lease.s->buf.p);
  double* dn = reinterpret_cast<double*>(b); b += al(nb);
  double* dT = reinterpret_cast<double*>(b); b += al(tb);
  double* ddt = reinterpret_cast<double*>(b); b += al(tb);
  double* dp = reinterpret_cast<double*>(b); b += al(pb);
  int* dfl = reinterpret_cast<int*>(b); b += al(fb);
  long* dst = sb ? reinterpret_cast<long*>(b) : nullptr; b += al(sb);
  double* dxs = reinterpret_cast<double*>(b); b += al(xb);
  double* dphi = reinterpret_cast<double*>(b); b += al(hb);
  unsigned* dcur = reinterpret_cast<unsigned*>(b);
  cudaStream_t s = lease.s->stream;
  Xfer x{lease.s, s};
  cudaError_t e = x.in(dn, n, nb);
  if (e == cudaSuccess) e = x.in(dT, Tgas, tb);
  if (e == cudaSuccess) e = x.in(ddt, dt, tb);
  if (e == cudaSuccess) e = x.in(dp, P, pb);
  PhotoArgs pa;
  if (B > 0) {
    if (e == cudaSuccess) e = x.in(dxs, h->photo.sigma.data(), xb);
    if (e == cudaSuccess) e = x.in(dphi, phi, hb);
    pa = PhotoArgs{dxs, dphi, B};
  }
  if (e == cudaSuccess)
    e = launch_any(*h, ncell, dn, dT, ddt, dp, ps, dfl, dst, dcur, s, pa);
  if (e == cudaSuccess) e = x.out(n, dn, nb);
  if (e == cudaSuccess) e = x.out(Tgas, dT, tb);
  int* hfl = flags != nullptr ? flags : fl.data();
  if (e == cudaSuccess) e = x.out(hfl, dfl, fb);
  if (e == cudaSuccess && sb) e = x.out(stats, dst, sb);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    std::fprintf(stderr, "krome_b200: CUDA error %s\n", cudaGetErrorString(e));
    return -104;
  }
  x.finish();
  for (int c = 0; c < ncell; ++c)
    if (hfl[c] != 0) return hfl[c];
  return 0;
}
}  // namespace

// ---- the equilibrium driver (reference krome.h:366-376, krome.cpp:
// 574-617, solve_equilibrium at solve_cell.hpp:2249-2301) ----
//
// Every cell integrates to steady state in intervals: outputs at t0,
// t0 factor, t0 factor^2, ... (each interval a full solve of the cell from
// its current state), converged when max_i |dn_i| / max(n_i, eatol ntot)
// (and |dTgas| / Tgas with evolve_T) between two outputs is below ertol,
// stopped (flag 1, the state returned) at t_max, or failed (a negative
// flag, the input restored). On the GPU all cells advance together: each
// interval is one launch of the solve over the batch, in which the cells
// already done have dt 0 and are skipped, bracketed by two small kernels
// that keep the per-cell bookkeeping on the device.
namespace {
struct EqCells {
  double* nin;   // [ncell][nspec] the input, restored on failure
  double* Tin;
  double* prev;  // the state before the interval
  double* Tprev;
  double* t;     // the time integrated
  double* dt;    // the next interval
  int* state;    // 0 integrating, 1 done
  int* out;      // the cell's flag
};
struct EqOpts {
  double t0, tmax, factor, rtol, atol;
  int evolve_T;
};

__global__ void kb_eq_init(int ncell, const double* n, const double* T,
                           EqCells e, double t0) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncell) return;
  for (int i = 0; i < kbnet::NSPEC; ++i)
    e.nin[(long)c * kbnet::NSPEC + i] = n[(long)c * kbnet::NSPEC + i];
  e.Tin[c] = T[c];
  e.t[c] = 0.0;
  e.dt[c] = t0;
  e.state[c] = 0;
  e.out[c] = 0;
}

__global__ void kb_eq_pre(int ncell, const double* n, const double* T,
                          EqCells e) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncell) return;
  if (e.state[c] != 0) {
    e.dt[c] = 0.0;  // done: the solve skips the cell
    return;
  }
  for (int i = 0; i < kbnet::NSPEC; ++i)
    e.prev[(long)c * kbnet::NSPEC + i] = n[(long)c * kbnet::NSPEC + i];
  e.Tprev[c] = T[c];
}

__global__ void kb_eq_post(int ncell, double* n, double* T, const int* fl,
                           EqCells e, EqOpts q, unsigned* active) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncell || e.state[c] != 0) return;
  double* nc = n + (long)c * kbnet::NSPEC;
  if (fl[c] != 0) {  // failed: the input back
    for (int i = 0; i < kbnet::NSPEC; ++i)
      nc[i] = e.nin[(long)c * kbnet::NSPEC + i];
    T[c] = e.Tin[c];
    e.out[c] = fl[c];
    e.state[c] = 1;
    return;
  }
  const double t = e.t[c] + e.dt[c];
  e.t[c] = t;
  const double floor = q.atol * kbnet::ntot_(nc);
  double w = q.evolve_T ? fabs(T[c] - e.Tprev[c]) / T[c] : 0.0;
  for (int i = 0; i < kbnet::NSPEC; ++i)
    w = fmax(w, fabs(nc[i] - e.prev[(long)c * kbnet::NSPEC + i])
                    / fmax(nc[i], floor));
  if (w < q.rtol) {
    e.out[c] = 0;
    e.state[c] = 1;
  } else if (t >= q.tmax) {
    e.out[c] = 1;
    e.state[c] = 1;
  } else {
    e.dt[c] = fmin((q.factor - 1.0) * t, q.tmax - t);
    atomicAdd(active, 1u);
  }
}
}  // namespace

// host arrays in place, the krome_solve_cells conventions; handle keys
// eq_t0, eq_tmax, eq_factor, eq_rtol, eq_atol; flags[c] 0 converged, 1
// t_max reached first (state returned), < 0 failed (cell untouched).
// Returns the flag of the first cell that did not converge (0 if all did).
KB_API int krome_equilibrium_cells(int ncell, double* n, double* Tgas,
                                   const double* par, int par_stride,
                                   const krome_cells* extra, int* flags,
                                   const krome_opts* h) {
  using namespace kbnet;
  if (h == nullptr || Tgas == nullptr || ncell < 0 || n == nullptr) return -1;
  if (par != nullptr && par_stride != 0 && par_stride != NPAR) return -1;
  const int B = h->photo.B;
  const double* phi = extra != nullptr ? extra->Phi : nullptr;
  if (B > 0 && phi == nullptr) return -103;
  if (ncell == 0) return 0;
  const int u = unsupported(*h);
  if (u != 0) {
    if (flags != nullptr)
      for (int c = 0; c < ncell; ++c) flags[c] = u;
    return u;
  }
  std::vector<double> dflt(NPAR);
  krome_params_default(dflt.data());
  const double* P = par != nullptr ? par : dflt.data();
  const int ps = par != nullptr ? par_stride : 0;
  const size_t nb = sizeof(double) * (size_t)ncell * NSPEC;
  const size_t tb = sizeof(double) * (size_t)ncell;
  const size_t ib = sizeof(int) * (size_t)ncell;
  const size_t pb = sizeof(double) * (ps ? (size_t)ncell * ps : (size_t)NPAR);
  const size_t xb = B > 0 ? sizeof(double) * (size_t)NPHOTO * B : 0;
  const size_t hb = B > 0 ? sizeof(double) * (size_t)ncell * B : 0;
  auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
  // n, T, dt, par, flags, cursor + counter, nin, Tin, prev, Tprev, t,
  // state, out, photon tables
  const size_t total = 3 * al(nb) + 6 * al(tb) + al(pb) + 3 * al(ib) + 256
                       + al(xb) + al(hb);
  SlotLease lease;
  if (lease.s == nullptr || lease.s->buf.ensure(total) != cudaSuccess) {
    if (flags != nullptr)
      for (int c = 0; c < ncell; ++c) flags[c] = -111;
    return -111;
  }
  char* b = static_cast<char*>(lease.s->buf.p);
  auto carve = [&](size_t bytes) { char* r = b; b += al(bytes); return r; };
  double* dn = reinterpret_cast<double*>(carve(nb));
  double* dT = reinterpret_cast<double*>(carve(tb));
  double* dp = reinterpret_cast<double*>(carve(pb));
  int* dfl = reinterpret_cast<int*>(carve(ib));
  EqCells e;
  e.nin = reinterpret_cast<double*>(carve(nb));
  e.Tin = reinterpret_cast<double*>(carve(tb));
  e.prev = reinterpret_cast<double*>(carve(nb));
  e.Tprev = reinterpret_cast<double*>(carve(tb));
  e.t = reinterpret_cast<double*>(carve(tb));
  e.dt = reinterpret_cast<double*>(carve(tb));
  e.state = reinterpret_cast<int*>(carve(ib));
  e.out = reinterpret_cast<int*>(carve(ib));
  double* dxs = reinterpret_cast<double*>(carve(xb));
  double* dphi = reinterpret_cast<double*>(carve(hb));
  unsigned* dcur = reinterpret_cast<unsigned*>(b);
  unsigned* dact = dcur + 1;
  const EqOpts q{h->eq_t0, h->eq_tmax, h->eq_factor, h->eq_rtol, h->eq_atol,
                 h->evolve_T};
  cudaStream_t s = lease.s->stream;
  cudaError_t err = cudaMemcpyAsync(dn, n, nb, cudaMemcpyHostToDevice, s);
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(dT, Tgas, tb, cudaMemcpyHostToDevice, s);
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(dp, P, pb, cudaMemcpyHostToDevice, s);
  PhotoArgs pa;
  if (B > 0) {
    if (err == cudaSuccess)
      err = cudaMemcpyAsync(dxs, h->photo.sigma.data(), xb,
                            cudaMemcpyHostToDevice, s);
    if (err == cudaSuccess)
      err = cudaMemcpyAsync(dphi, phi, hb, cudaMemcpyHostToDevice, s);
    pa = PhotoArgs{dxs, dphi, B};
  }
  const int tpb = 128, nblk = (ncell + tpb - 1) / tpb;
  if (err == cudaSuccess) {
    kb_eq_init<<<nblk, tpb, 0, s>>>(ncell, dn, dT, e, q.t0);
    err = cudaGetLastError();
  }
  // bounded: every interval at least multiplies t by factor (or converges
  // a cell whose interval is empty); 10,000 intervals is far beyond t_max
  for (int it = 0; it < 10000 && err == cudaSuccess; ++it) {
    kb_eq_pre<<<nblk, tpb, 0, s>>>(ncell, dn, dT, e);
    err = cudaGetLastError();
    if (err == cudaSuccess)
      err = launch_any(*h, ncell, dn, dT, e.dt, dp, ps, dfl, nullptr, dcur, s,
                       pa);
    if (err == cudaSuccess) err = cudaMemsetAsync(dact, 0, sizeof(unsigned), s);
    if (err == cudaSuccess) {
      kb_eq_post<<<nblk, tpb, 0, s>>>(ncell, dn, dT, dfl, e, q, dact);
      err = cudaGetLastError();
    }
    unsigned active = 0;
    if (err == cudaSuccess)
      err = cudaMemcpyAsync(&active, dact, sizeof(unsigned),
                            cudaMemcpyDeviceToHost, s);
    if (err == cudaSuccess) err = cudaStreamSynchronize(s);
    if (err == cudaSuccess && active == 0) break;
  }
  std::vector<double> hn(nb / sizeof(double)), hT(ncell);
  std::vector<int> hfl(ncell);
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(hn.data(), dn, nb, cudaMemcpyDeviceToHost, s);
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(hT.data(), dT, tb, cudaMemcpyDeviceToHost, s);
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(hfl.data(), e.out, ib, cudaMemcpyDeviceToHost, s);
  if (err == cudaSuccess) err = cudaStreamSynchronize(s);
  if (err != cudaSuccess) {
    std::fprintf(stderr, "krome_b200: CUDA error %s\n", cudaGetErrorString(err));
    return -104;
  }
  std::memcpy(n, hn.data(), nb);
  std::memcpy(Tgas, hT.data(), tb);
  int first = 0;
  for (int c = 0; c < ncell; ++c) {
    if (flags != nullptr) flags[c] = hfl[c];
    if (first == 0 && hfl[c] != 0) first = hfl[c];
  }
  return first;
}

KB_API int krome_b200_solve_batch(int ncell, double* n, double* Tgas,
                                  const double* dt, const double* par,
                                  int par_stride, int* flags, long* stats,
                                  const krome_opts* h) {
  return solve_host(ncell, n, Tgas, dt, par, par_stride, nullptr, flags,
                    stats, h);
}

// the reference's entry point (krome.h:291-294): host arrays, in place;
// extra->Phi [ncell][nbins] the photon field with photon bins on the handle
// (Td and adust: binned dust, not built, not read)
KB_API int krome_solve_cells(int ncell, double* n, double* Tgas,
                             const double* dt, const double* par,
                             int par_stride, const krome_cells* extra,
                             int* flags, const krome_opts* h) {
  return solve_host(ncell, n, Tgas, dt, par, par_stride,
                    extra != nullptr ? extra->Phi : nullptr, flags, nullptr, h);
}

// ---- mass fractions and device-resident arrays (reference krome.h:
// 296-349) ----

// the reference's count of a device call's cells (krome.h:339-343); host
// recovery does not exist in this library, so `host` stays 0
struct krome_device_summary {
  long device;
  long host;
  long failed;
};

namespace {
// species i of cell c in the caller's layout (krome.h:311-314): species-
// major n[i * ld + c] (0) or cell-major n[c * nspec + i] (1)
__device__ __forceinline__ long at_(int layout, long ld, int c, int i) {
  return layout == 0 ? (long)i * ld + c : (long)c * kbnet::NSPEC + i;
}
// the caller's species (densities, or fractions with rho) into the
// cell-major densities the solve takes; xin the fractions' input sums
__global__ void kb_gather_in(int ncell, const double* src, int layout, long ld,
                             const double* rho, double* n, double* xin) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncell) return;
  double v[kbnet::NSPEC];
  for (int i = 0; i < kbnet::NSPEC; ++i) v[i] = src[at_(layout, ld, c, i)];
  double* nc = n + (long)c * kbnet::NSPEC;
  if (rho == nullptr) {
    for (int i = 0; i < kbnet::NSPEC; ++i) nc[i] = v[i];
    return;
  }
  xin[c] = x_sum(v);
  x_to_n(v, rho[c], nc);
}
// the solved cells back into the caller's layout (a failed cell keeps its
// input)
__global__ void kb_scatter_out(int ncell, const double* n, const int* fl,
                               int layout, long ld, const double* rho,
                               const double* xin, int renormalize,
                               double* dst) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncell || fl[c] != 0) return;
  const double* nc = n + (long)c * kbnet::NSPEC;
  double v[kbnet::NSPEC];
  if (rho == nullptr) {
    for (int i = 0; i < kbnet::NSPEC; ++i) v[i] = nc[i];
  } else {
    n_to_x_out(nc, rho[c], xin[c], renormalize, v);
  }
  for (int i = 0; i < kbnet::NSPEC; ++i) dst[at_(layout, ld, c, i)] = v[i];
}

std::mutex g_dmu;  // the device entry points' scratch
DevBuf g_dbuf;

// krome_solve_cells_device and _x_device (krome.h:308-344): arrays in
// device memory; the device fenced before and after; no host recovery
int solve_device_entry(int ncell, double* arr, const double* rho, int layout,
                       long ld, double* Tgas, const double* dt,
                       const double* par, int par_stride, const krome_cells* extra,
                       int* flags, krome_device_summary* summary,
                       const krome_opts* h) {
  if (h == nullptr || ncell < 0 || arr == nullptr || Tgas == nullptr
      || dt == nullptr)
    return -1;
  if (layout != 0 && layout != 1) return -1;
  if (layout == 0) {
    if (ld == 0) ld = ncell;
    if (ld < ncell) return -1;
  }
  if (par != nullptr && par_stride != 0 && par_stride != kbnet::NPAR) return -1;
  if (summary != nullptr) *summary = krome_device_summary{0, 0, 0};
  if (ncell == 0) return 0;
  // extra->Phi [ncell][nbins] (device): the photon field, required with
  // photon bins on the handle; Td and adust (binned dust) are not read
  const int B = h->photo.B;
  const double* phi = extra != nullptr ? extra->Phi : nullptr;
  if (cudaDeviceSynchronize() != cudaSuccess) return -104;
  // the required-parameter rule on the caller's rows (a host copy)
  const int ps = par != nullptr ? par_stride : 0;
  std::vector<double> P(ps ? (size_t)ncell * ps : kbnet::NPAR);
  if (par != nullptr) {
    if (cudaMemcpy(P.data(), par, sizeof(double) * P.size(),
                   cudaMemcpyDeviceToHost) != cudaSuccess)
      return -1;
  } else {
    krome_params_default(P.data());
  }
  std::vector<int> hfl(ncell, 0);
  int ret = check_params(ncell, P.data(), ps, hfl.data());
  if (ret == 0) ret = unsupported(*h);
  if (ret == 0 && B > 0 && phi == nullptr) ret = -103;
  if (ret != 0 && ret != -105)
    for (int c = 0; c < ncell; ++c) hfl[c] = ret;
  const size_t fb = sizeof(int) * (size_t)ncell;
  if (ret != 0) {
    if (flags != nullptr
        && cudaMemcpy(flags, hfl.data(), fb, cudaMemcpyHostToDevice) != cudaSuccess)
      return -104;
    if (summary != nullptr)
      for (int c = 0; c < ncell; ++c) summary->failed += hfl[c] != 0;
    return ret;
  }
  // the lane kernel reads and writes the caller's layout (and converts
  // mass fractions) itself; the other kernels take staged cell-major
  // densities
  const bool fused = fuses_io(*h);
  const bool staged = !fused && (layout == 0 || rho != nullptr);
  const size_t nb = staged ? sizeof(double) * (size_t)ncell * kbnet::NSPEC : 0;
  const size_t xb = rho != nullptr ? sizeof(double) * (size_t)ncell : 0;
  const size_t pb = par == nullptr ? sizeof(double) * kbnet::NPAR : 0;
  const size_t sgb = B > 0 ? sizeof(double) * (size_t)kbnet::NPHOTO * B : 0;
  auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
  std::lock_guard<std::mutex> lock(g_dmu);
  if (g_dbuf.ensure(al(nb) + al(xb) + al(pb) + al(fb) + al(sgb) + 256)
      != cudaSuccess)
    return -111;
  char* b = static_cast<char*>(g_dbuf.p);
  double* dn = staged ? reinterpret_cast<double*>(b) : arr; b += al(nb);
  double* dx = reinterpret_cast<double*>(b); b += al(xb);
  double* dp = reinterpret_cast<double*>(b); b += al(pb);
  int* dfl = reinterpret_cast<int*>(b); b += al(fb);
  double* dsg = reinterpret_cast<double*>(b); b += al(sgb);
  unsigned* dcur = reinterpret_cast<unsigned*>(b);
  const double* Pd = par;
  cudaError_t e = cudaSuccess;
  if (par == nullptr) {
    e = cudaMemcpy(dp, P.data(), pb, cudaMemcpyHostToDevice);
    Pd = dp;
  }
  PhotoArgs pa;
  if (B > 0 && e == cudaSuccess) {
    e = cudaMemcpy(dsg, h->photo.sigma.data(), sgb, cudaMemcpyHostToDevice);
    pa = PhotoArgs{dsg, phi, B};
  }
  const int tpb = 128, nblk = (ncell + tpb - 1) / tpb;
  if (e == cudaSuccess && staged) {
    kb_gather_in<<<nblk, tpb>>>(ncell, arr, layout, ld, rho, dn, dx);
    e = cudaGetLastError();
  }
  CellIO io;
  if (fused) {
    io.layout = layout;
    io.ld = ld;
    io.rho = rho;
    io.renormalize = h->renormalize_x;
  }
  if (e == cudaSuccess)
    e = launch_any(*h, ncell, dn, Tgas, dt, Pd, ps, dfl, nullptr, dcur, 0, pa,
                   io);
  if (e == cudaSuccess && staged) {
    kb_scatter_out<<<nblk, tpb>>>(ncell, dn, dfl, layout, ld, rho, dx,
                                  h->renormalize_x, arr);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess && flags != nullptr)
    e = cudaMemcpyAsync(flags, dfl, fb, cudaMemcpyDeviceToDevice, 0);
  if (e == cudaSuccess)
    e = cudaMemcpy(hfl.data(), dfl, fb, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    std::fprintf(stderr, "krome_b200: CUDA error %s\n", cudaGetErrorString(e));
    return -104;
  }
  for (int c = 0; c < ncell; ++c) {
    if (summary != nullptr) {
      if (hfl[c] == 0) ++summary->device;
      else ++summary->failed;
    }
    if (ret == 0 && hfl[c] != 0) ret = hfl[c];
  }
  return ret;
}
}  // namespace

// krome_solve_cells with mass fractions x[ncell][nspec] and the gas density
// rho[ncell] [g cm^-3] (reference krome.h:302-306, krome.cpp:438-470): n =
// rho x / m on the way in, x = m n / rho on the way out (rescaled to the
// input sum with renormalize_x) for the cells that succeed; a failed cell
// keeps its input x
KB_API int krome_solve_cells_x(int ncell, double* x, const double* rho,
                               double* Tgas, const double* dt,
                               const double* par, int par_stride,
                               const krome_cells* extra, int* flags,
                               const krome_opts* h) {
  if (h == nullptr || ncell < 0 || x == nullptr || rho == nullptr
      || Tgas == nullptr || dt == nullptr)
    return -1;
  if (par != nullptr && par_stride != 0 && par_stride != kbnet::NPAR) return -1;
  if (ncell == 0) return 0;
  std::vector<double> n((size_t)ncell * kbnet::NSPEC), xin(ncell);
  for (int c = 0; c < ncell; ++c) {
    const double* xc = x + (size_t)c * kbnet::NSPEC;
    xin[c] = x_sum(xc);
    x_to_n(xc, rho[c], n.data() + (size_t)c * kbnet::NSPEC);
  }
  std::vector<int> fl(ncell, 0);
  int* f = flags != nullptr ? flags : fl.data();
  const int r = krome_solve_cells(ncell, n.data(), Tgas, dt, par, par_stride,
                                  extra, f, h);
  for (int c = 0; c < ncell; ++c)
    if (f[c] == 0)
      n_to_x_out(n.data() + (size_t)c * kbnet::NSPEC, rho[c], xin[c],
                 h->renormalize_x, x + (size_t)c * kbnet::NSPEC);
  return r;
}

// krome_solve_cells on device arrays (reference krome.h:308-349): n in the
// species-major (0, leading dimension ld >= ncell, 0 for ncell) or cell-
// major (1) layout, Tgas, dt [ncell], par rows or NULL (the defaults),
// flags (device, may be NULL), summary (host, may be NULL)
KB_API int krome_solve_cells_device(int ncell, double* n, int layout, long ld,
                                    double* Tgas, const double* dt,
                                    const double* par, int par_stride,
                                    const krome_cells* extra, int* flags,
                                    krome_device_summary* summary,
                                    const krome_opts* h) {
  return solve_device_entry(ncell, n, nullptr, layout, ld, Tgas, dt, par,
                            par_stride, extra, flags, summary, h);
}
// the same with mass fractions and rho [ncell] on the device
KB_API int krome_solve_cells_x_device(int ncell, double* x, const double* rho,
                                      int layout, long ld, double* Tgas,
                                      const double* dt, const double* par,
                                      int par_stride, const krome_cells* extra,
                                      int* flags,
                                      krome_device_summary* summary,
                                      const krome_opts* h) {
  if (rho == nullptr) return -1;
  return solve_device_entry(ncell, x, rho, layout, ld, Tgas, dt, par,
                            par_stride, extra, flags, summary, h);
}

// ---- host utilities of the reference's interface (krome.h:473-501, 539,
// 645-652): element totals, consistent advection, n <-> x, metadata ----

// tot[ncell][nelem] = sum_i (atoms of element e in species i) n_i
// (query.hpp:153-158), or per gram from mass fractions (162-170)
KB_API int krome_get_element_totals(int ncell, const double* n, double* tot) {
  if (ncell < 0 || n == nullptr || tot == nullptr) return -1;
  using namespace kbnet;
  for (int c = 0; c < ncell; ++c) {
    double* t = tot + (size_t)c * NELEM;
    for (int e = 0; e < NELEM; ++e) t[e] = 0.0;
    for (int i = 0; i < NSPEC; ++i)
      for (int e = 0; e < NELEM; ++e)
        t[e] += species_element(i, e) * n[(size_t)c * NSPEC + i];
  }
  return 0;
}
KB_API int krome_get_element_totals_x(int ncell, const double* x, double* tot) {
  if (ncell < 0 || x == nullptr || tot == nullptr) return -1;
  using namespace kbnet;
  for (int c = 0; c < ncell; ++c) {
    double* t = tot + (size_t)c * NELEM;
    for (int e = 0; e < NELEM; ++e) t[e] = 0.0;
    for (int i = 0; i < NSPEC; ++i) {
      if (!(species_mass_g(i) > 0.0)) continue;
      const double ni = x[(size_t)c * NSPEC + i] / species_mass_g(i);
      for (int e = 0; e < NELEM; ++e) t[e] += species_element(i, e) * ni;
    }
  }
  return 0;
}

// consistent advection (krome.h:478-497, solve_cells.hpp:215-243): each cell
// moved to its reference element totals ref (ref_stride 0: one row for all,
// nelem: a row per cell) and to zero charge; par (the freeze directives'
// rows: none in these networks) may be NULL; flags[ncell] (may be NULL) 0,
// -112 (unreachable) or the warning 2. Returns the lowest failing cell's
// flag (negative), else 0.
namespace {
int conserve_cells_host(int ncell, double* v, const double* ref,
                        int ref_stride, const double* par, int par_stride,
                        int* flags, bool x) {
  using namespace kbnet;
  if (ncell < 0 || v == nullptr || ref == nullptr || ref_stride < 0
      || par_stride < 0)
    return -1;
  if (ref_stride != 0 && ref_stride != NELEM) return -1;
  if (par != nullptr && par_stride != 0 && par_stride != NPAR) return -1;
  std::vector<double> dflt(NPAR);
  krome_params_default(dflt.data());
  int ret = 0;
  for (int c = 0; c < ncell; ++c) {
    double* vc = v + (size_t)c * NSPEC;
    const double* rc = ref + (size_t)c * ref_stride;
    Params p;  // the freeze directives' parameters (NULL: the defaults)
    params_from_row(par != nullptr ? par + (size_t)c * par_stride
                                   : dflt.data(), p);
    const int f = x ? conserve_to_x(vc, rc, p) : conserve_to(vc, rc, p);
    if (flags != nullptr) flags[c] = f;
    if (ret == 0 && f < 0) ret = f;
  }
  return ret;
}
}  // namespace
KB_API int krome_conserve_cells(int ncell, double* n, const double* ref,
                                int ref_stride, const double* par,
                                int par_stride, int* flags) {
  return conserve_cells_host(ncell, n, ref, ref_stride, par, par_stride,
                             flags, false);
}
KB_API int krome_conserve_cells_x(int ncell, double* x, const double* ref,
                                  int ref_stride, const double* par,
                                  int par_stride, int* flags) {
  return conserve_cells_host(ncell, x, ref, ref_stride, par, par_stride,
                             flags, true);
}

// consistent advection on device arrays (reference krome.h:351-360,
// runtime/core/solve_kokkos.hpp:1787-1823): one thread per cell reads the
// cell from the caller's layout, moves it to its reference totals with the
// host path's projection (kb_conserve.h) and writes it back; the lowest
// failing cell's flag comes back through one 64-bit atomic minimum of
// (cell << 32 | flag bits), so no second pass is needed
namespace {
__global__ void kb_conserve_cells(int ncell, double* v, int mass, int layout,
                                  long ld, const double* ref, int ref_stride,
                                  const double* par, int par_stride,
                                  int* flags, unsigned long long* lowest) {
  using namespace kbnet;
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncell) return;
  double x[NSPEC];
  for (int i = 0; i < NSPEC; ++i) x[i] = v[at_(layout, ld, c, i)];
  const double* r = ref + (long)c * ref_stride;
  Params p;  // the freeze directives' parameters
  params_from_row(par + (long)c * par_stride, p);
  const int f = mass ? conserve_to_x(x, r, p) : conserve_to(x, r, p);
  for (int i = 0; i < NSPEC; ++i) v[at_(layout, ld, c, i)] = x[i];
  if (flags != nullptr) flags[c] = f;
  if (f < 0)
    atomicMin(lowest, ((unsigned long long)c << 32) | (unsigned)f);
}

int conserve_cells_device(int ncell, double* v, bool mass, int layout,
                          long ld, const double* ref, int ref_stride,
                          const double* par, int par_stride, int* flags) {
  using namespace kbnet;
  if (ncell < 0 || v == nullptr || ref == nullptr || par_stride < 0)
    return -1;
  if (ref_stride != 0 && ref_stride != NELEM) return -1;
  if (par != nullptr && par_stride != 0 && par_stride != NPAR) return -1;
  if (layout != 0 && layout != 1) return -1;
  if (layout == 0) {
    if (ld == 0) ld = ncell;
    if (ld < ncell) return -1;
  }
  if (ncell == 0) return 0;
  if (cudaDeviceSynchronize() != cudaSuccess) return -104;
  std::lock_guard<std::mutex> lock(g_dmu);
  if (g_dbuf.ensure(256 + sizeof(double) * NPAR) != cudaSuccess) return -111;
  auto* lowest = static_cast<unsigned long long*>(g_dbuf.p);
  double* dflt = reinterpret_cast<double*>(static_cast<char*>(g_dbuf.p) + 256);
  cudaError_t e = cudaMemset(lowest, 0xff, sizeof(unsigned long long));
  if (e == cudaSuccess && par == nullptr) {  // the default parameter row
    std::vector<double> row(NPAR);
    krome_params_default(row.data());
    e = cudaMemcpy(dflt, row.data(), sizeof(double) * NPAR,
                   cudaMemcpyHostToDevice);
  }
  const int tpb = 128;
  if (e == cudaSuccess) {
    kb_conserve_cells<<<(ncell + tpb - 1) / tpb, tpb>>>(
        ncell, v, mass ? 1 : 0, layout, ld, ref, ref_stride,
        par != nullptr ? par : dflt, par != nullptr ? par_stride : 0, flags,
        lowest);
    e = cudaGetLastError();
  }
  unsigned long long key = ~0ull;
  if (e == cudaSuccess)
    e = cudaMemcpy(&key, lowest, sizeof(key), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) {
    std::fprintf(stderr, "krome_b200: CUDA error %s\n", cudaGetErrorString(e));
    return -104;
  }
  return key == ~0ull ? 0 : (int)(unsigned)(key & 0xffffffffull);
}
}  // namespace

// krome_conserve_cells and _x on device arrays (krome.h:351-360): v in the
// species-major (layout 0, leading dimension ld >= ncell, 0 for ncell) or
// cell-major (1) layout; ref, par and flags on the device too
KB_API int krome_conserve_cells_device(int ncell, double* n, int layout,
                                       long ld, const double* ref,
                                       int ref_stride, const double* par,
                                       int par_stride, int* flags) {
  return conserve_cells_device(ncell, n, false, layout, ld, ref, ref_stride,
                               par, par_stride, flags);
}
KB_API int krome_conserve_cells_x_device(int ncell, double* x, int layout,
                                         long ld, const double* ref,
                                         int ref_stride, const double* par,
                                         int par_stride, int* flags) {
  return conserve_cells_device(ncell, x, true, layout, ld, ref, ref_stride,
                               par, par_stride, flags);
}

// x = m n / rho and n = rho x / m (query.hpp:443-449)
KB_API int krome_n2x(int ncell, const double* n, const double* rho, double* x) {
  if (ncell < 0 || n == nullptr || rho == nullptr || x == nullptr) return -1;
  for (int c = 0; c < ncell; ++c)
    for (int i = 0; i < kbnet::NSPEC; ++i)
      x[(size_t)c * kbnet::NSPEC + i] =
          kbnet::species_mass_g(i) * n[(size_t)c * kbnet::NSPEC + i] / rho[c];
  return 0;
}
KB_API int krome_x2n(int ncell, const double* x, const double* rho, double* n) {
  if (ncell < 0 || x == nullptr || rho == nullptr || n == nullptr) return -1;
  for (int c = 0; c < ncell; ++c)
    x_to_n(x + (size_t)c * kbnet::NSPEC, rho[c], n + (size_t)c * kbnet::NSPEC);
  return 0;
}

KB_API double krome_species_mass(int i) {
  return (i >= 0 && i < kbnet::NSPEC) ? kbnet::species_mass_g(i) : std::nan("");
}
KB_API int krome_species_charge(int i) {
  return (i >= 0 && i < kbnet::NSPEC) ? kbnet::species_charge(i) : 0;
}
KB_API int krome_nelem(void) { return kbnet::NELEM; }
KB_API const char* krome_element_name(int e) {
  return (e >= 0 && e < kbnet::NELEM) ? kbnet::element_names[e] : nullptr;
}
KB_API int krome_species_natoms(int i, int e) {
  if (i < 0 || i >= kbnet::NSPEC || e < 0 || e >= kbnet::NELEM) return -1;
  return kbnet::species_element(i, e);
}

// the device backend's set-up calls (krome.h:187-201): this library needs
// none (the CUDA runtime initializes itself); 0 with a usable device, -104
// without one; _id makes device_id current for the calling thread
KB_API int krome_device_initialize(void) {
  int nd = 0;
  return cudaGetDeviceCount(&nd) == cudaSuccess && nd > 0 ? 0 : -104;
}
KB_API int krome_device_initialize_id(int device_id) {
  int nd = 0;
  if (cudaGetDeviceCount(&nd) != cudaSuccess || nd <= 0) return -104;
  if (device_id < 0) return 0;
  return cudaSetDevice(device_id) == cudaSuccess ? 0 : -1;
}
KB_API int krome_device_finalize(void) { return krome_device_initialize(); }

namespace {
// the rate coefficients of each cell at its rate temperature clamp(Tgas,
// Tcmb, 1e9) (the reference's krome_get_rates query, krome.h:387-389)
__global__ void kb_rates(int ncell, const double* n, const double* T,
                         const double* par, int pstride, double* k,
                         const double* sigma, const double* phi, int B) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncell) return;
  using namespace kbnet;
  double nv[NSPEC], kk[NREA + 1];
  KB_UNROLL for (int i = 0; i < NSPEC; ++i) nv[i] = n[(long)c * NSPEC + i];
  Params p;
  params_from_row(par + (long)c * pstride, p);
  if (B > 0) kbw::photo_rates_of_row(p, sigma, phi + (long)c * B, B);
  const double Tr = fmin(fmax(T[c], p.Tcmb), 1e9);
  KB_UNROLL for (int i = 0; i <= NREA; ++i) kk[i] = 0.0;
  rates_fixed(Tr, nv, p, kk);
  rates_var(Tr, nv, p, kk);
  KB_UNROLL for (int i = 0; i < NREA; ++i) k[(long)c * NREA + i] = kk[i];
}
}  // namespace

// krome_get_rates (reference krome.h:387-389): k[ncell][nrea], host arrays;
// the photo rates (no photon bins here) are 0. Phi and h are unused.
KB_API int krome_get_rates(int ncell, const double* n, const double* Tgas,
                           const double* par, int par_stride,
                           const double* Phi, const krome_opts* h, double* k) {
  if (ncell < 0 || n == nullptr || Tgas == nullptr || k == nullptr) return -1;
  const int B = h != nullptr ? h->photo.B : 0;
  if (B > 0 && Phi == nullptr) return -103;  // photon bins without a field
  if (par != nullptr && par_stride != 0 && par_stride != kbnet::NPAR) return -1;
  if (ncell == 0) return 0;
  std::vector<double> dflt(kbnet::NPAR);
  krome_params_default(dflt.data());
  const double* P = par != nullptr ? par : dflt.data();
  const int ps = par != nullptr ? par_stride : 0;
  for (int c = 0; c < ncell; ++c)
    if (row_missing(P + (long)c * ps)) return -105;
  const size_t nb = sizeof(double) * (size_t)ncell * kbnet::NSPEC;
  const size_t tb = sizeof(double) * (size_t)ncell;
  const size_t pb = sizeof(double) * (ps ? (size_t)ncell * ps : (size_t)kbnet::NPAR);
  const size_t kb = sizeof(double) * (size_t)ncell * kbnet::NREA;
  const size_t sgb = B > 0 ? sizeof(double) * (size_t)kbnet::NPHOTO * B : 0;
  const size_t phb = B > 0 ? sizeof(double) * (size_t)ncell * B : 0;
  auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
  std::lock_guard<std::mutex> lock(g_mu);
  if (g_buf.ensure(al(nb) + al(tb) + al(pb) + al(kb) + al(sgb) + al(phb))
      != cudaSuccess)
    return -111;
  char* b = static_cast<char*>(g_buf.p);
  double* dn = reinterpret_cast<double*>(b); b += al(nb);
  double* dT = reinterpret_cast<double*>(b); b += al(tb);
  double* dp = reinterpret_cast<double*>(b); b += al(pb);
  double* dk = reinterpret_cast<double*>(b); b += al(kb);
  double* dsg = reinterpret_cast<double*>(b); b += al(sgb);
  double* dph = reinterpret_cast<double*>(b);
  cudaError_t e = cudaMemcpy(dn, n, nb, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dT, Tgas, tb, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dp, P, pb, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && B > 0)
    e = cudaMemcpy(dsg, h->photo.sigma.data(), sgb, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && B > 0) e = cudaMemcpy(dph, Phi, phb, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    kb_rates<<<(ncell + 127) / 128, 128>>>(ncell, dn, dT, dp, ps, dk, dsg, dph, B);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(k, dk, kb, cudaMemcpyDeviceToHost);
  return e == cudaSuccess ? 0 : -104;
}

// ---------------------------------------------------------------------------
// the hydro loop of the collapse driver, on the device

namespace {
// one compression step of the reference's collapse driver
// (examples/tests/collapse/test.cpp:47-63): tff = sqrt(3 pi / (32 G rho))
// of the current state (rho = sum n_i m_i in species order, the reference's
// rho_), the parameter tff of the cell set to it, every density x factor,
// dt = dtfrac tff
__global__ void kb_compress(int ncell, double* n, double* par, int pstride,
                            int tff_index, double* dt, double factor,
                            double dtfrac) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncell) return;
  using namespace kbnet;
  double* nc = n + (long)c * NSPEC;
  double v[NSPEC];
  KB_UNROLL for (int i = 0; i < NSPEC; ++i) v[i] = nc[i];
  const double rho = rho_(v);
  const double tff = sqrt(3.0 * kbc::pi / (32.0 * kbc::gravity * fmax(rho, 1e-40)));
  if (pstride > 0) par[(long)c * pstride + tff_index] = tff;
  KB_UNROLL for (int i = 0; i < NSPEC; ++i) nc[i] = v[i] * factor;
  dt[c] = dtfrac * tff;
}

struct HydroGraph {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};
}  // namespace

// one device-resident hydro step: compression (kb_compress) then the solve,
// on `stream`, asynchronously (nothing allocated, no host synchronization)
KB_API int krome_b200_hydro_step(int ncell, double* n, double* Tgas,
                                 double* dt, double* par, int par_stride,
                                 int tff_index, double factor, double dtfrac,
                                 int* flags, long* stats, unsigned* cursor,
                                 const krome_opts* h, void* stream) {
  if (h == nullptr || ncell < 0 || par_stride != kbnet::NPAR
      || tff_index < 0 || tff_index >= kbnet::NPAR)
    return -1;
  if (ncell == 0) return 0;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  kb_compress<<<(ncell + 127) / 128, 128, 0, s>>>(
      ncell, n, par, par_stride, tff_index, dt, factor, dtfrac);
  if (cudaGetLastError() != cudaSuccess) return -104;
  return krome_b200_solve_device(ncell, n, Tgas, dt, par, par_stride, flags,
                                 stats, cursor, h, stream);
}

// the hydro step captured once as a CUDA graph (compression, work-queue
// reset, solve) and replayed by krome_b200_graph_launch; the arrays stay
// bound to the graph. Returns a handle or NULL.
KB_API void* krome_b200_graph_new(int ncell, double* n, double* Tgas,
                                  double* dt, double* par, int par_stride,
                                  int tff_index, double factor, double dtfrac,
                                  int* flags, long* stats, unsigned* cursor,
                                  const krome_opts* h, void* stream) {
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  auto* g = new HydroGraph();
  // occupancy queries are made before the capture
  (void)num_sms();
  if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    delete g;
    return nullptr;
  }
  const int r = krome_b200_hydro_step(ncell, n, Tgas, dt, par, par_stride,
                                      tff_index, factor, dtfrac, flags, stats,
                                      cursor, h, stream);
  const cudaError_t e = cudaStreamEndCapture(s, &g->graph);
  if (r != 0 || e != cudaSuccess
      || cudaGraphInstantiate(&g->exec, g->graph, 0) != cudaSuccess) {
    if (g->graph) cudaGraphDestroy(g->graph);
    delete g;
    return nullptr;
  }
  return g;
}

KB_API int krome_b200_graph_launch(void* handle, void* stream) {
  auto* g = static_cast<HydroGraph*>(handle);
  if (g == nullptr) return -1;
  return cudaGraphLaunch(g->exec, static_cast<cudaStream_t>(stream))
             == cudaSuccess ? 0 : -104;
}

KB_API void krome_b200_graph_free(void* handle) {
  auto* g = static_cast<HydroGraph*>(handle);
  if (g == nullptr) return;
  cudaGraphExecDestroy(g->exec);
  cudaGraphDestroy(g->graph);
  delete g;
}

// the network rhs alone at full SIMT width: every thread evaluates the rhs
// of its cell `reps` times (each evaluation feeds a negligible increment
// back into the state, so none can be hoisted); the rhs-throughput bound of
// the solve kernels
#ifndef KB_LARGE_NETWORK
namespace {
__global__ void kb_rhs_loop(int ncell, const double* n, const double* T,
                            const double* par, int pstride, int reps,
                            double* sink) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncell) return;
  using namespace kbnet;
  constexpr int N = NSPEC + 1;
  double yf[N], f[N], k[NREA + 1];
  KB_UNROLL for (int i = 0; i < NSPEC; ++i) yf[i] = n[(long)c * NSPEC + i];
  yf[N - 1] = T[c];
  Params p;
  params_from_row(par + (long)c * pstride, p);
  double acc = 0.0;
  for (int r = 0; r < reps; ++r) {
    kbw::full_rhs<N, true>(yf, f, p, 0.0, k);
    yf[0] += 1e-300 * f[0];
    acc += f[N - 1];
  }
  if (acc == 1.2345e-300) sink[c] = acc;
}
}  // namespace
#endif

KB_API int krome_b200_rhs_throughput(int ncell, const double* n,
                                     const double* Tgas, const double* par,
                                     int par_stride, int reps,
                                     double* rhs_per_s) {
  if (ncell <= 0 || reps <= 0 || rhs_per_s == nullptr) return -1;
#ifdef KB_LARGE_NETWORK
  (void)n; (void)Tgas; (void)par; (void)par_stride;
  return -104;  // the per-thread rhs of a large network is not a kernel here
#else
  const size_t nb = sizeof(double) * (size_t)ncell * kbnet::NSPEC;
  const size_t tb = sizeof(double) * (size_t)ncell;
  const size_t pb = sizeof(double) * (size_t)ncell * kbnet::NPAR;
  auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
  std::lock_guard<std::mutex> lock(g_mu);
  if (g_buf.ensure(al(nb) + 2 * al(tb) + al(pb)) != cudaSuccess) return -111;
  char* b = static_cast<char*>(g_buf.p);
  double* dn = reinterpret_cast<double*>(b); b += al(nb);
  double* dT = reinterpret_cast<double*>(b); b += al(tb);
  double* ds = reinterpret_cast<double*>(b); b += al(tb);
  double* dp = reinterpret_cast<double*>(b);
  cudaMemcpy(dn, n, nb, cudaMemcpyHostToDevice);
  cudaMemcpy(dT, Tgas, tb, cudaMemcpyHostToDevice);
  cudaMemcpy(dp, par, par_stride ? pb : sizeof(double) * kbnet::NPAR,
             cudaMemcpyHostToDevice);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  kb_rhs_loop<<<(ncell + 127) / 128, 128>>>(ncell, dn, dT, dp, par_stride, 1, ds);
  cudaEventRecord(e0);
  kb_rhs_loop<<<(ncell + 127) / 128, 128>>>(ncell, dn, dT, dp, par_stride, reps, ds);
  cudaEventRecord(e1);
  const cudaError_t e = cudaEventSynchronize(e1);
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (e != cudaSuccess || ms <= 0.0f) return -104;
  *rhs_per_s = (double)ncell * reps / (ms * 1e-3);
  return 0;
#endif
}

// the FP64 pipe's peak, measured: independent DFMA chains in registers,
// the whole GPU, timed with events. Writes TFLOP/s (2 flops per DFMA).
namespace {
__global__ void kb_dfma_chains(double* out, int iters, double a, double b) {
  double x0 = threadIdx.x, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3;
  double x4 = x0 + 4, x5 = x0 + 5, x6 = x0 + 6, x7 = x0 + 7;
  for (int i = 0; i < iters; ++i) {
    x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b);
    x3 = fma(x3, a, b); x4 = fma(x4, a, b); x5 = fma(x5, a, b);
    x6 = fma(x6, a, b); x7 = fma(x7, a, b);
  }
  const double s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
  if (s == 12345.678) out[0] = s;  // keeps the chains alive
}
}  // namespace

KB_API int krome_b200_fp64_peak(double* tflops) {
  if (tflops == nullptr) return -1;
  double* out = nullptr;
  if (cudaMalloc(&out, sizeof(double)) != cudaSuccess) return -104;
  const int blocks = num_sms() * 8, threads = 256, iters = 1 << 14;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  kb_dfma_chains<<<blocks, threads>>>(out, 256, 0.999999, 1e-7);
  cudaEventRecord(e0);
  kb_dfma_chains<<<blocks, threads>>>(out, iters, 0.999999, 1e-7);
  cudaEventRecord(e1);
  const cudaError_t e = cudaEventSynchronize(e1);
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  if (e != cudaSuccess || ms <= 0.0f) return -104;
  *tflops = 2.0 * 8.0 * (double)iters * blocks * threads / (ms * 1e-3) / 1e12;
  return 0;
}

// ---------------------------------------------------------------------------
// krome_solve_cells without device allocation
//
// Some callers cannot let a library call cudaMalloc: a hydro code that hands
// the whole GPU to its own memory pool at start-up (so a foreign allocation
// fails or fragments its pool), or a time step that must not pay
// cudaMalloc's implicit device-wide synchronization. For them this entry
// point stages the call's device copies in one fixed array compiled into
// the library instead of allocating: KB_NOALLOC_BYTES (16 MiB) of device
// memory that every GPU loading the library holds until the process exits.
// It holds, 256-byte aligned, the persistent kernel's work-queue cursor and
// the cells' n, Tgas, dt, parameter rows and flags; a call whose cells do not
// fit returns FLAG_DEVICE_MEMORY (-111) before touching anything.
//
// Host code never uses the array's name as an address (on the host it names
// a stand-in, not device memory): the first call on each device, with that
// device current, asks cudaGetSymbolAddress for the device address and
// keeps it. That lookup loads the library's device code (CUDA loads modules
// lazily), and the first launch of a kernel makes the driver reserve the
// kernel's per-thread local memory; both are device memory the driver takes
// itself. A call with ncell == 0 does both (the address lookup and one empty
// launch of the kernel the options select) and solves nothing: make it once
// per device before the caller's pool takes the GPU and before any stream
// capture. All calls share the one array and it keeps the previous call's
// contents; the cursor is zeroed by every launch and every cell's flag is
// written by the kernel. Calls that overlapped on the GPU would race on the
// array: the entry point serialises its own calls (a mutex held until the
// results are back on the host). Results come back through host staging, so
// a copy that fails part-way leaves the caller's arrays untouched.
// The large networks' sparse path needs its per-block workspace, which this
// entry point cannot provide: their builds return -104 and hold no array.

#ifndef KB_LARGE_NETWORK
#define KB_NOALLOC_BYTES (16u << 20)
static __device__ __align__(256) unsigned char kb_noalloc_scratch[KB_NOALLOC_BYTES];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
void* g_noalloc_ptr[kMaxDevices] = {};

// the device address of the scratch array on the current device
// (once per device), or nullptr
void* noalloc_scratch() {
  int d = 0;
  if (cudaGetDevice(&d) != cudaSuccess || d < 0 || d >= kMaxDevices)
    return nullptr;
  if (g_noalloc_ptr[d] == nullptr) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, kb_noalloc_scratch) != cudaSuccess)
      return nullptr;
    g_noalloc_ptr[d] = p;
  }
  return g_noalloc_ptr[d];
}
}  // namespace
#endif

KB_API int krome_b200_solve_cells_noalloc(int ncell, double* n, double* Tgas,
                                          const double* dt, const double* par,
                                          int par_stride, int* flags,
                                          const krome_opts* h) {
  if (h == nullptr || ncell < 0) return -1;
  if (ncell > 0 && (n == nullptr || Tgas == nullptr || dt == nullptr))
    return -1;
  if (par != nullptr && par_stride != 0 && par_stride != kbnet::NPAR)
    return -1;
#ifdef KB_LARGE_NETWORK
  (void)par;
  if (flags != nullptr)
    for (int c = 0; c < ncell; ++c) flags[c] = -104;
  return -104;  // a large network's solve needs its allocated workspace
#else
  if (ncell == 0) {
    // the warm-up: resolve the array, load the module, and launch the
    // selected kernel once with no cells (its local memory reserved now)
    if (const int u = unsupported(*h)) return u;  // it launches nothing
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    char* b = static_cast<char*>(noalloc_scratch());
    if (b == nullptr) return -104;
    unsigned* dcur = reinterpret_cast<unsigned*>(b);
    double* dd = reinterpret_cast<double*>(b + 256);
    cudaError_t e = launch_any(*h, 0, dd, dd, dd, dd, 0,
                               reinterpret_cast<int*>(b + 256), nullptr, dcur,
                               0);
    if (e == cudaSuccess) e = cudaStreamSynchronize(0);
    return e == cudaSuccess ? 0 : -104;
  }
  double dflt[kbnet::NPAR];
  for (int i = 0; i < kbnet::NPAR; ++i) dflt[i] = kbnet::param_default(i);
  const double* P = par != nullptr ? par : dflt;
  const int ps = par != nullptr ? par_stride : 0;
  bool missing = false;
  for (int c = 0; c < ncell; ++c) {
    const bool m = row_missing(P + (long)c * ps);
    if (flags != nullptr) flags[c] = m ? -105 : 0;
    missing |= m;
  }
  if (missing) return -105;
  int u = unsupported(*h);
  if (u == 0 && h->photo.B > 0) u = -103;  // no field argument here
  if (u != 0) {
    if (flags != nullptr)
      for (int c = 0; c < ncell; ++c) flags[c] = u;
    return u;
  }
  auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
  const size_t nb = sizeof(double) * (size_t)ncell * kbnet::NSPEC;
  const size_t tb = sizeof(double) * (size_t)ncell;
  const size_t pb = sizeof(double) * (ps ? (size_t)ncell * ps : (size_t)kbnet::NPAR);
  const size_t fb = sizeof(int) * (size_t)ncell;
  const size_t need = 256 + al(nb) + 2 * al(tb) + al(pb) + al(fb);
  if (need > KB_NOALLOC_BYTES) {
    if (flags != nullptr)
      for (int c = 0; c < ncell; ++c) flags[c] = -111;
    return -111;
  }
  // host staging of the results: committed to the caller's arrays only
  // once every copy has succeeded
  std::vector<double> hn((size_t)ncell * kbnet::NSPEC), hT(ncell);
  std::vector<int> hfl(ncell);
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  char* b = static_cast<char*>(noalloc_scratch());
  if (b == nullptr) {
    if (flags != nullptr)
      for (int c = 0; c < ncell; ++c) flags[c] = -104;
    return -104;
  }
  unsigned* dcur = reinterpret_cast<unsigned*>(b); b += 256;
  double* dn = reinterpret_cast<double*>(b); b += al(nb);
  double* dT = reinterpret_cast<double*>(b); b += al(tb);
  double* ddt = reinterpret_cast<double*>(b); b += al(tb);
  double* dp = reinterpret_cast<double*>(b); b += al(pb);
  int* dfl = reinterpret_cast<int*>(b);
  cudaStream_t s = 0;
  cudaError_t e = cudaMemcpyAsync(dn, n, nb, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dT, Tgas, tb, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(ddt, dt, tb, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dp, P, pb, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = launch_any(*h, ncell, dn, dT, ddt, dp, ps, dfl, nullptr, dcur, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(hn.data(), dn, nb, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(hT.data(), dT, tb, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(hfl.data(), dfl, fb, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    std::fprintf(stderr, "krome_b200: CUDA error %s\n", cudaGetErrorString(e));
    if (flags != nullptr)
      for (int c = 0; c < ncell; ++c) flags[c] = -104;
    return -104;
  }
  // a failed cell's device row still holds its input: copy every row
  std::memcpy(n, hn.data(), nb);
  std::memcpy(Tgas, hT.data(), tb);
  if (flags != nullptr) std::memcpy(flags, hfl.data(), fb);
  for (int c = 0; c < ncell; ++c)
    if (hfl[c] != 0) return hfl[c];
  return 0;
#endif
}

KB_API int krome_has_device(void) {
  int count = 0;
  return cudaGetDeviceCount(&count) == cudaSuccess && count > 0 ? 1 : 0;
}

KB_API int krome_b200_nstat(void) { return NSTAT; }
KB_API int krome_b200_neq(int evolve_T) {
  return kbnet::NSPEC + (evolve_T ? 1 : 0);
}
