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
#include <vector>

#include KB_NET_HEADER
#include "bdf_warp.cuh"
#include "bdf_lane.cuh"

#define KB_API extern "C" __attribute__((visibility("default")))

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
static_assert(kbnet::NSPEC + 3 <= 32,
              "warp-per-cell kernels need NEQ + 2 <= 32 lanes");

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
                                   par + (long)c * pstride, dtc, so, ws, sc);
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
  // per-warp shared memory: the Jacobian being assembled (column-major)
  // and two rhs vectors (the hybrid Jacobian's Tgas column)
  static constexpr int SMEM_DOUBLES = N * N + 2 * N;
};

// the warp serves lane `src`'s Jacobian request: lane j < N evaluates the
// rhs perturbed in component j (the difference-quotient column j,
// bdf_cell.hpp:1290-1311), or the hybrid analytic Jacobian's terms
// (solve_cell.hpp:883-1118: lane j < NSPEC the thermal row's species j,
// lane NSPEC the base state, lanes NSPEC+1 / NSPEC+2 the Tgas column at
// T + h / T - h; lane src the stoichiometric block); the result lands in
// lane src's savedJ
template <bool EVT>
__device__ void serve_jac(kbl::LaneCell<LaneGeo<EVT>::N>& s, int src,
                          const SolveOpts& so, double* sJ) {
  constexpr int N = LaneGeo<EVT>::N;
  using namespace kbnet;
  const unsigned FULLM = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  double yf[N], fy[N], f[N], k[NREA + 1];
  KB_UNROLL for (int i = 0; i < N; ++i) yf[i] = __shfl_sync(FULLM, s.y[i], src);
  Params p;
  {
    double row[NPAR];
    const double* ps = reinterpret_cast<const double*>(&s.p);
    KB_UNROLL for (int i = 0; i < NPAR; ++i) row[i] = __shfl_sync(FULLM, ps[i], src);
    params_from_row(row, p);
  }
  const double Tfix = __shfl_sync(FULLM, s.Tfix, src);
  bool hit = false;
  int ret = 0;
  long ndq = 0;
  if (so.jac == 2) {
    KB_UNROLL for (int i = 0; i < N; ++i) fy[i] = __shfl_sync(FULLM, s.ftemp[i], src);
    double ewtf[N];
    KB_UNROLL for (int i = 0; i < N; ++i) ewtf[i] = __shfl_sync(FULLM, s.ewt[i], src);
    const double h = __shfl_sync(FULLM, s.h, src);
    const double srur = kbw::ssqrt_(kbw::UROUND);
    double sum = 0.0;
    KB_UNROLL for (int i = 0; i < N; ++i) {
      const double pv = fy[i] * ewtf[i];
      sum += pv * pv;
    }
    const double fnorm = kbw::ssqrt_(sum / N);
    const double minInc = (fnorm != 0.0)
        ? (kbw::MIN_INC_MULT * fabs(h) * kbw::UROUND * (double)N * fnorm) : 1.0;
    const int j = lane < N ? lane : 0;
    const double yj = kbw::pick<N>(yf, j);
    const double ewj = kbw::pick<N>(ewtf, j);
    const double inc = kbw::smax_(srur * fabs(yj), minInc / ewj);
    KB_UNROLL for (int i = 0; i < N; ++i) yf[i] = (i == lane) ? yf[i] + inc : yf[i];
    int r = kbw::rhs_check<N, EVT>(yf, f, p, Tfix, k, hit);
    if (lane >= N) { r = 0; hit = false; }
    const unsigned bad = __ballot_sync(FULLM, r != 0);
    const int first_bad = bad ? __ffs(bad) - 1 : N;
    ndq = bad ? first_bad + 1 : N;
    ret = bad ? 1 : 0;
    hit = __any_sync(FULLM, hit && lane <= first_bad);
    if (lane < N && lane < first_bad) {
      const double inc_inv = 1.0 / inc;
      KB_UNROLL for (int i = 0; i < N; ++i) sJ[i + lane * N] = inc_inv * (f[i] - fy[i]);
    }
  } else {
    const double T = EVT ? fmin(fmax(yf[N - 1], p.Tcmb), 1e9)
                         : fmin(fmax(Tfix, p.Tcmb), 1e9);
    if (lane == 0) {
      KB_UNROLL for (int i = 0; i <= NREA; ++i) k[i] = 0.0;
      rates_fixed(T, yf, p, k);
      rates_var(T, yf, p, k);
      jac_stoich(yf, k, sJ, 1, N);  // column-major: (i, j) at i + j N
    }
    if (EVT) {
      constexpr int iT = N - 1;
      double sumabs = 0.0;
      KB_UNROLL for (int i = 0; i < NSPEC; ++i) sumabs += fabs(yf[i]);
      const double hT = fmax(1e-6 * fabs(yf[iT]), 1e-8);
      const double yjl = kbw::pick<N>(yf, lane < N ? lane : 0);
      const double hj = lane < NSPEC
          ? fmax(fmax(1e-7 * fabs(yjl), 1e-9 * sumabs), 1e-30) : 1.0;
      KB_UNROLL for (int i = 0; i < N; ++i) {
        double v = yf[i];
        if (lane < NSPEC && i == lane) v = yf[i] + hj;
        if (lane == NSPEC + 1 && i == iT) v = yf[iT] + hT;
        if (lane == NSPEC + 2 && i == iT) v = yf[iT] - hT;
        yf[i] = v;
      }
      const double Tl = (lane == NSPEC + 1 || lane == NSPEC + 2)
                            ? fmin(fmax(yf[iT], p.Tcmb), 1e9) : T;
      KB_UNROLL for (int i = 0; i <= NREA; ++i) k[i] = 0.0;
      rates_fixed(Tl, yf, p, k);
      rates_var(Tl, yf, p, k);
      rhs(yf, k, f);
      const double Tth = fmin(fmax(yf[iT], 2.73), 1e9);
      f[iT] = thermal_dTdt(Tth, yf, k, p);
      double* sv = sJ + N * N;
      __syncwarp();
      if (lane == NSPEC + 1) { KB_UNROLL for (int i = 0; i < N; ++i) sv[i] = f[i]; }
      if (lane == NSPEC + 2) { KB_UNROLL for (int i = 0; i < N; ++i) sv[N + i] = f[i]; }
      __syncwarp();
      if (lane < N) sJ[lane + iT * N] = (sv[lane] - sv[N + lane]) / (2.0 * hT);
      const double f0 = __shfl_sync(FULLM, f[iT], NSPEC);
      if (lane < NSPEC) sJ[iT + lane * N] = (f[iT] - f0) / hj;
    }
  }
  __syncwarp();
  if (lane == src) {
    for (int i = 0; i < N * N; ++i) s.savedJ[i] = sJ[i];
    s.ls_retval = ret;
    s.st[kbw::ST_NFEDQ] += ndq;
    s.hitT0 = s.hitT0 || hit;
  }
  __syncwarp();
}

// start cell c on this lane: false when the cell needs no integration
// (its flag is written here)
template <bool EVT>
__device__ bool lane_start(kbl::LaneCell<LaneGeo<EVT>::N>& s,
                           kbl::Machine<LaneGeo<EVT>::N, EVT>& m, int c,
                           const double* n, const double* T, const double* dt,
                           const double* par, int pstride, int* flags,
                           long* stats, const SolveOpts& so) {
  constexpr int N = LaneGeo<EVT>::N;
  using namespace kbnet;
  const double dtc = dt[c];
  int skip_flag = 1;
  if (so.fail_every > 0 && (c + 1) % so.fail_every == 0) skip_flag = kbw::TOO_MUCH_WORK;
  else if (!(dtc > 0.0)) skip_flag = 0;
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
  s.cell = c;
  s.dt = dtc;
  s.Tfix = T[c];
  s.hitT0 = false;
  s.restarts = 0;
  for (int i = 0; i < NSTAT; ++i) s.tot[i] = 0;
  double y0[N];
  KB_UNROLL for (int i = 0; i < NSPEC; ++i) y0[i] = n[(long)c * NSPEC + i];
  if (EVT) y0[N - 1] = T[c];
  KB_UNROLL for (int i = 0; i < N; ++i) s.atol[i] = i < NSPEC ? so.atol_n : so.atol_T;
  s.atolmin0 = (so.atol_n == 0.0) || (EVT && so.atol_T == 0.0);
  s.mxstep = so.max_steps == 0 ? 500
             : (so.max_steps < 0 ? KB_MAX_STEPS_CAP : so.max_steps);
  m.reinit(0.0, y0, 0.0);
  s.pc = kbl::PC_NEW;
  return true;
}

// the post-solve rules of solve() (solve_cell.hpp:2156-2176) and the
// write-back of a finished cell
template <bool EVT>
__device__ void lane_finish(kbl::LaneCell<LaneGeo<EVT>::N>& s, int flag,
                            double* n, double* T, int* flags, long* stats,
                            const SolveOpts& so) {
  constexpr int N = LaneGeo<EVT>::N;
  using namespace kbnet;
  const int c = s.cell;
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
    KB_UNROLL for (int i = 0; i < NSPEC; ++i) {
      double v = s.y[i];
      if (so.clip_negative && v < 0.0) v = 0.0;
      n[(long)c * NSPEC + i] = v;
    }
    if (EVT) T[c] = Tend;
  }
  if (flags != nullptr) flags[c] = flag;
  s.cell = -1;
}

// one warp = 32 cells in flight. persistent == 0: each lane integrates the
// cell of its global thread index; persistent == 1: lanes pull cells from
// the device work queue (`cursor`) until it is exhausted
template <bool EVT>
__global__ void __launch_bounds__(kWarpsPerBlock * 32)
kb_lane_cells(int ncell, double* n, double* T, const double* dt,
              const double* par, int pstride, int* flags, long* stats,
              SolveOpts so, unsigned* cursor, int persistent) {
  constexpr int N = LaneGeo<EVT>::N;
  extern __shared__ double smem[];
  const int warp = threadIdx.x >> 5;
  double* sJ = smem + warp * LaneGeo<EVT>::SMEM_DOUBLES;
  kbl::LaneCell<N> s;
  kbl::Machine<N, EVT> m(s, so);
  s.cell = -1;
  s.pc = kbl::PC_IDLE;
  bool static_taken = false;
  const int gtid = blockIdx.x * blockDim.x + threadIdx.x;
  bool exhausted = false;
  for (;;) {
    int req = kbl::REQ_NONE;
    // 1. advance this lane to its next request, taking new cells as the
    //    current one finishes
    while (!exhausted) {
      if (s.cell < 0) {
        int c;
        if (persistent) {
          c = (int)atomicAdd(cursor, 1u);
        } else {
          c = static_taken ? ncell : gtid;
          static_taken = true;
        }
        if (c >= ncell) { exhausted = true; break; }
        if (!lane_start<EVT>(s, m, c, n, T, dt, par, pstride, flags, stats, so))
          continue;
      }
      int flag = 0;
      req = m.advance(&flag);
      if (req == kbl::REQ_DONE) {
        lane_finish<EVT>(s, flag, n, T, flags, stats, so);
        req = kbl::REQ_NONE;
        continue;
      }
      break;
    }
    if (__all_sync(0xffffffffu, exhausted)) break;
    // 2. the warp serves the Jacobian requests, one cell at a time
    unsigned jm = __ballot_sync(0xffffffffu, req == kbl::REQ_JAC);
    while (jm) {
      const int src = __ffs(jm) - 1;
      jm &= jm - 1;
      serve_jac<EVT>(s, src, so, sJ);
    }
    // 3. the rhs requests, in one SIMT pass
    if (req == kbl::REQ_RHS) {
      double yf[N], f[N], k[kbnet::NREA + 1];
      KB_UNROLL for (int i = 0; i < N; ++i) yf[i] = s.yreq[i];
      bool hit = false;
      s.rhs_ret = kbw::rhs_check<N, EVT>(yf, f, s.p, s.Tfix, k, hit);
      if (hit) s.hitT0 = true;
      KB_UNROLL for (int i = 0; i < N; ++i) s.freq[i] = f[i];
    }
  }
}

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
  int queue_chunk = 1;     // cells per queue pop
  int blocks_per_sm = 0;   // persistent grid: 0 = occupancy limit
  int fail_every = 0;      // fault injection (tests)
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

int resolved_jac(const krome_opts& h) {
  if (h.jac == 1) return 1;
  if (h.jac == 2) return 2;
  return h.evolve_T ? 2 : 1;  // JAC_AUTO (solve_cell.hpp:2141-2142)
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
  return so;
}

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

template <bool EVT>
cudaError_t launch(const krome_opts& h, int ncell, double* n, double* T,
                   const double* dt, const double* par, int pstride,
                   int* flags, long* stats, unsigned* cursor,
                   cudaStream_t stream) {
  const SolveOpts so = to_solve_opts(h);
  if (h.layout == 1) {  // lane per cell
    const size_t lsmem =
        sizeof(double) * kWarpsPerBlock * LaneGeo<EVT>::SMEM_DOUBLES;
    const int threads = kWarpsPerBlock * 32;
    long blocks;
    if (h.kernel == 0) {
      blocks = ((long)ncell + threads - 1) / threads;
    } else {
      int per_sm = h.blocks_per_sm;
      if (per_sm <= 0) {
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &per_sm, kb_lane_cells<EVT>, threads, lsmem);
        if (per_sm <= 0) per_sm = 1;
      }
      blocks = (long)num_sms() * per_sm;
      const long need = ((long)ncell + threads - 1) / threads;
      if (blocks > need) blocks = need > 0 ? need : 1;
      cudaError_t e = cudaMemsetAsync(cursor, 0, sizeof(unsigned), stream);
      if (e != cudaSuccess) return e;
    }
    kb_lane_cells<EVT><<<(int)blocks, threads, lsmem, stream>>>(
        ncell, n, T, dt, par, pstride, flags, stats, so, cursor, h.kernel);
    return cudaGetLastError();
  }
  const size_t smem = sizeof(double) * kWarpsPerBlock * Geo<EVT>::SMEM_DOUBLES;
  if (h.kernel == 0) {
    const int blocks = (ncell + kWarpsPerBlock - 1) / kWarpsPerBlock;
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
}

cudaError_t launch_any(const krome_opts& h, int ncell, double* n, double* T,
                       const double* dt, const double* par, int pstride,
                       int* flags, long* stats, unsigned* cursor,
                       cudaStream_t stream) {
  return h.evolve_T
      ? launch<true>(h, ncell, n, T, dt, par, pstride, flags, stats, cursor,
                     stream)
      : launch<false>(h, ncell, n, T, dt, par, pstride, flags, stats, cursor,
                      stream);
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
      {"queue_chunk", offsetof(krome_opts, queue_chunk)},
      {"blocks_per_sm", offsetof(krome_opts, blocks_per_sm)},
      {"fail_every", offsetof(krome_opts, fail_every)},
  };
  for (const auto& e : keys)
    if (!std::strcmp(e.name, k))
      return reinterpret_cast<int*>(reinterpret_cast<char*>(h) + e.off);
  return nullptr;
}
double* dbl_key(krome_opts* h, const char* k) {
  if (!std::strcmp(k, "rtol")) return &h->rtol;
  if (!std::strcmp(k, "atol_n")) return &h->atol_n;
  if (!std::strcmp(k, "atol_T")) return &h->atol_T;
  if (!std::strcmp(k, "atol_u")) return &h->atol_u;
  return nullptr;
}
bool bool_key(const char* k) {
  return !std::strcmp(k, "evolve_T") || !std::strcmp(k, "clip_negative")
         || !std::strcmp(k, "error_report") || !std::strcmp(k, "renormalize_x")
         || !std::strcmp(k, "device_cache");
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
  if ((!std::strcmp(key, "max_err_fails") || !std::strcmp(key, "max_conv_fails")
       || !std::strcmp(key, "max_restarts") || !std::strcmp(key, "queue_chunk")
       || !std::strcmp(key, "fail_every") || !std::strcmp(key, "blocks_per_sm"))
      && v < 0.0)
    return -1;
  *iv = x;
  return 0;
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

// ---------------------------------------------------------------------------
// the solves

namespace {
// what this library does not implement returns FLAG_UNSUPPORTED before any
// work: LAPACK and the sparse LU (small networks use the dense LU),
// conservation, photon bins
int unsupported(const krome_opts& h) {
  if (h.linsol == 2 || h.linsol == 3) return -104;
  if (h.conserve != 0) return -104;
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
  if (cursor == nullptr && (h->kernel == 1)) return -1;
  if (const int u = unsupported(*h)) return u;
  const cudaError_t e = launch_any(*h, ncell, n, Tgas, dt, par, par_stride,
                                   flags, stats, cursor,
                                   static_cast<cudaStream_t>(stream));
  return e == cudaSuccess ? 0 : -104;
}

KB_API int krome_b200_solve_batch(int ncell, double* n, double* Tgas,
                                  const double* dt, const double* par,
                                  int par_stride, int* flags, long* stats,
                                  const krome_opts* h) {
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
  if (const int u = unsupported(*h)) {
    if (flags != nullptr)
      for (int c = 0; c < ncell; ++c) flags[c] = u;
    return u;
  }
  const size_t nb = sizeof(double) * (size_t)ncell * kbnet::NSPEC;
  const size_t tb = sizeof(double) * (size_t)ncell;
  const size_t pb = sizeof(double) * (size_t)(ps ? (size_t)ncell * ps : kbnet::NPAR);
  const size_t fb = sizeof(int) * (size_t)ncell;
  const size_t sb = stats != nullptr ? sizeof(long) * (size_t)ncell * NSTAT : 0;
  auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
  const size_t total = al(nb) + 2 * al(tb) + al(pb) + al(fb) + al(sb) + 256;
  std::lock_guard<std::mutex> lock(g_mu);
  if (g_buf.ensure(total) != cudaSuccess) {
    if (flags != nullptr)
      for (int c = 0; c < ncell; ++c) flags[c] = -111;
    return -111;
  }
  char* b = static_cast<char*>(g_buf.p);
  double* dn = reinterpret_cast<double*>(b); b += al(nb);
  double* dT = reinterpret_cast<double*>(b); b += al(tb);
  double* ddt = reinterpret_cast<double*>(b); b += al(tb);
  double* dp = reinterpret_cast<double*>(b); b += al(pb);
  int* dfl = reinterpret_cast<int*>(b); b += al(fb);
  long* dst = sb ? reinterpret_cast<long*>(b) : nullptr; b += al(sb);
  unsigned* dcur = reinterpret_cast<unsigned*>(b);
  cudaStream_t s = 0;
  cudaError_t e = cudaMemcpyAsync(dn, n, nb, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dT, Tgas, tb, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(ddt, dt, tb, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(dp, P, pb, cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess)
    e = launch_any(*h, ncell, dn, dT, ddt, dp, ps, dfl, dst, dcur, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(n, dn, nb, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(Tgas, dT, tb, cudaMemcpyDeviceToHost, s);
  int* hfl = flags != nullptr ? flags : fl.data();
  if (e == cudaSuccess) e = cudaMemcpyAsync(hfl, dfl, fb, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess && sb)
    e = cudaMemcpyAsync(stats, dst, sb, cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    std::fprintf(stderr, "krome_b200: CUDA error %s\n", cudaGetErrorString(e));
    return -104;
  }
  for (int c = 0; c < ncell; ++c)
    if (hfl[c] != 0) return hfl[c];
  return 0;
}

// the reference's entry point (krome.h:291-294): host arrays, in place
KB_API int krome_solve_cells(int ncell, double* n, double* Tgas,
                             const double* dt, const double* par,
                             int par_stride, const void* extra, int* flags,
                             const krome_opts* h) {
  (void)extra;  // no photon bins or dust bins in these networks
  return krome_b200_solve_batch(ncell, n, Tgas, dt, par, par_stride, flags,
                                nullptr, h);
}

KB_API int krome_has_device(void) {
  int count = 0;
  return cudaGetDeviceCount(&count) == cudaSuccess && count > 0 ? 1 : 0;
}

KB_API int krome_b200_nstat(void) { return NSTAT; }
KB_API int krome_b200_neq(int evolve_T) {
  return kbnet::NSPEC + (evolve_T ? 1 : 0);
}
