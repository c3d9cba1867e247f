// Conservation of a cell's element totals and net charge, for host and
// device (KB_HD): the post-solve `conserve` option and consistent advection
// (the behaviour of the reference's runtime/core/solve_cell.hpp:1333-1560,
// conserve_cell_ / conserve_to_n_ / conserve_to_x_).
//
// The behaviour, per mode of the post-solve option:
//
//   mode 1   the electrons restore the input net charge
//   mode 2   the densities moved onto the input element totals and net
//            charge by the least relative change
//   mode 3   the electrons neutralize the ions, n(e-) = max(sum q n, 0)
//
// The projection of mode 2 and of consistent advection, written for this
// library: with the conserved rows a_k (element counts, then the charge) of
// the movable species and the mismatch r = target - A n, the correction
// minimising sum_i d_i^2 / n_i under A d = r is d = W A^T lam with
// W = diag(n) (a species at zero stays zero) and the Gram system
// G lam = r, G = A W A^T: a symmetric positive semi-definite matrix of at
// most NELEM + 1 rows, built in one pass over the species and factored by
// LDL^T with diagonal pivoting. Rows whose remaining pivot falls to 1e-14
// of the largest diagonal have no independent freedom (no free carrier, or
// a combination of the other rows); their multiplier stays 0. The
// correction is unique whenever the system is consistent, so the choice of
// factorisation changes only the last bits. A correction that drives a
// species negative clips it to zero; the projection is then repeated from
// the clipped state, at most 20 passes, until the largest relative
// mismatch is below 1e-13.
//
// Opaque species never move, nor do the species a freeze directive holds
// for the cell's parameters (the reference's conserved_fixed_,
// solve_cell.hpp:1442-1450). Included inside the network namespace after
// the species tables and the parameters; n0 and n are a cell's NSPEC
// densities in any memory the caller can address.
#pragma once

namespace kbcons {
constexpr int kPasses = 20;          // projection passes after clipping
constexpr double kDone = 1e-13;      // mismatch that ends the passes
constexpr double kRankTol = 1e-14;   // pivot / largest diagonal: dependent
constexpr double kUnreached = 1e-12; // consistent advection: -112 above
}  // namespace kbcons

// conserved quantity k of species i: atoms of element k (k < NELEM), or the
// charge (k == NELEM)
KB_HD inline double cons_coef(int k, int i) {
  return k < NELEM ? (double)species_element(i, k) : (double)species_charge(i);
}

// largest relative mismatch of the first `rows` conserved totals of n
// against target: |target_k - (A n)_k| / max(|target_k|, sum_i |A_ki n_i|)
KB_HD inline double cons_mismatch(const double* n, const double* target,
                                  int rows) {
  double worst = 0.0;
  for (int k = 0; k < rows; ++k) {
    double sum = 0.0, mag = std::fabs(target[k]);
    for (int i = 0; i < NSPEC; ++i) {
      const double v = cons_coef(k, i) * n[i];
      sum += v;
      mag += std::fabs(v);
    }
    if (mag > 0.0) worst = std::fmax(worst, std::fabs(target[k] - sum) / mag);
  }
  return worst;
}

// one least-change correction of n towards target over the first `rows`
// conserved quantities; movable[i] marks the species that may move. Returns
// true when a correction clipped a species at zero.
KB_HD inline bool cons_correct(double* n, const double* target, int rows,
                               const bool* movable) {
  constexpr int R = NELEM + 1;
  double G[R][R], rhs[R], lam[R];
  int order[R];
  // the Gram matrix and the mismatch, one pass over the species
  for (int k = 0; k < rows; ++k) {
    rhs[k] = target[k];
    order[k] = k;
    lam[k] = 0.0;
    for (int l = 0; l < rows; ++l) G[k][l] = 0.0;
  }
  for (int i = 0; i < NSPEC; ++i) {
    double a[R];
    for (int k = 0; k < rows; ++k) a[k] = cons_coef(k, i);
    for (int k = 0; k < rows; ++k) rhs[k] -= a[k] * n[i];
    if (!movable[i]) continue;
    for (int k = 0; k < rows; ++k) {
      if (a[k] == 0.0) continue;
      const double ak = a[k] * n[i];
      for (int l = 0; l < rows; ++l) G[k][l] += ak * a[l];
    }
  }
  double dmax = 0.0;
  for (int k = 0; k < rows; ++k) dmax = std::fmax(dmax, G[k][k]);
  // LDL^T with diagonal pivoting: step s takes the largest remaining
  // diagonal; the trailing block is updated in place (upper triangle used)
  int rank = 0;
  for (int s = 0; s < rows; ++s) {
    int m = s;
    for (int k = s + 1; k < rows; ++k)
      if (G[k][k] > G[m][m]) m = k;
    if (!(G[m][m] > kbcons::kRankTol * dmax)) break;
    if (m != s) {
      for (int l = 0; l < rows; ++l) {
        const double t = G[s][l]; G[s][l] = G[m][l]; G[m][l] = t;
      }
      for (int l = 0; l < rows; ++l) {
        const double t = G[l][s]; G[l][s] = G[l][m]; G[l][m] = t;
      }
      const double t = rhs[s]; rhs[s] = rhs[m]; rhs[m] = t;
      const int o = order[s]; order[s] = order[m]; order[m] = o;
    }
    const double inv = 1.0 / G[s][s];
    for (int k = s + 1; k < rows; ++k) {
      const double f = G[k][s] * inv;
      if (f == 0.0) continue;
      for (int l = s + 1; l < rows; ++l) G[k][l] -= f * G[s][l];
      rhs[k] -= f * rhs[s];
    }
    rank = s + 1;
  }
  // back substitution over the independent rows
  double y[R];
  for (int s = rank - 1; s >= 0; --s) {
    double v = rhs[s];
    for (int l = s + 1; l < rank; ++l) v -= G[s][l] * y[l];
    y[s] = v / G[s][s];
  }
  for (int s = 0; s < rank; ++s) lam[order[s]] = y[s];
  // d_i = n_i sum_k a_ki lam_k
  bool clipped = false;
  for (int i = 0; i < NSPEC; ++i) {
    if (!movable[i]) continue;
    double g = 0.0;
    for (int k = 0; k < rows; ++k) g += cons_coef(k, i) * lam[k];
    const double v = n[i] + n[i] * g;
    clipped = clipped || v < 0.0;
    n[i] = v < 0.0 ? 0.0 : v;
  }
  return clipped;
}

// the projection with its passes; returns the final mismatch
KB_HD inline double cons_project(double* n, const double* target, int rows,
                                 const bool* movable) {
  for (int pass = 0; pass < kbcons::kPasses; ++pass) {
    const bool clipped = cons_correct(n, target, rows, movable);
    if (!clipped) break;
    if (cons_mismatch(n, target, rows) < kbcons::kDone) break;
  }
  return cons_mismatch(n, target, rows);
}

// the net charge sum_i q_i n_i, optionally without one species
KB_HD inline double cons_charge(const double* n, int skip = -1) {
  double q = 0.0;
  for (int i = 0; i < NSPEC; ++i)
    if (i != skip) q += species_charge(i) * n[i];
  return q;
}

// the species that do not move for a cell with parameters p: the opaque
// ones and those a freeze directive holds
KB_HD inline void conserved_fixed(const Params& p, bool* fixed) {
  for (int i = 0; i < NSPEC; ++i) fixed[i] = species_opaque(i) != 0;
#if KB_NFREEZE > 0
  int idx[KB_NFREEZE];
  const int m = frozen_species(p, idx);
  for (int q = 0; q < m; ++q) fixed[idx[q]] = true;
#else
  (void)p;
#endif
}

// the post-solve conservation of a solved cell n against its input n0
// (mode 0: none); mode 3 sets the electrons even while a freeze directive
// holds them (the reference's order: applied after the solve)
KB_HD inline void conserve_cell(const double* n0, double* n, int mode,
                                const Params& p) {
  if (mode <= 0) return;
  const int e = IDX_ELECTRON;
  if (mode == 3) {
    if (e >= 0) n[e] = std::fmax(cons_charge(n, e), 0.0);
    return;
  }
  bool fixed[NSPEC];
  conserved_fixed(p, fixed);
  if (mode == 1) {
    if (e >= 0 && !fixed[e])
      n[e] = std::fmax(n[e] + (cons_charge(n) - cons_charge(n0)), 0.0);
    return;
  }
  double target[NELEM + 1];
  for (int k = 0; k <= NELEM; ++k) {
    double t = 0.0;
    for (int i = 0; i < NSPEC; ++i) t += cons_coef(k, i) * n0[i];
    target[k] = t;
  }
  bool movable[NSPEC];
  for (int i = 0; i < NSPEC; ++i) movable[i] = !fixed[i];
  cons_project(n, target, NELEM + 1, movable);
}

// consistent advection (legacy krome_conserveLin_x): the advected cell n
// moved to the element totals ref[NELEM] and to zero net charge. fixed[i]
// marks the species that do not move. Steps: clip the movable species'
// negatives; the elements by the projection without the charge row (the
// ionization is kept); then the electrons from neutrality (the sum of the
// other charges) when that is non-negative, else the charge row joins the
// projection. Returns 0, -112 when the totals or neutrality stay out of
// reach (the cell corrected as far as possible), or the warning 2 when a
// species changed by more than half.
KB_HD inline int conserve_to_n(double* n, const double* ref,
                               const bool* fixed) {
  double start[NSPEC];
  bool movable[NSPEC];
  for (int i = 0; i < NSPEC; ++i) {
    movable[i] = !fixed[i];
    if (movable[i] && n[i] < 0.0) n[i] = 0.0;
    start[i] = n[i];
  }
  double target[NELEM + 1];
  for (int k = 0; k < NELEM; ++k) target[k] = ref[k];
  target[NELEM] = 0.0;
  cons_project(n, target, NELEM, movable);
  const int e = IDX_ELECTRON;
  bool neutral = false;
  if (e >= 0 && movable[e]) {
    const double q = cons_charge(n, e);
    neutral = q >= 0.0;
    n[e] = neutral ? q : 0.0;
  }
  if (!neutral) cons_project(n, target, NELEM + 1, movable);
  if (cons_mismatch(n, target, NELEM + 1) > kbcons::kUnreached) return -112;
  for (int i = 0; i < NSPEC; ++i)
    if (start[i] > 0.0 && std::fabs(n[i] - start[i]) > 0.5 * start[i])
      return 2;
  return 0;
}

// consistent advection of a cell with parameters p (its frozen species do
// not move)
KB_HD inline int conserve_to(double* n, const double* ref, const Params& p) {
  bool fixed[NSPEC];
  conserved_fixed(p, fixed);
  return conserve_to_n(n, ref, fixed);
}

// the same with mass fractions x and ref per gram: n = x / m per gram,
// corrected, x = m n; a species without mass does not move
KB_HD inline int conserve_to_x(double* x, const double* ref, const Params& p) {
  bool fixed[NSPEC];
  conserved_fixed(p, fixed);
  double n[NSPEC];
  for (int i = 0; i < NSPEC; ++i) {
    const double m = species_mass_g(i);
    if (!(m > 0.0)) fixed[i] = true;
    n[i] = m > 0.0 ? x[i] / m : 0.0;
  }
  const int f = conserve_to_n(n, ref, fixed);
  for (int i = 0; i < NSPEC; ++i)
    if (!fixed[i]) x[i] = species_mass_g(i) * n[i];
  return f;
}
