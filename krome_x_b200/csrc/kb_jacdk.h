// The analytic Jacobian's rate-derivative helpers: the terms d k_r / d n_j
// of the rate coefficients that depend on the densities (directly, or
// through the aggregates ntot, Hnuclei and rho). The emitted jac_dk()
// (networks/net_<net>.h) writes them as the reference's analytic Jacobian
// does (kromex/codegen.py:8462-8560, jacobian_split): symbolic derivatives
// of the rate expressions, and difference quotients of the rate function
// for rates that call a fitted function; the aggregate coupling is kept
// as the low-rank part U W^T, W_aj = d aggregate_a / d n_j.
//
// The difference-quotient rules are the reference's (its generated
// fd_dk_ / fd_dk_agg_), so that the Jacobian -- and with it the solve --
// is the reference's bit for bit. Included inside the network namespace.
#pragma once

// the aggregates a rate may depend on: 0 ntot, 1 Hnuclei, 2 rho; W_aj
constexpr int NAGG = 3;
KB_HD inline double agg_w_(int a, int j) {
  return a == 0 ? 1.0 : (a == 1 ? species_natoms_H(j) : species_mass_g(j));
}

// d(l^r) = l^r (dr ln l + r dl / l), with the limit 0 where l^r underflows
// to 0, is not finite, or l is not positive (the naive form is NaN there)
KB_HD inline double dpow_(double l, double r, double dl, double dr) {
  const double lr = kb_pow(l, r);
  if (l <= 0.0 || lr == 0.0 || !std::isfinite(lr)) return 0.0;
  return lr * (dr * kb_log(l) + r * dl / l);
}

// d rate / d n_j by a difference quotient of the rate function: a central
// difference with step max(1e-7 |n_j|, 1e-30) where n_j exceeds the step,
// else forward; a difference at the roundoff of k0 (1e-15 |k0|) is 0.
// np_ is a copy of n, restored on return
template <class F>
KB_HD inline double fd_dk_(F rate, double* np_, const double* n, double k0,
                           int j) {
  const double h = std::fmax(1e-7 * std::fabs(n[j]), 1e-30);
  np_[j] = n[j] + h;
  const double kp = rate(np_);
  double km = k0, den = h;
  if (n[j] > h) {
    np_[j] = n[j] - h;
    km = rate(np_);
    den = 2.0 * h;
  }
  np_[j] = n[j];
  if (std::fabs(kp - km) <= 1e-15 * std::fabs(k0)) return 0.0;
  return (kp - km) / den;
}

// d rate / d aggregate c[a] for the aggregates of `mask` (bit a): along
// each aggregate's dominant carrier j_q (the species of largest
// |W_aj n_j| outside the rate's direct species and the carriers already
// taken) the difference quotient g_q = sum_a c_a W_a,j_q; the m <= 3
// equations solved by elimination with partial pivoting. No carrier: no
// dependence to resolve (c stays 0)
template <class F>
KB_HD inline void fd_dk_agg_(F rate, double* np_, const double* n, double k0,
                             int mask, const int* dir, int ndir, double* c) {
  int am[NAGG], pj[NAGG], m = 0;
  for (int a = 0; a < NAGG; ++a) {
    c[a] = 0.0;
    if (mask & (1 << a)) am[m++] = a;
  }
  double M[NAGG][NAGG + 1];
  for (int q = 0; q < m; ++q) {
    int best = -1;
    double bv = 0.0;
    for (int j = 0; j < NSPEC; ++j) {
      bool skip = false;
      for (int t = 0; t < ndir; ++t) skip = skip || dir[t] == j;
      for (int t = 0; t < q; ++t) skip = skip || pj[t] == j;
      const double v = std::fabs(agg_w_(am[q], j) * n[j]);
      if (!skip && v > bv) {
        bv = v;
        best = j;
      }
    }
    if (best < 0) return;
    pj[q] = best;
    for (int r = 0; r < m; ++r) M[q][r] = agg_w_(am[r], best);
    M[q][m] = fd_dk_(rate, np_, n, k0, best);
  }
  for (int col = 0; col < m; ++col) {
    int piv = col;
    for (int r = col + 1; r < m; ++r)
      if (std::fabs(M[r][col]) > std::fabs(M[piv][col])) piv = r;
    if (M[piv][col] == 0.0) return;
    for (int t = 0; t <= m; ++t) {
      const double x = M[piv][t];
      M[piv][t] = M[col][t];
      M[col][t] = x;
    }
    for (int r = col + 1; r < m; ++r) {
      const double f = M[r][col] / M[col][col];
      for (int t = col; t <= m; ++t) M[r][t] -= f * M[col][t];
    }
  }
  double x[NAGG];
  for (int r = m - 1; r >= 0; --r) {
    double v = M[r][m];
    for (int t = r + 1; t < m; ++t) v -= M[r][t] * x[t];
    x[r] = v / M[r][r];
  }
  for (int r = 0; r < m; ++r) c[am[r]] = x[r];
}

// the aggregate part sum_a c_a W_aj of a total derivative along n_j
KB_HD inline double agg_part_(const double* c, int j) {
  double s = 0.0;
  for (int a = 0; a < NAGG; ++a) s += c[a] * agg_w_(a, j);
  return s;
}

// J += U W^T on the species block (J element (i, j) at J[i rs + j cs])
KB_HD inline void jac_agg_(double* J, const double* U, long rs, long cs) {
  for (int i = 0; i < NSPEC; ++i)
    for (int a = 0; a < NAGG; ++a) {
      const double u = U[i * NAGG + a];
      if (u == 0.0) continue;
      for (int j = 0; j < NSPEC; ++j) J[i * rs + j * cs] += u * agg_w_(a, j);
    }
}
