// The post-solve conservation of a cell (the conserve option), restated for
// host and device (KB_HD) from the reference's runtime
// (runtime/core/solve_cell.hpp:1333-1500, conserved_row_, totals_residual_,
// project_totals_, conserve_cell_):
//
//   mode 1   the electrons restore the input net charge
//   mode 2   the densities projected onto the input element totals and net
//            charge: the minimal relative correction d_i = n_i sum_k A_ki
//            lambda_k (a species at zero stays zero), lambda from the small
//            system (A W A^T) lambda = residual by Gaussian elimination with
//            partial pivoting (dependent rows skipped), repeated after
//            clipping negatives up to 20 times until the residual is below
//            1e-13
//   mode 3   the electrons neutralize the ions, n(e-) = max(sum q n, 0)
//
// Rows of A: the element counts (k < NELEM), then the charge. Opaque
// species do not move (the networks here have no freeze directives).
// Included inside the network namespace after the species tables; n0 and n
// are a cell's NSPEC densities (any memory the caller can address).
#pragma once

KB_HD inline double conserved_row_(int k, int i) {
  return k < NELEM ? (double)species_element(i, k) : (double)species_charge(i);
}

// the largest relative residual |target - sum A n| / max(|target|, sum |A n|)
KB_HD inline double totals_residual_(const double* n, const double* target,
                                     bool charge) {
  double worst = 0.0;
  for (int k = 0; k < NELEM + (charge ? 1 : 0); ++k) {
    double t = 0.0, sc = std::fabs(target[k]);
    for (int i = 0; i < NSPEC; ++i) {
      const double a = conserved_row_(k, i) * n[i];
      t += a;
      sc += std::fabs(a);
    }
    if (sc > 0.0) worst = std::fmax(worst, std::fabs(target[k] - t) / sc);
  }
  return worst;
}

// fixed: the species that do not move (nullptr: the opaque ones)
KB_HD inline double project_totals_(double* n, const double* target,
                                    bool charge, const bool* fixed = nullptr) {
  constexpr int NRMAX = NELEM + 1;
  const int NR = NELEM + (charge ? 1 : 0);
  for (int it = 0; it < 20; ++it) {
    double r[NRMAX], M[NRMAX][NRMAX];
    for (int k = 0; k < NR; ++k) {
      double t1 = 0.0;
      for (int i = 0; i < NSPEC; ++i) t1 += conserved_row_(k, i) * n[i];
      r[k] = target[k] - t1;
      for (int l = 0; l < NR; ++l) {
        double s = 0.0;
        for (int i = 0; i < NSPEC; ++i)
          if (!(fixed != nullptr ? fixed[i] : species_opaque(i)))
            s += conserved_row_(k, i) * conserved_row_(l, i) * n[i];
        M[k][l] = s;
      }
    }
    double lam[NRMAX];
    for (int k = 0; k < NR; ++k) lam[k] = 0.0;
    double scale = 0.0;
    for (int k = 0; k < NR; ++k) scale = std::fmax(scale, std::fabs(M[k][k]));
    bool used[NRMAX];
    for (int k = 0; k < NRMAX; ++k) used[k] = false;
    for (int col = 0; col < NR; ++col) {
      // a pivot below 1e-14 of the largest diagonal: the row depends on
      // the others (or has no free species), its lambda stays 0
      int piv = -1;
      double best = 1e-14 * scale;
      for (int row = col; row < NR; ++row)
        if (std::fabs(M[row][col]) > best) {
          best = std::fabs(M[row][col]);
          piv = row;
        }
      if (piv < 0) continue;
      if (piv != col) {
        for (int l = 0; l < NR; ++l) {
          const double t = M[piv][l];
          M[piv][l] = M[col][l];
          M[col][l] = t;
        }
        const double t = r[piv];
        r[piv] = r[col];
        r[col] = t;
      }
      used[col] = true;
      for (int row = col + 1; row < NR; ++row) {
        const double f = M[row][col] / M[col][col];
        for (int l = col; l < NR; ++l) M[row][l] -= f * M[col][l];
        r[row] -= f * r[col];
      }
    }
    for (int col = NR - 1; col >= 0; --col) {
      if (!used[col]) continue;
      double s = r[col];
      for (int l = col + 1; l < NR; ++l) s -= M[col][l] * lam[l];
      lam[col] = s / M[col][col];
    }
    bool clipped = false;
    for (int i = 0; i < NSPEC; ++i) {
      if (fixed != nullptr ? fixed[i] : species_opaque(i)) continue;
      double d = 0.0;
      for (int k = 0; k < NR; ++k) d += conserved_row_(k, i) * lam[k];
      n[i] += n[i] * d;
      if (n[i] < 0.0) {
        n[i] = 0.0;
        clipped = true;
      }
    }
    if (!clipped || totals_residual_(n, target, charge) < 1e-13) break;
  }
  return totals_residual_(n, target, charge);
}

// the conservation of a solved cell n against its input n0 (mode 0: none)
KB_HD inline void conserve_cell(const double* n0, double* n, int mode) {
  if (mode <= 0) return;
  if (mode == 3) {
    if (IDX_ELECTRON >= 0) {
      double qi = 0.0;
      for (int i = 0; i < NSPEC; ++i)
        if (i != IDX_ELECTRON) qi += species_charge(i) * n[i];
      n[IDX_ELECTRON] = std::fmax(qi, 0.0);
    }
    return;
  }
  if (mode == 1) {
    if (IDX_ELECTRON >= 0 && !species_opaque(IDX_ELECTRON)) {
      double q0 = 0.0, q = 0.0;
      for (int i = 0; i < NSPEC; ++i) {
        q0 += species_charge(i) * n0[i];
        q += species_charge(i) * n[i];
      }
      n[IDX_ELECTRON] = std::fmax(n[IDX_ELECTRON] + (q - q0), 0.0);
    }
    return;
  }
  double target[NELEM + 1];
  for (int k = 0; k <= NELEM; ++k) {
    target[k] = 0.0;
    for (int i = 0; i < NSPEC; ++i) target[k] += conserved_row_(k, i) * n0[i];
  }
  project_totals_(n, target, true);
}

// consistent advection (the reference's conserve_to_n_ / conserve_to_x_,
// solve_cell.hpp:1504-1560; legacy krome_conserveLin_x): the cell n moved
// to the element totals ref[NELEM] and to zero net charge. Negatives are
// clipped first; the elements by the projection without the charge row
// (the ionization is kept); then the electrons from neutrality, n(e-) =
// sum q n over the other species, or, when the electrons cannot do it
// (anions dominate, or no free electrons), the charge too by the
// projection. fixed species do not move. Returns 0, -112 when the totals
// or neutrality cannot be reached (corrected as far as possible), or the
// warning 2 when a species changed by more than 50 %.
KB_HD inline int conserve_to_n(double* n, const double* ref,
                               const bool* fixed) {
  double n0[NSPEC];
  for (int i = 0; i < NSPEC; ++i) {
    if (!fixed[i] && n[i] < 0.0) n[i] = 0.0;
    n0[i] = n[i];
  }
  double target[NELEM + 1];
  for (int k = 0; k < NELEM; ++k) target[k] = ref[k];
  target[NELEM] = 0.0;
  project_totals_(n, target, false, fixed);
  bool charge_done = false;
  if (IDX_ELECTRON >= 0 && !fixed[IDX_ELECTRON]) {
    double qi = 0.0;
    for (int i = 0; i < NSPEC; ++i)
      if (i != IDX_ELECTRON) qi += species_charge(i) * n[i];
    if (qi >= 0.0) {
      n[IDX_ELECTRON] = qi;
      charge_done = true;
    } else {
      n[IDX_ELECTRON] = 0.0;
    }
  }
  if (!charge_done) project_totals_(n, target, true, fixed);
  if (totals_residual_(n, target, true) > 1e-12) return -112;
  for (int i = 0; i < NSPEC; ++i)
    if (n0[i] > 0.0 && std::fabs(n[i] - n0[i]) > 0.5 * n0[i]) return 2;
  return 0;
}
// the same with mass fractions x and ref per gram: n = x / m per gram,
// corrected, x = m n; a species without mass does not move
KB_HD inline int conserve_to_x(double* x, const double* ref) {
  bool fixed[NSPEC];
  double n[NSPEC];
  for (int i = 0; i < NSPEC; ++i) {
    fixed[i] = species_opaque(i) || !(species_mass_g(i) > 0.0);
    n[i] = species_mass_g(i) > 0.0 ? x[i] / species_mass_g(i) : 0.0;
  }
  const int f = conserve_to_n(n, ref, fixed);
  for (int i = 0; i < NSPEC; ++i)
    if (!fixed[i]) x[i] = species_mass_g(i) * n[i];
  return f;
}
