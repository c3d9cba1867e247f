// Photon bins of a solve handle (krome_opts_set_photo): the per-bin
// averages of the network's photo cross sections that turn a cell's photon
// field Phi[B] (photons cm^-2 s^-1 per bin) into its photo rates
// k_r = sum_b sigma_rb Phi_b, the photoheating weights and the field's
// Habing and Lyman-Werner integrals. Host code; the kernels receive sigma
// and each cell's Phi row and form the rates once per cell (the field is
// fixed during a solve: Params::kph).
//
// The averages follow the reference's bin setup (runtime/core/photo.hpp:
// 145-260, PhotoModule::init), because the same bins must give the same
// rates: inside a bin the photon spectrum is dN/dE ~ E^-alpha, and
//   sigma_rb  = int_{bin ^ [Emin_r, Emax_r]} sigma_r(E) E^-alpha dE
//               / int_bin E^-alpha dE,
//   sigmaE_rb = the same with sigma_r(E) (E - Emin_r), the photoelectron
//               energy each absorption deposits,
// by the midpoint rule on 64 cells of the overlap (in E for alpha = 0,
// else in ln E with each cell's exact weight int E^-alpha dE). A tabulated
// cross section may be Doppler broadened: at E it is the table's mean over
// [E - w/2, E + w/2], w = E b / c, b^2 = 2 kB T / m + v_turb^2.
#pragma once

#include <cmath>
#include <vector>

namespace kbphoto {

constexpr int kQuad = 64;
constexpr double kLwLo = 11.2, kLwHi = 13.6;   // the Lyman-Werner band [eV]
constexpr double kHabLo = 6.0, kHabHi = 13.6;  // the Habing band [eV]
constexpr double kHabing = 1.6e-3;             // erg cm^-2 s^-1 per G0

// int_a^c E^-alpha dE
inline double in_bin_weight(double alpha, double a, double c) {
  if (alpha == 1.0) return std::log(c / a);
  if (alpha == 0.0) return c - a;
  const double q = 1.0 - alpha;
  return (std::pow(c, q) - std::pow(a, q)) / q;
}

struct Bins {
  int B = 0;
  double alpha = 1.0, broad_T = 0.0, broad_vturb = 0.0;
  std::vector<double> lo, hi;
  std::vector<double> sigma, sigmaE;  // [NPHOTO][B]
  std::vector<double> habw, lww;      // [B]: Habing flux and J_LW per Phi_b
  std::vector<double> kdust;          // [B] or empty: dust opacity per bin
};

// the bins' tables; false when a bin is not 0 < lo < hi
inline bool build(Bins& pb, int B, const double* lo, const double* hi,
                  double alpha, double broad_T, double broad_vturb) {
  for (int b = 0; b < B; ++b)
    if (!(lo[b] > 0.0 && hi[b] > lo[b])) return false;
  pb.B = B;
  pb.alpha = alpha;
  pb.broad_T = broad_T;
  pb.broad_vturb = broad_vturb;
  pb.lo.assign(lo, lo + B);
  pb.hi.assign(hi, hi + B);
  pb.sigma.assign((size_t)kbnet::NPHOTO * B, 0.0);
  pb.sigmaE.assign((size_t)kbnet::NPHOTO * B, 0.0);
  pb.habw.assign(B, 0.0);
  pb.lww.assign(B, 0.0);
  if (pb.kdust.size() != (size_t)B) pb.kdust.clear();
  for (int b = 0; b < B; ++b) {
    const double a = std::fmax(lo[b], kLwLo), c = std::fmin(hi[b], kLwHi);
    if (c <= a) continue;
    // J_LW per Phi_b: (h / 4 pi) int_overlap E^-alpha dE over the bin's
    // and the band's widths
    if (alpha == 1.0)
      pb.lww[b] = kbc::planck_eV * std::log(c / a)
          / (4.0 * kbc::pi * std::log(hi[b] / lo[b]) * std::log(kLwHi / kLwLo));
    else
      pb.lww[b] = kbc::planck_eV * in_bin_weight(alpha, a, c)
          / (4.0 * kbc::pi * in_bin_weight(alpha, lo[b], hi[b])
             * std::log(kLwHi / kLwLo));
  }
  for (int b = 0; b < B; ++b) {
    const double a = std::fmax(lo[b], kHabLo), c = std::fmin(hi[b], kHabHi);
    if (c <= a) continue;
    // the energy flux of the overlap per Phi_b, in Habing units
    if (alpha == 0.0)
      pb.habw[b] = (c * c - a * a) / (2.0 * (hi[b] - lo[b]))
          * kbc::eV_to_erg / kHabing;
    else
      pb.habw[b] = in_bin_weight(alpha - 1.0, a, c)
          / in_bin_weight(alpha, lo[b], hi[b]) * kbc::eV_to_erg / kHabing;
  }
  for (int r = 0; r < kbnet::NPHOTO; ++r) {
    const int sp = kbnet::photo_reactant_[r];
    const double b2 = (broad_T > 0.0
                           ? 2.0 * kbc::boltzmann_erg * broad_T
                                 / kbnet::species_mass_g(sp)
                           : 0.0) + broad_vturb * broad_vturb;
    const bool tab = kbnet::kbxs::photo_xsec_int[r] != nullptr;
    const double dsh = tab ? std::sqrt(b2) / kbc::clight : 0.0;
    auto xs = [&](double E) {
      if (dsh > 0.0) {
        const double wd = dsh * E;
        return kbnet::kbxs::photo_xsec_int[r](E - 0.5 * wd, E + 0.5 * wd) / wd;
      }
      return kbnet::kbxs::photo_xsec[r](E);
    };
    const double emin = kbnet::photo_Emin_[r];
    const double e_lo = emin * (1.0 - 0.5 * dsh);
    const double e_hi = kbnet::photo_Emax_[r] * (1.0 + 0.5 * dsh);
    for (int b = 0; b < B; ++b) {
      const double w = in_bin_weight(alpha, lo[b], hi[b]);
      const double a = std::fmax(lo[b], e_lo), c = std::fmin(hi[b], e_hi);
      if (c <= a) continue;
      const double dE = (c - a) / kQuad;
      const double dl = std::log(c / a) / kQuad;
      double s = 0.0, se = 0.0;
      for (int q = 0; q < kQuad; ++q) {
        const double E = alpha == 0.0 ? a + (q + 0.5) * dE
                                      : a * std::exp((q + 0.5) * dl);
        const double x = xs(E) * (alpha == 0.0 ? dE
            : in_bin_weight(alpha, a * std::exp(q * dl),
                            q + 1 == kQuad ? c : a * std::exp((q + 1) * dl)));
        const double Ee = std::fmax(E - emin, 0.0);
        s += x;
        se += x * Ee;
      }
      pb.sigma[(size_t)r * B + b] = s / w;
      pb.sigmaE[(size_t)r * B + b] = se / w;
    }
  }
  return true;
}

// the photo rates of one field row: k_r = sum_b sigma_rb Phi_b (sequential
// in b, the order the kernels use)
KB_HD inline void rates_of_field(const double* sigma, int B, const double* phi,
                                 double* kph) {
  for (int r = 0; r < kbnet::NPHOTO; ++r) {
    double s = 0.0;
    for (int b = 0; b < B; ++b) s += sigma[(size_t)r * B + b] * phi[b];
    kph[r] = s;
  }
}

}  // namespace kbphoto
