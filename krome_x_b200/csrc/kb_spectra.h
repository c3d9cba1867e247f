// Photon-field helpers of the reference's interface (the radiation part of
// runtime/interfaces/C/krome.h; reference runtime/core/spectra.hpp): bin
// edges, the conversion between a specific intensity constant across a bin
// and the bin's photon flux, and the analytic spectra, integrated over each
// bin. Host code only: a caller builds its photon field Phi[nbins] (photon
// flux per bin [cm^-2 s^-1]) with these before a solve.
//
// Convention (the reference's): a field is the bin integral
//   Phi_b = 4 pi / h  int_{Elo_b}^{Ehi_b} J(E) d ln E
// of the specific intensity J [eV s^-1 cm^-2 Hz^-1 sr^-1], so a J constant
// across a bin gives 4 pi J ln(Ehi/Elo) / h. The spectra with a closed-form
// integral (Draine 1978, a J21 power law, a piecewise-interpolated table)
// are integrated exactly; the blackbody by composite 4-point Gauss-Legendre
// quadrature in ln E with sub-intervals of at most 0.02.
#pragma once

#include <cmath>
#include <vector>

namespace kbspec {

constexpr double kPi4 = 4.0 * kbc::pi;

inline bool bins_valid(int B, const double* lo, const double* hi) {
  if (B <= 0 || lo == nullptr || hi == nullptr) return false;
  for (int b = 0; b < B; ++b)
    if (!(lo[b] > 0.0) || !(hi[b] > lo[b])) return false;
  return true;
}

// B equal bins of [lower, upper] in E, or in log10 E
inline void bins_linear(int B, double lower, double upper, double* lo,
                        double* hi) {
  const double w = (upper - lower) / B;
  for (int b = 0; b < B; ++b) {
    lo[b] = lower + b * w;
    hi[b] = lower + (b + 1) * w;
  }
}
inline void bins_logarithmic(int B, double lower, double upper, double* lo,
                             double* hi) {
  const double a = std::log10(lower), w = (std::log10(upper) - a) / B;
  for (int b = 0; b < B; ++b) {
    lo[b] = std::pow(10.0, a + b * w);
    hi[b] = std::pow(10.0, a + (b + 1) * w);
  }
}

inline double flux_of_intensity(double J, double lo, double hi) {
  return kPi4 * J * std::log(hi / lo) / kbc::planck_eV;
}
inline double intensity_of_flux(double phi, double lo, double hi) {
  return phi * kbc::planck_eV / (kPi4 * std::log(hi / lo));
}

// int f(E) d ln E over [lo, hi]: composite 4-point Gauss-Legendre in ln E
template <class F>
inline double integrate_dlnE(F f, double lo, double hi) {
  if (!(hi > lo)) return 0.0;
  // Gauss-Legendre nodes and weights on [-1, 1], 4 points
  const double x[4] = {-0.8611363115940526, -0.3399810435848563,
                       0.3399810435848563, 0.8611363115940526};
  const double wq[4] = {0.3478548451374538, 0.6521451548625461,
                        0.6521451548625461, 0.3478548451374538};
  const double a = std::log(lo), span = std::log(hi) - a;
  int m = (int)std::ceil(span / 0.02);
  if (m < 1) m = 1;
  const double h = span / m;
  double s = 0.0;
  for (int i = 0; i < m; ++i) {
    const double mid = a + (i + 0.5) * h;
    for (int q = 0; q < 4; ++q) s += wq[q] * f(std::exp(mid + 0.5 * h * x[q]));
  }
  return 0.5 * h * s;
}

// the Planck specific intensity B_nu(T) [eV s^-1 cm^-2 Hz^-1 sr^-1],
// 2 E^3 / (h^2 c^2) / (exp(E / kT) - 1), taken as 0 beyond E / kT = 300
inline double planck_intensity(double E, double T) {
  const double x = E / (kbc::boltzmann_eV * T);
  if (!(x < 300.0) || !(E > 1e-10)) return 0.0;
  return 2.0 * E * E * E
      / (kbc::planck_eV * kbc::planck_eV * kbc::clight * kbc::clight)
      / std::expm1(x);
}

inline void field_blackbody(int B, const double* lo, const double* hi,
                            double T, double* phi) {
  for (int b = 0; b < B; ++b)
    phi[b] = kPi4 / kbc::planck_eV
        * integrate_dlnE([T](double E) { return planck_intensity(E, T); },
                         lo[b], hi[b]);
}

// the photon range of a blackbody: from the Rayleigh-Jeans energy where
// B_nu falls to eps = 1e-6, to the energy above the peak where it falls to
// eps (bisection between the Wien-displacement estimate and 290 kT);
// -1 when B_nu never reaches eps
inline int blackbody_limits(double T, double* lower, double* upper) {
  const double eps = 1e-6;
  *lower = kbc::planck_eV * kbc::clight * std::sqrt(0.5 * eps / (T * kbc::boltzmann_eV));
  double a = T / 2.8977721e-1 * kbc::clight * kbc::planck_eV;
  double c = 290.0 * kbc::boltzmann_eV * T;
  if (planck_intensity(a, T) < eps || planck_intensity(c, T) > eps) return -1;
  double m = 0.5 * (a + c);
  for (int it = 0; it < 400; ++it) {
    m = 0.5 * (a + c);
    const double f = planck_intensity(m, T) - eps;
    if (std::fabs(f) < 1e-9 * eps) break;
    if (f > 0.0) a = m;
    else c = m;
  }
  *upper = m;
  return 0;
}

// Draine (1978) interstellar field: photon intensity
// 1.658e6 E - 2.152e5 E^2 + 6.919e3 E^3 [cm^-2 s^-1 sr^-1 eV^-1] over
// 5-13.6 eV; Phi_b = 4 pi times its exact integral over the overlap
inline void field_draine(int B, const double* lo, const double* hi,
                         double* phi) {
  auto prim = [](double E) {
    return E * E * (1.658e6 / 2.0 + E * (-2.152e5 / 3.0 + E * (6.919e3 / 4.0)));
  };
  for (int b = 0; b < B; ++b) {
    const double a = std::fmax(lo[b], 5.0), c = std::fmin(hi[b], 13.6);
    phi[b] = c > a ? kPi4 * (prim(c) - prim(a)) : 0.0;
  }
}

// a J21 power law J = J21 1e-21 erg s^-1 cm^-2 Hz^-1 sr^-1 (13.6 eV / E)^alpha
// (1e-21 erg taken as 6.2415e-10 eV), integrated exactly
inline void field_j21(int B, const double* lo, const double* hi, double J21,
                      double alpha, double* phi) {
  const double J0 = J21 * 6.2415e-10;
  for (int b = 0; b < B; ++b) {
    const double I = alpha == 0.0
        ? std::log(hi[b] / lo[b])
        : (std::pow(13.6 / lo[b], alpha) - std::pow(13.6 / hi[b], alpha)) / alpha;
    phi[b] = kPi4 / kbc::planck_eV * J0 * I;
  }
}

// int_{e0}^{e1} J d ln E of J interpolated between the nodes (E0, J0) and
// (E1, J1): linearly in E, or as a power law (log-log: 0 where a node is
// not positive), in closed form
inline double segment_dlnE(double e0, double e1, double E0, double J0,
                           double E1, double J1, bool loglog) {
  if (!(e1 > e0)) return 0.0;
  if (!loglog) {
    const double g = (J1 - J0) / (E1 - E0);
    return (J0 - g * E0) * std::log(e1 / e0) + g * (e1 - e0);
  }
  if (!(J0 > 0.0) || !(J1 > 0.0)) return 0.0;
  const double beta = std::log(J1 / J0) / std::log(E1 / E0);
  const double L = std::log(e1 / e0);
  const double base = J0 * std::pow(e0 / E0, beta);
  if (std::fabs(beta * L) < 1e-8) return base * L * (1.0 + 0.5 * beta * L);
  return base * std::expm1(beta * L) / beta;
}

// a tabulated J(E) at nE ascending energies, zero outside the table
inline void field_table(int B, const double* lo, const double* hi, int nE,
                        const double* E, const double* J, bool loglog,
                        double* phi) {
  for (int b = 0; b < B; ++b) {
    double s = 0.0;
    for (int i = 0; i + 1 < nE; ++i)
      s += segment_dlnE(std::fmax(lo[b], E[i]), std::fmin(hi[b], E[i + 1]),
                        E[i], J[i], E[i + 1], J[i + 1], loglog);
    phi[b] = kPi4 / kbc::planck_eV * s;
  }
}

// the bin-mean of a tabulated dust opacity kappa(E) [cm^2 g^-1] (E
// ascending): the trapezoid rule over the linear interpolant on each bin,
// with the table's nodes inside the bin as breakpoints; -1 when a bin
// leaves the table
inline int dust_opacity_bins(int nE, const double* E, const double* kap,
                             int B, const double* lo, const double* hi,
                             double* out) {
  auto at = [&](double x) {
    int i = 0;
    while (i < nE - 2 && E[i + 1] < x) ++i;
    return kap[i] + (x - E[i]) / (E[i + 1] - E[i]) * (kap[i + 1] - kap[i]);
  };
  for (int b = 0; b < B; ++b) {
    if (lo[b] < E[0] || hi[b] > E[nE - 1]) return -1;
    double s = 0.0, x0 = lo[b], k0 = at(x0);
    for (int i = 0; i < nE; ++i) {
      if (!(E[i] > lo[b] && E[i] < hi[b])) continue;
      s += 0.5 * (k0 + kap[i]) * (E[i] - x0);
      x0 = E[i];
      k0 = kap[i];
    }
    s += 0.5 * (k0 + at(hi[b])) * (hi[b] - x0);
    out[b] = s / (hi[b] - lo[b]);
  }
  return 0;
}

// G0 and Av of a field: the least-squares line through
// ln(Phi_b / Phi_Draine,b) = ln G0 - kappa_b d2g 1.8e21 m_p Av / xH over the
// bins where the Draine field is nonzero, with ln G0 held to [-7, 7] (Av
// refitted at the bound) and Av >= 0 (then ln G0 the mean, held to the
// same range); -1 with fewer than 2 such bins
inline int fit_G0_Av(int B, const double* lo, const double* hi,
                     const double* phi, const double* kap, double d2g,
                     double xH, double* G0, double* Av) {
  std::vector<double> dr(B);
  field_draine(B, lo, hi, dr.data());
  double sx = 0.0, sy = 0.0, sxx = 0.0, sxy = 0.0;
  int m = 0;
  std::vector<double> xs, ys;
  for (int b = 0; b < B; ++b) {
    if (!(dr[b] > 0.0)) continue;
    const double x = -kap[b] * 1.8e21 * kbc::p_mass * d2g / xH;
    const double y = std::log(phi[b] + 1e-200) - std::log(dr[b]);
    xs.push_back(x);
    ys.push_back(y);
    sx += x; sy += y; sxx += x * x; sxy += x * y;
    ++m;
  }
  if (m < 2) return -1;
  const double den = m * sxx - sx * sx;
  double slope = den != 0.0 ? (m * sxy - sx * sy) / den : 0.0;
  double lg = (sy - slope * sx) / m;
  if (lg < -7.0 || lg > 7.0) {
    lg = std::fmin(std::fmax(lg, -7.0), 7.0);
    double num = 0.0;
    for (int i = 0; i < m; ++i) num += (ys[i] - lg) * xs[i];
    slope = sxx > 0.0 ? num / sxx : 0.0;
  }
  if (slope < 0.0) {
    slope = 0.0;
    lg = std::fmin(std::fmax(sy / m, -7.0), 7.0);
  }
  *Av = slope;
  *G0 = std::exp(lg);
  return 0;
}

}  // namespace kbspec
