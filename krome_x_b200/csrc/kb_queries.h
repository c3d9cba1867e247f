// The rest of the reference's C interface (runtime/interfaces/C/krome.h):
// network metadata, the per-cell queries, the photon-field helpers and the
// option setters a caller of the reference's bindings reaches, so that the
// reference's own ctypes binding (runtime/interfaces/python/krome.py) loads
// this library and finds every entry point it prototypes.
//
// The queries are diagnostics, evaluated on the host with the network
// header's scalar (KB_HD) functions: rates at the rate temperature
// clamp(Tgas, Tcmb, 1e9), thermal terms at the thermal temperature
// clamp(Tgas, 2.73, 1e9), as the solve's right-hand side does
// (reference runtime/core/query.hpp). What this library does not build --
// binned dust and per-coolant line data -- answers as the reference does
// when it is not configured (-1, 0 or NULL), and the setters that would
// configure it return -104. Included by krome_b200.cu after krome_opts.
#pragma once

#include "kb_spectra.h"

namespace {

// f(c, n_c, Tgas_c, params_c) for every cell with the solve's parameter
// conventions (rows, or one row with stride 0, or NULL for the defaults);
// returns -1 for bad arguments, else the first nonzero flag of f
template <class F>
int for_each_cell(int ncell, const double* n, const double* Tgas,
                  const double* par, int par_stride, F f) {
  if (ncell < 0 || n == nullptr) return -1;
  if (par != nullptr && par_stride != 0 && par_stride != kbnet::NPAR) return -1;
  double dflt[kbnet::NPAR > 0 ? kbnet::NPAR : 1];
  for (int i = 0; i < kbnet::NPAR; ++i) dflt[i] = kbnet::param_default(i);
  int first = 0;
  for (int c = 0; c < ncell; ++c) {
    kbnet::Params P;
    kbnet::params_from_row(par != nullptr ? par + (size_t)c * par_stride : dflt, P);
    const int fl = f(c, n + (size_t)c * kbnet::NSPEC,
                     Tgas != nullptr ? Tgas[c] : 0.0, P);
    if (fl != 0 && first == 0) first = fl;
  }
  return first;
}

inline double rate_T(double Tgas, const kbnet::Params& P) {
  return std::fmin(std::fmax(Tgas, P.Tcmb), 1e9);
}
inline double thermal_T(double Tgas) {
  return std::fmin(std::fmax(Tgas, 2.73), 1e9);
}

// the rate coefficients of a cell as the solve sees them (no photon field)
inline void cell_rates(const double* n, double T, const kbnet::Params& P,
                       double* k) {
  for (int r = 0; r <= kbnet::NREA; ++r) k[r] = 0.0;
  kbnet::rates_fixed(T, n, P, k);
  kbnet::rates_var(T, n, P, k);
}

inline double cell_rho(const double* n) { return kbnet::rho_(n); }
inline double cell_ntot(const double* n) { return kbnet::ntot_(n); }
inline double cell_mu(const double* n) {
  return std::fmax(kbnet::rho_(n), 1e-40)
      / (std::fmax(kbnet::ntot_(n), 1e-40) * kbc::p_mass);
}
inline double cell_charge(const double* n) {
  double q = 0.0;
  for (int i = 0; i < kbnet::NSPEC; ++i) q += kbnet::species_charge(i) * n[i];
  return q;
}
// the electron density that makes the cell neutral: the charge of every
// species but the electrons, floored at 0
inline double cell_electrons(const double* n) {
  double q = cell_charge(n);
  if (kbnet::IDX_ELECTRON >= 0) q += n[kbnet::IDX_ELECTRON];
  return std::fmax(q, 0.0);
}
inline double freefall_rho(double rho) {
  return std::sqrt(3.0 * kbc::pi / (32.0 * kbc::gravity * std::fmax(rho, 1e-40)));
}

template <double (*G)(const double*)>
int cellwise(int ncell, const double* n, double* out) {
  if (ncell < 0 || n == nullptr || out == nullptr) return -1;
  for (int c = 0; c < ncell; ++c) out[c] = G(n + (size_t)c * kbnet::NSPEC);
  return 0;
}
// a cell's photo rates from its field row, on the host (the queries)
template <class P>
void host_photo_rates(P& p, const krome_opts* h, const double* Phi, int c) {
  if constexpr (kbnet::NPHOTO > 0) {
    if (h == nullptr || h->photo.B <= 0 || Phi == nullptr) return;
    kbphoto::rates_of_field(h->photo.sigma.data(), h->photo.B,
                            Phi + (size_t)c * h->photo.B, p.kph);
  } else {
    (void)p; (void)h; (void)Phi; (void)c;
  }
}
inline double cell_hnuclei(const double* n) { return kbnet::Hnuclei_(n); }
inline double cell_freefall(const double* n) { return freefall_rho(kbnet::rho_(n)); }

}  // namespace

// ---- metadata (reference krome.h:114-121, 580-652) ----

KB_API const char* krome_reaction_name(int r) {
  return (r >= 0 && r < kbnet::NREA) ? kbnet::reaction_names[r] : nullptr;
}
KB_API int krome_nheat(void) { return kbnet::NHEAT; }
KB_API int krome_ncool(void) { return kbnet::NCOOL; }
KB_API const char* krome_heating_name(int i) {
  return (i >= 0 && i < kbnet::NHEAT) ? kbnet::heat_names[i] : nullptr;
}
KB_API const char* krome_cooling_name(int i) {
  return (i >= 0 && i < kbnet::NCOOL) ? kbnet::cool_names[i] : nullptr;
}
// line coolants of coolant files (thermal.coolant_files): none here
KB_API int krome_ncoolant(void) { return 0; }
KB_API const char* krome_coolant_name(int) { return nullptr; }
KB_API int krome_coolant_species(int) { return -1; }
KB_API int krome_coolant_nlev(int) { return -1; }
KB_API int krome_coolant_levels(int, double*, double*) { return -1; }

// ---- per-cell quantities of the densities (reference krome.h:520-560;
// query.hpp:120-195) ----

KB_API int krome_get_mu(int ncell, const double* n, double* out) {
  return cellwise<cell_mu>(ncell, n, out);
}
KB_API int krome_get_rho(int ncell, const double* n, double* out) {
  return cellwise<cell_rho>(ncell, n, out);
}
KB_API int krome_get_ntot(int ncell, const double* n, double* out) {
  return cellwise<cell_ntot>(ncell, n, out);
}
KB_API int krome_get_Hnuclei(int ncell, const double* n, double* out) {
  return cellwise<cell_hnuclei>(ncell, n, out);
}
KB_API int krome_get_charge(int ncell, const double* n, double* out) {
  return cellwise<cell_charge>(ncell, n, out);
}
KB_API int krome_get_electrons(int ncell, const double* n, double* out) {
  return cellwise<cell_electrons>(ncell, n, out);
}
KB_API int krome_get_free_fall_time(int ncell, const double* n, double* out) {
  return cellwise<cell_freefall>(ncell, n, out);
}
KB_API int krome_get_free_fall_time_rho(int ncell, const double* rho,
                                        double* out) {
  if (ncell < 0 || rho == nullptr || out == nullptr) return -1;
  for (int c = 0; c < ncell; ++c) out[c] = freefall_rho(rho[c]);
  return 0;
}
// sqrt(pi kB T / (G rho mu m_p)) [cm]
KB_API int krome_get_jeans_length(int ncell, const double* n,
                                  const double* Tgas, double* out) {
  if (ncell < 0 || n == nullptr || Tgas == nullptr || out == nullptr) return -1;
  for (int c = 0; c < ncell; ++c) {
    const double* nc = n + (size_t)c * kbnet::NSPEC;
    const double rr = std::fmax(kbnet::rho_(nc), 1e-40);
    out[c] = std::sqrt(kbc::pi * kbc::boltzmann_erg * Tgas[c]
                       / (kbc::gravity * rr * cell_mu(nc) * kbc::p_mass));
  }
  return 0;
}
// the neutral atomic metals at a metallicity Z = log10(Z / Z_sun)
KB_API int krome_scale_Z(int ncell, double* n, double Z) {
  if (ncell < 0 || n == nullptr) return -1;
  for (int c = 0; c < ncell; ++c) kbnet::scale_Z(n + (size_t)c * kbnet::NSPEC, Z);
  return 0;
}
// the column density [cm^-2] the network's estimator gives num [cm^-3]
KB_API int krome_num2col(int ncell, const double* num, const double* n,
                         const double* Tgas, const double* par,
                         int par_stride, double* out) {
  if (num == nullptr || Tgas == nullptr || out == nullptr) return -1;
  return for_each_cell(ncell, n, Tgas, par, par_stride,
                       [&](int c, const double*, double, const kbnet::Params&) {
                         out[c] = kbnet::num2col_(num[c]);
                         return 0;
                       });
}

// ---- queries at (n, Tgas, par) (reference krome.h:387-470) ----

// the adiabatic index at the thermal temperature
KB_API int krome_get_gamma(int ncell, const double* n, const double* Tgas,
                           const double* par, int par_stride, double* gamma) {
  if (Tgas == nullptr || gamma == nullptr) return -1;
  return for_each_cell(
      ncell, n, Tgas, par, par_stride,
      [&](int c, const double* nc, double T, const kbnet::Params& P) {
        if (kbnet::params_missing(P) >= 0) return -105;
        gamma[c] = kbnet::gamma_index(thermal_T(T), nc, P);
        return 0;
      });
}

// reaction fluxes k prod(n) [cm^-3 s^-1], fl[ncell][nrea]
KB_API int krome_get_fluxes(int ncell, const double* n, const double* Tgas,
                            const double* par, int par_stride,
                            const double* Phi, const krome_opts* h,
                            double* fl) {
  if (Tgas == nullptr || fl == nullptr) return -1;
  if (h != nullptr && h->photo.B > 0 && Phi == nullptr) return -103;
  return for_each_cell(
      ncell, n, Tgas, par, par_stride,
      [&](int c, const double* nc, double T, const kbnet::Params& P) {
        if (kbnet::params_missing(P) >= 0) return -105;
        kbnet::Params Q = P;
        host_photo_rates(Q, h, Phi, c);
        double k[kbnet::NREA + 1];
        cell_rates(nc, rate_T(T, Q), Q, k);
        kbnet::reaction_fluxes(nc, k, fl + (size_t)c * kbnet::NREA);
        return 0;
      });
}

// the thermal balance: totals, the active terms (heats[ncell][nheat],
// cools[ncell][ncool], each may be NULL) and dTgas/dt [K s^-1]
KB_API int krome_get_thermal(int ncell, const double* n, const double* Tgas,
                             const double* par, int par_stride,
                             const double* Phi, const krome_opts* h,
                             double* heat, double* cool, double* heats,
                             double* cools, double* dTdt) {
  if (Tgas == nullptr) return -1;
  if (h != nullptr && h->photo.B > 0 && Phi == nullptr) return -103;
  return for_each_cell(
      ncell, n, Tgas, par, par_stride,
      [&](int c, const double* nc, double T, const kbnet::Params& P) {
        if (kbnet::params_missing(P) >= 0) return -105;
        kbnet::Params Q = P;
        host_photo_rates(Q, h, Phi, c);
        double k[kbnet::NREA + 1];
        cell_rates(nc, rate_T(T, Q), Q, k);
        const double Tth = thermal_T(T);
        double H[kbnet::NHEAT > 0 ? kbnet::NHEAT : 1];
        double C[kbnet::NCOOL > 0 ? kbnet::NCOOL : 1];
        kbnet::thermal_terms(Tth, nc, k, P, H, C);
        double hs = 0.0, cs = 0.0;
        for (int i = 0; i < kbnet::NHEAT; ++i) {
          hs += H[i];
          if (heats != nullptr) heats[(size_t)c * kbnet::NHEAT + i] = H[i];
        }
        for (int i = 0; i < kbnet::NCOOL; ++i) {
          cs += C[i];
          if (cools != nullptr) cools[(size_t)c * kbnet::NCOOL + i] = C[i];
        }
        if (heat != nullptr) heat[c] = hs;
        if (cool != nullptr) cool[c] = cs;
        if (dTdt != nullptr)
          dTdt[c] = (kbnet::gamma_index(Tth, nc, P) - 1.0) * (hs - cs)
              / (kbc::boltzmann_erg * kbnet::ntot_(nc));
        return 0;
      });
}

// the dust temperature the rates see: the Tdust parameter where the
// network has one, else -1
KB_API int krome_get_Tdust(int ncell, const double* n, const double* Tgas,
                           const double* par, int par_stride,
                           const double* Phi, const krome_opts* h,
                           double* Td) {
  (void)Phi; (void)h;
  if (Tgas == nullptr || Td == nullptr) return -1;
  int it = -1;
  for (int i = 0; i < kbnet::NPAR; ++i)
    if (!std::strcmp(kbnet::param_names[i], "Tdust")) it = i;
  if (it < 0) return -1;
  return for_each_cell(
      ncell, n, Tgas, par, par_stride,
      [&](int c, const double*, double, const kbnet::Params& P) {
        if (kbnet::params_missing(P) >= 0) return -105;
        const double* row = reinterpret_cast<const double*>(&P);
        Td[c] = row[it];
        return 0;
      });
}

// the energy released per reaction event [MeV]: no reaction of these
// networks carries one
KB_API int krome_get_qeff(int ncell, const double* n, const double* Tgas,
                          const double* par, int par_stride, double* q) {
  if (Tgas == nullptr || q == nullptr) return -1;
  return for_each_cell(
      ncell, n, Tgas, par, par_stride,
      [&](int c, const double*, double, const kbnet::Params& P) {
        if (kbnet::params_missing(P) >= 0) return -105;
        for (int r = 0; r < kbnet::NREA; ++r) q[(size_t)c * kbnet::NREA + r] = 0.0;
        return 0;
      });
}

KB_API int krome_get_coolant_cooling(int ncell, const double* n,
                                     const double* Tgas, const double* par,
                                     int par_stride, const double* Phi,
                                     const krome_opts* h, double* cool) {
  (void)Phi; (void)h;
  if (Tgas == nullptr || cool == nullptr) return -1;
  return for_each_cell(ncell, n, Tgas, par, par_stride,
                       [&](int, const double*, double, const kbnet::Params& P) {
                         return kbnet::params_missing(P) >= 0 ? -105 : 0;
                       });
}
KB_API int krome_get_coolant_populations(int, const double*, const double*,
                                         const double*, int, const double*,
                                         const krome_opts*, int, double*) {
  return -1;  // no coolant
}

// ---- photon-field helpers (reference krome.h:560-640) ----

KB_API int krome_bins_lin(int nbins, double lower, double upper, double* Elo,
                          double* Ehi) {
  if (nbins <= 0 || !(upper > lower) || !(lower > 0.0) || !Elo || !Ehi) return -1;
  kbspec::bins_linear(nbins, lower, upper, Elo, Ehi);
  return 0;
}
KB_API int krome_bins_log(int nbins, double lower, double upper, double* Elo,
                          double* Ehi) {
  if (nbins <= 0 || !(upper > lower) || !(lower > 0.0) || !Elo || !Ehi) return -1;
  kbspec::bins_logarithmic(nbins, lower, upper, Elo, Ehi);
  return 0;
}
KB_API int krome_J_to_phi(int nbins, const double* Elo, const double* Ehi,
                          const double* J, double* phi) {
  if (!kbspec::bins_valid(nbins, Elo, Ehi) || !J || !phi) return -1;
  for (int b = 0; b < nbins; ++b)
    phi[b] = kbspec::flux_of_intensity(J[b], Elo[b], Ehi[b]);
  return 0;
}
KB_API int krome_phi_to_J(int nbins, const double* Elo, const double* Ehi,
                          const double* phi, double* J) {
  if (!kbspec::bins_valid(nbins, Elo, Ehi) || !J || !phi) return -1;
  for (int b = 0; b < nbins; ++b)
    J[b] = kbspec::intensity_of_flux(phi[b], Elo[b], Ehi[b]);
  return 0;
}
KB_API int krome_spectrum_blackbody(int nbins, const double* Elo,
                                    const double* Ehi, double Tbb,
                                    double* phi) {
  if (!kbspec::bins_valid(nbins, Elo, Ehi) || !(Tbb > 0.0) || !phi) return -1;
  kbspec::field_blackbody(nbins, Elo, Ehi, Tbb, phi);
  return 0;
}
KB_API int krome_blackbody_range(double Tbb, double* lower, double* upper) {
  if (!(Tbb > 0.0) || !lower || !upper) return -1;
  return kbspec::blackbody_limits(Tbb, lower, upper);
}
KB_API int krome_spectrum_draine(int nbins, const double* Elo,
                                 const double* Ehi, double* phi) {
  if (!kbspec::bins_valid(nbins, Elo, Ehi) || !phi) return -1;
  kbspec::field_draine(nbins, Elo, Ehi, phi);
  return 0;
}
KB_API int krome_spectrum_j21(int nbins, const double* Elo, const double* Ehi,
                              double J21, double alpha, double* phi) {
  if (!kbspec::bins_valid(nbins, Elo, Ehi) || !phi) return -1;
  kbspec::field_j21(nbins, Elo, Ehi, J21, alpha, phi);
  return 0;
}
// the Haardt & Madau 2012 background needs its tabulated spectra, which
// this library does not carry
KB_API int krome_spectrum_hm2012(int nbins, const double* Elo,
                                 const double* Ehi, double, double* phi) {
  if (!kbspec::bins_valid(nbins, Elo, Ehi) || !phi) return -1;
  return -104;
}
KB_API int krome_spectrum_table(int nbins, const double* Elo,
                                const double* Ehi, int nE, const double* E,
                                const double* J, int loglog, double* phi) {
  if (!kbspec::bins_valid(nbins, Elo, Ehi) || nE < 2 || !E || !J || !phi)
    return -1;
  for (int i = 1; i < nE; ++i)
    if (!(E[i] > E[i - 1])) return -1;
  kbspec::field_table(nbins, Elo, Ehi, nE, E, J, loglog != 0, phi);
  return 0;
}
KB_API int krome_dust_kappa_bins(int nE, const double* E, const double* kappa,
                                 int nbins, const double* Elo,
                                 const double* Ehi, double* kbin) {
  if (!kbspec::bins_valid(nbins, Elo, Ehi) || nE < 2 || !E || !kappa || !kbin)
    return -1;
  for (int i = 1; i < nE; ++i)
    if (!(E[i] > E[i - 1])) return -1;
  return kbspec::dust_opacity_bins(nE, E, kappa, nbins, Elo, Ehi, kbin);
}
// the Draine R_V = 3.1 dust opacity needs its table, not carried here
KB_API int krome_dust_kappa_draine(int nbins, const double* Elo,
                                   const double* Ehi, double* kbin) {
  if (!kbspec::bins_valid(nbins, Elo, Ehi) || !kbin) return -1;
  return -104;
}
KB_API int krome_find_G0_Av(int nbins, const double* Elo, const double* Ehi,
                            const double* phi, const double* kbin, double d2g,
                            double xH, double* G0, double* Av) {
  if (!kbspec::bins_valid(nbins, Elo, Ehi) || !phi || !kbin || !G0 || !Av
      || !(d2g > 0.0) || !(xH > 0.0))
    return -1;
  return kbspec::fit_G0_Av(nbins, Elo, Ehi, phi, kbin, d2g, xH, G0, Av);
}

// ---- the photo reactions (reference krome.h:600-640) ----

KB_API int krome_nphoto(void) { return kbnet::NPHOTO; }
KB_API int krome_photo_reaction(int r) {
  return (r >= 0 && r < kbnet::NPHOTO) ? kbnet::photo_reaction_[r] : -1;
}
KB_API int krome_photo_reactant(int r) {
  return (r >= 0 && r < kbnet::NPHOTO) ? kbnet::photo_reactant_[r] : -1;
}
KB_API double krome_photo_pdiss(int r) {
  return (r >= 0 && r < kbnet::NPHOTO) ? kbnet::photo_pdiss_[r] : std::nan("");
}
// J_LW rates: none in these networks
KB_API int krome_nlw(void) { return kbnet::NLW; }
KB_API int krome_lw_reaction(int) { return -1; }
KB_API int krome_lw_reactant(int) { return -1; }
KB_API double krome_lw_pdiss(int) { return std::nan(""); }

// ---- binned dust (krome.h:230-256): not built in this library ----

KB_API int krome_opts_set_dustbins(krome_opts* h, int nd, int use_Si,
                                   int use_C, double alow, double aup,
                                   double phi) {
  (void)phi;
  if (h == nullptr || nd <= 0 || !(use_Si || use_C) || !(aup > alow)) return -1;
  return -104;
}
KB_API int krome_opts_ndust(const krome_opts*) { return 0; }
KB_API int krome_opts_set_dust_Td(krome_opts*, const double*) { return -1; }
KB_API int krome_opts_get_dust_Td(const krome_opts*, double*) { return -1; }
KB_API int krome_opts_set_dust_a(krome_opts*, const double*) { return -1; }
KB_API int krome_opts_get_dust_a(const krome_opts*, double*) { return -1; }
KB_API int krome_opts_get_dust_counts(const krome_opts*, double, double,
                                      double*) {
  return -1;
}
KB_API int krome_opts_get_dust_types(const krome_opts*, int*) { return -1; }

// the error-report file (the error_report key): the name is kept; this
// library writes no report (a failed cell's flag is the report)
KB_API int krome_opts_set_error_file(krome_opts* h, const char* path) {
  if (h == nullptr || path == nullptr) return -1;
  h->error_file = path;
  return 0;
}

// ---- photon bins (krome.h:203-228, 600-640) ----

namespace {
int rebuild_photo(krome_opts* h) {
  if (h->photo.B <= 0) return 0;  // applied when the bins are set
  const std::vector<double> lo = h->photo.lo, hi = h->photo.hi;
  return kbphoto::build(h->photo, (int)lo.size(), lo.data(), hi.data(),
                        h->photo_alpha, h->broad_T, h->broad_vturb) ? 0 : -1;
}
}  // namespace

// nbins bins [Elo, Ehi] [eV]: the cross sections averaged over them; a
// solve then needs each cell's field (krome_cells Phi, -103 without)
KB_API int krome_opts_set_photo(krome_opts* h, int nbins, const double* Elo,
                                const double* Ehi) {
  if (h == nullptr || !kbspec::bins_valid(nbins, Elo, Ehi)) return -1;
  return kbphoto::build(h->photo, nbins, Elo, Ehi, h->photo_alpha, h->broad_T,
                        h->broad_vturb) ? 0 : -1;
}
KB_API int krome_opts_nbins(const krome_opts* h) {
  return h != nullptr ? h->photo.B : 0;
}
// Doppler broadening of the tabulated cross sections (Tgas [K], vturb
// [cm/s]); rebuilds the bins already set
KB_API int krome_opts_set_photo_broadening(krome_opts* h, double Tgas,
                                           double vturb) {
  if (h == nullptr || !(Tgas >= 0.0) || !(vturb >= 0.0)) return -1;
  h->broad_T = Tgas;
  h->broad_vturb = vturb;
  return rebuild_photo(h);
}
// the in-bin spectrum dN/dE ~ E^-alpha; rebuilds the bins already set
KB_API int krome_opts_set_photo_alpha(krome_opts* h, double alpha) {
  if (h == nullptr || !std::isfinite(alpha)) return -1;
  h->photo_alpha = alpha;
  return rebuild_photo(h);
}
// the dust opacity per bin [cm^2 per g of dust] (NULL: none), the dust
// term of krome_get_absorption
KB_API int krome_opts_set_photo_dust_opacity(krome_opts* h,
                                             const double* kappa) {
  if (h == nullptr || h->photo.B <= 0) return -1;
  if (kappa == nullptr) {
    h->photo.kdust.clear();
    return 0;
  }
  for (int b = 0; b < h->photo.B; ++b)
    if (!(kappa[b] >= 0.0)) return -1;
  h->photo.kdust.assign(kappa, kappa + h->photo.B);
  return 0;
}
// J_LW = sum_b w_b Phi_b
KB_API int krome_opts_lw_weights(const krome_opts* h, double* w) {
  if (h == nullptr || h->photo.B <= 0 || w == nullptr) return -1;
  for (int b = 0; b < h->photo.B; ++b) w[b] = h->photo.lww[b];
  return 0;
}
// the bin-averaged cross sections sigma[nphoto][nbins] [cm^2]
KB_API int krome_opts_photo_sigma(const krome_opts* h, double* sigma) {
  if (h == nullptr || h->photo.B <= 0 || sigma == nullptr) return -1;
  for (size_t i = 0; i < h->photo.sigma.size(); ++i) sigma[i] = h->photo.sigma[i];
  return 0;
}
// the cross section of photo reaction r at E [eV] (0 outside its range)
KB_API double krome_photo_xsec(int r, double E) {
  if (r < 0 || r >= kbnet::NPHOTO) return std::nan("");
  if (kbnet::kbxs::photo_xsec[r] == nullptr) return std::nan("");
  return (E >= kbnet::photo_Emin_[r] && E <= kbnet::photo_Emax_[r])
      ? kbnet::kbxs::photo_xsec[r](E) : 0.0;
}
// the Habing flux G of each cell's field (6-13.6 eV over 1.6e-3 erg
// cm^-2 s^-1), and its ratio to the Draine field (the photon flux summed
// over the bins as h / (4 pi) sum Phi_b over 7.95e-8)
KB_API int krome_get_habing(int ncell, const double* Phi, const krome_opts* h,
                            double* G) {
  if (ncell < 0 || h == nullptr || h->photo.B <= 0 || !Phi || !G) return -1;
  const int B = h->photo.B;
  for (int c = 0; c < ncell; ++c) {
    double g = 0.0;
    for (int b = 0; b < B; ++b) g += h->photo.habw[b] * Phi[(size_t)c * B + b];
    G[c] = g;
  }
  return 0;
}
KB_API int krome_get_ratio_flux_draine(int ncell, const double* Phi,
                                       const krome_opts* h, double* ratio) {
  if (ncell < 0 || Phi == nullptr || ratio == nullptr || h == nullptr
      || h->photo.B <= 0)
    return -1;
  const int B = h->photo.B;
  for (int c = 0; c < ncell; ++c) {
    double s = 0.0;
    for (int b = 0; b < B; ++b) s += Phi[(size_t)c * B + b];
    ratio[c] = s * kbc::planck_eV / (4.0 * kbc::pi) / 7.95e-8;
  }
  return 0;
}
// the photoheating of each photo reaction [erg cm^-3 s^-1],
// heat[ncell][nphoto]: its photoelectrons' deposit (0 for the Solomon
// process)
KB_API int krome_get_photo_heating(int ncell, const double* n,
                                   const double* Tgas, const double* par,
                                   int par_stride, const double* Phi,
                                   const krome_opts* h, double* heat) {
  if (Tgas == nullptr || heat == nullptr || h == nullptr || h->photo.B <= 0)
    return -1;
  if (Phi == nullptr) return -103;
  const int B = h->photo.B;
  return for_each_cell(
      ncell, n, Tgas, par, par_stride,
      [&](int c, const double* nc, double, const kbnet::Params& P) {
        if (kbnet::params_missing(P) >= 0) return -105;
        for (int r = 0; r < kbnet::NPHOTO; ++r) {
          double& o = heat[(size_t)c * kbnet::NPHOTO + r];
          o = 0.0;
          if (!kbnet::photo_deposit_[r]) continue;
          double se = 0.0;
          for (int b = 0; b < B; ++b)
            se += h->photo.sigmaE[(size_t)r * B + b] * Phi[(size_t)c * B + b];
          o = se * nc[kbnet::photo_reactant_[r]] * kbc::eV_to_erg;
        }
        return 0;
      });
}

namespace {
// the d2g parameter of a cell, or 0 where the network has none
double cell_d2g(const kbnet::Params& P) {
  for (int i = 0; i < kbnet::NPAR; ++i)
    if (!std::strcmp(kbnet::param_names[i], "d2g"))
      return reinterpret_cast<const double*>(&P)[i];
  return 0.0;
}
bool has_d2g() {
  for (int i = 0; i < kbnet::NPAR; ++i)
    if (!std::strcmp(kbnet::param_names[i], "d2g")) return true;
  return false;
}
}  // namespace

// the photon removal per bin [cm^-1], kabs[ncell][nbins]: the photo
// reactions' sigma_rb n_r / pdiss_r, the handle's dust opacity times the
// dust mass density (the d2g parameter), and rho_gas kdust_b when given
KB_API int krome_get_absorption(int ncell, const double* n, const double* Tgas,
                                const double* par, int par_stride,
                                const krome_opts* h, const double* kdust,
                                double* kabs) {
  if (Tgas == nullptr || kabs == nullptr || h == nullptr || h->photo.B <= 0)
    return -1;
  const int B = h->photo.B;
  return for_each_cell(
      ncell, n, Tgas, par, par_stride,
      [&](int c, const double* nc, double, const kbnet::Params& P) {
        if (kbnet::params_missing(P) >= 0) return -105;
        double* kc = kabs + (size_t)c * B;
        for (int b = 0; b < B; ++b) kc[b] = 0.0;
        for (int r = 0; r < kbnet::NPHOTO; ++r) {
          const double f = nc[kbnet::photo_reactant_[r]] * 1.0 / kbnet::photo_pdiss_[r];
          for (int b = 0; b < B; ++b) kc[b] += h->photo.sigma[(size_t)r * B + b] * f;
        }
        if (has_d2g() && !h->photo.kdust.empty())
          for (int b = 0; b < B; ++b)
            kc[b] += kbnet::rho_(nc) * cell_d2g(P) * h->photo.kdust[b];
        if (kdust != nullptr) {
          const double rr = kbnet::rho_(nc);
          for (int b = 0; b < B; ++b) kc[b] += rr * kdust[b];
        }
        return 0;
      });
}
// the optical depth per bin with the column estimates, tau[ncell][nbins]:
// sigma_rb N_r / pdiss_r (N_r the column of the reactant's density) and,
// with d2g[ncell], kdust_b d2g Sigma_gas (Sigma_gas = N_H rho / n_H); the
// reference's default dust opacity (the Draine table) is not carried here:
// d2g without kdust returns -1
KB_API int krome_get_opacity(int ncell, const double* n, const double* Tgas,
                             const double* par, int par_stride,
                             const krome_opts* h, const double* d2g,
                             const double* kdust, double* tau) {
  if (Tgas == nullptr || tau == nullptr || h == nullptr || h->photo.B <= 0)
    return -1;
  if (d2g != nullptr && kdust == nullptr) return -1;
  const int B = h->photo.B;
  return for_each_cell(
      ncell, n, Tgas, par, par_stride,
      [&](int c, const double* nc, double, const kbnet::Params& P) {
        if (kbnet::params_missing(P) >= 0) return -105;
        double* tc = tau + (size_t)c * B;
        for (int b = 0; b < B; ++b) tc[b] = 0.0;
        for (int r = 0; r < kbnet::NPHOTO; ++r) {
          const double Ncol = kbnet::num2col_(nc[kbnet::photo_reactant_[r]]);
          const double I = 1.0 * Ncol;
          for (int b = 0; b < B; ++b)
            tc[b] += h->photo.sigma[(size_t)r * B + b] * I / kbnet::photo_pdiss_[r];
        }
        const double dg = d2g != nullptr ? d2g[c] : 0.0;
        if (dg > 0.0) {
          const double nH = kbnet::Hnuclei_(nc);
          const double Sg = nH > 0.0 ? kbnet::NH_col_(nc) * kbnet::rho_(nc) / nH : 0.0;
          for (int b = 0; b < B; ++b) tc[b] += kdust[b] * dg * Sg;
        }
        return 0;
      });
}

// (the equilibrium driver, krome_equilibrium_cells, is in krome_b200.cu:
// it runs the device solve)
