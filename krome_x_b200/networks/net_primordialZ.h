// Generated by krome_x_b200.emit from the network 'primordialZ' -- do not edit.
// One host/device (KB_HD) scalar form of the network: species,
// parameters, rate coefficients, mass-action rhs, stoichiometric
// Jacobian and the thermal equation (see krome_x_b200/emit/
// emitter.py for the layout and the reference rules it follows).
#pragma once
#include "../csrc/kb_common.h"

namespace kbnet {

constexpr const char* NETWORK_NAME = "primordialZ";
constexpr const char* NETWORK_KEY = "primordialZ";
constexpr int NSPEC = 27;
constexpr int NREA = 74;
constexpr int KB_RATE_NDEP = 43;
#define KB_NFREEZE 0
constexpr int IDX_C = 0;
constexpr int IDX_Cj = 1;
constexpr int IDX_CH = 2;
constexpr int IDX_CH2 = 3;
constexpr int IDX_CH3 = 4;
constexpr int IDX_CH4 = 5;
constexpr int IDX_CO = 6;
constexpr int IDX_COj = 7;
constexpr int IDX_CO2 = 8;
constexpr int IDX_H = 9;
constexpr int IDX_Hj = 10;
constexpr int IDX_Hk = 11;
constexpr int IDX_H2 = 12;
constexpr int IDX_H2j = 13;
constexpr int IDX_H2O = 14;
constexpr int IDX_H2Oj = 15;
constexpr int IDX_H3Oj = 16;
constexpr int IDX_He = 17;
constexpr int IDX_Hej = 18;
constexpr int IDX_Hejj = 19;
constexpr int IDX_O = 20;
constexpr int IDX_Oj = 21;
constexpr int IDX_O2 = 22;
constexpr int IDX_O2j = 23;
constexpr int IDX_OH = 24;
constexpr int IDX_OHj = 25;
constexpr int IDX_E = 26;
#define KB_HAS_C 1
#define KB_HAS_Cj 1
#define KB_HAS_CH 1
#define KB_HAS_CH2 1
#define KB_HAS_CH3 1
#define KB_HAS_CH4 1
#define KB_HAS_CO 1
#define KB_HAS_COj 1
#define KB_HAS_CO2 1
#define KB_HAS_H 1
#define KB_HAS_Hj 1
#define KB_HAS_Hk 1
#define KB_HAS_H2 1
#define KB_HAS_H2j 1
#define KB_HAS_H2O 1
#define KB_HAS_H2Oj 1
#define KB_HAS_H3Oj 1
#define KB_HAS_He 1
#define KB_HAS_Hej 1
#define KB_HAS_Hejj 1
#define KB_HAS_O 1
#define KB_HAS_Oj 1
#define KB_HAS_O2 1
#define KB_HAS_O2j 1
#define KB_HAS_OH 1
#define KB_HAS_OHj 1
#define KB_HAS_E 1
#define KB_EXTERN_dissH2_Martin96 1
constexpr int IDX_ELECTRON = 26;

inline const char* const species_names[NSPEC] = {"C", "C+", "CH", "CH2", "CH3", "CH4", "CO", "CO+", "CO2", "H", "H+", "H-", "H2", "H2+", "H2O", "H2O+", "H3O+", "He", "He+", "He++", "O", "O+", "O2", "O2+", "OH", "OH+", "e-"};
constexpr int NELEM = 4;
inline const char* const element_names[4] = {"C", "H", "He", "O"};
KB_HD inline double species_mass_g(int i) {
  constexpr double t_[NSPEC] = {1.99447347289326e-23, 1.9943823790562555e-23, 2.1618558108065398e-23, 2.32923814871982e-23, 2.4966204866331e-23, 2.6640028245463796e-23, 4.6511699255465995e-23, 4.651078831709595e-23, 7.30786637819994e-23, 1.6738233791328e-24, 1.6729124407627538e-24, 1.6747343175028463e-24, 3.3476467582656e-24, 3.346735819895553e-24, 2.9914611284799e-23, 2.9913700346428956e-23, 3.1587523725561754e-23, 6.64647366797316e-24, 6.645562729603113e-24, 6.644651791233067e-24, 2.65669645265334e-23, 2.6566053588163353e-23, 5.31339290530668e-23, 5.313301811469676e-23, 2.82407879056662e-23, 2.823987696729615e-23, 9.10938370046373e-28};
  return t_[i];
}
KB_HD inline int species_charge(int i) {
  constexpr int t_[NSPEC] = {0, 1, 0, 0, 0, 0, 0, 1, 0, 0, 1, -1, 0, 1, 0, 1, 1, 0, 1, 2, 0, 1, 0, 1, 0, 1, -1};
  return t_[i];
}
KB_HD inline double species_natoms_H(int i) {
  constexpr double t_[NSPEC] = {0.0, 0.0, 1.0, 2.0, 3.0, 4.0, 0.0, 0.0, 0.0, 1.0, 1.0, 1.0, 2.0, 2.0, 2.0, 2.0, 3.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 1.0, 1.0, 0.0};
  return t_[i];
}
KB_HD inline int species_opaque(int i) {
  constexpr int t_[NSPEC] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  return t_[i];
}
inline constexpr int species_elements_t_[108] = {1, 0, 0, 0, 1, 0, 0, 0, 1, 1, 0, 0, 1, 2, 0, 0, 1, 3, 0, 0, 1, 4, 0, 0, 1, 0, 0, 1, 1, 0, 0, 1, 1, 0, 0, 2, 0, 1, 0, 0, 0, 1, 0, 0, 0, 1, 0, 0, 0, 2, 0, 0, 0, 2, 0, 0, 0, 2, 0, 1, 0, 2, 0, 1, 0, 3, 0, 1, 0, 0, 1, 0, 0, 0, 1, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 1, 0, 0, 0, 2, 0, 0, 0, 2, 0, 1, 0, 1, 0, 1, 0, 1, 0, 0, 0, 0};
#ifdef __CUDACC__
__device__ const int d_species_elements_[108] = {1, 0, 0, 0, 1, 0, 0, 0, 1, 1, 0, 0, 1, 2, 0, 0, 1, 3, 0, 0, 1, 4, 0, 0, 1, 0, 0, 1, 1, 0, 0, 1, 1, 0, 0, 2, 0, 1, 0, 0, 0, 1, 0, 0, 0, 1, 0, 0, 0, 2, 0, 0, 0, 2, 0, 0, 0, 2, 0, 1, 0, 2, 0, 1, 0, 3, 0, 1, 0, 0, 1, 0, 0, 0, 1, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 1, 0, 0, 0, 2, 0, 0, 0, 2, 0, 1, 0, 1, 0, 1, 0, 1, 0, 0, 0, 0};
#endif
KB_HD inline int species_element(int i, int e) {
#ifdef __CUDA_ARCH__
  return d_species_elements_[i * NELEM + e];
#else
  return species_elements_t_[i * NELEM + e];
#endif
}
KB_HD inline double ntot_(const double* n) {
  double s = 0.0;
KB_UNROLL
  for (int i = 0; i < NSPEC; ++i) s += n[i];
  return s;
}
KB_HD inline double Hnuclei_(const double* n) {
  double s = 0.0;
KB_UNROLL
  for (int i = 0; i < NSPEC; ++i) s += n[i] * species_natoms_H(i);
  return s;
}
KB_HD inline double rho_(const double* n) {
  double s = 0.0;
KB_UNROLL
  for (int i = 0; i < NSPEC; ++i) s += n[i] * species_mass_g(i);
  return s;
}

constexpr int NPAR = 2;
constexpr int NPHOTO = 0;
struct Params {
  double gamma_ad;
  double Tcmb;
};
inline const char* const param_names[NPAR] = {"gamma_ad", "Tcmb"};
// the defaults of a parameter row; NaN marks a REQUIRED parameter
inline double param_default(int i) {
  const double t_[NPAR] = {1.6666666666666667, 2.725};
  return t_[i];
}
inline const char* const param_required_by[NPAR] = {"", ""};
KB_HD inline void params_from_row(const double* row, Params& p) {
  p.gamma_ad = row[0];
  p.Tcmb = row[1];
}
KB_HD inline int params_missing(const Params& p) {
  (void)p;
  return -1;
}

#include "../csrc/kb_physics.h"
#include "../csrc/kb_conserve.h"
#include "../csrc/kb_jacdk.h"

KB_HD inline double v_Te(double Tgas, const double* n, const Params& p) {
  (void)Tgas; (void)n; (void)p;
  return Tgas*kbc::boltzmann_eV;
}
KB_HD inline double v_lnTe(double Tgas, const double* n, const Params& p) {
  (void)Tgas; (void)n; (void)p;
  return kb_log(Tgas*kbc::boltzmann_eV);
}
KB_HD inline double v_invTe(double Tgas, const double* n, const Params& p) {
  (void)Tgas; (void)n; (void)p;
  return 1.0 / (Tgas*kbc::boltzmann_eV);
}
KB_HD inline double v_invT(double Tgas, const double* n, const Params& p) {
  (void)Tgas; (void)n; (void)p;
  return 1.0 / Tgas;
}
KB_HD inline double v_T32(double Tgas, const double* n, const Params& p) {
  (void)Tgas; (void)n; (void)p;
  return Tgas / 300.0;
}
KB_HD inline double v_T(double Tgas, const double* n, const Params& p) {
  (void)Tgas; (void)n; (void)p;
  return Tgas;
}
KB_HD inline double v_a1(double Tgas, const double* n, const Params& p) {
  (void)Tgas; (void)n; (void)p;
  return 1.35e-09;
}
KB_HD inline double v_a2(double Tgas, const double* n, const Params& p) {
  (void)Tgas; (void)n; (void)p;
  return 0.098493;
}
KB_HD inline double v_a3(double Tgas, const double* n, const Params& p) {
  (void)Tgas; (void)n; (void)p;
  return 0.32852;
}
KB_HD inline double v_a4(double Tgas, const double* n, const Params& p) {
  (void)Tgas; (void)n; (void)p;
  return 0.5561;
}
KB_HD inline double v_a5(double Tgas, const double* n, const Params& p) {
  (void)Tgas; (void)n; (void)p;
  return 2.771e-07;
}
KB_HD inline double v_a6(double Tgas, const double* n, const Params& p) {
  (void)Tgas; (void)n; (void)p;
  return 2.1826;
}
KB_HD inline double v_a7(double Tgas, const double* n, const Params& p) {
  (void)Tgas; (void)n; (void)p;
  return 0.006191;
}
KB_HD inline double v_a8(double Tgas, const double* n, const Params& p) {
  (void)Tgas; (void)n; (void)p;
  return 1.0461;
}
KB_HD inline double v_a9(double Tgas, const double* n, const Params& p) {
  (void)Tgas; (void)n; (void)p;
  return 8.9712e-11;
}
KB_HD inline double v_a10(double Tgas, const double* n, const Params& p) {
  (void)Tgas; (void)n; (void)p;
  return 3.0424;
}
KB_HD inline double v_a11(double Tgas, const double* n, const Params& p) {
  (void)Tgas; (void)n; (void)p;
  return 3.2576e-14;
}
KB_HD inline double v_a12(double Tgas, const double* n, const Params& p) {
  (void)Tgas; (void)n; (void)p;
  return 3.7741;
}
KB_HD inline double v_asav(double Tgas, const double* n, const Params& p) {
  (void)Tgas; (void)n; (void)p;
  return 21237.15;
}
KB_HD inline double v_bsav1(double Tgas, const double* n, const Params& p) {
  (void)Tgas; (void)n; (void)p;
  return -3.3232183e-07;
}
KB_HD inline double v_bsav2(double Tgas, const double* n, const Params& p) {
  (void)Tgas; (void)n; (void)p;
  return 3.3735382e-07;
}
KB_HD inline double v_bsav3(double Tgas, const double* n, const Params& p) {
  (void)Tgas; (void)n; (void)p;
  return -1.4491368e-07;
}
KB_HD inline double v_bsav4(double Tgas, const double* n, const Params& p) {
  (void)Tgas; (void)n; (void)p;
  return 3.4172805e-08;
}
KB_HD inline double v_bsav5(double Tgas, const double* n, const Params& p) {
  (void)Tgas; (void)n; (void)p;
  return -4.7813728e-09;
}
KB_HD inline double v_bsav6(double Tgas, const double* n, const Params& p) {
  (void)Tgas; (void)n; (void)p;
  return 3.9731542e-10;
}
KB_HD inline double v_bsav7(double Tgas, const double* n, const Params& p) {
  (void)Tgas; (void)n; (void)p;
  return -1.8171411e-11;
}
KB_HD inline double v_bsav8(double Tgas, const double* n, const Params& p) {
  (void)Tgas; (void)n; (void)p;
  return 3.5311932e-13;
}
KB_HD inline double v_sumsav(double Tgas, const double* n, const Params& p) {
  (void)Tgas; (void)n; (void)p;
  return v_bsav1(Tgas, n, p) + v_bsav2(Tgas, n, p) * kb_log(Tgas) + v_bsav3(Tgas, n, p) * kb_log(Tgas)*kb_log(Tgas) + v_bsav4(Tgas, n, p) * kb_log(Tgas)*kb_log(Tgas)*kb_log(Tgas) + v_bsav5(Tgas, n, p) * kb_log(Tgas)*kb_log(Tgas)*kb_log(Tgas)*kb_log(Tgas) + v_bsav6(Tgas, n, p) * ipow_<5>(kb_log(Tgas)) + v_bsav7(Tgas, n, p) * ipow_<6>(kb_log(Tgas)) + v_bsav8(Tgas, n, p) * ipow_<7>(kb_log(Tgas));
}
KB_HD inline double v_kl21(double Tgas, const double* n, const Params& p) {
  (void)Tgas; (void)n; (void)p;
  return 1.18e-10 * kb_exp(-69500.0 * v_invT(Tgas, n, p));
}
KB_HD inline double v_kh21(double Tgas, const double* n, const Params& p) {
  (void)Tgas; (void)n; (void)p;
  return 8.125e-08 * 1.0/(std::sqrt(v_T(Tgas, n, p))) * kb_exp(-52000.0 * v_invT(Tgas, n, p)) * (1.0 - kb_exp(-6000.0 * v_invT(Tgas, n, p)));
}
KB_HD inline double v_ncr21(double Tgas, const double* n, const Params& p) {
  (void)Tgas; (void)n; (void)p;
  return kb_exp10(4.845 - 1.3 * kb_log10(v_T(Tgas, n, p) * 0.0001) + 1.62 * kb_log10(v_T(Tgas, n, p) * 0.0001)*kb_log10(v_T(Tgas, n, p) * 0.0001));
}
KB_HD inline double v_a21(double Tgas, const double* n, const Params& p) {
  (void)Tgas; (void)n; (void)p;
  return 1.0 / (1.0 + Hnuclei_(n) / v_ncr21(Tgas, n, p));
}

// rate coefficients of Tgas and the parameters only
KB_HD inline void rates_fixed(double Tgas, const double* n, const Params& p, double* k) {
  (void)Tgas; (void)n; (void)p; (void)k;
  const double vh_a1 = v_a1(Tgas, n, p);
  (void)vh_a1;
  const double vh_a10 = v_a10(Tgas, n, p);
  (void)vh_a10;
  const double vh_a11 = v_a11(Tgas, n, p);
  (void)vh_a11;
  const double vh_a12 = v_a12(Tgas, n, p);
  (void)vh_a12;
  const double vh_a2 = v_a2(Tgas, n, p);
  (void)vh_a2;
  const double vh_a3 = v_a3(Tgas, n, p);
  (void)vh_a3;
  const double vh_a4 = v_a4(Tgas, n, p);
  (void)vh_a4;
  const double vh_a5 = v_a5(Tgas, n, p);
  (void)vh_a5;
  const double vh_a6 = v_a6(Tgas, n, p);
  (void)vh_a6;
  const double vh_a7 = v_a7(Tgas, n, p);
  (void)vh_a7;
  const double vh_a8 = v_a8(Tgas, n, p);
  (void)vh_a8;
  const double vh_a9 = v_a9(Tgas, n, p);
  (void)vh_a9;
  const double vh_invT = v_invT(Tgas, n, p);
  (void)vh_invT;
  const double vh_lnTe = v_lnTe(Tgas, n, p);
  (void)vh_lnTe;
  k[0] = kb_exp(-32.71396786 + 13.536556 * vh_lnTe - 5.73932875 * vh_lnTe*vh_lnTe + 1.56315498 * vh_lnTe*vh_lnTe*vh_lnTe - 0.2877056 * vh_lnTe*vh_lnTe*vh_lnTe*vh_lnTe + 0.0348255977 * ipow_<5>(vh_lnTe) - 0.00263197617 * ipow_<6>(vh_lnTe) + 0.000111954395 * ipow_<7>(vh_lnTe) - 2.03914985e-06 * ipow_<8>(vh_lnTe));  // H + e- -> H+ + e- + e-
  k[3] = kb_exp(-44.09864886 + 23.91596563 * vh_lnTe - 10.7532302 * vh_lnTe*vh_lnTe + 3.05803875 * vh_lnTe*vh_lnTe*vh_lnTe - 0.56851189 * vh_lnTe*vh_lnTe*vh_lnTe*vh_lnTe + 0.0679539123 * ipow_<5>(vh_lnTe) - 0.0050090561 * ipow_<6>(vh_lnTe) + 0.000206723616 * ipow_<7>(vh_lnTe) - 3.64916141e-06 * ipow_<8>(vh_lnTe));  // He + e- -> He+ + e- + e-
  k[6] = kb_exp(-68.71040990212 + 43.93347632635 * vh_lnTe - 18.48066993568 * vh_lnTe*vh_lnTe + 4.701626486759002 * vh_lnTe*vh_lnTe*vh_lnTe - 0.7692466334492 * vh_lnTe*vh_lnTe*vh_lnTe*vh_lnTe + 0.08113042097303 * ipow_<5>(vh_lnTe) - 0.005324020628287001 * ipow_<6>(vh_lnTe) + 0.0001975705312221 * ipow_<7>(vh_lnTe) - 3.165581065665e-06 * ipow_<8>(vh_lnTe));  // He+ + e- -> He++ + e- + e-
  k[7] = 1.891e-10 / (std::sqrt(Tgas / 9.37) * kb_pow(1.0 + std::sqrt(Tgas / 9.37), 0.2476) * kb_pow(1.0 + std::sqrt(Tgas / 2774000.0), 1.7524));  // He++ + e- -> He+
  k[8] = 1.4e-18 * kb_pow(Tgas, 0.928) * kb_exp(-Tgas / 16200.0);  // H + e- -> H-
  k[9] = vh_a1 * (kb_pow(Tgas, vh_a2) + vh_a3 * kb_pow(Tgas, vh_a4) + vh_a5 * kb_pow(Tgas, vh_a6)) / (1.0 + vh_a7 * kb_pow(Tgas, vh_a8) + vh_a9 * kb_pow(Tgas, vh_a10) + vh_a11 * kb_pow(Tgas, vh_a12));  // H- + H -> H2 + e-
  k[12] = 6e-10;  // H2+ + H -> H2 + H+
  k[14] = 35.5 * kb_pow(Tgas, -2.28) * kb_exp(-46707.0 / Tgas);  // H2 + e- -> H + H-
  k[15] = 4.38e-10 * kb_exp(-102000.0 / Tgas) * kb_pow(Tgas, 0.35);  // H2 + e- -> H + H + e-
  k[17] = kb_exp(-18.01849334273 + 2.360852208681 * vh_lnTe - 0.2827443061704 * vh_lnTe*vh_lnTe + 0.01623316639567 * vh_lnTe*vh_lnTe*vh_lnTe - 0.03365012031362999 * vh_lnTe*vh_lnTe*vh_lnTe*vh_lnTe + 0.01178329782711 * ipow_<5>(vh_lnTe) - 0.001656194699504 * ipow_<6>(vh_lnTe) + 0.0001068275202678 * ipow_<7>(vh_lnTe) - 2.631285809207e-06 * ipow_<8>(vh_lnTe));  // H- + e- -> H + e- + e-
  k[20] = 2.96e-06 / std::sqrt(Tgas) - 1.73e-09 + 2.5e-10 * std::sqrt(Tgas) - 7.77e-13 * Tgas;  // H- + H+ -> H + H
  k[21] = 1e-08 * kb_pow(Tgas, -0.4);  // H- + H+ -> H2+ + e-
  k[22] = 1000000.0 * (4.2278e-14 - 2.3088e-17 * Tgas + 7.3428e-21 * Tgas*Tgas - 7.5474e-25 * Tgas*Tgas*Tgas + 3.3468e-29 * Tgas*Tgas*Tgas*Tgas - 5.528e-34 * ipow_<5>(Tgas));  // H2+ + e- -> H + H
  k[23] = 5e-07 * std::sqrt(100.0 * vh_invT);  // H2+ + H- -> H + H2
  k[24] = 6e-32 * kb_pow(Tgas, -0.25) + 2e-31 * 1.0/(std::sqrt(Tgas));  // H + H + H -> H2 + H
  k[25] = (6e-32 * kb_pow(Tgas, -0.25) + 2e-31 * 1.0/(std::sqrt(Tgas))) / 8.0;  // H2 + H + H -> H2 + H2
  k[27] = 1.2e-15 * kb_pow(Tgas / 300.0, 0.25);  // He+ + H -> He + H+
  k[71] = 6.622e-11 / (std::sqrt(Tgas / 4.136) * kb_pow(1.0 + std::sqrt(Tgas / 4.136), 1.0 - (0.6109 + 0.4093 * kb_exp(-87700.0 / Tgas))) * kb_pow(1.0 + std::sqrt(Tgas / 4214000.0), 1.0 + (0.6109 + 0.4093 * kb_exp(-87700.0 / Tgas)))) + 1.0/(ipow_<1>(Tgas) * std::sqrt(Tgas)) * (5.629e-08 * kb_exp(-5395.0 / Tgas) + 2.55e-07 * kb_exp(-17700.0 / Tgas) + 0.0006173 * kb_exp(-167100.0 / Tgas) + 0.0001627 * kb_exp(-268700.0 / Tgas));  // O+ + e- -> O
  k[72] = 0.0;  // CO+ + e- -> CO
  k[73] = 2.75e-07 * kb_pow(Tgas / 300.0, -0.55);  // CO+ + e- -> C + O
  {  // group 1: H+ + e- -> H
    double T = Tgas;
    const double vh_invTe = v_invTe(T, n, p);
    (void)vh_invTe;
    const double vh_lnTe = v_lnTe(T, n, p);
    (void)vh_lnTe;
    if (T < 5500.0) {
      k[1] = 3.92e-13 * kb_pow(vh_invTe, 0.6353);  // H+ + e- -> H
    }
    else if (T >= 5500.0) {
      k[2] = kb_exp(-28.61303380689232 - 0.7241125657826851 * vh_lnTe - 0.02026044731984691 * vh_lnTe*vh_lnTe - 0.002380861877349834 * vh_lnTe*vh_lnTe*vh_lnTe - 0.0003212605213188796 * vh_lnTe*vh_lnTe*vh_lnTe*vh_lnTe - 1.421502914054107e-05 * ipow_<5>(vh_lnTe) + 4.989108920299513e-06 * ipow_<6>(vh_lnTe) + 5.755614137575758e-07 * ipow_<7>(vh_lnTe) - 1.856767039775261e-08 * ipow_<8>(vh_lnTe) - 3.071135243196595e-09 * ipow_<9>(vh_lnTe));  // H+ + e- -> H
    }
  }
  {  // group 2: He+ + e- -> He
    double T = Tgas;
    const double vh_Te = v_Te(T, n, p);
    (void)vh_Te;
    const double vh_invTe = v_invTe(T, n, p);
    (void)vh_invTe;
    if (T < 9280.0) {
      k[4] = 3.92e-13 * kb_pow(vh_invTe, 0.6353);  // He+ + e- -> He
    }
    else if (T >= 9280.0) {
      k[5] = 1.54e-09 * (1.0 + 0.3 / kb_exp(8.099328789667 * vh_invTe)) / (kb_exp(40.49664394833662 * vh_invTe) * ipow_<1>(vh_Te) * std::sqrt(vh_Te)) + 3.92e-13 / kb_pow(vh_Te, 0.6353);  // He+ + e- -> He
    }
  }
  {  // group 3: H + H+ -> H2+
    double T = Tgas;
    if (T < 30.0) {
      k[10] = 2.1e-20 * kb_pow(T / 30.0, -0.15);  // H + H+ -> H2+
    }
    else if (T >= 30.0) {
      k[11] = kb_exp10(-18.2 - 3.194 * kb_log10(T) + 1.786 * kb_log10(T)*kb_log10(T) - 0.2072 * kb_log10(T)*kb_log10(T)*kb_log10(T));  // H + H+ -> H2+
    }
  }
  {  // group 4: H2 + H+ -> H2+ + H
    double T = Tgas;
    if (T > 30000.0) T = 30000.0;
    const double vh_asav = v_asav(T, n, p);
    (void)vh_asav;
    const double vh_bsav1 = v_bsav1(T, n, p);
    (void)vh_bsav1;
    const double vh_bsav2 = v_bsav2(T, n, p);
    (void)vh_bsav2;
    const double vh_bsav3 = v_bsav3(T, n, p);
    (void)vh_bsav3;
    const double vh_bsav4 = v_bsav4(T, n, p);
    (void)vh_bsav4;
    const double vh_bsav5 = v_bsav5(T, n, p);
    (void)vh_bsav5;
    const double vh_bsav6 = v_bsav6(T, n, p);
    (void)vh_bsav6;
    const double vh_bsav7 = v_bsav7(T, n, p);
    (void)vh_bsav7;
    const double vh_bsav8 = v_bsav8(T, n, p);
    (void)vh_bsav8;
    const double vh_invT = v_invT(T, n, p);
    (void)vh_invT;
    const double vh_sumsav = v_sumsav(T, n, p);
    (void)vh_sumsav;
    if (T >= 100.0 && T >= 100.0) {
      k[13] = vh_sumsav * kb_exp(-vh_asav * vh_invT);  // H2 + H+ -> H2+ + H
    }
  }
  {  // group 5: H- + H -> H + H + e-
    double T = Tgas;
    const double vh_Te = v_Te(T, n, p);
    (void)vh_Te;
    const double vh_lnTe = v_lnTe(T, n, p);
    (void)vh_lnTe;
    if (T < 1160.0) {
      k[18] = 2.56e-09 * kb_pow(vh_Te, 1.78186);  // H- + H -> H + H + e-
    }
    else if (T >= 1160.0) {
      k[19] = kb_exp(-20.37260896533324 + 1.139449335841631 * vh_lnTe - 0.1421013521554148 * vh_lnTe*vh_lnTe + 0.00846445538663 * vh_lnTe*vh_lnTe*vh_lnTe - 0.0014327641212992 * vh_lnTe*vh_lnTe*vh_lnTe*vh_lnTe + 0.0002012250284791 * ipow_<5>(vh_lnTe) + 8.66396324309e-05 * ipow_<6>(vh_lnTe) - 2.585009680264e-05 * ipow_<7>(vh_lnTe) + 2.4555011970392e-06 * ipow_<8>(vh_lnTe) - 8.06838246118e-08 * ipow_<9>(vh_lnTe));  // H- + H -> H + H + e-
    }
  }
  {  // group 6: He + H+ -> He+ + H
    double T = Tgas;
    const double vh_invT = v_invT(T, n, p);
    (void)vh_invT;
    if (T < 10000.0) {
      k[28] = 1.26e-09 * kb_pow(T, -0.75) * kb_exp(-127500.0 * vh_invT);  // He + H+ -> He+ + H
    }
    else if (T >= 10000.0) {
      k[29] = 4e-37 * kb_pow(T, 4.74);  // He + H+ -> He+ + H
    }
  }
}
// rate coefficients that also depend on the densities
KB_HD inline void rates_var(double Tgas, const double* n, const Params& p, double* k) {
  (void)Tgas; (void)n; (void)p; (void)k;
  const double vh_T = v_T(Tgas, n, p);
  (void)vh_T;
  const double vh_T32 = v_T32(Tgas, n, p);
  (void)vh_T32;
  const double vh_a21 = v_a21(Tgas, n, p);
  (void)vh_a21;
  const double vh_invT = v_invT(Tgas, n, p);
  (void)vh_invT;
  const double vh_kh21 = v_kh21(Tgas, n, p);
  (void)vh_kh21;
  const double vh_kl21 = v_kl21(Tgas, n, p);
  (void)vh_kl21;
  const double vh_ncr21 = v_ncr21(Tgas, n, p);
  (void)vh_ncr21;
  k[16] = dissH2_Martin96(Tgas, n, p);  // H2 + H -> H + H + H
  k[26] = kb_pow(vh_kh21, 1.0 - vh_a21) * kb_pow(vh_kl21, vh_a21);  // H2 + H2 -> H + H + H2
  k[30] = (ntot_(n) > 100000000000000.0 ? 0.0 : 6.8e-10);  // O+ + H -> H+ + O
  k[31] = (ntot_(n) > 100000000000000.0 ? 0.0 : 7e-10 * kb_exp(-232.0 * vh_invT));  // H+ + O -> O+ + H
  k[32] = (ntot_(n) > 100000000000000.0 ? 0.0 : 1.7e-09);  // O+ + H2 -> OH+ + H
  k[33] = (ntot_(n) > 100000000000000.0 ? 0.0 : 1.01e-09);  // OH+ + H2 -> H2O+ + H
  k[34] = (ntot_(n) > 100000000000000.0 ? 0.0 : 8.3e-10);  // H2O+ + H2 -> H3O+ + H
  k[35] = (ntot_(n) > 100000000000000.0 ? 0.0 : 2e-07 * 1.0/(std::sqrt(vh_T32)));  // H2O+ + e- -> O + H2
  k[36] = (ntot_(n) > 100000000000000.0 ? 0.0 : 1.6e-07 * 1.0/(std::sqrt(vh_T32)));  // H2O+ + e- -> OH + H
  k[37] = (ntot_(n) > 100000000000000.0 ? 0.0 : 3.5e-07 * 1.0/(std::sqrt(vh_T32)));  // H3O+ + e- -> H2O + H
  k[38] = (ntot_(n) > 100000000000000.0 ? 0.0 : 9.9e-19 * kb_pow(vh_T32, -0.38));  // O + H -> OH
  k[39] = (ntot_(n) > 100000000000000.0 ? 0.0 : 3.43e-13 * kb_pow(vh_T32, 2.67) * kb_exp(-3160.0 * vh_invT));  // O + H2 -> OH + H
  k[40] = (ntot_(n) > 100000000000000.0 ? 0.0 : 1.55e-12 * kb_pow(vh_T32, 1.6) * kb_exp(-1660.0 * vh_invT));  // H2 + OH -> H2O + H
  k[41] = (ntot_(n) > 100000000000000.0 ? 0.0 : 1.65e-12 * kb_pow(vh_T32, 1.14) * kb_exp(-50.0 * vh_invT));  // OH + OH -> H2O + O
  k[42] = (ntot_(n) > 100000000000000.0 ? 0.0 : 2.1e-09);  // H+ + OH -> OH+ + H
  k[43] = (ntot_(n) > 100000000000000.0 ? 0.0 : 6.9e-09);  // H+ + H2O -> H2O+ + H
  k[44] = (ntot_(n) > 100000000000000.0 ? 0.0 : 7e-14 * kb_pow(vh_T32, 2.8) * kb_exp(-1950.0 * vh_invT));  // H + OH -> H2 + O
  k[45] = (ntot_(n) > 100000000000000.0 ? 0.0 : 6.83e-12 * kb_pow(vh_T32, 1.6) * kb_exp(-9720.0 * vh_invT));  // H + H2O -> OH + H2
  k[46] = (ntot_(n) > 100000000000000.0 ? 0.0 : 4.9e-20 * kb_pow(vh_T32, 1.58));  // O + O -> O2
  k[47] = (ntot_(n) > 100000000000000.0 ? 0.0 : 4.34e-11 * 1.0/(std::sqrt(vh_T32)) * kb_exp(-30.0 * vh_invT));  // O + OH -> O2 + H
  k[48] = (ntot_(n) > 100000000000000.0 ? 0.0 : 3.3e-10 * kb_exp(-8460.0 * vh_invT));  // H + O2 -> OH + O
  k[49] = (ntot_(n) > 100000000000000.0 ? 0.0 : 2e-09);  // H+ + O2 -> O2+ + H
  k[50] = (ntot_(n) > 100000000000000.0 ? 0.0 : 1.95e-07 * kb_pow(vh_T32, -0.7));  // O2+ + e- -> O + O
  k[51] = (ntot_(n) > 100000000000000.0 ? 0.0 : 6.6e-11);  // O + CH -> CO + H
  k[52] = (ntot_(n) > 100000000000000.0 ? 0.0 : 1.1e-10 * std::sqrt(vh_T32));  // C + OH -> CO + H
  k[53] = (ntot_(n) > 100000000000000.0 ? 0.0 : 3.3e-11);  // C + O2 -> CO + O
  k[54] = (ntot_(n) > 100000000000000.0 ? 0.0 : 6.2e-10);  // C+ + O2 -> O+ + CO
  k[55] = (ntot_(n) > 100000000000000.0 ? 0.0 : 1e-13);  // OH + CO -> CO2 + H
  k[56] = (ntot_(n) > 100000000000000.0 ? 0.0 : 4.4e-12 * kb_pow(vh_T32, -0.61));  // C+ + e- -> C
  k[57] = (ntot_(n) > 100000000000000.0 ? 0.0 : 7.7e-10);  // C+ + OH -> CO+ + H
  k[58] = (ntot_(n) > 100000000000000.0 ? 0.0 : 7.5e-10);  // CO+ + H -> H+ + CO
  k[59] = (ntot_(n) > 100000000000000.0 ? 0.0 : 1e-17);  // C + H -> CH
  k[60] = (ntot_(n) > 100000000000000.0 ? 0.0 : 6.64e-10 * kb_exp(-11700.0 * vh_invT));  // C + H2 -> CH + H
  k[61] = (ntot_(n) > 100000000000000.0 ? 0.0 : 4.98e-11);  // H + CH -> C + H2
  k[62] = (ntot_(n) > 100000000000000.0 ? 0.0 : 2.38e-10 * kb_exp(-1760.0 * vh_invT));  // H2 + CH -> CH2 + H
  k[63] = (ntot_(n) > 100000000000000.0 ? 0.0 : 2.7e-10);  // H + CH2 -> CH + H2
  k[64] = (ntot_(n) > 100000000000000.0 ? 0.0 : 5.18e-11 * kb_pow(vh_T32, 0.17) * kb_exp(-6400.0 * vh_invT));  // H2 + CH2 -> CH3 + H
  k[65] = (ntot_(n) > 100000000000000.0 ? 0.0 : 1e-10 * kb_exp(-7600.0 * vh_invT));  // H + CH3 -> CH2 + H2
  k[66] = (ntot_(n) > 100000000000000.0 ? 0.0 : 6.86e-14 * kb_pow(vh_T32, 2.74) * kb_exp(-4740.0 * vh_invT));  // H2 + CH3 -> CH4 + H
  k[67] = (ntot_(n) > 100000000000000.0 ? 0.0 : 5.82e-13 * vh_T32*vh_T32*vh_T32 * kb_exp(-4045.0 * vh_invT));  // H + CH4 -> H2 + CH3
  k[68] = (ntot_(n) > 100000000000000.0 ? 0.0 : 1e-17);  // H2 + C -> CH2
  k[69] = (ntot_(n) > 100000000000000.0 ? 0.0 : 6.5e-07 * 1.0/(std::sqrt(vh_T32)));  // H3O+ + e- -> OH + H + H
  k[70] = (ntot_(n) > 100000000000000.0 ? 0.0 : 6.3e-09 * kb_pow(vh_T32, -0.48));  // OH+ + e- -> O + H
}
constexpr int NREA_FIXED = 31;
KB_HD inline bool rate_is_fixed(int r) {
  switch (r) {
    case 0:
    case 1:
    case 2:
    case 3:
    case 4:
    case 5:
    case 6:
    case 7:
    case 8:
    case 9:
    case 10:
    case 11:
    case 12:
    case 13:
    case 14:
    case 15:
    case 17:
    case 18:
    case 19:
    case 20:
    case 21:
    case 22:
    case 23:
    case 24:
    case 25:
    case 27:
    case 28:
    case 29:
    case 71:
    case 72:
    case 73:
      return true;
    default: return false;
  }
}

// mass-action dn/dt: per species, the flux terms in reaction order
KB_HD inline void rhs(const double* n, const double* k, double* dn) {
KB_UNROLL
  for (int i = 0; i < NSPEC; ++i) dn[i] = 0.0;
  double flux;
  (void)flux;
  flux = k[0]*n[IDX_H]*n[IDX_E];
  dn[IDX_H] -= flux;
  dn[IDX_E] -= flux;
  dn[IDX_Hj] += flux;
  dn[IDX_E] += flux;
  dn[IDX_E] += flux;
  flux = k[1]*n[IDX_Hj]*n[IDX_E];
  dn[IDX_Hj] -= flux;
  dn[IDX_E] -= flux;
  dn[IDX_H] += flux;
  flux = k[2]*n[IDX_Hj]*n[IDX_E];
  dn[IDX_Hj] -= flux;
  dn[IDX_E] -= flux;
  dn[IDX_H] += flux;
  flux = k[3]*n[IDX_He]*n[IDX_E];
  dn[IDX_He] -= flux;
  dn[IDX_E] -= flux;
  dn[IDX_Hej] += flux;
  dn[IDX_E] += flux;
  dn[IDX_E] += flux;
  flux = k[4]*n[IDX_Hej]*n[IDX_E];
  dn[IDX_Hej] -= flux;
  dn[IDX_E] -= flux;
  dn[IDX_He] += flux;
  flux = k[5]*n[IDX_Hej]*n[IDX_E];
  dn[IDX_Hej] -= flux;
  dn[IDX_E] -= flux;
  dn[IDX_He] += flux;
  flux = k[6]*n[IDX_Hej]*n[IDX_E];
  dn[IDX_Hej] -= flux;
  dn[IDX_E] -= flux;
  dn[IDX_Hejj] += flux;
  dn[IDX_E] += flux;
  dn[IDX_E] += flux;
  flux = k[7]*n[IDX_Hejj]*n[IDX_E];
  dn[IDX_Hejj] -= flux;
  dn[IDX_E] -= flux;
  dn[IDX_Hej] += flux;
  flux = k[8]*n[IDX_H]*n[IDX_E];
  dn[IDX_H] -= flux;
  dn[IDX_E] -= flux;
  dn[IDX_Hk] += flux;
  flux = k[9]*n[IDX_Hk]*n[IDX_H];
  dn[IDX_Hk] -= flux;
  dn[IDX_H] -= flux;
  dn[IDX_H2] += flux;
  dn[IDX_E] += flux;
  flux = k[10]*n[IDX_H]*n[IDX_Hj];
  dn[IDX_H] -= flux;
  dn[IDX_Hj] -= flux;
  dn[IDX_H2j] += flux;
  flux = k[11]*n[IDX_H]*n[IDX_Hj];
  dn[IDX_H] -= flux;
  dn[IDX_Hj] -= flux;
  dn[IDX_H2j] += flux;
  flux = k[12]*n[IDX_H2j]*n[IDX_H];
  dn[IDX_H2j] -= flux;
  dn[IDX_H] -= flux;
  dn[IDX_H2] += flux;
  dn[IDX_Hj] += flux;
  flux = k[13]*n[IDX_H2]*n[IDX_Hj];
  dn[IDX_H2] -= flux;
  dn[IDX_Hj] -= flux;
  dn[IDX_H2j] += flux;
  dn[IDX_H] += flux;
  flux = k[14]*n[IDX_H2]*n[IDX_E];
  dn[IDX_H2] -= flux;
  dn[IDX_E] -= flux;
  dn[IDX_H] += flux;
  dn[IDX_Hk] += flux;
  flux = k[15]*n[IDX_H2]*n[IDX_E];
  dn[IDX_H2] -= flux;
  dn[IDX_E] -= flux;
  dn[IDX_H] += flux;
  dn[IDX_H] += flux;
  dn[IDX_E] += flux;
  flux = k[16]*n[IDX_H2]*n[IDX_H];
  dn[IDX_H2] -= flux;
  dn[IDX_H] -= flux;
  dn[IDX_H] += flux;
  dn[IDX_H] += flux;
  dn[IDX_H] += flux;
  flux = k[17]*n[IDX_Hk]*n[IDX_E];
  dn[IDX_Hk] -= flux;
  dn[IDX_E] -= flux;
  dn[IDX_H] += flux;
  dn[IDX_E] += flux;
  dn[IDX_E] += flux;
  flux = k[18]*n[IDX_Hk]*n[IDX_H];
  dn[IDX_Hk] -= flux;
  dn[IDX_H] -= flux;
  dn[IDX_H] += flux;
  dn[IDX_H] += flux;
  dn[IDX_E] += flux;
  flux = k[19]*n[IDX_Hk]*n[IDX_H];
  dn[IDX_Hk] -= flux;
  dn[IDX_H] -= flux;
  dn[IDX_H] += flux;
  dn[IDX_H] += flux;
  dn[IDX_E] += flux;
  flux = k[20]*n[IDX_Hk]*n[IDX_Hj];
  dn[IDX_Hk] -= flux;
  dn[IDX_Hj] -= flux;
  dn[IDX_H] += flux;
  dn[IDX_H] += flux;
  flux = k[21]*n[IDX_Hk]*n[IDX_Hj];
  dn[IDX_Hk] -= flux;
  dn[IDX_Hj] -= flux;
  dn[IDX_H2j] += flux;
  dn[IDX_E] += flux;
  flux = k[22]*n[IDX_H2j]*n[IDX_E];
  dn[IDX_H2j] -= flux;
  dn[IDX_E] -= flux;
  dn[IDX_H] += flux;
  dn[IDX_H] += flux;
  flux = k[23]*n[IDX_H2j]*n[IDX_Hk];
  dn[IDX_H2j] -= flux;
  dn[IDX_Hk] -= flux;
  dn[IDX_H] += flux;
  dn[IDX_H2] += flux;
  flux = k[24]*n[IDX_H]*n[IDX_H]*n[IDX_H];
  dn[IDX_H] -= flux;
  dn[IDX_H] -= flux;
  dn[IDX_H] -= flux;
  dn[IDX_H2] += flux;
  dn[IDX_H] += flux;
  flux = k[25]*n[IDX_H2]*n[IDX_H]*n[IDX_H];
  dn[IDX_H2] -= flux;
  dn[IDX_H] -= flux;
  dn[IDX_H] -= flux;
  dn[IDX_H2] += flux;
  dn[IDX_H2] += flux;
  flux = k[26]*n[IDX_H2]*n[IDX_H2];
  dn[IDX_H2] -= flux;
  dn[IDX_H2] -= flux;
  dn[IDX_H] += flux;
  dn[IDX_H] += flux;
  dn[IDX_H2] += flux;
  flux = k[27]*n[IDX_Hej]*n[IDX_H];
  dn[IDX_Hej] -= flux;
  dn[IDX_H] -= flux;
  dn[IDX_He] += flux;
  dn[IDX_Hj] += flux;
  flux = k[28]*n[IDX_He]*n[IDX_Hj];
  dn[IDX_He] -= flux;
  dn[IDX_Hj] -= flux;
  dn[IDX_Hej] += flux;
  dn[IDX_H] += flux;
  flux = k[29]*n[IDX_He]*n[IDX_Hj];
  dn[IDX_He] -= flux;
  dn[IDX_Hj] -= flux;
  dn[IDX_Hej] += flux;
  dn[IDX_H] += flux;
  flux = k[30]*n[IDX_Oj]*n[IDX_H];
  dn[IDX_Oj] -= flux;
  dn[IDX_H] -= flux;
  dn[IDX_Hj] += flux;
  dn[IDX_O] += flux;
  flux = k[31]*n[IDX_Hj]*n[IDX_O];
  dn[IDX_Hj] -= flux;
  dn[IDX_O] -= flux;
  dn[IDX_Oj] += flux;
  dn[IDX_H] += flux;
  flux = k[32]*n[IDX_Oj]*n[IDX_H2];
  dn[IDX_Oj] -= flux;
  dn[IDX_H2] -= flux;
  dn[IDX_OHj] += flux;
  dn[IDX_H] += flux;
  flux = k[33]*n[IDX_OHj]*n[IDX_H2];
  dn[IDX_OHj] -= flux;
  dn[IDX_H2] -= flux;
  dn[IDX_H2Oj] += flux;
  dn[IDX_H] += flux;
  flux = k[34]*n[IDX_H2Oj]*n[IDX_H2];
  dn[IDX_H2Oj] -= flux;
  dn[IDX_H2] -= flux;
  dn[IDX_H3Oj] += flux;
  dn[IDX_H] += flux;
  flux = k[35]*n[IDX_H2Oj]*n[IDX_E];
  dn[IDX_H2Oj] -= flux;
  dn[IDX_E] -= flux;
  dn[IDX_O] += flux;
  dn[IDX_H2] += flux;
  flux = k[36]*n[IDX_H2Oj]*n[IDX_E];
  dn[IDX_H2Oj] -= flux;
  dn[IDX_E] -= flux;
  dn[IDX_OH] += flux;
  dn[IDX_H] += flux;
  flux = k[37]*n[IDX_H3Oj]*n[IDX_E];
  dn[IDX_H3Oj] -= flux;
  dn[IDX_E] -= flux;
  dn[IDX_H2O] += flux;
  dn[IDX_H] += flux;
  flux = k[38]*n[IDX_O]*n[IDX_H];
  dn[IDX_O] -= flux;
  dn[IDX_H] -= flux;
  dn[IDX_OH] += flux;
  flux = k[39]*n[IDX_O]*n[IDX_H2];
  dn[IDX_O] -= flux;
  dn[IDX_H2] -= flux;
  dn[IDX_OH] += flux;
  dn[IDX_H] += flux;
  flux = k[40]*n[IDX_H2]*n[IDX_OH];
  dn[IDX_H2] -= flux;
  dn[IDX_OH] -= flux;
  dn[IDX_H2O] += flux;
  dn[IDX_H] += flux;
  flux = k[41]*n[IDX_OH]*n[IDX_OH];
  dn[IDX_OH] -= flux;
  dn[IDX_OH] -= flux;
  dn[IDX_H2O] += flux;
  dn[IDX_O] += flux;
  flux = k[42]*n[IDX_Hj]*n[IDX_OH];
  dn[IDX_Hj] -= flux;
  dn[IDX_OH] -= flux;
  dn[IDX_OHj] += flux;
  dn[IDX_H] += flux;
  flux = k[43]*n[IDX_Hj]*n[IDX_H2O];
  dn[IDX_Hj] -= flux;
  dn[IDX_H2O] -= flux;
  dn[IDX_H2Oj] += flux;
  dn[IDX_H] += flux;
  flux = k[44]*n[IDX_H]*n[IDX_OH];
  dn[IDX_H] -= flux;
  dn[IDX_OH] -= flux;
  dn[IDX_H2] += flux;
  dn[IDX_O] += flux;
  flux = k[45]*n[IDX_H]*n[IDX_H2O];
  dn[IDX_H] -= flux;
  dn[IDX_H2O] -= flux;
  dn[IDX_OH] += flux;
  dn[IDX_H2] += flux;
  flux = k[46]*n[IDX_O]*n[IDX_O];
  dn[IDX_O] -= flux;
  dn[IDX_O] -= flux;
  dn[IDX_O2] += flux;
  flux = k[47]*n[IDX_O]*n[IDX_OH];
  dn[IDX_O] -= flux;
  dn[IDX_OH] -= flux;
  dn[IDX_O2] += flux;
  dn[IDX_H] += flux;
  flux = k[48]*n[IDX_H]*n[IDX_O2];
  dn[IDX_H] -= flux;
  dn[IDX_O2] -= flux;
  dn[IDX_OH] += flux;
  dn[IDX_O] += flux;
  flux = k[49]*n[IDX_Hj]*n[IDX_O2];
  dn[IDX_Hj] -= flux;
  dn[IDX_O2] -= flux;
  dn[IDX_O2j] += flux;
  dn[IDX_H] += flux;
  flux = k[50]*n[IDX_O2j]*n[IDX_E];
  dn[IDX_O2j] -= flux;
  dn[IDX_E] -= flux;
  dn[IDX_O] += flux;
  dn[IDX_O] += flux;
  flux = k[51]*n[IDX_O]*n[IDX_CH];
  dn[IDX_O] -= flux;
  dn[IDX_CH] -= flux;
  dn[IDX_CO] += flux;
  dn[IDX_H] += flux;
  flux = k[52]*n[IDX_C]*n[IDX_OH];
  dn[IDX_C] -= flux;
  dn[IDX_OH] -= flux;
  dn[IDX_CO] += flux;
  dn[IDX_H] += flux;
  flux = k[53]*n[IDX_C]*n[IDX_O2];
  dn[IDX_C] -= flux;
  dn[IDX_O2] -= flux;
  dn[IDX_CO] += flux;
  dn[IDX_O] += flux;
  flux = k[54]*n[IDX_Cj]*n[IDX_O2];
  dn[IDX_Cj] -= flux;
  dn[IDX_O2] -= flux;
  dn[IDX_Oj] += flux;
  dn[IDX_CO] += flux;
  flux = k[55]*n[IDX_OH]*n[IDX_CO];
  dn[IDX_OH] -= flux;
  dn[IDX_CO] -= flux;
  dn[IDX_CO2] += flux;
  dn[IDX_H] += flux;
  flux = k[56]*n[IDX_Cj]*n[IDX_E];
  dn[IDX_Cj] -= flux;
  dn[IDX_E] -= flux;
  dn[IDX_C] += flux;
  flux = k[57]*n[IDX_Cj]*n[IDX_OH];
  dn[IDX_Cj] -= flux;
  dn[IDX_OH] -= flux;
  dn[IDX_COj] += flux;
  dn[IDX_H] += flux;
  flux = k[58]*n[IDX_COj]*n[IDX_H];
  dn[IDX_COj] -= flux;
  dn[IDX_H] -= flux;
  dn[IDX_Hj] += flux;
  dn[IDX_CO] += flux;
  flux = k[59]*n[IDX_C]*n[IDX_H];
  dn[IDX_C] -= flux;
  dn[IDX_H] -= flux;
  dn[IDX_CH] += flux;
  flux = k[60]*n[IDX_C]*n[IDX_H2];
  dn[IDX_C] -= flux;
  dn[IDX_H2] -= flux;
  dn[IDX_CH] += flux;
  dn[IDX_H] += flux;
  flux = k[61]*n[IDX_H]*n[IDX_CH];
  dn[IDX_H] -= flux;
  dn[IDX_CH] -= flux;
  dn[IDX_C] += flux;
  dn[IDX_H2] += flux;
  flux = k[62]*n[IDX_H2]*n[IDX_CH];
  dn[IDX_H2] -= flux;
  dn[IDX_CH] -= flux;
  dn[IDX_CH2] += flux;
  dn[IDX_H] += flux;
  flux = k[63]*n[IDX_H]*n[IDX_CH2];
  dn[IDX_H] -= flux;
  dn[IDX_CH2] -= flux;
  dn[IDX_CH] += flux;
  dn[IDX_H2] += flux;
  flux = k[64]*n[IDX_H2]*n[IDX_CH2];
  dn[IDX_H2] -= flux;
  dn[IDX_CH2] -= flux;
  dn[IDX_CH3] += flux;
  dn[IDX_H] += flux;
  flux = k[65]*n[IDX_H]*n[IDX_CH3];
  dn[IDX_H] -= flux;
  dn[IDX_CH3] -= flux;
  dn[IDX_CH2] += flux;
  dn[IDX_H2] += flux;
  flux = k[66]*n[IDX_H2]*n[IDX_CH3];
  dn[IDX_H2] -= flux;
  dn[IDX_CH3] -= flux;
  dn[IDX_CH4] += flux;
  dn[IDX_H] += flux;
  flux = k[67]*n[IDX_H]*n[IDX_CH4];
  dn[IDX_H] -= flux;
  dn[IDX_CH4] -= flux;
  dn[IDX_H2] += flux;
  dn[IDX_CH3] += flux;
  flux = k[68]*n[IDX_H2]*n[IDX_C];
  dn[IDX_H2] -= flux;
  dn[IDX_C] -= flux;
  dn[IDX_CH2] += flux;
  flux = k[69]*n[IDX_H3Oj]*n[IDX_E];
  dn[IDX_H3Oj] -= flux;
  dn[IDX_E] -= flux;
  dn[IDX_OH] += flux;
  dn[IDX_H] += flux;
  dn[IDX_H] += flux;
  flux = k[70]*n[IDX_OHj]*n[IDX_E];
  dn[IDX_OHj] -= flux;
  dn[IDX_E] -= flux;
  dn[IDX_O] += flux;
  dn[IDX_H] += flux;
  flux = k[71]*n[IDX_Oj]*n[IDX_E];
  dn[IDX_Oj] -= flux;
  dn[IDX_E] -= flux;
  dn[IDX_O] += flux;
  flux = k[72]*n[IDX_COj]*n[IDX_E];
  dn[IDX_COj] -= flux;
  dn[IDX_E] -= flux;
  dn[IDX_CO] += flux;
  flux = k[73]*n[IDX_COj]*n[IDX_E];
  dn[IDX_COj] -= flux;
  dn[IDX_E] -= flux;
  dn[IDX_C] += flux;
  dn[IDX_O] += flux;
}

KB_HD inline void jac_stoich(const double* n, const double* k, double* J, int rs, int cs) {
  for (int i = 0; i < NSPEC; ++i)
    for (int j = 0; j < NSPEC; ++j) J[i*rs + j*cs] = 0.0;
  double d;
  (void)d; (void)n; (void)k;
  d = k[0]*n[IDX_E];
  J[IDX_H*rs + IDX_H*cs] -= d;
  J[IDX_E*rs + IDX_H*cs] -= d;
  J[IDX_Hj*rs + IDX_H*cs] += d;
  J[IDX_E*rs + IDX_H*cs] += d;
  J[IDX_E*rs + IDX_H*cs] += d;
  d = k[0]*n[IDX_H];
  J[IDX_H*rs + IDX_E*cs] -= d;
  J[IDX_E*rs + IDX_E*cs] -= d;
  J[IDX_Hj*rs + IDX_E*cs] += d;
  J[IDX_E*rs + IDX_E*cs] += d;
  J[IDX_E*rs + IDX_E*cs] += d;
  d = k[1]*n[IDX_E];
  J[IDX_Hj*rs + IDX_Hj*cs] -= d;
  J[IDX_E*rs + IDX_Hj*cs] -= d;
  J[IDX_H*rs + IDX_Hj*cs] += d;
  d = k[1]*n[IDX_Hj];
  J[IDX_Hj*rs + IDX_E*cs] -= d;
  J[IDX_E*rs + IDX_E*cs] -= d;
  J[IDX_H*rs + IDX_E*cs] += d;
  d = k[2]*n[IDX_E];
  J[IDX_Hj*rs + IDX_Hj*cs] -= d;
  J[IDX_E*rs + IDX_Hj*cs] -= d;
  J[IDX_H*rs + IDX_Hj*cs] += d;
  d = k[2]*n[IDX_Hj];
  J[IDX_Hj*rs + IDX_E*cs] -= d;
  J[IDX_E*rs + IDX_E*cs] -= d;
  J[IDX_H*rs + IDX_E*cs] += d;
  d = k[3]*n[IDX_E];
  J[IDX_He*rs + IDX_He*cs] -= d;
  J[IDX_E*rs + IDX_He*cs] -= d;
  J[IDX_Hej*rs + IDX_He*cs] += d;
  J[IDX_E*rs + IDX_He*cs] += d;
  J[IDX_E*rs + IDX_He*cs] += d;
  d = k[3]*n[IDX_He];
  J[IDX_He*rs + IDX_E*cs] -= d;
  J[IDX_E*rs + IDX_E*cs] -= d;
  J[IDX_Hej*rs + IDX_E*cs] += d;
  J[IDX_E*rs + IDX_E*cs] += d;
  J[IDX_E*rs + IDX_E*cs] += d;
  d = k[4]*n[IDX_E];
  J[IDX_Hej*rs + IDX_Hej*cs] -= d;
  J[IDX_E*rs + IDX_Hej*cs] -= d;
  J[IDX_He*rs + IDX_Hej*cs] += d;
  d = k[4]*n[IDX_Hej];
  J[IDX_Hej*rs + IDX_E*cs] -= d;
  J[IDX_E*rs + IDX_E*cs] -= d;
  J[IDX_He*rs + IDX_E*cs] += d;
  d = k[5]*n[IDX_E];
  J[IDX_Hej*rs + IDX_Hej*cs] -= d;
  J[IDX_E*rs + IDX_Hej*cs] -= d;
  J[IDX_He*rs + IDX_Hej*cs] += d;
  d = k[5]*n[IDX_Hej];
  J[IDX_Hej*rs + IDX_E*cs] -= d;
  J[IDX_E*rs + IDX_E*cs] -= d;
  J[IDX_He*rs + IDX_E*cs] += d;
  d = k[6]*n[IDX_E];
  J[IDX_Hej*rs + IDX_Hej*cs] -= d;
  J[IDX_E*rs + IDX_Hej*cs] -= d;
  J[IDX_Hejj*rs + IDX_Hej*cs] += d;
  J[IDX_E*rs + IDX_Hej*cs] += d;
  J[IDX_E*rs + IDX_Hej*cs] += d;
  d = k[6]*n[IDX_Hej];
  J[IDX_Hej*rs + IDX_E*cs] -= d;
  J[IDX_E*rs + IDX_E*cs] -= d;
  J[IDX_Hejj*rs + IDX_E*cs] += d;
  J[IDX_E*rs + IDX_E*cs] += d;
  J[IDX_E*rs + IDX_E*cs] += d;
  d = k[7]*n[IDX_E];
  J[IDX_Hejj*rs + IDX_Hejj*cs] -= d;
  J[IDX_E*rs + IDX_Hejj*cs] -= d;
  J[IDX_Hej*rs + IDX_Hejj*cs] += d;
  d = k[7]*n[IDX_Hejj];
  J[IDX_Hejj*rs + IDX_E*cs] -= d;
  J[IDX_E*rs + IDX_E*cs] -= d;
  J[IDX_Hej*rs + IDX_E*cs] += d;
  d = k[8]*n[IDX_E];
  J[IDX_H*rs + IDX_H*cs] -= d;
  J[IDX_E*rs + IDX_H*cs] -= d;
  J[IDX_Hk*rs + IDX_H*cs] += d;
  d = k[8]*n[IDX_H];
  J[IDX_H*rs + IDX_E*cs] -= d;
  J[IDX_E*rs + IDX_E*cs] -= d;
  J[IDX_Hk*rs + IDX_E*cs] += d;
  d = k[9]*n[IDX_Hk];
  J[IDX_Hk*rs + IDX_H*cs] -= d;
  J[IDX_H*rs + IDX_H*cs] -= d;
  J[IDX_H2*rs + IDX_H*cs] += d;
  J[IDX_E*rs + IDX_H*cs] += d;
  d = k[9]*n[IDX_H];
  J[IDX_Hk*rs + IDX_Hk*cs] -= d;
  J[IDX_H*rs + IDX_Hk*cs] -= d;
  J[IDX_H2*rs + IDX_Hk*cs] += d;
  J[IDX_E*rs + IDX_Hk*cs] += d;
  d = k[10]*n[IDX_Hj];
  J[IDX_H*rs + IDX_H*cs] -= d;
  J[IDX_Hj*rs + IDX_H*cs] -= d;
  J[IDX_H2j*rs + IDX_H*cs] += d;
  d = k[10]*n[IDX_H];
  J[IDX_H*rs + IDX_Hj*cs] -= d;
  J[IDX_Hj*rs + IDX_Hj*cs] -= d;
  J[IDX_H2j*rs + IDX_Hj*cs] += d;
  d = k[11]*n[IDX_Hj];
  J[IDX_H*rs + IDX_H*cs] -= d;
  J[IDX_Hj*rs + IDX_H*cs] -= d;
  J[IDX_H2j*rs + IDX_H*cs] += d;
  d = k[11]*n[IDX_H];
  J[IDX_H*rs + IDX_Hj*cs] -= d;
  J[IDX_Hj*rs + IDX_Hj*cs] -= d;
  J[IDX_H2j*rs + IDX_Hj*cs] += d;
  d = k[12]*n[IDX_H2j];
  J[IDX_H2j*rs + IDX_H*cs] -= d;
  J[IDX_H*rs + IDX_H*cs] -= d;
  J[IDX_H2*rs + IDX_H*cs] += d;
  J[IDX_Hj*rs + IDX_H*cs] += d;
  d = k[12]*n[IDX_H];
  J[IDX_H2j*rs + IDX_H2j*cs] -= d;
  J[IDX_H*rs + IDX_H2j*cs] -= d;
  J[IDX_H2*rs + IDX_H2j*cs] += d;
  J[IDX_Hj*rs + IDX_H2j*cs] += d;
  d = k[13]*n[IDX_H2];
  J[IDX_H2*rs + IDX_Hj*cs] -= d;
  J[IDX_Hj*rs + IDX_Hj*cs] -= d;
  J[IDX_H2j*rs + IDX_Hj*cs] += d;
  J[IDX_H*rs + IDX_Hj*cs] += d;
  d = k[13]*n[IDX_Hj];
  J[IDX_H2*rs + IDX_H2*cs] -= d;
  J[IDX_Hj*rs + IDX_H2*cs] -= d;
  J[IDX_H2j*rs + IDX_H2*cs] += d;
  J[IDX_H*rs + IDX_H2*cs] += d;
  d = k[14]*n[IDX_E];
  J[IDX_H2*rs + IDX_H2*cs] -= d;
  J[IDX_E*rs + IDX_H2*cs] -= d;
  J[IDX_H*rs + IDX_H2*cs] += d;
  J[IDX_Hk*rs + IDX_H2*cs] += d;
  d = k[14]*n[IDX_H2];
  J[IDX_H2*rs + IDX_E*cs] -= d;
  J[IDX_E*rs + IDX_E*cs] -= d;
  J[IDX_H*rs + IDX_E*cs] += d;
  J[IDX_Hk*rs + IDX_E*cs] += d;
  d = k[15]*n[IDX_E];
  J[IDX_H2*rs + IDX_H2*cs] -= d;
  J[IDX_E*rs + IDX_H2*cs] -= d;
  J[IDX_H*rs + IDX_H2*cs] += d;
  J[IDX_H*rs + IDX_H2*cs] += d;
  J[IDX_E*rs + IDX_H2*cs] += d;
  d = k[15]*n[IDX_H2];
  J[IDX_H2*rs + IDX_E*cs] -= d;
  J[IDX_E*rs + IDX_E*cs] -= d;
  J[IDX_H*rs + IDX_E*cs] += d;
  J[IDX_H*rs + IDX_E*cs] += d;
  J[IDX_E*rs + IDX_E*cs] += d;
  d = k[16]*n[IDX_H2];
  J[IDX_H2*rs + IDX_H*cs] -= d;
  J[IDX_H*rs + IDX_H*cs] -= d;
  J[IDX_H*rs + IDX_H*cs] += d;
  J[IDX_H*rs + IDX_H*cs] += d;
  J[IDX_H*rs + IDX_H*cs] += d;
  d = k[16]*n[IDX_H];
  J[IDX_H2*rs + IDX_H2*cs] -= d;
  J[IDX_H*rs + IDX_H2*cs] -= d;
  J[IDX_H*rs + IDX_H2*cs] += d;
  J[IDX_H*rs + IDX_H2*cs] += d;
  J[IDX_H*rs + IDX_H2*cs] += d;
  d = k[17]*n[IDX_E];
  J[IDX_Hk*rs + IDX_Hk*cs] -= d;
  J[IDX_E*rs + IDX_Hk*cs] -= d;
  J[IDX_H*rs + IDX_Hk*cs] += d;
  J[IDX_E*rs + IDX_Hk*cs] += d;
  J[IDX_E*rs + IDX_Hk*cs] += d;
  d = k[17]*n[IDX_Hk];
  J[IDX_Hk*rs + IDX_E*cs] -= d;
  J[IDX_E*rs + IDX_E*cs] -= d;
  J[IDX_H*rs + IDX_E*cs] += d;
  J[IDX_E*rs + IDX_E*cs] += d;
  J[IDX_E*rs + IDX_E*cs] += d;
  d = k[18]*n[IDX_Hk];
  J[IDX_Hk*rs + IDX_H*cs] -= d;
  J[IDX_H*rs + IDX_H*cs] -= d;
  J[IDX_H*rs + IDX_H*cs] += d;
  J[IDX_H*rs + IDX_H*cs] += d;
  J[IDX_E*rs + IDX_H*cs] += d;
  d = k[18]*n[IDX_H];
  J[IDX_Hk*rs + IDX_Hk*cs] -= d;
  J[IDX_H*rs + IDX_Hk*cs] -= d;
  J[IDX_H*rs + IDX_Hk*cs] += d;
  J[IDX_H*rs + IDX_Hk*cs] += d;
  J[IDX_E*rs + IDX_Hk*cs] += d;
  d = k[19]*n[IDX_Hk];
  J[IDX_Hk*rs + IDX_H*cs] -= d;
  J[IDX_H*rs + IDX_H*cs] -= d;
  J[IDX_H*rs + IDX_H*cs] += d;
  J[IDX_H*rs + IDX_H*cs] += d;
  J[IDX_E*rs + IDX_H*cs] += d;
  d = k[19]*n[IDX_H];
  J[IDX_Hk*rs + IDX_Hk*cs] -= d;
  J[IDX_H*rs + IDX_Hk*cs] -= d;
  J[IDX_H*rs + IDX_Hk*cs] += d;
  J[IDX_H*rs + IDX_Hk*cs] += d;
  J[IDX_E*rs + IDX_Hk*cs] += d;
  d = k[20]*n[IDX_Hk];
  J[IDX_Hk*rs + IDX_Hj*cs] -= d;
  J[IDX_Hj*rs + IDX_Hj*cs] -= d;
  J[IDX_H*rs + IDX_Hj*cs] += d;
  J[IDX_H*rs + IDX_Hj*cs] += d;
  d = k[20]*n[IDX_Hj];
  J[IDX_Hk*rs + IDX_Hk*cs] -= d;
  J[IDX_Hj*rs + IDX_Hk*cs] -= d;
  J[IDX_H*rs + IDX_Hk*cs] += d;
  J[IDX_H*rs + IDX_Hk*cs] += d;
  d = k[21]*n[IDX_Hk];
  J[IDX_Hk*rs + IDX_Hj*cs] -= d;
  J[IDX_Hj*rs + IDX_Hj*cs] -= d;
  J[IDX_H2j*rs + IDX_Hj*cs] += d;
  J[IDX_E*rs + IDX_Hj*cs] += d;
  d = k[21]*n[IDX_Hj];
  J[IDX_Hk*rs + IDX_Hk*cs] -= d;
  J[IDX_Hj*rs + IDX_Hk*cs] -= d;
  J[IDX_H2j*rs + IDX_Hk*cs] += d;
  J[IDX_E*rs + IDX_Hk*cs] += d;
  d = k[22]*n[IDX_E];
  J[IDX_H2j*rs + IDX_H2j*cs] -= d;
  J[IDX_E*rs + IDX_H2j*cs] -= d;
  J[IDX_H*rs + IDX_H2j*cs] += d;
  J[IDX_H*rs + IDX_H2j*cs] += d;
  d = k[22]*n[IDX_H2j];
  J[IDX_H2j*rs + IDX_E*cs] -= d;
  J[IDX_E*rs + IDX_E*cs] -= d;
  J[IDX_H*rs + IDX_E*cs] += d;
  J[IDX_H*rs + IDX_E*cs] += d;
  d = k[23]*n[IDX_H2j];
  J[IDX_H2j*rs + IDX_Hk*cs] -= d;
  J[IDX_Hk*rs + IDX_Hk*cs] -= d;
  J[IDX_H*rs + IDX_Hk*cs] += d;
  J[IDX_H2*rs + IDX_Hk*cs] += d;
  d = k[23]*n[IDX_Hk];
  J[IDX_H2j*rs + IDX_H2j*cs] -= d;
  J[IDX_Hk*rs + IDX_H2j*cs] -= d;
  J[IDX_H*rs + IDX_H2j*cs] += d;
  J[IDX_H2*rs + IDX_H2j*cs] += d;
  d = 3.0*k[24]*n[IDX_H]*n[IDX_H];
  J[IDX_H*rs + IDX_H*cs] -= d;
  J[IDX_H*rs + IDX_H*cs] -= d;
  J[IDX_H*rs + IDX_H*cs] -= d;
  J[IDX_H2*rs + IDX_H*cs] += d;
  J[IDX_H*rs + IDX_H*cs] += d;
  d = 2.0*k[25]*n[IDX_H]*n[IDX_H2];
  J[IDX_H2*rs + IDX_H*cs] -= d;
  J[IDX_H*rs + IDX_H*cs] -= d;
  J[IDX_H*rs + IDX_H*cs] -= d;
  J[IDX_H2*rs + IDX_H*cs] += d;
  J[IDX_H2*rs + IDX_H*cs] += d;
  d = k[25]*n[IDX_H]*n[IDX_H];
  J[IDX_H2*rs + IDX_H2*cs] -= d;
  J[IDX_H*rs + IDX_H2*cs] -= d;
  J[IDX_H*rs + IDX_H2*cs] -= d;
  J[IDX_H2*rs + IDX_H2*cs] += d;
  J[IDX_H2*rs + IDX_H2*cs] += d;
  d = 2.0*k[26]*n[IDX_H2];
  J[IDX_H2*rs + IDX_H2*cs] -= d;
  J[IDX_H2*rs + IDX_H2*cs] -= d;
  J[IDX_H*rs + IDX_H2*cs] += d;
  J[IDX_H*rs + IDX_H2*cs] += d;
  J[IDX_H2*rs + IDX_H2*cs] += d;
  d = k[27]*n[IDX_Hej];
  J[IDX_Hej*rs + IDX_H*cs] -= d;
  J[IDX_H*rs + IDX_H*cs] -= d;
  J[IDX_He*rs + IDX_H*cs] += d;
  J[IDX_Hj*rs + IDX_H*cs] += d;
  d = k[27]*n[IDX_H];
  J[IDX_Hej*rs + IDX_Hej*cs] -= d;
  J[IDX_H*rs + IDX_Hej*cs] -= d;
  J[IDX_He*rs + IDX_Hej*cs] += d;
  J[IDX_Hj*rs + IDX_Hej*cs] += d;
  d = k[28]*n[IDX_He];
  J[IDX_He*rs + IDX_Hj*cs] -= d;
  J[IDX_Hj*rs + IDX_Hj*cs] -= d;
  J[IDX_Hej*rs + IDX_Hj*cs] += d;
  J[IDX_H*rs + IDX_Hj*cs] += d;
  d = k[28]*n[IDX_Hj];
  J[IDX_He*rs + IDX_He*cs] -= d;
  J[IDX_Hj*rs + IDX_He*cs] -= d;
  J[IDX_Hej*rs + IDX_He*cs] += d;
  J[IDX_H*rs + IDX_He*cs] += d;
  d = k[29]*n[IDX_He];
  J[IDX_He*rs + IDX_Hj*cs] -= d;
  J[IDX_Hj*rs + IDX_Hj*cs] -= d;
  J[IDX_Hej*rs + IDX_Hj*cs] += d;
  J[IDX_H*rs + IDX_Hj*cs] += d;
  d = k[29]*n[IDX_Hj];
  J[IDX_He*rs + IDX_He*cs] -= d;
  J[IDX_Hj*rs + IDX_He*cs] -= d;
  J[IDX_Hej*rs + IDX_He*cs] += d;
  J[IDX_H*rs + IDX_He*cs] += d;
  d = k[30]*n[IDX_Oj];
  J[IDX_Oj*rs + IDX_H*cs] -= d;
  J[IDX_H*rs + IDX_H*cs] -= d;
  J[IDX_Hj*rs + IDX_H*cs] += d;
  J[IDX_O*rs + IDX_H*cs] += d;
  d = k[30]*n[IDX_H];
  J[IDX_Oj*rs + IDX_Oj*cs] -= d;
  J[IDX_H*rs + IDX_Oj*cs] -= d;
  J[IDX_Hj*rs + IDX_Oj*cs] += d;
  J[IDX_O*rs + IDX_Oj*cs] += d;
  d = k[31]*n[IDX_O];
  J[IDX_Hj*rs + IDX_Hj*cs] -= d;
  J[IDX_O*rs + IDX_Hj*cs] -= d;
  J[IDX_Oj*rs + IDX_Hj*cs] += d;
  J[IDX_H*rs + IDX_Hj*cs] += d;
  d = k[31]*n[IDX_Hj];
  J[IDX_Hj*rs + IDX_O*cs] -= d;
  J[IDX_O*rs + IDX_O*cs] -= d;
  J[IDX_Oj*rs + IDX_O*cs] += d;
  J[IDX_H*rs + IDX_O*cs] += d;
  d = k[32]*n[IDX_Oj];
  J[IDX_Oj*rs + IDX_H2*cs] -= d;
  J[IDX_H2*rs + IDX_H2*cs] -= d;
  J[IDX_OHj*rs + IDX_H2*cs] += d;
  J[IDX_H*rs + IDX_H2*cs] += d;
  d = k[32]*n[IDX_H2];
  J[IDX_Oj*rs + IDX_Oj*cs] -= d;
  J[IDX_H2*rs + IDX_Oj*cs] -= d;
  J[IDX_OHj*rs + IDX_Oj*cs] += d;
  J[IDX_H*rs + IDX_Oj*cs] += d;
  d = k[33]*n[IDX_OHj];
  J[IDX_OHj*rs + IDX_H2*cs] -= d;
  J[IDX_H2*rs + IDX_H2*cs] -= d;
  J[IDX_H2Oj*rs + IDX_H2*cs] += d;
  J[IDX_H*rs + IDX_H2*cs] += d;
  d = k[33]*n[IDX_H2];
  J[IDX_OHj*rs + IDX_OHj*cs] -= d;
  J[IDX_H2*rs + IDX_OHj*cs] -= d;
  J[IDX_H2Oj*rs + IDX_OHj*cs] += d;
  J[IDX_H*rs + IDX_OHj*cs] += d;
  d = k[34]*n[IDX_H2Oj];
  J[IDX_H2Oj*rs + IDX_H2*cs] -= d;
  J[IDX_H2*rs + IDX_H2*cs] -= d;
  J[IDX_H3Oj*rs + IDX_H2*cs] += d;
  J[IDX_H*rs + IDX_H2*cs] += d;
  d = k[34]*n[IDX_H2];
  J[IDX_H2Oj*rs + IDX_H2Oj*cs] -= d;
  J[IDX_H2*rs + IDX_H2Oj*cs] -= d;
  J[IDX_H3Oj*rs + IDX_H2Oj*cs] += d;
  J[IDX_H*rs + IDX_H2Oj*cs] += d;
  d = k[35]*n[IDX_E];
  J[IDX_H2Oj*rs + IDX_H2Oj*cs] -= d;
  J[IDX_E*rs + IDX_H2Oj*cs] -= d;
  J[IDX_O*rs + IDX_H2Oj*cs] += d;
  J[IDX_H2*rs + IDX_H2Oj*cs] += d;
  d = k[35]*n[IDX_H2Oj];
  J[IDX_H2Oj*rs + IDX_E*cs] -= d;
  J[IDX_E*rs + IDX_E*cs] -= d;
  J[IDX_O*rs + IDX_E*cs] += d;
  J[IDX_H2*rs + IDX_E*cs] += d;
  d = k[36]*n[IDX_E];
  J[IDX_H2Oj*rs + IDX_H2Oj*cs] -= d;
  J[IDX_E*rs + IDX_H2Oj*cs] -= d;
  J[IDX_OH*rs + IDX_H2Oj*cs] += d;
  J[IDX_H*rs + IDX_H2Oj*cs] += d;
  d = k[36]*n[IDX_H2Oj];
  J[IDX_H2Oj*rs + IDX_E*cs] -= d;
  J[IDX_E*rs + IDX_E*cs] -= d;
  J[IDX_OH*rs + IDX_E*cs] += d;
  J[IDX_H*rs + IDX_E*cs] += d;
  d = k[37]*n[IDX_E];
  J[IDX_H3Oj*rs + IDX_H3Oj*cs] -= d;
  J[IDX_E*rs + IDX_H3Oj*cs] -= d;
  J[IDX_H2O*rs + IDX_H3Oj*cs] += d;
  J[IDX_H*rs + IDX_H3Oj*cs] += d;
  d = k[37]*n[IDX_H3Oj];
  J[IDX_H3Oj*rs + IDX_E*cs] -= d;
  J[IDX_E*rs + IDX_E*cs] -= d;
  J[IDX_H2O*rs + IDX_E*cs] += d;
  J[IDX_H*rs + IDX_E*cs] += d;
  d = k[38]*n[IDX_O];
  J[IDX_O*rs + IDX_H*cs] -= d;
  J[IDX_H*rs + IDX_H*cs] -= d;
  J[IDX_OH*rs + IDX_H*cs] += d;
  d = k[38]*n[IDX_H];
  J[IDX_O*rs + IDX_O*cs] -= d;
  J[IDX_H*rs + IDX_O*cs] -= d;
  J[IDX_OH*rs + IDX_O*cs] += d;
  d = k[39]*n[IDX_O];
  J[IDX_O*rs + IDX_H2*cs] -= d;
  J[IDX_H2*rs + IDX_H2*cs] -= d;
  J[IDX_OH*rs + IDX_H2*cs] += d;
  J[IDX_H*rs + IDX_H2*cs] += d;
  d = k[39]*n[IDX_H2];
  J[IDX_O*rs + IDX_O*cs] -= d;
  J[IDX_H2*rs + IDX_O*cs] -= d;
  J[IDX_OH*rs + IDX_O*cs] += d;
  J[IDX_H*rs + IDX_O*cs] += d;
  d = k[40]*n[IDX_OH];
  J[IDX_H2*rs + IDX_H2*cs] -= d;
  J[IDX_OH*rs + IDX_H2*cs] -= d;
  J[IDX_H2O*rs + IDX_H2*cs] += d;
  J[IDX_H*rs + IDX_H2*cs] += d;
  d = k[40]*n[IDX_H2];
  J[IDX_H2*rs + IDX_OH*cs] -= d;
  J[IDX_OH*rs + IDX_OH*cs] -= d;
  J[IDX_H2O*rs + IDX_OH*cs] += d;
  J[IDX_H*rs + IDX_OH*cs] += d;
  d = 2.0*k[41]*n[IDX_OH];
  J[IDX_OH*rs + IDX_OH*cs] -= d;
  J[IDX_OH*rs + IDX_OH*cs] -= d;
  J[IDX_H2O*rs + IDX_OH*cs] += d;
  J[IDX_O*rs + IDX_OH*cs] += d;
  d = k[42]*n[IDX_OH];
  J[IDX_Hj*rs + IDX_Hj*cs] -= d;
  J[IDX_OH*rs + IDX_Hj*cs] -= d;
  J[IDX_OHj*rs + IDX_Hj*cs] += d;
  J[IDX_H*rs + IDX_Hj*cs] += d;
  d = k[42]*n[IDX_Hj];
  J[IDX_Hj*rs + IDX_OH*cs] -= d;
  J[IDX_OH*rs + IDX_OH*cs] -= d;
  J[IDX_OHj*rs + IDX_OH*cs] += d;
  J[IDX_H*rs + IDX_OH*cs] += d;
  d = k[43]*n[IDX_H2O];
  J[IDX_Hj*rs + IDX_Hj*cs] -= d;
  J[IDX_H2O*rs + IDX_Hj*cs] -= d;
  J[IDX_H2Oj*rs + IDX_Hj*cs] += d;
  J[IDX_H*rs + IDX_Hj*cs] += d;
  d = k[43]*n[IDX_Hj];
  J[IDX_Hj*rs + IDX_H2O*cs] -= d;
  J[IDX_H2O*rs + IDX_H2O*cs] -= d;
  J[IDX_H2Oj*rs + IDX_H2O*cs] += d;
  J[IDX_H*rs + IDX_H2O*cs] += d;
  d = k[44]*n[IDX_OH];
  J[IDX_H*rs + IDX_H*cs] -= d;
  J[IDX_OH*rs + IDX_H*cs] -= d;
  J[IDX_H2*rs + IDX_H*cs] += d;
  J[IDX_O*rs + IDX_H*cs] += d;
  d = k[44]*n[IDX_H];
  J[IDX_H*rs + IDX_OH*cs] -= d;
  J[IDX_OH*rs + IDX_OH*cs] -= d;
  J[IDX_H2*rs + IDX_OH*cs] += d;
  J[IDX_O*rs + IDX_OH*cs] += d;
  d = k[45]*n[IDX_H2O];
  J[IDX_H*rs + IDX_H*cs] -= d;
  J[IDX_H2O*rs + IDX_H*cs] -= d;
  J[IDX_OH*rs + IDX_H*cs] += d;
  J[IDX_H2*rs + IDX_H*cs] += d;
  d = k[45]*n[IDX_H];
  J[IDX_H*rs + IDX_H2O*cs] -= d;
  J[IDX_H2O*rs + IDX_H2O*cs] -= d;
  J[IDX_OH*rs + IDX_H2O*cs] += d;
  J[IDX_H2*rs + IDX_H2O*cs] += d;
  d = 2.0*k[46]*n[IDX_O];
  J[IDX_O*rs + IDX_O*cs] -= d;
  J[IDX_O*rs + IDX_O*cs] -= d;
  J[IDX_O2*rs + IDX_O*cs] += d;
  d = k[47]*n[IDX_OH];
  J[IDX_O*rs + IDX_O*cs] -= d;
  J[IDX_OH*rs + IDX_O*cs] -= d;
  J[IDX_O2*rs + IDX_O*cs] += d;
  J[IDX_H*rs + IDX_O*cs] += d;
  d = k[47]*n[IDX_O];
  J[IDX_O*rs + IDX_OH*cs] -= d;
  J[IDX_OH*rs + IDX_OH*cs] -= d;
  J[IDX_O2*rs + IDX_OH*cs] += d;
  J[IDX_H*rs + IDX_OH*cs] += d;
  d = k[48]*n[IDX_O2];
  J[IDX_H*rs + IDX_H*cs] -= d;
  J[IDX_O2*rs + IDX_H*cs] -= d;
  J[IDX_OH*rs + IDX_H*cs] += d;
  J[IDX_O*rs + IDX_H*cs] += d;
  d = k[48]*n[IDX_H];
  J[IDX_H*rs + IDX_O2*cs] -= d;
  J[IDX_O2*rs + IDX_O2*cs] -= d;
  J[IDX_OH*rs + IDX_O2*cs] += d;
  J[IDX_O*rs + IDX_O2*cs] += d;
  d = k[49]*n[IDX_O2];
  J[IDX_Hj*rs + IDX_Hj*cs] -= d;
  J[IDX_O2*rs + IDX_Hj*cs] -= d;
  J[IDX_O2j*rs + IDX_Hj*cs] += d;
  J[IDX_H*rs + IDX_Hj*cs] += d;
  d = k[49]*n[IDX_Hj];
  J[IDX_Hj*rs + IDX_O2*cs] -= d;
  J[IDX_O2*rs + IDX_O2*cs] -= d;
  J[IDX_O2j*rs + IDX_O2*cs] += d;
  J[IDX_H*rs + IDX_O2*cs] += d;
  d = k[50]*n[IDX_E];
  J[IDX_O2j*rs + IDX_O2j*cs] -= d;
  J[IDX_E*rs + IDX_O2j*cs] -= d;
  J[IDX_O*rs + IDX_O2j*cs] += d;
  J[IDX_O*rs + IDX_O2j*cs] += d;
  d = k[50]*n[IDX_O2j];
  J[IDX_O2j*rs + IDX_E*cs] -= d;
  J[IDX_E*rs + IDX_E*cs] -= d;
  J[IDX_O*rs + IDX_E*cs] += d;
  J[IDX_O*rs + IDX_E*cs] += d;
  d = k[51]*n[IDX_O];
  J[IDX_O*rs + IDX_CH*cs] -= d;
  J[IDX_CH*rs + IDX_CH*cs] -= d;
  J[IDX_CO*rs + IDX_CH*cs] += d;
  J[IDX_H*rs + IDX_CH*cs] += d;
  d = k[51]*n[IDX_CH];
  J[IDX_O*rs + IDX_O*cs] -= d;
  J[IDX_CH*rs + IDX_O*cs] -= d;
  J[IDX_CO*rs + IDX_O*cs] += d;
  J[IDX_H*rs + IDX_O*cs] += d;
  d = k[52]*n[IDX_OH];
  J[IDX_C*rs + IDX_C*cs] -= d;
  J[IDX_OH*rs + IDX_C*cs] -= d;
  J[IDX_CO*rs + IDX_C*cs] += d;
  J[IDX_H*rs + IDX_C*cs] += d;
  d = k[52]*n[IDX_C];
  J[IDX_C*rs + IDX_OH*cs] -= d;
  J[IDX_OH*rs + IDX_OH*cs] -= d;
  J[IDX_CO*rs + IDX_OH*cs] += d;
  J[IDX_H*rs + IDX_OH*cs] += d;
  d = k[53]*n[IDX_O2];
  J[IDX_C*rs + IDX_C*cs] -= d;
  J[IDX_O2*rs + IDX_C*cs] -= d;
  J[IDX_CO*rs + IDX_C*cs] += d;
  J[IDX_O*rs + IDX_C*cs] += d;
  d = k[53]*n[IDX_C];
  J[IDX_C*rs + IDX_O2*cs] -= d;
  J[IDX_O2*rs + IDX_O2*cs] -= d;
  J[IDX_CO*rs + IDX_O2*cs] += d;
  J[IDX_O*rs + IDX_O2*cs] += d;
  d = k[54]*n[IDX_O2];
  J[IDX_Cj*rs + IDX_Cj*cs] -= d;
  J[IDX_O2*rs + IDX_Cj*cs] -= d;
  J[IDX_Oj*rs + IDX_Cj*cs] += d;
  J[IDX_CO*rs + IDX_Cj*cs] += d;
  d = k[54]*n[IDX_Cj];
  J[IDX_Cj*rs + IDX_O2*cs] -= d;
  J[IDX_O2*rs + IDX_O2*cs] -= d;
  J[IDX_Oj*rs + IDX_O2*cs] += d;
  J[IDX_CO*rs + IDX_O2*cs] += d;
  d = k[55]*n[IDX_OH];
  J[IDX_OH*rs + IDX_CO*cs] -= d;
  J[IDX_CO*rs + IDX_CO*cs] -= d;
  J[IDX_CO2*rs + IDX_CO*cs] += d;
  J[IDX_H*rs + IDX_CO*cs] += d;
  d = k[55]*n[IDX_CO];
  J[IDX_OH*rs + IDX_OH*cs] -= d;
  J[IDX_CO*rs + IDX_OH*cs] -= d;
  J[IDX_CO2*rs + IDX_OH*cs] += d;
  J[IDX_H*rs + IDX_OH*cs] += d;
  d = k[56]*n[IDX_E];
  J[IDX_Cj*rs + IDX_Cj*cs] -= d;
  J[IDX_E*rs + IDX_Cj*cs] -= d;
  J[IDX_C*rs + IDX_Cj*cs] += d;
  d = k[56]*n[IDX_Cj];
  J[IDX_Cj*rs + IDX_E*cs] -= d;
  J[IDX_E*rs + IDX_E*cs] -= d;
  J[IDX_C*rs + IDX_E*cs] += d;
  d = k[57]*n[IDX_OH];
  J[IDX_Cj*rs + IDX_Cj*cs] -= d;
  J[IDX_OH*rs + IDX_Cj*cs] -= d;
  J[IDX_COj*rs + IDX_Cj*cs] += d;
  J[IDX_H*rs + IDX_Cj*cs] += d;
  d = k[57]*n[IDX_Cj];
  J[IDX_Cj*rs + IDX_OH*cs] -= d;
  J[IDX_OH*rs + IDX_OH*cs] -= d;
  J[IDX_COj*rs + IDX_OH*cs] += d;
  J[IDX_H*rs + IDX_OH*cs] += d;
  d = k[58]*n[IDX_H];
  J[IDX_COj*rs + IDX_COj*cs] -= d;
  J[IDX_H*rs + IDX_COj*cs] -= d;
  J[IDX_Hj*rs + IDX_COj*cs] += d;
  J[IDX_CO*rs + IDX_COj*cs] += d;
  d = k[58]*n[IDX_COj];
  J[IDX_COj*rs + IDX_H*cs] -= d;
  J[IDX_H*rs + IDX_H*cs] -= d;
  J[IDX_Hj*rs + IDX_H*cs] += d;
  J[IDX_CO*rs + IDX_H*cs] += d;
  d = k[59]*n[IDX_H];
  J[IDX_C*rs + IDX_C*cs] -= d;
  J[IDX_H*rs + IDX_C*cs] -= d;
  J[IDX_CH*rs + IDX_C*cs] += d;
  d = k[59]*n[IDX_C];
  J[IDX_C*rs + IDX_H*cs] -= d;
  J[IDX_H*rs + IDX_H*cs] -= d;
  J[IDX_CH*rs + IDX_H*cs] += d;
  d = k[60]*n[IDX_H2];
  J[IDX_C*rs + IDX_C*cs] -= d;
  J[IDX_H2*rs + IDX_C*cs] -= d;
  J[IDX_CH*rs + IDX_C*cs] += d;
  J[IDX_H*rs + IDX_C*cs] += d;
  d = k[60]*n[IDX_C];
  J[IDX_C*rs + IDX_H2*cs] -= d;
  J[IDX_H2*rs + IDX_H2*cs] -= d;
  J[IDX_CH*rs + IDX_H2*cs] += d;
  J[IDX_H*rs + IDX_H2*cs] += d;
  d = k[61]*n[IDX_H];
  J[IDX_H*rs + IDX_CH*cs] -= d;
  J[IDX_CH*rs + IDX_CH*cs] -= d;
  J[IDX_C*rs + IDX_CH*cs] += d;
  J[IDX_H2*rs + IDX_CH*cs] += d;
  d = k[61]*n[IDX_CH];
  J[IDX_H*rs + IDX_H*cs] -= d;
  J[IDX_CH*rs + IDX_H*cs] -= d;
  J[IDX_C*rs + IDX_H*cs] += d;
  J[IDX_H2*rs + IDX_H*cs] += d;
  d = k[62]*n[IDX_H2];
  J[IDX_H2*rs + IDX_CH*cs] -= d;
  J[IDX_CH*rs + IDX_CH*cs] -= d;
  J[IDX_CH2*rs + IDX_CH*cs] += d;
  J[IDX_H*rs + IDX_CH*cs] += d;
  d = k[62]*n[IDX_CH];
  J[IDX_H2*rs + IDX_H2*cs] -= d;
  J[IDX_CH*rs + IDX_H2*cs] -= d;
  J[IDX_CH2*rs + IDX_H2*cs] += d;
  J[IDX_H*rs + IDX_H2*cs] += d;
  d = k[63]*n[IDX_H];
  J[IDX_H*rs + IDX_CH2*cs] -= d;
  J[IDX_CH2*rs + IDX_CH2*cs] -= d;
  J[IDX_CH*rs + IDX_CH2*cs] += d;
  J[IDX_H2*rs + IDX_CH2*cs] += d;
  d = k[63]*n[IDX_CH2];
  J[IDX_H*rs + IDX_H*cs] -= d;
  J[IDX_CH2*rs + IDX_H*cs] -= d;
  J[IDX_CH*rs + IDX_H*cs] += d;
  J[IDX_H2*rs + IDX_H*cs] += d;
  d = k[64]*n[IDX_H2];
  J[IDX_H2*rs + IDX_CH2*cs] -= d;
  J[IDX_CH2*rs + IDX_CH2*cs] -= d;
  J[IDX_CH3*rs + IDX_CH2*cs] += d;
  J[IDX_H*rs + IDX_CH2*cs] += d;
  d = k[64]*n[IDX_CH2];
  J[IDX_H2*rs + IDX_H2*cs] -= d;
  J[IDX_CH2*rs + IDX_H2*cs] -= d;
  J[IDX_CH3*rs + IDX_H2*cs] += d;
  J[IDX_H*rs + IDX_H2*cs] += d;
  d = k[65]*n[IDX_H];
  J[IDX_H*rs + IDX_CH3*cs] -= d;
  J[IDX_CH3*rs + IDX_CH3*cs] -= d;
  J[IDX_CH2*rs + IDX_CH3*cs] += d;
  J[IDX_H2*rs + IDX_CH3*cs] += d;
  d = k[65]*n[IDX_CH3];
  J[IDX_H*rs + IDX_H*cs] -= d;
  J[IDX_CH3*rs + IDX_H*cs] -= d;
  J[IDX_CH2*rs + IDX_H*cs] += d;
  J[IDX_H2*rs + IDX_H*cs] += d;
  d = k[66]*n[IDX_H2];
  J[IDX_H2*rs + IDX_CH3*cs] -= d;
  J[IDX_CH3*rs + IDX_CH3*cs] -= d;
  J[IDX_CH4*rs + IDX_CH3*cs] += d;
  J[IDX_H*rs + IDX_CH3*cs] += d;
  d = k[66]*n[IDX_CH3];
  J[IDX_H2*rs + IDX_H2*cs] -= d;
  J[IDX_CH3*rs + IDX_H2*cs] -= d;
  J[IDX_CH4*rs + IDX_H2*cs] += d;
  J[IDX_H*rs + IDX_H2*cs] += d;
  d = k[67]*n[IDX_H];
  J[IDX_H*rs + IDX_CH4*cs] -= d;
  J[IDX_CH4*rs + IDX_CH4*cs] -= d;
  J[IDX_H2*rs + IDX_CH4*cs] += d;
  J[IDX_CH3*rs + IDX_CH4*cs] += d;
  d = k[67]*n[IDX_CH4];
  J[IDX_H*rs + IDX_H*cs] -= d;
  J[IDX_CH4*rs + IDX_H*cs] -= d;
  J[IDX_H2*rs + IDX_H*cs] += d;
  J[IDX_CH3*rs + IDX_H*cs] += d;
  d = k[68]*n[IDX_H2];
  J[IDX_H2*rs + IDX_C*cs] -= d;
  J[IDX_C*rs + IDX_C*cs] -= d;
  J[IDX_CH2*rs + IDX_C*cs] += d;
  d = k[68]*n[IDX_C];
  J[IDX_H2*rs + IDX_H2*cs] -= d;
  J[IDX_C*rs + IDX_H2*cs] -= d;
  J[IDX_CH2*rs + IDX_H2*cs] += d;
  d = k[69]*n[IDX_E];
  J[IDX_H3Oj*rs + IDX_H3Oj*cs] -= d;
  J[IDX_E*rs + IDX_H3Oj*cs] -= d;
  J[IDX_OH*rs + IDX_H3Oj*cs] += d;
  J[IDX_H*rs + IDX_H3Oj*cs] += d;
  J[IDX_H*rs + IDX_H3Oj*cs] += d;
  d = k[69]*n[IDX_H3Oj];
  J[IDX_H3Oj*rs + IDX_E*cs] -= d;
  J[IDX_E*rs + IDX_E*cs] -= d;
  J[IDX_OH*rs + IDX_E*cs] += d;
  J[IDX_H*rs + IDX_E*cs] += d;
  J[IDX_H*rs + IDX_E*cs] += d;
  d = k[70]*n[IDX_E];
  J[IDX_OHj*rs + IDX_OHj*cs] -= d;
  J[IDX_E*rs + IDX_OHj*cs] -= d;
  J[IDX_O*rs + IDX_OHj*cs] += d;
  J[IDX_H*rs + IDX_OHj*cs] += d;
  d = k[70]*n[IDX_OHj];
  J[IDX_OHj*rs + IDX_E*cs] -= d;
  J[IDX_E*rs + IDX_E*cs] -= d;
  J[IDX_O*rs + IDX_E*cs] += d;
  J[IDX_H*rs + IDX_E*cs] += d;
  d = k[71]*n[IDX_E];
  J[IDX_Oj*rs + IDX_Oj*cs] -= d;
  J[IDX_E*rs + IDX_Oj*cs] -= d;
  J[IDX_O*rs + IDX_Oj*cs] += d;
  d = k[71]*n[IDX_Oj];
  J[IDX_Oj*rs + IDX_E*cs] -= d;
  J[IDX_E*rs + IDX_E*cs] -= d;
  J[IDX_O*rs + IDX_E*cs] += d;
  d = k[72]*n[IDX_E];
  J[IDX_COj*rs + IDX_COj*cs] -= d;
  J[IDX_E*rs + IDX_COj*cs] -= d;
  J[IDX_CO*rs + IDX_COj*cs] += d;
  d = k[72]*n[IDX_COj];
  J[IDX_COj*rs + IDX_E*cs] -= d;
  J[IDX_E*rs + IDX_E*cs] -= d;
  J[IDX_CO*rs + IDX_E*cs] += d;
  d = k[73]*n[IDX_E];
  J[IDX_COj*rs + IDX_COj*cs] -= d;
  J[IDX_E*rs + IDX_COj*cs] -= d;
  J[IDX_C*rs + IDX_COj*cs] += d;
  J[IDX_O*rs + IDX_COj*cs] += d;
  d = k[73]*n[IDX_COj];
  J[IDX_COj*rs + IDX_E*cs] -= d;
  J[IDX_E*rs + IDX_E*cs] -= d;
  J[IDX_C*rs + IDX_E*cs] += d;
  J[IDX_O*rs + IDX_E*cs] += d;
}

// H2 + H -> H + H + H
KB_HD inline double rate_16(double Tgas, const double* n, const Params& p, double Tg_) {
  (void)Tgas; (void)n; (void)p; (void)Tg_;
  return dissH2_Martin96(Tgas, n, p);
}
// the rate-derivative part of the analytic Jacobian (J[i*jrs_ + j*cs], added to;
// U[NSPEC][NAGG] written), gated and clamped like the rates
KB_HD inline void jac_dk(double Tgas, const double* n, const Params& p, const double* k, double* J, double* U, long jrs_, long jcs_) {
  (void)Tgas; (void)n; (void)p; (void)k; (void)J; (void)jrs_; (void)jcs_;
  for (int i = 0; i < NSPEC * NAGG; ++i) U[i] = 0.0;
  double d;
  (void)d;
  { // numerical dk/dn: H2 + H -> H + H + H (extern/table in rate, all species)
    double np_[NSPEC];
    for (int q = 0; q < NSPEC; ++q) np_[q] = n[q];
    auto rf_ = [&](const double* x) { return rate_16(Tgas, x, p, Tgas); };
    const double pr_ = n[IDX_H]*n[IDX_H2];
    for (int jj = 0; jj < NSPEC; ++jj) {
      const double dk_ = fd_dk_(rf_, np_, n, k[16], jj);
      if (dk_ == 0.0) continue;
      d = dk_ * pr_;
      J[IDX_H2*jrs_ + jj*jcs_] -= d;
      J[IDX_H*jrs_ + jj*jcs_] -= d;
      J[IDX_H*jrs_ + jj*jcs_] += d;
      J[IDX_H*jrs_ + jj*jcs_] += d;
      J[IDX_H*jrs_ + jj*jcs_] += d;
    }
  }
  d = (dpow_(v_kh21(Tgas, n, p), 1.0 - v_a21(Tgas, n, p), (8.125e-08 * dpow_(v_T(Tgas, n, p), -0.5, 0.0, -0.0) * kb_exp(-52000.0 * v_invT(Tgas, n, p)) + 8.125e-08 * 1.0/(std::sqrt(v_T(Tgas, n, p))) * kb_exp(-52000.0 * v_invT(Tgas, n, p)) * -0.0 * v_invT(Tgas, n, p)) * (1.0 - kb_exp(-6000.0 * v_invT(Tgas, n, p))) + 8.125e-08 * 1.0/(std::sqrt(v_T(Tgas, n, p))) * kb_exp(-52000.0 * v_invT(Tgas, n, p)) * -(kb_exp(-6000.0 * v_invT(Tgas, n, p)) * -0.0 * v_invT(Tgas, n, p)), -(-(1.0 / v_ncr21(Tgas, n, p) / ((1.0 + Hnuclei_(n) / v_ncr21(Tgas, n, p)) * (1.0 + Hnuclei_(n) / v_ncr21(Tgas, n, p)))))) * kb_pow(v_kl21(Tgas, n, p), v_a21(Tgas, n, p)) + kb_pow(v_kh21(Tgas, n, p), 1.0 - v_a21(Tgas, n, p)) * dpow_(v_kl21(Tgas, n, p), v_a21(Tgas, n, p), 1.18e-10 * kb_exp(-69500.0 * v_invT(Tgas, n, p)) * -0.0 * v_invT(Tgas, n, p), -(1.0 / v_ncr21(Tgas, n, p) / ((1.0 + Hnuclei_(n) / v_ncr21(Tgas, n, p)) * (1.0 + Hnuclei_(n) / v_ncr21(Tgas, n, p))))))*n[IDX_H2]*n[IDX_H2];  // dk of H2 + H2 -> H + H + H2 wrt Hnuclei
  U[IDX_H2*NAGG + 1] -= d;
  U[IDX_H2*NAGG + 1] -= d;
  U[IDX_H*NAGG + 1] += d;
  U[IDX_H*NAGG + 1] += d;
  U[IDX_H2*NAGG + 1] += d;
  d = ((ntot_(n) > 100000000000000.0 ? 0.0 : 0.0))*n[IDX_H]*n[IDX_Oj];  // dk of O+ + H -> H+ + O wrt ntot
  U[IDX_Oj*NAGG + 0] -= d;
  U[IDX_H*NAGG + 0] -= d;
  U[IDX_Hj*NAGG + 0] += d;
  U[IDX_O*NAGG + 0] += d;
  d = ((ntot_(n) > 100000000000000.0 ? 0.0 : 7e-10 * kb_exp(-232.0 * v_invT(Tgas, n, p)) * -0.0 * v_invT(Tgas, n, p)))*n[IDX_Hj]*n[IDX_O];  // dk of H+ + O -> O+ + H wrt ntot
  U[IDX_Hj*NAGG + 0] -= d;
  U[IDX_O*NAGG + 0] -= d;
  U[IDX_Oj*NAGG + 0] += d;
  U[IDX_H*NAGG + 0] += d;
  d = ((ntot_(n) > 100000000000000.0 ? 0.0 : 0.0))*n[IDX_H2]*n[IDX_Oj];  // dk of O+ + H2 -> OH+ + H wrt ntot
  U[IDX_Oj*NAGG + 0] -= d;
  U[IDX_H2*NAGG + 0] -= d;
  U[IDX_OHj*NAGG + 0] += d;
  U[IDX_H*NAGG + 0] += d;
  d = ((ntot_(n) > 100000000000000.0 ? 0.0 : 0.0))*n[IDX_H2]*n[IDX_OHj];  // dk of OH+ + H2 -> H2O+ + H wrt ntot
  U[IDX_OHj*NAGG + 0] -= d;
  U[IDX_H2*NAGG + 0] -= d;
  U[IDX_H2Oj*NAGG + 0] += d;
  U[IDX_H*NAGG + 0] += d;
  d = ((ntot_(n) > 100000000000000.0 ? 0.0 : 0.0))*n[IDX_H2]*n[IDX_H2Oj];  // dk of H2O+ + H2 -> H3O+ + H wrt ntot
  U[IDX_H2Oj*NAGG + 0] -= d;
  U[IDX_H2*NAGG + 0] -= d;
  U[IDX_H3Oj*NAGG + 0] += d;
  U[IDX_H*NAGG + 0] += d;
  d = ((ntot_(n) > 100000000000000.0 ? 0.0 : 2e-07 * dpow_(v_T32(Tgas, n, p), -0.5, 0.0, -0.0)))*n[IDX_H2Oj]*n[IDX_E];  // dk of H2O+ + e- -> O + H2 wrt ntot
  U[IDX_H2Oj*NAGG + 0] -= d;
  U[IDX_E*NAGG + 0] -= d;
  U[IDX_O*NAGG + 0] += d;
  U[IDX_H2*NAGG + 0] += d;
  d = ((ntot_(n) > 100000000000000.0 ? 0.0 : 1.6e-07 * dpow_(v_T32(Tgas, n, p), -0.5, 0.0, -0.0)))*n[IDX_H2Oj]*n[IDX_E];  // dk of H2O+ + e- -> OH + H wrt ntot
  U[IDX_H2Oj*NAGG + 0] -= d;
  U[IDX_E*NAGG + 0] -= d;
  U[IDX_OH*NAGG + 0] += d;
  U[IDX_H*NAGG + 0] += d;
  d = ((ntot_(n) > 100000000000000.0 ? 0.0 : 3.5e-07 * dpow_(v_T32(Tgas, n, p), -0.5, 0.0, -0.0)))*n[IDX_H3Oj]*n[IDX_E];  // dk of H3O+ + e- -> H2O + H wrt ntot
  U[IDX_H3Oj*NAGG + 0] -= d;
  U[IDX_E*NAGG + 0] -= d;
  U[IDX_H2O*NAGG + 0] += d;
  U[IDX_H*NAGG + 0] += d;
  d = ((ntot_(n) > 100000000000000.0 ? 0.0 : 9.9e-19 * dpow_(v_T32(Tgas, n, p), -0.38, 0.0, -0.0)))*n[IDX_H]*n[IDX_O];  // dk of O + H -> OH wrt ntot
  U[IDX_O*NAGG + 0] -= d;
  U[IDX_H*NAGG + 0] -= d;
  U[IDX_OH*NAGG + 0] += d;
  d = ((ntot_(n) > 100000000000000.0 ? 0.0 : 3.43e-13 * kb_pow(v_T32(Tgas, n, p), 2.67) * kb_exp(-3160.0 * v_invT(Tgas, n, p)) * -0.0 * v_invT(Tgas, n, p)))*n[IDX_H2]*n[IDX_O];  // dk of O + H2 -> OH + H wrt ntot
  U[IDX_O*NAGG + 0] -= d;
  U[IDX_H2*NAGG + 0] -= d;
  U[IDX_OH*NAGG + 0] += d;
  U[IDX_H*NAGG + 0] += d;
  d = ((ntot_(n) > 100000000000000.0 ? 0.0 : 1.55e-12 * kb_pow(v_T32(Tgas, n, p), 1.6) * kb_exp(-1660.0 * v_invT(Tgas, n, p)) * -0.0 * v_invT(Tgas, n, p)))*n[IDX_H2]*n[IDX_OH];  // dk of H2 + OH -> H2O + H wrt ntot
  U[IDX_H2*NAGG + 0] -= d;
  U[IDX_OH*NAGG + 0] -= d;
  U[IDX_H2O*NAGG + 0] += d;
  U[IDX_H*NAGG + 0] += d;
  d = ((ntot_(n) > 100000000000000.0 ? 0.0 : 1.65e-12 * kb_pow(v_T32(Tgas, n, p), 1.14) * kb_exp(-50.0 * v_invT(Tgas, n, p)) * -0.0 * v_invT(Tgas, n, p)))*n[IDX_OH]*n[IDX_OH];  // dk of OH + OH -> H2O + O wrt ntot
  U[IDX_OH*NAGG + 0] -= d;
  U[IDX_OH*NAGG + 0] -= d;
  U[IDX_H2O*NAGG + 0] += d;
  U[IDX_O*NAGG + 0] += d;
  d = ((ntot_(n) > 100000000000000.0 ? 0.0 : 0.0))*n[IDX_Hj]*n[IDX_OH];  // dk of H+ + OH -> OH+ + H wrt ntot
  U[IDX_Hj*NAGG + 0] -= d;
  U[IDX_OH*NAGG + 0] -= d;
  U[IDX_OHj*NAGG + 0] += d;
  U[IDX_H*NAGG + 0] += d;
  d = ((ntot_(n) > 100000000000000.0 ? 0.0 : 0.0))*n[IDX_Hj]*n[IDX_H2O];  // dk of H+ + H2O -> H2O+ + H wrt ntot
  U[IDX_Hj*NAGG + 0] -= d;
  U[IDX_H2O*NAGG + 0] -= d;
  U[IDX_H2Oj*NAGG + 0] += d;
  U[IDX_H*NAGG + 0] += d;
  d = ((ntot_(n) > 100000000000000.0 ? 0.0 : 7e-14 * kb_pow(v_T32(Tgas, n, p), 2.8) * kb_exp(-1950.0 * v_invT(Tgas, n, p)) * -0.0 * v_invT(Tgas, n, p)))*n[IDX_H]*n[IDX_OH];  // dk of H + OH -> H2 + O wrt ntot
  U[IDX_H*NAGG + 0] -= d;
  U[IDX_OH*NAGG + 0] -= d;
  U[IDX_H2*NAGG + 0] += d;
  U[IDX_O*NAGG + 0] += d;
  d = ((ntot_(n) > 100000000000000.0 ? 0.0 : 6.83e-12 * kb_pow(v_T32(Tgas, n, p), 1.6) * kb_exp(-9720.0 * v_invT(Tgas, n, p)) * -0.0 * v_invT(Tgas, n, p)))*n[IDX_H]*n[IDX_H2O];  // dk of H + H2O -> OH + H2 wrt ntot
  U[IDX_H*NAGG + 0] -= d;
  U[IDX_H2O*NAGG + 0] -= d;
  U[IDX_OH*NAGG + 0] += d;
  U[IDX_H2*NAGG + 0] += d;
  d = ((ntot_(n) > 100000000000000.0 ? 0.0 : 0.0))*n[IDX_O]*n[IDX_O];  // dk of O + O -> O2 wrt ntot
  U[IDX_O*NAGG + 0] -= d;
  U[IDX_O*NAGG + 0] -= d;
  U[IDX_O2*NAGG + 0] += d;
  d = ((ntot_(n) > 100000000000000.0 ? 0.0 : 4.34e-11 * dpow_(v_T32(Tgas, n, p), -0.5, 0.0, -0.0) * kb_exp(-30.0 * v_invT(Tgas, n, p)) + 4.34e-11 * 1.0/(std::sqrt(v_T32(Tgas, n, p))) * kb_exp(-30.0 * v_invT(Tgas, n, p)) * -0.0 * v_invT(Tgas, n, p)))*n[IDX_O]*n[IDX_OH];  // dk of O + OH -> O2 + H wrt ntot
  U[IDX_O*NAGG + 0] -= d;
  U[IDX_OH*NAGG + 0] -= d;
  U[IDX_O2*NAGG + 0] += d;
  U[IDX_H*NAGG + 0] += d;
  d = ((ntot_(n) > 100000000000000.0 ? 0.0 : 3.3e-10 * kb_exp(-8460.0 * v_invT(Tgas, n, p)) * -0.0 * v_invT(Tgas, n, p)))*n[IDX_H]*n[IDX_O2];  // dk of H + O2 -> OH + O wrt ntot
  U[IDX_H*NAGG + 0] -= d;
  U[IDX_O2*NAGG + 0] -= d;
  U[IDX_OH*NAGG + 0] += d;
  U[IDX_O*NAGG + 0] += d;
  d = ((ntot_(n) > 100000000000000.0 ? 0.0 : 0.0))*n[IDX_Hj]*n[IDX_O2];  // dk of H+ + O2 -> O2+ + H wrt ntot
  U[IDX_Hj*NAGG + 0] -= d;
  U[IDX_O2*NAGG + 0] -= d;
  U[IDX_O2j*NAGG + 0] += d;
  U[IDX_H*NAGG + 0] += d;
  d = ((ntot_(n) > 100000000000000.0 ? 0.0 : 1.95e-07 * dpow_(v_T32(Tgas, n, p), -0.7, 0.0, -0.0)))*n[IDX_O2j]*n[IDX_E];  // dk of O2+ + e- -> O + O wrt ntot
  U[IDX_O2j*NAGG + 0] -= d;
  U[IDX_E*NAGG + 0] -= d;
  U[IDX_O*NAGG + 0] += d;
  U[IDX_O*NAGG + 0] += d;
  d = ((ntot_(n) > 100000000000000.0 ? 0.0 : 0.0))*n[IDX_CH]*n[IDX_O];  // dk of O + CH -> CO + H wrt ntot
  U[IDX_O*NAGG + 0] -= d;
  U[IDX_CH*NAGG + 0] -= d;
  U[IDX_CO*NAGG + 0] += d;
  U[IDX_H*NAGG + 0] += d;
  d = ((ntot_(n) > 100000000000000.0 ? 0.0 : 0.0))*n[IDX_C]*n[IDX_OH];  // dk of C + OH -> CO + H wrt ntot
  U[IDX_C*NAGG + 0] -= d;
  U[IDX_OH*NAGG + 0] -= d;
  U[IDX_CO*NAGG + 0] += d;
  U[IDX_H*NAGG + 0] += d;
  d = ((ntot_(n) > 100000000000000.0 ? 0.0 : 0.0))*n[IDX_C]*n[IDX_O2];  // dk of C + O2 -> CO + O wrt ntot
  U[IDX_C*NAGG + 0] -= d;
  U[IDX_O2*NAGG + 0] -= d;
  U[IDX_CO*NAGG + 0] += d;
  U[IDX_O*NAGG + 0] += d;
  d = ((ntot_(n) > 100000000000000.0 ? 0.0 : 0.0))*n[IDX_Cj]*n[IDX_O2];  // dk of C+ + O2 -> O+ + CO wrt ntot
  U[IDX_Cj*NAGG + 0] -= d;
  U[IDX_O2*NAGG + 0] -= d;
  U[IDX_Oj*NAGG + 0] += d;
  U[IDX_CO*NAGG + 0] += d;
  d = ((ntot_(n) > 100000000000000.0 ? 0.0 : 0.0))*n[IDX_CO]*n[IDX_OH];  // dk of OH + CO -> CO2 + H wrt ntot
  U[IDX_OH*NAGG + 0] -= d;
  U[IDX_CO*NAGG + 0] -= d;
  U[IDX_CO2*NAGG + 0] += d;
  U[IDX_H*NAGG + 0] += d;
  d = ((ntot_(n) > 100000000000000.0 ? 0.0 : 4.4e-12 * dpow_(v_T32(Tgas, n, p), -0.61, 0.0, -0.0)))*n[IDX_Cj]*n[IDX_E];  // dk of C+ + e- -> C wrt ntot
  U[IDX_Cj*NAGG + 0] -= d;
  U[IDX_E*NAGG + 0] -= d;
  U[IDX_C*NAGG + 0] += d;
  d = ((ntot_(n) > 100000000000000.0 ? 0.0 : 0.0))*n[IDX_Cj]*n[IDX_OH];  // dk of C+ + OH -> CO+ + H wrt ntot
  U[IDX_Cj*NAGG + 0] -= d;
  U[IDX_OH*NAGG + 0] -= d;
  U[IDX_COj*NAGG + 0] += d;
  U[IDX_H*NAGG + 0] += d;
  d = ((ntot_(n) > 100000000000000.0 ? 0.0 : 0.0))*n[IDX_COj]*n[IDX_H];  // dk of CO+ + H -> H+ + CO wrt ntot
  U[IDX_COj*NAGG + 0] -= d;
  U[IDX_H*NAGG + 0] -= d;
  U[IDX_Hj*NAGG + 0] += d;
  U[IDX_CO*NAGG + 0] += d;
  d = ((ntot_(n) > 100000000000000.0 ? 0.0 : 0.0))*n[IDX_C]*n[IDX_H];  // dk of C + H -> CH wrt ntot
  U[IDX_C*NAGG + 0] -= d;
  U[IDX_H*NAGG + 0] -= d;
  U[IDX_CH*NAGG + 0] += d;
  d = ((ntot_(n) > 100000000000000.0 ? 0.0 : 6.64e-10 * kb_exp(-11700.0 * v_invT(Tgas, n, p)) * -0.0 * v_invT(Tgas, n, p)))*n[IDX_C]*n[IDX_H2];  // dk of C + H2 -> CH + H wrt ntot
  U[IDX_C*NAGG + 0] -= d;
  U[IDX_H2*NAGG + 0] -= d;
  U[IDX_CH*NAGG + 0] += d;
  U[IDX_H*NAGG + 0] += d;
  d = ((ntot_(n) > 100000000000000.0 ? 0.0 : 0.0))*n[IDX_CH]*n[IDX_H];  // dk of H + CH -> C + H2 wrt ntot
  U[IDX_H*NAGG + 0] -= d;
  U[IDX_CH*NAGG + 0] -= d;
  U[IDX_C*NAGG + 0] += d;
  U[IDX_H2*NAGG + 0] += d;
  d = ((ntot_(n) > 100000000000000.0 ? 0.0 : 2.38e-10 * kb_exp(-1760.0 * v_invT(Tgas, n, p)) * -0.0 * v_invT(Tgas, n, p)))*n[IDX_CH]*n[IDX_H2];  // dk of H2 + CH -> CH2 + H wrt ntot
  U[IDX_H2*NAGG + 0] -= d;
  U[IDX_CH*NAGG + 0] -= d;
  U[IDX_CH2*NAGG + 0] += d;
  U[IDX_H*NAGG + 0] += d;
  d = ((ntot_(n) > 100000000000000.0 ? 0.0 : 0.0))*n[IDX_CH2]*n[IDX_H];  // dk of H + CH2 -> CH + H2 wrt ntot
  U[IDX_H*NAGG + 0] -= d;
  U[IDX_CH2*NAGG + 0] -= d;
  U[IDX_CH*NAGG + 0] += d;
  U[IDX_H2*NAGG + 0] += d;
  d = ((ntot_(n) > 100000000000000.0 ? 0.0 : 5.18e-11 * kb_pow(v_T32(Tgas, n, p), 0.17) * kb_exp(-6400.0 * v_invT(Tgas, n, p)) * -0.0 * v_invT(Tgas, n, p)))*n[IDX_CH2]*n[IDX_H2];  // dk of H2 + CH2 -> CH3 + H wrt ntot
  U[IDX_H2*NAGG + 0] -= d;
  U[IDX_CH2*NAGG + 0] -= d;
  U[IDX_CH3*NAGG + 0] += d;
  U[IDX_H*NAGG + 0] += d;
  d = ((ntot_(n) > 100000000000000.0 ? 0.0 : 1e-10 * kb_exp(-7600.0 * v_invT(Tgas, n, p)) * -0.0 * v_invT(Tgas, n, p)))*n[IDX_CH3]*n[IDX_H];  // dk of H + CH3 -> CH2 + H2 wrt ntot
  U[IDX_H*NAGG + 0] -= d;
  U[IDX_CH3*NAGG + 0] -= d;
  U[IDX_CH2*NAGG + 0] += d;
  U[IDX_H2*NAGG + 0] += d;
  d = ((ntot_(n) > 100000000000000.0 ? 0.0 : 6.86e-14 * kb_pow(v_T32(Tgas, n, p), 2.74) * kb_exp(-4740.0 * v_invT(Tgas, n, p)) * -0.0 * v_invT(Tgas, n, p)))*n[IDX_CH3]*n[IDX_H2];  // dk of H2 + CH3 -> CH4 + H wrt ntot
  U[IDX_H2*NAGG + 0] -= d;
  U[IDX_CH3*NAGG + 0] -= d;
  U[IDX_CH4*NAGG + 0] += d;
  U[IDX_H*NAGG + 0] += d;
  d = ((ntot_(n) > 100000000000000.0 ? 0.0 : 5.82e-13 * v_T32(Tgas, n, p)*v_T32(Tgas, n, p)*v_T32(Tgas, n, p) * kb_exp(-4045.0 * v_invT(Tgas, n, p)) * -0.0 * v_invT(Tgas, n, p)))*n[IDX_CH4]*n[IDX_H];  // dk of H + CH4 -> H2 + CH3 wrt ntot
  U[IDX_H*NAGG + 0] -= d;
  U[IDX_CH4*NAGG + 0] -= d;
  U[IDX_H2*NAGG + 0] += d;
  U[IDX_CH3*NAGG + 0] += d;
  d = ((ntot_(n) > 100000000000000.0 ? 0.0 : 0.0))*n[IDX_C]*n[IDX_H2];  // dk of H2 + C -> CH2 wrt ntot
  U[IDX_H2*NAGG + 0] -= d;
  U[IDX_C*NAGG + 0] -= d;
  U[IDX_CH2*NAGG + 0] += d;
  d = ((ntot_(n) > 100000000000000.0 ? 0.0 : 6.5e-07 * dpow_(v_T32(Tgas, n, p), -0.5, 0.0, -0.0)))*n[IDX_H3Oj]*n[IDX_E];  // dk of H3O+ + e- -> OH + H + H wrt ntot
  U[IDX_H3Oj*NAGG + 0] -= d;
  U[IDX_E*NAGG + 0] -= d;
  U[IDX_OH*NAGG + 0] += d;
  U[IDX_H*NAGG + 0] += d;
  U[IDX_H*NAGG + 0] += d;
  d = ((ntot_(n) > 100000000000000.0 ? 0.0 : 6.3e-09 * dpow_(v_T32(Tgas, n, p), -0.48, 0.0, -0.0)))*n[IDX_OHj]*n[IDX_E];  // dk of OH+ + e- -> O + H wrt ntot
  U[IDX_OHj*NAGG + 0] -= d;
  U[IDX_E*NAGG + 0] -= d;
  U[IDX_O*NAGG + 0] += d;
  U[IDX_H*NAGG + 0] += d;
  {  // group 1: H+ + e- -> H
    double T = Tgas;
    if (T < 5500.0) {
    }
    else if (T >= 5500.0) {
    }
  }
  {  // group 2: He+ + e- -> He
    double T = Tgas;
    if (T < 9280.0) {
    }
    else if (T >= 9280.0) {
    }
  }
  {  // group 3: H + H+ -> H2+
    double T = Tgas;
    if (T < 30.0) {
    }
    else if (T >= 30.0) {
    }
  }
  {  // group 4: H2 + H+ -> H2+ + H
    double T = Tgas;
    if (T > 30000.0) T = 30000.0;
    if (T >= 100.0 && T >= 100.0) {
    }
  }
  {  // group 5: H- + H -> H + H + e-
    double T = Tgas;
    if (T < 1160.0) {
    }
    else if (T >= 1160.0) {
    }
  }
  {  // group 6: He + H+ -> He+ + H
    double T = Tgas;
    if (T < 10000.0) {
    }
    else if (T >= 10000.0) {
    }
  }
}

KB_HD inline double gamma_index(double Tgas, const double* n, const Params& p) {
  (void)Tgas; (void)n;
  return p.gamma_ad;
}
// dTgas/dt at the thermal temperature T (capped to [2.73, 1e9] K by
// the caller) with the rates k of the rate temperature
KB_HD inline double thermal_dTdt(double T, const double* n, const double* k, const Params& p) {
  (void)k; (void)p;
  double heat = 0.0, cool = 0.0;
  return (gamma_index(T, n, p) - 1.0) * (heat - cool)
      / (kbc::boltzmann_erg * ntot_(n));
}
// the cooling's temperature-only parts at one T (a row of density
// derivatives at that T evaluates them once): thermal_dTdt_with of
// thermal_pre(T) equals thermal_dTdt bit for bit
struct ThermalPre {
  int unused_;
};
KB_HD inline void thermal_pre(double T, const double* n, const Params& p, ThermalPre& q) {
  (void)T; (void)n; (void)p; (void)q;
}
KB_HD inline double thermal_dTdt_with(const ThermalPre& q, double T, const double* n, const double* k, const Params& p) {
  (void)q; (void)k; (void)p;
  double heat = 0.0, cool = 0.0;
  return (gamma_index(T, n, p) - 1.0) * (heat - cool)
      / (kbc::boltzmann_erg * ntot_(n));
}

// g[r] += sum_i mu_i d f_i / d ln k_r at the state n with the rates k;
// muT: mu of the Tgas row (0 without it), Tth the thermal temperature
KB_HD inline void lnk_vjp(const double* n, const double* k, double Tth, const Params& p, const double* mu, double muT, double* g) {
  (void)Tth; (void)p; (void)muT;
  double flux;
  (void)flux;
  flux = k[0]*n[IDX_H]*n[IDX_E];
  g[0] += flux * (mu[IDX_Hj] + mu[IDX_E] + mu[IDX_E] - mu[IDX_H] - mu[IDX_E]);
  flux = k[1]*n[IDX_Hj]*n[IDX_E];
  g[1] += flux * (mu[IDX_H] - mu[IDX_Hj] - mu[IDX_E]);
  flux = k[2]*n[IDX_Hj]*n[IDX_E];
  g[2] += flux * (mu[IDX_H] - mu[IDX_Hj] - mu[IDX_E]);
  flux = k[3]*n[IDX_He]*n[IDX_E];
  g[3] += flux * (mu[IDX_Hej] + mu[IDX_E] + mu[IDX_E] - mu[IDX_He] - mu[IDX_E]);
  flux = k[4]*n[IDX_Hej]*n[IDX_E];
  g[4] += flux * (mu[IDX_He] - mu[IDX_Hej] - mu[IDX_E]);
  flux = k[5]*n[IDX_Hej]*n[IDX_E];
  g[5] += flux * (mu[IDX_He] - mu[IDX_Hej] - mu[IDX_E]);
  flux = k[6]*n[IDX_Hej]*n[IDX_E];
  g[6] += flux * (mu[IDX_Hejj] + mu[IDX_E] + mu[IDX_E] - mu[IDX_Hej] - mu[IDX_E]);
  flux = k[7]*n[IDX_Hejj]*n[IDX_E];
  g[7] += flux * (mu[IDX_Hej] - mu[IDX_Hejj] - mu[IDX_E]);
  flux = k[8]*n[IDX_H]*n[IDX_E];
  g[8] += flux * (mu[IDX_Hk] - mu[IDX_H] - mu[IDX_E]);
  flux = k[9]*n[IDX_Hk]*n[IDX_H];
  g[9] += flux * (mu[IDX_H2] + mu[IDX_E] - mu[IDX_Hk] - mu[IDX_H]);
  flux = k[10]*n[IDX_H]*n[IDX_Hj];
  g[10] += flux * (mu[IDX_H2j] - mu[IDX_H] - mu[IDX_Hj]);
  flux = k[11]*n[IDX_H]*n[IDX_Hj];
  g[11] += flux * (mu[IDX_H2j] - mu[IDX_H] - mu[IDX_Hj]);
  flux = k[12]*n[IDX_H2j]*n[IDX_H];
  g[12] += flux * (mu[IDX_H2] + mu[IDX_Hj] - mu[IDX_H2j] - mu[IDX_H]);
  flux = k[13]*n[IDX_H2]*n[IDX_Hj];
  g[13] += flux * (mu[IDX_H2j] + mu[IDX_H] - mu[IDX_H2] - mu[IDX_Hj]);
  flux = k[14]*n[IDX_H2]*n[IDX_E];
  g[14] += flux * (mu[IDX_H] + mu[IDX_Hk] - mu[IDX_H2] - mu[IDX_E]);
  flux = k[15]*n[IDX_H2]*n[IDX_E];
  g[15] += flux * (mu[IDX_H] + mu[IDX_H] + mu[IDX_E] - mu[IDX_H2] - mu[IDX_E]);
  flux = k[16]*n[IDX_H2]*n[IDX_H];
  g[16] += flux * (mu[IDX_H] + mu[IDX_H] + mu[IDX_H] - mu[IDX_H2] - mu[IDX_H]);
  flux = k[17]*n[IDX_Hk]*n[IDX_E];
  g[17] += flux * (mu[IDX_H] + mu[IDX_E] + mu[IDX_E] - mu[IDX_Hk] - mu[IDX_E]);
  flux = k[18]*n[IDX_Hk]*n[IDX_H];
  g[18] += flux * (mu[IDX_H] + mu[IDX_H] + mu[IDX_E] - mu[IDX_Hk] - mu[IDX_H]);
  flux = k[19]*n[IDX_Hk]*n[IDX_H];
  g[19] += flux * (mu[IDX_H] + mu[IDX_H] + mu[IDX_E] - mu[IDX_Hk] - mu[IDX_H]);
  flux = k[20]*n[IDX_Hk]*n[IDX_Hj];
  g[20] += flux * (mu[IDX_H] + mu[IDX_H] - mu[IDX_Hk] - mu[IDX_Hj]);
  flux = k[21]*n[IDX_Hk]*n[IDX_Hj];
  g[21] += flux * (mu[IDX_H2j] + mu[IDX_E] - mu[IDX_Hk] - mu[IDX_Hj]);
  flux = k[22]*n[IDX_H2j]*n[IDX_E];
  g[22] += flux * (mu[IDX_H] + mu[IDX_H] - mu[IDX_H2j] - mu[IDX_E]);
  flux = k[23]*n[IDX_H2j]*n[IDX_Hk];
  g[23] += flux * (mu[IDX_H] + mu[IDX_H2] - mu[IDX_H2j] - mu[IDX_Hk]);
  flux = k[24]*n[IDX_H]*n[IDX_H]*n[IDX_H];
  g[24] += flux * (mu[IDX_H2] + mu[IDX_H] - mu[IDX_H] - mu[IDX_H] - mu[IDX_H]);
  flux = k[25]*n[IDX_H2]*n[IDX_H]*n[IDX_H];
  g[25] += flux * (mu[IDX_H2] + mu[IDX_H2] - mu[IDX_H2] - mu[IDX_H] - mu[IDX_H]);
  flux = k[26]*n[IDX_H2]*n[IDX_H2];
  g[26] += flux * (mu[IDX_H] + mu[IDX_H] + mu[IDX_H2] - mu[IDX_H2] - mu[IDX_H2]);
  flux = k[27]*n[IDX_Hej]*n[IDX_H];
  g[27] += flux * (mu[IDX_He] + mu[IDX_Hj] - mu[IDX_Hej] - mu[IDX_H]);
  flux = k[28]*n[IDX_He]*n[IDX_Hj];
  g[28] += flux * (mu[IDX_Hej] + mu[IDX_H] - mu[IDX_He] - mu[IDX_Hj]);
  flux = k[29]*n[IDX_He]*n[IDX_Hj];
  g[29] += flux * (mu[IDX_Hej] + mu[IDX_H] - mu[IDX_He] - mu[IDX_Hj]);
  flux = k[30]*n[IDX_Oj]*n[IDX_H];
  g[30] += flux * (mu[IDX_Hj] + mu[IDX_O] - mu[IDX_Oj] - mu[IDX_H]);
  flux = k[31]*n[IDX_Hj]*n[IDX_O];
  g[31] += flux * (mu[IDX_Oj] + mu[IDX_H] - mu[IDX_Hj] - mu[IDX_O]);
  flux = k[32]*n[IDX_Oj]*n[IDX_H2];
  g[32] += flux * (mu[IDX_OHj] + mu[IDX_H] - mu[IDX_Oj] - mu[IDX_H2]);
  flux = k[33]*n[IDX_OHj]*n[IDX_H2];
  g[33] += flux * (mu[IDX_H2Oj] + mu[IDX_H] - mu[IDX_OHj] - mu[IDX_H2]);
  flux = k[34]*n[IDX_H2Oj]*n[IDX_H2];
  g[34] += flux * (mu[IDX_H3Oj] + mu[IDX_H] - mu[IDX_H2Oj] - mu[IDX_H2]);
  flux = k[35]*n[IDX_H2Oj]*n[IDX_E];
  g[35] += flux * (mu[IDX_O] + mu[IDX_H2] - mu[IDX_H2Oj] - mu[IDX_E]);
  flux = k[36]*n[IDX_H2Oj]*n[IDX_E];
  g[36] += flux * (mu[IDX_OH] + mu[IDX_H] - mu[IDX_H2Oj] - mu[IDX_E]);
  flux = k[37]*n[IDX_H3Oj]*n[IDX_E];
  g[37] += flux * (mu[IDX_H2O] + mu[IDX_H] - mu[IDX_H3Oj] - mu[IDX_E]);
  flux = k[38]*n[IDX_O]*n[IDX_H];
  g[38] += flux * (mu[IDX_OH] - mu[IDX_O] - mu[IDX_H]);
  flux = k[39]*n[IDX_O]*n[IDX_H2];
  g[39] += flux * (mu[IDX_OH] + mu[IDX_H] - mu[IDX_O] - mu[IDX_H2]);
  flux = k[40]*n[IDX_H2]*n[IDX_OH];
  g[40] += flux * (mu[IDX_H2O] + mu[IDX_H] - mu[IDX_H2] - mu[IDX_OH]);
  flux = k[41]*n[IDX_OH]*n[IDX_OH];
  g[41] += flux * (mu[IDX_H2O] + mu[IDX_O] - mu[IDX_OH] - mu[IDX_OH]);
  flux = k[42]*n[IDX_Hj]*n[IDX_OH];
  g[42] += flux * (mu[IDX_OHj] + mu[IDX_H] - mu[IDX_Hj] - mu[IDX_OH]);
  flux = k[43]*n[IDX_Hj]*n[IDX_H2O];
  g[43] += flux * (mu[IDX_H2Oj] + mu[IDX_H] - mu[IDX_Hj] - mu[IDX_H2O]);
  flux = k[44]*n[IDX_H]*n[IDX_OH];
  g[44] += flux * (mu[IDX_H2] + mu[IDX_O] - mu[IDX_H] - mu[IDX_OH]);
  flux = k[45]*n[IDX_H]*n[IDX_H2O];
  g[45] += flux * (mu[IDX_OH] + mu[IDX_H2] - mu[IDX_H] - mu[IDX_H2O]);
  flux = k[46]*n[IDX_O]*n[IDX_O];
  g[46] += flux * (mu[IDX_O2] - mu[IDX_O] - mu[IDX_O]);
  flux = k[47]*n[IDX_O]*n[IDX_OH];
  g[47] += flux * (mu[IDX_O2] + mu[IDX_H] - mu[IDX_O] - mu[IDX_OH]);
  flux = k[48]*n[IDX_H]*n[IDX_O2];
  g[48] += flux * (mu[IDX_OH] + mu[IDX_O] - mu[IDX_H] - mu[IDX_O2]);
  flux = k[49]*n[IDX_Hj]*n[IDX_O2];
  g[49] += flux * (mu[IDX_O2j] + mu[IDX_H] - mu[IDX_Hj] - mu[IDX_O2]);
  flux = k[50]*n[IDX_O2j]*n[IDX_E];
  g[50] += flux * (mu[IDX_O] + mu[IDX_O] - mu[IDX_O2j] - mu[IDX_E]);
  flux = k[51]*n[IDX_O]*n[IDX_CH];
  g[51] += flux * (mu[IDX_CO] + mu[IDX_H] - mu[IDX_O] - mu[IDX_CH]);
  flux = k[52]*n[IDX_C]*n[IDX_OH];
  g[52] += flux * (mu[IDX_CO] + mu[IDX_H] - mu[IDX_C] - mu[IDX_OH]);
  flux = k[53]*n[IDX_C]*n[IDX_O2];
  g[53] += flux * (mu[IDX_CO] + mu[IDX_O] - mu[IDX_C] - mu[IDX_O2]);
  flux = k[54]*n[IDX_Cj]*n[IDX_O2];
  g[54] += flux * (mu[IDX_Oj] + mu[IDX_CO] - mu[IDX_Cj] - mu[IDX_O2]);
  flux = k[55]*n[IDX_OH]*n[IDX_CO];
  g[55] += flux * (mu[IDX_CO2] + mu[IDX_H] - mu[IDX_OH] - mu[IDX_CO]);
  flux = k[56]*n[IDX_Cj]*n[IDX_E];
  g[56] += flux * (mu[IDX_C] - mu[IDX_Cj] - mu[IDX_E]);
  flux = k[57]*n[IDX_Cj]*n[IDX_OH];
  g[57] += flux * (mu[IDX_COj] + mu[IDX_H] - mu[IDX_Cj] - mu[IDX_OH]);
  flux = k[58]*n[IDX_COj]*n[IDX_H];
  g[58] += flux * (mu[IDX_Hj] + mu[IDX_CO] - mu[IDX_COj] - mu[IDX_H]);
  flux = k[59]*n[IDX_C]*n[IDX_H];
  g[59] += flux * (mu[IDX_CH] - mu[IDX_C] - mu[IDX_H]);
  flux = k[60]*n[IDX_C]*n[IDX_H2];
  g[60] += flux * (mu[IDX_CH] + mu[IDX_H] - mu[IDX_C] - mu[IDX_H2]);
  flux = k[61]*n[IDX_H]*n[IDX_CH];
  g[61] += flux * (mu[IDX_C] + mu[IDX_H2] - mu[IDX_H] - mu[IDX_CH]);
  flux = k[62]*n[IDX_H2]*n[IDX_CH];
  g[62] += flux * (mu[IDX_CH2] + mu[IDX_H] - mu[IDX_H2] - mu[IDX_CH]);
  flux = k[63]*n[IDX_H]*n[IDX_CH2];
  g[63] += flux * (mu[IDX_CH] + mu[IDX_H2] - mu[IDX_H] - mu[IDX_CH2]);
  flux = k[64]*n[IDX_H2]*n[IDX_CH2];
  g[64] += flux * (mu[IDX_CH3] + mu[IDX_H] - mu[IDX_H2] - mu[IDX_CH2]);
  flux = k[65]*n[IDX_H]*n[IDX_CH3];
  g[65] += flux * (mu[IDX_CH2] + mu[IDX_H2] - mu[IDX_H] - mu[IDX_CH3]);
  flux = k[66]*n[IDX_H2]*n[IDX_CH3];
  g[66] += flux * (mu[IDX_CH4] + mu[IDX_H] - mu[IDX_H2] - mu[IDX_CH3]);
  flux = k[67]*n[IDX_H]*n[IDX_CH4];
  g[67] += flux * (mu[IDX_H2] + mu[IDX_CH3] - mu[IDX_H] - mu[IDX_CH4]);
  flux = k[68]*n[IDX_H2]*n[IDX_C];
  g[68] += flux * (mu[IDX_CH2] - mu[IDX_H2] - mu[IDX_C]);
  flux = k[69]*n[IDX_H3Oj]*n[IDX_E];
  g[69] += flux * (mu[IDX_OH] + mu[IDX_H] + mu[IDX_H] - mu[IDX_H3Oj] - mu[IDX_E]);
  flux = k[70]*n[IDX_OHj]*n[IDX_E];
  g[70] += flux * (mu[IDX_O] + mu[IDX_H] - mu[IDX_OHj] - mu[IDX_E]);
  flux = k[71]*n[IDX_Oj]*n[IDX_E];
  g[71] += flux * (mu[IDX_O] - mu[IDX_Oj] - mu[IDX_E]);
  flux = k[72]*n[IDX_COj]*n[IDX_E];
  g[72] += flux * (mu[IDX_CO] - mu[IDX_COj] - mu[IDX_E]);
  flux = k[73]*n[IDX_COj]*n[IDX_E];
  g[73] += flux * (mu[IDX_C] + mu[IDX_O] - mu[IDX_COj] - mu[IDX_E]);
}

// reaction labels: the equation, and the T range of a piece
inline const char* const reaction_names[74] = {"H + e- -> H+ + e- + e-", "H+ + e- -> H [0.0, 5500.0]", "H+ + e- -> H [5500.0, INFINITY]", "He + e- -> He+ + e- + e-", "He+ + e- -> He [0.0, 9280.0]", "He+ + e- -> He [9280.0, INFINITY]", "He+ + e- -> He++ + e- + e-", "He++ + e- -> He+", "H + e- -> H-", "H- + H -> H2 + e-", "H + H+ -> H2+ [0.0, 30.0]", "H + H+ -> H2+ [30.0, INFINITY]", "H2+ + H -> H2 + H+", "H2 + H+ -> H2+ + H [100.0, 30000.0]", "H2 + e- -> H + H-", "H2 + e- -> H + H + e-", "H2 + H -> H + H + H", "H- + e- -> H + e- + e-", "H- + H -> H + H + e- [0.0, 1160.0]", "H- + H -> H + H + e- [1160.0, INFINITY]", "H- + H+ -> H + H", "H- + H+ -> H2+ + e-", "H2+ + e- -> H + H", "H2+ + H- -> H + H2", "H + H + H -> H2 + H", "H2 + H + H -> H2 + H2", "H2 + H2 -> H + H + H2", "He+ + H -> He + H+", "He + H+ -> He+ + H [0.0, 10000.0]", "He + H+ -> He+ + H [10000.0, INFINITY]", "O+ + H -> H+ + O", "H+ + O -> O+ + H", "O+ + H2 -> OH+ + H", "OH+ + H2 -> H2O+ + H", "H2O+ + H2 -> H3O+ + H", "H2O+ + e- -> O + H2", "H2O+ + e- -> OH + H", "H3O+ + e- -> H2O + H", "O + H -> OH", "O + H2 -> OH + H", "H2 + OH -> H2O + H", "OH + OH -> H2O + O", "H+ + OH -> OH+ + H", "H+ + H2O -> H2O+ + H", "H + OH -> H2 + O", "H + H2O -> OH + H2", "O + O -> O2", "O + OH -> O2 + H", "H + O2 -> OH + O", "H+ + O2 -> O2+ + H", "O2+ + e- -> O + O", "O + CH -> CO + H", "C + OH -> CO + H", "C + O2 -> CO + O", "C+ + O2 -> O+ + CO", "OH + CO -> CO2 + H", "C+ + e- -> C", "C+ + OH -> CO+ + H", "CO+ + H -> H+ + CO", "C + H -> CH", "C + H2 -> CH + H", "H + CH -> C + H2", "H2 + CH -> CH2 + H", "H + CH2 -> CH + H2", "H2 + CH2 -> CH3 + H", "H + CH3 -> CH2 + H2", "H2 + CH3 -> CH4 + H", "H + CH4 -> H2 + CH3", "H2 + C -> CH2", "H3O+ + e- -> OH + H + H", "OH+ + e- -> O + H", "O+ + e- -> O", "CO+ + e- -> CO", "CO+ + e- -> C + O"};
constexpr int NHEAT = 0;
constexpr int NCOOL = 0;
inline const char* const heat_names[1] = {""};
inline const char* const cool_names[1] = {""};
// the thermal terms one by one [erg cm^-3 s^-1] at the thermal
// temperature T with the rates k: H[NHEAT], C[NCOOL] in the order
// of heat_names / cool_names (their sums are thermal_dTdt's)
KB_HD inline void thermal_terms(double T, const double* n, const double* k, const Params& p, double* H, double* C) {
  (void)T; (void)n; (void)k; (void)p; (void)H; (void)C;
}
// reaction fluxes k prod(n) [cm^-3 s^-1], fl[NREA]
KB_HD inline void reaction_fluxes(const double* n, const double* k, double* fl) {
  fl[0] = k[0]*n[IDX_H]*n[IDX_E];
  fl[1] = k[1]*n[IDX_Hj]*n[IDX_E];
  fl[2] = k[2]*n[IDX_Hj]*n[IDX_E];
  fl[3] = k[3]*n[IDX_He]*n[IDX_E];
  fl[4] = k[4]*n[IDX_Hej]*n[IDX_E];
  fl[5] = k[5]*n[IDX_Hej]*n[IDX_E];
  fl[6] = k[6]*n[IDX_Hej]*n[IDX_E];
  fl[7] = k[7]*n[IDX_Hejj]*n[IDX_E];
  fl[8] = k[8]*n[IDX_H]*n[IDX_E];
  fl[9] = k[9]*n[IDX_Hk]*n[IDX_H];
  fl[10] = k[10]*n[IDX_H]*n[IDX_Hj];
  fl[11] = k[11]*n[IDX_H]*n[IDX_Hj];
  fl[12] = k[12]*n[IDX_H2j]*n[IDX_H];
  fl[13] = k[13]*n[IDX_H2]*n[IDX_Hj];
  fl[14] = k[14]*n[IDX_H2]*n[IDX_E];
  fl[15] = k[15]*n[IDX_H2]*n[IDX_E];
  fl[16] = k[16]*n[IDX_H2]*n[IDX_H];
  fl[17] = k[17]*n[IDX_Hk]*n[IDX_E];
  fl[18] = k[18]*n[IDX_Hk]*n[IDX_H];
  fl[19] = k[19]*n[IDX_Hk]*n[IDX_H];
  fl[20] = k[20]*n[IDX_Hk]*n[IDX_Hj];
  fl[21] = k[21]*n[IDX_Hk]*n[IDX_Hj];
  fl[22] = k[22]*n[IDX_H2j]*n[IDX_E];
  fl[23] = k[23]*n[IDX_H2j]*n[IDX_Hk];
  fl[24] = k[24]*n[IDX_H]*n[IDX_H]*n[IDX_H];
  fl[25] = k[25]*n[IDX_H2]*n[IDX_H]*n[IDX_H];
  fl[26] = k[26]*n[IDX_H2]*n[IDX_H2];
  fl[27] = k[27]*n[IDX_Hej]*n[IDX_H];
  fl[28] = k[28]*n[IDX_He]*n[IDX_Hj];
  fl[29] = k[29]*n[IDX_He]*n[IDX_Hj];
  fl[30] = k[30]*n[IDX_Oj]*n[IDX_H];
  fl[31] = k[31]*n[IDX_Hj]*n[IDX_O];
  fl[32] = k[32]*n[IDX_Oj]*n[IDX_H2];
  fl[33] = k[33]*n[IDX_OHj]*n[IDX_H2];
  fl[34] = k[34]*n[IDX_H2Oj]*n[IDX_H2];
  fl[35] = k[35]*n[IDX_H2Oj]*n[IDX_E];
  fl[36] = k[36]*n[IDX_H2Oj]*n[IDX_E];
  fl[37] = k[37]*n[IDX_H3Oj]*n[IDX_E];
  fl[38] = k[38]*n[IDX_O]*n[IDX_H];
  fl[39] = k[39]*n[IDX_O]*n[IDX_H2];
  fl[40] = k[40]*n[IDX_H2]*n[IDX_OH];
  fl[41] = k[41]*n[IDX_OH]*n[IDX_OH];
  fl[42] = k[42]*n[IDX_Hj]*n[IDX_OH];
  fl[43] = k[43]*n[IDX_Hj]*n[IDX_H2O];
  fl[44] = k[44]*n[IDX_H]*n[IDX_OH];
  fl[45] = k[45]*n[IDX_H]*n[IDX_H2O];
  fl[46] = k[46]*n[IDX_O]*n[IDX_O];
  fl[47] = k[47]*n[IDX_O]*n[IDX_OH];
  fl[48] = k[48]*n[IDX_H]*n[IDX_O2];
  fl[49] = k[49]*n[IDX_Hj]*n[IDX_O2];
  fl[50] = k[50]*n[IDX_O2j]*n[IDX_E];
  fl[51] = k[51]*n[IDX_O]*n[IDX_CH];
  fl[52] = k[52]*n[IDX_C]*n[IDX_OH];
  fl[53] = k[53]*n[IDX_C]*n[IDX_O2];
  fl[54] = k[54]*n[IDX_Cj]*n[IDX_O2];
  fl[55] = k[55]*n[IDX_OH]*n[IDX_CO];
  fl[56] = k[56]*n[IDX_Cj]*n[IDX_E];
  fl[57] = k[57]*n[IDX_Cj]*n[IDX_OH];
  fl[58] = k[58]*n[IDX_COj]*n[IDX_H];
  fl[59] = k[59]*n[IDX_C]*n[IDX_H];
  fl[60] = k[60]*n[IDX_C]*n[IDX_H2];
  fl[61] = k[61]*n[IDX_H]*n[IDX_CH];
  fl[62] = k[62]*n[IDX_H2]*n[IDX_CH];
  fl[63] = k[63]*n[IDX_H]*n[IDX_CH2];
  fl[64] = k[64]*n[IDX_H2]*n[IDX_CH2];
  fl[65] = k[65]*n[IDX_H]*n[IDX_CH3];
  fl[66] = k[66]*n[IDX_H2]*n[IDX_CH3];
  fl[67] = k[67]*n[IDX_H]*n[IDX_CH4];
  fl[68] = k[68]*n[IDX_H2]*n[IDX_C];
  fl[69] = k[69]*n[IDX_H3Oj]*n[IDX_E];
  fl[70] = k[70]*n[IDX_OHj]*n[IDX_E];
  fl[71] = k[71]*n[IDX_Oj]*n[IDX_E];
  fl[72] = k[72]*n[IDX_COj]*n[IDX_E];
  fl[73] = k[73]*n[IDX_COj]*n[IDX_E];
}
// the neutral atomic metals (C, O) at n_H 10^(Z + kb_log10(n/n_H)_sun)
// of the Asplund+09 photospheric abundances, floored at 1e-40
KB_HD inline void scale_Z(double* n, double Z) {
  (void)n; (void)Z;
  const double Htot = Hnuclei_(n);
  n[IDX_C] = std::fmax(Htot * kb_exp10(Z + (-3.5700000000000003)), 1e-40);
  n[IDX_O] = std::fmax(Htot * kb_exp10(Z + (-3.3100000000000005)), 1e-40);
}
// the column density [cm^-2] of a number density x [cm^-3]
// (the default estimator: 1.87e21 (x / 1e3)^(2/3))
KB_HD inline double num2col_(double x) {
  return 1.87e21 * kb_pow(std::fmax(x, 1e-40) * 1e-3, 2.0/3.0);
}
KB_HD inline double NH_col_(const double* n) {
  (void)n;
  return num2col_(n[IDX_H]) + num2col_(n[IDX_Hj]) + 2.0 * num2col_(n[IDX_H2]);
}
constexpr int NLW = 0;
inline const int photo_reaction_[1] = {-1};
inline const int photo_reactant_[1] = {-1};
inline const double photo_pdiss_[1] = {1.0};
// the photoelectron deposit (E - Eth) of each photo rate: none for
// the Solomon process (line pumping)
inline const bool photo_deposit_[1] = {true};
inline const double photo_Emin_[1] = {0.0};
inline const double photo_Emax_[1] = {0.0};
namespace kbxs {  // no photo reactions
inline double (*const photo_xsec[1])(double) = {nullptr};
inline double (*const photo_xsec_int[1])(double, double) = {nullptr};
}  // namespace kbxs

constexpr bool HAS_THERMAL_TERMS = false;
// a rate coefficient depends on the densities (the species block
// of jac_stoich, taken at fixed k, is then not the exact dF/dn)
constexpr bool RATES_DEPEND_ON_N = true;
}  // namespace kbnet
