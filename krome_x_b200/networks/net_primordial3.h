// Generated by krome_x_b200.emit from the network 'primordial3' -- do not edit.
// One host/device (KB_HD) scalar form of the network: species,
// parameters, rate coefficients, mass-action rhs, stoichiometric
// Jacobian and the thermal equation (see krome_x_b200/emit/
// emitter.py for the layout and the reference rules it follows).
#pragma once
#include "../csrc/kb_common.h"

namespace kbnet {

constexpr const char* NETWORK_NAME = "primordial3";
constexpr const char* NETWORK_KEY = "primordial3";
constexpr int NSPEC = 9;
constexpr int NREA = 27;
constexpr int KB_RATE_NDEP = 2;
#define KB_NFREEZE 0
constexpr int IDX_H = 0;
constexpr int IDX_Hj = 1;
constexpr int IDX_Hk = 2;
constexpr int IDX_H2 = 3;
constexpr int IDX_H2j = 4;
constexpr int IDX_He = 5;
constexpr int IDX_Hej = 6;
constexpr int IDX_Hejj = 7;
constexpr int IDX_E = 8;
#define KB_HAS_H 1
#define KB_HAS_Hj 1
#define KB_HAS_Hk 1
#define KB_HAS_H2 1
#define KB_HAS_H2j 1
#define KB_HAS_He 1
#define KB_HAS_Hej 1
#define KB_HAS_Hejj 1
#define KB_HAS_E 1
#define KB_EXTERN_dissH2_Martin96 1
constexpr int IDX_ELECTRON = 8;

inline const char* const species_names[NSPEC] = {"H", "H+", "H-", "H2", "H2+", "He", "He+", "He++", "e-"};
constexpr int NELEM = 2;
inline const char* const element_names[2] = {"H", "He"};
KB_HD inline double species_mass_g(int i) {
  constexpr double t_[NSPEC] = {1.6738233791328e-24, 1.6729124407627538e-24, 1.6747343175028463e-24, 3.3476467582656e-24, 3.346735819895553e-24, 6.64647366797316e-24, 6.645562729603113e-24, 6.644651791233067e-24, 9.10938370046373e-28};
  return t_[i];
}
KB_HD inline int species_charge(int i) {
  constexpr int t_[NSPEC] = {0, 1, -1, 0, 1, 0, 1, 2, -1};
  return t_[i];
}
KB_HD inline double species_natoms_H(int i) {
  constexpr double t_[NSPEC] = {1.0, 1.0, 1.0, 2.0, 2.0, 0.0, 0.0, 0.0, 0.0};
  return t_[i];
}
KB_HD inline int species_opaque(int i) {
  constexpr int t_[NSPEC] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  return t_[i];
}
inline constexpr int species_elements_t_[18] = {1, 0, 1, 0, 1, 0, 2, 0, 2, 0, 0, 1, 0, 1, 0, 1, 0, 0};
#ifdef __CUDACC__
__device__ const int d_species_elements_[18] = {1, 0, 1, 0, 1, 0, 2, 0, 2, 0, 0, 1, 0, 1, 0, 1, 0, 0};
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

constexpr int NPAR = 3;
constexpr int NPHOTO = 0;
struct Params {
  double Tcmb;
  double tff;
  double opratio;
};
inline const char* const param_names[NPAR] = {"Tcmb", "tff", "opratio"};
// the defaults of a parameter row; NaN marks a REQUIRED parameter
inline double param_default(int i) {
  const double t_[NPAR] = {2.725, NAN, 3.0};
  return t_[i];
}
inline const char* const param_required_by[NPAR] = {"", "thermal.heating = ['COMPRESS']", ""};
KB_HD inline void params_from_row(const double* row, Params& p) {
  p.Tcmb = row[0];
  p.tff = row[1];
  p.opratio = row[2];
}
KB_HD inline int params_missing(const Params& p) {
  (void)p;
  if (p.tff != p.tff) return 1;
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
  k[21] = 1e-08 * kb_pow(Tgas, -0.4);  // H- + H+ -> H2+ + e-
  k[23] = 5e-07 * std::sqrt(100.0 * vh_invT);  // H2+ + H- -> H + H2
  k[24] = 6e-32 * kb_pow(Tgas, -0.25) + 2e-31 * 1.0/(std::sqrt(Tgas));  // H + H + H -> H2 + H
  k[25] = (6e-32 * kb_pow(Tgas, -0.25) + 2e-31 * 1.0/(std::sqrt(Tgas))) / 8.0;  // H2 + H + H -> H2 + H2
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
  {  // group 6: H- + H+ -> H + H
    double T = Tgas;
    if (T > 100000.0) T = 100000.0;
    if (T >= 10.0 && T >= 10.0) {
      k[20] = 2.96e-06 / std::sqrt(T) - 1.73e-09 + 2.5e-10 * std::sqrt(T) - 7.77e-13 * T;  // H- + H+ -> H + H
    }
  }
  {  // group 7: H2+ + e- -> H + H
    double T = Tgas;
    if (T > 10000.0) T = 10000.0;
    if (true) {
      k[22] = 1000000.0 * (4.2278e-14 - 2.3088e-17 * T + 7.3428e-21 * T*T - 7.5474e-25 * T*T*T + 3.3468e-29 * T*T*T*T - 5.528e-34 * ipow_<5>(T));  // H2+ + e- -> H + H
    }
  }
}
// rate coefficients that also depend on the densities
KB_HD inline void rates_var(double Tgas, const double* n, const Params& p, double* k) {
  (void)Tgas; (void)n; (void)p; (void)k;
  const double vh_T = v_T(Tgas, n, p);
  (void)vh_T;
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
}
constexpr int NREA_FIXED = 25;
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
  {  // group 6: H- + H+ -> H + H
    double T = Tgas;
    if (T > 100000.0) T = 100000.0;
    if (T >= 10.0 && T >= 10.0) {
    }
  }
  {  // group 7: H2+ + e- -> H + H
    double T = Tgas;
    if (T > 10000.0) T = 10000.0;
    if (true) {
    }
  }
}

KB_HD inline double cooling_chem(const double* n, const double* k) {
  double c = 0.0;
  c += k[15] * 4.48 * n[IDX_H2]*n[IDX_E];
  c += k[16] * 4.48 * n[IDX_H2]*n[IDX_H];
  c += k[26] * 4.48 * n[IDX_H2]*n[IDX_H2];
  c *= kbc::eV_to_erg;
  return c;
}
KB_HD inline double heating_chem(double Tgas, const double* n, const double* k) {
  double h = 0.0;
  const double ev2erg = kbc::eV_to_erg;
  const double dd = Hnuclei_(n);
  const double ncr = 1.0e6 / std::sqrt(Tgas)
      / (1.6 * kb_exp(-kb_pow(4.0e2 / Tgas, 2.0)) * n[IDX_H] / dd
         + 1.4 * kb_exp(-1.2e4 / (Tgas + 1.2e3)) * n[IDX_H2] / dd);
  const double ffac = 1.0 / (1.0 + ncr / dd);
  h += k[9] * (3.53*ffac) * n[IDX_Hk]*n[IDX_H];
  h += k[12] * (1.83*ffac) * n[IDX_H2j]*n[IDX_H];
  h += k[24] * (4.48*ffac) * n[IDX_H]*n[IDX_H]*n[IDX_H];
  h += k[25] * (4.48*ffac) * n[IDX_H2]*n[IDX_H]*n[IDX_H];
  h *= ev2erg;
  return h;
}
KB_HD inline double h2_opacity_(const double* n) {
  (void)n;
  return std::fmin(1.0, kb_pow(std::fmax(1.25e-10 * ntot_(n), 1e-40), -0.45));
}
KB_HD inline double gamma_rot_(double Tin, double brot) {
  const double ib = brot / std::fmax(Tin, 10.0);
  double z = 0.0, e1 = 0.0, e2 = 0.0;
KB_UNROLL
  for (int j = 0; j <= 10; ++j) {
    const double E = j * (j + 1.0) * ib;
    const double g = (2.0 * j + 1.0) * kb_exp(-E);
    z += g; e1 += g * E; e2 += g * E * E;
  }
  const double m = e1 / z;
  return e2 / z - m * m;
}
KB_HD inline double gamma_rotop_(double Tin, double a) {
  const double ib = 85.4 / std::fmax(Tin, 10.0);
  double zp = 0.0, p1 = 0.0, p2 = 0.0, zo = 0.0, o1 = 0.0, o2 = 0.0;
KB_UNROLL
  for (int j = 0; j <= 10; j += 2) {
    const int j1 = j + 1;
    const double Ep = j * (j + 1.0) * ib;
    const double Eo = j1 * (j1 + 1.0) * ib;
    const double gp = (2.0 * j + 1.0) * kb_exp(-Ep);
    const double go = 3.0 * (2.0 * j1 + 1.0) * kb_exp(-Eo);
    zp += gp; p1 += gp * Ep; p2 += gp * Ep * Ep;
    zo += go; o1 += go * Eo; o2 += go * Eo * Eo;
  }
  const double b = 1.0 - a;
  const double mp = p1 / zp, mo = o1 / zo;
  return b * (p2 / zp - mp * mp) + a * (o2 / zo - mo * mo);
}
KB_HD inline double gamma_index(double Tgas, const double* n, const Params& p) {
  (void)Tgas; (void)n; (void)p;
  const double iTv = 1.0 / std::fmax(Tgas, 63.3236349736972);
  const double x_H2 = 6332.36349736972 * iTv, e_H2 = kb_exp(x_H2);
  const double gi_H2 = 0.5 * (3.0 + 2.0 * gamma_rotop_(Tgas, p.opratio / (p.opratio + 1.0)) + 2.0 * x_H2 * x_H2 * e_H2 / ((e_H2 - 1.0) * (e_H2 - 1.0)));
  const double gi_H2j = 0.5 * (3.0 + 2.0 * gamma_rot_(Tgas, 61.72352804491875) + 0.0);
  const double mosum = n[IDX_H] + n[IDX_Hj] + n[IDX_Hk] + n[IDX_He] + n[IDX_Hej] + n[IDX_Hejj] + n[IDX_E];
  const double ysum = mosum + n[IDX_H2] + n[IDX_H2j];
  const double gsum = 1.5 * mosum + n[IDX_H2] * gi_H2 + n[IDX_H2j] * gi_H2j;
  return gsum > 0.0 ? 1.0 + ysum / gsum : 5.0 / 3.0;
}
// dTgas/dt at the thermal temperature T (capped to [2.73, 1e9] K by
// the caller) with the rates k of the rate temperature
KB_HD inline double thermal_dTdt(double T, const double* n, const double* k, const Params& p) {
  (void)k; (void)p;
  double heat = 0.0, cool = 0.0;
  heat += heating_chem(T, n, k);
  heat += ntot_(n) * kbc::boltzmann_erg * T / p.tff;
  cool += cooling_H2(T, n) * h2_opacity_(n);
  cool += cooling_chem(n, k);
  cool += cooling_Continuum(T, n);
  return (gamma_index(T, n, p) - 1.0) * (heat - cool)
      / (kbc::boltzmann_erg * ntot_(n));
}
// the cooling's temperature-only parts at one T (a row of density
// derivatives at that T evaluates them once): thermal_dTdt_with of
// thermal_pre(T) equals thermal_dTdt bit for bit
struct ThermalPre {
  CoolH2C h2;
  int unused_;
};
KB_HD inline void thermal_pre(double T, const double* n, const Params& p, ThermalPre& q) {
  (void)T; (void)n; (void)p; (void)q;
  q.h2 = cooling_H2_coef(T);
}
KB_HD inline double thermal_dTdt_with(const ThermalPre& q, double T, const double* n, const double* k, const Params& p) {
  (void)q; (void)k; (void)p;
  double heat = 0.0, cool = 0.0;
  heat += heating_chem(T, n, k);
  heat += ntot_(n) * kbc::boltzmann_erg * T / p.tff;
  cool += cooling_H2_with(q.h2, n) * h2_opacity_(n);
  cool += cooling_chem(n, k);
  cool += cooling_Continuum(T, n);
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
  if (muT != 0.0) {
    const double c = muT * (gamma_index(Tth, n, p) - 1.0) / (kbc::boltzmann_erg * ntot_(n)) * kbc::eV_to_erg;
    g[15] -= c * k[15] * 4.48 * n[IDX_H2]*n[IDX_E];
    g[16] -= c * k[16] * 4.48 * n[IDX_H2]*n[IDX_H];
    g[26] -= c * k[26] * 4.48 * n[IDX_H2]*n[IDX_H2];
    const double dd = Hnuclei_(n);
    const double ncr = 1.0e6 / std::sqrt(Tth)
        / (1.6 * kb_exp(-kb_pow(4.0e2 / Tth, 2.0)) * n[IDX_H] / dd
           + 1.4 * kb_exp(-1.2e4 / (Tth + 1.2e3)) * n[IDX_H2] / dd);
    const double ffac = 1.0 / (1.0 + ncr / dd);
    (void)ffac;
    g[9] += c * k[9] * (3.53*ffac) * n[IDX_Hk]*n[IDX_H];
    g[12] += c * k[12] * (1.83*ffac) * n[IDX_H2j]*n[IDX_H];
    g[24] += c * k[24] * (4.48*ffac) * n[IDX_H]*n[IDX_H]*n[IDX_H];
    g[25] += c * k[25] * (4.48*ffac) * n[IDX_H2]*n[IDX_H]*n[IDX_H];
  }
}

// reaction labels: the equation, and the T range of a piece
inline const char* const reaction_names[27] = {"H + e- -> H+ + e- + e-", "H+ + e- -> H [0.0, 5500.0]", "H+ + e- -> H [5500.0, INFINITY]", "He + e- -> He+ + e- + e-", "He+ + e- -> He [0.0, 9280.0]", "He+ + e- -> He [9280.0, INFINITY]", "He+ + e- -> He++ + e- + e-", "He++ + e- -> He+", "H + e- -> H-", "H- + H -> H2 + e-", "H + H+ -> H2+ [0.0, 30.0]", "H + H+ -> H2+ [30.0, INFINITY]", "H2+ + H -> H2 + H+", "H2 + H+ -> H2+ + H [100.0, 30000.0]", "H2 + e- -> H + H-", "H2 + e- -> H + H + e-", "H2 + H -> H + H + H", "H- + e- -> H + e- + e-", "H- + H -> H + H + e- [0.0, 1160.0]", "H- + H -> H + H + e- [1160.0, INFINITY]", "H- + H+ -> H + H [10.0, 100000.0]", "H- + H+ -> H2+ + e-", "H2+ + e- -> H + H [0.0, 10000.0]", "H2+ + H- -> H + H2", "H + H + H -> H2 + H", "H2 + H + H -> H2 + H2", "H2 + H2 -> H + H + H2"};
constexpr int NHEAT = 2;
constexpr int NCOOL = 3;
inline const char* const heat_names[2] = {"CHEM", "COMPRESS"};
inline const char* const cool_names[3] = {"H2", "CHEM", "CONT"};
// the thermal terms one by one [erg cm^-3 s^-1] at the thermal
// temperature T with the rates k: H[NHEAT], C[NCOOL] in the order
// of heat_names / cool_names (their sums are thermal_dTdt's)
KB_HD inline void thermal_terms(double T, const double* n, const double* k, const Params& p, double* H, double* C) {
  (void)T; (void)n; (void)k; (void)p; (void)H; (void)C;
  H[0] = heating_chem(T, n, k);
  H[1] = ntot_(n) * kbc::boltzmann_erg * T / p.tff;
  C[0] = cooling_H2(T, n) * h2_opacity_(n);
  C[1] = cooling_chem(n, k);
  C[2] = cooling_Continuum(T, n);
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
}
// the neutral atomic metals (none) at n_H 10^(Z + kb_log10(n/n_H)_sun)
// of the Asplund+09 photospheric abundances, floored at 1e-40
KB_HD inline void scale_Z(double* n, double Z) {
  (void)n; (void)Z;
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

constexpr bool HAS_THERMAL_TERMS = true;
// a rate coefficient depends on the densities (the species block
// of jac_stoich, taken at fixed k, is then not the exact dF/dn)
constexpr bool RATES_DEPEND_ON_N = true;
}  // namespace kbnet
