// Generated by krome_x_b200.emit from the network 'galaxy_ism' -- do not edit.
// One host/device (KB_HD) scalar form of the network: species,
// parameters, rate coefficients, mass-action rhs, stoichiometric
// Jacobian and the thermal equation (see krome_x_b200/emit/
// emitter.py for the layout and the reference rules it follows).
#pragma once
#include "../csrc/kb_common.h"

namespace kbnet {

constexpr const char* NETWORK_NAME = "galaxy_ism";
constexpr const char* NETWORK_KEY = "galaxy_ism";
constexpr int NSPEC = 9;
constexpr int NREA = 46;
constexpr int KB_RATE_NDEP = 3;
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
#define KB_EXTERN_H2_sigmaLW 1
#define KB_EXTERN_H2_solomonLW 1
#define KB_EXTERN_H_recombination_on_dust 1
#define KB_EXTERN_He_recombination_on_dust 1
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

constexpr int NPAR = 5;
constexpr int NPHOTO = 8;
struct Params {
  double crate;
  double G0;
  double d2g;
  double gamma_ad;
  double Tcmb;
  // the photo rates sum_b sigma_rb Phi_b of the cell's field
  double kph[NPHOTO];
};
inline const char* const param_names[NPAR] = {"crate", "G0", "d2g", "gamma_ad", "Tcmb"};
// the defaults of a parameter row; NaN marks a REQUIRED parameter
inline double param_default(int i) {
  const double t_[NPAR] = {0.0, 0.0, 0.01, 1.6666666666666667, 2.725};
  return t_[i];
}
inline const char* const param_required_by[NPAR] = {"", "", "", "", ""};
KB_HD inline void params_from_row(const double* row, Params& p) {
  p.crate = row[0];
  p.G0 = row[1];
  p.d2g = row[2];
  p.gamma_ad = row[3];
  p.Tcmb = row[4];
  p.kph[0] = 0.0;
  p.kph[1] = 0.0;
  p.kph[2] = 0.0;
  p.kph[3] = 0.0;
  p.kph[4] = 0.0;
  p.kph[5] = 0.0;
  p.kph[6] = 0.0;
  p.kph[7] = 0.0;
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
KB_HD inline double v_asav0(double Tgas, const double* n, const Params& p) {
  (void)Tgas; (void)n; (void)p;
  return -191.53214;
}
KB_HD inline double v_asav1(double Tgas, const double* n, const Params& p) {
  (void)Tgas; (void)n; (void)p;
  return 401.29114;
}
KB_HD inline double v_asav2(double Tgas, const double* n, const Params& p) {
  (void)Tgas; (void)n; (void)p;
  return -374.46991;
}
KB_HD inline double v_asav3(double Tgas, const double* n, const Params& p) {
  (void)Tgas; (void)n; (void)p;
  return 190.7841;
}
KB_HD inline double v_asav4(double Tgas, const double* n, const Params& p) {
  (void)Tgas; (void)n; (void)p;
  return -57.263467;
}
KB_HD inline double v_asav5(double Tgas, const double* n, const Params& p) {
  (void)Tgas; (void)n; (void)p;
  return 10.13321;
}
KB_HD inline double v_asav6(double Tgas, const double* n, const Params& p) {
  (void)Tgas; (void)n; (void)p;
  return -0.98012853;
}
KB_HD inline double v_asav7(double Tgas, const double* n, const Params& p) {
  (void)Tgas; (void)n; (void)p;
  return 0.040023414;
}
KB_HD inline double v_bsav0(double Tgas, const double* n, const Params& p) {
  (void)Tgas; (void)n; (void)p;
  return -8875.5774;
}
KB_HD inline double v_bsav1(double Tgas, const double* n, const Params& p) {
  (void)Tgas; (void)n; (void)p;
  return 10081.246;
}
KB_HD inline double v_bsav2(double Tgas, const double* n, const Params& p) {
  (void)Tgas; (void)n; (void)p;
  return -4860.6622;
}
KB_HD inline double v_bsav3(double Tgas, const double* n, const Params& p) {
  (void)Tgas; (void)n; (void)p;
  return 1288.9659;
}
KB_HD inline double v_bsav4(double Tgas, const double* n, const Params& p) {
  (void)Tgas; (void)n; (void)p;
  return -203.19575;
}
KB_HD inline double v_bsav5(double Tgas, const double* n, const Params& p) {
  (void)Tgas; (void)n; (void)p;
  return 19.057493;
}
KB_HD inline double v_bsav6(double Tgas, const double* n, const Params& p) {
  (void)Tgas; (void)n; (void)p;
  return -0.98530668;
}
KB_HD inline double v_bsav7(double Tgas, const double* n, const Params& p) {
  (void)Tgas; (void)n; (void)p;
  return 0.021675387;
}
KB_HD inline double v_sumsav(double Tgas, const double* n, const Params& p) {
  (void)Tgas; (void)n; (void)p;
  return v_asav0(Tgas, n, p) + v_asav1(Tgas, n, p) * kb_log10(Tgas) + v_asav2(Tgas, n, p) * kb_log10(Tgas)*kb_log10(Tgas) + v_asav3(Tgas, n, p) * kb_log10(Tgas)*kb_log10(Tgas)*kb_log10(Tgas) + v_asav4(Tgas, n, p) * kb_log10(Tgas)*kb_log10(Tgas)*kb_log10(Tgas)*kb_log10(Tgas) + v_asav5(Tgas, n, p) * ipow_<5>(kb_log10(Tgas)) + v_asav6(Tgas, n, p) * ipow_<6>(kb_log10(Tgas)) + v_asav7(Tgas, n, p) * ipow_<7>(kb_log10(Tgas));
}
KB_HD inline double v_sumsbv(double Tgas, const double* n, const Params& p) {
  (void)Tgas; (void)n; (void)p;
  return v_bsav0(Tgas, n, p) + v_bsav1(Tgas, n, p) * kb_log10(Tgas) + v_bsav2(Tgas, n, p) * kb_log10(Tgas)*kb_log10(Tgas) + v_bsav3(Tgas, n, p) * kb_log10(Tgas)*kb_log10(Tgas)*kb_log10(Tgas) + v_bsav4(Tgas, n, p) * kb_log10(Tgas)*kb_log10(Tgas)*kb_log10(Tgas)*kb_log10(Tgas) + v_bsav5(Tgas, n, p) * ipow_<5>(kb_log10(Tgas)) + v_bsav6(Tgas, n, p) * ipow_<6>(kb_log10(Tgas)) + v_bsav7(Tgas, n, p) * ipow_<7>(kb_log10(Tgas));
}
KB_HD inline double v_myflux_eV(double Tgas, const double* n, const Params& p) {
  (void)Tgas; (void)n; (void)p;
  return 2.01235e-10;
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
  k[15] = 35.5 * kb_pow(Tgas, -2.28) * kb_exp(-46707.0 / Tgas);  // H2 + e- -> H + H-
  k[16] = 4.38e-10 * kb_exp(-102000.0 / Tgas) * kb_pow(Tgas, 0.35);  // H2 + e- -> H + H + e-
  k[17] = 6.67e-12 * std::sqrt(Tgas) * kb_exp(-(1.0 + 63593.0 / Tgas));  // H2 + H -> H + H + H
  k[18] = kb_exp(-18.01849334273 + 2.360852208681 * vh_lnTe - 0.2827443061704 * vh_lnTe*vh_lnTe + 0.01623316639567 * vh_lnTe*vh_lnTe*vh_lnTe - 0.03365012031362999 * vh_lnTe*vh_lnTe*vh_lnTe*vh_lnTe + 0.01178329782711 * ipow_<5>(vh_lnTe) - 0.001656194699504 * ipow_<6>(vh_lnTe) + 0.0001068275202678 * ipow_<7>(vh_lnTe) - 2.631285809207e-06 * ipow_<8>(vh_lnTe));  // H- + e- -> H + e- + e-
  k[22] = 1e-08 * kb_pow(Tgas, -0.4);  // H- + H+ -> H2+ + e-
  k[25] = 5e-07 * std::sqrt(100.0 * vh_invT);  // H2+ + H- -> H + H2
  k[26] = 5.996e-30 * kb_pow(Tgas, 4.1881) * kb_pow(1.0 + 6.761e-06 * Tgas, -5.6881) * kb_exp(-54657.4 * vh_invT);  // H2 + H2 -> H + H + H2
  k[27] = 1.2e-15 * kb_pow(Tgas / 300.0, 0.25);  // He+ + H -> He + H+
  k[30] = 3.7e-14 * kb_exp(-35.0 / Tgas);  // H2 + He+ -> He + H + H+
  k[31] = kb_exp10(-27.029 + 3.801 * kb_log10(Tgas) - 29487.0 / Tgas);  // H2 + He -> H + H + He
  k[32] = 7.2e-15;  // H2 + He+ -> H2+ + He
  k[33] = 1.2e-17 * kb_pow(Tgas, 1.2) * kb_exp(-157800.0 * vh_invT);  // H + H -> H + H+ + e-
  k[34] = 1.75e-17 * kb_pow(Tgas, 1.3) * kb_exp(-157800.0 * vh_invT);  // H + He -> He + H+ + e-
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
    if (T < 9284.0) {
      k[4] = 3.92e-13 * kb_pow(vh_invTe, 0.6353);  // He+ + e- -> He
    }
    else if (T >= 9284.0) {
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
    if (T > 100000000.0) T = 100000000.0;
    const double vh_asav0 = v_asav0(T, n, p);
    (void)vh_asav0;
    const double vh_asav1 = v_asav1(T, n, p);
    (void)vh_asav1;
    const double vh_asav2 = v_asav2(T, n, p);
    (void)vh_asav2;
    const double vh_asav3 = v_asav3(T, n, p);
    (void)vh_asav3;
    const double vh_asav4 = v_asav4(T, n, p);
    (void)vh_asav4;
    const double vh_asav5 = v_asav5(T, n, p);
    (void)vh_asav5;
    const double vh_asav6 = v_asav6(T, n, p);
    (void)vh_asav6;
    const double vh_asav7 = v_asav7(T, n, p);
    (void)vh_asav7;
    const double vh_bsav0 = v_bsav0(T, n, p);
    (void)vh_bsav0;
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
    const double vh_sumsav = v_sumsav(T, n, p);
    (void)vh_sumsav;
    const double vh_sumsbv = v_sumsbv(T, n, p);
    (void)vh_sumsbv;
    if (T >= 100.0 && T >= 100.0 && T < 100000.0) {
      k[13] = kb_exp10(vh_sumsav);  // H2 + H+ -> H2+ + H
    }
    else if (T >= 100000.0) {
      k[14] = kb_exp10(vh_sumsbv);  // H2 + H+ -> H2+ + H
    }
  }
  {  // group 5: H- + H -> H + H + e-
    double T = Tgas;
    const double vh_Te = v_Te(T, n, p);
    (void)vh_Te;
    const double vh_lnTe = v_lnTe(T, n, p);
    (void)vh_lnTe;
    if (T < 1160.0) {
      k[19] = 2.56e-09 * kb_pow(vh_Te, 1.78186);  // H- + H -> H + H + e-
    }
    else if (T >= 1160.0) {
      k[20] = kb_exp(-20.37260896533324 + 1.139449335841631 * vh_lnTe - 0.1421013521554148 * vh_lnTe*vh_lnTe + 0.00846445538663 * vh_lnTe*vh_lnTe*vh_lnTe - 0.0014327641212992 * vh_lnTe*vh_lnTe*vh_lnTe*vh_lnTe + 0.0002012250284791 * ipow_<5>(vh_lnTe) + 8.66396324309e-05 * ipow_<6>(vh_lnTe) - 2.585009680264e-05 * ipow_<7>(vh_lnTe) + 2.4555011970392e-06 * ipow_<8>(vh_lnTe) - 8.06838246118e-08 * ipow_<9>(vh_lnTe));  // H- + H -> H + H + e-
    }
  }
  {  // group 6: H- + H+ -> H + H
    double T = Tgas;
    if (T > 10000000.0) T = 10000000.0;
    if (T >= 10.0 && T >= 10.0) {
      k[21] = 2.96e-06 / std::sqrt(T) - 1.73e-09 + 2.5e-10 * std::sqrt(T) - 7.77e-13;  // H- + H+ -> H + H
    }
  }
  {  // group 7: H2+ + e- -> H + H
    double T = Tgas;
    if (T < 617.0) {
      k[23] = 1e-08;  // H2+ + e- -> H + H
    }
    else if (T >= 617.0) {
      k[24] = 1.32e-06 * kb_pow(T, -0.76);  // H2+ + e- -> H + H
    }
  }
  {  // group 8: He + H+ -> He+ + H
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
  const double vh_myflux_eV = v_myflux_eV(Tgas, n, p);
  (void)vh_myflux_eV;
  k[43] = H2_solomonLW(vh_myflux_eV, Tgas, n, p);  // H2 -> H + H
  k[44] = H_recombination_on_dust(Tgas, n, p);  // H+ + e- -> H
  k[45] = He_recombination_on_dust(Tgas, n, p);  // He+ + e- -> He
  k[35] += p.kph[0];  // H -> H+ + e-
  k[36] += p.kph[1];  // He -> He+ + e-
  k[37] += p.kph[2];  // He+ -> He++ + e-
  k[38] += p.kph[3];  // H- -> H + e-
  k[39] += p.kph[4];  // H2 -> H2+ + e-
  k[40] += p.kph[5];  // H2+ -> H+ + H
  k[41] += p.kph[6];  // H2+ -> H+ + H+ + e-
  k[42] += p.kph[7];  // H2 -> H + H
}
constexpr int NREA_FIXED = 35;
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
    case 16:
    case 17:
    case 18:
    case 19:
    case 20:
    case 21:
    case 22:
    case 23:
    case 24:
    case 25:
    case 26:
    case 27:
    case 28:
    case 29:
    case 30:
    case 31:
    case 32:
    case 33:
    case 34:
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
  flux = k[14]*n[IDX_H2]*n[IDX_Hj];
  dn[IDX_H2] -= flux;
  dn[IDX_Hj] -= flux;
  dn[IDX_H2j] += flux;
  dn[IDX_H] += flux;
  flux = k[15]*n[IDX_H2]*n[IDX_E];
  dn[IDX_H2] -= flux;
  dn[IDX_E] -= flux;
  dn[IDX_H] += flux;
  dn[IDX_Hk] += flux;
  flux = k[16]*n[IDX_H2]*n[IDX_E];
  dn[IDX_H2] -= flux;
  dn[IDX_E] -= flux;
  dn[IDX_H] += flux;
  dn[IDX_H] += flux;
  dn[IDX_E] += flux;
  flux = k[17]*n[IDX_H2]*n[IDX_H];
  dn[IDX_H2] -= flux;
  dn[IDX_H] -= flux;
  dn[IDX_H] += flux;
  dn[IDX_H] += flux;
  dn[IDX_H] += flux;
  flux = k[18]*n[IDX_Hk]*n[IDX_E];
  dn[IDX_Hk] -= flux;
  dn[IDX_E] -= flux;
  dn[IDX_H] += flux;
  dn[IDX_E] += flux;
  dn[IDX_E] += flux;
  flux = k[19]*n[IDX_Hk]*n[IDX_H];
  dn[IDX_Hk] -= flux;
  dn[IDX_H] -= flux;
  dn[IDX_H] += flux;
  dn[IDX_H] += flux;
  dn[IDX_E] += flux;
  flux = k[20]*n[IDX_Hk]*n[IDX_H];
  dn[IDX_Hk] -= flux;
  dn[IDX_H] -= flux;
  dn[IDX_H] += flux;
  dn[IDX_H] += flux;
  dn[IDX_E] += flux;
  flux = k[21]*n[IDX_Hk]*n[IDX_Hj];
  dn[IDX_Hk] -= flux;
  dn[IDX_Hj] -= flux;
  dn[IDX_H] += flux;
  dn[IDX_H] += flux;
  flux = k[22]*n[IDX_Hk]*n[IDX_Hj];
  dn[IDX_Hk] -= flux;
  dn[IDX_Hj] -= flux;
  dn[IDX_H2j] += flux;
  dn[IDX_E] += flux;
  flux = k[23]*n[IDX_H2j]*n[IDX_E];
  dn[IDX_H2j] -= flux;
  dn[IDX_E] -= flux;
  dn[IDX_H] += flux;
  dn[IDX_H] += flux;
  flux = k[24]*n[IDX_H2j]*n[IDX_E];
  dn[IDX_H2j] -= flux;
  dn[IDX_E] -= flux;
  dn[IDX_H] += flux;
  dn[IDX_H] += flux;
  flux = k[25]*n[IDX_H2j]*n[IDX_Hk];
  dn[IDX_H2j] -= flux;
  dn[IDX_Hk] -= flux;
  dn[IDX_H] += flux;
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
  flux = k[30]*n[IDX_H2]*n[IDX_Hej];
  dn[IDX_H2] -= flux;
  dn[IDX_Hej] -= flux;
  dn[IDX_He] += flux;
  dn[IDX_H] += flux;
  dn[IDX_Hj] += flux;
  flux = k[31]*n[IDX_H2]*n[IDX_He];
  dn[IDX_H2] -= flux;
  dn[IDX_He] -= flux;
  dn[IDX_H] += flux;
  dn[IDX_H] += flux;
  dn[IDX_He] += flux;
  flux = k[32]*n[IDX_H2]*n[IDX_Hej];
  dn[IDX_H2] -= flux;
  dn[IDX_Hej] -= flux;
  dn[IDX_H2j] += flux;
  dn[IDX_He] += flux;
  flux = k[33]*n[IDX_H]*n[IDX_H];
  dn[IDX_H] -= flux;
  dn[IDX_H] -= flux;
  dn[IDX_H] += flux;
  dn[IDX_Hj] += flux;
  dn[IDX_E] += flux;
  flux = k[34]*n[IDX_H]*n[IDX_He];
  dn[IDX_H] -= flux;
  dn[IDX_He] -= flux;
  dn[IDX_He] += flux;
  dn[IDX_Hj] += flux;
  dn[IDX_E] += flux;
  flux = k[35]*n[IDX_H];
  dn[IDX_H] -= flux;
  dn[IDX_Hj] += flux;
  dn[IDX_E] += flux;
  flux = k[36]*n[IDX_He];
  dn[IDX_He] -= flux;
  dn[IDX_Hej] += flux;
  dn[IDX_E] += flux;
  flux = k[37]*n[IDX_Hej];
  dn[IDX_Hej] -= flux;
  dn[IDX_Hejj] += flux;
  dn[IDX_E] += flux;
  flux = k[38]*n[IDX_Hk];
  dn[IDX_Hk] -= flux;
  dn[IDX_H] += flux;
  dn[IDX_E] += flux;
  flux = k[39]*n[IDX_H2];
  dn[IDX_H2] -= flux;
  dn[IDX_H2j] += flux;
  dn[IDX_E] += flux;
  flux = k[40]*n[IDX_H2j];
  dn[IDX_H2j] -= flux;
  dn[IDX_Hj] += flux;
  dn[IDX_H] += flux;
  flux = k[41]*n[IDX_H2j];
  dn[IDX_H2j] -= flux;
  dn[IDX_Hj] += flux;
  dn[IDX_Hj] += flux;
  dn[IDX_E] += flux;
  flux = k[42]*n[IDX_H2];
  dn[IDX_H2] -= flux;
  dn[IDX_H] += flux;
  dn[IDX_H] += flux;
  flux = k[43]*n[IDX_H2];
  dn[IDX_H2] -= flux;
  dn[IDX_H] += flux;
  dn[IDX_H] += flux;
  flux = k[44]*n[IDX_Hj]*n[IDX_E];
  dn[IDX_Hj] -= flux;
  dn[IDX_E] -= flux;
  dn[IDX_H] += flux;
  flux = k[45]*n[IDX_Hej]*n[IDX_E];
  dn[IDX_Hej] -= flux;
  dn[IDX_E] -= flux;
  dn[IDX_He] += flux;
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
  d = k[14]*n[IDX_H2];
  J[IDX_H2*rs + IDX_Hj*cs] -= d;
  J[IDX_Hj*rs + IDX_Hj*cs] -= d;
  J[IDX_H2j*rs + IDX_Hj*cs] += d;
  J[IDX_H*rs + IDX_Hj*cs] += d;
  d = k[14]*n[IDX_Hj];
  J[IDX_H2*rs + IDX_H2*cs] -= d;
  J[IDX_Hj*rs + IDX_H2*cs] -= d;
  J[IDX_H2j*rs + IDX_H2*cs] += d;
  J[IDX_H*rs + IDX_H2*cs] += d;
  d = k[15]*n[IDX_E];
  J[IDX_H2*rs + IDX_H2*cs] -= d;
  J[IDX_E*rs + IDX_H2*cs] -= d;
  J[IDX_H*rs + IDX_H2*cs] += d;
  J[IDX_Hk*rs + IDX_H2*cs] += d;
  d = k[15]*n[IDX_H2];
  J[IDX_H2*rs + IDX_E*cs] -= d;
  J[IDX_E*rs + IDX_E*cs] -= d;
  J[IDX_H*rs + IDX_E*cs] += d;
  J[IDX_Hk*rs + IDX_E*cs] += d;
  d = k[16]*n[IDX_E];
  J[IDX_H2*rs + IDX_H2*cs] -= d;
  J[IDX_E*rs + IDX_H2*cs] -= d;
  J[IDX_H*rs + IDX_H2*cs] += d;
  J[IDX_H*rs + IDX_H2*cs] += d;
  J[IDX_E*rs + IDX_H2*cs] += d;
  d = k[16]*n[IDX_H2];
  J[IDX_H2*rs + IDX_E*cs] -= d;
  J[IDX_E*rs + IDX_E*cs] -= d;
  J[IDX_H*rs + IDX_E*cs] += d;
  J[IDX_H*rs + IDX_E*cs] += d;
  J[IDX_E*rs + IDX_E*cs] += d;
  d = k[17]*n[IDX_H2];
  J[IDX_H2*rs + IDX_H*cs] -= d;
  J[IDX_H*rs + IDX_H*cs] -= d;
  J[IDX_H*rs + IDX_H*cs] += d;
  J[IDX_H*rs + IDX_H*cs] += d;
  J[IDX_H*rs + IDX_H*cs] += d;
  d = k[17]*n[IDX_H];
  J[IDX_H2*rs + IDX_H2*cs] -= d;
  J[IDX_H*rs + IDX_H2*cs] -= d;
  J[IDX_H*rs + IDX_H2*cs] += d;
  J[IDX_H*rs + IDX_H2*cs] += d;
  J[IDX_H*rs + IDX_H2*cs] += d;
  d = k[18]*n[IDX_E];
  J[IDX_Hk*rs + IDX_Hk*cs] -= d;
  J[IDX_E*rs + IDX_Hk*cs] -= d;
  J[IDX_H*rs + IDX_Hk*cs] += d;
  J[IDX_E*rs + IDX_Hk*cs] += d;
  J[IDX_E*rs + IDX_Hk*cs] += d;
  d = k[18]*n[IDX_Hk];
  J[IDX_Hk*rs + IDX_E*cs] -= d;
  J[IDX_E*rs + IDX_E*cs] -= d;
  J[IDX_H*rs + IDX_E*cs] += d;
  J[IDX_E*rs + IDX_E*cs] += d;
  J[IDX_E*rs + IDX_E*cs] += d;
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
  J[IDX_Hk*rs + IDX_H*cs] -= d;
  J[IDX_H*rs + IDX_H*cs] -= d;
  J[IDX_H*rs + IDX_H*cs] += d;
  J[IDX_H*rs + IDX_H*cs] += d;
  J[IDX_E*rs + IDX_H*cs] += d;
  d = k[20]*n[IDX_H];
  J[IDX_Hk*rs + IDX_Hk*cs] -= d;
  J[IDX_H*rs + IDX_Hk*cs] -= d;
  J[IDX_H*rs + IDX_Hk*cs] += d;
  J[IDX_H*rs + IDX_Hk*cs] += d;
  J[IDX_E*rs + IDX_Hk*cs] += d;
  d = k[21]*n[IDX_Hk];
  J[IDX_Hk*rs + IDX_Hj*cs] -= d;
  J[IDX_Hj*rs + IDX_Hj*cs] -= d;
  J[IDX_H*rs + IDX_Hj*cs] += d;
  J[IDX_H*rs + IDX_Hj*cs] += d;
  d = k[21]*n[IDX_Hj];
  J[IDX_Hk*rs + IDX_Hk*cs] -= d;
  J[IDX_Hj*rs + IDX_Hk*cs] -= d;
  J[IDX_H*rs + IDX_Hk*cs] += d;
  J[IDX_H*rs + IDX_Hk*cs] += d;
  d = k[22]*n[IDX_Hk];
  J[IDX_Hk*rs + IDX_Hj*cs] -= d;
  J[IDX_Hj*rs + IDX_Hj*cs] -= d;
  J[IDX_H2j*rs + IDX_Hj*cs] += d;
  J[IDX_E*rs + IDX_Hj*cs] += d;
  d = k[22]*n[IDX_Hj];
  J[IDX_Hk*rs + IDX_Hk*cs] -= d;
  J[IDX_Hj*rs + IDX_Hk*cs] -= d;
  J[IDX_H2j*rs + IDX_Hk*cs] += d;
  J[IDX_E*rs + IDX_Hk*cs] += d;
  d = k[23]*n[IDX_E];
  J[IDX_H2j*rs + IDX_H2j*cs] -= d;
  J[IDX_E*rs + IDX_H2j*cs] -= d;
  J[IDX_H*rs + IDX_H2j*cs] += d;
  J[IDX_H*rs + IDX_H2j*cs] += d;
  d = k[23]*n[IDX_H2j];
  J[IDX_H2j*rs + IDX_E*cs] -= d;
  J[IDX_E*rs + IDX_E*cs] -= d;
  J[IDX_H*rs + IDX_E*cs] += d;
  J[IDX_H*rs + IDX_E*cs] += d;
  d = k[24]*n[IDX_E];
  J[IDX_H2j*rs + IDX_H2j*cs] -= d;
  J[IDX_E*rs + IDX_H2j*cs] -= d;
  J[IDX_H*rs + IDX_H2j*cs] += d;
  J[IDX_H*rs + IDX_H2j*cs] += d;
  d = k[24]*n[IDX_H2j];
  J[IDX_H2j*rs + IDX_E*cs] -= d;
  J[IDX_E*rs + IDX_E*cs] -= d;
  J[IDX_H*rs + IDX_E*cs] += d;
  J[IDX_H*rs + IDX_E*cs] += d;
  d = k[25]*n[IDX_H2j];
  J[IDX_H2j*rs + IDX_Hk*cs] -= d;
  J[IDX_Hk*rs + IDX_Hk*cs] -= d;
  J[IDX_H*rs + IDX_Hk*cs] += d;
  J[IDX_H2*rs + IDX_Hk*cs] += d;
  d = k[25]*n[IDX_Hk];
  J[IDX_H2j*rs + IDX_H2j*cs] -= d;
  J[IDX_Hk*rs + IDX_H2j*cs] -= d;
  J[IDX_H*rs + IDX_H2j*cs] += d;
  J[IDX_H2*rs + IDX_H2j*cs] += d;
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
  d = k[30]*n[IDX_Hej];
  J[IDX_H2*rs + IDX_H2*cs] -= d;
  J[IDX_Hej*rs + IDX_H2*cs] -= d;
  J[IDX_He*rs + IDX_H2*cs] += d;
  J[IDX_H*rs + IDX_H2*cs] += d;
  J[IDX_Hj*rs + IDX_H2*cs] += d;
  d = k[30]*n[IDX_H2];
  J[IDX_H2*rs + IDX_Hej*cs] -= d;
  J[IDX_Hej*rs + IDX_Hej*cs] -= d;
  J[IDX_He*rs + IDX_Hej*cs] += d;
  J[IDX_H*rs + IDX_Hej*cs] += d;
  J[IDX_Hj*rs + IDX_Hej*cs] += d;
  d = k[31]*n[IDX_He];
  J[IDX_H2*rs + IDX_H2*cs] -= d;
  J[IDX_He*rs + IDX_H2*cs] -= d;
  J[IDX_H*rs + IDX_H2*cs] += d;
  J[IDX_H*rs + IDX_H2*cs] += d;
  J[IDX_He*rs + IDX_H2*cs] += d;
  d = k[31]*n[IDX_H2];
  J[IDX_H2*rs + IDX_He*cs] -= d;
  J[IDX_He*rs + IDX_He*cs] -= d;
  J[IDX_H*rs + IDX_He*cs] += d;
  J[IDX_H*rs + IDX_He*cs] += d;
  J[IDX_He*rs + IDX_He*cs] += d;
  d = k[32]*n[IDX_Hej];
  J[IDX_H2*rs + IDX_H2*cs] -= d;
  J[IDX_Hej*rs + IDX_H2*cs] -= d;
  J[IDX_H2j*rs + IDX_H2*cs] += d;
  J[IDX_He*rs + IDX_H2*cs] += d;
  d = k[32]*n[IDX_H2];
  J[IDX_H2*rs + IDX_Hej*cs] -= d;
  J[IDX_Hej*rs + IDX_Hej*cs] -= d;
  J[IDX_H2j*rs + IDX_Hej*cs] += d;
  J[IDX_He*rs + IDX_Hej*cs] += d;
  d = 2.0*k[33]*n[IDX_H];
  J[IDX_H*rs + IDX_H*cs] -= d;
  J[IDX_H*rs + IDX_H*cs] -= d;
  J[IDX_H*rs + IDX_H*cs] += d;
  J[IDX_Hj*rs + IDX_H*cs] += d;
  J[IDX_E*rs + IDX_H*cs] += d;
  d = k[34]*n[IDX_He];
  J[IDX_H*rs + IDX_H*cs] -= d;
  J[IDX_He*rs + IDX_H*cs] -= d;
  J[IDX_He*rs + IDX_H*cs] += d;
  J[IDX_Hj*rs + IDX_H*cs] += d;
  J[IDX_E*rs + IDX_H*cs] += d;
  d = k[34]*n[IDX_H];
  J[IDX_H*rs + IDX_He*cs] -= d;
  J[IDX_He*rs + IDX_He*cs] -= d;
  J[IDX_He*rs + IDX_He*cs] += d;
  J[IDX_Hj*rs + IDX_He*cs] += d;
  J[IDX_E*rs + IDX_He*cs] += d;
  d = k[35];
  J[IDX_H*rs + IDX_H*cs] -= d;
  J[IDX_Hj*rs + IDX_H*cs] += d;
  J[IDX_E*rs + IDX_H*cs] += d;
  d = k[36];
  J[IDX_He*rs + IDX_He*cs] -= d;
  J[IDX_Hej*rs + IDX_He*cs] += d;
  J[IDX_E*rs + IDX_He*cs] += d;
  d = k[37];
  J[IDX_Hej*rs + IDX_Hej*cs] -= d;
  J[IDX_Hejj*rs + IDX_Hej*cs] += d;
  J[IDX_E*rs + IDX_Hej*cs] += d;
  d = k[38];
  J[IDX_Hk*rs + IDX_Hk*cs] -= d;
  J[IDX_H*rs + IDX_Hk*cs] += d;
  J[IDX_E*rs + IDX_Hk*cs] += d;
  d = k[39];
  J[IDX_H2*rs + IDX_H2*cs] -= d;
  J[IDX_H2j*rs + IDX_H2*cs] += d;
  J[IDX_E*rs + IDX_H2*cs] += d;
  d = k[40];
  J[IDX_H2j*rs + IDX_H2j*cs] -= d;
  J[IDX_Hj*rs + IDX_H2j*cs] += d;
  J[IDX_H*rs + IDX_H2j*cs] += d;
  d = k[41];
  J[IDX_H2j*rs + IDX_H2j*cs] -= d;
  J[IDX_Hj*rs + IDX_H2j*cs] += d;
  J[IDX_Hj*rs + IDX_H2j*cs] += d;
  J[IDX_E*rs + IDX_H2j*cs] += d;
  d = k[42];
  J[IDX_H2*rs + IDX_H2*cs] -= d;
  J[IDX_H*rs + IDX_H2*cs] += d;
  J[IDX_H*rs + IDX_H2*cs] += d;
  d = k[43];
  J[IDX_H2*rs + IDX_H2*cs] -= d;
  J[IDX_H*rs + IDX_H2*cs] += d;
  J[IDX_H*rs + IDX_H2*cs] += d;
  d = k[44]*n[IDX_E];
  J[IDX_Hj*rs + IDX_Hj*cs] -= d;
  J[IDX_E*rs + IDX_Hj*cs] -= d;
  J[IDX_H*rs + IDX_Hj*cs] += d;
  d = k[44]*n[IDX_Hj];
  J[IDX_Hj*rs + IDX_E*cs] -= d;
  J[IDX_E*rs + IDX_E*cs] -= d;
  J[IDX_H*rs + IDX_E*cs] += d;
  d = k[45]*n[IDX_E];
  J[IDX_Hej*rs + IDX_Hej*cs] -= d;
  J[IDX_E*rs + IDX_Hej*cs] -= d;
  J[IDX_He*rs + IDX_Hej*cs] += d;
  d = k[45]*n[IDX_Hej];
  J[IDX_Hej*rs + IDX_E*cs] -= d;
  J[IDX_E*rs + IDX_E*cs] -= d;
  J[IDX_He*rs + IDX_E*cs] += d;
}

// H2 -> H + H
KB_HD inline double rate_43(double Tgas, const double* n, const Params& p, double Tg_) {
  (void)Tgas; (void)n; (void)p; (void)Tg_;
  return H2_solomonLW(v_myflux_eV(Tgas, n, p), Tgas, n, p);
}
// H+ + e- -> H
KB_HD inline double rate_44(double Tgas, const double* n, const Params& p, double Tg_) {
  (void)Tgas; (void)n; (void)p; (void)Tg_;
  return H_recombination_on_dust(Tgas, n, p);
}
// He+ + e- -> He
KB_HD inline double rate_45(double Tgas, const double* n, const Params& p, double Tg_) {
  (void)Tgas; (void)n; (void)p; (void)Tg_;
  return He_recombination_on_dust(Tgas, n, p);
}
// the rate-derivative part of the analytic Jacobian (J[i*jrs_ + j*cs], added to;
// U[NSPEC][NAGG] written), gated and clamped like the rates
KB_HD inline void jac_dk(double Tgas, const double* n, const Params& p, const double* k, double* J, double* U, long jrs_, long jcs_) {
  (void)Tgas; (void)n; (void)p; (void)k; (void)J; (void)jrs_; (void)jcs_;
  for (int i = 0; i < NSPEC * NAGG; ++i) U[i] = 0.0;
  double d;
  (void)d;
  { // numerical dk/dn: H2 -> H + H (extern/table in rate, all species)
    double np_[NSPEC];
    for (int q = 0; q < NSPEC; ++q) np_[q] = n[q];
    auto rf_ = [&](const double* x) { return rate_43(Tgas, x, p, Tgas); };
    const double pr_ = n[IDX_H2];
    for (int jj = 0; jj < NSPEC; ++jj) {
      const double dk_ = fd_dk_(rf_, np_, n, k[43], jj);
      if (dk_ == 0.0) continue;
      d = dk_ * pr_;
      J[IDX_H2*jrs_ + jj*jcs_] -= d;
      J[IDX_H*jrs_ + jj*jcs_] += d;
      J[IDX_H*jrs_ + jj*jcs_] += d;
    }
  }
  { // numerical dk/dn: H+ + e- -> H (extern/table in rate, all species)
    double np_[NSPEC];
    for (int q = 0; q < NSPEC; ++q) np_[q] = n[q];
    auto rf_ = [&](const double* x) { return rate_44(Tgas, x, p, Tgas); };
    const double pr_ = n[IDX_Hj]*n[IDX_E];
    for (int jj = 0; jj < NSPEC; ++jj) {
      const double dk_ = fd_dk_(rf_, np_, n, k[44], jj);
      if (dk_ == 0.0) continue;
      d = dk_ * pr_;
      J[IDX_Hj*jrs_ + jj*jcs_] -= d;
      J[IDX_E*jrs_ + jj*jcs_] -= d;
      J[IDX_H*jrs_ + jj*jcs_] += d;
    }
  }
  { // numerical dk/dn: He+ + e- -> He (extern/table in rate, all species)
    double np_[NSPEC];
    for (int q = 0; q < NSPEC; ++q) np_[q] = n[q];
    auto rf_ = [&](const double* x) { return rate_45(Tgas, x, p, Tgas); };
    const double pr_ = n[IDX_Hej]*n[IDX_E];
    for (int jj = 0; jj < NSPEC; ++jj) {
      const double dk_ = fd_dk_(rf_, np_, n, k[45], jj);
      if (dk_ == 0.0) continue;
      d = dk_ * pr_;
      J[IDX_Hej*jrs_ + jj*jcs_] -= d;
      J[IDX_E*jrs_ + jj*jcs_] -= d;
      J[IDX_He*jrs_ + jj*jcs_] += d;
    }
  }
  {  // group 1: H+ + e- -> H
    double T = Tgas;
    if (T < 5500.0) {
    }
    else if (T >= 5500.0) {
    }
  }
  {  // group 2: He+ + e- -> He
    double T = Tgas;
    if (T < 9284.0) {
    }
    else if (T >= 9284.0) {
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
    if (T > 100000000.0) T = 100000000.0;
    if (T >= 100.0 && T >= 100.0 && T < 100000.0) {
    }
    else if (T >= 100000.0) {
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
    if (T > 10000000.0) T = 10000000.0;
    if (T >= 10.0 && T >= 10.0) {
    }
  }
  {  // group 7: H2+ + e- -> H + H
    double T = Tgas;
    if (T < 617.0) {
    }
    else if (T >= 617.0) {
    }
  }
  {  // group 8: He + H+ -> He+ + H
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
  flux = k[14]*n[IDX_H2]*n[IDX_Hj];
  g[14] += flux * (mu[IDX_H2j] + mu[IDX_H] - mu[IDX_H2] - mu[IDX_Hj]);
  flux = k[15]*n[IDX_H2]*n[IDX_E];
  g[15] += flux * (mu[IDX_H] + mu[IDX_Hk] - mu[IDX_H2] - mu[IDX_E]);
  flux = k[16]*n[IDX_H2]*n[IDX_E];
  g[16] += flux * (mu[IDX_H] + mu[IDX_H] + mu[IDX_E] - mu[IDX_H2] - mu[IDX_E]);
  flux = k[17]*n[IDX_H2]*n[IDX_H];
  g[17] += flux * (mu[IDX_H] + mu[IDX_H] + mu[IDX_H] - mu[IDX_H2] - mu[IDX_H]);
  flux = k[18]*n[IDX_Hk]*n[IDX_E];
  g[18] += flux * (mu[IDX_H] + mu[IDX_E] + mu[IDX_E] - mu[IDX_Hk] - mu[IDX_E]);
  flux = k[19]*n[IDX_Hk]*n[IDX_H];
  g[19] += flux * (mu[IDX_H] + mu[IDX_H] + mu[IDX_E] - mu[IDX_Hk] - mu[IDX_H]);
  flux = k[20]*n[IDX_Hk]*n[IDX_H];
  g[20] += flux * (mu[IDX_H] + mu[IDX_H] + mu[IDX_E] - mu[IDX_Hk] - mu[IDX_H]);
  flux = k[21]*n[IDX_Hk]*n[IDX_Hj];
  g[21] += flux * (mu[IDX_H] + mu[IDX_H] - mu[IDX_Hk] - mu[IDX_Hj]);
  flux = k[22]*n[IDX_Hk]*n[IDX_Hj];
  g[22] += flux * (mu[IDX_H2j] + mu[IDX_E] - mu[IDX_Hk] - mu[IDX_Hj]);
  flux = k[23]*n[IDX_H2j]*n[IDX_E];
  g[23] += flux * (mu[IDX_H] + mu[IDX_H] - mu[IDX_H2j] - mu[IDX_E]);
  flux = k[24]*n[IDX_H2j]*n[IDX_E];
  g[24] += flux * (mu[IDX_H] + mu[IDX_H] - mu[IDX_H2j] - mu[IDX_E]);
  flux = k[25]*n[IDX_H2j]*n[IDX_Hk];
  g[25] += flux * (mu[IDX_H] + mu[IDX_H2] - mu[IDX_H2j] - mu[IDX_Hk]);
  flux = k[26]*n[IDX_H2]*n[IDX_H2];
  g[26] += flux * (mu[IDX_H] + mu[IDX_H] + mu[IDX_H2] - mu[IDX_H2] - mu[IDX_H2]);
  flux = k[27]*n[IDX_Hej]*n[IDX_H];
  g[27] += flux * (mu[IDX_He] + mu[IDX_Hj] - mu[IDX_Hej] - mu[IDX_H]);
  flux = k[28]*n[IDX_He]*n[IDX_Hj];
  g[28] += flux * (mu[IDX_Hej] + mu[IDX_H] - mu[IDX_He] - mu[IDX_Hj]);
  flux = k[29]*n[IDX_He]*n[IDX_Hj];
  g[29] += flux * (mu[IDX_Hej] + mu[IDX_H] - mu[IDX_He] - mu[IDX_Hj]);
  flux = k[30]*n[IDX_H2]*n[IDX_Hej];
  g[30] += flux * (mu[IDX_He] + mu[IDX_H] + mu[IDX_Hj] - mu[IDX_H2] - mu[IDX_Hej]);
  flux = k[31]*n[IDX_H2]*n[IDX_He];
  g[31] += flux * (mu[IDX_H] + mu[IDX_H] + mu[IDX_He] - mu[IDX_H2] - mu[IDX_He]);
  flux = k[32]*n[IDX_H2]*n[IDX_Hej];
  g[32] += flux * (mu[IDX_H2j] + mu[IDX_He] - mu[IDX_H2] - mu[IDX_Hej]);
  flux = k[33]*n[IDX_H]*n[IDX_H];
  g[33] += flux * (mu[IDX_H] + mu[IDX_Hj] + mu[IDX_E] - mu[IDX_H] - mu[IDX_H]);
  flux = k[34]*n[IDX_H]*n[IDX_He];
  g[34] += flux * (mu[IDX_He] + mu[IDX_Hj] + mu[IDX_E] - mu[IDX_H] - mu[IDX_He]);
  flux = k[35]*n[IDX_H];
  g[35] += flux * (mu[IDX_Hj] + mu[IDX_E] - mu[IDX_H]);
  flux = k[36]*n[IDX_He];
  g[36] += flux * (mu[IDX_Hej] + mu[IDX_E] - mu[IDX_He]);
  flux = k[37]*n[IDX_Hej];
  g[37] += flux * (mu[IDX_Hejj] + mu[IDX_E] - mu[IDX_Hej]);
  flux = k[38]*n[IDX_Hk];
  g[38] += flux * (mu[IDX_H] + mu[IDX_E] - mu[IDX_Hk]);
  flux = k[39]*n[IDX_H2];
  g[39] += flux * (mu[IDX_H2j] + mu[IDX_E] - mu[IDX_H2]);
  flux = k[40]*n[IDX_H2j];
  g[40] += flux * (mu[IDX_Hj] + mu[IDX_H] - mu[IDX_H2j]);
  flux = k[41]*n[IDX_H2j];
  g[41] += flux * (mu[IDX_Hj] + mu[IDX_Hj] + mu[IDX_E] - mu[IDX_H2j]);
  flux = k[42]*n[IDX_H2];
  g[42] += flux * (mu[IDX_H] + mu[IDX_H] - mu[IDX_H2]);
  flux = k[43]*n[IDX_H2];
  g[43] += flux * (mu[IDX_H] + mu[IDX_H] - mu[IDX_H2]);
  flux = k[44]*n[IDX_Hj]*n[IDX_E];
  g[44] += flux * (mu[IDX_H] - mu[IDX_Hj] - mu[IDX_E]);
  flux = k[45]*n[IDX_Hej]*n[IDX_E];
  g[45] += flux * (mu[IDX_He] - mu[IDX_Hej] - mu[IDX_E]);
}

// reaction labels: the equation, and the T range of a piece
inline const char* const reaction_names[46] = {"H + e- -> H+ + e- + e-", "H+ + e- -> H [0.0, 5500.0]", "H+ + e- -> H [5500.0, INFINITY]", "He + e- -> He+ + e- + e-", "He+ + e- -> He [0.0, 9284.0]", "He+ + e- -> He [9284.0, INFINITY]", "He+ + e- -> He++ + e- + e-", "He++ + e- -> He+", "H + e- -> H-", "H- + H -> H2 + e-", "H + H+ -> H2+ [0.0, 30.0]", "H + H+ -> H2+ [30.0, INFINITY]", "H2+ + H -> H2 + H+", "H2 + H+ -> H2+ + H [100.0, 100000.0]", "H2 + H+ -> H2+ + H [100000.0, 100000000.0]", "H2 + e- -> H + H-", "H2 + e- -> H + H + e-", "H2 + H -> H + H + H", "H- + e- -> H + e- + e-", "H- + H -> H + H + e- [0.0, 1160.0]", "H- + H -> H + H + e- [1160.0, INFINITY]", "H- + H+ -> H + H [10.0, 10000000.0]", "H- + H+ -> H2+ + e-", "H2+ + e- -> H + H [0.0, 617.0]", "H2+ + e- -> H + H [617.0, INFINITY]", "H2+ + H- -> H + H2", "H2 + H2 -> H + H + H2", "He+ + H -> He + H+", "He + H+ -> He+ + H [0.0, 10000.0]", "He + H+ -> He+ + H [10000.0, INFINITY]", "H2 + He+ -> He + H + H+", "H2 + He -> H + H + He", "H2 + He+ -> H2+ + He", "H + H -> H + H+ + e-", "H + He -> He + H+ + e-", "H -> H+ + e-", "He -> He+ + e-", "He+ -> He++ + e-", "H- -> H + e-", "H2 -> H2+ + e-", "H2+ -> H+ + H", "H2+ -> H+ + H+ + e-", "H2 -> H + H", "H2 -> H + H", "H+ + e- -> H", "He+ + e- -> He"};
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
  fl[14] = k[14]*n[IDX_H2]*n[IDX_Hj];
  fl[15] = k[15]*n[IDX_H2]*n[IDX_E];
  fl[16] = k[16]*n[IDX_H2]*n[IDX_E];
  fl[17] = k[17]*n[IDX_H2]*n[IDX_H];
  fl[18] = k[18]*n[IDX_Hk]*n[IDX_E];
  fl[19] = k[19]*n[IDX_Hk]*n[IDX_H];
  fl[20] = k[20]*n[IDX_Hk]*n[IDX_H];
  fl[21] = k[21]*n[IDX_Hk]*n[IDX_Hj];
  fl[22] = k[22]*n[IDX_Hk]*n[IDX_Hj];
  fl[23] = k[23]*n[IDX_H2j]*n[IDX_E];
  fl[24] = k[24]*n[IDX_H2j]*n[IDX_E];
  fl[25] = k[25]*n[IDX_H2j]*n[IDX_Hk];
  fl[26] = k[26]*n[IDX_H2]*n[IDX_H2];
  fl[27] = k[27]*n[IDX_Hej]*n[IDX_H];
  fl[28] = k[28]*n[IDX_He]*n[IDX_Hj];
  fl[29] = k[29]*n[IDX_He]*n[IDX_Hj];
  fl[30] = k[30]*n[IDX_H2]*n[IDX_Hej];
  fl[31] = k[31]*n[IDX_H2]*n[IDX_He];
  fl[32] = k[32]*n[IDX_H2]*n[IDX_Hej];
  fl[33] = k[33]*n[IDX_H]*n[IDX_H];
  fl[34] = k[34]*n[IDX_H]*n[IDX_He];
  fl[35] = k[35]*n[IDX_H];
  fl[36] = k[36]*n[IDX_He];
  fl[37] = k[37]*n[IDX_Hej];
  fl[38] = k[38]*n[IDX_Hk];
  fl[39] = k[39]*n[IDX_H2];
  fl[40] = k[40]*n[IDX_H2j];
  fl[41] = k[41]*n[IDX_H2j];
  fl[42] = k[42]*n[IDX_H2];
  fl[43] = k[43]*n[IDX_H2];
  fl[44] = k[44]*n[IDX_Hj]*n[IDX_E];
  fl[45] = k[45]*n[IDX_Hej]*n[IDX_E];
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
inline const int photo_reaction_[8] = {35, 36, 37, 38, 39, 40, 41, 42};
inline const int photo_reactant_[8] = {IDX_H, IDX_He, IDX_Hej, IDX_Hk, IDX_H2, IDX_H2j, IDX_H2j, IDX_H2};
inline const double photo_pdiss_[8] = {1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0};
// the photoelectron deposit (E - Eth) of each photo rate: none for
// the Solomon process (line pumping)
inline const bool photo_deposit_[8] = {true, true, true, true, true, true, true, true};
inline const double photo_Emin_[8] = {13.6, 24.59, 54.42, 0.755, 15.4, 2.65, 30.0, 14.159};
inline const double photo_Emax_[8] = {INFINITY, INFINITY, INFINITY, 12398.419843320025, 1239.8419843320025, 13.776022048133363, 90.0, 17.7};
// ---- host: the photo cross sections (photon-bin setup) ----
namespace kbxs {
inline double H2_sigmaLW(double E) {
  auto band = [](double lg) { return 1e-18 * kb_exp10(lg); };
  double l0 = 0.0, w0 = 0.0, l1 = 0.0, w1 = 0.0;
  if (E > 14.675 && E < 16.820) l0 = band(15.1289 - 1.05139 * E);
  else if (E > 16.820 && E < 17.6)
    l0 = band(-31.41 + 1.8042e-2 * E * E * E - 4.2339e-5 * kb_pow(E, 5.0));
  if (E > 14.675 && E < 17.7) w0 = band(13.5311 - 0.9182618 * E);
  if (E > 14.159 && E < 15.302) l1 = band(12.0218406 - 0.819429 * E);
  else if (E > 15.302 && E < 17.2) l1 = band(16.04644 - 1.082438 * E);
  if (E > 14.159 && E < 17.2) w1 = band(12.87367 - 0.85088597 * E);
  const double para = 1.0 / (3.0 + 1.0);
  return para * (l0 + w0) + (1.0 - para) * (l1 + w1);
}
// Verner+96 cross-section fit [cm^2] (as in legacy KROME)
static inline double sigma_v96(double E, double E0, double s0, double ya, double P, double yw, double y0, double y1) {
  const double x = E/E0 - y0;
  const double y = std::sqrt(x*x + y1*y1);
  const double Fy = ((x - 1.0)*(x - 1.0) + yw*yw)
      * kb_pow(y, 0.5*P - 5.5)
      * kb_pow(1.0 + std::sqrt(y/ya), -P);
  return 1e-18 * s0 * Fy;
}

// Verner & Yakovlev 1995 fit of one shell [cm^2], 0 below its
// threshold Eth; above the inner-shell edge the database sums
// them over the shells (Verner's phfit2.f)
static inline double sigma_vy95(double E, double Eth, double E0, double s0, double ya, double P, double yw, double l) {
  if (E < Eth) return 0.0;
  const double y = E/E0;
  return 1e-18 * s0 * ((y - 1.0)*(y - 1.0) + yw*yw)
      * kb_pow(y, 0.5*P - 5.5 - l)
      * kb_pow(1.0 + std::sqrt(y/ya), -P);
}

// linear interpolation on a tabulated cross section;
// zero outside the tabulated range
static inline double xsec_interp(double E, const double* tE, const double* tS, int n) {
  if (E < tE[0] || E > tE[n-1]) return 0.0;
  int lo = 0, hi = n - 1;
  while (hi - lo > 1) {
    int m = (lo + hi) / 2;
    if (tE[m] <= E) lo = m; else hi = m;
  }
  const double f = (E - tE[lo]) / (tE[lo+1] - tE[lo]);
  return tS[lo] + f * (tS[lo+1] - tS[lo]);
}
// exact integral of that interpolant over [a, b] [cm^2 eV]
// (the Doppler broadening of PhotoModule::init)
static inline double xsec_int(double a, double b, const double* tE, const double* tS, int n) {
  a = std::fmax(a, tE[0]);
  b = std::fmin(b, tE[n-1]);
  if (!(b > a)) return 0.0;
  int i = 0, hi = n - 1;
  while (hi - i > 1) {
    int m = (i + hi) / 2;
    if (tE[m] <= a) i = m; else hi = m;
  }
  double s = 0.0;
  for (; i < n - 1 && tE[i] < b; ++i) {
    const double l = std::fmax(a, tE[i]);
    const double r = std::fmin(b, tE[i+1]);
    if (!(r > l)) continue;
    const double g = (tS[i+1] - tS[i]) / (tE[i+1] - tE[i]);
    s += 0.5 * (2.0 * tS[i] + g * (l + r - 2.0 * tE[i])) * (r - l);
  }
  return s;
}

// xsec of H -> H+ + e- [cm^2]
static inline double photo_xsec_0(double E_eV) {
  (void)E_eV;
  return sigma_v96(E_eV, 4.298e-01, 5.475e+04, 3.288e+01, 2.963e+00, 0.000e+00, 0.000e+00, 0.000e+00);
}
// xsec of He -> He+ + e- [cm^2]
static inline double photo_xsec_1(double E_eV) {
  (void)E_eV;
  return sigma_v96(E_eV, 1.361e+01, 9.492e+02, 1.469e+00, 3.188e+00, 2.039e+00, 4.434e-01, 2.136e+00);
}
// xsec of He+ -> He++ + e- [cm^2]
static inline double photo_xsec_2(double E_eV) {
  (void)E_eV;
  return sigma_v96(E_eV, 1.720e+00, 1.369e+04, 3.288e+01, 2.963e+00, 0.000e+00, 0.000e+00, 0.000e+00);
}
// tabulated xsec of H- -> H + e-: 116 points, 0.7542-1.24e+04 eV
inline const double xsec_tab_3_E[116] = {
  0.7542076673349976, 0.7749012402075016, 0.7998980544077435, 0.8265613228880017, 0.8550634374703466, 0.8856014173800019, 0.9184014698755575, 0.9537246033323097,
  0.9918735874656021, 1.0170976081476641, 1.0332016536100022, 1.0781234646365239, 1.127129076665457, 1.1808018898400023, 1.2398419843320025, 1.2888170315301481,
  1.377602204813336, 1.4586376286258853, 1.5498024804150032, 1.5615138341712878, 1.6531226457760033, 1.7712028347600037, 1.834085775639057, 1.8505104243761232,
  1.9074492066646194, 2.0664033072200043, 2.254258153330914, 2.3481855763863684, 2.4310627143764756, 2.479683968664005, 2.637961668791495, 2.755204409626672,
  2.8833534519348896, 3.0996049608300065, 3.179082011107699, 3.46324576629051, 3.5424056695200075, 3.999490272038718, 4.132806614440009, 4.592007349377787,
  4.82428787677822, 4.95936793732801, 5.39061732318262, 6.199209921660013, 6.888011024066681, 7.293188143129426, 7.560012099585381, 7.7490124020750155,
  8.265613228880017, 8.856014173800018, 8.91972650598563, 9.537246033323097, 10.24662796968597, 10.33201653610002, 11.271290766654568, 12.398419843320026,
  13.594758600131607, 14.359995185684532, 14.631130331980206, 15.720070804260207, 16.535635960682885, 17.080065908968212, 19.805782497316333, 22.522106890681243,
  24.796839686640052, 25.251364243014308, 27.97477401471125, 30.689158028019865, 32.321219612408825, 36.14699662775518, 41.605435715839015, 46.96371152772737,
  48.374638483496, 52.535677302203496, 55.177658403738434, 57.936541323925354, 63.25724409857156, 68.76550107221311, 68.88011024066681, 69.81092254121636,
  72.80340483452746, 75.92418765045943, 79.22312998926533, 82.60106491219204, 86.1599711141072, 89.84362205304366, 93.71443570158749, 97.70228402931461,
  101.87690914806923, 106.33293176089217, 110.89820968980345, 115.54911317166847, 120.6071969194555, 125.74462315740392, 131.2002099822225, 136.84790114039765,
  142.67456666651353, 148.84057434958015, 155.1742158112644, 161.85926688407346, 168.6859842628575, 175.86411125276632, 191.62936388438987, 208.3768040894122,
  226.66215435685604, 246.48946010576591, 279.2436901648654, 303.8828392970595, 359.37448821217464, 426.0625375711349, 504.00080663902537, 619.9209921660013,
  799.8980544077435, 1239.8419843320025, 2384.311508330774, 12398.419843320025
};
inline const double xsec_tab_3_S[116] = {
  1e-25, 1.69e-18, 4e-18, 7.11e-18, 1.06e-17, 1.45e-17, 1.83e-17, 2.19e-17,
  2.54e-17, 2.81e-17, 2.86e-17, 3.14e-17, 3.39e-17, 3.59e-17, 3.74e-17, 3.99e-17,
  3.94e-17, 3.95e-17, 3.92e-17, 3.95e-17, 3.91e-17, 3.7e-17, 3.75e-17, 3.69e-17,
  3.55e-17, 3.35e-17, 3.18e-17, 3.02e-17, 2.97e-17, 2.84e-17, 2.74e-17, 2.56e-17,
  2.49e-17, 2.23e-17, 2.21e-17, 1.97e-17, 1.89e-17, 1.69e-17, 1.65e-17, 1.42e-17,
  1.31e-17, 1.29e-17, 1.15e-17, 9.53e-18, 8.25e-18, 7.62e-18, 7.29e-18, 7e-18,
  6.4e-18, 5.81e-18, 5.91e-18, 5.23e-18, 4.93e-18, 4.67e-18, 4.12e-18, 3.65e-18,
  3.5e-18, 3.4e-18, 3.07e-18, 2.88e-18, 2.69e-18, 2.54e-18, 2.33e-18, 1.83e-18,
  1.5e-18, 1.24e-18, 9.46e-19, 7.03e-19, 6.06e-19, 4.14e-19, 2.83e-19, 2.06e-19,
  1.92e-19, 1.55e-19, 1.35e-19, 1.17e-19, 8.79e-20, 6.73e-20, 6.48e-20, 5.62e-20,
  4.95e-20, 4.36e-20, 3.84e-20, 3.38e-20, 2.98e-20, 2.62e-20, 2.3e-20, 2.02e-20,
  1.78e-20, 1.57e-20, 1.37e-20, 1.21e-20, 1.06e-20, 9.31e-21, 8.17e-21, 7.16e-21,
  6.28e-21, 5.51e-21, 4.83e-21, 4.23e-21, 3.71e-21, 3.25e-21, 2.49e-21, 1.91e-21,
  1.46e-21, 1.12e-21, 7.44e-22, 5.68e-22, 3.3e-22, 1.91e-22, 8.34e-23, 5.51e-23,
  2.39e-23, 5.59e-24, 6.11e-25, 2e-27
};
static inline double photo_xsec_3(double E_eV) {
  return xsec_interp(E_eV, xsec_tab_3_E, xsec_tab_3_S, 116);
}
static inline double photo_xsec_int_3(double a, double b) {
  return xsec_int(a, b, xsec_tab_3_E, xsec_tab_3_S, 116);
}
// tabulated xsec of H2 -> H2+ + e-: 40 points, 15.46-1240 eV
inline const double xsec_tab_4_E[40] = {
  15.459376363241926, 15.603347399093915, 15.634829562824748, 15.77206442350849, 15.794165405503216, 15.930129568701048, 15.956782295135168, 16.070537710071324,
  16.10184395236367, 16.531226457760035, 17.712028347600036, 19.074492066646194, 20.66403307220004, 21.230170964589085, 22.542581533309136, 24.796839686640052,
  27.418000538080552, 28.548053979553362, 28.954740409434905, 32.00418131987617, 33.07127192136577, 34.16483836682289, 34.58415576937246, 35.92703518782969,
  36.999163960966946, 38.314029182076716, 39.37256222076858, 40.90537724618946, 41.66135700040331, 43.733403327407494, 46.5580917886595, 47.5947018937429,
  50.155420078155444, 51.74632655809693, 52.939452789581665, 59.237553002006806, 61.992099216600124, 123.98419843320025, 247.9683968664005, 1239.8419843320025
};
inline const double xsec_tab_4_S[40] = {
  1.71e-18, 5.19e-18, 3.72e-18, 7.1e-18, 5.21e-18, 8.11e-18, 5.21e-18, 7.85e-18,
  7.44e-18, 9e-18, 9.29e-18, 9.15e-18, 7.06e-18, 6.35e-18, 5.09e-18, 3.64e-18,
  3.29e-18, 2.94e-18, 2.8e-18, 2.02e-18, 1.74e-18, 1.46e-18, 1.35e-18, 1.02e-18,
  8.02e-19, 6.08e-19, 4.87e-19, 3.52e-19, 2.87e-19, 1.61e-19, 6.28e-20, 4.17e-20,
  1.57e-20, 8.56e-21, 5.83e-21, 2.38e-21, 1.42e-21, 8.51e-23, 4.63e-24, 4.33e-28
};
static inline double photo_xsec_4(double E_eV) {
  return xsec_interp(E_eV, xsec_tab_4_E, xsec_tab_4_S, 40);
}
static inline double photo_xsec_int_4(double a, double b) {
  return xsec_int(a, b, xsec_tab_4_E, xsec_tab_4_S, 40);
}
// tabulated xsec of H2+ -> H+ + H: 2102 points, 4.133-13.78 eV
inline const double xsec_tab_5_E[2102] = {
  4.132668858811383, 4.1328066144400095, 4.134184675998676, 4.1355636568779275, 4.136943557998007, 4.138324380280383, 4.139706124647756, 4.141088792024058,
  4.142472383334456, 4.143856899505357, 4.145242341464402, 4.146628710140478, 4.14801600646371, 4.149404231365471, 4.150793385778383, 4.152183470636312,
  4.153574486874381, 4.154966435428964, 4.15635931723769, 4.157753133239446, 4.15914788437438, 4.160543571583902, 4.1619401958106845, 4.163337757998666,
  4.164736259093056, 4.166135700040331, 4.167536081788245, 4.16893740528582, 4.170339671483359, 4.171742881332445, 4.17314703578594, 4.174552135797989,
  4.175958182324025, 4.177365176320764, 4.178773118746218, 4.180182010559685, 4.1815918527217635, 4.183002646194342, 4.18441439194061, 4.18582709092506,
  4.187240744113484, 4.188655352472982, 4.190070916971959, 4.191487438580131, 4.192904918268525, 4.194323357009481, 4.195742755776659, 4.197163115545034,
  4.1985844372909, 4.20000672199188, 4.201429970626915, 4.202854184176281, 4.204279363621576, 4.205705509945735, 4.207132624133026, 4.208560707169052,
  4.209989760040757, 4.211419783736423, 4.212850779245677, 4.214282747559493, 4.21571568967019, 4.217149606571438, 4.218584499258261, 4.220020368727035,
  4.221457215975494, 4.222895042002734, 4.224333847809209, 4.225773634396738, 4.227214402768506, 4.228656153929069, 4.230098888884349, 4.231542608641647,
  4.2329873142096375, 4.23443300659837, 4.2358796868192785, 4.237327355885177, 4.238776014810266, 4.240225664610133, 4.241676306301754, 4.2431279409035,
  4.244580569435134, 4.246034192917818, 4.247488812374111, 4.248944428827974, 4.250401043304775, 4.251858656831285, 4.253317270435687, 4.254776885147574,
  4.2562375019979495, 4.257699122019241, 4.259161746245286, 4.26062537571135, 4.262090011454117, 4.263555654511701, 4.265022305923642, 4.26648996673091,
  4.267958637975913, 4.269428320702489, 4.2708990159559175, 4.272370724782918, 4.273843448231654, 4.2753171873517335, 4.2767919431942145, 4.2782677168116034,
  4.2797445092578625, 4.281222321588407, 4.2827011548601135, 4.2841810101313165, 4.285661888461814, 4.2871437909128725, 4.288626718547225, 4.290110672429075,
  4.291595653624102, 4.293081663199455, 4.2945687022237715, 4.296056771767161, 4.297545872901223, 4.299036006699039, 4.300527174235181, 4.302019376585714,
  4.303512614828194, 4.3050068900416765, 4.306502203306714, 4.30799855570536, 4.309495948321178, 4.3109943822392305, 4.312493858546096, 4.3139943783298635,
  4.315495942680135, 4.316998552688032, 4.318502209446195, 4.32000691404879, 4.321512667591505, 4.323019471171557, 4.324527325887697, 4.326036232840205,
  4.3275461931309, 4.329057207863139, 4.330569278141819, 4.332082405073385, 4.3335965897658255, 4.335111833328681, 4.336628136873043, 4.338145501511556,
  4.339663928358428, 4.341183418529421, 4.342703973141866, 4.344225593314656, 4.345748280168253, 4.3472720348246945, 4.348796858407586, 4.350322752042115,
  4.351849716855047, 4.353377753974729, 4.354906864531095, 4.356437049655667, 4.3579683104815565, 4.35950064814347, 4.361034063777709, 4.362568558522177,
  4.364104133516377, 4.365640789901418, 4.367178528820017, 4.3687173514165, 4.370257258836809, 4.3717982522285, 4.37334033274075, 4.374883501524358,
  4.376427759731743, 4.377973108516959, 4.3795195490356855, 4.38106708244524, 4.38261570990457, 4.384165432574267, 4.385716251616564, 4.387268168195338,
  4.388821183476116, 4.390375298626073, 4.391930514814037, 4.393486833210499, 4.395044254987602, 4.396602781319158, 4.398162413380642, 4.3997231523491935,
  4.4012849994036305, 4.402847955724441, 4.404412022493793, 4.405977200895532, 4.407543492115189, 4.409110897339982, 4.410679417758814, 4.412249054562287,
  4.413819808942694, 4.415391682094027, 4.41696467521198, 4.418538789493951, 4.420114026139047, 4.421690386348084, 4.423267871323592, 4.4248464822698175,
  4.4264262203927265, 4.42800708690001, 4.4295890830010825, 4.4311722099070865, 4.432756468830901, 4.434341860987134, 4.4359283875921385, 4.437516049864005,
  4.439104849022566, 4.440694786289408, 4.442285862887863, 4.443878080043021, 4.445471438981724, 4.4470659409325775, 4.448661587125952, 4.450258378793979,
  4.4518563171705665, 4.45345540349139, 4.455055638993901, 4.456657024917336, 4.458259562502707, 4.4598632529928155, 4.4614680976322525, 4.463074097667397,
  4.464681254346427, 4.466289568919318, 4.467899042637848, 4.469509676755598, 4.471121472527958, 4.472734431212132, 4.4743485540671335, 4.4759638423538,
  4.4775802973347885, 4.479197920274577, 4.480816712439475, 4.482436675097624, 4.484057809518998, 4.485680116975408, 4.487303598740509, 4.4889282560898005,
  4.490554090300625, 4.492181102652184, 4.493809294425527, 4.4954386669035635, 4.497069221371066, 4.498700959114669, 4.500333881422877, 4.501967989586067,
  4.503603284896487, 4.505239768648266, 4.506877442137414, 4.508516306661829, 4.510156363521291, 4.511797614017477, 4.51344005945396, 4.5150837011362075,
  4.516728540371595, 4.518374578469398, 4.520021816740805, 4.521670256498917, 4.523319899058747, 4.524970745737236, 4.526622797853242, 4.528276056727548,
  4.529930523682875, 4.531586200043869, 4.533243087137121, 4.534901186291159, 4.536560498836454, 4.538221026105427, 4.539882769432452, 4.541545730153857,
  4.543209909607926, 4.544875309134907, 4.5465419300770185, 4.5482097737784395, 4.549878841585331, 4.551549134845826, 4.553220654910036, 4.554893403130062,
  4.556567380859987, 4.558242589455893, 4.559919030275847, 4.561596704679921, 4.563275614030191, 4.564955759690731, 4.566637143027634, 4.568319765409001,
  4.570003628204949, 4.571688732787621, 4.5733750805311795, 4.575062672811819, 4.576751511007762, 4.578441596499271, 4.580132930668647, 4.581825514900231,
  4.583519350580417, 4.585214439097644, 4.586910781842407, 4.588608380207265, 4.590307235586829, 4.592007349377788, 4.593708722978891, 4.595411357790966,
  4.597115255216918, 4.598820416661731, 4.600526843532478, 4.602234537238318, 4.603943499190504, 4.605653730802388, 4.607365233489419, 4.609078008669155,
  4.61079205776126, 4.61250738218751, 4.614223983371801, 4.615941862740144, 4.61766102172068, 4.619381461743677, 4.621103184241531, 4.62282619064878,
  4.624550482402099, 4.626276060940309, 4.628002927704378, 4.629731084137426, 4.631460531684732, 4.633191271793732, 4.634923305914029, 4.636656635497393,
  4.638391261997765, 4.640127186871268, 4.641864411576199, 4.643602937573044, 4.645342766324477, 4.647083899295363, 4.648826337952767, 4.650570083765952,
  4.652315138206389, 4.6540615027477585, 4.655809178865951, 4.657558168039079, 4.659308471747473, 4.661060091473694, 4.662813028702531, 4.664567284921003,
  4.666322861618378, 4.668079760286155, 4.669837982418089, 4.671597529510184, 4.673358403060696, 4.6751206045701466, 4.676884135541315, 4.6786489974792556,
  4.68041519189129, 4.682182720287019, 4.683951584178326, 4.685721785079375, 4.687493324506627, 4.689266203978831, 4.691040425017037, 4.692815989144598,
  4.694592897887174, 4.696371152772738, 4.698150755331576, 4.699931707096296, 4.701714009601831, 4.703497664385442, 4.705282672986728, 4.707069036947619,
  4.708856757812391, 4.710645837127671, 4.7124362764424275, 4.714228077307995, 4.716021241278064, 4.717815769908686, 4.71961166475829, 4.721408927387672,
  4.72320755936001, 4.725007562240864, 4.7268089375981805, 4.728611687002299, 4.730415812025955, 4.732221314244286, 4.734028195234833, 4.735836456577551,
  4.737646099854806, 4.739457126651386, 4.741269538554504, 4.743083337153799, 4.744898524041342, 4.74671510081165, 4.748533069061672, 4.750352430390815,
  4.752173186400931, 4.753995338696329, 4.755818888883785, 4.757643838572535, 4.759470189374291, 4.761297942903237, 4.763127100776038, 4.764957664611848,
  4.766789636032305, 4.768623016661549, 4.7704578081262135, 4.772294012055438, 4.774131630080873, 4.775970663836682, 4.777811114959548, 4.779652985088677,
  4.781496275865803, 4.783340988935196, 4.785187125943661, 4.787034688540551, 4.788883678377763, 4.790734097109747, 4.792585946393517, 4.794439227888641,
  4.796293943257264, 4.7981500941640975, 4.8000076822764335, 4.801866709264147, 4.8037271767997005, 4.80558908655815, 4.8074524402171495, 4.809317239456954,
  4.81118348596043, 4.813051181413054, 4.814920327502923, 4.816790925920757, 4.818662978359901, 4.820536486516341, 4.822411452088692, 4.824287876778221,
  4.82616576228884, 4.828045110327113, 4.82992592260227, 4.831808200826199, 4.833691946713461, 4.83557716198129, 4.837463848349601, 4.839352007540994,
  4.84124164128076, 4.843132751296886, 4.845025339320058, 4.84691940708367, 4.848814956323828, 4.850711988779354, 4.852610506191792, 4.854510510305414,
  4.856412002867225, 4.85831498562697, 4.860219460337134, 4.862125428752952, 4.864032892632416, 4.865941853736274, 4.867852313828044, 4.86976427467401,
  4.871677738043233, 4.873592705707558, 4.875509179441615, 4.877427161022828, 4.879346652231416, 4.881267654850404, 4.883190170665627, 4.885114201465732,
  4.887039749042187, 4.888966815189286, 4.890895401704153, 4.892825510386751, 4.894757143039884, 4.896690301469206, 4.8986249874832195, 4.900561202893291,
  4.902498949513652, 4.9044382291614035, 4.9063790436565204, 4.908321394821864, 4.910265284483179, 4.912210714469108, 4.914157686611188, 4.916106202743865,
  4.918056264704494, 4.920007874333344, 4.921961033473612, 4.923915743971417, 4.925872007675816, 4.927829826438803, 4.92978920211532, 4.931750136563257,
  4.9337126316434645, 4.935676689219757, 4.937642311158912, 4.939609499330689, 4.941578255607823, 4.94354858186604, 4.945520479984056, 4.947493951843587,
  4.949468999329352, 4.951445624329084, 4.953423828733531, 4.955403614436462, 4.957384983334677, 4.959367937328011, 4.961352478319339, 4.963338608214583,
  4.9653263289227185, 4.96731564235578, 4.969306550428869, 4.971299055060156, 4.97329315817089, 4.975288861685405, 4.9772861675311235, 4.979285077638566,
  4.981285593941353, 4.983287718376217, 4.985291452883003, 4.987296799404677, 4.989303759887335, 4.991312336280204, 4.993322530535654, 4.995334344609198,
  4.997347780459504, 4.9993628400483985, 5.001379525340874, 5.003397838305096, 5.005417780912405, 5.00743935513733, 5.009462562957587, 5.011487406354093,
  5.013513887310969, 5.0155420078155455, 5.017571769858368, 5.019603175433209, 5.021636226537071, 5.023670925170189, 5.025707273336047, 5.027745273041374,
  5.029784926296157, 5.031826235113647, 5.033869201510364, 5.035913827506104, 5.037960115123945, 5.040008066390255, 5.0420576833347, 5.044108967990247,
  5.046161922393174, 5.048216548583073, 5.050272848602862, 5.052330824498789, 5.054390478320435, 5.056451812120729, 5.058514827955948, 5.060579527885726,
  5.0626459139730615, 5.064713988284325, 5.066783752889264, 5.068855209861009, 5.070928361276085, 5.073003209214414, 5.075079755759323, 5.077158002997555,
  5.079237953019266, 5.0813196079180445, 5.083402969790909, 5.085488040738321, 5.087574822864189, 5.089663318275874, 5.0917535290842, 5.093845457403463,
  5.095939105351429, 5.098034475049354, 5.100131568621978, 5.102230388197542, 5.104330935907792, 5.106433213887985, 5.108537224276897, 5.110642969216829,
  5.1127504508536195, 5.114859671336645, 5.1169706328188305, 5.119083337456659, 5.121197787410173, 5.123313984842986, 5.125431931922293, 5.1275516308188696,
  5.129673083707087, 5.131796292764912, 5.133921260173924, 5.136047988119316, 5.138176478789899, 5.140306734378121, 5.142438757080061, 5.1445725490954475,
  5.146708112627658, 5.148845449883733, 5.1509845630743785, 5.153125454413977, 5.1552681261205935, 5.1574125804159845, 5.159558819525604, 5.161706845678613,
  5.163856661107883, 5.166008268050011, 5.168161668745322, 5.170316865437877, 5.172473860375481, 5.1746326558096944, 5.176793253995836, 5.1789556571929936,
  5.181119867664031, 5.183285887675597, 5.185453719498129, 5.187623365405869, 5.189794827676864, 5.1919681085929765, 5.194143210439894, 5.196320135507136,
  5.198498886088062, 5.200679464479877, 5.202861872983646, 5.205046113904294, 5.207232189550621, 5.209420102235306, 5.211609854274917, 5.213801447989919,
  5.215994885704681, 5.218190169747486, 5.220387302450538, 5.222586286149969, 5.224787123185852, 5.226989815902204, 5.229194366646996, 5.231400777772164,
  5.2336090516336125, 5.2358191905912275, 5.238031197008884, 5.240245073254449, 5.2424608216998, 5.244678444720824, 5.24689794469743, 5.249119324013559,
  5.251342585057191, 5.25356773022035, 5.255794761899121, 5.258023682493651, 5.260254494408158, 5.262487200050946, 5.264721801834407, 5.266958302175033,
  5.269196703493424, 5.271437008214297, 5.273679218766494, 5.275923337582991, 5.278169367100905, 5.280417309761511, 5.282667168010238, 5.284918944296687,
  5.287172641074639, 5.289428260802059, 5.291685805941112, 5.293945278958168, 5.296206682323805, 5.298470018512832, 5.300735290004287, 5.303002499281448,
  5.305271648831848, 5.307542741147272, 5.309815778723781, 5.3120907640617085, 5.314367699665678, 5.316646588044609, 5.318927431711724, 5.321210233184561,
  5.3234949949849835, 5.325781719639187, 5.328070409677709, 5.330361067635438, 5.332653696051625, 5.334948297469891, 5.337244874438238, 5.339543429509056,
  5.341843965239133, 5.344146484189667, 5.346450988926273, 5.348757482018994, 5.3510659660423086, 5.353376443575142, 5.355688917200876, 5.358003389507358,
  5.360319863086912, 5.3626383405363445, 5.3649588244569575, 5.367281317454557, 5.369605822139466, 5.371932341126528, 5.374260877035123, 5.376591432489171,
  5.3789240101171485, 5.381258612552095, 5.383595242431623, 5.385933902397928, 5.388274595097796, 5.390617323182621, 5.392962089308407, 5.395308896135782,
  5.397657746330008, 5.400008642560988, 5.40236158750328, 5.404716583836106, 5.407073634243361, 5.4094327414136245, 5.41179390804017, 5.414157136820973,
  5.416522430458728, 5.418889791660851, 5.421259223139496, 5.4236307276115605, 5.426004307798699, 5.4283799664273324, 5.4307577062286585, 5.433137529938663,
  5.435519440298127, 5.437903440052644, 5.440289531952623, 5.442677718753305, 5.445068003214769, 5.447460388101946, 5.449854876184627, 5.452251470237479,
  5.454650173040047, 5.457050987376773, 5.459453916037001, 5.46185896181499, 5.464266127509928, 5.466675415925938, 5.46908682987209, 5.471500372162413,
  5.473916045615907, 5.476333853056549, 5.4787537973133125, 5.481175881220172, 5.483600107616112, 5.486026479345145, 5.48845499925632, 5.490885670203732,
  5.493318495046535, 5.495753476648948, 5.498190617880279, 5.500629921614919, 5.5030713907323685, 5.505515028117242, 5.507960836659275, 5.510408819253346,
  5.512858978799478, 5.515311318202859, 5.517765840373844, 5.520222548227974, 5.522681444685981, 5.525142532673809, 5.527605815122616, 5.53007129496879,
  5.532538975153962, 5.535008858625012, 5.53748094833409, 5.539955247238618, 5.542431758301309, 5.544910484490173, 5.5473914287785355, 5.549874594145043,
  5.552359983573679, 5.554847600053776, 5.557337446580021, 5.559829526152479, 5.5623238417765934, 5.564820396463208, 5.567319193228571, 5.569820235094352,
  5.572323525087653, 5.574829066241019, 5.577336861592455, 5.579846914185431, 5.582359227068901, 5.5848738032973095, 5.587390645930611, 5.589909758034278,
  5.592431142679309, 5.594954802942251, 5.597480741905204, 5.6000089626558385, 5.602539468287405, 5.605072261898747, 5.607607346594314, 5.610144725484175,
  5.6126844016840325, 5.61522637831523, 5.61777065850477, 5.620317245385325, 5.62286614209525, 5.625417351778597, 5.627970877585123, 5.630526722670313,
  5.633084890195378, 5.635645383327286, 5.638208205238757, 5.640773359108293, 5.643340848120177, 5.645910675464494, 5.648482844337143, 5.651057357939848,
  5.6536342194801765, 5.656213432171546, 5.65879499923324, 5.661378923890424, 5.663965209374156, 5.666553858921402, 5.669144875775047, 5.671738263183911,
  5.674334024402759, 5.67693216269232, 5.679532681319298, 5.682135583556383, 5.684740872682268, 5.687348551981664, 5.689958624745309, 5.692571094269985,
  5.695185963858534, 5.6978032368198654, 5.700422916468979, 5.703045006126968, 5.705669509121043, 5.708296428784544, 5.710925768456945, 5.713557531483883,
  5.716191721217164, 5.718828341014772, 5.721467394240899, 5.724108884265941, 5.726752814466526, 5.729399188225521, 5.732048008932051, 5.734699279981512,
  5.73735300477558, 5.740009186722235, 5.74266782923577, 5.745328935736806, 5.747992509652308, 5.7506585544155975, 5.75332707346637, 5.755998070250709,
  5.758671548221099, 5.761347510836444, 5.764025961562077, 5.76670690386978, 5.769390341237798, 5.772076277150851, 5.774764715100153, 5.777455658583424,
  5.780149111104908, 5.782845076175386, 5.785543557312192, 5.788244558039229, 5.790948081886982, 5.793654132392536, 5.796362713099592, 5.7990738275584786,
  5.801787479326172, 5.804503671966305, 5.807222409049193, 5.8099436941518405, 5.81266753085796, 5.815393922757987, 5.818122873449098, 5.820854386535224,
  5.823588465627068, 5.826325114342118, 5.8290643363046675, 5.831806135145827, 5.834550514503542, 5.837297478022612, 5.840047029354699, 5.8427991721583545,
  5.8455539100990235, 5.84831124684907, 5.85107118608779, 5.853833731501429, 5.856598886783197, 5.859366655633283, 5.862137041758879, 5.864910048874185,
  5.867685680700439, 5.870463940965923, 5.873244833405982, 5.876028361763046, 5.878814529786641, 5.88160334123341, 5.884394799867123, 5.887188909458703,
  5.889985673786237, 5.892785096634994, 5.8955871817974455, 5.8983919330732775, 5.901199354269409, 5.9040094492000135, 5.9068222216865305, 5.909637675557687,
  5.912455814649513, 5.915276642805357, 5.918100163875908, 5.920926381719211, 5.923755300200682, 5.92658692319313, 5.929421254576771, 5.9322582982392476,
  5.935098058075647, 5.937940537988519, 5.940785741887891, 5.943633673691289, 5.946484337323755, 5.9493377367178635, 5.952193875813744, 5.955052758559091,
  5.957914388909192, 5.960778770826936, 5.9636459082828415, 5.9665158052550655, 5.969388465729431, 5.972263893699435, 5.975142093166278, 5.978023068138875,
  5.980906822633877, 5.98379336067569, 5.986682686296489, 5.989574803536245, 5.992469716442739, 5.99536742907158, 5.9982679454862255, 6.001171269758,
  6.0040774059661155, 6.006986358197688, 6.009898130547759, 6.012812727119315, 6.015730152023303, 6.018650409378655, 6.0215735033123, 6.0244994379591965,
  6.0274282174623375, 6.030359845972776, 6.0332943276496485, 6.036231666660188, 6.03917186717975, 6.042114933391827, 6.0450608694880685, 6.048009679668306,
  6.05096136814057, 6.053915939121107, 6.056873396834406, 6.0598337455132105, 6.062796989398547, 6.06576313273974, 6.068732179794433, 6.071704134828614,
  6.074679002116623, 6.07765678594119, 6.080637490593442, 6.083621120372928, 6.086607679587643, 6.089597172554042, 6.092589603597065, 6.095584977050161,
  6.098583297255301, 6.101584568563006, 6.104588795332362, 6.107595981931048, 6.110606132735351, 6.11361925213019, 6.116635344509141, 6.1196544142744465,
  6.122676465837051, 6.1257015036166145, 6.128729532041536, 6.131760555548976, 6.134794578584873, 6.137831605603974, 6.14087164106985, 6.1439146894549195,
  6.14696075524047, 6.15000984291668, 6.153061956982644, 6.156117101946389, 6.1591752823249015, 6.1622365026441495, 6.165300767439099, 6.168368081253745,
  6.171438448641129, 6.17451187416336, 6.177588362391643, 6.1806679179062955, 6.183750545296772, 6.18683624916169, 6.1899250341088505, 6.193016904755259,
  6.196111865727151, 6.199209921660014, 6.202311077198613, 6.20541533699701, 6.208522705718592, 6.211633188036086, 6.214746788631593, 6.217863512196604,
  6.220983363432025, 6.224106347048207, 6.227232467764956, 6.2303617303115715, 6.2334941394268615, 6.236629699859169, 6.239768416366395, 6.242910293716026,
  6.246055336685153, 6.249203550060497, 6.25235493863844, 6.25550950722504, 6.258667260636057, 6.261828203696983, 6.264992341243066, 6.268159678119326,
  6.271330219180591, 6.274503969291512, 6.277680933326597, 6.280861116170227, 6.284044522716688, 6.287231157870197, 6.290421026544915, 6.293614133664988,
  6.296810484164564, 6.300010082987819, 6.3032129350889825, 6.3064190454323645, 6.30962841899238, 6.312841060753578, 6.31605697571066, 6.319276168868516,
  6.322498645242238, 6.325724409857157, 6.328953467748866, 6.332185823963242, 6.335421483556479, 6.338660451595106, 6.341902733156024, 6.345148333326524,
  6.348397257204315, 6.351649509897555, 6.354905096524873, 6.358164022215399, 6.361426292108788, 6.36469191135525, 6.367960885115577, 6.371233218561166,
  6.37450891687405, 6.377787985246927, 6.381070428883184, 6.384356252996925, 6.387645462812998, 6.390938063567025, 6.394234060505429, 6.397533458885463,
  6.400836263975234, 6.404142481053733, 6.407452115410867, 6.410765172347481, 6.414081657175389, 6.417401575217406, 6.420724931807368, 6.424051732290169,
  6.427381982021787, 6.430715686369308, 6.434052850710964, 6.4373934804361514, 6.440737580945469, 6.444085157650742, 6.447436215975053, 6.450790761352772,
  6.454148799229583, 6.457510335062515, 6.460875374319973, 6.464243922481766, 6.467615985039139, 6.470991567494796, 6.474370675362938, 6.477753314169293,
  6.481139489451138, 6.484529206757337, 6.487922471648366, 6.491319289696349, 6.494719666485085, 6.498123607610077, 6.501531118678567, 6.504942205309564,
  6.508356873133873, 6.511775127794132, 6.515196974944838, 6.518622420252381, 6.52205146939507, 6.525484128063172, 6.52892040195894, 6.532360296796642,
  6.535803818302598, 6.539250972215204, 6.542701764284975, 6.546156200274566, 6.54961428595881, 6.55307602712475, 6.55654142957167, 6.560010499111126,
  6.563483241566981, 6.566959662775438, 6.570439768585071, 6.573923564856854, 6.5774110574642055, 6.580902252293008, 6.58439715524165, 6.5878957722210565,
  6.59139810915472, 6.5949041719787385, 6.5984139666418455, 6.601927499105446, 6.605444775343648, 6.608965801343299, 6.612490583104015, 6.616019126638221,
  6.619551437971183, 6.623087523141041, 6.626627388198839, 6.630171039208571, 6.633718482247206, 6.637269723404725, 6.640824768784161, 6.644383624501622,
  6.647946296686342, 6.651512791480702, 6.655083115040272, 6.65865727353385, 6.662235273143486, 6.665817120064531, 6.669402820505663, 6.672992380688927,
  6.676585806849773, 6.680183105237084, 6.683784282113223, 6.68738934375406, 6.690998296449016, 6.694611146501095, 6.69822790022692, 6.701848563956772,
  6.705473144034628, 6.709101646818197, 6.712734078678954, 6.716370446002182, 6.7200107551870065, 6.723655012646436, 6.727303224807394, 6.730955398110765,
  6.734611539011422, 6.738271653978276, 6.7419357494943055, 6.745603832056598, 6.74927590817639, 6.7529519843791, 6.756632067204375, 6.760316163206122,
  6.764004278952552, 6.7676964210262165, 6.771392596024046, 6.775092810557392, 6.7787970712520655, 6.782505384748373, 6.786217757701165, 6.789934196779862,
  6.793654708668508, 6.7973793000658045, 6.801107977685149, 6.804840748254681, 6.8085776185173135, 6.812318595230784, 6.8160636851676895, 6.819812895115526,
  6.823566231876735, 6.827323702268738, 6.831085313123983, 6.834851071289982, 6.838620983629358, 6.842395057019883, 6.846173298354516, 6.849955714541451,
  6.853742312504161, 6.857533099181431, 6.861328081527409, 6.865127266511643, 6.868930661119129, 6.872738272350348, 6.876550107221313, 6.880366172763612,
  6.884186476024446, 6.888011024066682, 6.891839823968887, 6.895672882825377, 6.89951020774626, 6.9033518058574765, 6.907197684300851, 6.911047850234129,
  6.914902310831025, 6.918761073281265, 6.922624144790635, 6.9264915325810215, 6.930363243890457, 6.934239285973169, 6.938119666099624, 6.942004391556567,
  6.945893469647074, 6.949786907690598, 6.95368471302301, 6.957586892996649, 6.9614934549803635, 6.965404406359566, 6.969319754536271, 6.973239506929149,
  6.977163670973567, 6.981092254121638, 6.985025263842269, 6.98896270762121, 6.992904592961098, 6.996850927381506, 7.000801718418988, 7.004756973627134,
  7.0087167005766124, 7.012680906855219, 7.016649600067928, 7.020622787836936, 7.024600477801715, 7.028582677619063, 7.032569394963146, 7.036560637525556,
  7.040556413015348, 7.0445567291591065, 7.048561593700982, 7.052571014402746, 7.0565849990438405, 7.060603555421428, 7.064626691350443, 7.068654414663642,
  7.072686733211652, 7.07672365486303, 7.0807651875043, 7.084811339040016, 7.088862117392812, 7.092917530503448, 7.096977586330869, 7.10104229285225,
  7.105111658063053, 7.10918568997708, 7.113264396626521, 7.117347786062014, 7.121435866352687, 7.125528645586223, 7.129626131868906, 7.133728333325677,
  7.137835258100189, 7.141946914354855, 7.146063310270909, 7.150184454048459, 7.154310353906536, 7.158441018083157, 7.162576454835372, 7.166716672439322,
  7.170861679190299, 7.175011483402793, 7.179166093410555, 7.183325517566645, 7.1874897642434945, 7.191658841832963, 7.195832758746389, 7.200011523414651,
  7.204195144288221, 7.2083836298372255, 7.2125769885515, 7.216775228940644, 7.2209783595340875, 7.225186388881135, 7.229399325551037, 7.233617178133038,
  7.237839955236443, 7.242067665490671, 7.246300317545312, 7.250537920070192, 7.254780481755429, 7.259028011311491, 7.263280517469261, 7.267538008980087,
  7.271800494615852, 7.27606798316903, 7.280340483452746, 7.28461800430084, 7.288900554567918, 7.293188143129428, 7.297480778881711, 7.301778470742065,
  7.306081227648809, 7.310389058561337, 7.314701972460194, 7.319019978347123, 7.323343085245143, 7.327671302198598, 7.332004638273228, 7.33634310255623,
  7.3406867041563215, 7.345035452203807, 7.349389355850639, 7.35374842427048, 7.35811266665877, 7.362482092232796, 7.366856710231745, 7.371236529916783,
  7.375621560571106, 7.380011811500016, 7.384407292030987, 7.3888080115137225, 7.393213979320231, 7.397625204844886, 7.402041697504494, 7.4064634667383675,
  7.410890522008384, 7.41532287279906, 7.419760528617611, 7.424203498994029, 7.4286517934811425, 7.433105421654692, 7.437564393113394, 7.442028717479008,
  7.446498404396413, 7.45097346353367, 7.455453904582097, 7.4599397372563345, 7.4644309712944175, 7.468927616457848, 7.473429682531662, 7.4779371793245035,
  7.482450116668695, 7.4869685044203065, 7.491492352459232, 7.496021670689255, 7.500556469038129, 7.505096757457644, 7.5096425459236995, 7.51419384443638,
  7.518750663020029, 7.523313011723317, 7.5278809006193255, 7.532454339805606, 7.537033339404272, 7.541617909562061, 7.546208060450412, 7.5508038022655475,
  7.555405145228536, 7.560012099585383, 7.564624675607094, 7.56924288358976, 7.573866733854629, 7.578496236748183, 7.583131402642219, 7.587772241933921,
  7.592418765045944, 7.597070982426488, 7.601728904549374, 7.606392541914127, 7.611061905046057, 7.615737004496331, 7.620417850842058, 7.625104454686364,
  7.629796826658478, 7.63449497741381, 7.639198917634028, 7.6439086580271445, 7.648624209327593, 7.653345582296313, 7.658072787720832, 7.662805836415344,
  7.667544739220797, 7.672289507004968, 7.677040150662556, 7.681796681115259, 7.686559109311858, 7.691327446228305, 7.696101702867802, 7.700881890260887,
  7.705668019465524, 7.710460101567181, 7.715258147678923, 7.720062168941487, 7.724872176523382, 7.729688181620965, 7.734510195458532, 7.739338229288407,
  7.744172294391023, 7.749012402075017, 7.753858563677316, 7.758710790563221, 7.763569094126505, 7.768433485789491, 7.7733039770031525, 7.778180579247194,
  7.783063304030149, 7.787952162889465, 7.792847167391595, 7.797748329132093, 7.8026556597356995, 7.80756917085644, 7.812488874177712, 7.817414781412376,
  7.822346904302856, 7.82728525462123, 7.832229844169316, 7.8371806847787795, 7.842137788311213, 7.847101166658246, 7.852070831741626, 7.857046795513325,
  7.86202906995563, 7.867017667081236, 7.872012598933351, 7.877013877585786, 7.882021515143056, 7.887035523740476, 7.892055915544257, 7.89708270275161,
  7.902115897590839, 7.907155512321445, 7.912201559234224, 7.917254050651359, 7.922312998926535, 7.9273784164450305, 7.932450315623817, 7.93752870891167,
  7.942613608789256, 7.947705027769248, 7.952802978396425, 7.95790747324777, 7.963018524932581, 7.968136146092563, 7.973260349401947, 7.978391147567585,
  7.983528553329058, 7.988672579458782, 7.993823238762107, 7.998980544077437, 8.004144508276324, 8.009315144263583, 8.014492464977394, 8.01967648338941,
  8.024867212504873, 8.030064665362712, 8.035268855035662, 8.040479794630368, 8.045697497287494, 8.050921976181836, 8.056153244522434, 8.061391315552683,
  8.066636202550441, 8.071887918828143, 8.077146477732917, 8.082411892646693, 8.087684176986318, 8.092963344203675, 8.09824940778578, 8.10354238125492,
  8.108842278168755, 8.114149112120437, 8.119462896738723, 8.124783645688092, 8.130111372668871, 8.135446091417341, 8.140787815705862, 8.146136559342988,
  8.151492336173588, 8.156855160078965, 8.162225044976976, 8.167602004822152, 8.17298605360582, 8.178377205356218, 8.183775474138631, 8.1891808740555,
  8.194593419246548, 8.200013123888908, 8.20544000219724, 8.210874068423859, 8.216315336858864, 8.221763821830256, 8.227219537704066, 8.232682498884481,
  8.238152719813971, 8.243630214973422, 8.249114998882254, 8.254607086098554, 8.260106491219206, 8.265613228880019, 8.271127313755855, 8.276648760560766,
  8.282177584048116, 8.287713799010714, 8.293257420280955, 8.298808462730943, 8.304366941272624, 8.309932870857928, 8.315506266478891, 8.321087143167803,
  8.326675515997332, 8.332271400080662, 8.33787481057164, 8.34348576266489, 8.349104271595978, 8.354730352641528, 8.36036402111937, 8.366005292388683,
  8.37165418185012, 8.377310704945964, 8.382974877160262, 8.388646714018963, 8.394326231090067, 8.40001344398376, 8.405708368352562, 8.41141101989147,
  8.417121414338103, 8.422839567472845, 8.428565495118987, 8.434299213142875, 8.44004073745407, 8.445790084005468, 8.451547268793476, 8.457312307858137,
  8.463085217283295, 8.46886601319674, 8.474654711770354, 8.480451329220266, 8.486255881807, 8.492068385835635, 8.497888857655948, 8.50371731366257,
  8.509553770295147, 8.515398244038481, 8.5212507514227, 8.527111309023402, 8.53297993346182, 8.538856641404978, 8.544741449565835, 8.550634374703467,
  8.556535433623207, 8.562444643176814, 8.568362020262633, 8.574287581825745, 8.58022134485815, 8.58616332639891, 8.592113543534323, 8.598072013398077,
  8.604038753171428, 8.610013780083353, 8.61599711141072, 8.621988764478461, 8.627988756659727, 8.633997105376064, 8.64001382809758, 8.646038942343115,
  8.65207246568041, 8.658114415726278, 8.66416481014677, 8.670223666657362, 8.676291003023112, 8.682366837058842, 8.688451186629312, 8.694544069649389,
  8.70064550408423, 8.706755507949458, 8.712874099311334, 8.71900129628694, 8.725137117044355, 8.731281579802836, 8.737434702833, 8.743596504457,
  8.749767003048715, 8.755946217033918, 8.76213416489048, 8.768330865148535, 8.774536336390677, 8.780750597252146, 8.786973666420998, 8.793205562638317,
  8.799446304698387, 8.805695911448883, 8.811954401791064, 8.818221794679964, 8.824498109124574, 8.830783364188054, 8.837077578987902, 8.843380772696168,
  8.849692964539635, 8.85601417380002, 8.862344419814173, 8.868683721974268, 8.87503209972801, 8.881389572578817, 8.887756160086042, 8.894131881865155,
  8.900516757587958, 8.90691080698278, 8.913314049834671, 8.919726505985631, 8.926148195334793, 8.932579137838635, 8.939019353511195, 8.945468862424264,
  8.9519276847076, 8.958395840549153, 8.964873350195248, 8.971360233950817, 8.977856512179601, 8.984362205304368, 8.990877333807127, 8.997401918229338,
  9.003935979172134, 9.010479537296533, 9.017032613323657, 9.023595228034955, 9.030167402272415, 9.036749156938797, 9.043340512997833, 9.049941491474472,
  9.056552113455096, 9.063172400087739, 9.069802372582318, 9.076442052210854, 9.083091460307713, 9.089750618269814, 9.096419547556879, 9.103098269691651,
  9.109786806260123, 9.116485178911786, 9.123193409359843, 9.129911519381462, 9.136639530818002, 9.143377465575242, 9.150125345623637, 9.156883192998542,
  9.163651029800462, 9.170428878195288, 9.17721676041453, 9.184014698755576, 9.190822715581932, 9.197640833323462, 9.204469074476636, 9.211307461604775,
  9.21815601733831, 9.22501476437502, 9.231883725480287, 9.238762923487354, 9.24565238129756, 9.252552121880617, 9.259462168274853, 9.266382543587463,
  9.273313270994786, 9.280254373742537, 9.287205875146087, 9.294167798590726, 9.301140167531903, 9.308123005495517, 9.315116336078159, 9.322120182947389,
  9.329134569842006, 9.33615952057231, 9.343195059020369, 9.350241209140293, 9.357297994958511, 9.364365440574039, 9.37144357015875, 9.378532407957662,
  9.385631978289195, 9.392742305545475, 9.399863414192591, 9.406995328770885, 9.414138073895238, 9.421291674255341, 9.42845615461599, 9.435631539817372,
  9.442817854775344, 9.450015124481729, 9.457223374004599, 9.464442628488571, 9.471672913155102, 9.478914253302772, 9.486166674307597, 9.4934302016233,
  9.50070486078163, 9.507990677392659, 9.51528767714507, 9.522595885806474, 9.529915329223696, 9.537246033323099, 9.544588024110876, 9.551941327673363,
  9.559305970177354, 9.566681977870392, 9.574069377081102, 9.581468194219495, 9.588878455777282, 9.596300188328195, 9.603733418528295, 9.6111781731163,
  9.618634478913908, 9.626102362826108, 9.633581851841514, 9.641072973032681, 9.648575753556441, 9.656090220654226, 9.663616401652398, 9.67115432396258,
  9.678704015081989, 9.686265502593772, 9.69383881416734, 9.701423977558708, 9.709021020610829, 9.71662997125394, 9.724250857505904, 9.731883707472548,
  9.73952854934802, 9.747185411415115, 9.754854322045656, 9.762535309700809, 9.770228402931464, 9.777933630378572, 9.785651020773502, 9.793380602938411,
  9.801122405786582, 9.808876458322807, 9.816642789643728, 9.824421428938216, 9.83221240548773, 9.840015748666689, 9.847831487942834, 9.855659652877605,
  9.863500273126514, 9.871353378439514, 9.879218998661377, 9.88709716373208, 9.894987903687174, 9.902891248658168, 9.910807228872924, 9.918735874656022,
  9.926677216429166, 9.93463128471156, 9.942598110120311, 9.95057772337081, 9.958570155277132, 9.966575436752434, 9.974593598809355, 9.982624672560409,
  9.990668689218396, 9.998725680096797, 10.006795676610192, 10.01487871027466, 10.022974812708187, 10.031084015631091, 10.039206350866419, 10.047341850340379,
  10.055490546082748, 10.063652470227295, 10.071827655012209, 10.08001613278051, 10.088217935980493, 10.096433097166146, 10.104661648997578, 10.112903624241458,
  10.121159055771452, 10.12942797656865, 10.137710419722017, 10.146006418428827, 10.15431600599511, 10.162639215836089, 10.170976081476642, 10.179326636551748,
  10.187690914806925, 10.196068950098708, 10.204460776395084, 10.21286642777597, 10.221285938433658, 10.22971934267329, 10.238166674913318, 10.246627969685973,
  10.255103261637739, 10.263592585529825, 10.272095976238631, 10.280613468756242, 10.289145098190895, 10.297690899767465, 10.306250908827954, 10.314825160831969,
  10.323413691357226, 10.332016536100022, 10.340633730875753, 10.349265311619389, 10.357911314385987, 10.366571775351193, 10.375246730811739, 10.383936217185953,
  10.392640271014272, 10.401358928959754, 10.410092227808589, 10.418840204470612, 10.427602895979838, 10.436380339494972, 10.445172572299938, 10.453979631804408,
  10.462801555544328, 10.471638381182455, 10.480490146508899, 10.489356889441648, 10.498238648027119, 10.5071354604407, 10.516047364987301, 10.524974400101891,
  10.533916604350066, 10.542874016428595, 10.551846675165981, 10.560834619523021, 10.569837888593375, 10.578856521604118, 10.587890557916335, 10.596940037025664,
  10.606004998562897, 10.615085482294544, 10.624181528123417, 10.633293176089218, 10.642420466369122, 10.651563439278373, 10.660722135270875, 10.669896594939782,
  10.679086859018112, 10.688292968379335, 10.697514964037987, 10.706752887150284, 10.716006779014716, 10.725276681072689, 10.734562634909114, 10.743864682253056,
  10.753182864978342, 10.76251722510419, 10.771867804795855, 10.781234646365242, 10.790617792271563, 10.800017285121976, 10.809433167672212, 10.818865482827249,
  10.828314273641945, 10.837779583321701, 10.847261455223121, 10.856759932854665, 10.866275059877326, 10.875806880105287, 10.88535543750661, 10.894920776203891,
  10.904502940474957, 10.914101974753546, 10.92371792362998, 10.933350831851875, 10.943000744324825, 10.952667706113099, 10.962351762440344, 10.97205295869029,
  10.981771340407464, 10.991506953297897, 11.001259843229837, 11.011030056234484, 11.020817638506692, 11.030622636405718, 11.040445096455947, 11.050285065347618,
  11.06014258993758, 11.070017717250025, 11.079910494477236, 11.089820968980346, 11.099749188290087, 11.109695200107552, 11.119659052304957, 11.129640792926416,
  11.139640470188704, 11.149658132482038, 11.159693828370862, 11.169747606594619, 11.179819516068555, 11.189909605884502, 11.200017925311677, 11.210144523797494,
  11.22028945096835, 11.23045275663046, 11.24063449077065, 11.250834703557194, 11.261053445340625, 11.271290766654571, 11.281546718216585, 11.291821350928988,
  11.302114715879696, 11.312426864343092, 11.322757847780847, 11.333107717842804, 11.343476526367821, 11.35386432538464, 11.364271167112767, 11.374697103963328,
  11.38514218853997, 11.395606473639731, 11.406090012253935, 11.416592857569087, 11.427115062967767, 11.437656682029544, 11.448217768531881, 11.458798376451043,
  11.469398559963023, 11.48001837344447, 11.490657871473612, 11.501317108831195, 11.511996140501418, 11.522695021672888, 11.53341380773956, 11.544152554301702,
  11.554911317166848, 11.565690152350772, 11.576489116078458, 11.587308264785072, 11.598147655116957, 11.60900734393261, 11.619887388303681, 11.630787845515973,
  11.641708773070448, 11.652650228684236, 11.663612270291654, 11.674594956045224, 11.685598344316709, 11.69662249369814, 11.707667463002858, 11.718733311266567,
  11.72982009774837, 11.740927881931846, 11.752056723526092, 11.76320668246682, 11.774377818917406, 11.785570193269988, 11.796783866146555, 11.808018898400027,
  11.819275351115374, 11.830553285610714, 11.841852763438421, 11.85317384638626, 11.864516596478495, 11.875881075977038, 11.887267347382577, 11.898675473435727,
  11.910105517118183, 11.921557541653872, 11.933031610510131, 11.94452778739887, 11.95604613627775, 11.96758672135138, 11.97914960707249, 11.99073485814316,
  12.002342539516, 12.013972716395376, 12.02562545423863, 12.03730081875731, 12.048998875918393, 12.060719691945552, 12.072463333320377, 12.084229866783653,
  12.096019359336612, 12.107831878242214, 12.119667491026421, 12.13152626547948, 12.143408269657227, 12.15531357188238, 12.167242240745855, 12.179194345108083,
  12.191169954100323, 12.203169137126013, 12.215191963862097, 12.22723850426038, 12.239308828548893, 12.251403007233229, 12.263521111097951, 12.275663211207949,
  12.287829378909839, 12.30001968583336, 12.312234203892778, 12.324473005288299, 12.33673616250749, 12.34902374832672, 12.361335835812591, 12.37367249832338,
  12.386033809510518, 12.398419843320028, 12.41083067399402, 12.423266376072172, 12.435727024393207, 12.448212694096414, 12.460723460623143, 12.473259399718337,
  12.485820587432052, 12.498407100120994, 12.51101901445008, 12.523656407393966, 12.536319356238652, 12.549007938583024, 12.561722232340454, 12.574462315740394,
  12.587228267329976, 12.600020165975637, 12.612838090864729, 12.625682121507156, 12.638552337737032, 12.651448819714314, 12.664371647926483, 12.677320903190212,
  12.690296666653047, 12.70329901979511, 12.716328044430798, 12.7293838227105, 12.742466437122332, 12.755575970493854, 12.76871250599385, 12.78187612713405,
  12.795066917770926, 12.808284962107466, 12.821530344694962, 12.834803150434812, 12.848103464580339, 12.861431372738616, 12.874786960872303, 12.888170315301483,
  12.901581522705545, 12.91502067012503, 12.928487844963533, 12.941983134989592, 12.955506628338586, 12.969058413514674, 12.982638579392699, 12.996247215220153,
  13.009884410619128, 13.023550255588264, 13.037244840504762, 13.050968256126344, 13.064720593593284, 13.078501944430409, 13.092312400549131, 13.1061520542495,
  13.120020998222252, 13.133919325550876, 13.147847129713709, 13.161804504586016, 13.175791544442113, 13.189808343957477, 13.203854998210891, 13.217931602686598,
  13.232038253276443, 13.246175046282081, 13.260342078417143, 13.27453944680945, 13.288767249003245, 13.303025582961403, 13.3173145470677, 13.331634240129063,
  13.345984761377855, 13.360366210474169, 13.37477868750812, 13.38922229300219, 13.403697127913544, 13.418203293636394, 13.432740892004364, 13.447310025292872,
  13.46191079622153, 13.476543307956552, 13.491207664113196, 13.5059039687582, 13.520632326412244, 13.535392842052433, 13.550185621114784, 13.565010769496746,
  13.579868393559725, 13.594758600131609, 13.609681496509362, 13.624637190461568, 13.639625790231053, 13.654647404537476, 13.669702142579965, 13.684790114039766,
  13.699911429082903, 13.715066198362862, 13.730254533023286, 13.745476544700695, 13.760732345527224, 13.776022048133363
};
inline const double xsec_tab_5_S[2102] = {
  0.0, -3.23351e-25, 1.0895e-25, 1.179e-25, 1.2685e-25, 1.358e-25, 1.4475e-25, 1.537e-25,
  1.6265e-25, 1.716e-25, 1.8055e-25, 1.895e-25, 1.9845e-25, 2.074e-25, 2.1635e-25, 2.253e-25,
  2.3425e-25, 2.432e-25, 2.5215e-25, 2.611e-25, 2.7005e-25, 2.79e-25, 2.8795e-25, 2.969e-25,
  3.0585e-25, 3.148e-25, 3.2375e-25, 3.327e-25, 3.4165e-25, 3.506e-25, 3.5955e-25, 3.685e-25,
  3.7745e-25, 3.864e-25, 3.9535e-25, 4.043e-25, 4.1325e-25, 4.222e-25, 4.3115e-25, 4.401e-25,
  4.4905e-25, 4.58e-25, 4.6695e-25, 4.759e-25, 4.8485e-25, 4.938e-25, 5.0275e-25, 5.117e-25,
  5.2065e-25, 5.296e-25, 5.3855e-25, 5.475e-25, 5.5645e-25, 5.654e-25, 5.7435e-25, 5.833e-25,
  5.9225e-25, 6.012e-25, 6.1015e-25, 6.191e-25, 6.2805e-25, 6.37e-25, 6.4595e-25, 6.549e-25,
  6.6385e-25, 6.728e-25, 6.8175e-25, 6.907e-25, 6.9965e-25, 7.086e-25, 7.1755e-25, 7.265e-25,
  7.3545e-25, 7.444e-25, 7.5335e-25, 7.623e-25, 7.7125e-25, 7.802e-25, 7.8915e-25, 7.981e-25,
  8.0705e-25, 8.16e-25, 8.2495e-25, 8.339e-25, 8.4285e-25, 8.518e-25, 8.6075e-25, 8.697e-25,
  8.7865e-25, 8.876e-25, 8.9655e-25, 9.055e-25, 9.1445e-25, 9.234e-25, 9.3235e-25, 9.413e-25,
  9.5025e-25, 9.592e-25, 9.6815e-25, 9.771e-25, 9.8605e-25, 9.95e-25, 1.00395e-24, 1.0129e-24,
  1.02185e-24, 1.0308e-24, 1.03975e-24, 1.0487e-24, 1.05765e-24, 1.0666e-24, 1.07555e-24, 1.0845e-24,
  1.09345e-24, 1.1024e-24, 1.11135e-24, 1.1203e-24, 1.12925e-24, 1.1382e-24, 1.14715e-24, 1.1561e-24,
  1.16505e-24, 1.174e-24, 1.18295e-24, 1.1919e-24, 1.20085e-24, 1.2098e-24, 1.21875e-24, 1.2277e-24,
  1.23665e-24, 1.2456e-24, 1.25455e-24, 1.2635e-24, 1.27245e-24, 1.2814e-24, 1.29035e-24, 1.2993e-24,
  1.30825e-24, 1.3172e-24, 1.32615e-24, 1.3351e-24, 1.34405e-24, 1.353e-24, 1.36195e-24, 1.3709e-24,
  1.37985e-24, 1.3888e-24, 1.39775e-24, 1.4067e-24, 1.41565e-24, 1.4246e-24, 1.43355e-24, 1.4425e-24,
  1.45145e-24, 1.4604e-24, 1.46935e-24, 1.4783e-24, 1.48725e-24, 1.4962e-24, 1.50515e-24, 1.5141e-24,
  1.52305e-24, 1.532e-24, 1.54095e-24, 1.5499e-24, 1.55885e-24, 1.5678e-24, 1.57675e-24, 1.5857e-24,
  1.59465e-24, 1.6036e-24, 1.61255e-24, 1.6215e-24, 1.63045e-24, 1.6394e-24, 1.64835e-24, 1.6573e-24,
  1.66625e-24, 1.6752e-24, 1.68415e-24, 1.6931e-24, 1.70205e-24, 1.711e-24, 1.71995e-24, 1.7289e-24,
  1.73785e-24, 1.7468e-24, 1.75575e-24, 1.7647e-24, 1.77365e-24, 1.7826e-24, 1.79155e-24, 1.8005e-24,
  1.80945e-24, 1.8184e-24, 1.82735e-24, 1.8363e-24, 1.84525e-24, 1.8542e-24, 1.86315e-24, 1.8721e-24,
  1.88105e-24, 1.89e-24, 2.00755e-24, 2.1251e-24, 2.24265e-24, 2.3602e-24, 2.47775e-24, 2.5953e-24,
  2.71285e-24, 2.8304e-24, 2.94795e-24, 3.0655e-24, 3.18305e-24, 3.3006e-24, 3.41815e-24, 3.5357e-24,
  3.65325e-24, 3.7708e-24, 3.88835e-24, 4.0059e-24, 4.12345e-24, 4.241e-24, 4.35855e-24, 4.4761e-24,
  4.59365e-24, 4.7112e-24, 4.82875e-24, 4.9463e-24, 5.06385e-24, 5.1814e-24, 5.29895e-24, 5.4165e-24,
  5.53405e-24, 5.6516e-24, 5.76915e-24, 5.8867e-24, 6.00425e-24, 6.1218e-24, 6.23935e-24, 6.3569e-24,
  6.47445e-24, 6.592e-24, 6.70955e-24, 6.8271e-24, 6.94465e-24, 7.0622e-24, 7.17975e-24, 7.2973e-24,
  7.41485e-24, 7.5324e-24, 7.64995e-24, 7.7675e-24, 7.88505e-24, 8.0026e-24, 8.12015e-24, 8.2377e-24,
  8.35525e-24, 8.4728e-24, 8.59035e-24, 8.7079e-24, 8.82545e-24, 8.943e-24, 9.06055e-24, 9.1781e-24,
  9.29565e-24, 9.4132e-24, 9.53075e-24, 9.6483e-24, 9.76585e-24, 9.8834e-24, 1.000095e-23, 1.01185e-23,
  1.023605e-23, 1.03536e-23, 1.047115e-23, 1.05887e-23, 1.070625e-23, 1.08238e-23, 1.094135e-23, 1.10589e-23,
  1.117645e-23, 1.1294e-23, 1.141155e-23, 1.15291e-23, 1.164665e-23, 1.17642e-23, 1.188175e-23, 1.19993e-23,
  1.211685e-23, 1.22344e-23, 1.235195e-23, 1.24695e-23, 1.258705e-23, 1.27046e-23, 1.282215e-23, 1.29397e-23,
  1.305725e-23, 1.31748e-23, 1.329235e-23, 1.34099e-23, 1.352745e-23, 1.3645e-23, 1.376255e-23, 1.38801e-23,
  1.399765e-23, 1.41152e-23, 1.423275e-23, 1.43503e-23, 1.446785e-23, 1.45854e-23, 1.470295e-23, 1.48205e-23,
  1.493805e-23, 1.50556e-23, 1.517315e-23, 1.52907e-23, 1.540825e-23, 1.55258e-23, 1.564335e-23, 1.57609e-23,
  1.587845e-23, 1.5996e-23, 1.611355e-23, 1.62311e-23, 1.634865e-23, 1.64662e-23, 1.658375e-23, 1.67013e-23,
  1.681885e-23, 1.69364e-23, 1.705395e-23, 1.71715e-23, 1.728905e-23, 1.74066e-23, 1.752415e-23, 1.76417e-23,
  1.775925e-23, 1.78768e-23, 1.799435e-23, 1.81119e-23, 1.822945e-23, 1.8347e-23, 1.846455e-23, 1.85821e-23,
  1.869965e-23, 1.88172e-23, 1.893475e-23, 1.90523e-23, 1.916985e-23, 1.92874e-23, 1.940495e-23, 1.95225e-23,
  1.964005e-23, 1.97576e-23, 1.987515e-23, 1.99927e-23, 2.011025e-23, 2.02278e-23, 2.034535e-23, 2.04629e-23,
  2.058045e-23, 2.0698e-23, 2.081555e-23, 2.09331e-23, 2.105065e-23, 2.11682e-23, 2.128575e-23, 2.14033e-23,
  2.152085e-23, 2.16384e-23, 2.175595e-23, 2.18735e-23, 2.199105e-23, 2.21086e-23, 2.222615e-23, 2.23437e-23,
  2.246125e-23, 2.25788e-23, 2.269635e-23, 2.28139e-23, 2.293145e-23, 2.3049e-23, 2.316655e-23, 2.32841e-23,
  2.340165e-23, 2.35192e-23, 2.363675e-23, 2.37543e-23, 2.387185e-23, 2.39894e-23, 2.410695e-23, 2.42245e-23,
  2.434205e-23, 2.44596e-23, 2.457715e-23, 2.46947e-23, 2.481225e-23, 2.49298e-23, 2.504735e-23, 2.51649e-23,
  2.528245e-23, 2.54e-23, 2.6718e-23, 2.8036e-23, 2.9354e-23, 3.0672e-23, 3.199e-23, 3.3308e-23,
  3.4626e-23, 3.5944e-23, 3.7262e-23, 3.858e-23, 3.9898e-23, 4.1216e-23, 4.2534e-23, 4.3852e-23,
  4.517e-23, 4.6488e-23, 4.7806e-23, 4.9124e-23, 5.0442e-23, 5.176e-23, 5.3078e-23, 5.4396e-23,
  5.5714e-23, 5.7032e-23, 5.835e-23, 5.9668e-23, 6.0986e-23, 6.2304e-23, 6.3622e-23, 6.494e-23,
  6.6258e-23, 6.7576e-23, 6.8894e-23, 7.0212e-23, 7.153e-23, 7.2848e-23, 7.4166e-23, 7.5484e-23,
  7.6802e-23, 7.812e-23, 7.9438e-23, 8.0756e-23, 8.2074e-23, 8.3392e-23, 8.471e-23, 8.6028e-23,
  8.7346e-23, 8.8664e-23, 8.9982e-23, 9.13e-23, 9.2618e-23, 9.3936e-23, 9.5254e-23, 9.6572e-23,
  9.789e-23, 9.9208e-23, 1.00526e-22, 1.01844e-22, 1.03162e-22, 1.0448e-22, 1.05798e-22, 1.07116e-22,
  1.08434e-22, 1.09752e-22, 1.1107e-22, 1.12388e-22, 1.13706e-22, 1.15024e-22, 1.16342e-22, 1.1766e-22,
  1.18978e-22, 1.20296e-22, 1.21614e-22, 1.22932e-22, 1.2425e-22, 1.25568e-22, 1.26886e-22, 1.28204e-22,
  1.29522e-22, 1.3084e-22, 1.32158e-22, 1.33476e-22, 1.34794e-22, 1.36112e-22, 1.3743e-22, 1.38748e-22,
  1.40066e-22, 1.41384e-22, 1.42702e-22, 1.4402e-22, 1.45338e-22, 1.46656e-22, 1.47974e-22, 1.49292e-22,
  1.5061e-22, 1.51928e-22, 1.53246e-22, 1.54564e-22, 1.55882e-22, 1.572e-22, 1.58518e-22, 1.59836e-22,
  1.61154e-22, 1.62472e-22, 1.6379e-22, 1.65108e-22, 1.66426e-22, 1.67744e-22, 1.69062e-22, 1.7038e-22,
  1.71698e-22, 1.73016e-22, 1.74334e-22, 1.75652e-22, 1.7697e-22, 1.78288e-22, 1.79606e-22, 1.80924e-22,
  1.82242e-22, 1.8356e-22, 1.84878e-22, 1.86196e-22, 1.87514e-22, 1.88832e-22, 1.9015e-22, 1.91468e-22,
  1.92786e-22, 1.94104e-22, 1.95422e-22, 1.9674e-22, 1.98058e-22, 1.99376e-22, 2.00694e-22, 2.02012e-22,
  2.0333e-22, 2.04648e-22, 2.05966e-22, 2.07284e-22, 2.08602e-22, 2.0992e-22, 2.11238e-22, 2.12556e-22,
  2.13874e-22, 2.15192e-22, 2.1651e-22, 2.17828e-22, 2.19146e-22, 2.20464e-22, 2.21782e-22, 2.231e-22,
  2.24418e-22, 2.25736e-22, 2.27054e-22, 2.28372e-22, 2.2969e-22, 2.31008e-22, 2.32326e-22, 2.33644e-22,
  2.34962e-22, 2.3628e-22, 2.37598e-22, 2.38916e-22, 2.40234e-22, 2.41552e-22, 2.4287e-22, 2.44188e-22,
  2.45506e-22, 2.46824e-22, 2.48142e-22, 2.4946e-22, 2.50778e-22, 2.52096e-22, 2.53414e-22, 2.54732e-22,
  2.5605e-22, 2.57368e-22, 2.58686e-22, 2.60004e-22, 2.61322e-22, 2.6264e-22, 2.63958e-22, 2.65276e-22,
  2.66594e-22, 2.67912e-22, 2.6923e-22, 2.70548e-22, 2.71866e-22, 2.73184e-22, 2.74502e-22, 2.7582e-22,
  2.77138e-22, 2.78456e-22, 2.79774e-22, 2.81092e-22, 2.8241e-22, 2.83728e-22, 2.85046e-22, 2.86364e-22,
  2.87682e-22, 2.89e-22, 3.01705e-22, 3.1441e-22, 3.27115e-22, 3.3982e-22, 3.52525e-22, 3.6523e-22,
  3.77935e-22, 3.9064e-22, 4.03345e-22, 4.1605e-22, 4.28755e-22, 4.4146e-22, 4.54165e-22, 4.6687e-22,
  4.79575e-22, 4.9228e-22, 5.04985e-22, 5.1769e-22, 5.30395e-22, 5.431e-22, 5.55805e-22, 5.6851e-22,
  5.81215e-22, 5.9392e-22, 6.06625e-22, 6.1933e-22, 6.32035e-22, 6.4474e-22, 6.57445e-22, 6.7015e-22,
  6.82855e-22, 6.9556e-22, 7.08265e-22, 7.2097e-22, 7.33675e-22, 7.4638e-22, 7.59085e-22, 7.7179e-22,
  7.84495e-22, 7.972e-22, 8.09905e-22, 8.2261e-22, 8.35315e-22, 8.4802e-22, 8.60725e-22, 8.7343e-22,
  8.86135e-22, 8.9884e-22, 9.11545e-22, 9.2425e-22, 9.36955e-22, 9.4966e-22, 9.62365e-22, 9.7507e-22,
  9.87775e-22, 1.00048e-21, 1.013185e-21, 1.02589e-21, 1.038595e-21, 1.0513e-21, 1.064005e-21, 1.07671e-21,
  1.089415e-21, 1.10212e-21, 1.114825e-21, 1.12753e-21, 1.140235e-21, 1.15294e-21, 1.165645e-21, 1.17835e-21,
  1.191055e-21, 1.20376e-21, 1.216465e-21, 1.22917e-21, 1.241875e-21, 1.25458e-21, 1.267285e-21, 1.27999e-21,
  1.292695e-21, 1.3054e-21, 1.318105e-21, 1.33081e-21, 1.343515e-21, 1.35622e-21, 1.368925e-21, 1.38163e-21,
  1.394335e-21, 1.40704e-21, 1.419745e-21, 1.43245e-21, 1.445155e-21, 1.45786e-21, 1.470565e-21, 1.48327e-21,
  1.495975e-21, 1.50868e-21, 1.521385e-21, 1.53409e-21, 1.546795e-21, 1.5595e-21, 1.572205e-21, 1.58491e-21,
  1.597615e-21, 1.61032e-21, 1.623025e-21, 1.63573e-21, 1.648435e-21, 1.66114e-21, 1.673845e-21, 1.68655e-21,
  1.699255e-21, 1.71196e-21, 1.724665e-21, 1.73737e-21, 1.750075e-21, 1.76278e-21, 1.775485e-21, 1.78819e-21,
  1.800895e-21, 1.8136e-21, 1.826305e-21, 1.83901e-21, 1.851715e-21, 1.86442e-21, 1.877125e-21, 1.88983e-21,
  1.902535e-21, 1.91524e-21, 1.927945e-21, 1.94065e-21, 1.953355e-21, 1.96606e-21, 1.978765e-21, 1.99147e-21,
  2.004175e-21, 2.01688e-21, 2.029585e-21, 2.04229e-21, 2.054995e-21, 2.0677e-21, 2.080405e-21, 2.09311e-21,
  2.105815e-21, 2.11852e-21, 2.131225e-21, 2.14393e-21, 2.156635e-21, 2.16934e-21, 2.182045e-21, 2.19475e-21,
  2.207455e-21, 2.22016e-21, 2.232865e-21, 2.24557e-21, 2.258275e-21, 2.27098e-21, 2.283685e-21, 2.29639e-21,
  2.309095e-21, 2.3218e-21, 2.334505e-21, 2.34721e-21, 2.359915e-21, 2.37262e-21, 2.385325e-21, 2.39803e-21,
  2.410735e-21, 2.42344e-21, 2.436145e-21, 2.44885e-21, 2.461555e-21, 2.47426e-21, 2.486965e-21, 2.49967e-21,
  2.512375e-21, 2.52508e-21, 2.537785e-21, 2.55049e-21, 2.563195e-21, 2.5759e-21, 2.588605e-21, 2.60131e-21,
  2.614015e-21, 2.62672e-21, 2.639425e-21, 2.65213e-21, 2.664835e-21, 2.67754e-21, 2.690245e-21, 2.70295e-21,
  2.715655e-21, 2.72836e-21, 2.741065e-21, 2.75377e-21, 2.766475e-21, 2.77918e-21, 2.791885e-21, 2.80459e-21,
  2.817295e-21, 2.83e-21, 2.8862e-21, 2.9424e-21, 2.9986e-21, 3.0548e-21, 3.111e-21, 3.1672e-21,
  3.2234e-21, 3.2796e-21, 3.3358e-21, 3.392e-21, 3.4482e-21, 3.5044e-21, 3.5606e-21, 3.6168e-21,
  3.673e-21, 3.7292e-21, 3.7854e-21, 3.8416e-21, 3.8978e-21, 3.954e-21, 4.0102e-21, 4.0664e-21,
  4.1226e-21, 4.1788e-21, 4.235e-21, 4.2912e-21, 4.3474e-21, 4.4036e-21, 4.4598e-21, 4.516e-21,
  4.5722e-21, 4.6284e-21, 4.6846e-21, 4.7408e-21, 4.797e-21, 4.8532e-21, 4.9094e-21, 4.9656e-21,
  5.0218e-21, 5.078e-21, 5.1342e-21, 5.1904e-21, 5.2466e-21, 5.3028e-21, 5.359e-21, 5.4152e-21,
  5.4714e-21, 5.5276e-21, 5.5838e-21, 5.64e-21, 5.6962e-21, 5.7524e-21, 5.8086e-21, 5.8648e-21,
  5.921e-21, 5.9772e-21, 6.0334e-21, 6.0896e-21, 6.1458e-21, 6.202e-21, 6.2582e-21, 6.3144e-21,
  6.3706e-21, 6.4268e-21, 6.483e-21, 6.5392e-21, 6.5954e-21, 6.6516e-21, 6.7078e-21, 6.764e-21,
  6.8202e-21, 6.8764e-21, 6.9326e-21, 6.9888e-21, 7.045e-21, 7.1012e-21, 7.1574e-21, 7.2136e-21,
  7.2698e-21, 7.326e-21, 7.3822e-21, 7.4384e-21, 7.4946e-21, 7.5508e-21, 7.607e-21, 7.6632e-21,
  7.7194e-21, 7.7756e-21, 7.8318e-21, 7.888e-21, 7.9442e-21, 8.0004e-21, 8.0566e-21, 8.1128e-21,
  8.169e-21, 8.2252e-21, 8.2814e-21, 8.3376e-21, 8.3938e-21, 8.45e-21, 8.6045e-21, 8.759e-21,
  8.9135e-21, 9.068e-21, 9.2225e-21, 9.377e-21, 9.5315e-21, 9.686e-21, 9.8405e-21, 9.995e-21,
  1.01495e-20, 1.0304e-20, 1.04585e-20, 1.0613e-20, 1.07675e-20, 1.0922e-20, 1.10765e-20, 1.1231e-20,
  1.13855e-20, 1.154e-20, 1.16945e-20, 1.1849e-20, 1.20035e-20, 1.2158e-20, 1.23125e-20, 1.2467e-20,
  1.26215e-20, 1.2776e-20, 1.29305e-20, 1.3085e-20, 1.32395e-20, 1.3394e-20, 1.35485e-20, 1.3703e-20,
  1.38575e-20, 1.4012e-20, 1.41665e-20, 1.4321e-20, 1.44755e-20, 1.463e-20, 1.47845e-20, 1.4939e-20,
  1.50935e-20, 1.5248e-20, 1.54025e-20, 1.5557e-20, 1.57115e-20, 1.5866e-20, 1.60205e-20, 1.6175e-20,
  1.63295e-20, 1.6484e-20, 1.66385e-20, 1.6793e-20, 1.69475e-20, 1.7102e-20, 1.72565e-20, 1.7411e-20,
  1.75655e-20, 1.772e-20, 1.78745e-20, 1.8029e-20, 1.81835e-20, 1.8338e-20, 1.84925e-20, 1.8647e-20,
  1.88015e-20, 1.8956e-20, 1.91105e-20, 1.9265e-20, 1.94195e-20, 1.9574e-20, 1.97285e-20, 1.9883e-20,
  2.00375e-20, 2.0192e-20, 2.03465e-20, 2.0501e-20, 2.06555e-20, 2.081e-20, 2.09645e-20, 2.1119e-20,
  2.12735e-20, 2.1428e-20, 2.15825e-20, 2.1737e-20, 2.18915e-20, 2.2046e-20, 2.22005e-20, 2.2355e-20,
  2.25095e-20, 2.2664e-20, 2.28185e-20, 2.2973e-20, 2.31275e-20, 2.3282e-20, 2.34365e-20, 2.3591e-20,
  2.37455e-20, 2.39e-20, 2.4304e-20, 2.4708e-20, 2.5112e-20, 2.5516e-20, 2.592e-20, 2.6324e-20,
  2.6728e-20, 2.7132e-20, 2.7536e-20, 2.794e-20, 2.8344e-20, 2.8748e-20, 2.9152e-20, 2.9556e-20,
  2.996e-20, 3.0364e-20, 3.0768e-20, 3.1172e-20, 3.1576e-20, 3.198e-20, 3.2384e-20, 3.2788e-20,
  3.3192e-20, 3.3596e-20, 3.4e-20, 3.4404e-20, 3.4808e-20, 3.5212e-20, 3.5616e-20, 3.602e-20,
  3.6424e-20, 3.6828e-20, 3.7232e-20, 3.7636e-20, 3.804e-20, 3.8444e-20, 3.8848e-20, 3.9252e-20,
  3.9656e-20, 4.006e-20, 4.0464e-20, 4.0868e-20, 4.1272e-20, 4.1676e-20, 4.208e-20, 4.2484e-20,
  4.2888e-20, 4.3292e-20, 4.3696e-20, 4.41e-20, 4.4504e-20, 4.4908e-20, 4.5312e-20, 4.5716e-20,
  4.612e-20, 4.6524e-20, 4.6928e-20, 4.7332e-20, 4.7736e-20, 4.814e-20, 4.8544e-20, 4.8948e-20,
  4.9352e-20, 4.9756e-20, 5.016e-20, 5.0564e-20, 5.0968e-20, 5.1372e-20, 5.1776e-20, 5.218e-20,
  5.2584e-20, 5.2988e-20, 5.3392e-20, 5.3796e-20, 5.42e-20, 5.4604e-20, 5.5008e-20, 5.5412e-20,
  5.5816e-20, 5.622e-20, 5.6624e-20, 5.7028e-20, 5.7432e-20, 5.7836e-20, 5.824e-20, 5.8644e-20,
  5.9048e-20, 5.9452e-20, 5.9856e-20, 6.026e-20, 6.0664e-20, 6.1068e-20, 6.1472e-20, 6.1876e-20,
  6.228e-20, 6.2684e-20, 6.3088e-20, 6.3492e-20, 6.3896e-20, 6.43e-20, 6.5094e-20, 6.5888e-20,
  6.6682e-20, 6.7476e-20, 6.827e-20, 6.9064e-20, 6.9858e-20, 7.0652e-20, 7.1446e-20, 7.224e-20,
  7.3034e-20, 7.3828e-20, 7.4622e-20, 7.5416e-20, 7.621e-20, 7.7004e-20, 7.7798e-20, 7.8592e-20,
  7.9386e-20, 8.018e-20, 8.0974e-20, 8.1768e-20, 8.2562e-20, 8.3356e-20, 8.415e-20, 8.4944e-20,
  8.5738e-20, 8.6532e-20, 8.7326e-20, 8.812e-20, 8.8914e-20, 8.9708e-20, 9.0502e-20, 9.1296e-20,
  9.209e-20, 9.2884e-20, 9.3678e-20, 9.4472e-20, 9.5266e-20, 9.606e-20, 9.6854e-20, 9.7648e-20,
  9.8442e-20, 9.9236e-20, 1.0003e-19, 1.00824e-19, 1.01618e-19, 1.02412e-19, 1.03206e-19, 1.04e-19,
  1.0522e-19, 1.0644e-19, 1.0766e-19, 1.0888e-19, 1.101e-19, 1.1132e-19, 1.1254e-19, 1.1376e-19,
  1.1498e-19, 1.162e-19, 1.1742e-19, 1.1864e-19, 1.1986e-19, 1.2108e-19, 1.223e-19, 1.2352e-19,
  1.2474e-19, 1.2596e-19, 1.2718e-19, 1.284e-19, 1.2962e-19, 1.3084e-19, 1.3206e-19, 1.3328e-19,
  1.345e-19, 1.3572e-19, 1.3694e-19, 1.3816e-19, 1.3938e-19, 1.406e-19, 1.4182e-19, 1.4304e-19,
  1.4426e-19, 1.4548e-19, 1.467e-19, 1.4792e-19, 1.4914e-19, 1.5036e-19, 1.5158e-19, 1.528e-19,
  1.5402e-19, 1.5524e-19, 1.5646e-19, 1.5768e-19, 1.589e-19, 1.6012e-19, 1.6134e-19, 1.6256e-19,
  1.6378e-19, 1.65e-19, 1.6688e-19, 1.6876e-19, 1.7064e-19, 1.7252e-19, 1.744e-19, 1.7628e-19,
  1.7816e-19, 1.8004e-19, 1.8192e-19, 1.838e-19, 1.8568e-19, 1.8756e-19, 1.8944e-19, 1.9132e-19,
  1.932e-19, 1.9508e-19, 1.9696e-19, 1.9884e-19, 2.0072e-19, 2.026e-19, 2.0448e-19, 2.0636e-19,
  2.0824e-19, 2.1012e-19, 2.12e-19, 2.1388e-19, 2.1576e-19, 2.1764e-19, 2.1952e-19, 2.214e-19,
  2.2328e-19, 2.2516e-19, 2.2704e-19, 2.2892e-19, 2.308e-19, 2.3268e-19, 2.3456e-19, 2.3644e-19,
  2.3832e-19, 2.402e-19, 2.4208e-19, 2.4396e-19, 2.4584e-19, 2.4772e-19, 2.496e-19, 2.5148e-19,
  2.5336e-19, 2.5524e-19, 2.5712e-19, 2.59e-19, 2.618e-19, 2.646e-19, 2.674e-19, 2.702e-19,
  2.73e-19, 2.758e-19, 2.786e-19, 2.814e-19, 2.842e-19, 2.87e-19, 2.898e-19, 2.926e-19,
  2.954e-19, 2.982e-19, 3.01e-19, 3.038e-19, 3.066e-19, 3.094e-19, 3.122e-19, 3.15e-19,
  3.178e-19, 3.206e-19, 3.234e-19, 3.262e-19, 3.29e-19, 3.318e-19, 3.346e-19, 3.374e-19,
  3.402e-19, 3.43e-19, 3.458e-19, 3.486e-19, 3.514e-19, 3.542e-19, 3.57e-19, 3.598e-19,
  3.626e-19, 3.654e-19, 3.682e-19, 3.71e-19, 3.738e-19, 3.766e-19, 3.794e-19, 3.822e-19,
  3.85e-19, 3.878e-19, 3.906e-19, 3.934e-19, 3.962e-19, 3.99e-19, 4.0308e-19, 4.0716e-19,
  4.1124e-19, 4.1532e-19, 4.194e-19, 4.2348e-19, 4.2756e-19, 4.3164e-19, 4.3572e-19, 4.398e-19,
  4.4388e-19, 4.4796e-19, 4.5204e-19, 4.5612e-19, 4.602e-19, 4.6428e-19, 4.6836e-19, 4.7244e-19,
  4.7652e-19, 4.806e-19, 4.8468e-19, 4.8876e-19, 4.9284e-19, 4.9692e-19, 5.01e-19, 5.0508e-19,
  5.0916e-19, 5.1324e-19, 5.1732e-19, 5.214e-19, 5.2548e-19, 5.2956e-19, 5.3364e-19, 5.3772e-19,
  5.418e-19, 5.4588e-19, 5.4996e-19, 5.5404e-19, 5.5812e-19, 5.622e-19, 5.6628e-19, 5.7036e-19,
  5.7444e-19, 5.7852e-19, 5.826e-19, 5.8668e-19, 5.9076e-19, 5.9484e-19, 5.9892e-19, 6.03e-19,
  6.0876e-19, 6.1452e-19, 6.2028e-19, 6.2604e-19, 6.318e-19, 6.3756e-19, 6.4332e-19, 6.4908e-19,
  6.5484e-19, 6.606e-19, 6.6636e-19, 6.7212e-19, 6.7788e-19, 6.8364e-19, 6.894e-19, 6.9516e-19,
  7.0092e-19, 7.0668e-19, 7.1244e-19, 7.182e-19, 7.2396e-19, 7.2972e-19, 7.3548e-19, 7.4124e-19,
  7.47e-19, 7.5276e-19, 7.5852e-19, 7.6428e-19, 7.7004e-19, 7.758e-19, 7.8156e-19, 7.8732e-19,
  7.9308e-19, 7.9884e-19, 8.046e-19, 8.1036e-19, 8.1612e-19, 8.2188e-19, 8.2764e-19, 8.334e-19,
  8.3916e-19, 8.4492e-19, 8.5068e-19, 8.5644e-19, 8.622e-19, 8.6796e-19, 8.7372e-19, 8.7948e-19,
  8.8524e-19, 8.91e-19, 8.9878e-19, 9.0656e-19, 9.1434e-19, 9.2212e-19, 9.299e-19, 9.3768e-19,
  9.4546e-19, 9.5324e-19, 9.6102e-19, 9.688e-19, 9.7658e-19, 9.8436e-19, 9.9214e-19, 9.9992e-19,
  1.0077e-18, 1.01548e-18, 1.02326e-18, 1.03104e-18, 1.03882e-18, 1.0466e-18, 1.05438e-18, 1.06216e-18,
  1.06994e-18, 1.07772e-18, 1.0855e-18, 1.09328e-18, 1.10106e-18, 1.10884e-18, 1.11662e-18, 1.1244e-18,
  1.13218e-18, 1.13996e-18, 1.14774e-18, 1.15552e-18, 1.1633e-18, 1.17108e-18, 1.17886e-18, 1.18664e-18,
  1.19442e-18, 1.2022e-18, 1.20998e-18, 1.21776e-18, 1.22554e-18, 1.23332e-18, 1.2411e-18, 1.24888e-18,
  1.25666e-18, 1.26444e-18, 1.27222e-18, 1.28e-18, 1.2906e-18, 1.3012e-18, 1.3118e-18, 1.3224e-18,
  1.333e-18, 1.3436e-18, 1.3542e-18, 1.3648e-18, 1.3754e-18, 1.386e-18, 1.3966e-18, 1.4072e-18,
  1.4178e-18, 1.4284e-18, 1.439e-18, 1.4496e-18, 1.4602e-18, 1.4708e-18, 1.4814e-18, 1.492e-18,
  1.5026e-18, 1.5132e-18, 1.5238e-18, 1.5344e-18, 1.545e-18, 1.5556e-18, 1.5662e-18, 1.5768e-18,
  1.5874e-18, 1.598e-18, 1.6086e-18, 1.6192e-18, 1.6298e-18, 1.6404e-18, 1.651e-18, 1.6616e-18,
  1.6722e-18, 1.6828e-18, 1.6934e-18, 1.704e-18, 1.7146e-18, 1.7252e-18, 1.7358e-18, 1.7464e-18,
  1.757e-18, 1.7676e-18, 1.7782e-18, 1.7888e-18, 1.7994e-18, 1.81e-18, 1.8234e-18, 1.8368e-18,
  1.8502e-18, 1.8636e-18, 1.877e-18, 1.8904e-18, 1.9038e-18, 1.9172e-18, 1.9306e-18, 1.944e-18,
  1.9574e-18, 1.9708e-18, 1.9842e-18, 1.9976e-18, 2.011e-18, 2.0244e-18, 2.0378e-18, 2.0512e-18,
  2.0646e-18, 2.078e-18, 2.0914e-18, 2.1048e-18, 2.1182e-18, 2.1316e-18, 2.145e-18, 2.1584e-18,
  2.1718e-18, 2.1852e-18, 2.1986e-18, 2.212e-18, 2.2254e-18, 2.2388e-18, 2.2522e-18, 2.2656e-18,
  2.279e-18, 2.2924e-18, 2.3058e-18, 2.3192e-18, 2.3326e-18, 2.346e-18, 2.3594e-18, 2.3728e-18,
  2.3862e-18, 2.3996e-18, 2.413e-18, 2.4264e-18, 2.4398e-18, 2.4532e-18, 2.4666e-18, 2.48e-18,
  2.4966e-18, 2.5132e-18, 2.5298e-18, 2.5464e-18, 2.563e-18, 2.5796e-18, 2.5962e-18, 2.6128e-18,
  2.6294e-18, 2.646e-18, 2.6626e-18, 2.6792e-18, 2.6958e-18, 2.7124e-18, 2.729e-18, 2.7456e-18,
  2.7622e-18, 2.7788e-18, 2.7954e-18, 2.812e-18, 2.8286e-18, 2.8452e-18, 2.8618e-18, 2.8784e-18,
  2.895e-18, 2.9116e-18, 2.9282e-18, 2.9448e-18, 2.9614e-18, 2.978e-18, 2.9946e-18, 3.0112e-18,
  3.0278e-18, 3.0444e-18, 3.061e-18, 3.0776e-18, 3.0942e-18, 3.1108e-18, 3.1274e-18, 3.144e-18,
  3.1606e-18, 3.1772e-18, 3.1938e-18, 3.2104e-18, 3.227e-18, 3.2436e-18, 3.2602e-18, 3.2768e-18,
  3.2934e-18, 3.31e-18, 3.3342e-18, 3.3584e-18, 3.3826e-18, 3.4068e-18, 3.431e-18, 3.4552e-18,
  3.4794e-18, 3.5036e-18, 3.5278e-18, 3.552e-18, 3.5762e-18, 3.6004e-18, 3.6246e-18, 3.6488e-18,
  3.673e-18, 3.6972e-18, 3.7214e-18, 3.7456e-18, 3.7698e-18, 3.794e-18, 3.8182e-18, 3.8424e-18,
  3.8666e-18, 3.8908e-18, 3.915e-18, 3.9392e-18, 3.9634e-18, 3.9876e-18, 4.0118e-18, 4.036e-18,
  4.0602e-18, 4.0844e-18, 4.1086e-18, 4.1328e-18, 4.157e-18, 4.1812e-18, 4.2054e-18, 4.2296e-18,
  4.2538e-18, 4.278e-18, 4.3022e-18, 4.3264e-18, 4.3506e-18, 4.3748e-18, 4.399e-18, 4.4232e-18,
  4.4474e-18, 4.4716e-18, 4.4958e-18, 4.52e-18, 4.5354e-18, 4.5508e-18, 4.5662e-18, 4.5816e-18,
  4.597e-18, 4.6124e-18, 4.6278e-18, 4.6432e-18, 4.6586e-18, 4.674e-18, 4.6894e-18, 4.7048e-18,
  4.7202e-18, 4.7356e-18, 4.751e-18, 4.7664e-18, 4.7818e-18, 4.7972e-18, 4.8126e-18, 4.828e-18,
  4.8434e-18, 4.8588e-18, 4.8742e-18, 4.8896e-18, 4.905e-18, 4.9204e-18, 4.9358e-18, 4.9512e-18,
  4.9666e-18, 4.982e-18, 4.9974e-18, 5.0128e-18, 5.0282e-18, 5.0436e-18, 5.059e-18, 5.0744e-18,
  5.0898e-18, 5.1052e-18, 5.1206e-18, 5.136e-18, 5.1514e-18, 5.1668e-18, 5.1822e-18, 5.1976e-18,
  5.213e-18, 5.2284e-18, 5.2438e-18, 5.2592e-18, 5.2746e-18, 5.29e-18, 5.3098e-18, 5.3296e-18,
  5.3494e-18, 5.3692e-18, 5.389e-18, 5.4088e-18, 5.4286e-18, 5.4484e-18, 5.4682e-18, 5.488e-18,
  5.5078e-18, 5.5276e-18, 5.5474e-18, 5.5672e-18, 5.587e-18, 5.6068e-18, 5.6266e-18, 5.6464e-18,
  5.6662e-18, 5.686e-18, 5.7058e-18, 5.7256e-18, 5.7454e-18, 5.7652e-18, 5.785e-18, 5.8048e-18,
  5.8246e-18, 5.8444e-18, 5.8642e-18, 5.884e-18, 5.9038e-18, 5.9236e-18, 5.9434e-18, 5.9632e-18,
  5.983e-18, 6.0028e-18, 6.0226e-18, 6.0424e-18, 6.0622e-18, 6.082e-18, 6.1018e-18, 6.1216e-18,
  6.1414e-18, 6.1612e-18, 6.181e-18, 6.2008e-18, 6.2206e-18, 6.2404e-18, 6.2602e-18, 6.28e-18,
  6.296e-18, 6.312e-18, 6.328e-18, 6.344e-18, 6.36e-18, 6.376e-18, 6.392e-18, 6.408e-18,
  6.424e-18, 6.44e-18, 6.456e-18, 6.472e-18, 6.488e-18, 6.504e-18, 6.52e-18, 6.536e-18,
  6.552e-18, 6.568e-18, 6.584e-18, 6.6e-18, 6.616e-18, 6.632e-18, 6.648e-18, 6.664e-18,
  6.68e-18, 6.696e-18, 6.712e-18, 6.728e-18, 6.744e-18, 6.76e-18, 6.776e-18, 6.792e-18,
  6.808e-18, 6.824e-18, 6.84e-18, 6.856e-18, 6.872e-18, 6.888e-18, 6.904e-18, 6.92e-18,
  6.936e-18, 6.952e-18, 6.968e-18, 6.984e-18, 7e-18, 7.016e-18, 7.032e-18, 7.048e-18,
  7.064e-18, 7.08e-18, 7.0898e-18, 7.0996e-18, 7.1094e-18, 7.1192e-18, 7.129e-18, 7.1388e-18,
  7.1486e-18, 7.1584e-18, 7.1682e-18, 7.178e-18, 7.1878e-18, 7.1976e-18, 7.2074e-18, 7.2172e-18,
  7.227e-18, 7.2368e-18, 7.2466e-18, 7.2564e-18, 7.2662e-18, 7.276e-18, 7.2858e-18, 7.2956e-18,
  7.3054e-18, 7.3152e-18, 7.325e-18, 7.3348e-18, 7.3446e-18, 7.3544e-18, 7.3642e-18, 7.374e-18,
  7.3838e-18, 7.3936e-18, 7.4034e-18, 7.4132e-18, 7.423e-18, 7.4328e-18, 7.4426e-18, 7.4524e-18,
  7.4622e-18, 7.472e-18, 7.4818e-18, 7.4916e-18, 7.5014e-18, 7.5112e-18, 7.521e-18, 7.5308e-18,
  7.5406e-18, 7.5504e-18, 7.5602e-18, 7.57e-18, 7.5708e-18, 7.5716e-18, 7.5724e-18, 7.5732e-18,
  7.574e-18, 7.5748e-18, 7.5756e-18, 7.5764e-18, 7.5772e-18, 7.578e-18, 7.5788e-18, 7.5796e-18,
  7.5804e-18, 7.5812e-18, 7.582e-18, 7.5828e-18, 7.5836e-18, 7.5844e-18, 7.5852e-18, 7.586e-18,
  7.5868e-18, 7.5876e-18, 7.5884e-18, 7.5892e-18, 7.59e-18, 7.5908e-18, 7.5916e-18, 7.5924e-18,
  7.5932e-18, 7.594e-18, 7.5948e-18, 7.5956e-18, 7.5964e-18, 7.5972e-18, 7.598e-18, 7.5988e-18,
  7.5996e-18, 7.6004e-18, 7.6012e-18, 7.602e-18, 7.6028e-18, 7.6036e-18, 7.6044e-18, 7.6052e-18,
  7.606e-18, 7.6068e-18, 7.6076e-18, 7.6084e-18, 7.6092e-18, 7.61e-18, 7.6006e-18, 7.5912e-18,
  7.5818e-18, 7.5724e-18, 7.563e-18, 7.5536e-18, 7.5442e-18, 7.5348e-18, 7.5254e-18, 7.516e-18,
  7.5066e-18, 7.4972e-18, 7.4878e-18, 7.4784e-18, 7.469e-18, 7.4596e-18, 7.4502e-18, 7.4408e-18,
  7.4314e-18, 7.422e-18, 7.4126e-18, 7.4032e-18, 7.3938e-18, 7.3844e-18, 7.375e-18, 7.3656e-18,
  7.3562e-18, 7.3468e-18, 7.3374e-18, 7.328e-18, 7.3186e-18, 7.3092e-18, 7.2998e-18, 7.2904e-18,
  7.281e-18, 7.2716e-18, 7.2622e-18, 7.2528e-18, 7.2434e-18, 7.234e-18, 7.2246e-18, 7.2152e-18,
  7.2058e-18, 7.1964e-18, 7.187e-18, 7.1776e-18, 7.1682e-18, 7.1588e-18, 7.1494e-18, 7.14e-18,
  7.1184e-18, 7.0968e-18, 7.0752e-18, 7.0536e-18, 7.032e-18, 7.0104e-18, 6.9888e-18, 6.9672e-18,
  6.9456e-18, 6.924e-18, 6.9024e-18, 6.8808e-18, 6.8592e-18, 6.8376e-18, 6.816e-18, 6.7944e-18,
  6.7728e-18, 6.7512e-18, 6.7296e-18, 6.708e-18, 6.6864e-18, 6.6648e-18, 6.6432e-18, 6.6216e-18,
  6.6e-18, 6.5784e-18, 6.5568e-18, 6.5352e-18, 6.5136e-18, 6.492e-18, 6.4704e-18, 6.4488e-18,
  6.4272e-18, 6.4056e-18, 6.384e-18, 6.3624e-18, 6.3408e-18, 6.3192e-18, 6.2976e-18, 6.276e-18,
  6.2544e-18, 6.2328e-18, 6.2112e-18, 6.1896e-18, 6.168e-18, 6.1464e-18, 6.1248e-18, 6.1032e-18,
  6.0816e-18, 6.06e-18, 6.0324e-18, 6.0048e-18, 5.9772e-18, 5.9496e-18, 5.922e-18, 5.8944e-18,
  5.8668e-18, 5.8392e-18, 5.8116e-18, 5.784e-18, 5.7564e-18, 5.7288e-18, 5.7012e-18, 5.6736e-18,
  5.646e-18, 5.6184e-18, 5.5908e-18, 5.5632e-18, 5.5356e-18, 5.508e-18, 5.4804e-18, 5.4528e-18,
  5.4252e-18, 5.3976e-18, 5.37e-18, 5.3396e-18, 5.3092e-18, 5.2788e-18, 5.2484e-18, 5.218e-18,
  5.1876e-18, 5.1572e-18, 5.1268e-18, 5.0964e-18, 5.066e-18, 5.0356e-18, 5.0052e-18, 4.9748e-18,
  4.9444e-18, 4.914e-18, 4.8836e-18, 4.8532e-18, 4.8228e-18, 4.7924e-18, 4.762e-18, 4.7316e-18,
  4.7012e-18, 4.6708e-18, 4.6404e-18, 4.61e-18, 4.5784e-18, 4.5468e-18, 4.5152e-18, 4.4836e-18,
  4.452e-18, 4.4204e-18, 4.3888e-18, 4.3572e-18, 4.3256e-18, 4.294e-18, 4.2624e-18, 4.2308e-18,
  4.1992e-18, 4.1676e-18, 4.136e-18, 4.1044e-18, 4.0728e-18, 4.0412e-18, 4.0096e-18, 3.978e-18,
  3.9464e-18, 3.9148e-18, 3.8832e-18, 3.8516e-18, 3.82e-18, 3.7904e-18, 3.7608e-18, 3.7312e-18,
  3.7016e-18, 3.672e-18, 3.6424e-18, 3.6128e-18, 3.5832e-18, 3.5536e-18, 3.524e-18, 3.4944e-18,
  3.4648e-18, 3.4352e-18, 3.4056e-18, 3.376e-18, 3.3464e-18, 3.3168e-18, 3.2872e-18, 3.2576e-18,
  3.228e-18, 3.1984e-18, 3.1688e-18, 3.1392e-18, 3.1096e-18, 3.08e-18
};
static inline double photo_xsec_5(double E_eV) {
  return xsec_interp(E_eV, xsec_tab_5_E, xsec_tab_5_S, 2102);
}
static inline double photo_xsec_int_5(double a, double b) {
  return xsec_int(a, b, xsec_tab_5_E, xsec_tab_5_S, 2102);
}
// xsec of H2+ -> H+ + H+ + e- [cm^2]
static inline double photo_xsec_6(double E_eV) {
  (void)E_eV;
  return kb_exp10(-16.926 - 0.04528 * E_eV + 0.0002238 * E_eV*E_eV + 4.245e-07 * E_eV*E_eV*E_eV);
}
// xsec of H2 -> H + H [cm^2]
static inline double photo_xsec_7(double E_eV) {
  (void)E_eV;
  return H2_sigmaLW(E_eV);
}

inline double (*const photo_xsec[8])(double) = {photo_xsec_0, photo_xsec_1, photo_xsec_2, photo_xsec_3, photo_xsec_4, photo_xsec_5, photo_xsec_6, photo_xsec_7};
inline double (*const photo_xsec_int[8])(double, double) = {nullptr, nullptr, nullptr, photo_xsec_int_3, photo_xsec_int_4, photo_xsec_int_5, nullptr, nullptr};
}  // namespace kbxs

constexpr bool HAS_THERMAL_TERMS = false;
// a rate coefficient depends on the densities (the species block
// of jac_stoich, taken at fixed k, is then not the exact dF/dn)
constexpr bool RATES_DEPEND_ON_N = false;
}  // namespace kbnet
