// Generated by krome_x_b200.emit from the network 'primordial' -- do not edit.
// One host/device (KB_HD) scalar form of the network: species,
// parameters, rate coefficients, mass-action rhs, stoichiometric
// Jacobian and the thermal equation (see krome_x_b200/emit/
// emitter.py for the layout and the reference rules it follows).
#pragma once
#include "../csrc/kb_common.h"

namespace kbnet {

constexpr const char* NETWORK_NAME = "primordial";
constexpr const char* NETWORK_KEY = "primordial";
constexpr int NSPEC = 12;
constexpr int NREA = 38;
constexpr int KB_RATE_NDEP = 0;
#define KB_NFREEZE 0
constexpr int IDX_D = 0;
constexpr int IDX_Dj = 1;
constexpr int IDX_H = 2;
constexpr int IDX_Hj = 3;
constexpr int IDX_Hk = 4;
constexpr int IDX_H2 = 5;
constexpr int IDX_H2j = 6;
constexpr int IDX_HD = 7;
constexpr int IDX_He = 8;
constexpr int IDX_Hej = 9;
constexpr int IDX_Hejj = 10;
constexpr int IDX_E = 11;
#define KB_HAS_D 1
#define KB_HAS_Dj 1
#define KB_HAS_H 1
#define KB_HAS_Hj 1
#define KB_HAS_Hk 1
#define KB_HAS_H2 1
#define KB_HAS_H2j 1
#define KB_HAS_HD 1
#define KB_HAS_He 1
#define KB_HAS_Hej 1
#define KB_HAS_Hejj 1
#define KB_HAS_E 1
constexpr int IDX_ELECTRON = 11;

inline const char* const species_names[NSPEC] = {"D", "D+", "H", "H+", "H-", "H2", "H2+", "HD", "He", "He+", "He++", "e-"};
constexpr int NELEM = 3;
inline const char* const element_names[3] = {"D", "H", "He"};
KB_HD inline double species_mass_g(int i) {
  constexpr double t_[NSPEC] = {3.3443256801323995e-24, 3.343414741762353e-24, 1.6738233791328e-24, 1.6729124407627538e-24, 1.6747343175028463e-24, 3.3476467582656e-24, 3.346735819895553e-24, 5.0181490592651994e-24, 6.64647366797316e-24, 6.645562729603113e-24, 6.644651791233067e-24, 9.10938370046373e-28};
  return t_[i];
}
KB_HD inline int species_charge(int i) {
  constexpr int t_[NSPEC] = {0, 1, 0, 1, -1, 0, 1, 0, 0, 1, 2, -1};
  return t_[i];
}
KB_HD inline double species_natoms_H(int i) {
  constexpr double t_[NSPEC] = {0.0, 0.0, 1.0, 1.0, 1.0, 2.0, 2.0, 1.0, 0.0, 0.0, 0.0, 0.0};
  return t_[i];
}
KB_HD inline int species_opaque(int i) {
  constexpr int t_[NSPEC] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  return t_[i];
}
inline constexpr int species_elements_t_[36] = {1, 0, 0, 1, 0, 0, 0, 1, 0, 0, 1, 0, 0, 1, 0, 0, 2, 0, 0, 2, 0, 1, 1, 0, 0, 0, 1, 0, 0, 1, 0, 0, 1, 0, 0, 0};
#ifdef __CUDACC__
__device__ const int d_species_elements_[36] = {1, 0, 0, 1, 0, 0, 0, 1, 0, 0, 1, 0, 0, 1, 0, 0, 2, 0, 0, 2, 0, 1, 1, 0, 0, 0, 1, 0, 0, 1, 0, 0, 1, 0, 0, 0};
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
  double gamma_ad;
  double Tcmb;
  double tff;
};
inline const char* const param_names[NPAR] = {"gamma_ad", "Tcmb", "tff"};
// the defaults of a parameter row; NaN marks a REQUIRED parameter
inline double param_default(int i) {
  const double t_[NPAR] = {1.6666666666666667, 2.725, NAN};
  return t_[i];
}
inline const char* const param_required_by[NPAR] = {"", "", "thermal.heating = ['COMPRESS']"};
KB_HD inline void params_from_row(const double* row, Params& p) {
  p.gamma_ad = row[0];
  p.Tcmb = row[1];
  p.tff = row[2];
}
KB_HD inline int params_missing(const Params& p) {
  (void)p;
  if (p.tff != p.tff) return 2;
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
KB_HD inline double v_sqrTgas(double Tgas, const double* n, const Params& p) {
  (void)Tgas; (void)n; (void)p;
  return std::sqrt(Tgas);
}
KB_HD inline double v_T32(double Tgas, const double* n, const Params& p) {
  (void)Tgas; (void)n; (void)p;
  return Tgas / 300.0;
}

// rate coefficients of Tgas and the parameters only
KB_HD inline void rates_fixed(double Tgas, const double* n, const Params& p, double* k) {
  (void)Tgas; (void)n; (void)p; (void)k;
  const double vh_T32 = v_T32(Tgas, n, p);
  (void)vh_T32;
  const double vh_Te = v_Te(Tgas, n, p);
  (void)vh_Te;
  const double vh_invT = v_invT(Tgas, n, p);
  (void)vh_invT;
  const double vh_invTe = v_invTe(Tgas, n, p);
  (void)vh_invTe;
  const double vh_lnTe = v_lnTe(Tgas, n, p);
  (void)vh_lnTe;
  const double vh_sqrTgas = v_sqrTgas(Tgas, n, p);
  (void)vh_sqrTgas;
  k[0] = kb_exp(-32.71396786 + 13.536556 * vh_lnTe - 5.73932875 * vh_lnTe*vh_lnTe + 1.56315498 * vh_lnTe*vh_lnTe*vh_lnTe - 0.2877056 * vh_lnTe*vh_lnTe*vh_lnTe*vh_lnTe + 0.0348255977 * ipow_<5>(vh_lnTe) - 0.00263197617 * ipow_<6>(vh_lnTe) + 0.000111954395 * ipow_<7>(vh_lnTe) - 2.03914985e-06 * ipow_<8>(vh_lnTe));  // H + e- -> H+ + e- + e-
  k[3] = kb_exp(-44.09864886 + 23.91596563 * vh_lnTe - 10.7532302 * vh_lnTe*vh_lnTe + 3.05803875 * vh_lnTe*vh_lnTe*vh_lnTe - 0.56851189 * vh_lnTe*vh_lnTe*vh_lnTe*vh_lnTe + 0.0679539123 * ipow_<5>(vh_lnTe) - 0.0050090561 * ipow_<6>(vh_lnTe) + 0.000206723616 * ipow_<7>(vh_lnTe) - 3.64916141e-06 * ipow_<8>(vh_lnTe));  // He + e- -> He+ + e- + e-
  k[6] = kb_exp(-68.71040990212 + 43.93347632635 * vh_lnTe - 18.48066993568 * vh_lnTe*vh_lnTe + 4.701626486759002 * vh_lnTe*vh_lnTe*vh_lnTe - 0.7692466334492 * vh_lnTe*vh_lnTe*vh_lnTe*vh_lnTe + 0.08113042097303 * ipow_<5>(vh_lnTe) - 0.005324020628287001 * ipow_<6>(vh_lnTe) + 0.0001975705312221 * ipow_<7>(vh_lnTe) - 3.165581065665e-06 * ipow_<8>(vh_lnTe));  // He+ + e- -> He++ + e- + e-
  k[7] = 3.36e-10 / vh_sqrTgas / kb_pow(Tgas / 1000.0, 0.2) / (1.0 + kb_pow(Tgas / 1000000.0, 0.7));  // He++ + e- -> He+
  k[8] = 6.77e-15 * kb_pow(vh_Te, 0.8779);  // H + e- -> H-
  k[13] = 6e-10;  // H2+ + H -> H2 + H+
  k[15] = 5.6e-11 * kb_exp(-102124.0 * vh_invT) * std::sqrt(Tgas);  // H2 + e- -> H + H + e-
  k[16] = 1.0670825e-10 * kb_pow(vh_Te, 2.012) * kb_exp(-4.463 * vh_invTe) / kb_pow(1.0 + 0.2472 * vh_Te, 3.512);  // H2 + H -> H + H + H
  k[17] = kb_exp(-18.01849334273 + 2.360852208681 * vh_lnTe - 0.2827443061704 * vh_lnTe*vh_lnTe + 0.01623316639567 * vh_lnTe*vh_lnTe*vh_lnTe - 0.03365012031362999 * vh_lnTe*vh_lnTe*vh_lnTe*vh_lnTe + 0.01178329782711 * ipow_<5>(vh_lnTe) - 0.001656194699504 * ipow_<6>(vh_lnTe) + 0.0001068275202678 * ipow_<7>(vh_lnTe) - 2.631285809207e-06 * ipow_<8>(vh_lnTe));  // H- + e- -> H + e- + e-
  k[20] = 6.5e-09 / std::sqrt(vh_Te);  // H- + H+ -> H + H
  k[21] = 1e-08 * kb_pow(Tgas, -0.4);  // H- + H+ -> H2+ + e-
  k[24] = 5e-07 * std::sqrt(100.0 * vh_invT);  // H2+ + H- -> H + H2
  k[31] = 1e-09 * (0.417 + 0.846 * kb_log10(Tgas) - 0.137 * kb_log10(Tgas)*kb_log10(Tgas));  // H2 + D+ -> HD + H+
  k[32] = 1e-09 * kb_exp(-457.0 * vh_invT);  // HD + H+ -> H2 + D+
  k[36] = 1.5e-09 * kb_pow(vh_T32, -0.1);  // D + H- -> HD + e-
  k[37] = 3.6e-12 * kb_pow(Tgas / 300.0, -0.75);  // D+ + e- -> D
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
  {  // group 3: H- + H -> H2 + e-
    double T = Tgas;
    const double vh_lnTe = v_lnTe(T, n, p);
    (void)vh_lnTe;
    if (T < 1160.0) {
      k[9] = 1.43e-09;  // H- + H -> H2 + e-
    }
    else if (T >= 1160.0) {
      k[10] = kb_exp(-20.06913897587003 + 0.2289800603272916 * vh_lnTe + 0.03599837721023835 * vh_lnTe*vh_lnTe - 0.004555120027032095 * vh_lnTe*vh_lnTe*vh_lnTe - 0.0003105115447124016 * vh_lnTe*vh_lnTe*vh_lnTe*vh_lnTe + 0.0001073294010367247 * ipow_<5>(vh_lnTe) - 8.36671960467864e-06 * ipow_<6>(vh_lnTe) + 2.238306228891639e-07 * ipow_<7>(vh_lnTe));  // H- + H -> H2 + e-
    }
  }
  {  // group 4: H + H+ -> H2+
    double T = Tgas;
    if (T < 6700.0) {
      k[11] = 1.85e-23 * kb_pow(T, 1.8);  // H + H+ -> H2+
    }
    else if (T >= 6700.0) {
      k[12] = 5.81e-16 * kb_pow(T / 56200.0, -0.6657 * kb_log10(T / 56200.0));  // H + H+ -> H2+
    }
  }
  {  // group 5: H2 + H+ -> H2+ + H
    double T = Tgas;
    const double vh_lnTe = v_lnTe(T, n, p);
    (void)vh_lnTe;
    if (T >= 3480.0 && T >= 3480.0) {
      k[14] = kb_exp(-24.24914687731536 + 3.400824447095291 * vh_lnTe - 3.898003964650152 * vh_lnTe*vh_lnTe + 2.045587822403071 * vh_lnTe*vh_lnTe*vh_lnTe - 0.5416182856220388 * vh_lnTe*vh_lnTe*vh_lnTe*vh_lnTe + 0.0841077503763412 * ipow_<5>(vh_lnTe) - 0.007879026154483455 * ipow_<6>(vh_lnTe) + 0.0004138398421504563 * ipow_<7>(vh_lnTe) - 9.36345888928611e-06 * ipow_<8>(vh_lnTe));  // H2 + H+ -> H2+ + H
    }
  }
  {  // group 6: H- + H -> H + H + e-
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
  {  // group 7: H2+ + e- -> H + H
    double T = Tgas;
    if (T < 617.0) {
      k[22] = 1e-08;  // H2+ + e- -> H + H
    }
    else if (T >= 617.0) {
      k[23] = 1.32e-06 * kb_pow(T, -0.76);  // H2+ + e- -> H + H
    }
  }
  {  // group 8: H + H + H -> H2 + H
    double T = Tgas;
    const double vh_T32 = v_T32(T, n, p);
    (void)vh_T32;
    if (T < 300.0) {
      k[25] = 1.3e-32 * kb_pow(vh_T32, -0.38);  // H + H + H -> H2 + H
    }
    else if (T >= 300.0) {
      k[26] = 1.3e-32 * ipow_<-1>(vh_T32);  // H + H + H -> H2 + H
    }
  }
  {  // group 9: H2 + H + H -> H2 + H2
    double T = Tgas;
    const double vh_T32 = v_T32(T, n, p);
    (void)vh_T32;
    if (T < 300.0) {
      k[27] = 1.3e-32 * kb_pow(vh_T32, -0.38) / 8.0;  // H2 + H + H -> H2 + H2
    }
    else if (T >= 300.0) {
      k[28] = 1.3e-32 * ipow_<-1>(vh_T32) / 8.0;  // H2 + H + H -> H2 + H2
    }
  }
  {  // group 10: H+ + D -> H + D+
    double T = Tgas;
    const double vh_invT = v_invT(T, n, p);
    (void)vh_invT;
    if (T >= 50.0 && T >= 50.0) {
      k[29] = 2e-10 * kb_pow(T, 0.402) * kb_exp(-37.1 * vh_invT) - 3.31e-17 * kb_pow(T, 1.48);  // H+ + D -> H + D+
    }
  }
  {  // group 11: H + D+ -> H+ + D
    double T = Tgas;
    const double vh_invT = v_invT(T, n, p);
    (void)vh_invT;
    if (T >= 50.0 && T >= 50.0) {
      k[30] = 2.06e-10 * kb_pow(T, 0.396) * kb_exp(-33.0 * vh_invT) + 2.03e-09 * kb_pow(T, -0.332);  // H + D+ -> H+ + D
    }
  }
  {  // group 12: H2 + D -> HD + H
    double T = Tgas;
    const double vh_invT = v_invT(T, n, p);
    (void)vh_invT;
    if (T < 2000.0) {
      k[33] = kb_exp10(-56.4737 + 5.88886 * kb_log10(T) + 7.19692 * kb_log10(T)*kb_log10(T) + 2.25069 * kb_log10(T)*kb_log10(T)*kb_log10(T) - 2.16903 * kb_log10(T)*kb_log10(T)*kb_log10(T)*kb_log10(T) + 0.317887 * ipow_<5>(kb_log10(T)));  // H2 + D -> HD + H
    }
    else if (T >= 2000.0) {
      k[34] = 3.17e-10 * kb_exp(-5207.0 * vh_invT);  // H2 + D -> HD + H
    }
  }
  {  // group 13: HD + H -> H2 + D
    double T = Tgas;
    const double vh_invT = v_invT(T, n, p);
    (void)vh_invT;
    if (T >= 200.0 && T >= 200.0) {
      k[35] = 5.25e-11 * kb_exp(-4430.0 * vh_invT + 173900.0 * vh_invT*vh_invT);  // HD + H -> H2 + D
    }
  }
}
// rate coefficients that also depend on the densities
KB_HD inline void rates_var(double Tgas, const double* n, const Params& p, double* k) {
  (void)Tgas; (void)n; (void)p; (void)k;
}
constexpr int NREA_FIXED = 38;
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
    case 35:
    case 36:
    case 37:
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
  flux = k[10]*n[IDX_Hk]*n[IDX_H];
  dn[IDX_Hk] -= flux;
  dn[IDX_H] -= flux;
  dn[IDX_H2] += flux;
  dn[IDX_E] += flux;
  flux = k[11]*n[IDX_H]*n[IDX_Hj];
  dn[IDX_H] -= flux;
  dn[IDX_Hj] -= flux;
  dn[IDX_H2j] += flux;
  flux = k[12]*n[IDX_H]*n[IDX_Hj];
  dn[IDX_H] -= flux;
  dn[IDX_Hj] -= flux;
  dn[IDX_H2j] += flux;
  flux = k[13]*n[IDX_H2j]*n[IDX_H];
  dn[IDX_H2j] -= flux;
  dn[IDX_H] -= flux;
  dn[IDX_H2] += flux;
  dn[IDX_Hj] += flux;
  flux = k[14]*n[IDX_H2]*n[IDX_Hj];
  dn[IDX_H2] -= flux;
  dn[IDX_Hj] -= flux;
  dn[IDX_H2j] += flux;
  dn[IDX_H] += flux;
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
  flux = k[23]*n[IDX_H2j]*n[IDX_E];
  dn[IDX_H2j] -= flux;
  dn[IDX_E] -= flux;
  dn[IDX_H] += flux;
  dn[IDX_H] += flux;
  flux = k[24]*n[IDX_H2j]*n[IDX_Hk];
  dn[IDX_H2j] -= flux;
  dn[IDX_Hk] -= flux;
  dn[IDX_H] += flux;
  dn[IDX_H2] += flux;
  flux = k[25]*n[IDX_H]*n[IDX_H]*n[IDX_H];
  dn[IDX_H] -= flux;
  dn[IDX_H] -= flux;
  dn[IDX_H] -= flux;
  dn[IDX_H2] += flux;
  dn[IDX_H] += flux;
  flux = k[26]*n[IDX_H]*n[IDX_H]*n[IDX_H];
  dn[IDX_H] -= flux;
  dn[IDX_H] -= flux;
  dn[IDX_H] -= flux;
  dn[IDX_H2] += flux;
  dn[IDX_H] += flux;
  flux = k[27]*n[IDX_H2]*n[IDX_H]*n[IDX_H];
  dn[IDX_H2] -= flux;
  dn[IDX_H] -= flux;
  dn[IDX_H] -= flux;
  dn[IDX_H2] += flux;
  dn[IDX_H2] += flux;
  flux = k[28]*n[IDX_H2]*n[IDX_H]*n[IDX_H];
  dn[IDX_H2] -= flux;
  dn[IDX_H] -= flux;
  dn[IDX_H] -= flux;
  dn[IDX_H2] += flux;
  dn[IDX_H2] += flux;
  flux = k[29]*n[IDX_Hj]*n[IDX_D];
  dn[IDX_Hj] -= flux;
  dn[IDX_D] -= flux;
  dn[IDX_H] += flux;
  dn[IDX_Dj] += flux;
  flux = k[30]*n[IDX_H]*n[IDX_Dj];
  dn[IDX_H] -= flux;
  dn[IDX_Dj] -= flux;
  dn[IDX_Hj] += flux;
  dn[IDX_D] += flux;
  flux = k[31]*n[IDX_H2]*n[IDX_Dj];
  dn[IDX_H2] -= flux;
  dn[IDX_Dj] -= flux;
  dn[IDX_HD] += flux;
  dn[IDX_Hj] += flux;
  flux = k[32]*n[IDX_HD]*n[IDX_Hj];
  dn[IDX_HD] -= flux;
  dn[IDX_Hj] -= flux;
  dn[IDX_H2] += flux;
  dn[IDX_Dj] += flux;
  flux = k[33]*n[IDX_H2]*n[IDX_D];
  dn[IDX_H2] -= flux;
  dn[IDX_D] -= flux;
  dn[IDX_HD] += flux;
  dn[IDX_H] += flux;
  flux = k[34]*n[IDX_H2]*n[IDX_D];
  dn[IDX_H2] -= flux;
  dn[IDX_D] -= flux;
  dn[IDX_HD] += flux;
  dn[IDX_H] += flux;
  flux = k[35]*n[IDX_HD]*n[IDX_H];
  dn[IDX_HD] -= flux;
  dn[IDX_H] -= flux;
  dn[IDX_H2] += flux;
  dn[IDX_D] += flux;
  flux = k[36]*n[IDX_D]*n[IDX_Hk];
  dn[IDX_D] -= flux;
  dn[IDX_Hk] -= flux;
  dn[IDX_HD] += flux;
  dn[IDX_E] += flux;
  flux = k[37]*n[IDX_Dj]*n[IDX_E];
  dn[IDX_Dj] -= flux;
  dn[IDX_E] -= flux;
  dn[IDX_D] += flux;
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
  d = k[10]*n[IDX_Hk];
  J[IDX_Hk*rs + IDX_H*cs] -= d;
  J[IDX_H*rs + IDX_H*cs] -= d;
  J[IDX_H2*rs + IDX_H*cs] += d;
  J[IDX_E*rs + IDX_H*cs] += d;
  d = k[10]*n[IDX_H];
  J[IDX_Hk*rs + IDX_Hk*cs] -= d;
  J[IDX_H*rs + IDX_Hk*cs] -= d;
  J[IDX_H2*rs + IDX_Hk*cs] += d;
  J[IDX_E*rs + IDX_Hk*cs] += d;
  d = k[11]*n[IDX_Hj];
  J[IDX_H*rs + IDX_H*cs] -= d;
  J[IDX_Hj*rs + IDX_H*cs] -= d;
  J[IDX_H2j*rs + IDX_H*cs] += d;
  d = k[11]*n[IDX_H];
  J[IDX_H*rs + IDX_Hj*cs] -= d;
  J[IDX_Hj*rs + IDX_Hj*cs] -= d;
  J[IDX_H2j*rs + IDX_Hj*cs] += d;
  d = k[12]*n[IDX_Hj];
  J[IDX_H*rs + IDX_H*cs] -= d;
  J[IDX_Hj*rs + IDX_H*cs] -= d;
  J[IDX_H2j*rs + IDX_H*cs] += d;
  d = k[12]*n[IDX_H];
  J[IDX_H*rs + IDX_Hj*cs] -= d;
  J[IDX_Hj*rs + IDX_Hj*cs] -= d;
  J[IDX_H2j*rs + IDX_Hj*cs] += d;
  d = k[13]*n[IDX_H2j];
  J[IDX_H2j*rs + IDX_H*cs] -= d;
  J[IDX_H*rs + IDX_H*cs] -= d;
  J[IDX_H2*rs + IDX_H*cs] += d;
  J[IDX_Hj*rs + IDX_H*cs] += d;
  d = k[13]*n[IDX_H];
  J[IDX_H2j*rs + IDX_H2j*cs] -= d;
  J[IDX_H*rs + IDX_H2j*cs] -= d;
  J[IDX_H2*rs + IDX_H2j*cs] += d;
  J[IDX_Hj*rs + IDX_H2j*cs] += d;
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
  d = k[24]*n[IDX_H2j];
  J[IDX_H2j*rs + IDX_Hk*cs] -= d;
  J[IDX_Hk*rs + IDX_Hk*cs] -= d;
  J[IDX_H*rs + IDX_Hk*cs] += d;
  J[IDX_H2*rs + IDX_Hk*cs] += d;
  d = k[24]*n[IDX_Hk];
  J[IDX_H2j*rs + IDX_H2j*cs] -= d;
  J[IDX_Hk*rs + IDX_H2j*cs] -= d;
  J[IDX_H*rs + IDX_H2j*cs] += d;
  J[IDX_H2*rs + IDX_H2j*cs] += d;
  d = 3.0*k[25]*n[IDX_H]*n[IDX_H];
  J[IDX_H*rs + IDX_H*cs] -= d;
  J[IDX_H*rs + IDX_H*cs] -= d;
  J[IDX_H*rs + IDX_H*cs] -= d;
  J[IDX_H2*rs + IDX_H*cs] += d;
  J[IDX_H*rs + IDX_H*cs] += d;
  d = 3.0*k[26]*n[IDX_H]*n[IDX_H];
  J[IDX_H*rs + IDX_H*cs] -= d;
  J[IDX_H*rs + IDX_H*cs] -= d;
  J[IDX_H*rs + IDX_H*cs] -= d;
  J[IDX_H2*rs + IDX_H*cs] += d;
  J[IDX_H*rs + IDX_H*cs] += d;
  d = 2.0*k[27]*n[IDX_H]*n[IDX_H2];
  J[IDX_H2*rs + IDX_H*cs] -= d;
  J[IDX_H*rs + IDX_H*cs] -= d;
  J[IDX_H*rs + IDX_H*cs] -= d;
  J[IDX_H2*rs + IDX_H*cs] += d;
  J[IDX_H2*rs + IDX_H*cs] += d;
  d = k[27]*n[IDX_H]*n[IDX_H];
  J[IDX_H2*rs + IDX_H2*cs] -= d;
  J[IDX_H*rs + IDX_H2*cs] -= d;
  J[IDX_H*rs + IDX_H2*cs] -= d;
  J[IDX_H2*rs + IDX_H2*cs] += d;
  J[IDX_H2*rs + IDX_H2*cs] += d;
  d = 2.0*k[28]*n[IDX_H]*n[IDX_H2];
  J[IDX_H2*rs + IDX_H*cs] -= d;
  J[IDX_H*rs + IDX_H*cs] -= d;
  J[IDX_H*rs + IDX_H*cs] -= d;
  J[IDX_H2*rs + IDX_H*cs] += d;
  J[IDX_H2*rs + IDX_H*cs] += d;
  d = k[28]*n[IDX_H]*n[IDX_H];
  J[IDX_H2*rs + IDX_H2*cs] -= d;
  J[IDX_H*rs + IDX_H2*cs] -= d;
  J[IDX_H*rs + IDX_H2*cs] -= d;
  J[IDX_H2*rs + IDX_H2*cs] += d;
  J[IDX_H2*rs + IDX_H2*cs] += d;
  d = k[29]*n[IDX_Hj];
  J[IDX_Hj*rs + IDX_D*cs] -= d;
  J[IDX_D*rs + IDX_D*cs] -= d;
  J[IDX_H*rs + IDX_D*cs] += d;
  J[IDX_Dj*rs + IDX_D*cs] += d;
  d = k[29]*n[IDX_D];
  J[IDX_Hj*rs + IDX_Hj*cs] -= d;
  J[IDX_D*rs + IDX_Hj*cs] -= d;
  J[IDX_H*rs + IDX_Hj*cs] += d;
  J[IDX_Dj*rs + IDX_Hj*cs] += d;
  d = k[30]*n[IDX_H];
  J[IDX_H*rs + IDX_Dj*cs] -= d;
  J[IDX_Dj*rs + IDX_Dj*cs] -= d;
  J[IDX_Hj*rs + IDX_Dj*cs] += d;
  J[IDX_D*rs + IDX_Dj*cs] += d;
  d = k[30]*n[IDX_Dj];
  J[IDX_H*rs + IDX_H*cs] -= d;
  J[IDX_Dj*rs + IDX_H*cs] -= d;
  J[IDX_Hj*rs + IDX_H*cs] += d;
  J[IDX_D*rs + IDX_H*cs] += d;
  d = k[31]*n[IDX_H2];
  J[IDX_H2*rs + IDX_Dj*cs] -= d;
  J[IDX_Dj*rs + IDX_Dj*cs] -= d;
  J[IDX_HD*rs + IDX_Dj*cs] += d;
  J[IDX_Hj*rs + IDX_Dj*cs] += d;
  d = k[31]*n[IDX_Dj];
  J[IDX_H2*rs + IDX_H2*cs] -= d;
  J[IDX_Dj*rs + IDX_H2*cs] -= d;
  J[IDX_HD*rs + IDX_H2*cs] += d;
  J[IDX_Hj*rs + IDX_H2*cs] += d;
  d = k[32]*n[IDX_HD];
  J[IDX_HD*rs + IDX_Hj*cs] -= d;
  J[IDX_Hj*rs + IDX_Hj*cs] -= d;
  J[IDX_H2*rs + IDX_Hj*cs] += d;
  J[IDX_Dj*rs + IDX_Hj*cs] += d;
  d = k[32]*n[IDX_Hj];
  J[IDX_HD*rs + IDX_HD*cs] -= d;
  J[IDX_Hj*rs + IDX_HD*cs] -= d;
  J[IDX_H2*rs + IDX_HD*cs] += d;
  J[IDX_Dj*rs + IDX_HD*cs] += d;
  d = k[33]*n[IDX_H2];
  J[IDX_H2*rs + IDX_D*cs] -= d;
  J[IDX_D*rs + IDX_D*cs] -= d;
  J[IDX_HD*rs + IDX_D*cs] += d;
  J[IDX_H*rs + IDX_D*cs] += d;
  d = k[33]*n[IDX_D];
  J[IDX_H2*rs + IDX_H2*cs] -= d;
  J[IDX_D*rs + IDX_H2*cs] -= d;
  J[IDX_HD*rs + IDX_H2*cs] += d;
  J[IDX_H*rs + IDX_H2*cs] += d;
  d = k[34]*n[IDX_H2];
  J[IDX_H2*rs + IDX_D*cs] -= d;
  J[IDX_D*rs + IDX_D*cs] -= d;
  J[IDX_HD*rs + IDX_D*cs] += d;
  J[IDX_H*rs + IDX_D*cs] += d;
  d = k[34]*n[IDX_D];
  J[IDX_H2*rs + IDX_H2*cs] -= d;
  J[IDX_D*rs + IDX_H2*cs] -= d;
  J[IDX_HD*rs + IDX_H2*cs] += d;
  J[IDX_H*rs + IDX_H2*cs] += d;
  d = k[35]*n[IDX_HD];
  J[IDX_HD*rs + IDX_H*cs] -= d;
  J[IDX_H*rs + IDX_H*cs] -= d;
  J[IDX_H2*rs + IDX_H*cs] += d;
  J[IDX_D*rs + IDX_H*cs] += d;
  d = k[35]*n[IDX_H];
  J[IDX_HD*rs + IDX_HD*cs] -= d;
  J[IDX_H*rs + IDX_HD*cs] -= d;
  J[IDX_H2*rs + IDX_HD*cs] += d;
  J[IDX_D*rs + IDX_HD*cs] += d;
  d = k[36]*n[IDX_Hk];
  J[IDX_D*rs + IDX_D*cs] -= d;
  J[IDX_Hk*rs + IDX_D*cs] -= d;
  J[IDX_HD*rs + IDX_D*cs] += d;
  J[IDX_E*rs + IDX_D*cs] += d;
  d = k[36]*n[IDX_D];
  J[IDX_D*rs + IDX_Hk*cs] -= d;
  J[IDX_Hk*rs + IDX_Hk*cs] -= d;
  J[IDX_HD*rs + IDX_Hk*cs] += d;
  J[IDX_E*rs + IDX_Hk*cs] += d;
  d = k[37]*n[IDX_E];
  J[IDX_Dj*rs + IDX_Dj*cs] -= d;
  J[IDX_E*rs + IDX_Dj*cs] -= d;
  J[IDX_D*rs + IDX_Dj*cs] += d;
  d = k[37]*n[IDX_Dj];
  J[IDX_Dj*rs + IDX_E*cs] -= d;
  J[IDX_E*rs + IDX_E*cs] -= d;
  J[IDX_D*rs + IDX_E*cs] += d;
}

// the rate-derivative part of the analytic Jacobian (J[i*jrs_ + j*cs], added to;
// U[NSPEC][NAGG] written), gated and clamped like the rates
KB_HD inline void jac_dk(double Tgas, const double* n, const Params& p, const double* k, double* J, double* U, long jrs_, long jcs_) {
  (void)Tgas; (void)n; (void)p; (void)k; (void)J; (void)jrs_; (void)jcs_;
  for (int i = 0; i < NSPEC * NAGG; ++i) U[i] = 0.0;
  double d;
  (void)d;
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
  {  // group 3: H- + H -> H2 + e-
    double T = Tgas;
    if (T < 1160.0) {
    }
    else if (T >= 1160.0) {
    }
  }
  {  // group 4: H + H+ -> H2+
    double T = Tgas;
    if (T < 6700.0) {
    }
    else if (T >= 6700.0) {
    }
  }
  {  // group 5: H2 + H+ -> H2+ + H
    double T = Tgas;
    if (T >= 3480.0 && T >= 3480.0) {
    }
  }
  {  // group 6: H- + H -> H + H + e-
    double T = Tgas;
    if (T < 1160.0) {
    }
    else if (T >= 1160.0) {
    }
  }
  {  // group 7: H2+ + e- -> H + H
    double T = Tgas;
    if (T < 617.0) {
    }
    else if (T >= 617.0) {
    }
  }
  {  // group 8: H + H + H -> H2 + H
    double T = Tgas;
    if (T < 300.0) {
    }
    else if (T >= 300.0) {
    }
  }
  {  // group 9: H2 + H + H -> H2 + H2
    double T = Tgas;
    if (T < 300.0) {
    }
    else if (T >= 300.0) {
    }
  }
  {  // group 10: H+ + D -> H + D+
    double T = Tgas;
    if (T >= 50.0 && T >= 50.0) {
    }
  }
  {  // group 11: H + D+ -> H+ + D
    double T = Tgas;
    if (T >= 50.0 && T >= 50.0) {
    }
  }
  {  // group 12: H2 + D -> HD + H
    double T = Tgas;
    if (T < 2000.0) {
    }
    else if (T >= 2000.0) {
    }
  }
  {  // group 13: HD + H -> H2 + D
    double T = Tgas;
    if (T >= 200.0 && T >= 200.0) {
    }
  }
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
  h += k[10] * (3.53*ffac) * n[IDX_Hk]*n[IDX_H];
  h += k[13] * (1.83*ffac) * n[IDX_H2j]*n[IDX_H];
  h += k[25] * (4.48*ffac) * n[IDX_H]*n[IDX_H]*n[IDX_H];
  h += k[26] * (4.48*ffac) * n[IDX_H]*n[IDX_H]*n[IDX_H];
  h += k[27] * (4.48*ffac) * n[IDX_H2]*n[IDX_H]*n[IDX_H];
  h += k[28] * (4.48*ffac) * n[IDX_H2]*n[IDX_H]*n[IDX_H];
  h *= ev2erg;
  return h;
}
// recombination rates of the ATOMIC cooling and T dk/dT of the
// piece active at T (central difference, relative step 1e-4;
// 0 where the rate's temperature is clamped)
KB_HD inline void recomb_rates_(double Tgas, const double* n, const Params& p, double* kr, double* tdk) {
  (void)n; (void)p;
  const double h = 1e-4;
  for (int j = 0; j < 6; ++j) kr[j] = tdk[j] = 0.0;
  kr[4] = 3.36e-10 / v_sqrTgas(Tgas, n, p) / kb_pow(Tgas / 1000.0, 0.2) / (1.0 + kb_pow(Tgas / 1000000.0, 0.7));
  { const double Tp_ = Tgas * (1.0 + h), Tm_ = Tgas * (1.0 - h);
    tdk[4] = ((3.36e-10 / v_sqrTgas(Tp_, n, p) / kb_pow(Tp_ / 1000.0, 0.2) / (1.0 + kb_pow(Tp_ / 1000000.0, 0.7))) - (3.36e-10 / v_sqrTgas(Tm_, n, p) / kb_pow(Tm_ / 1000.0, 0.2) / (1.0 + kb_pow(Tm_ / 1000000.0, 0.7)))) / (2.0 * h); }
  kr[5] = 3.6e-12 * kb_pow(Tgas / 300.0, -0.75);
  { const double Tp_ = Tgas * (1.0 + h), Tm_ = Tgas * (1.0 - h);
    tdk[5] = ((3.6e-12 * kb_pow(Tp_ / 300.0, -0.75)) - (3.6e-12 * kb_pow(Tm_ / 300.0, -0.75))) / (2.0 * h); }
  {  // group 1: H+ + e- -> H
    double T = Tgas;
    if (T < 5500.0) {
      kr[0] = 3.92e-13 * kb_pow(v_invTe(T, n, p), 0.6353);
      if (T == Tgas) { const double Tp_ = T * (1.0 + h), Tm_ = T * (1.0 - h);
        tdk[0] = ((3.92e-13 * kb_pow(v_invTe(Tp_, n, p), 0.6353)) - (3.92e-13 * kb_pow(v_invTe(Tm_, n, p), 0.6353))) / (2.0 * h); }
    }
    else if (T >= 5500.0) {
      kr[1] = kb_exp(-28.61303380689232 - 0.7241125657826851 * v_lnTe(T, n, p) - 0.02026044731984691 * v_lnTe(T, n, p)*v_lnTe(T, n, p) - 0.002380861877349834 * v_lnTe(T, n, p)*v_lnTe(T, n, p)*v_lnTe(T, n, p) - 0.0003212605213188796 * v_lnTe(T, n, p)*v_lnTe(T, n, p)*v_lnTe(T, n, p)*v_lnTe(T, n, p) - 1.421502914054107e-05 * ipow_<5>(v_lnTe(T, n, p)) + 4.989108920299513e-06 * ipow_<6>(v_lnTe(T, n, p)) + 5.755614137575758e-07 * ipow_<7>(v_lnTe(T, n, p)) - 1.856767039775261e-08 * ipow_<8>(v_lnTe(T, n, p)) - 3.071135243196595e-09 * ipow_<9>(v_lnTe(T, n, p)));
      if (T == Tgas) { const double Tp_ = T * (1.0 + h), Tm_ = T * (1.0 - h);
        tdk[1] = ((kb_exp(-28.61303380689232 - 0.7241125657826851 * v_lnTe(Tp_, n, p) - 0.02026044731984691 * v_lnTe(Tp_, n, p)*v_lnTe(Tp_, n, p) - 0.002380861877349834 * v_lnTe(Tp_, n, p)*v_lnTe(Tp_, n, p)*v_lnTe(Tp_, n, p) - 0.0003212605213188796 * v_lnTe(Tp_, n, p)*v_lnTe(Tp_, n, p)*v_lnTe(Tp_, n, p)*v_lnTe(Tp_, n, p) - 1.421502914054107e-05 * ipow_<5>(v_lnTe(Tp_, n, p)) + 4.989108920299513e-06 * ipow_<6>(v_lnTe(Tp_, n, p)) + 5.755614137575758e-07 * ipow_<7>(v_lnTe(Tp_, n, p)) - 1.856767039775261e-08 * ipow_<8>(v_lnTe(Tp_, n, p)) - 3.071135243196595e-09 * ipow_<9>(v_lnTe(Tp_, n, p)))) - (kb_exp(-28.61303380689232 - 0.7241125657826851 * v_lnTe(Tm_, n, p) - 0.02026044731984691 * v_lnTe(Tm_, n, p)*v_lnTe(Tm_, n, p) - 0.002380861877349834 * v_lnTe(Tm_, n, p)*v_lnTe(Tm_, n, p)*v_lnTe(Tm_, n, p) - 0.0003212605213188796 * v_lnTe(Tm_, n, p)*v_lnTe(Tm_, n, p)*v_lnTe(Tm_, n, p)*v_lnTe(Tm_, n, p) - 1.421502914054107e-05 * ipow_<5>(v_lnTe(Tm_, n, p)) + 4.989108920299513e-06 * ipow_<6>(v_lnTe(Tm_, n, p)) + 5.755614137575758e-07 * ipow_<7>(v_lnTe(Tm_, n, p)) - 1.856767039775261e-08 * ipow_<8>(v_lnTe(Tm_, n, p)) - 3.071135243196595e-09 * ipow_<9>(v_lnTe(Tm_, n, p))))) / (2.0 * h); }
    }
  }
  {  // group 2: He+ + e- -> He
    double T = Tgas;
    if (T < 9280.0) {
      kr[2] = 3.92e-13 * kb_pow(v_invTe(T, n, p), 0.6353);
      if (T == Tgas) { const double Tp_ = T * (1.0 + h), Tm_ = T * (1.0 - h);
        tdk[2] = ((3.92e-13 * kb_pow(v_invTe(Tp_, n, p), 0.6353)) - (3.92e-13 * kb_pow(v_invTe(Tm_, n, p), 0.6353))) / (2.0 * h); }
    }
    else if (T >= 9280.0) {
      kr[3] = 1.54e-09 * (1.0 + 0.3 / kb_exp(8.099328789667 * v_invTe(T, n, p))) / (kb_exp(40.49664394833662 * v_invTe(T, n, p)) * ipow_<1>(v_Te(T, n, p)) * std::sqrt(v_Te(T, n, p))) + 3.92e-13 / kb_pow(v_Te(T, n, p), 0.6353);
      if (T == Tgas) { const double Tp_ = T * (1.0 + h), Tm_ = T * (1.0 - h);
        tdk[3] = ((1.54e-09 * (1.0 + 0.3 / kb_exp(8.099328789667 * v_invTe(Tp_, n, p))) / (kb_exp(40.49664394833662 * v_invTe(Tp_, n, p)) * ipow_<1>(v_Te(Tp_, n, p)) * std::sqrt(v_Te(Tp_, n, p))) + 3.92e-13 / kb_pow(v_Te(Tp_, n, p), 0.6353)) - (1.54e-09 * (1.0 + 0.3 / kb_exp(8.099328789667 * v_invTe(Tm_, n, p))) / (kb_exp(40.49664394833662 * v_invTe(Tm_, n, p)) * ipow_<1>(v_Te(Tm_, n, p)) * std::sqrt(v_Te(Tm_, n, p))) + 3.92e-13 / kb_pow(v_Te(Tm_, n, p), 0.6353))) / (2.0 * h); }
    }
  }
}
KB_HD inline double cooling_recomb_(double Tgas, const double* n, const Params& p) {
  const double T = std::fmin(std::fmax(Tgas, p.Tcmb), 1e9);
  double k0[6], tdk[6];
  recomb_rates_(T, n, p, k0, tdk);
  double c = 0.0;
  c += n[IDX_E] * n[IDX_Hj] * std::fmax(0.0, 1.5 * k0[0] + tdk[0]);
  c += n[IDX_E] * n[IDX_Hj] * std::fmax(0.0, 1.5 * k0[1] + tdk[1]);
  c += n[IDX_E] * n[IDX_Hej] * std::fmax(0.0, 1.5 * k0[2] + tdk[2]);
  c += n[IDX_E] * n[IDX_Hej] * std::fmax(0.0, 1.5 * k0[3] + tdk[3]);
  c += n[IDX_E] * n[IDX_Hejj] * std::fmax(0.0, 1.5 * k0[4] + tdk[4]);
  c += n[IDX_E] * n[IDX_Dj] * std::fmax(0.0, 1.5 * k0[5] + tdk[5]);
  return kbc::boltzmann_erg * T * c;
}
KB_HD inline double cooling_recomb_with_(const double* k0, const double* tdk, double Tgas, const double* n, const Params& p) {
  const double T = std::fmin(std::fmax(Tgas, p.Tcmb), 1e9);
  double c = 0.0;
  c += n[IDX_E] * n[IDX_Hj] * std::fmax(0.0, 1.5 * k0[0] + tdk[0]);
  c += n[IDX_E] * n[IDX_Hj] * std::fmax(0.0, 1.5 * k0[1] + tdk[1]);
  c += n[IDX_E] * n[IDX_Hej] * std::fmax(0.0, 1.5 * k0[2] + tdk[2]);
  c += n[IDX_E] * n[IDX_Hej] * std::fmax(0.0, 1.5 * k0[3] + tdk[3]);
  c += n[IDX_E] * n[IDX_Hejj] * std::fmax(0.0, 1.5 * k0[4] + tdk[4]);
  c += n[IDX_E] * n[IDX_Dj] * std::fmax(0.0, 1.5 * k0[5] + tdk[5]);
  return kbc::boltzmann_erg * T * c;
}
KB_HD inline double h2_opacity_(const double* n) {
  (void)n;
  return 1.0;
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
  heat += heating_chem(T, n, k);
  heat += ntot_(n) * kbc::boltzmann_erg * T / p.tff;
  cool += cooling_Atomic(T, n) + cooling_recomb_(T, n, p);
  cool += cooling_H2(T, n) * h2_opacity_(n);
  return (gamma_index(T, n, p) - 1.0) * (heat - cool)
      / (kbc::boltzmann_erg * ntot_(n));
}
// the cooling's temperature-only parts at one T (a row of density
// derivatives at that T evaluates them once): thermal_dTdt_with of
// thermal_pre(T) equals thermal_dTdt bit for bit
struct ThermalPre {
  CoolAtomicC atomic;
  double k0[6], tdk[6];
  CoolH2C h2;
  int unused_;
};
KB_HD inline void thermal_pre(double T, const double* n, const Params& p, ThermalPre& q) {
  (void)T; (void)n; (void)p; (void)q;
  q.atomic = cooling_Atomic_coef(T);
  recomb_rates_(std::fmin(std::fmax(T, p.Tcmb), 1e9), n, p, q.k0, q.tdk);
  q.h2 = cooling_H2_coef(T);
}
KB_HD inline double thermal_dTdt_with(const ThermalPre& q, double T, const double* n, const double* k, const Params& p) {
  (void)q; (void)k; (void)p;
  double heat = 0.0, cool = 0.0;
  heat += heating_chem(T, n, k);
  heat += ntot_(n) * kbc::boltzmann_erg * T / p.tff;
  cool += cooling_Atomic_with(q.atomic, n) + cooling_recomb_with_(q.k0, q.tdk, T, n, p);
  cool += cooling_H2_with(q.h2, n) * h2_opacity_(n);
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
  flux = k[10]*n[IDX_Hk]*n[IDX_H];
  g[10] += flux * (mu[IDX_H2] + mu[IDX_E] - mu[IDX_Hk] - mu[IDX_H]);
  flux = k[11]*n[IDX_H]*n[IDX_Hj];
  g[11] += flux * (mu[IDX_H2j] - mu[IDX_H] - mu[IDX_Hj]);
  flux = k[12]*n[IDX_H]*n[IDX_Hj];
  g[12] += flux * (mu[IDX_H2j] - mu[IDX_H] - mu[IDX_Hj]);
  flux = k[13]*n[IDX_H2j]*n[IDX_H];
  g[13] += flux * (mu[IDX_H2] + mu[IDX_Hj] - mu[IDX_H2j] - mu[IDX_H]);
  flux = k[14]*n[IDX_H2]*n[IDX_Hj];
  g[14] += flux * (mu[IDX_H2j] + mu[IDX_H] - mu[IDX_H2] - mu[IDX_Hj]);
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
  flux = k[23]*n[IDX_H2j]*n[IDX_E];
  g[23] += flux * (mu[IDX_H] + mu[IDX_H] - mu[IDX_H2j] - mu[IDX_E]);
  flux = k[24]*n[IDX_H2j]*n[IDX_Hk];
  g[24] += flux * (mu[IDX_H] + mu[IDX_H2] - mu[IDX_H2j] - mu[IDX_Hk]);
  flux = k[25]*n[IDX_H]*n[IDX_H]*n[IDX_H];
  g[25] += flux * (mu[IDX_H2] + mu[IDX_H] - mu[IDX_H] - mu[IDX_H] - mu[IDX_H]);
  flux = k[26]*n[IDX_H]*n[IDX_H]*n[IDX_H];
  g[26] += flux * (mu[IDX_H2] + mu[IDX_H] - mu[IDX_H] - mu[IDX_H] - mu[IDX_H]);
  flux = k[27]*n[IDX_H2]*n[IDX_H]*n[IDX_H];
  g[27] += flux * (mu[IDX_H2] + mu[IDX_H2] - mu[IDX_H2] - mu[IDX_H] - mu[IDX_H]);
  flux = k[28]*n[IDX_H2]*n[IDX_H]*n[IDX_H];
  g[28] += flux * (mu[IDX_H2] + mu[IDX_H2] - mu[IDX_H2] - mu[IDX_H] - mu[IDX_H]);
  flux = k[29]*n[IDX_Hj]*n[IDX_D];
  g[29] += flux * (mu[IDX_H] + mu[IDX_Dj] - mu[IDX_Hj] - mu[IDX_D]);
  flux = k[30]*n[IDX_H]*n[IDX_Dj];
  g[30] += flux * (mu[IDX_Hj] + mu[IDX_D] - mu[IDX_H] - mu[IDX_Dj]);
  flux = k[31]*n[IDX_H2]*n[IDX_Dj];
  g[31] += flux * (mu[IDX_HD] + mu[IDX_Hj] - mu[IDX_H2] - mu[IDX_Dj]);
  flux = k[32]*n[IDX_HD]*n[IDX_Hj];
  g[32] += flux * (mu[IDX_H2] + mu[IDX_Dj] - mu[IDX_HD] - mu[IDX_Hj]);
  flux = k[33]*n[IDX_H2]*n[IDX_D];
  g[33] += flux * (mu[IDX_HD] + mu[IDX_H] - mu[IDX_H2] - mu[IDX_D]);
  flux = k[34]*n[IDX_H2]*n[IDX_D];
  g[34] += flux * (mu[IDX_HD] + mu[IDX_H] - mu[IDX_H2] - mu[IDX_D]);
  flux = k[35]*n[IDX_HD]*n[IDX_H];
  g[35] += flux * (mu[IDX_H2] + mu[IDX_D] - mu[IDX_HD] - mu[IDX_H]);
  flux = k[36]*n[IDX_D]*n[IDX_Hk];
  g[36] += flux * (mu[IDX_HD] + mu[IDX_E] - mu[IDX_D] - mu[IDX_Hk]);
  flux = k[37]*n[IDX_Dj]*n[IDX_E];
  g[37] += flux * (mu[IDX_D] - mu[IDX_Dj] - mu[IDX_E]);
  if (muT != 0.0) {
    const double c = muT * (gamma_index(Tth, n, p) - 1.0) / (kbc::boltzmann_erg * ntot_(n)) * kbc::eV_to_erg;
    const double dd = Hnuclei_(n);
    const double ncr = 1.0e6 / std::sqrt(Tth)
        / (1.6 * kb_exp(-kb_pow(4.0e2 / Tth, 2.0)) * n[IDX_H] / dd
           + 1.4 * kb_exp(-1.2e4 / (Tth + 1.2e3)) * n[IDX_H2] / dd);
    const double ffac = 1.0 / (1.0 + ncr / dd);
    (void)ffac;
    g[9] += c * k[9] * (3.53*ffac) * n[IDX_Hk]*n[IDX_H];
    g[10] += c * k[10] * (3.53*ffac) * n[IDX_Hk]*n[IDX_H];
    g[13] += c * k[13] * (1.83*ffac) * n[IDX_H2j]*n[IDX_H];
    g[25] += c * k[25] * (4.48*ffac) * n[IDX_H]*n[IDX_H]*n[IDX_H];
    g[26] += c * k[26] * (4.48*ffac) * n[IDX_H]*n[IDX_H]*n[IDX_H];
    g[27] += c * k[27] * (4.48*ffac) * n[IDX_H2]*n[IDX_H]*n[IDX_H];
    g[28] += c * k[28] * (4.48*ffac) * n[IDX_H2]*n[IDX_H]*n[IDX_H];
  }
}

// reaction labels: the equation, and the T range of a piece
inline const char* const reaction_names[38] = {"H + e- -> H+ + e- + e-", "H+ + e- -> H [0.0, 5500.0]", "H+ + e- -> H [5500.0, INFINITY]", "He + e- -> He+ + e- + e-", "He+ + e- -> He [0.0, 9280.0]", "He+ + e- -> He [9280.0, INFINITY]", "He+ + e- -> He++ + e- + e-", "He++ + e- -> He+", "H + e- -> H-", "H- + H -> H2 + e- [0.0, 1160.0]", "H- + H -> H2 + e- [1160.0, INFINITY]", "H + H+ -> H2+ [0.0, 6700.0]", "H + H+ -> H2+ [6700.0, INFINITY]", "H2+ + H -> H2 + H+", "H2 + H+ -> H2+ + H [3480.0, INFINITY]", "H2 + e- -> H + H + e-", "H2 + H -> H + H + H", "H- + e- -> H + e- + e-", "H- + H -> H + H + e- [0.0, 1160.0]", "H- + H -> H + H + e- [1160.0, INFINITY]", "H- + H+ -> H + H", "H- + H+ -> H2+ + e-", "H2+ + e- -> H + H [0.0, 617.0]", "H2+ + e- -> H + H [617.0, INFINITY]", "H2+ + H- -> H + H2", "H + H + H -> H2 + H [0.0, 300.0]", "H + H + H -> H2 + H [300.0, INFINITY]", "H2 + H + H -> H2 + H2 [0.0, 300.0]", "H2 + H + H -> H2 + H2 [300.0, INFINITY]", "H+ + D -> H + D+ [50.0, INFINITY]", "H + D+ -> H+ + D [50.0, INFINITY]", "H2 + D+ -> HD + H+", "HD + H+ -> H2 + D+", "H2 + D -> HD + H [0.0, 2000.0]", "H2 + D -> HD + H [2000.0, INFINITY]", "HD + H -> H2 + D [200.0, INFINITY]", "D + H- -> HD + e-", "D+ + e- -> D"};
constexpr int NHEAT = 2;
constexpr int NCOOL = 2;
inline const char* const heat_names[2] = {"CHEM", "COMPRESS"};
inline const char* const cool_names[2] = {"ATOMIC", "H2"};
// the thermal terms one by one [erg cm^-3 s^-1] at the thermal
// temperature T with the rates k: H[NHEAT], C[NCOOL] in the order
// of heat_names / cool_names (their sums are thermal_dTdt's)
KB_HD inline void thermal_terms(double T, const double* n, const double* k, const Params& p, double* H, double* C) {
  (void)T; (void)n; (void)k; (void)p; (void)H; (void)C;
  H[0] = heating_chem(T, n, k);
  H[1] = ntot_(n) * kbc::boltzmann_erg * T / p.tff;
  C[0] = cooling_Atomic(T, n) + cooling_recomb_(T, n, p);
  C[1] = cooling_H2(T, n) * h2_opacity_(n);
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
  fl[10] = k[10]*n[IDX_Hk]*n[IDX_H];
  fl[11] = k[11]*n[IDX_H]*n[IDX_Hj];
  fl[12] = k[12]*n[IDX_H]*n[IDX_Hj];
  fl[13] = k[13]*n[IDX_H2j]*n[IDX_H];
  fl[14] = k[14]*n[IDX_H2]*n[IDX_Hj];
  fl[15] = k[15]*n[IDX_H2]*n[IDX_E];
  fl[16] = k[16]*n[IDX_H2]*n[IDX_H];
  fl[17] = k[17]*n[IDX_Hk]*n[IDX_E];
  fl[18] = k[18]*n[IDX_Hk]*n[IDX_H];
  fl[19] = k[19]*n[IDX_Hk]*n[IDX_H];
  fl[20] = k[20]*n[IDX_Hk]*n[IDX_Hj];
  fl[21] = k[21]*n[IDX_Hk]*n[IDX_Hj];
  fl[22] = k[22]*n[IDX_H2j]*n[IDX_E];
  fl[23] = k[23]*n[IDX_H2j]*n[IDX_E];
  fl[24] = k[24]*n[IDX_H2j]*n[IDX_Hk];
  fl[25] = k[25]*n[IDX_H]*n[IDX_H]*n[IDX_H];
  fl[26] = k[26]*n[IDX_H]*n[IDX_H]*n[IDX_H];
  fl[27] = k[27]*n[IDX_H2]*n[IDX_H]*n[IDX_H];
  fl[28] = k[28]*n[IDX_H2]*n[IDX_H]*n[IDX_H];
  fl[29] = k[29]*n[IDX_Hj]*n[IDX_D];
  fl[30] = k[30]*n[IDX_H]*n[IDX_Dj];
  fl[31] = k[31]*n[IDX_H2]*n[IDX_Dj];
  fl[32] = k[32]*n[IDX_HD]*n[IDX_Hj];
  fl[33] = k[33]*n[IDX_H2]*n[IDX_D];
  fl[34] = k[34]*n[IDX_H2]*n[IDX_D];
  fl[35] = k[35]*n[IDX_HD]*n[IDX_H];
  fl[36] = k[36]*n[IDX_D]*n[IDX_Hk];
  fl[37] = k[37]*n[IDX_Dj]*n[IDX_E];
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
constexpr bool RATES_DEPEND_ON_N = false;
}  // namespace kbnet
