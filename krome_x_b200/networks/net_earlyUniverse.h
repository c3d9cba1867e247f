// Generated by krome_x_b200.emit from the network 'earlyUniverse' -- do not edit.
// One host/device (KB_HD) scalar form of the network: species,
// parameters, rate coefficients, mass-action rhs, stoichiometric
// Jacobian and the thermal equation (see krome_x_b200/emit/
// emitter.py for the layout and the reference rules it follows).
#pragma once
#include "../csrc/kb_common.h"

namespace kbnet {

constexpr const char* NETWORK_NAME = "earlyUniverse";
constexpr const char* NETWORK_KEY = "earlyUniverse";
constexpr int NSPEC = 16;
constexpr int NREA = 64;
constexpr int KB_RATE_NDEP = 6;
#define KB_NFREEZE 12
constexpr int IDX_D = 0;
constexpr int IDX_Dj = 1;
constexpr int IDX_H = 2;
constexpr int IDX_Hj = 3;
constexpr int IDX_Hk = 4;
constexpr int IDX_H2 = 5;
constexpr int IDX_H2j = 6;
constexpr int IDX_H2Dj = 7;
constexpr int IDX_H3j = 8;
constexpr int IDX_HD = 9;
constexpr int IDX_HDj = 10;
constexpr int IDX_He = 11;
constexpr int IDX_Hej = 12;
constexpr int IDX_Hejj = 13;
constexpr int IDX_HeHj = 14;
constexpr int IDX_E = 15;
#define KB_HAS_D 1
#define KB_HAS_Dj 1
#define KB_HAS_H 1
#define KB_HAS_Hj 1
#define KB_HAS_Hk 1
#define KB_HAS_H2 1
#define KB_HAS_H2j 1
#define KB_HAS_H2Dj 1
#define KB_HAS_H3j 1
#define KB_HAS_HD 1
#define KB_HAS_HDj 1
#define KB_HAS_He 1
#define KB_HAS_Hej 1
#define KB_HAS_Hejj 1
#define KB_HAS_HeHj 1
#define KB_HAS_E 1
#define KB_EXTERN_recfast_H_ion 1
#define KB_EXTERN_recfast_H_rec 1
#define KB_EXTERN_recfast_He_ion 1
#define KB_EXTERN_recfast_He_rec 1
constexpr int IDX_ELECTRON = 15;

inline const char* const species_names[NSPEC] = {"D", "D+", "H", "H+", "H-", "H2", "H2+", "H2D+", "H3+", "HD", "HD+", "He", "He+", "He++", "HeH+", "e-"};
constexpr int NELEM = 3;
inline const char* const element_names[3] = {"D", "H", "He"};
KB_HD inline double species_mass_g(int i) {
  constexpr double t_[NSPEC] = {3.3443256801323995e-24, 3.343414741762353e-24, 1.6738233791328e-24, 1.6729124407627538e-24, 1.6747343175028463e-24, 3.3476467582656e-24, 3.346735819895553e-24, 6.691061500027952e-24, 5.020559199028353e-24, 5.0181490592651994e-24, 5.017238120895153e-24, 6.64647366797316e-24, 6.645562729603113e-24, 6.644651791233067e-24, 8.319386108735913e-24, 9.10938370046373e-28};
  return t_[i];
}
KB_HD inline int species_charge(int i) {
  constexpr int t_[NSPEC] = {0, 1, 0, 1, -1, 0, 1, 1, 1, 0, 1, 0, 1, 2, 1, -1};
  return t_[i];
}
KB_HD inline double species_natoms_H(int i) {
  constexpr double t_[NSPEC] = {0.0, 0.0, 1.0, 1.0, 1.0, 2.0, 2.0, 2.0, 3.0, 1.0, 1.0, 0.0, 0.0, 0.0, 1.0, 0.0};
  return t_[i];
}
KB_HD inline int species_opaque(int i) {
  constexpr int t_[NSPEC] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
  return t_[i];
}
inline constexpr int species_elements_t_[48] = {1, 0, 0, 1, 0, 0, 0, 1, 0, 0, 1, 0, 0, 1, 0, 0, 2, 0, 0, 2, 0, 1, 2, 0, 0, 3, 0, 1, 1, 0, 1, 1, 0, 0, 0, 1, 0, 0, 1, 0, 0, 1, 0, 1, 1, 0, 0, 0};
#ifdef __CUDACC__
__device__ const int d_species_elements_[48] = {1, 0, 0, 1, 0, 0, 0, 1, 0, 0, 1, 0, 0, 1, 0, 0, 2, 0, 0, 2, 0, 1, 2, 0, 0, 3, 0, 1, 1, 0, 1, 1, 0, 0, 0, 1, 0, 0, 1, 0, 0, 1, 0, 1, 1, 0, 0, 0};
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

constexpr int NPAR = 6;
constexpr int NPHOTO = 0;
struct Params {
  double Trad;
  double gamma_ad;
  double Tcmb;
  double zredshift;
  double hubble0;
  double omega0;
};
inline const char* const param_names[NPAR] = {"Trad", "gamma_ad", "Tcmb", "zredshift", "hubble0", "omega0"};
// the defaults of a parameter row; NaN marks a REQUIRED parameter
inline double param_default(int i) {
  const double t_[NPAR] = {0.0, 1.6666666666666667, 2.725, 0.0, NAN, NAN};
  return t_[i];
}
inline const char* const param_required_by[NPAR] = {"", "", "", "", "recfast_H_ion(), recfast_H_rec(), recfast_He_ion(), recfast_He_rec()", "recfast_H_ion(), recfast_H_rec(), recfast_He_ion(), recfast_He_rec()"};
KB_HD inline void params_from_row(const double* row, Params& p) {
  p.Trad = row[0];
  p.gamma_ad = row[1];
  p.Tcmb = row[2];
  p.zredshift = row[3];
  p.hubble0 = row[4];
  p.omega0 = row[5];
}
KB_HD inline int params_missing(const Params& p) {
  (void)p;
  if (p.hubble0 != p.hubble0) return 4;
  if (p.omega0 != p.omega0) return 5;
  return -1;
}
KB_HD inline bool freeze_active(const Params& p) {
  (void)p;
  if (p.zredshift > 2243.0) return true;  // knet line 45
  return false;
}
KB_HD inline int frozen_species(const Params& p, int* idx) {
  (void)p; (void)idx;
  int m = 0;
  if (p.zredshift > 2243.0) {  // knet line 45
    idx[m++] = IDX_E; idx[m++] = IDX_H; idx[m++] = IDX_H2; idx[m++] = IDX_Hj; idx[m++] = IDX_H2j; idx[m++] = IDX_Hk; idx[m++] = IDX_D; idx[m++] = IDX_Dj; idx[m++] = IDX_HD; idx[m++] = IDX_HDj; idx[m++] = IDX_H2Dj; idx[m++] = IDX_H3j;
  }
  return m;
}

#include "../csrc/kb_physics.h"
#include "../csrc/kb_conserve.h"
#include "../csrc/kb_jacdk.h"

KB_HD inline double v_invTgas(double Tgas, const double* n, const Params& p) {
  (void)Tgas; (void)n; (void)p;
  return 1.0 / Tgas;
}

// rate coefficients of Tgas and the parameters only
KB_HD inline void rates_fixed(double Tgas, const double* n, const Params& p, double* k) {
  (void)Tgas; (void)n; (void)p; (void)k;
  const double vh_invTgas = v_invTgas(Tgas, n, p);
  (void)vh_invTgas;
  k[2] = 1.4e-18 * kb_pow(Tgas, 0.928) * kb_exp(-Tgas / 16200.0);  // H + e- -> H-
  k[3] = 0.11 * kb_pow(p.Trad, 2.13) * kb_exp(-8823.0 / p.Trad);  // H- -> H + e-
  k[8] = 5.7e-06 * 1.0/(std::sqrt(Tgas)) + 6.3e-08 - 9.2e-11 * std::sqrt(Tgas) + 4.4e-13 * Tgas;  // H- + H+ -> H + H
  k[9] = kb_exp10(-19.38 - 1.523 * kb_log10(Tgas) + 1.118 * kb_log10(Tgas)*kb_log10(Tgas) - 0.1269 * kb_log10(Tgas)*kb_log10(Tgas)*kb_log10(Tgas));  // H + H+ -> H2+
  k[10] = 16300000.0 * kb_exp(-32400.0 / p.Trad);  // H2+ -> H + H+
  k[11] = 6.4e-10;  // H2+ + H -> H2 + H+
  k[12] = 2e-07 * 1.0/(std::sqrt(Tgas));  // H2+ + e- -> H + H
  k[13] = 90.0 * kb_pow(p.Trad, 1.48) * kb_exp(-335000.0 / p.Trad);  // H2+ -> H+ + H+ + e-
  k[14] = 2e-09;  // H2+ + H2 -> H3+ + H
  k[17] = 2.7e-08 * kb_pow(Tgas, -1.27) * kb_exp(-43000.0 * vh_invTgas);  // H2 + e- -> H + H-
  k[18] = 4.4e-10 * kb_pow(Tgas, 0.35) * kb_exp(-102000.0 * vh_invTgas);  // H2 + e- -> H + H + e-
  k[19] = 290.0 * kb_pow(p.Trad, 1.56) * kb_exp(-178500.0 / p.Trad);  // H2 -> H2+ + e-
  k[20] = 7.7e-09 * kb_exp(-17560.0 * vh_invTgas);  // H3+ + H -> H2+ + H2
  k[21] = 4.6e-06 * kb_pow(Tgas, -0.65);  // H3+ + e- -> H2 + H
  k[22] = 1e-16;  // H2 + H+ -> H3+
  k[23] = 1.891e-10 * ipow_<-1>(std::sqrt(Tgas / 9.37) * kb_pow(1.0 + std::sqrt(Tgas / 9.37), 0.2476) * kb_pow(1.0 + std::sqrt(Tgas / 2774000.0), 1.7524));  // He++ + e- -> He+
  k[24] = (p.Trad > 1000.0 ? 50.0 * kb_pow(p.Trad, 1.63) * kb_exp(-590000.0 / p.Trad) : 0.0);  // He+ -> He++ + e-
  k[31] = 3e-10 * kb_exp(-6717.0 * vh_invTgas);  // He + H2+ -> HeH+ + H
  k[34] = 9.1e-10;  // HeH+ + H -> He + H2+
  k[35] = 1.7e-07 * 1.0/(std::sqrt(Tgas));  // HeH+ + e- -> He + H
  k[36] = 1.3e-09;  // HeH+ + H2 -> H3+ + He
  k[37] = 0.68 * ipow_<1>(p.Trad) * std::sqrt(p.Trad) * kb_exp(-22750.0 / p.Trad);  // HeH+ -> He + H+
  k[38] = 7800.0 * kb_pow(p.Trad, 1.2) * kb_exp(-240000.0 / p.Trad);  // HeH+ -> He+ + H
  k[41] = 3.7e-10 * kb_pow(Tgas, 0.28) * kb_exp(-43.0 * vh_invTgas);  // D + H+ -> D+ + H
  k[42] = 3.7e-10 * kb_pow(Tgas, 0.28);  // D+ + H -> D + H+
  k[43] = 1e-25;  // D + H -> HD
  k[45] = 6.4e-10;  // HD+ + H -> H+ + HD
  k[46] = 2.1e-09;  // D+ + H2 -> H+ + HD
  k[48] = 1e-09 * kb_exp(-464.0 * vh_invTgas);  // HD + H+ -> H2 + D+
  k[49] = (2.1 - 0.4 * kb_log10(Tgas)) * 1e-09;  // HD + H3+ -> H2 + H2D+
  k[50] = kb_exp10(-19.38 - 1.523 * kb_log10(Tgas) + 1.118 * kb_log10(Tgas)*kb_log10(Tgas) - 0.1269 * kb_log10(Tgas)*kb_log10(Tgas)*kb_log10(Tgas));  // D + H+ -> HD+
  k[51] = kb_exp10(-19.38 - 1.523 * kb_log10(Tgas) + 1.118 * kb_log10(Tgas)*kb_log10(Tgas) - 0.1269 * kb_log10(Tgas)*kb_log10(Tgas)*kb_log10(Tgas));  // D+ + H -> HD+
  k[52] = 16300000.0 * kb_exp(-32400.0 / p.Trad);  // HD+ -> H + D+
  k[53] = 16300000.0 * kb_exp(-32400.0 / p.Trad);  // HD+ -> H+ + D
  k[54] = 7.2e-08 * 1.0/(std::sqrt(Tgas));  // HD+ + e- -> H + D
  k[55] = 2e-09;  // HD+ + H2 -> H2D+ + H
  k[56] = 2e-09;  // HD+ + H2 -> H3+ + D
  k[57] = 1e-09;  // D + H3+ -> H2D+ + H
  k[58] = 1e-06 * 1.0/(std::sqrt(Tgas)) * 0.73;  // H2D+ + e- -> H + H + D
  k[59] = 1e-06 * 1.0/(std::sqrt(Tgas)) * 0.07;  // H2D+ + e- -> H2 + D
  k[60] = 1e-06 * 1.0/(std::sqrt(Tgas)) * 0.2;  // H2D+ + e- -> HD + H
  k[63] = 1e-09 * kb_exp(-598.0 * vh_invTgas);  // H2D+ + H -> H3+ + D
  {  // group 1: H- + H -> H2 + e-
    double T = Tgas;
    if (T < 300.0) {
      k[4] = 1.5e-09;  // H- + H -> H2 + e-
    }
    else if (T >= 300.0) {
      k[5] = 4e-09 * kb_pow(T, -0.17);  // H- + H -> H2 + e-
    }
  }
  {  // group 2: H- + H+ -> H2+ + e-
    double T = Tgas;
    if (T < 8000.0) {
      k[6] = 6.9e-09 * kb_pow(T, -0.35);  // H- + H+ -> H2+ + e-
    }
    else if (T >= 8000.0) {
      k[7] = 9.6e-07 * kb_pow(T, -0.9);  // H- + H+ -> H2+ + e-
    }
  }
  {  // group 3: H2 + H+ -> H2+ + H
    double T = Tgas;
    const double vh_invTgas = v_invTgas(T, n, p);
    (void)vh_invTgas;
    if (T < 10000.0) {
      k[15] = 3e-10 * kb_exp(-21050.0 * vh_invTgas);  // H2 + H+ -> H2+ + H
    }
    else if (T >= 10000.0) {
      k[16] = 1.5e-10 * kb_exp(-14000.0 * vh_invTgas);  // H2 + H+ -> H2+ + H
    }
  }
  {  // group 4: He + H+ -> He+ + H
    double T = Tgas;
    if (T >= 10000.0 && T >= 10000.0) {
      k[27] = 4e-37 * kb_pow(T, 4.74);  // He + H+ -> He+ + H
    }
  }
  {  // group 5: He+ + H -> He + H+
    double T = Tgas;
    if (T >= 6000.0 && T >= 6000.0) {
      k[28] = 3.7e-25 * kb_pow(T, 2.06) * (1.0 + 9.9 * kb_exp(-T / 2570.0));  // He+ + H -> He + H+
    }
  }
  {  // group 6: He + H+ -> HeH+
    double T = Tgas;
    if (T < 1000.0) {
      k[29] = 7.6e-18 * 1.0/(std::sqrt(T)) + 5e-21;  // He + H+ -> HeH+
    }
    else if (T >= 1000.0) {
      k[30] = 3.45e-16 * kb_pow(T, -1.06) + 5e-21;  // He + H+ -> HeH+
    }
  }
  {  // group 7: He+ + H -> HeH+
    double T = Tgas;
    if (T < 4000.0) {
      k[32] = 1.6e-14 * kb_pow(T, -0.33);  // He+ + H -> HeH+
    }
    else if (T >= 4000.0) {
      k[33] = 1e-15;  // He+ + H -> HeH+
    }
  }
  {  // group 8: D + H2 -> H + HD
    double T = Tgas;
    const double vh_invTgas = v_invTgas(T, n, p);
    (void)vh_invTgas;
    if (T >= 250.0 && T >= 250.0) {
      k[44] = 9e-11 * kb_exp(-3876.0 * vh_invTgas);  // D + H2 -> H + HD
    }
  }
  {  // group 9: HD + H -> H2 + D
    double T = Tgas;
    const double vh_invTgas = v_invTgas(T, n, p);
    (void)vh_invTgas;
    if (T >= 200.0 && T >= 200.0) {
      k[47] = 3.2e-11 * kb_exp(-3624.0 * vh_invTgas);  // HD + H -> H2 + D
    }
  }
  {  // group 10: H2D+ + H2 -> H3+ + HD
    double T = Tgas;
    const double vh_invTgas = v_invTgas(T, n, p);
    (void)vh_invTgas;
    if (T < 100.0) {
      k[61] = 4.7e-09 * kb_exp(-215.0 * vh_invTgas);  // H2D+ + H2 -> H3+ + HD
    }
    else if (T >= 100.0) {
      k[62] = 5.5e-10;  // H2D+ + H2 -> H3+ + HD
    }
  }
}
// rate coefficients that also depend on the densities
KB_HD inline void rates_var(double Tgas, const double* n, const Params& p, double* k) {
  (void)Tgas; (void)n; (void)p; (void)k;
  k[0] = recfast_H_rec(n[IDX_H], Tgas, n, p);  // H+ + e- -> H
  k[1] = recfast_H_ion(n[IDX_H], Tgas, n, p);  // H -> H+ + e-
  k[25] = recfast_He_rec(n[IDX_He], n[IDX_H], Tgas, n, p);  // He+ + e- -> He
  k[26] = recfast_He_ion(n[IDX_He], n[IDX_H], Tgas, n, p);  // He -> He+ + e-
  k[39] = recfast_H_rec(n[IDX_D], Tgas, n, p);  // D+ + e- -> D
  k[40] = recfast_H_ion(n[IDX_D], Tgas, n, p);  // D -> D+ + e-
}
constexpr int NREA_FIXED = 58;
KB_HD inline bool rate_is_fixed(int r) {
  switch (r) {
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
    case 38:
    case 41:
    case 42:
    case 43:
    case 44:
    case 45:
    case 46:
    case 47:
    case 48:
    case 49:
    case 50:
    case 51:
    case 52:
    case 53:
    case 54:
    case 55:
    case 56:
    case 57:
    case 58:
    case 59:
    case 60:
    case 61:
    case 62:
    case 63:
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
  flux = k[0]*n[IDX_Hj]*n[IDX_E];
  dn[IDX_Hj] -= flux;
  dn[IDX_E] -= flux;
  dn[IDX_H] += flux;
  flux = k[1]*n[IDX_H];
  dn[IDX_H] -= flux;
  dn[IDX_Hj] += flux;
  dn[IDX_E] += flux;
  flux = k[2]*n[IDX_H]*n[IDX_E];
  dn[IDX_H] -= flux;
  dn[IDX_E] -= flux;
  dn[IDX_Hk] += flux;
  flux = k[3]*n[IDX_Hk];
  dn[IDX_Hk] -= flux;
  dn[IDX_H] += flux;
  dn[IDX_E] += flux;
  flux = k[4]*n[IDX_Hk]*n[IDX_H];
  dn[IDX_Hk] -= flux;
  dn[IDX_H] -= flux;
  dn[IDX_H2] += flux;
  dn[IDX_E] += flux;
  flux = k[5]*n[IDX_Hk]*n[IDX_H];
  dn[IDX_Hk] -= flux;
  dn[IDX_H] -= flux;
  dn[IDX_H2] += flux;
  dn[IDX_E] += flux;
  flux = k[6]*n[IDX_Hk]*n[IDX_Hj];
  dn[IDX_Hk] -= flux;
  dn[IDX_Hj] -= flux;
  dn[IDX_H2j] += flux;
  dn[IDX_E] += flux;
  flux = k[7]*n[IDX_Hk]*n[IDX_Hj];
  dn[IDX_Hk] -= flux;
  dn[IDX_Hj] -= flux;
  dn[IDX_H2j] += flux;
  dn[IDX_E] += flux;
  flux = k[8]*n[IDX_Hk]*n[IDX_Hj];
  dn[IDX_Hk] -= flux;
  dn[IDX_Hj] -= flux;
  dn[IDX_H] += flux;
  dn[IDX_H] += flux;
  flux = k[9]*n[IDX_H]*n[IDX_Hj];
  dn[IDX_H] -= flux;
  dn[IDX_Hj] -= flux;
  dn[IDX_H2j] += flux;
  flux = k[10]*n[IDX_H2j];
  dn[IDX_H2j] -= flux;
  dn[IDX_H] += flux;
  dn[IDX_Hj] += flux;
  flux = k[11]*n[IDX_H2j]*n[IDX_H];
  dn[IDX_H2j] -= flux;
  dn[IDX_H] -= flux;
  dn[IDX_H2] += flux;
  dn[IDX_Hj] += flux;
  flux = k[12]*n[IDX_H2j]*n[IDX_E];
  dn[IDX_H2j] -= flux;
  dn[IDX_E] -= flux;
  dn[IDX_H] += flux;
  dn[IDX_H] += flux;
  flux = k[13]*n[IDX_H2j];
  dn[IDX_H2j] -= flux;
  dn[IDX_Hj] += flux;
  dn[IDX_Hj] += flux;
  dn[IDX_E] += flux;
  flux = k[14]*n[IDX_H2j]*n[IDX_H2];
  dn[IDX_H2j] -= flux;
  dn[IDX_H2] -= flux;
  dn[IDX_H3j] += flux;
  dn[IDX_H] += flux;
  flux = k[15]*n[IDX_H2]*n[IDX_Hj];
  dn[IDX_H2] -= flux;
  dn[IDX_Hj] -= flux;
  dn[IDX_H2j] += flux;
  dn[IDX_H] += flux;
  flux = k[16]*n[IDX_H2]*n[IDX_Hj];
  dn[IDX_H2] -= flux;
  dn[IDX_Hj] -= flux;
  dn[IDX_H2j] += flux;
  dn[IDX_H] += flux;
  flux = k[17]*n[IDX_H2]*n[IDX_E];
  dn[IDX_H2] -= flux;
  dn[IDX_E] -= flux;
  dn[IDX_H] += flux;
  dn[IDX_Hk] += flux;
  flux = k[18]*n[IDX_H2]*n[IDX_E];
  dn[IDX_H2] -= flux;
  dn[IDX_E] -= flux;
  dn[IDX_H] += flux;
  dn[IDX_H] += flux;
  dn[IDX_E] += flux;
  flux = k[19]*n[IDX_H2];
  dn[IDX_H2] -= flux;
  dn[IDX_H2j] += flux;
  dn[IDX_E] += flux;
  flux = k[20]*n[IDX_H3j]*n[IDX_H];
  dn[IDX_H3j] -= flux;
  dn[IDX_H] -= flux;
  dn[IDX_H2j] += flux;
  dn[IDX_H2] += flux;
  flux = k[21]*n[IDX_H3j]*n[IDX_E];
  dn[IDX_H3j] -= flux;
  dn[IDX_E] -= flux;
  dn[IDX_H2] += flux;
  dn[IDX_H] += flux;
  flux = k[22]*n[IDX_H2]*n[IDX_Hj];
  dn[IDX_H2] -= flux;
  dn[IDX_Hj] -= flux;
  dn[IDX_H3j] += flux;
  flux = k[23]*n[IDX_Hejj]*n[IDX_E];
  dn[IDX_Hejj] -= flux;
  dn[IDX_E] -= flux;
  dn[IDX_Hej] += flux;
  flux = k[24]*n[IDX_Hej];
  dn[IDX_Hej] -= flux;
  dn[IDX_Hejj] += flux;
  dn[IDX_E] += flux;
  flux = k[25]*n[IDX_Hej]*n[IDX_E];
  dn[IDX_Hej] -= flux;
  dn[IDX_E] -= flux;
  dn[IDX_He] += flux;
  flux = k[26]*n[IDX_He];
  dn[IDX_He] -= flux;
  dn[IDX_Hej] += flux;
  dn[IDX_E] += flux;
  flux = k[27]*n[IDX_He]*n[IDX_Hj];
  dn[IDX_He] -= flux;
  dn[IDX_Hj] -= flux;
  dn[IDX_Hej] += flux;
  dn[IDX_H] += flux;
  flux = k[28]*n[IDX_Hej]*n[IDX_H];
  dn[IDX_Hej] -= flux;
  dn[IDX_H] -= flux;
  dn[IDX_He] += flux;
  dn[IDX_Hj] += flux;
  flux = k[29]*n[IDX_He]*n[IDX_Hj];
  dn[IDX_He] -= flux;
  dn[IDX_Hj] -= flux;
  dn[IDX_HeHj] += flux;
  flux = k[30]*n[IDX_He]*n[IDX_Hj];
  dn[IDX_He] -= flux;
  dn[IDX_Hj] -= flux;
  dn[IDX_HeHj] += flux;
  flux = k[31]*n[IDX_He]*n[IDX_H2j];
  dn[IDX_He] -= flux;
  dn[IDX_H2j] -= flux;
  dn[IDX_HeHj] += flux;
  dn[IDX_H] += flux;
  flux = k[32]*n[IDX_Hej]*n[IDX_H];
  dn[IDX_Hej] -= flux;
  dn[IDX_H] -= flux;
  dn[IDX_HeHj] += flux;
  flux = k[33]*n[IDX_Hej]*n[IDX_H];
  dn[IDX_Hej] -= flux;
  dn[IDX_H] -= flux;
  dn[IDX_HeHj] += flux;
  flux = k[34]*n[IDX_HeHj]*n[IDX_H];
  dn[IDX_HeHj] -= flux;
  dn[IDX_H] -= flux;
  dn[IDX_He] += flux;
  dn[IDX_H2j] += flux;
  flux = k[35]*n[IDX_HeHj]*n[IDX_E];
  dn[IDX_HeHj] -= flux;
  dn[IDX_E] -= flux;
  dn[IDX_He] += flux;
  dn[IDX_H] += flux;
  flux = k[36]*n[IDX_HeHj]*n[IDX_H2];
  dn[IDX_HeHj] -= flux;
  dn[IDX_H2] -= flux;
  dn[IDX_H3j] += flux;
  dn[IDX_He] += flux;
  flux = k[37]*n[IDX_HeHj];
  dn[IDX_HeHj] -= flux;
  dn[IDX_He] += flux;
  dn[IDX_Hj] += flux;
  flux = k[38]*n[IDX_HeHj];
  dn[IDX_HeHj] -= flux;
  dn[IDX_Hej] += flux;
  dn[IDX_H] += flux;
  flux = k[39]*n[IDX_Dj]*n[IDX_E];
  dn[IDX_Dj] -= flux;
  dn[IDX_E] -= flux;
  dn[IDX_D] += flux;
  flux = k[40]*n[IDX_D];
  dn[IDX_D] -= flux;
  dn[IDX_Dj] += flux;
  dn[IDX_E] += flux;
  flux = k[41]*n[IDX_D]*n[IDX_Hj];
  dn[IDX_D] -= flux;
  dn[IDX_Hj] -= flux;
  dn[IDX_Dj] += flux;
  dn[IDX_H] += flux;
  flux = k[42]*n[IDX_Dj]*n[IDX_H];
  dn[IDX_Dj] -= flux;
  dn[IDX_H] -= flux;
  dn[IDX_D] += flux;
  dn[IDX_Hj] += flux;
  flux = k[43]*n[IDX_D]*n[IDX_H];
  dn[IDX_D] -= flux;
  dn[IDX_H] -= flux;
  dn[IDX_HD] += flux;
  flux = k[44]*n[IDX_D]*n[IDX_H2];
  dn[IDX_D] -= flux;
  dn[IDX_H2] -= flux;
  dn[IDX_H] += flux;
  dn[IDX_HD] += flux;
  flux = k[45]*n[IDX_HDj]*n[IDX_H];
  dn[IDX_HDj] -= flux;
  dn[IDX_H] -= flux;
  dn[IDX_Hj] += flux;
  dn[IDX_HD] += flux;
  flux = k[46]*n[IDX_Dj]*n[IDX_H2];
  dn[IDX_Dj] -= flux;
  dn[IDX_H2] -= flux;
  dn[IDX_Hj] += flux;
  dn[IDX_HD] += flux;
  flux = k[47]*n[IDX_HD]*n[IDX_H];
  dn[IDX_HD] -= flux;
  dn[IDX_H] -= flux;
  dn[IDX_H2] += flux;
  dn[IDX_D] += flux;
  flux = k[48]*n[IDX_HD]*n[IDX_Hj];
  dn[IDX_HD] -= flux;
  dn[IDX_Hj] -= flux;
  dn[IDX_H2] += flux;
  dn[IDX_Dj] += flux;
  flux = k[49]*n[IDX_HD]*n[IDX_H3j];
  dn[IDX_HD] -= flux;
  dn[IDX_H3j] -= flux;
  dn[IDX_H2] += flux;
  dn[IDX_H2Dj] += flux;
  flux = k[50]*n[IDX_D]*n[IDX_Hj];
  dn[IDX_D] -= flux;
  dn[IDX_Hj] -= flux;
  dn[IDX_HDj] += flux;
  flux = k[51]*n[IDX_Dj]*n[IDX_H];
  dn[IDX_Dj] -= flux;
  dn[IDX_H] -= flux;
  dn[IDX_HDj] += flux;
  flux = k[52]*n[IDX_HDj];
  dn[IDX_HDj] -= flux;
  dn[IDX_H] += flux;
  dn[IDX_Dj] += flux;
  flux = k[53]*n[IDX_HDj];
  dn[IDX_HDj] -= flux;
  dn[IDX_Hj] += flux;
  dn[IDX_D] += flux;
  flux = k[54]*n[IDX_HDj]*n[IDX_E];
  dn[IDX_HDj] -= flux;
  dn[IDX_E] -= flux;
  dn[IDX_H] += flux;
  dn[IDX_D] += flux;
  flux = k[55]*n[IDX_HDj]*n[IDX_H2];
  dn[IDX_HDj] -= flux;
  dn[IDX_H2] -= flux;
  dn[IDX_H2Dj] += flux;
  dn[IDX_H] += flux;
  flux = k[56]*n[IDX_HDj]*n[IDX_H2];
  dn[IDX_HDj] -= flux;
  dn[IDX_H2] -= flux;
  dn[IDX_H3j] += flux;
  dn[IDX_D] += flux;
  flux = k[57]*n[IDX_D]*n[IDX_H3j];
  dn[IDX_D] -= flux;
  dn[IDX_H3j] -= flux;
  dn[IDX_H2Dj] += flux;
  dn[IDX_H] += flux;
  flux = k[58]*n[IDX_H2Dj]*n[IDX_E];
  dn[IDX_H2Dj] -= flux;
  dn[IDX_E] -= flux;
  dn[IDX_H] += flux;
  dn[IDX_H] += flux;
  dn[IDX_D] += flux;
  flux = k[59]*n[IDX_H2Dj]*n[IDX_E];
  dn[IDX_H2Dj] -= flux;
  dn[IDX_E] -= flux;
  dn[IDX_H2] += flux;
  dn[IDX_D] += flux;
  flux = k[60]*n[IDX_H2Dj]*n[IDX_E];
  dn[IDX_H2Dj] -= flux;
  dn[IDX_E] -= flux;
  dn[IDX_HD] += flux;
  dn[IDX_H] += flux;
  flux = k[61]*n[IDX_H2Dj]*n[IDX_H2];
  dn[IDX_H2Dj] -= flux;
  dn[IDX_H2] -= flux;
  dn[IDX_H3j] += flux;
  dn[IDX_HD] += flux;
  flux = k[62]*n[IDX_H2Dj]*n[IDX_H2];
  dn[IDX_H2Dj] -= flux;
  dn[IDX_H2] -= flux;
  dn[IDX_H3j] += flux;
  dn[IDX_HD] += flux;
  flux = k[63]*n[IDX_H2Dj]*n[IDX_H];
  dn[IDX_H2Dj] -= flux;
  dn[IDX_H] -= flux;
  dn[IDX_H3j] += flux;
  dn[IDX_D] += flux;
}

KB_HD inline void jac_stoich(const double* n, const double* k, double* J, int rs, int cs) {
  for (int i = 0; i < NSPEC; ++i)
    for (int j = 0; j < NSPEC; ++j) J[i*rs + j*cs] = 0.0;
  double d;
  (void)d; (void)n; (void)k;
  d = k[0]*n[IDX_E];
  J[IDX_Hj*rs + IDX_Hj*cs] -= d;
  J[IDX_E*rs + IDX_Hj*cs] -= d;
  J[IDX_H*rs + IDX_Hj*cs] += d;
  d = k[0]*n[IDX_Hj];
  J[IDX_Hj*rs + IDX_E*cs] -= d;
  J[IDX_E*rs + IDX_E*cs] -= d;
  J[IDX_H*rs + IDX_E*cs] += d;
  d = k[1];
  J[IDX_H*rs + IDX_H*cs] -= d;
  J[IDX_Hj*rs + IDX_H*cs] += d;
  J[IDX_E*rs + IDX_H*cs] += d;
  d = k[2]*n[IDX_E];
  J[IDX_H*rs + IDX_H*cs] -= d;
  J[IDX_E*rs + IDX_H*cs] -= d;
  J[IDX_Hk*rs + IDX_H*cs] += d;
  d = k[2]*n[IDX_H];
  J[IDX_H*rs + IDX_E*cs] -= d;
  J[IDX_E*rs + IDX_E*cs] -= d;
  J[IDX_Hk*rs + IDX_E*cs] += d;
  d = k[3];
  J[IDX_Hk*rs + IDX_Hk*cs] -= d;
  J[IDX_H*rs + IDX_Hk*cs] += d;
  J[IDX_E*rs + IDX_Hk*cs] += d;
  d = k[4]*n[IDX_Hk];
  J[IDX_Hk*rs + IDX_H*cs] -= d;
  J[IDX_H*rs + IDX_H*cs] -= d;
  J[IDX_H2*rs + IDX_H*cs] += d;
  J[IDX_E*rs + IDX_H*cs] += d;
  d = k[4]*n[IDX_H];
  J[IDX_Hk*rs + IDX_Hk*cs] -= d;
  J[IDX_H*rs + IDX_Hk*cs] -= d;
  J[IDX_H2*rs + IDX_Hk*cs] += d;
  J[IDX_E*rs + IDX_Hk*cs] += d;
  d = k[5]*n[IDX_Hk];
  J[IDX_Hk*rs + IDX_H*cs] -= d;
  J[IDX_H*rs + IDX_H*cs] -= d;
  J[IDX_H2*rs + IDX_H*cs] += d;
  J[IDX_E*rs + IDX_H*cs] += d;
  d = k[5]*n[IDX_H];
  J[IDX_Hk*rs + IDX_Hk*cs] -= d;
  J[IDX_H*rs + IDX_Hk*cs] -= d;
  J[IDX_H2*rs + IDX_Hk*cs] += d;
  J[IDX_E*rs + IDX_Hk*cs] += d;
  d = k[6]*n[IDX_Hk];
  J[IDX_Hk*rs + IDX_Hj*cs] -= d;
  J[IDX_Hj*rs + IDX_Hj*cs] -= d;
  J[IDX_H2j*rs + IDX_Hj*cs] += d;
  J[IDX_E*rs + IDX_Hj*cs] += d;
  d = k[6]*n[IDX_Hj];
  J[IDX_Hk*rs + IDX_Hk*cs] -= d;
  J[IDX_Hj*rs + IDX_Hk*cs] -= d;
  J[IDX_H2j*rs + IDX_Hk*cs] += d;
  J[IDX_E*rs + IDX_Hk*cs] += d;
  d = k[7]*n[IDX_Hk];
  J[IDX_Hk*rs + IDX_Hj*cs] -= d;
  J[IDX_Hj*rs + IDX_Hj*cs] -= d;
  J[IDX_H2j*rs + IDX_Hj*cs] += d;
  J[IDX_E*rs + IDX_Hj*cs] += d;
  d = k[7]*n[IDX_Hj];
  J[IDX_Hk*rs + IDX_Hk*cs] -= d;
  J[IDX_Hj*rs + IDX_Hk*cs] -= d;
  J[IDX_H2j*rs + IDX_Hk*cs] += d;
  J[IDX_E*rs + IDX_Hk*cs] += d;
  d = k[8]*n[IDX_Hk];
  J[IDX_Hk*rs + IDX_Hj*cs] -= d;
  J[IDX_Hj*rs + IDX_Hj*cs] -= d;
  J[IDX_H*rs + IDX_Hj*cs] += d;
  J[IDX_H*rs + IDX_Hj*cs] += d;
  d = k[8]*n[IDX_Hj];
  J[IDX_Hk*rs + IDX_Hk*cs] -= d;
  J[IDX_Hj*rs + IDX_Hk*cs] -= d;
  J[IDX_H*rs + IDX_Hk*cs] += d;
  J[IDX_H*rs + IDX_Hk*cs] += d;
  d = k[9]*n[IDX_Hj];
  J[IDX_H*rs + IDX_H*cs] -= d;
  J[IDX_Hj*rs + IDX_H*cs] -= d;
  J[IDX_H2j*rs + IDX_H*cs] += d;
  d = k[9]*n[IDX_H];
  J[IDX_H*rs + IDX_Hj*cs] -= d;
  J[IDX_Hj*rs + IDX_Hj*cs] -= d;
  J[IDX_H2j*rs + IDX_Hj*cs] += d;
  d = k[10];
  J[IDX_H2j*rs + IDX_H2j*cs] -= d;
  J[IDX_H*rs + IDX_H2j*cs] += d;
  J[IDX_Hj*rs + IDX_H2j*cs] += d;
  d = k[11]*n[IDX_H2j];
  J[IDX_H2j*rs + IDX_H*cs] -= d;
  J[IDX_H*rs + IDX_H*cs] -= d;
  J[IDX_H2*rs + IDX_H*cs] += d;
  J[IDX_Hj*rs + IDX_H*cs] += d;
  d = k[11]*n[IDX_H];
  J[IDX_H2j*rs + IDX_H2j*cs] -= d;
  J[IDX_H*rs + IDX_H2j*cs] -= d;
  J[IDX_H2*rs + IDX_H2j*cs] += d;
  J[IDX_Hj*rs + IDX_H2j*cs] += d;
  d = k[12]*n[IDX_E];
  J[IDX_H2j*rs + IDX_H2j*cs] -= d;
  J[IDX_E*rs + IDX_H2j*cs] -= d;
  J[IDX_H*rs + IDX_H2j*cs] += d;
  J[IDX_H*rs + IDX_H2j*cs] += d;
  d = k[12]*n[IDX_H2j];
  J[IDX_H2j*rs + IDX_E*cs] -= d;
  J[IDX_E*rs + IDX_E*cs] -= d;
  J[IDX_H*rs + IDX_E*cs] += d;
  J[IDX_H*rs + IDX_E*cs] += d;
  d = k[13];
  J[IDX_H2j*rs + IDX_H2j*cs] -= d;
  J[IDX_Hj*rs + IDX_H2j*cs] += d;
  J[IDX_Hj*rs + IDX_H2j*cs] += d;
  J[IDX_E*rs + IDX_H2j*cs] += d;
  d = k[14]*n[IDX_H2j];
  J[IDX_H2j*rs + IDX_H2*cs] -= d;
  J[IDX_H2*rs + IDX_H2*cs] -= d;
  J[IDX_H3j*rs + IDX_H2*cs] += d;
  J[IDX_H*rs + IDX_H2*cs] += d;
  d = k[14]*n[IDX_H2];
  J[IDX_H2j*rs + IDX_H2j*cs] -= d;
  J[IDX_H2*rs + IDX_H2j*cs] -= d;
  J[IDX_H3j*rs + IDX_H2j*cs] += d;
  J[IDX_H*rs + IDX_H2j*cs] += d;
  d = k[15]*n[IDX_H2];
  J[IDX_H2*rs + IDX_Hj*cs] -= d;
  J[IDX_Hj*rs + IDX_Hj*cs] -= d;
  J[IDX_H2j*rs + IDX_Hj*cs] += d;
  J[IDX_H*rs + IDX_Hj*cs] += d;
  d = k[15]*n[IDX_Hj];
  J[IDX_H2*rs + IDX_H2*cs] -= d;
  J[IDX_Hj*rs + IDX_H2*cs] -= d;
  J[IDX_H2j*rs + IDX_H2*cs] += d;
  J[IDX_H*rs + IDX_H2*cs] += d;
  d = k[16]*n[IDX_H2];
  J[IDX_H2*rs + IDX_Hj*cs] -= d;
  J[IDX_Hj*rs + IDX_Hj*cs] -= d;
  J[IDX_H2j*rs + IDX_Hj*cs] += d;
  J[IDX_H*rs + IDX_Hj*cs] += d;
  d = k[16]*n[IDX_Hj];
  J[IDX_H2*rs + IDX_H2*cs] -= d;
  J[IDX_Hj*rs + IDX_H2*cs] -= d;
  J[IDX_H2j*rs + IDX_H2*cs] += d;
  J[IDX_H*rs + IDX_H2*cs] += d;
  d = k[17]*n[IDX_E];
  J[IDX_H2*rs + IDX_H2*cs] -= d;
  J[IDX_E*rs + IDX_H2*cs] -= d;
  J[IDX_H*rs + IDX_H2*cs] += d;
  J[IDX_Hk*rs + IDX_H2*cs] += d;
  d = k[17]*n[IDX_H2];
  J[IDX_H2*rs + IDX_E*cs] -= d;
  J[IDX_E*rs + IDX_E*cs] -= d;
  J[IDX_H*rs + IDX_E*cs] += d;
  J[IDX_Hk*rs + IDX_E*cs] += d;
  d = k[18]*n[IDX_E];
  J[IDX_H2*rs + IDX_H2*cs] -= d;
  J[IDX_E*rs + IDX_H2*cs] -= d;
  J[IDX_H*rs + IDX_H2*cs] += d;
  J[IDX_H*rs + IDX_H2*cs] += d;
  J[IDX_E*rs + IDX_H2*cs] += d;
  d = k[18]*n[IDX_H2];
  J[IDX_H2*rs + IDX_E*cs] -= d;
  J[IDX_E*rs + IDX_E*cs] -= d;
  J[IDX_H*rs + IDX_E*cs] += d;
  J[IDX_H*rs + IDX_E*cs] += d;
  J[IDX_E*rs + IDX_E*cs] += d;
  d = k[19];
  J[IDX_H2*rs + IDX_H2*cs] -= d;
  J[IDX_H2j*rs + IDX_H2*cs] += d;
  J[IDX_E*rs + IDX_H2*cs] += d;
  d = k[20]*n[IDX_H3j];
  J[IDX_H3j*rs + IDX_H*cs] -= d;
  J[IDX_H*rs + IDX_H*cs] -= d;
  J[IDX_H2j*rs + IDX_H*cs] += d;
  J[IDX_H2*rs + IDX_H*cs] += d;
  d = k[20]*n[IDX_H];
  J[IDX_H3j*rs + IDX_H3j*cs] -= d;
  J[IDX_H*rs + IDX_H3j*cs] -= d;
  J[IDX_H2j*rs + IDX_H3j*cs] += d;
  J[IDX_H2*rs + IDX_H3j*cs] += d;
  d = k[21]*n[IDX_E];
  J[IDX_H3j*rs + IDX_H3j*cs] -= d;
  J[IDX_E*rs + IDX_H3j*cs] -= d;
  J[IDX_H2*rs + IDX_H3j*cs] += d;
  J[IDX_H*rs + IDX_H3j*cs] += d;
  d = k[21]*n[IDX_H3j];
  J[IDX_H3j*rs + IDX_E*cs] -= d;
  J[IDX_E*rs + IDX_E*cs] -= d;
  J[IDX_H2*rs + IDX_E*cs] += d;
  J[IDX_H*rs + IDX_E*cs] += d;
  d = k[22]*n[IDX_H2];
  J[IDX_H2*rs + IDX_Hj*cs] -= d;
  J[IDX_Hj*rs + IDX_Hj*cs] -= d;
  J[IDX_H3j*rs + IDX_Hj*cs] += d;
  d = k[22]*n[IDX_Hj];
  J[IDX_H2*rs + IDX_H2*cs] -= d;
  J[IDX_Hj*rs + IDX_H2*cs] -= d;
  J[IDX_H3j*rs + IDX_H2*cs] += d;
  d = k[23]*n[IDX_E];
  J[IDX_Hejj*rs + IDX_Hejj*cs] -= d;
  J[IDX_E*rs + IDX_Hejj*cs] -= d;
  J[IDX_Hej*rs + IDX_Hejj*cs] += d;
  d = k[23]*n[IDX_Hejj];
  J[IDX_Hejj*rs + IDX_E*cs] -= d;
  J[IDX_E*rs + IDX_E*cs] -= d;
  J[IDX_Hej*rs + IDX_E*cs] += d;
  d = k[24];
  J[IDX_Hej*rs + IDX_Hej*cs] -= d;
  J[IDX_Hejj*rs + IDX_Hej*cs] += d;
  J[IDX_E*rs + IDX_Hej*cs] += d;
  d = k[25]*n[IDX_E];
  J[IDX_Hej*rs + IDX_Hej*cs] -= d;
  J[IDX_E*rs + IDX_Hej*cs] -= d;
  J[IDX_He*rs + IDX_Hej*cs] += d;
  d = k[25]*n[IDX_Hej];
  J[IDX_Hej*rs + IDX_E*cs] -= d;
  J[IDX_E*rs + IDX_E*cs] -= d;
  J[IDX_He*rs + IDX_E*cs] += d;
  d = k[26];
  J[IDX_He*rs + IDX_He*cs] -= d;
  J[IDX_Hej*rs + IDX_He*cs] += d;
  J[IDX_E*rs + IDX_He*cs] += d;
  d = k[27]*n[IDX_He];
  J[IDX_He*rs + IDX_Hj*cs] -= d;
  J[IDX_Hj*rs + IDX_Hj*cs] -= d;
  J[IDX_Hej*rs + IDX_Hj*cs] += d;
  J[IDX_H*rs + IDX_Hj*cs] += d;
  d = k[27]*n[IDX_Hj];
  J[IDX_He*rs + IDX_He*cs] -= d;
  J[IDX_Hj*rs + IDX_He*cs] -= d;
  J[IDX_Hej*rs + IDX_He*cs] += d;
  J[IDX_H*rs + IDX_He*cs] += d;
  d = k[28]*n[IDX_Hej];
  J[IDX_Hej*rs + IDX_H*cs] -= d;
  J[IDX_H*rs + IDX_H*cs] -= d;
  J[IDX_He*rs + IDX_H*cs] += d;
  J[IDX_Hj*rs + IDX_H*cs] += d;
  d = k[28]*n[IDX_H];
  J[IDX_Hej*rs + IDX_Hej*cs] -= d;
  J[IDX_H*rs + IDX_Hej*cs] -= d;
  J[IDX_He*rs + IDX_Hej*cs] += d;
  J[IDX_Hj*rs + IDX_Hej*cs] += d;
  d = k[29]*n[IDX_He];
  J[IDX_He*rs + IDX_Hj*cs] -= d;
  J[IDX_Hj*rs + IDX_Hj*cs] -= d;
  J[IDX_HeHj*rs + IDX_Hj*cs] += d;
  d = k[29]*n[IDX_Hj];
  J[IDX_He*rs + IDX_He*cs] -= d;
  J[IDX_Hj*rs + IDX_He*cs] -= d;
  J[IDX_HeHj*rs + IDX_He*cs] += d;
  d = k[30]*n[IDX_He];
  J[IDX_He*rs + IDX_Hj*cs] -= d;
  J[IDX_Hj*rs + IDX_Hj*cs] -= d;
  J[IDX_HeHj*rs + IDX_Hj*cs] += d;
  d = k[30]*n[IDX_Hj];
  J[IDX_He*rs + IDX_He*cs] -= d;
  J[IDX_Hj*rs + IDX_He*cs] -= d;
  J[IDX_HeHj*rs + IDX_He*cs] += d;
  d = k[31]*n[IDX_He];
  J[IDX_He*rs + IDX_H2j*cs] -= d;
  J[IDX_H2j*rs + IDX_H2j*cs] -= d;
  J[IDX_HeHj*rs + IDX_H2j*cs] += d;
  J[IDX_H*rs + IDX_H2j*cs] += d;
  d = k[31]*n[IDX_H2j];
  J[IDX_He*rs + IDX_He*cs] -= d;
  J[IDX_H2j*rs + IDX_He*cs] -= d;
  J[IDX_HeHj*rs + IDX_He*cs] += d;
  J[IDX_H*rs + IDX_He*cs] += d;
  d = k[32]*n[IDX_Hej];
  J[IDX_Hej*rs + IDX_H*cs] -= d;
  J[IDX_H*rs + IDX_H*cs] -= d;
  J[IDX_HeHj*rs + IDX_H*cs] += d;
  d = k[32]*n[IDX_H];
  J[IDX_Hej*rs + IDX_Hej*cs] -= d;
  J[IDX_H*rs + IDX_Hej*cs] -= d;
  J[IDX_HeHj*rs + IDX_Hej*cs] += d;
  d = k[33]*n[IDX_Hej];
  J[IDX_Hej*rs + IDX_H*cs] -= d;
  J[IDX_H*rs + IDX_H*cs] -= d;
  J[IDX_HeHj*rs + IDX_H*cs] += d;
  d = k[33]*n[IDX_H];
  J[IDX_Hej*rs + IDX_Hej*cs] -= d;
  J[IDX_H*rs + IDX_Hej*cs] -= d;
  J[IDX_HeHj*rs + IDX_Hej*cs] += d;
  d = k[34]*n[IDX_HeHj];
  J[IDX_HeHj*rs + IDX_H*cs] -= d;
  J[IDX_H*rs + IDX_H*cs] -= d;
  J[IDX_He*rs + IDX_H*cs] += d;
  J[IDX_H2j*rs + IDX_H*cs] += d;
  d = k[34]*n[IDX_H];
  J[IDX_HeHj*rs + IDX_HeHj*cs] -= d;
  J[IDX_H*rs + IDX_HeHj*cs] -= d;
  J[IDX_He*rs + IDX_HeHj*cs] += d;
  J[IDX_H2j*rs + IDX_HeHj*cs] += d;
  d = k[35]*n[IDX_E];
  J[IDX_HeHj*rs + IDX_HeHj*cs] -= d;
  J[IDX_E*rs + IDX_HeHj*cs] -= d;
  J[IDX_He*rs + IDX_HeHj*cs] += d;
  J[IDX_H*rs + IDX_HeHj*cs] += d;
  d = k[35]*n[IDX_HeHj];
  J[IDX_HeHj*rs + IDX_E*cs] -= d;
  J[IDX_E*rs + IDX_E*cs] -= d;
  J[IDX_He*rs + IDX_E*cs] += d;
  J[IDX_H*rs + IDX_E*cs] += d;
  d = k[36]*n[IDX_HeHj];
  J[IDX_HeHj*rs + IDX_H2*cs] -= d;
  J[IDX_H2*rs + IDX_H2*cs] -= d;
  J[IDX_H3j*rs + IDX_H2*cs] += d;
  J[IDX_He*rs + IDX_H2*cs] += d;
  d = k[36]*n[IDX_H2];
  J[IDX_HeHj*rs + IDX_HeHj*cs] -= d;
  J[IDX_H2*rs + IDX_HeHj*cs] -= d;
  J[IDX_H3j*rs + IDX_HeHj*cs] += d;
  J[IDX_He*rs + IDX_HeHj*cs] += d;
  d = k[37];
  J[IDX_HeHj*rs + IDX_HeHj*cs] -= d;
  J[IDX_He*rs + IDX_HeHj*cs] += d;
  J[IDX_Hj*rs + IDX_HeHj*cs] += d;
  d = k[38];
  J[IDX_HeHj*rs + IDX_HeHj*cs] -= d;
  J[IDX_Hej*rs + IDX_HeHj*cs] += d;
  J[IDX_H*rs + IDX_HeHj*cs] += d;
  d = k[39]*n[IDX_E];
  J[IDX_Dj*rs + IDX_Dj*cs] -= d;
  J[IDX_E*rs + IDX_Dj*cs] -= d;
  J[IDX_D*rs + IDX_Dj*cs] += d;
  d = k[39]*n[IDX_Dj];
  J[IDX_Dj*rs + IDX_E*cs] -= d;
  J[IDX_E*rs + IDX_E*cs] -= d;
  J[IDX_D*rs + IDX_E*cs] += d;
  d = k[40];
  J[IDX_D*rs + IDX_D*cs] -= d;
  J[IDX_Dj*rs + IDX_D*cs] += d;
  J[IDX_E*rs + IDX_D*cs] += d;
  d = k[41]*n[IDX_Hj];
  J[IDX_D*rs + IDX_D*cs] -= d;
  J[IDX_Hj*rs + IDX_D*cs] -= d;
  J[IDX_Dj*rs + IDX_D*cs] += d;
  J[IDX_H*rs + IDX_D*cs] += d;
  d = k[41]*n[IDX_D];
  J[IDX_D*rs + IDX_Hj*cs] -= d;
  J[IDX_Hj*rs + IDX_Hj*cs] -= d;
  J[IDX_Dj*rs + IDX_Hj*cs] += d;
  J[IDX_H*rs + IDX_Hj*cs] += d;
  d = k[42]*n[IDX_H];
  J[IDX_Dj*rs + IDX_Dj*cs] -= d;
  J[IDX_H*rs + IDX_Dj*cs] -= d;
  J[IDX_D*rs + IDX_Dj*cs] += d;
  J[IDX_Hj*rs + IDX_Dj*cs] += d;
  d = k[42]*n[IDX_Dj];
  J[IDX_Dj*rs + IDX_H*cs] -= d;
  J[IDX_H*rs + IDX_H*cs] -= d;
  J[IDX_D*rs + IDX_H*cs] += d;
  J[IDX_Hj*rs + IDX_H*cs] += d;
  d = k[43]*n[IDX_H];
  J[IDX_D*rs + IDX_D*cs] -= d;
  J[IDX_H*rs + IDX_D*cs] -= d;
  J[IDX_HD*rs + IDX_D*cs] += d;
  d = k[43]*n[IDX_D];
  J[IDX_D*rs + IDX_H*cs] -= d;
  J[IDX_H*rs + IDX_H*cs] -= d;
  J[IDX_HD*rs + IDX_H*cs] += d;
  d = k[44]*n[IDX_H2];
  J[IDX_D*rs + IDX_D*cs] -= d;
  J[IDX_H2*rs + IDX_D*cs] -= d;
  J[IDX_H*rs + IDX_D*cs] += d;
  J[IDX_HD*rs + IDX_D*cs] += d;
  d = k[44]*n[IDX_D];
  J[IDX_D*rs + IDX_H2*cs] -= d;
  J[IDX_H2*rs + IDX_H2*cs] -= d;
  J[IDX_H*rs + IDX_H2*cs] += d;
  J[IDX_HD*rs + IDX_H2*cs] += d;
  d = k[45]*n[IDX_HDj];
  J[IDX_HDj*rs + IDX_H*cs] -= d;
  J[IDX_H*rs + IDX_H*cs] -= d;
  J[IDX_Hj*rs + IDX_H*cs] += d;
  J[IDX_HD*rs + IDX_H*cs] += d;
  d = k[45]*n[IDX_H];
  J[IDX_HDj*rs + IDX_HDj*cs] -= d;
  J[IDX_H*rs + IDX_HDj*cs] -= d;
  J[IDX_Hj*rs + IDX_HDj*cs] += d;
  J[IDX_HD*rs + IDX_HDj*cs] += d;
  d = k[46]*n[IDX_H2];
  J[IDX_Dj*rs + IDX_Dj*cs] -= d;
  J[IDX_H2*rs + IDX_Dj*cs] -= d;
  J[IDX_Hj*rs + IDX_Dj*cs] += d;
  J[IDX_HD*rs + IDX_Dj*cs] += d;
  d = k[46]*n[IDX_Dj];
  J[IDX_Dj*rs + IDX_H2*cs] -= d;
  J[IDX_H2*rs + IDX_H2*cs] -= d;
  J[IDX_Hj*rs + IDX_H2*cs] += d;
  J[IDX_HD*rs + IDX_H2*cs] += d;
  d = k[47]*n[IDX_HD];
  J[IDX_HD*rs + IDX_H*cs] -= d;
  J[IDX_H*rs + IDX_H*cs] -= d;
  J[IDX_H2*rs + IDX_H*cs] += d;
  J[IDX_D*rs + IDX_H*cs] += d;
  d = k[47]*n[IDX_H];
  J[IDX_HD*rs + IDX_HD*cs] -= d;
  J[IDX_H*rs + IDX_HD*cs] -= d;
  J[IDX_H2*rs + IDX_HD*cs] += d;
  J[IDX_D*rs + IDX_HD*cs] += d;
  d = k[48]*n[IDX_HD];
  J[IDX_HD*rs + IDX_Hj*cs] -= d;
  J[IDX_Hj*rs + IDX_Hj*cs] -= d;
  J[IDX_H2*rs + IDX_Hj*cs] += d;
  J[IDX_Dj*rs + IDX_Hj*cs] += d;
  d = k[48]*n[IDX_Hj];
  J[IDX_HD*rs + IDX_HD*cs] -= d;
  J[IDX_Hj*rs + IDX_HD*cs] -= d;
  J[IDX_H2*rs + IDX_HD*cs] += d;
  J[IDX_Dj*rs + IDX_HD*cs] += d;
  d = k[49]*n[IDX_HD];
  J[IDX_HD*rs + IDX_H3j*cs] -= d;
  J[IDX_H3j*rs + IDX_H3j*cs] -= d;
  J[IDX_H2*rs + IDX_H3j*cs] += d;
  J[IDX_H2Dj*rs + IDX_H3j*cs] += d;
  d = k[49]*n[IDX_H3j];
  J[IDX_HD*rs + IDX_HD*cs] -= d;
  J[IDX_H3j*rs + IDX_HD*cs] -= d;
  J[IDX_H2*rs + IDX_HD*cs] += d;
  J[IDX_H2Dj*rs + IDX_HD*cs] += d;
  d = k[50]*n[IDX_Hj];
  J[IDX_D*rs + IDX_D*cs] -= d;
  J[IDX_Hj*rs + IDX_D*cs] -= d;
  J[IDX_HDj*rs + IDX_D*cs] += d;
  d = k[50]*n[IDX_D];
  J[IDX_D*rs + IDX_Hj*cs] -= d;
  J[IDX_Hj*rs + IDX_Hj*cs] -= d;
  J[IDX_HDj*rs + IDX_Hj*cs] += d;
  d = k[51]*n[IDX_H];
  J[IDX_Dj*rs + IDX_Dj*cs] -= d;
  J[IDX_H*rs + IDX_Dj*cs] -= d;
  J[IDX_HDj*rs + IDX_Dj*cs] += d;
  d = k[51]*n[IDX_Dj];
  J[IDX_Dj*rs + IDX_H*cs] -= d;
  J[IDX_H*rs + IDX_H*cs] -= d;
  J[IDX_HDj*rs + IDX_H*cs] += d;
  d = k[52];
  J[IDX_HDj*rs + IDX_HDj*cs] -= d;
  J[IDX_H*rs + IDX_HDj*cs] += d;
  J[IDX_Dj*rs + IDX_HDj*cs] += d;
  d = k[53];
  J[IDX_HDj*rs + IDX_HDj*cs] -= d;
  J[IDX_Hj*rs + IDX_HDj*cs] += d;
  J[IDX_D*rs + IDX_HDj*cs] += d;
  d = k[54]*n[IDX_E];
  J[IDX_HDj*rs + IDX_HDj*cs] -= d;
  J[IDX_E*rs + IDX_HDj*cs] -= d;
  J[IDX_H*rs + IDX_HDj*cs] += d;
  J[IDX_D*rs + IDX_HDj*cs] += d;
  d = k[54]*n[IDX_HDj];
  J[IDX_HDj*rs + IDX_E*cs] -= d;
  J[IDX_E*rs + IDX_E*cs] -= d;
  J[IDX_H*rs + IDX_E*cs] += d;
  J[IDX_D*rs + IDX_E*cs] += d;
  d = k[55]*n[IDX_HDj];
  J[IDX_HDj*rs + IDX_H2*cs] -= d;
  J[IDX_H2*rs + IDX_H2*cs] -= d;
  J[IDX_H2Dj*rs + IDX_H2*cs] += d;
  J[IDX_H*rs + IDX_H2*cs] += d;
  d = k[55]*n[IDX_H2];
  J[IDX_HDj*rs + IDX_HDj*cs] -= d;
  J[IDX_H2*rs + IDX_HDj*cs] -= d;
  J[IDX_H2Dj*rs + IDX_HDj*cs] += d;
  J[IDX_H*rs + IDX_HDj*cs] += d;
  d = k[56]*n[IDX_HDj];
  J[IDX_HDj*rs + IDX_H2*cs] -= d;
  J[IDX_H2*rs + IDX_H2*cs] -= d;
  J[IDX_H3j*rs + IDX_H2*cs] += d;
  J[IDX_D*rs + IDX_H2*cs] += d;
  d = k[56]*n[IDX_H2];
  J[IDX_HDj*rs + IDX_HDj*cs] -= d;
  J[IDX_H2*rs + IDX_HDj*cs] -= d;
  J[IDX_H3j*rs + IDX_HDj*cs] += d;
  J[IDX_D*rs + IDX_HDj*cs] += d;
  d = k[57]*n[IDX_H3j];
  J[IDX_D*rs + IDX_D*cs] -= d;
  J[IDX_H3j*rs + IDX_D*cs] -= d;
  J[IDX_H2Dj*rs + IDX_D*cs] += d;
  J[IDX_H*rs + IDX_D*cs] += d;
  d = k[57]*n[IDX_D];
  J[IDX_D*rs + IDX_H3j*cs] -= d;
  J[IDX_H3j*rs + IDX_H3j*cs] -= d;
  J[IDX_H2Dj*rs + IDX_H3j*cs] += d;
  J[IDX_H*rs + IDX_H3j*cs] += d;
  d = k[58]*n[IDX_E];
  J[IDX_H2Dj*rs + IDX_H2Dj*cs] -= d;
  J[IDX_E*rs + IDX_H2Dj*cs] -= d;
  J[IDX_H*rs + IDX_H2Dj*cs] += d;
  J[IDX_H*rs + IDX_H2Dj*cs] += d;
  J[IDX_D*rs + IDX_H2Dj*cs] += d;
  d = k[58]*n[IDX_H2Dj];
  J[IDX_H2Dj*rs + IDX_E*cs] -= d;
  J[IDX_E*rs + IDX_E*cs] -= d;
  J[IDX_H*rs + IDX_E*cs] += d;
  J[IDX_H*rs + IDX_E*cs] += d;
  J[IDX_D*rs + IDX_E*cs] += d;
  d = k[59]*n[IDX_E];
  J[IDX_H2Dj*rs + IDX_H2Dj*cs] -= d;
  J[IDX_E*rs + IDX_H2Dj*cs] -= d;
  J[IDX_H2*rs + IDX_H2Dj*cs] += d;
  J[IDX_D*rs + IDX_H2Dj*cs] += d;
  d = k[59]*n[IDX_H2Dj];
  J[IDX_H2Dj*rs + IDX_E*cs] -= d;
  J[IDX_E*rs + IDX_E*cs] -= d;
  J[IDX_H2*rs + IDX_E*cs] += d;
  J[IDX_D*rs + IDX_E*cs] += d;
  d = k[60]*n[IDX_E];
  J[IDX_H2Dj*rs + IDX_H2Dj*cs] -= d;
  J[IDX_E*rs + IDX_H2Dj*cs] -= d;
  J[IDX_HD*rs + IDX_H2Dj*cs] += d;
  J[IDX_H*rs + IDX_H2Dj*cs] += d;
  d = k[60]*n[IDX_H2Dj];
  J[IDX_H2Dj*rs + IDX_E*cs] -= d;
  J[IDX_E*rs + IDX_E*cs] -= d;
  J[IDX_HD*rs + IDX_E*cs] += d;
  J[IDX_H*rs + IDX_E*cs] += d;
  d = k[61]*n[IDX_H2Dj];
  J[IDX_H2Dj*rs + IDX_H2*cs] -= d;
  J[IDX_H2*rs + IDX_H2*cs] -= d;
  J[IDX_H3j*rs + IDX_H2*cs] += d;
  J[IDX_HD*rs + IDX_H2*cs] += d;
  d = k[61]*n[IDX_H2];
  J[IDX_H2Dj*rs + IDX_H2Dj*cs] -= d;
  J[IDX_H2*rs + IDX_H2Dj*cs] -= d;
  J[IDX_H3j*rs + IDX_H2Dj*cs] += d;
  J[IDX_HD*rs + IDX_H2Dj*cs] += d;
  d = k[62]*n[IDX_H2Dj];
  J[IDX_H2Dj*rs + IDX_H2*cs] -= d;
  J[IDX_H2*rs + IDX_H2*cs] -= d;
  J[IDX_H3j*rs + IDX_H2*cs] += d;
  J[IDX_HD*rs + IDX_H2*cs] += d;
  d = k[62]*n[IDX_H2];
  J[IDX_H2Dj*rs + IDX_H2Dj*cs] -= d;
  J[IDX_H2*rs + IDX_H2Dj*cs] -= d;
  J[IDX_H3j*rs + IDX_H2Dj*cs] += d;
  J[IDX_HD*rs + IDX_H2Dj*cs] += d;
  d = k[63]*n[IDX_H2Dj];
  J[IDX_H2Dj*rs + IDX_H*cs] -= d;
  J[IDX_H*rs + IDX_H*cs] -= d;
  J[IDX_H3j*rs + IDX_H*cs] += d;
  J[IDX_D*rs + IDX_H*cs] += d;
  d = k[63]*n[IDX_H];
  J[IDX_H2Dj*rs + IDX_H2Dj*cs] -= d;
  J[IDX_H*rs + IDX_H2Dj*cs] -= d;
  J[IDX_H3j*rs + IDX_H2Dj*cs] += d;
  J[IDX_D*rs + IDX_H2Dj*cs] += d;
}

// H+ + e- -> H
KB_HD inline double rate_0(double Tgas, const double* n, const Params& p, double Tg_) {
  (void)Tgas; (void)n; (void)p; (void)Tg_;
  return recfast_H_rec(n[IDX_H], Tgas, n, p);
}
// H -> H+ + e-
KB_HD inline double rate_1(double Tgas, const double* n, const Params& p, double Tg_) {
  (void)Tgas; (void)n; (void)p; (void)Tg_;
  return recfast_H_ion(n[IDX_H], Tgas, n, p);
}
// He+ + e- -> He
KB_HD inline double rate_25(double Tgas, const double* n, const Params& p, double Tg_) {
  (void)Tgas; (void)n; (void)p; (void)Tg_;
  return recfast_He_rec(n[IDX_He], n[IDX_H], Tgas, n, p);
}
// He -> He+ + e-
KB_HD inline double rate_26(double Tgas, const double* n, const Params& p, double Tg_) {
  (void)Tgas; (void)n; (void)p; (void)Tg_;
  return recfast_He_ion(n[IDX_He], n[IDX_H], Tgas, n, p);
}
// D+ + e- -> D
KB_HD inline double rate_39(double Tgas, const double* n, const Params& p, double Tg_) {
  (void)Tgas; (void)n; (void)p; (void)Tg_;
  return recfast_H_rec(n[IDX_D], Tgas, n, p);
}
// D -> D+ + e-
KB_HD inline double rate_40(double Tgas, const double* n, const Params& p, double Tg_) {
  (void)Tgas; (void)n; (void)p; (void)Tg_;
  return recfast_H_ion(n[IDX_D], Tgas, n, p);
}
// the rate-derivative part of the analytic Jacobian (J[i*jrs_ + j*cs], added to;
// U[NSPEC][NAGG] written), gated and clamped like the rates
KB_HD inline void jac_dk(double Tgas, const double* n, const Params& p, const double* k, double* J, double* U, long jrs_, long jcs_) {
  (void)Tgas; (void)n; (void)p; (void)k; (void)J; (void)jrs_; (void)jcs_;
  for (int i = 0; i < NSPEC * NAGG; ++i) U[i] = 0.0;
  double d;
  (void)d;
  { // numerical dk/dn: H+ + e- -> H (extern/table in rate, all species)
    double np_[NSPEC];
    for (int q = 0; q < NSPEC; ++q) np_[q] = n[q];
    auto rf_ = [&](const double* x) { return rate_0(Tgas, x, p, Tgas); };
    const double pr_ = n[IDX_Hj]*n[IDX_E];
    for (int jj = 0; jj < NSPEC; ++jj) {
      const double dk_ = fd_dk_(rf_, np_, n, k[0], jj);
      if (dk_ == 0.0) continue;
      d = dk_ * pr_;
      J[IDX_Hj*jrs_ + jj*jcs_] -= d;
      J[IDX_E*jrs_ + jj*jcs_] -= d;
      J[IDX_H*jrs_ + jj*jcs_] += d;
    }
  }
  { // numerical dk/dn: H -> H+ + e- (extern/table in rate, all species)
    double np_[NSPEC];
    for (int q = 0; q < NSPEC; ++q) np_[q] = n[q];
    auto rf_ = [&](const double* x) { return rate_1(Tgas, x, p, Tgas); };
    const double pr_ = n[IDX_H];
    for (int jj = 0; jj < NSPEC; ++jj) {
      const double dk_ = fd_dk_(rf_, np_, n, k[1], jj);
      if (dk_ == 0.0) continue;
      d = dk_ * pr_;
      J[IDX_H*jrs_ + jj*jcs_] -= d;
      J[IDX_Hj*jrs_ + jj*jcs_] += d;
      J[IDX_E*jrs_ + jj*jcs_] += d;
    }
  }
  { // numerical dk/dn: He+ + e- -> He (extern/table in rate, all species)
    double np_[NSPEC];
    for (int q = 0; q < NSPEC; ++q) np_[q] = n[q];
    auto rf_ = [&](const double* x) { return rate_25(Tgas, x, p, Tgas); };
    const double pr_ = n[IDX_Hej]*n[IDX_E];
    for (int jj = 0; jj < NSPEC; ++jj) {
      const double dk_ = fd_dk_(rf_, np_, n, k[25], jj);
      if (dk_ == 0.0) continue;
      d = dk_ * pr_;
      J[IDX_Hej*jrs_ + jj*jcs_] -= d;
      J[IDX_E*jrs_ + jj*jcs_] -= d;
      J[IDX_He*jrs_ + jj*jcs_] += d;
    }
  }
  { // numerical dk/dn: He -> He+ + e- (extern/table in rate, all species)
    double np_[NSPEC];
    for (int q = 0; q < NSPEC; ++q) np_[q] = n[q];
    auto rf_ = [&](const double* x) { return rate_26(Tgas, x, p, Tgas); };
    const double pr_ = n[IDX_He];
    for (int jj = 0; jj < NSPEC; ++jj) {
      const double dk_ = fd_dk_(rf_, np_, n, k[26], jj);
      if (dk_ == 0.0) continue;
      d = dk_ * pr_;
      J[IDX_He*jrs_ + jj*jcs_] -= d;
      J[IDX_Hej*jrs_ + jj*jcs_] += d;
      J[IDX_E*jrs_ + jj*jcs_] += d;
    }
  }
  { // numerical dk/dn: D+ + e- -> D (extern/table in rate, all species)
    double np_[NSPEC];
    for (int q = 0; q < NSPEC; ++q) np_[q] = n[q];
    auto rf_ = [&](const double* x) { return rate_39(Tgas, x, p, Tgas); };
    const double pr_ = n[IDX_Dj]*n[IDX_E];
    for (int jj = 0; jj < NSPEC; ++jj) {
      const double dk_ = fd_dk_(rf_, np_, n, k[39], jj);
      if (dk_ == 0.0) continue;
      d = dk_ * pr_;
      J[IDX_Dj*jrs_ + jj*jcs_] -= d;
      J[IDX_E*jrs_ + jj*jcs_] -= d;
      J[IDX_D*jrs_ + jj*jcs_] += d;
    }
  }
  { // numerical dk/dn: D -> D+ + e- (extern/table in rate, all species)
    double np_[NSPEC];
    for (int q = 0; q < NSPEC; ++q) np_[q] = n[q];
    auto rf_ = [&](const double* x) { return rate_40(Tgas, x, p, Tgas); };
    const double pr_ = n[IDX_D];
    for (int jj = 0; jj < NSPEC; ++jj) {
      const double dk_ = fd_dk_(rf_, np_, n, k[40], jj);
      if (dk_ == 0.0) continue;
      d = dk_ * pr_;
      J[IDX_D*jrs_ + jj*jcs_] -= d;
      J[IDX_Dj*jrs_ + jj*jcs_] += d;
      J[IDX_E*jrs_ + jj*jcs_] += d;
    }
  }
  {  // group 1: H- + H -> H2 + e-
    double T = Tgas;
    if (T < 300.0) {
    }
    else if (T >= 300.0) {
    }
  }
  {  // group 2: H- + H+ -> H2+ + e-
    double T = Tgas;
    if (T < 8000.0) {
    }
    else if (T >= 8000.0) {
    }
  }
  {  // group 3: H2 + H+ -> H2+ + H
    double T = Tgas;
    if (T < 10000.0) {
    }
    else if (T >= 10000.0) {
    }
  }
  {  // group 4: He + H+ -> He+ + H
    double T = Tgas;
    if (T >= 10000.0 && T >= 10000.0) {
    }
  }
  {  // group 5: He+ + H -> He + H+
    double T = Tgas;
    if (T >= 6000.0 && T >= 6000.0) {
    }
  }
  {  // group 6: He + H+ -> HeH+
    double T = Tgas;
    if (T < 1000.0) {
    }
    else if (T >= 1000.0) {
    }
  }
  {  // group 7: He+ + H -> HeH+
    double T = Tgas;
    if (T < 4000.0) {
    }
    else if (T >= 4000.0) {
    }
  }
  {  // group 8: D + H2 -> H + HD
    double T = Tgas;
    if (T >= 250.0 && T >= 250.0) {
    }
  }
  {  // group 9: HD + H -> H2 + D
    double T = Tgas;
    if (T >= 200.0 && T >= 200.0) {
    }
  }
  {  // group 10: H2D+ + H2 -> H3+ + HD
    double T = Tgas;
    if (T < 100.0) {
    }
    else if (T >= 100.0) {
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
  flux = k[0]*n[IDX_Hj]*n[IDX_E];
  g[0] += flux * (mu[IDX_H] - mu[IDX_Hj] - mu[IDX_E]);
  flux = k[1]*n[IDX_H];
  g[1] += flux * (mu[IDX_Hj] + mu[IDX_E] - mu[IDX_H]);
  flux = k[2]*n[IDX_H]*n[IDX_E];
  g[2] += flux * (mu[IDX_Hk] - mu[IDX_H] - mu[IDX_E]);
  flux = k[3]*n[IDX_Hk];
  g[3] += flux * (mu[IDX_H] + mu[IDX_E] - mu[IDX_Hk]);
  flux = k[4]*n[IDX_Hk]*n[IDX_H];
  g[4] += flux * (mu[IDX_H2] + mu[IDX_E] - mu[IDX_Hk] - mu[IDX_H]);
  flux = k[5]*n[IDX_Hk]*n[IDX_H];
  g[5] += flux * (mu[IDX_H2] + mu[IDX_E] - mu[IDX_Hk] - mu[IDX_H]);
  flux = k[6]*n[IDX_Hk]*n[IDX_Hj];
  g[6] += flux * (mu[IDX_H2j] + mu[IDX_E] - mu[IDX_Hk] - mu[IDX_Hj]);
  flux = k[7]*n[IDX_Hk]*n[IDX_Hj];
  g[7] += flux * (mu[IDX_H2j] + mu[IDX_E] - mu[IDX_Hk] - mu[IDX_Hj]);
  flux = k[8]*n[IDX_Hk]*n[IDX_Hj];
  g[8] += flux * (mu[IDX_H] + mu[IDX_H] - mu[IDX_Hk] - mu[IDX_Hj]);
  flux = k[9]*n[IDX_H]*n[IDX_Hj];
  g[9] += flux * (mu[IDX_H2j] - mu[IDX_H] - mu[IDX_Hj]);
  flux = k[10]*n[IDX_H2j];
  g[10] += flux * (mu[IDX_H] + mu[IDX_Hj] - mu[IDX_H2j]);
  flux = k[11]*n[IDX_H2j]*n[IDX_H];
  g[11] += flux * (mu[IDX_H2] + mu[IDX_Hj] - mu[IDX_H2j] - mu[IDX_H]);
  flux = k[12]*n[IDX_H2j]*n[IDX_E];
  g[12] += flux * (mu[IDX_H] + mu[IDX_H] - mu[IDX_H2j] - mu[IDX_E]);
  flux = k[13]*n[IDX_H2j];
  g[13] += flux * (mu[IDX_Hj] + mu[IDX_Hj] + mu[IDX_E] - mu[IDX_H2j]);
  flux = k[14]*n[IDX_H2j]*n[IDX_H2];
  g[14] += flux * (mu[IDX_H3j] + mu[IDX_H] - mu[IDX_H2j] - mu[IDX_H2]);
  flux = k[15]*n[IDX_H2]*n[IDX_Hj];
  g[15] += flux * (mu[IDX_H2j] + mu[IDX_H] - mu[IDX_H2] - mu[IDX_Hj]);
  flux = k[16]*n[IDX_H2]*n[IDX_Hj];
  g[16] += flux * (mu[IDX_H2j] + mu[IDX_H] - mu[IDX_H2] - mu[IDX_Hj]);
  flux = k[17]*n[IDX_H2]*n[IDX_E];
  g[17] += flux * (mu[IDX_H] + mu[IDX_Hk] - mu[IDX_H2] - mu[IDX_E]);
  flux = k[18]*n[IDX_H2]*n[IDX_E];
  g[18] += flux * (mu[IDX_H] + mu[IDX_H] + mu[IDX_E] - mu[IDX_H2] - mu[IDX_E]);
  flux = k[19]*n[IDX_H2];
  g[19] += flux * (mu[IDX_H2j] + mu[IDX_E] - mu[IDX_H2]);
  flux = k[20]*n[IDX_H3j]*n[IDX_H];
  g[20] += flux * (mu[IDX_H2j] + mu[IDX_H2] - mu[IDX_H3j] - mu[IDX_H]);
  flux = k[21]*n[IDX_H3j]*n[IDX_E];
  g[21] += flux * (mu[IDX_H2] + mu[IDX_H] - mu[IDX_H3j] - mu[IDX_E]);
  flux = k[22]*n[IDX_H2]*n[IDX_Hj];
  g[22] += flux * (mu[IDX_H3j] - mu[IDX_H2] - mu[IDX_Hj]);
  flux = k[23]*n[IDX_Hejj]*n[IDX_E];
  g[23] += flux * (mu[IDX_Hej] - mu[IDX_Hejj] - mu[IDX_E]);
  flux = k[24]*n[IDX_Hej];
  g[24] += flux * (mu[IDX_Hejj] + mu[IDX_E] - mu[IDX_Hej]);
  flux = k[25]*n[IDX_Hej]*n[IDX_E];
  g[25] += flux * (mu[IDX_He] - mu[IDX_Hej] - mu[IDX_E]);
  flux = k[26]*n[IDX_He];
  g[26] += flux * (mu[IDX_Hej] + mu[IDX_E] - mu[IDX_He]);
  flux = k[27]*n[IDX_He]*n[IDX_Hj];
  g[27] += flux * (mu[IDX_Hej] + mu[IDX_H] - mu[IDX_He] - mu[IDX_Hj]);
  flux = k[28]*n[IDX_Hej]*n[IDX_H];
  g[28] += flux * (mu[IDX_He] + mu[IDX_Hj] - mu[IDX_Hej] - mu[IDX_H]);
  flux = k[29]*n[IDX_He]*n[IDX_Hj];
  g[29] += flux * (mu[IDX_HeHj] - mu[IDX_He] - mu[IDX_Hj]);
  flux = k[30]*n[IDX_He]*n[IDX_Hj];
  g[30] += flux * (mu[IDX_HeHj] - mu[IDX_He] - mu[IDX_Hj]);
  flux = k[31]*n[IDX_He]*n[IDX_H2j];
  g[31] += flux * (mu[IDX_HeHj] + mu[IDX_H] - mu[IDX_He] - mu[IDX_H2j]);
  flux = k[32]*n[IDX_Hej]*n[IDX_H];
  g[32] += flux * (mu[IDX_HeHj] - mu[IDX_Hej] - mu[IDX_H]);
  flux = k[33]*n[IDX_Hej]*n[IDX_H];
  g[33] += flux * (mu[IDX_HeHj] - mu[IDX_Hej] - mu[IDX_H]);
  flux = k[34]*n[IDX_HeHj]*n[IDX_H];
  g[34] += flux * (mu[IDX_He] + mu[IDX_H2j] - mu[IDX_HeHj] - mu[IDX_H]);
  flux = k[35]*n[IDX_HeHj]*n[IDX_E];
  g[35] += flux * (mu[IDX_He] + mu[IDX_H] - mu[IDX_HeHj] - mu[IDX_E]);
  flux = k[36]*n[IDX_HeHj]*n[IDX_H2];
  g[36] += flux * (mu[IDX_H3j] + mu[IDX_He] - mu[IDX_HeHj] - mu[IDX_H2]);
  flux = k[37]*n[IDX_HeHj];
  g[37] += flux * (mu[IDX_He] + mu[IDX_Hj] - mu[IDX_HeHj]);
  flux = k[38]*n[IDX_HeHj];
  g[38] += flux * (mu[IDX_Hej] + mu[IDX_H] - mu[IDX_HeHj]);
  flux = k[39]*n[IDX_Dj]*n[IDX_E];
  g[39] += flux * (mu[IDX_D] - mu[IDX_Dj] - mu[IDX_E]);
  flux = k[40]*n[IDX_D];
  g[40] += flux * (mu[IDX_Dj] + mu[IDX_E] - mu[IDX_D]);
  flux = k[41]*n[IDX_D]*n[IDX_Hj];
  g[41] += flux * (mu[IDX_Dj] + mu[IDX_H] - mu[IDX_D] - mu[IDX_Hj]);
  flux = k[42]*n[IDX_Dj]*n[IDX_H];
  g[42] += flux * (mu[IDX_D] + mu[IDX_Hj] - mu[IDX_Dj] - mu[IDX_H]);
  flux = k[43]*n[IDX_D]*n[IDX_H];
  g[43] += flux * (mu[IDX_HD] - mu[IDX_D] - mu[IDX_H]);
  flux = k[44]*n[IDX_D]*n[IDX_H2];
  g[44] += flux * (mu[IDX_H] + mu[IDX_HD] - mu[IDX_D] - mu[IDX_H2]);
  flux = k[45]*n[IDX_HDj]*n[IDX_H];
  g[45] += flux * (mu[IDX_Hj] + mu[IDX_HD] - mu[IDX_HDj] - mu[IDX_H]);
  flux = k[46]*n[IDX_Dj]*n[IDX_H2];
  g[46] += flux * (mu[IDX_Hj] + mu[IDX_HD] - mu[IDX_Dj] - mu[IDX_H2]);
  flux = k[47]*n[IDX_HD]*n[IDX_H];
  g[47] += flux * (mu[IDX_H2] + mu[IDX_D] - mu[IDX_HD] - mu[IDX_H]);
  flux = k[48]*n[IDX_HD]*n[IDX_Hj];
  g[48] += flux * (mu[IDX_H2] + mu[IDX_Dj] - mu[IDX_HD] - mu[IDX_Hj]);
  flux = k[49]*n[IDX_HD]*n[IDX_H3j];
  g[49] += flux * (mu[IDX_H2] + mu[IDX_H2Dj] - mu[IDX_HD] - mu[IDX_H3j]);
  flux = k[50]*n[IDX_D]*n[IDX_Hj];
  g[50] += flux * (mu[IDX_HDj] - mu[IDX_D] - mu[IDX_Hj]);
  flux = k[51]*n[IDX_Dj]*n[IDX_H];
  g[51] += flux * (mu[IDX_HDj] - mu[IDX_Dj] - mu[IDX_H]);
  flux = k[52]*n[IDX_HDj];
  g[52] += flux * (mu[IDX_H] + mu[IDX_Dj] - mu[IDX_HDj]);
  flux = k[53]*n[IDX_HDj];
  g[53] += flux * (mu[IDX_Hj] + mu[IDX_D] - mu[IDX_HDj]);
  flux = k[54]*n[IDX_HDj]*n[IDX_E];
  g[54] += flux * (mu[IDX_H] + mu[IDX_D] - mu[IDX_HDj] - mu[IDX_E]);
  flux = k[55]*n[IDX_HDj]*n[IDX_H2];
  g[55] += flux * (mu[IDX_H2Dj] + mu[IDX_H] - mu[IDX_HDj] - mu[IDX_H2]);
  flux = k[56]*n[IDX_HDj]*n[IDX_H2];
  g[56] += flux * (mu[IDX_H3j] + mu[IDX_D] - mu[IDX_HDj] - mu[IDX_H2]);
  flux = k[57]*n[IDX_D]*n[IDX_H3j];
  g[57] += flux * (mu[IDX_H2Dj] + mu[IDX_H] - mu[IDX_D] - mu[IDX_H3j]);
  flux = k[58]*n[IDX_H2Dj]*n[IDX_E];
  g[58] += flux * (mu[IDX_H] + mu[IDX_H] + mu[IDX_D] - mu[IDX_H2Dj] - mu[IDX_E]);
  flux = k[59]*n[IDX_H2Dj]*n[IDX_E];
  g[59] += flux * (mu[IDX_H2] + mu[IDX_D] - mu[IDX_H2Dj] - mu[IDX_E]);
  flux = k[60]*n[IDX_H2Dj]*n[IDX_E];
  g[60] += flux * (mu[IDX_HD] + mu[IDX_H] - mu[IDX_H2Dj] - mu[IDX_E]);
  flux = k[61]*n[IDX_H2Dj]*n[IDX_H2];
  g[61] += flux * (mu[IDX_H3j] + mu[IDX_HD] - mu[IDX_H2Dj] - mu[IDX_H2]);
  flux = k[62]*n[IDX_H2Dj]*n[IDX_H2];
  g[62] += flux * (mu[IDX_H3j] + mu[IDX_HD] - mu[IDX_H2Dj] - mu[IDX_H2]);
  flux = k[63]*n[IDX_H2Dj]*n[IDX_H];
  g[63] += flux * (mu[IDX_H3j] + mu[IDX_D] - mu[IDX_H2Dj] - mu[IDX_H]);
}

// reaction labels: the equation, and the T range of a piece
inline const char* const reaction_names[64] = {"H+ + e- -> H", "H -> H+ + e-", "H + e- -> H-", "H- -> H + e-", "H- + H -> H2 + e- [0.0, 300.0]", "H- + H -> H2 + e- [300.0, INFINITY]", "H- + H+ -> H2+ + e- [0.0, 8000.0]", "H- + H+ -> H2+ + e- [8000.0, INFINITY]", "H- + H+ -> H + H", "H + H+ -> H2+", "H2+ -> H + H+", "H2+ + H -> H2 + H+", "H2+ + e- -> H + H", "H2+ -> H+ + H+ + e-", "H2+ + H2 -> H3+ + H", "H2 + H+ -> H2+ + H [0.0, 10000.0]", "H2 + H+ -> H2+ + H [10000.0, INFINITY]", "H2 + e- -> H + H-", "H2 + e- -> H + H + e-", "H2 -> H2+ + e-", "H3+ + H -> H2+ + H2", "H3+ + e- -> H2 + H", "H2 + H+ -> H3+", "He++ + e- -> He+", "He+ -> He++ + e-", "He+ + e- -> He", "He -> He+ + e-", "He + H+ -> He+ + H [10000.0, INFINITY]", "He+ + H -> He + H+ [6000.0, INFINITY]", "He + H+ -> HeH+ [0.0, 1000.0]", "He + H+ -> HeH+ [1000.0, INFINITY]", "He + H2+ -> HeH+ + H", "He+ + H -> HeH+ [0.0, 4000.0]", "He+ + H -> HeH+ [4000.0, INFINITY]", "HeH+ + H -> He + H2+", "HeH+ + e- -> He + H", "HeH+ + H2 -> H3+ + He", "HeH+ -> He + H+", "HeH+ -> He+ + H", "D+ + e- -> D", "D -> D+ + e-", "D + H+ -> D+ + H", "D+ + H -> D + H+", "D + H -> HD", "D + H2 -> H + HD [250.0, INFINITY]", "HD+ + H -> H+ + HD", "D+ + H2 -> H+ + HD", "HD + H -> H2 + D [200.0, INFINITY]", "HD + H+ -> H2 + D+", "HD + H3+ -> H2 + H2D+", "D + H+ -> HD+", "D+ + H -> HD+", "HD+ -> H + D+", "HD+ -> H+ + D", "HD+ + e- -> H + D", "HD+ + H2 -> H2D+ + H", "HD+ + H2 -> H3+ + D", "D + H3+ -> H2D+ + H", "H2D+ + e- -> H + H + D", "H2D+ + e- -> H2 + D", "H2D+ + e- -> HD + H", "H2D+ + H2 -> H3+ + HD [0.0, 100.0]", "H2D+ + H2 -> H3+ + HD [100.0, INFINITY]", "H2D+ + H -> H3+ + D"};
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
  fl[0] = k[0]*n[IDX_Hj]*n[IDX_E];
  fl[1] = k[1]*n[IDX_H];
  fl[2] = k[2]*n[IDX_H]*n[IDX_E];
  fl[3] = k[3]*n[IDX_Hk];
  fl[4] = k[4]*n[IDX_Hk]*n[IDX_H];
  fl[5] = k[5]*n[IDX_Hk]*n[IDX_H];
  fl[6] = k[6]*n[IDX_Hk]*n[IDX_Hj];
  fl[7] = k[7]*n[IDX_Hk]*n[IDX_Hj];
  fl[8] = k[8]*n[IDX_Hk]*n[IDX_Hj];
  fl[9] = k[9]*n[IDX_H]*n[IDX_Hj];
  fl[10] = k[10]*n[IDX_H2j];
  fl[11] = k[11]*n[IDX_H2j]*n[IDX_H];
  fl[12] = k[12]*n[IDX_H2j]*n[IDX_E];
  fl[13] = k[13]*n[IDX_H2j];
  fl[14] = k[14]*n[IDX_H2j]*n[IDX_H2];
  fl[15] = k[15]*n[IDX_H2]*n[IDX_Hj];
  fl[16] = k[16]*n[IDX_H2]*n[IDX_Hj];
  fl[17] = k[17]*n[IDX_H2]*n[IDX_E];
  fl[18] = k[18]*n[IDX_H2]*n[IDX_E];
  fl[19] = k[19]*n[IDX_H2];
  fl[20] = k[20]*n[IDX_H3j]*n[IDX_H];
  fl[21] = k[21]*n[IDX_H3j]*n[IDX_E];
  fl[22] = k[22]*n[IDX_H2]*n[IDX_Hj];
  fl[23] = k[23]*n[IDX_Hejj]*n[IDX_E];
  fl[24] = k[24]*n[IDX_Hej];
  fl[25] = k[25]*n[IDX_Hej]*n[IDX_E];
  fl[26] = k[26]*n[IDX_He];
  fl[27] = k[27]*n[IDX_He]*n[IDX_Hj];
  fl[28] = k[28]*n[IDX_Hej]*n[IDX_H];
  fl[29] = k[29]*n[IDX_He]*n[IDX_Hj];
  fl[30] = k[30]*n[IDX_He]*n[IDX_Hj];
  fl[31] = k[31]*n[IDX_He]*n[IDX_H2j];
  fl[32] = k[32]*n[IDX_Hej]*n[IDX_H];
  fl[33] = k[33]*n[IDX_Hej]*n[IDX_H];
  fl[34] = k[34]*n[IDX_HeHj]*n[IDX_H];
  fl[35] = k[35]*n[IDX_HeHj]*n[IDX_E];
  fl[36] = k[36]*n[IDX_HeHj]*n[IDX_H2];
  fl[37] = k[37]*n[IDX_HeHj];
  fl[38] = k[38]*n[IDX_HeHj];
  fl[39] = k[39]*n[IDX_Dj]*n[IDX_E];
  fl[40] = k[40]*n[IDX_D];
  fl[41] = k[41]*n[IDX_D]*n[IDX_Hj];
  fl[42] = k[42]*n[IDX_Dj]*n[IDX_H];
  fl[43] = k[43]*n[IDX_D]*n[IDX_H];
  fl[44] = k[44]*n[IDX_D]*n[IDX_H2];
  fl[45] = k[45]*n[IDX_HDj]*n[IDX_H];
  fl[46] = k[46]*n[IDX_Dj]*n[IDX_H2];
  fl[47] = k[47]*n[IDX_HD]*n[IDX_H];
  fl[48] = k[48]*n[IDX_HD]*n[IDX_Hj];
  fl[49] = k[49]*n[IDX_HD]*n[IDX_H3j];
  fl[50] = k[50]*n[IDX_D]*n[IDX_Hj];
  fl[51] = k[51]*n[IDX_Dj]*n[IDX_H];
  fl[52] = k[52]*n[IDX_HDj];
  fl[53] = k[53]*n[IDX_HDj];
  fl[54] = k[54]*n[IDX_HDj]*n[IDX_E];
  fl[55] = k[55]*n[IDX_HDj]*n[IDX_H2];
  fl[56] = k[56]*n[IDX_HDj]*n[IDX_H2];
  fl[57] = k[57]*n[IDX_D]*n[IDX_H3j];
  fl[58] = k[58]*n[IDX_H2Dj]*n[IDX_E];
  fl[59] = k[59]*n[IDX_H2Dj]*n[IDX_E];
  fl[60] = k[60]*n[IDX_H2Dj]*n[IDX_E];
  fl[61] = k[61]*n[IDX_H2Dj]*n[IDX_H2];
  fl[62] = k[62]*n[IDX_H2Dj]*n[IDX_H2];
  fl[63] = k[63]*n[IDX_H2Dj]*n[IDX_H];
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

constexpr bool HAS_THERMAL_TERMS = false;
// a rate coefficient depends on the densities (the species block
// of jac_stoich, taken at fixed k, is then not the exact dF/dn)
constexpr bool RATES_DEPEND_ON_N = true;
}  // namespace kbnet
