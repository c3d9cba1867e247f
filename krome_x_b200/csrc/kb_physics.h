// Runtime physics the benchmark networks call from their rates and thermal
// terms, restated for host and device (KB_HD). Each function evaluates the
// published fit the reference's runtime module evaluates, with the same
// constants and the same operation order (the CPU checker compiles this
// file too and must reproduce the reference's numbers bit for bit):
//
//   cooling_Atomic     Cen 1992 collisional ionization + excitation
//                      (reference runtime/core/cooling.hpp:32-68)
//   cooling_H2         Glover & Abel 2008 low-density colliders, HM79 /
//                      Glover 2015 LTE limit (cooling.hpp:74-177)
//   cooling_Continuum  Lenzuni+1996 Planck opacity, Jeans-length escape
//                      (cooling.hpp:282-303)
//   dissH2_Martin96    Martin, Schwarz & Mandy 1996 H2 collisional
//                      dissociation (special_rates.hpp:20-63)
//   H/He_recombination_on_dust  Weingartner & Draine 2001
//                      (dust_rates.hpp:37-66)
//   H2_solomonLW       Solomon-process H2 photodissociation
//                      (h2_shielding.hpp:84-93)
//   recfast_*          RECFAST 1.5.2 H and He I recombination and CMB
//                      photoionization (special_rates.hpp:106-288)
//
// Included inside the network namespace after the generated indices; the
// KB_HAS_<species> macros select the terms a network has.
#pragma once

KB_HD inline double cool_sigmoid_(double x, double x0, double s) {
  return 10.0 / (10.0 + kb_exp(-s * (x - x0)));
}

KB_HD inline double wCool_(double logT, double logTmin, double logTmax) {
  const double x = (logT - logTmin) / (logTmax - logTmin);
  const double w = kb_exp10(200.0 * (cool_sigmoid_(x, -0.2, 50.0)
                            * cool_sigmoid_(-x, -1.2, 50.0) - 1.0));
  return (w < 1e-199) ? 0.0 : w;
}

#ifdef KB_HAS_E
KB_HD inline double cooling_Atomic(double Tgas, const double* n) {
  const double temp = std::fmax(Tgas, 10.0);
  const double T5 = temp / 1e5;
  const double ne = n[IDX_E];
  (void)T5; (void)ne;
  double cool = 0.0;
#ifdef KB_HAS_H
  cool += 1.27e-21 * std::sqrt(temp) / (1.0 + std::sqrt(T5))
          * kb_exp(-1.578091e5 / temp) * ne * n[IDX_H];
#endif
#ifdef KB_HAS_He
  cool += 9.38e-22 * std::sqrt(temp) / (1.0 + std::sqrt(T5))
          * kb_exp(-2.853354e5 / temp) * ne * n[IDX_He];
#endif
#ifdef KB_HAS_Hej
  cool += 4.95e-22 * std::sqrt(temp) / (1.0 + std::sqrt(T5))
          * kb_exp(-6.31515e5 / temp) * ne * n[IDX_Hej];
  cool += 5.01e-27 * kb_pow(temp, -0.1687) / (1.0 + std::sqrt(T5))
          * kb_exp(-5.5338e4 / temp) * ne * ne * n[IDX_Hej];
#endif
#ifdef KB_HAS_H
  cool += 7.5e-19 / (1.0 + std::sqrt(T5)) * kb_exp(-1.18348e5 / temp)
          * ne * n[IDX_H];
#endif
#ifdef KB_HAS_Hej
  cool += 9.1e-27 * kb_pow(temp, -0.1687) / (1.0 + std::sqrt(T5))
          * kb_exp(-1.3179e4 / temp) * ne * ne * n[IDX_Hej];
  cool += 5.54e-17 * kb_pow(temp, -0.397) / (1.0 + std::sqrt(T5))
          * kb_exp(-4.73638e5 / temp) * ne * n[IDX_Hej];
#endif
  return std::fmax(cool, 0.0);
}
#else
KB_HD inline double cooling_Atomic(double, const double*) { return 0.0; }
#endif

#ifdef KB_HAS_H2
KB_HD inline double cooling_H2(double Tgas, const double* n) {
  const double temp = Tgas;
  const double T3 = temp * 1e-3;
  const double logt3 = kb_log10(T3);
  const double logt = kb_log10(temp);
  const double logt32 = logt3 * logt3, logt33 = logt32 * logt3,
               logt34 = logt33 * logt3, logt35 = logt34 * logt3,
               logt36 = logt35 * logt3, logt37 = logt36 * logt3,
               logt38 = logt37 * logt3;
  const double w14 = wCool_(logt, 1.0, 4.0);
  const double w24 = wCool_(logt, 2.0, 4.0);
  (void)w14; (void)w24; (void)logt36; (void)logt37; (void)logt38;
  double cool = 0.0;
#ifdef KB_HAS_H
  double fH2H;
  if (temp <= 1e2)
    fH2H = kb_exp10(-16.818342 + 37.383713 * logt3
           + 58.145166 * logt32 + 48.656103 * logt33
           + 20.159831 * logt34 + 3.8479610 * logt35) * n[IDX_H];
  else if (temp <= 1e3)
    fH2H = kb_exp10(-24.311209 + 3.5692468 * logt3
           - 11.332860 * logt32 - 27.850082 * logt33
           - 21.328264 * logt34 - 4.2519023 * logt35) * n[IDX_H];
  else if (temp <= 6e3)
    fH2H = kb_exp10(-24.311209 + 4.6450521 * logt3
           - 3.7209846 * logt32 + 5.9369081 * logt33
           - 5.5108049 * logt34 + 1.5538288 * logt35) * n[IDX_H];
  else
    fH2H = 1.862314467912518e-22 * wCool_(logt, 1.0, kb_log10(6e3))
           * n[IDX_H];
  cool += fH2H;
#endif
#ifdef KB_HAS_Hj
  double fH2Hp;
  if (temp > 1e1 && temp <= 1e4)
    fH2Hp = kb_exp10(-22.089523 + 1.5714711 * logt3
            + 0.015391166 * logt32 - 0.23619985 * logt33
            - 0.51002221 * logt34 + 0.32168730 * logt35) * n[IDX_Hj];
  else
    fH2Hp = 1.182509139382060e-21 * n[IDX_Hj] * w14;
  cool += fH2Hp;
#endif
  cool += w24 * kb_exp10(-23.962112 + 2.09433740 * logt3
          - 0.77151436 * logt32 + 0.43693353 * logt33
          - 0.14913216 * logt34 - 0.033638326 * logt35) * n[IDX_H2];
#ifdef KB_HAS_E
  double fH2e;
  if (temp <= 5e2)
    fH2e = kb_exp10(std::fmin(-21.928796 + 16.815730 * logt3
           + 96.743155 * logt32 + 343.19180 * logt33
           + 734.71651 * logt34 + 983.67576 * logt35
           + 801.81247 * logt36 + 364.14446 * logt37
           + 70.609154 * logt38, 30.0)) * n[IDX_E];
  else
    fH2e = kb_exp10(-22.921189 + 1.6802758 * logt3
           + 0.93310622 * logt32 + 4.0406627 * logt33
           - 4.7274036 * logt34 - 8.8077017 * logt35
           + 8.9167183 * logt36 + 6.4380698 * logt37
           - 6.3701156 * logt38) * n[IDX_E];
  cool += fH2e * w24;
#endif
#ifdef KB_HAS_He
  double fH2He;
  if (temp > 1e1 && temp <= 1e4)
    fH2He = kb_exp10(-23.689237 + 2.1892372 * logt3
            - 0.81520438 * logt32 + 0.29036281 * logt33
            - 0.16596184 * logt34 + 0.19191375 * logt35) * n[IDX_He];
  else
    fH2He = 1.002560385050777e-22 * n[IDX_He] * w14;
  cool += fH2He;
#endif
  if (cool <= 0.0) return 0.0;
  double HDL;
  if (temp < 2e3) {
    const double HDLR = 9.5e-22 * kb_pow(T3, 3.76)
                        / (1.0 + 0.12 * kb_pow(T3, 2.1))
                        * kb_exp(-kb_pow(0.13 / T3, 3.0))
                        + 3e-24 * kb_exp(-0.51 / T3);
    const double HDLV = 6.7e-19 * kb_exp(-5.86 / T3)
                        + 1.6e-18 * kb_exp(-11.7 / T3);
    HDL = HDLR + HDLV;
  } else if (temp <= 1e4) {
    HDL = kb_exp10(-20.584225 + 5.0194035 * logt3
          - 1.5738805 * logt32 - 4.7155769 * logt33
          + 2.4714161 * logt34 + 5.4710750 * logt35
          - 3.9467356 * logt36 - 2.2148338 * logt37
          + 1.8161874 * logt38);
  } else {
    const double dump14 = 1.0
        / (1.0 + kb_exp(std::fmin((temp - 3e4) * 2e-4, 3e2)));
    HDL = 5.531333679406485e-19 * dump14;
  }
  if (HDL == 0.0) return 0.0;
  return n[IDX_H2] / (1.0 / HDL + 1.0 / cool);
}
#else
KB_HD inline double cooling_H2(double, const double*) { return 0.0; }
#endif

// ---- the same two fits split at a fixed temperature ----
// cooling_X_coef(T) evaluates a fit's temperature-only factors once and
// cooling_X_with(c, n) combines them with the densities in the original
// expressions' order of operations, so that
// cooling_X_with(cooling_X_coef(T), n) == cooling_X(T, n) bit for bit: a
// row of density derivatives at one T (the adjoint's Jacobian) then
// evaluates the transcendental part once instead of once per column.
struct CoolAtomicC {
  double c[7];
};
KB_HD inline CoolAtomicC cooling_Atomic_coef(double Tgas) {
  CoolAtomicC q{};
#ifdef KB_HAS_E
  const double temp = std::fmax(Tgas, 10.0);
  const double T5 = temp / 1e5;
  q.c[0] = 1.27e-21 * std::sqrt(temp) / (1.0 + std::sqrt(T5))
           * kb_exp(-1.578091e5 / temp);
  q.c[1] = 9.38e-22 * std::sqrt(temp) / (1.0 + std::sqrt(T5))
           * kb_exp(-2.853354e5 / temp);
  q.c[2] = 4.95e-22 * std::sqrt(temp) / (1.0 + std::sqrt(T5))
           * kb_exp(-6.31515e5 / temp);
  q.c[3] = 5.01e-27 * kb_pow(temp, -0.1687) / (1.0 + std::sqrt(T5))
           * kb_exp(-5.5338e4 / temp);
  q.c[4] = 7.5e-19 / (1.0 + std::sqrt(T5)) * kb_exp(-1.18348e5 / temp);
  q.c[5] = 9.1e-27 * kb_pow(temp, -0.1687) / (1.0 + std::sqrt(T5))
           * kb_exp(-1.3179e4 / temp);
  q.c[6] = 5.54e-17 * kb_pow(temp, -0.397) / (1.0 + std::sqrt(T5))
           * kb_exp(-4.73638e5 / temp);
#else
  (void)Tgas;
#endif
  return q;
}
KB_HD inline double cooling_Atomic_with(const CoolAtomicC& q, const double* n) {
#ifdef KB_HAS_E
  const double ne = n[IDX_E];
  (void)ne;
  double cool = 0.0;
#ifdef KB_HAS_H
  cool += q.c[0] * ne * n[IDX_H];
#endif
#ifdef KB_HAS_He
  cool += q.c[1] * ne * n[IDX_He];
#endif
#ifdef KB_HAS_Hej
  cool += q.c[2] * ne * n[IDX_Hej];
  cool += q.c[3] * ne * ne * n[IDX_Hej];
#endif
#ifdef KB_HAS_H
  cool += q.c[4] * ne * n[IDX_H];
#endif
#ifdef KB_HAS_Hej
  cool += q.c[5] * ne * ne * n[IDX_Hej];
  cool += q.c[6] * ne * n[IDX_Hej];
#endif
  return std::fmax(cool, 0.0);
#else
  (void)q; (void)n;
  return 0.0;
#endif
}

// H2: per collider the factor a (and b: the fits whose density multiplies
// before the w14 / w24 weight), the H2-H2 term's w24 x fit, the LTE HDL
struct CoolH2C {
  double aH, aHp, bHp, aH2, ae, be, aHe, bHe, HDL;
  int fHp, fHe;  // 1: the fit is a (x n); 0: (a x n) x b
};
KB_HD inline CoolH2C cooling_H2_coef(double Tgas) {
  CoolH2C q{};
#ifdef KB_HAS_H2
  const double temp = Tgas;
  const double T3 = temp * 1e-3;
  const double logt3 = kb_log10(T3);
  const double logt = kb_log10(temp);
  const double logt32 = logt3 * logt3, logt33 = logt32 * logt3,
               logt34 = logt33 * logt3, logt35 = logt34 * logt3,
               logt36 = logt35 * logt3, logt37 = logt36 * logt3,
               logt38 = logt37 * logt3;
  const double w14 = wCool_(logt, 1.0, 4.0);
  const double w24 = wCool_(logt, 2.0, 4.0);
  (void)w14; (void)logt36; (void)logt37; (void)logt38;
  if (temp <= 1e2)
    q.aH = kb_exp10(-16.818342 + 37.383713 * logt3
           + 58.145166 * logt32 + 48.656103 * logt33
           + 20.159831 * logt34 + 3.8479610 * logt35);
  else if (temp <= 1e3)
    q.aH = kb_exp10(-24.311209 + 3.5692468 * logt3
           - 11.332860 * logt32 - 27.850082 * logt33
           - 21.328264 * logt34 - 4.2519023 * logt35);
  else if (temp <= 6e3)
    q.aH = kb_exp10(-24.311209 + 4.6450521 * logt3
           - 3.7209846 * logt32 + 5.9369081 * logt33
           - 5.5108049 * logt34 + 1.5538288 * logt35);
  else
    q.aH = 1.862314467912518e-22 * wCool_(logt, 1.0, kb_log10(6e3));
  if (temp > 1e1 && temp <= 1e4) {
    q.fHp = 1;
    q.aHp = kb_exp10(-22.089523 + 1.5714711 * logt3
            + 0.015391166 * logt32 - 0.23619985 * logt33
            - 0.51002221 * logt34 + 0.32168730 * logt35);
  } else {
    q.fHp = 0;
    q.aHp = 1.182509139382060e-21;
    q.bHp = w14;
  }
  q.aH2 = w24 * kb_exp10(-23.962112 + 2.09433740 * logt3
          - 0.77151436 * logt32 + 0.43693353 * logt33
          - 0.14913216 * logt34 - 0.033638326 * logt35);
  if (temp <= 5e2)
    q.ae = kb_exp10(std::fmin(-21.928796 + 16.815730 * logt3
           + 96.743155 * logt32 + 343.19180 * logt33
           + 734.71651 * logt34 + 983.67576 * logt35
           + 801.81247 * logt36 + 364.14446 * logt37
           + 70.609154 * logt38, 30.0));
  else
    q.ae = kb_exp10(-22.921189 + 1.6802758 * logt3
           + 0.93310622 * logt32 + 4.0406627 * logt33
           - 4.7274036 * logt34 - 8.8077017 * logt35
           + 8.9167183 * logt36 + 6.4380698 * logt37
           - 6.3701156 * logt38);
  q.be = w24;
  if (temp > 1e1 && temp <= 1e4) {
    q.fHe = 1;
    q.aHe = kb_exp10(-23.689237 + 2.1892372 * logt3
            - 0.81520438 * logt32 + 0.29036281 * logt33
            - 0.16596184 * logt34 + 0.19191375 * logt35);
  } else {
    q.fHe = 0;
    q.aHe = 1.002560385050777e-22;
    q.bHe = w14;
  }
  if (temp < 2e3) {
    const double HDLR = 9.5e-22 * kb_pow(T3, 3.76)
                        / (1.0 + 0.12 * kb_pow(T3, 2.1))
                        * kb_exp(-kb_pow(0.13 / T3, 3.0))
                        + 3e-24 * kb_exp(-0.51 / T3);
    const double HDLV = 6.7e-19 * kb_exp(-5.86 / T3)
                        + 1.6e-18 * kb_exp(-11.7 / T3);
    q.HDL = HDLR + HDLV;
  } else if (temp <= 1e4) {
    q.HDL = kb_exp10(-20.584225 + 5.0194035 * logt3
          - 1.5738805 * logt32 - 4.7155769 * logt33
          + 2.4714161 * logt34 + 5.4710750 * logt35
          - 3.9467356 * logt36 - 2.2148338 * logt37
          + 1.8161874 * logt38);
  } else {
    const double dump14 = 1.0
        / (1.0 + kb_exp(std::fmin((temp - 3e4) * 2e-4, 3e2)));
    q.HDL = 5.531333679406485e-19 * dump14;
  }
#else
  (void)Tgas;
#endif
  return q;
}
KB_HD inline double cooling_H2_with(const CoolH2C& q, const double* n) {
#ifdef KB_HAS_H2
  double cool = 0.0;
#ifdef KB_HAS_H
  const double fH2H = q.aH * n[IDX_H];
  cool += fH2H;
#endif
#ifdef KB_HAS_Hj
  const double fH2Hp = q.fHp ? q.aHp * n[IDX_Hj] : q.aHp * n[IDX_Hj] * q.bHp;
  cool += fH2Hp;
#endif
  cool += q.aH2 * n[IDX_H2];
#ifdef KB_HAS_E
  const double fH2e = q.ae * n[IDX_E];
  cool += fH2e * q.be;
#endif
#ifdef KB_HAS_He
  const double fH2He = q.fHe ? q.aHe * n[IDX_He] : q.aHe * n[IDX_He] * q.bHe;
  cool += fH2He;
#endif
  if (cool <= 0.0) return 0.0;
  if (q.HDL == 0.0) return 0.0;
  return n[IDX_H2] / (1.0 / q.HDL + 1.0 / cool);
#else
  (void)q; (void)n;
  return 0.0;
#endif
}

// Planck mean opacity (Lenzuni+1996, density-only fit)
KB_HD inline double kpla_(const double* n) {
  const double rho = rho_(n);
  if (rho < 1e-12) return 0.0;
  const double y = kb_log10(std::fmin(rho, 0.5));
  return kb_exp10(1.000042 * y + 2.14989);
}

KB_HD inline double cooling_Continuum(double Tgas, const double* n) {
  const double rho = std::fmax(rho_(n), 1e-40);
  const double kgas = kpla_(n);
  const double mu = rho / std::fmax(ntot_(n), 1e-40) / kbc::p_mass;
  const double lj = std::sqrt(kbc::pi * kbc::boltzmann_erg * Tgas
                              / rho / kbc::p_mass / kbc::gravity / mu);
  const double tau = lj * kgas * rho + 1e-40;
  const double beta = std::fmin(1.0, 1.0 / (tau * tau));
  return 4.0 * kbc::stefboltz_erg * Tgas * Tgas * Tgas * Tgas
      * kgas * rho * beta;
}

#ifdef KB_EXTERN_dissH2_Martin96
KB_HD inline double dissH2_Martin96(double Tgas_in, const double* n,
                                    const Params& p) {
  (void)p;
  const double Tgas = std::fmin(Tgas_in, 4.5e4);
  constexpr double m[2][21] = {
      {-178.4239, -68.42243, 43.20243, -4.633167, 69.70086, 40870.38,
       -23705.70, 128.8953, -53.91334, 5.315517, -19.73427, 16780.95,
       -25786.11, 14.82123, -4.890915, 0.4749030, -133.8283, -1.164408,
       0.8227443, 0.5864073, -2.056313},
      {-142.7664, 42.70741, -2.027365, -0.2582097, 21.36094, 27535.31,
       -21467.79, 60.34928, -27.43096, 2.676150, -11.28215, 14254.55,
       -23125.20, 9.305564, -2.464009, 0.1985955, 743.0600, -1.174242,
       0.7502286, 0.2358848, 2.937507}};
  const double n_H = Hnuclei_(n);
  const double logT = kb_log10(Tgas);
  const double invT = 1.0 / Tgas;
  const double logT2 = logT * logT;
  const double logT3 = logT2 * logT;
  double k_CID = 0.0;
KB_UNROLL
  for (int i = 0; i < 2; ++i) {
    const double* c = m[i];
    const double logk_h1 = c[0] + c[1] * logT + c[2] * logT2
        + c[3] * logT3 + c[4] * kb_log10(1.0 + c[5] * invT);
    const double logk_h2 = c[6] * invT;
    const double logk_l1 = c[7] + c[8] * logT + c[9] * logT2
        + c[10] * kb_log10(1.0 + c[11] * invT);
    const double logk_l2 = c[12] * invT;
    const double logn_c1 = c[13] + c[14] * logT + c[15] * logT2
        + c[16] * invT;
    const double logn_c2 = c[17] + logn_c1;
    const double pp = c[18] + c[19] * kb_exp(-Tgas / 1.850e3)
        + c[20] * kb_exp(-Tgas / 4.40e2);
    const double n_c1 = kb_exp10(logn_c1);
    const double n_c2 = kb_exp10(logn_c2);
    const double logk_CID = logk_h1
        - (logk_h1 - logk_l1) / (1.0 + kb_pow(n_H / n_c1, pp))
        + logk_h2
        - (logk_h2 - logk_l2) / (1.0 + kb_pow(n_H / n_c2, pp));
    k_CID += kb_exp10(logk_CID);
  }
  return k_CID;
}
#endif

#if defined(KB_EXTERN_H_recombination_on_dust) \
    || defined(KB_EXTERN_He_recombination_on_dust)
KB_HD inline double wd01_fit_(double pre, double c1, double p1, double c2,
                              double q, double p2a, double p2b, double Tgas,
                              const double* n, const Params& p) {
  if (n[IDX_E] < 1e-20) return 0.0;
  const double scale = pre * (p.d2g / 1e-2);
  const double psi = p.G0 * std::sqrt(Tgas) / n[IDX_E];
  if (psi <= 0.0) return scale;
  return scale / (1.0 + c1 * kb_pow(psi, p1)
                  * (1.0 + c2 * kb_pow(Tgas, q)
                     * kb_pow(psi, p2a + p2b * kb_log(Tgas))));
}
#endif
#ifdef KB_EXTERN_H_recombination_on_dust
KB_HD inline double H_recombination_on_dust(double Tgas, const double* n,
                                            const Params& p) {
  return wd01_fit_(1.225e-13, 8.074e-6, 1.378, 5.087e2, 0.01586, -0.4723,
                   -1.102e-5, Tgas, n, p);
}
#endif
#ifdef KB_EXTERN_He_recombination_on_dust
KB_HD inline double He_recombination_on_dust(double Tgas, const double* n,
                                             const Params& p) {
  return wd01_fit_(5.572e-14, 3.185e-7, 1.512, 5.115e3, 3.903e-7, -0.4956,
                   -5.494e-7, Tgas, n, p);
}
#endif
#ifdef KB_EXTERN_H2_solomonLW
KB_HD inline double H2_solomonLW(double flux_eV, double Tgas, const double* n,
                                 const Params& p) {
  (void)Tgas; (void)n; (void)p;
  return 1.38e9 * flux_eV * kbc::eV_to_erg;
}
#endif

#if defined(KB_EXTERN_recfast_H_rec) || defined(KB_EXTERN_recfast_H_ion) \
    || defined(KB_EXTERN_recfast_He_rec) || defined(KB_EXTERN_recfast_He_ion)
// Cosmological recombination of H and He I after RECFAST 1.5.2 (Seager,
// Sasselov & Scott 1999, 2000; Wong, Moss & Scott 2008), as the reference's
// runtime states it (special_rates.hpp:106-224): each net RECFAST rate
// C (n_e n_X+ alpha - n_X beta e^(-E/kT)) split into a recombination
// coefficient C alpha and a CMB photoionization rate C beta e^(-E/kT).
// The escape factors C use H(z) = hubble0 (1 + z) sqrt(1 + omega0 z).
// RECFAST's atomic data in cgs (wavenumbers in cm^-1, rates in s^-1,
// cross sections in cm^2):
namespace rf {
constexpr double kH_ion = 1.096787737e5, kH_alpha = 8.225916453e4;
constexpr double kHe1_ion = 1.98310772e5, kHe_2s = 1.66277434e5;
constexpr double kHe_2p = 1.71134891e5, kHe_2Pt = 1.690871466e5;
constexpr double kHe_2St = 1.5985597526e5, kHe2St_ion = 3.8454693845e4;
constexpr double two_photon_H = 8.2245809, two_photon_He = 51.3;
constexpr double A2P_singlet = 1.798287e9, A2P_triplet = 177.58;
constexpr double sigma_2Ps = 1.436289e-18, sigma_2Pt = 1.484872e-18;
constexpr double mass_ratio_He = 3.9715;
constexpr double fudge_H = 1.125, fudge_He = 0.86;

struct Rates {
  double alpha, beta, C;
};
struct Common {
  double T, z, Hz, hck, crT15;
};

KB_HD inline Common common(double Tgas, const Params& p) {
  Common c;
  c.T = Tgas;
  c.z = p.zredshift;
  c.Hz = p.hubble0 * (1.0 + c.z) * std::sqrt(1.0 + p.omega0 * c.z);
  c.hck = kbc::hc_k;
  // (2 pi m_e k T / h^2)^(3/2)
  const double cr = 2.0 * kbc::pi * kbc::e_mass * kbc::boltzmann_erg
      / (kbc::planck_erg * kbc::planck_erg);
  c.crT15 = kb_pow(cr * c.T, 1.5);
  return c;
}

// H: case-B alpha of Pequignot, Petitjean & Boisson, the Peebles factor
// with the fudge and the double-Gaussian correction of K
KB_HD inline Rates hydrogen(const Common& c, double nH0) {
  Rates r;
  const double t4 = c.T * 1e-4;
  r.alpha = 1e-13 * 4.309 * kb_pow(t4, -0.6166)
      / (1.0 + 0.6703 * kb_pow(t4, 0.53));
  const double up = r.alpha * c.crT15
      * kb_exp(-c.hck * (kH_ion - kH_alpha) / c.T);
  r.beta = up * kb_exp(-c.hck * kH_alpha / c.T);
  const double lz = kb_log(1.0 + c.z);
  const double g1 = (lz - 7.28) / 0.18, g2 = (lz - 6.73) / 0.33;
  const double K = 1.0 / (kH_alpha * kH_alpha * kH_alpha)
      / (8.0 * kbc::pi * c.Hz)
      * (1.0 - 0.14 * kb_exp(-g1 * g1) + 0.079 * kb_exp(-g2 * g2));
  const double KL = K * two_photon_H * nH0;
  r.C = fudge_H * (1.0 + KL) / (1.0 + KL + fudge_H * K * up * nH0);
  return r;
}

// the Sobolev continuum-opacity term of a He I 2P line (Kholupenko,
// Ivanchik & Varshalovich 2007): A / (1 + a g^b), 0 without neutral H
KB_HD inline double he_continuum(const Common& c, double nH0, double nHe0,
                                 double k_line, double A, double sigma,
                                 double a, double b) {
  if (!(nH0 > 0.0)) return 0.0;
  const double mH = kbc::p_mass + kbc::e_mass;
  const double doppler = kbc::clight * k_line
      * std::sqrt(2.0 * kbc::boltzmann_erg * c.T
                  / (mH * mass_ratio_He * kbc::clight * kbc::clight));
  const double g = 3.0 * A * nHe0 / nH0
      / (std::sqrt(kbc::pi) * sigma * 8.0 * kbc::pi * doppler * k_line * k_line);
  return A / (1.0 + a * kb_pow(g, b));
}

// (1 - e^-tau) / tau, 1 for an optically thin line
KB_HD inline double escape(double tau) {
  return tau > 1e-8 ? -std::expm1(-tau) / tau : 1.0;
}

// the He I recombination fits (square-root terms shared by both)
KB_HD inline double he_alpha(double s0, double s1, double lg, double e) {
  return kb_exp10(lg) / (s0 * kb_pow(1.0 + s0, 1.0 - e))
      / kb_pow(1.0 + s1, 1.0 + e);
}

// He I singlet: the Sobolev escape of 2^1P - 1^1S with the H continuum
KB_HD inline Rates helium_singlet(const Common& c, double nH0, double nHe0,
                                  double s0, double s1) {
  Rates r;
  r.alpha = he_alpha(s0, s1, -10.744, 0.711);
  const double up = 4.0 * r.alpha * c.crT15
      * kb_exp(-c.hck * (kHe1_ion - kHe_2s) / c.T);
  r.beta = up * kb_exp(-c.hck * kHe_2s / c.T);
  const double boltz = kb_exp(std::fmin(c.hck * (kHe_2p - kHe_2s) / c.T, 680.0));
  const double tau = A2P_singlet / (kHe_2p * kHe_2p * kHe_2p)
      / (8.0 * kbc::pi) * 3.0 * nHe0 / c.Hz;
  const double cont = he_continuum(c, nH0, nHe0, kHe_2p, A2P_singlet,
                                   sigma_2Ps, 0.36, fudge_He);
  // K_He n_He0 = 1 / (3 (A p + A_cont)), finite as n_He0 -> 0
  const double kn = 1.0 / (3.0 * (A2P_singlet * escape(tau) + cont));
  r.C = (1.0 + kn * two_photon_He * boltz)
      / (1.0 + kn * (two_photon_He + up) * boltz);
  return r;
}

// He I triplets, C = 1 / (1 + up / cf) with the two Boltzmann factors
// combined (each alone underflows at low T)
KB_HD inline Rates helium_triplet(const Common& c, double nH0, double nHe0,
                                  double s0, double s1) {
  Rates r;
  r.alpha = he_alpha(s0, s1, -10.306, 0.761);
  const double up = r.alpha * kb_exp(-c.hck * kHe2St_ion / c.T) * c.crT15
      * (4.0 / 3.0);
  r.beta = 3.0 * up * kb_exp(-c.hck * kHe_2St / c.T);
  const double tau = A2P_triplet * nHe0 * 3.0
      / (8.0 * kbc::pi * c.Hz * kHe_2Pt * kHe_2Pt * kHe_2Pt);
  const double cont = he_continuum(c, nH0, nHe0, kHe_2Pt, A2P_triplet,
                                   sigma_2Pt, 0.66, 0.9) / 3.0;
  const double ru = r.alpha * c.crT15 * (4.0 / 3.0)
      / (A2P_triplet * escape(tau) + cont)
      * kb_exp(-c.hck * (kHe2St_ion - (kHe_2Pt - kHe_2St)) / c.T);
  r.C = 1.0 / (1.0 + ru);
  return r;
}

KB_HD inline void helium(double Tgas, double nH0, double nHe0,
                         const Params& p, Rates& s, Rates& t) {
  const Common c = common(Tgas, p);
  const double s0 = std::sqrt(c.T / kb_exp10(0.477121));
  const double s1 = std::sqrt(c.T / kb_exp10(5.114));
  s = helium_singlet(c, nH0, nHe0, s0, s1);
  t = helium_triplet(c, nH0, nHe0, s0, s1);
}
}  // namespace rf

// H+ + e- -> H: C alpha_B [cm^3 s^-1] (nH0 the neutral H density)
KB_HD inline double recfast_H_rec(double nH0, double Tgas, const double* n,
                                  const Params& p) {
  (void)n;
  const rf::Rates r = rf::hydrogen(rf::common(Tgas, p), nH0);
  return r.C * r.alpha;
}
// H -> H+ + e- by the CMB: C beta e^(-h nu_a / kT) [s^-1]
KB_HD inline double recfast_H_ion(double nH0, double Tgas, const double* n,
                                  const Params& p) {
  (void)n;
  const rf::Rates r = rf::hydrogen(rf::common(Tgas, p), nH0);
  return r.C * r.beta;
}
// He+ + e- -> He: singlet + triplet C alpha [cm^3 s^-1]
KB_HD inline double recfast_He_rec(double nHe0, double nH0, double Tgas,
                                   const double* n, const Params& p) {
  (void)n;
  rf::Rates s, t;
  rf::helium(Tgas, nH0, nHe0, p, s, t);
  return s.C * s.alpha + t.C * t.alpha;
}
// He -> He+ + e- by the CMB: singlet + triplet [s^-1]
KB_HD inline double recfast_He_ion(double nHe0, double nH0, double Tgas,
                                   const double* n, const Params& p) {
  (void)n;
  rf::Rates s, t;
  rf::helium(Tgas, nH0, nHe0, p, s, t);
  return s.C * s.beta + t.C * t.beta;
}
#endif
