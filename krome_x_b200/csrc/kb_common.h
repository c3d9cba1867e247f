// Common definitions of the B200 chemistry integrator: the host/device
// qualifier, the physical constants the network physics uses, and the
// integer-power helper the generated rate expressions call.
//
// The constants are the CODATA 2018 / IAU values the reference network
// generator writes into every project (reference: kromex/constants.py, the
// `constants` namespace of each generated net_<name>_core.hpp); they have
// to be the same numbers for the rates to agree.
#pragma once
#include <cmath>

#if defined(__CUDACC__)
#define KB_HD __host__ __device__
#define KB_DEV __device__
#define KB_UNROLL _Pragma("unroll")
#else
#define KB_HD
#define KB_DEV
#define KB_UNROLL
#endif

// The special functions of the network math (rates, cooling, heating) are
// called through these wrappers, which the device code keeps out of line:
// the generated rates and thermal terms call exp / log / pow at ~130 sites
// per rhs, and CUDA's math routines inlined at every site made the rhs code
// larger than the instruction caches serve, so the lane kernel stalled on
// instruction fetch. Out of line, the primordial3 hydro-loop calls ran
// 16-20 % faster on the B200. The values are the math library's, unchanged.
#if defined(__CUDACC__)
#define KB_MATH static __host__ __device__ __noinline__
#else
#define KB_MATH static inline
#endif
KB_MATH double kb_exp(double x) { return std::exp(x); }
KB_MATH double kb_log(double x) { return std::log(x); }
KB_MATH double kb_log10(double x) { return std::log10(x); }
KB_MATH double kb_pow(double x, double y) { return std::pow(x, y); }
// 10^x: on the device CUDA's exp10 (the cost of an exp, where pow(10, x)
// takes a logarithm and an exponential in extended precision: the
// thermal fits evaluate ~26 of them per rhs; 2-3 % on the primordial3
// hydro calls), on the host pow(10, x) as the reference writes it
#if defined(__CUDACC__)
static __host__ __device__ __noinline__ double kb_exp10(double x) {
#ifdef __CUDA_ARCH__
  return exp10(x);
#else
  return std::pow(10.0, x);
#endif
}
#else
static inline double kb_exp10(double x) { return std::pow(10.0, x); }
#endif

namespace kbc {
constexpr double boltzmann_eV = 8.617333262145179e-05;
constexpr double boltzmann_erg = 1.380649e-16;
constexpr double planck_erg = 6.62607015e-27;
constexpr double hc_k = 1.4387768775039336;  // cm K: E/k [K] = hc_k E [cm^-1]
constexpr double e_mass = 9.1093837015e-28;
constexpr double planck_eV = 4.135667696923859e-15;
constexpr double gravity = 6.6743e-08;
constexpr double p_mass = 1.67262192369e-24;
constexpr double amu = 1.6605390666e-24;
constexpr double clight = 29979245800.0;
constexpr double pi = 3.141592653589793;
constexpr double eV_to_erg = 1.602176634e-12;
constexpr double stefboltz_erg = 5.6703744191844286e-05;
constexpr double seconds_per_year = 31557600.0;
}  // namespace kbc

// x^N for a literal integer exponent by binary powering (the evaluation the
// generated expressions assume: products, not pow, so the roundoff is the
// reference's; reference: generated net_<name>_core.hpp ipow_)
template <int N>
KB_HD inline double ipow_(double x) {
  if constexpr (N < 0) {
    return 1.0 / ipow_<-N>(x);
  } else if constexpr (N == 0) {
    (void)x;
    return 1.0;
  } else if constexpr (N == 1) {
    return x;
  } else {
    const double h = ipow_<N / 2>(x);
    if constexpr (N % 2 == 1) return h * h * x;
    else return h * h;
  }
}
