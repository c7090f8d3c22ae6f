// device_math.cuh - FP64 special functions for the SHORE basis, on the device.
//
// Device restatements of the scalar recurrences cs_dmri evaluates while it
// builds a design matrix (src/math.rs:8-166): exact factorial table with a
// Gamma fallback, the Lanczos Gamma approximation (g = 7, the nine published
// coefficients of Numerical Recipes / Godfrey), associated Legendre functions
// with the Condon-Shortley phase, generalised Laguerre polynomials, and the
// Cartesian -> spherical conversion.
#pragma once

#include <cuda_runtime.h>
#include <math_constants.h>

namespace csd {

__device__ __forceinline__ double lanczos_gamma(double x);

// factorial(n): table below 21, Gamma(n + 1) above (src/math.rs:8-37).
__device__ __forceinline__ double dev_factorial(unsigned n) {
  const double t[21] = {1.0,
                        1.0,
                        2.0,
                        6.0,
                        24.0,
                        120.0,
                        720.0,
                        5040.0,
                        40320.0,
                        362880.0,
                        3628800.0,
                        39916800.0,
                        479001600.0,
                        6227020800.0,
                        87178291200.0,
                        1307674368000.0,
                        20922789888000.0,
                        355687428096000.0,
                        6402373705728000.0,
                        121645100408832000.0,
                        2432902008176640000.0};
  if (n < 21) return t[n];
  return lanczos_gamma(static_cast<double>(n + 1));
}

// Lanczos Gamma for x >= 0.5 (every argument the basis uses is >= 1.5);
// src/math.rs:40-64.
__device__ __forceinline__ double lanczos_gamma(double x) {
  const double c[9] = {0.99999999999980993,  676.5203681218851,     -1259.1392167224028,
                       771.32342877765313,   -176.61502916214059,   12.507343278686905,
                       -0.13857109526572012, 9.9843695780195716e-6, 1.5056327351493116e-7};
  x -= 1.0;
  double a = c[0];
  const double t = x + 7.0 + 0.5;
#pragma unroll
  for (int i = 1; i < 9; ++i) a += c[i] / (x + static_cast<double>(i));
  return sqrt(2.0 * CUDART_PI) * pow(t, x + 0.5) * exp(-t) * a;
}

// P_l^m(x) with the Condon-Shortley phase (src/math.rs:70-100).
__device__ __forceinline__ double dev_assoc_legendre(unsigned l, unsigned m, double x) {
  double pmm = 1.0;
  if (m > 0) {
    const double somx2 = sqrt(fmax((1.0 - x) * (1.0 + x), 0.0));
    double fact = 1.0;
    for (unsigned i = 0; i < m; ++i) {
      pmm *= -fact * somx2;
      fact += 2.0;
    }
  }
  if (l == m) return pmm;
  double pmmp1 = x * (2.0 * m + 1.0) * pmm;
  if (l == m + 1) return pmmp1;
  double pll = 0.0;
  for (unsigned ll = m + 2; ll <= l; ++ll) {
    const double llf = ll, mf = m;
    pll = ((2.0 * llf - 1.0) * x * pmmp1 - (llf + mf - 1.0) * pmm) / (llf - mf);
    pmm = pmmp1;
    pmmp1 = pll;
  }
  return pll;
}

// L_n^alpha(x) by three-term recurrence (src/math.rs:108-124).
__device__ __forceinline__ double dev_gen_laguerre(unsigned n, double alpha, double x) {
  if (n == 0) return 1.0;
  double lkm1 = 1.0;
  double lk = 1.0 + alpha - x;
  if (n == 1) return lk;
  for (unsigned k = 1; k < n; ++k) {
    const double kf = k;
    const double lkp1 = ((2.0 * kf + 1.0 + alpha - x) * lk - (kf + alpha) * lkm1) / (kf + 1.0);
    lkm1 = lk;
    lk = lkp1;
  }
  return lk;
}

// kappa(zeta, n, l) = sqrt(2 (n-l)! / (zeta^1.5 Gamma(n + 3/2)))
// (src/basis/shore.rs:56-61).
__device__ __forceinline__ double dev_kappa(double zeta, unsigned n, unsigned l) {
  const double num = 2.0 * dev_factorial(n - l);
  const double den = pow(zeta, 1.5) * lanczos_gamma(static_cast<double>(n) + 1.5);
  return sqrt(num / den);
}

// R_nl(q) (src/basis/shore.rs:64-70).
__device__ __forceinline__ double dev_shore_radial(unsigned n, unsigned l, double q, double zeta) {
  const double u = q * q / zeta;
  const double lag = dev_gen_laguerre(n - l, static_cast<double>(l) + 0.5, u);
  const double env = exp(-u * 0.5);
  const double rp = pow(u, static_cast<double>(l) / 2.0);
  return dev_kappa(zeta, n, l) * lag * env * rp;
}

// One entry (column k of the 2l+1 block) of the BrainSuite real SH block
// (src/basis/shore.rs:76-115): cosine terms m = l..1 in columns 0..l-1, the
// m = 0 term in column l, signed sine terms m = 1..l in columns l+1..2l.
__device__ __forceinline__ double dev_brainsuite_sh(unsigned l, unsigned k, double theta,
                                                    double phi) {
  if (l == 0) return 1.0 / sqrt(4.0 * CUDART_PI);
  const double cphi = cos(phi);
  const double tlp1 = 2.0 * l + 1.0;
  unsigned m;
  if (k < l)
    m = l - k;
  else if (k == l)
    m = 0;
  else
    m = k - l;
  const double norm =
      sqrt(tlp1 / (4.0 * CUDART_PI) * dev_factorial(l - m) / dev_factorial(l + m));
  const double p = norm * dev_assoc_legendre(l, m, cphi);
  const double s2 = sqrt(2.0);
  if (k < l) return s2 * p * cos(static_cast<double>(m) * theta);
  if (k == l) return p;
  const double sign = ((m + 1) % 2 == 0) ? 1.0 : -1.0;
  return s2 * sign * p * sin(static_cast<double>(m) * theta);
}

}  // namespace csd
