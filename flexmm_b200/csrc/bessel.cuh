// Modified Bessel functions K0 and K1 in FP64 for the modified Helmholtz
// kernel K0(k r) / (2 pi) (examples/kifmm_modified_helmholtz.py:25-39; its
// gradient uses K1, examples/pure_kifmm_modified_helmholtz_gradient.py:45-70).
//
// The reference evaluates K0 through piecewise Chebyshev tables fitted to
// scipy.special.k0 (function_generator, examples/kifmm_modified_helmholtz.py:28).
// Here, likewise tabulated but built without a third-party library:
//  * x < 1: the ascending series (Abramowitz & Stegun 9.6.13 and 9.6.11),
//      K0 = -(ln(x/2) + gamma) I0(x) + sum_k H_k y^k / (k!)^2,
//      K1 = 1/x + ln(x/2) I1(x) - (x/4) sum_k (psi(k+1) + psi(k+2)) y^k / (k!(k+1)!),
//    y = x^2/4, H_k the harmonic numbers, psi(n+1) = -gamma + H_n;
//  * 1 <= x < 1024: g_n(x) = sqrt(x) e^x K_n(x) as a degree-19 Chebyshev
//    series on each octave [2^j, 2^(j+1)), j = 0..9, with K_n = g_n e^-x / sqrt(x).
//    The coefficients are computed on the host (bessel_tables()) from the
//    integral representations e^x K0(x) = int_0^inf exp(-2x sinh^2(t/2)) dt,
//    e^x K1(x) = int_0^inf exp(-2x sinh^2(t/2)) cosh t dt, by the trapezoidal
//    rule (exponentially convergent for these analytic integrands);
//  * x >= 1024: 0 (below the smallest double).
// Relative error against scipy: ~5e-15 (series near x = 1), ~3e-15 (tables).
#pragma once
#include <math.h>

namespace fmmb {

constexpr int BESSEL_OCTAVES = 10;  // [1, 2) ... [512, 1024)
constexpr int BESSEL_NCHEB = 20;    // Chebyshev coefficients per octave
// table layout: [function n = 0, 1][octave][coefficient]
constexpr int BESSEL_TABLE_DOUBLES = 2 * BESSEL_OCTAVES * BESSEL_NCHEB;
constexpr double EULER_GAMMA = 0.57721566490153286061;

// g_n(x) on octave j from the table, Clenshaw recurrence
__device__ __forceinline__ double bessel_cheb(const double *__restrict__ tab, int n, int j,
                                              double x) {
  const double a = ldexp(1.0, j);
  const double u = (2.0 * x - 3.0 * a) / a;  // [a, 2a) -> [-1, 1)
  const double *c = tab + (n * BESSEL_OCTAVES + j) * BESSEL_NCHEB;
  double b1 = 0.0, b2 = 0.0;
#pragma unroll
  for (int i = BESSEL_NCHEB - 1; i >= 1; --i) {
    const double b0 = fma(2.0 * u, b1, -b2) + __ldg(c + i);
    b2 = b1;
    b1 = b0;
  }
  return fma(u, b1, -b2) + __ldg(c);
}

// K0(x) and, with K1 = true, K1(x) as well, for x > 0
template <bool K1>
__device__ __forceinline__ void bessel_k01(double x, const double *__restrict__ tab, double &k0,
                                           double &k1) {
  if (x < 1.0) {
    const double y = 0.25 * x * x;
    double t = 1.0, h = 0.0, i0 = 1.0, s0 = 0.0;  // t = y^k / (k!)^2
    double t1 = 1.0, i1 = 1.0, s1 = 2.0 * (-EULER_GAMMA) + 1.0;  // t1 = y^k / (k!(k+1)!)
#pragma unroll
    for (int k = 1; k <= 16; ++k) {
      t *= y / double(k * k);
      h += 1.0 / double(k);
      i0 += t;
      s0 = fma(t, h, s0);
      if (K1) {
        t1 *= y / double(k * (k + 1));
        i1 += t1;
        s1 = fma(t1, 2.0 * (h - EULER_GAMMA) + 1.0 / double(k + 1), s1);
      }
    }
    const double lg = log(0.5 * x);
    k0 = -(lg + EULER_GAMMA) * i0 + s0;
    if (K1) k1 = 1.0 / x + 0.5 * x * i1 * lg - 0.25 * x * s1;
    return;
  }
  if (x >= 1024.0) {
    k0 = 0.0;
    if (K1) k1 = 0.0;
    return;
  }
  int e;
  frexp(x, &e);  // x in [2^(e-1), 2^e)
  const int j = e - 1;
  const double w = exp(-x) * rsqrt(x);
  k0 = bessel_cheb(tab, 0, j, x) * w;
  if (K1) k1 = bessel_cheb(tab, 1, j, x) * w;
}

}  // namespace fmmb
