// Device kernel functors, registered under the reference's example names.
//
//   Laplace_Eval: -log(|t-s|^2) / (4 pi)       examples/kifmm_laplace.py:24-29
//   Modified_Helmholtz_Eval: K0(k |t-s|) / (2 pi)  examples/kifmm_modified_helmholtz.py:33-39
//   a tabulated radial kernel f(|t-s|), as the reference's examples build
//   with function_generator (e.g. the Struve kernel, examples/bbfmm_struve.py:29-46)
//
// A functor evaluates K(source, target) for source (sx, sy) and target
// (tx, ty); the FMM kernels are templated on it, so the functor inlines into
// every loop the way the reference's numba kernel inlines into its closures
// (flexmm/flexmm2d/helpers.py:87-151).
#pragma once
#include <math.h>

#include <cmath>

#include "bessel.cuh"
#include "common.cuh"

namespace fmmb {

enum KernelId : int { KERNEL_LAPLACE = 0, KERNEL_MOD_HELMHOLTZ = 1, KERNEL_RADIAL_TABLE = 2 };

// the caller's parameters (p[0] = helmholtz k for the modified Helmholtz
// kernel) and the device's Bessel tables (bessel.cuh)
struct KernelParams {
  double p[4];
  const double *table;
};

struct LaplaceF64 {
  __host__ __device__ explicit LaplaceF64(const KernelParams &) {}
  __device__ __forceinline__ double operator()(double sx, double sy, double tx, double ty) const {
    const double dx = tx - sx, dy = ty - sy;
    return -log(dx * dx + dy * dy) * (1.0 / (4.0 * M_PI));
  }
  // potential and its gradient in the target position, times q, added to
  // (u, ux, uy) (Gradient_Eval, examples/pure_kifmm_laplace_gradient.py:32-55)
  __device__ __forceinline__ void grad(double sx, double sy, double tx, double ty, double q,
                                       double &u, double &ux, double &uy) const {
    const double dx = tx - sx, dy = ty - sy, d2 = dx * dx + dy * dy;
    const double s = -(1.0 / (2.0 * M_PI)) / d2 * q;
    u += -log(d2) * (1.0 / (4.0 * M_PI)) * q;
    ux += s * dx;
    uy += s * dy;
  }
};

struct ModHelmholtzF64 {
  double k;
  const double *tab;
  __host__ __device__ explicit ModHelmholtzF64(const KernelParams &kp) : k(kp.p[0]), tab(kp.table) {}
  __device__ __forceinline__ double operator()(double sx, double sy, double tx, double ty) const {
    const double dx = tx - sx, dy = ty - sy;
    double k0, k1;
    bessel_k01<false>(k * sqrt(dx * dx + dy * dy), tab, k0, k1);
    return k0 * (1.0 / (2.0 * M_PI));
  }
  // potential and its gradient in the target position, times q:
  // d/dt K0(k r) = -k K1(k r) (t - s) / r
  // (examples/pure_kifmm_modified_helmholtz_gradient.py:45-70)
  __device__ __forceinline__ void grad(double sx, double sy, double tx, double ty, double q,
                                       double &u, double &ux, double &uy) const {
    const double dx = tx - sx, dy = ty - sy, r = sqrt(dx * dx + dy * dy);
    double k0, k1;
    bessel_k01<true>(k * r, tab, k0, k1);
    const double s = -k * k1 / r * (1.0 / (2.0 * M_PI)) * q;
    u += k0 * (1.0 / (2.0 * M_PI)) * q;
    ux += s * dx;
    uy += s * dy;
  }
};

// K(s, t) = f(|t - s|) with f tabulated as Chebyshev series on the octaves
// [2^j, 2^(j+1)), j = j0 .. j0 + noct - 1 (table [noct][ncheb], built on the
// host from any function; the octave grid resolves power-law and log
// behaviour at 0).  Distances outside the tabulated range are clamped to it.
struct RadialTableF64 {
  const double *tab;
  int j0, noct, ncheb;
  __host__ __device__ explicit RadialTableF64(const KernelParams &kp)
      : tab(kp.table), j0(int(kp.p[1])), noct(int(kp.p[2])), ncheb(int(kp.p[3])) {}
  __device__ __forceinline__ double f(double r) const {
    const double lo = ldexp(1.0, j0), hi = ldexp(1.0, j0 + noct);
    r = fmin(fmax(r, lo), hi * (1.0 - 1e-16));
    int e;
    frexp(r, &e);
    const int oct = e - 1 - j0;
    const double a = ldexp(1.0, e - 1);
    const double u = (2.0 * r - 3.0 * a) / a;
    const double *c = tab + oct * ncheb;
    double b1 = 0.0, b2 = 0.0;
    for (int i = ncheb - 1; i >= 1; --i) {
      const double b0 = fma(2.0 * u, b1, -b2) + __ldg(c + i);
      b2 = b1;
      b1 = b0;
    }
    return fma(u, b1, -b2) + __ldg(c);
  }
  __device__ __forceinline__ double operator()(double sx, double sy, double tx, double ty) const {
    const double dx = tx - sx, dy = ty - sy;
    return f(sqrt(dx * dx + dy * dy));
  }
  // a tabulated kernel carries no derivative table: gradients are not offered
  __device__ __forceinline__ void grad(double, double, double, double, double, double &, double &,
                                       double &) const {}
};

// log2 on the special-function unit, denormal inputs flushed to zero
// (lg2.approx.ftz.f32: relative error ~2^-22 on normal inputs).
__device__ __forceinline__ float lg2_ftz(float x) {
  float r;
  asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// FP32 evaluation for the mixed-precision passes.  The log kernel is scale
// invariant up to a constant, K(w r) = offset(w) + K(r) with offset(w) =
// -log(w^2)/(4 pi): the mixed passes evaluate K in FP32 on coordinates divided
// by the box width (O(1) arguments, so FP32 keeps the kernel's variation to
// ~1e-7 absolute) and add offset(w) times the charge sum in FP64.  Kernels
// without such a decomposition set kScaled = false and offset() = 0.
//
// Radial form used by the P2P loop: K(dx, dy) = kScale * radial(dx^2 + dy^2),
// with kScale folded into the staged charges.  radial() is only called on
// squared distances >= FLT_MIN (smaller ones are coincident pairs, handled
// apart in FP64).
struct LaplaceF32 {
  static constexpr bool kScaled = true;
  // radial(d2) is -inf for d2 below FLT_MIN (the flushed log2 of 0)
  static constexpr bool kInfAtZero = true;
  static constexpr float kScale = (float)(-0.69314718055994531 / (4.0 * M_PI));  // -ln2 / (4 pi)
  __host__ __device__ explicit LaplaceF32(const KernelParams &) {}
  // -log(d2)/(4 pi) = -(ln 2 / 4 pi) * log2(d2); on width-scaled coordinates
  // the hardware log2's error is ~2e-7 of log2, ~1e-8 of K
  // (dx, dy) = target - source
  __device__ __forceinline__ float operator()(float dx, float dy) const {
    return lg2_ftz(dx * dx + dy * dy) * kScale;
  }
  __device__ __forceinline__ float radial(float d2) const { return lg2_ftz(d2); }
  // gradient in the target position: kGradScale * (dx, dy) / d2 on width-scaled
  // coordinates (times 1/w for absolute units)
  static constexpr double kGradScale = -1.0 / (2.0 * M_PI);
  static double offset(double w, const KernelParams &) { return -std::log(w * w) / (4.0 * M_PI); }
};

}  // namespace fmmb
