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

#include <cfloat>
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

// ---------------------------------------------------------------------------
// Table-driven FP64 log2, after P. T. P. Tang, "Table-driven implementation
// of the logarithm function in IEEE floating-point arithmetic", ACM TOMS 16
// (1990): d = 2^e m, m in [1, 2); F = 1 + j/256 is the table point nearest m,
// so r = (m - F) / F has |r| <= 2^-9 and
//   log2 d = e + log2 F + log2(1 + r),
//   log2(1 + r) = r (c1 + r (c2 + r (c3 + r (c4 + r c5)))),  c_k = (-1)^(k+1) / (k ln 2),
// the Taylor series of log(1 + r) / ln 2 cut after r^5 (the first dropped
// term, r^6 / (6 ln 2), is below 1.3e-17).  m - F is exact; the table holds
// 1/F (IEEE division) and log2 F (CUDA's log2) for j = 0..256, filled in
// shared memory by each block.  Absolute error about one ulp of the result
// (~1e-16 relative to max(1, |log2 d|)): far inside the 1e-12 parity bar,
// at about a third of the FP64 instructions of the library log.  Zero,
// subnormal, infinite and NaN arguments take the library log2 instead.
constexpr int LOG2_TAB_N = 256;
struct Log2Table {
  double2 t[LOG2_TAB_N + 1];
  __device__ void fill() {
    for (int i = threadIdx.x; i <= LOG2_TAB_N; i += blockDim.x) {
      const double F = 1.0 + i * (1.0 / LOG2_TAB_N);
      t[i] = make_double2(1.0 / F, log2(F));
    }
  }
};

// true for arguments outside the table path: zero, subnormal, negative,
// infinite or NaN (one unsigned compare of the high word)
__device__ __forceinline__ bool log2_tab_rare(double d) {
  return (unsigned)(__double2hiint(d) - 0x00100000) >= 0x7FE00000u;
}

// log2 of a positive normal finite d (callers route log2_tab_rare arguments
// elsewhere)
__device__ __forceinline__ double log2_tab(double d, const double2 *__restrict__ tab) {
  constexpr double LN2 = 0.69314718055994530942;
  constexpr double C1 = 1.0 / LN2, C2 = -1.0 / (2.0 * LN2), C3 = 1.0 / (3.0 * LN2),
                   C4 = -1.0 / (4.0 * LN2), C5 = 1.0 / (5.0 * LN2);
  const int hi = __double2hiint(d), lo = __double2loint(d);
  const int mh = hi & 0x000FFFFF;
  const int j = (mh + (1 << 11)) >> 12;                           // nearest 1/256 step: 0..256
  const double m = __hiloint2double(mh | 0x3FF00000, lo);         // [1, 2)
  const double F = __hiloint2double(0x3FF00000 + (j << 12), 0);   // 1 + j/256 (j = 256: 2)
  const double2 tj = tab[j];
  const double r = (m - F) * tj.x;
  // the exponent as a double without a conversion instruction:
  // bits (0x43300000, e + 2^31) are 2^52 + 2^31 + e
  const double e = __hiloint2double(0x43300000, ((hi >> 20) - 1023) ^ (int)0x80000000) -
                   4503601774854144.0;
  double q = fma(r, C5, C4);
  q = fma(r, q, C3);
  q = fma(r, q, C2);
  q = fma(r, q, C1);
  return fma(r, q, e + tj.y);
}

// Shared-memory state a functor needs inside a kernel (the log2 table of
// LaplaceF64T); empty for the other functors.  bind() is called by every
// thread of the block before the functor's first use.
template <class KF, bool = KF::kLogTable>
struct FunctorSmem {
  __device__ void bind(KF &) {}
};

struct LaplaceF64 {
  static constexpr bool kLogTable = false;
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

// The Laplace kernel of the FP64 passes: LaplaceF64 with the table-driven
// log2 above.  raw(dx, dy) = log2(dx^2 + dy^2), so K = kFold * raw; the P2P
// and L2T loops fold kFold into their staged charges / locals.
struct LaplaceF64T {
  static constexpr bool kLogTable = true;
  static constexpr double kFold = -0.69314718055994530942 / (4.0 * M_PI);  // -ln2 / (4 pi)
  const double2 *lt = nullptr;  // the block's table (FunctorSmem::bind)
  __host__ __device__ explicit LaplaceF64T(const KernelParams &) {}
  __device__ __forceinline__ double raw(double dx, double dy) const {
    const double d2 = dx * dx + dy * dy;
    return log2_tab_rare(d2) ? log2(d2) : log2_tab(d2, lt);
  }
  // raw value of a P2P pair, 0 for a coincident pair when check is set
  // (flexmm/flexmm2d/helpers.py:99-107): a coincident pair has d2 = 0, so
  // the test only runs on the rare path
  __device__ __forceinline__ double raw_checked(double sx, double sy, double tx, double ty,
                                                int check) const {
    const double dx = tx - sx, dy = ty - sy, d2 = dx * dx + dy * dy;
    if (!log2_tab_rare(d2)) return log2_tab(d2, lt);
    return (check && dx == 0.0 && dy == 0.0) ? 0.0 : log2(d2);
  }
  __device__ __forceinline__ double operator()(double sx, double sy, double tx, double ty) const {
    return kFold * raw(tx - sx, ty - sy);
  }
  __device__ __forceinline__ void grad(double sx, double sy, double tx, double ty, double q,
                                       double &u, double &ux, double &uy) const {
    const double dx = tx - sx, dy = ty - sy, d2 = dx * dx + dy * dy;
    const double s = -(1.0 / (2.0 * M_PI)) / d2 * q;
    u += kFold * raw(dx, dy) * q;
    ux += s * dx;
    uy += s * dy;
  }
};

template <class KF>
struct FunctorSmem<KF, true> {
  Log2Table tab;
  __device__ void bind(KF &k) {
    tab.fill();
    __syncthreads();
    k.lt = tab.t;
  }
};

struct ModHelmholtzF64 {
  static constexpr bool kLogTable = false;
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
  static constexpr bool kLogTable = false;
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

// K0 in FP32 (A&S 9.8.1, 9.8.5, 9.8.6: Abramowitz & Stegun, Handbook of
// Mathematical Functions, polynomial approximations of I0 and K0):
//   x <= 2: K0(x) = -ln(x/2) I0(x) + P(t^2), t = x/2 (|error| < 1e-8), with
//           I0(x) = Q((x/3.75)^2) (relative error < 1.6e-7);
//   x > 2:  K0(x) = exp(-x) / sqrt(x) R(2/x) (relative error < 1.9e-7).
// Both branches are computed and one selected (no divergence within a warp
// of pairs at mixed distances).  K0(0) = +inf (the flushed log of 0).
__device__ __forceinline__ float bessel_k0_f32(float x) {
  const float y = (x * (1.f / 3.75f)) * (x * (1.f / 3.75f));
  const float i0 = fmaf(y, fmaf(y, fmaf(y, fmaf(y, fmaf(y, fmaf(y, 0.0045813f, 0.0360768f), 0.2659732f),
                                                   1.2067492f), 3.0899424f), 3.5156229f), 1.f);
  const float t2 = 0.25f * x * x;
  const float p = fmaf(t2, fmaf(t2, fmaf(t2, fmaf(t2, fmaf(t2, fmaf(t2, 0.0000074f, 0.0001075f), 0.00262698f),
                                                   0.0348859f), 0.23069756f), 0.4227842f), -0.57721566f);
  // -ln(x/2) = (1 - log2 x) ln 2
  const float small = fmaf((1.f - lg2_ftz(x)) * 0.69314718f, i0, p);
  const float z = 2.f * __frcp_rn(fmaxf(x, 2.f));
  const float r = fmaf(z, fmaf(z, fmaf(z, fmaf(z, fmaf(z, fmaf(z, 0.00053208f, -0.0025154f), 0.00587872f),
                                                  -0.01062446f), 0.02189568f), -0.07832358f), 1.25331414f);
  const float large = __expf(-x) * rsqrtf(fmaxf(x, 2.f)) * r;
  return x <= 2.f ? small : large;
}

// FP32 evaluation of K0(k r) / (2 pi) for the mixed passes.  K0 has no scale
// decomposition: the passes evaluate it on box-centred coordinates in the
// caller's units (kScaled = false, offset 0); FP32 keeps a pair's distance
// to ~1e-7 of the box width, which bounds the per-pair error as for the log
// kernel on width-scaled coordinates.
struct ModHelmholtzF32 {
  static constexpr bool kScaled = false;
  // radial(d2) is +inf for d2 below FLT_MIN (K0 at a flushed 0)
  static constexpr bool kInfAtZero = true;
  static constexpr float kScale = (float)(1.0 / (2.0 * M_PI));
  float k;
  __host__ __device__ explicit ModHelmholtzF32(const KernelParams &kp) : k((float)kp.p[0]) {}
  // (squared distances below FLT_MIN flushed to 0: K0 = +inf there)
  __device__ __forceinline__ float radial(float d2) const {
    return bessel_k0_f32(k * (d2 < FLT_MIN ? 0.f : sqrtf(d2)));
  }
  // (dx, dy) = target - source
  __device__ __forceinline__ float operator()(float dx, float dy) const {
    return radial(dx * dx + dy * dy) * kScale;
  }
  static double offset(double, const KernelParams &) { return 0.0; }
};

}  // namespace fmmb
