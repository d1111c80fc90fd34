// Device kernel functors, registered under the reference's example names.
//
//   Laplace_Eval: -log(|t-s|^2) / (4 pi)       examples/kifmm_laplace.py:24-29
//
// A functor evaluates K(source, target) for source (sx, sy) and target
// (tx, ty); the FMM kernels are templated on it, so the functor inlines into
// every loop the way the reference's numba kernel inlines into its closures
// (flexmm/flexmm2d/helpers.py:87-151).
#pragma once
#include <math.h>

#include "common.cuh"

namespace fmmb {

enum KernelId : int { KERNEL_LAPLACE = 0 };

struct KernelParams {
  double p[4];
};

struct LaplaceF64 {
  __host__ __device__ explicit LaplaceF64(const KernelParams &) {}
  __device__ __forceinline__ double operator()(double sx, double sy, double tx, double ty) const {
    const double dx = tx - sx, dy = ty - sy;
    return -log(dx * dx + dy * dy) * (1.0 / (4.0 * M_PI));
  }
};

}  // namespace fmmb
