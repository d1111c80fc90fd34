// Helpers shared by the dense-operator FMM forms (black-box, Stokes); their
// translations are row GEMMs (rowgemm.cuh).
#pragma once
#include "fmm.cuh"

namespace fmmb {
namespace {

__device__ __forceinline__ int node_level_of(const int *__restrict__ off, int L, int g) {
  int lo = 0, hi = L;  // largest l with off[l] <= g
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (off[mid] <= g)
      lo = mid;
    else
      hi = mid;
  }
  return lo;
}

}  // namespace
}  // namespace fmmb
