// Gathers and scatters shared by the dense-operator FMM forms (black-box,
// Stokes): their translations are GEMMs over node rows of np doubles, and
// these kernels move rows between the node arrays and the GEMM operands.
// Real sibling groups (children of split boxes) are listed in the tree's rg
// array; a group's 4 children are consecutive nodes.
#pragma once
#include <cublas_v2.h>

#include <string>

#include "fmm.cuh"

namespace fmmb {
namespace {

#define FMMB_BLAS(call)                                                                     \
  do {                                                                                      \
    cublasStatus_t st_ = (call);                                                            \
    if (st_ != CUBLAS_STATUS_SUCCESS)                                                       \
      throw Error(ERR_CUDA, std::string("cuBLAS error ") + std::to_string(int(st_)) + " in " \
                                + #call);                                                   \
  } while (0)

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

// rows[e] -> dst row node(e) = parent[c_first + 4 e]  (M2M results to parent rows)
__global__ void k_rows_to_parents(int n_groups, int np, int c_first, const int *__restrict__ parent,
                                const double *__restrict__ rows, double *__restrict__ dst) {
  const int64_t total = (int64_t)n_groups * np;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int e = int(i / np), q = int(i - (int64_t)e * np);
    dst[(size_t)parent[c_first + 4 * e] * np + q] = rows[i];
  }
}

// M2L gather of a level: row 4 g + c (node rg[g] + c) holds, for each offset
// o, the source multipole il[node][o] (zeros if none) at columns o np .. o np + np
__global__ void k_m2l_gather_cat(int n_groups, int np, const int *__restrict__ rg, int rg_lo,
                                const int *__restrict__ il, const double *__restrict__ mult,
                                double *__restrict__ sbig) {
  const int64_t rowlen = (int64_t)N_OFFSETS * np;
  const int64_t total = (int64_t)n_groups * 4 * rowlen;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t row = i / rowlen;
    const int col = int(i - row * rowlen), o = col / np, q = col - o * np;
    const int node = rg[rg_lo + int(row >> 2)] + int(row & 3);
    const int s = il[(size_t)node * N_OFFSETS + o];
    sbig[i] = s >= 0 ? mult[(size_t)s * np + q] : 0.0;
  }
}

// ple[node(row)] += y[row]
__global__ void k_add_group_rows(int n_groups, int np, const int *__restrict__ rg, int rg_lo,
                              const double *__restrict__ y, double *__restrict__ ple) {
  const int64_t total = (int64_t)n_groups * 4 * np;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t row = i / np;
    const int q = int(i - row * np);
    const int node = rg[rg_lo + int(row >> 2)] + int(row & 3);
    ple[(size_t)node * np + q] += y[i];
  }
}

// L2L gather: the parent local of every real group of a level
__global__ void k_gather_parent_rows(int n_groups, int np, const int *__restrict__ rg, int rg_lo,
                                   const int *__restrict__ parent, const double *__restrict__ ple,
                                   double *__restrict__ lp) {
  const int64_t total = (int64_t)n_groups * np;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int g = int(i / np), q = int(i - (int64_t)g * np);
    lp[i] = ple[(size_t)parent[rg[rg_lo + g]] * np + q];
  }
}

// L2L scatter: the 4 children of group g are the consecutive rows rg[g] .. rg[g] + 3
__global__ void k_add_child_rows(int n_groups, int np, const int *__restrict__ rg, int rg_lo,
                                  const double *__restrict__ c, double *__restrict__ ple) {
  const int64_t rowlen = 4 * (int64_t)np;
  const int64_t total = (int64_t)n_groups * rowlen;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int g = int(i / rowlen);
    const int64_t k = i - (int64_t)g * rowlen;
    ple[(size_t)rg[rg_lo + g] * np + k] += c[i];
  }
}

}  // namespace
}  // namespace fmmb
