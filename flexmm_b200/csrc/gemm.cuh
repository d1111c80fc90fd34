// Warp-level tensor-core GEMM helpers shared by the FMM passes.
#pragma once
#include "fmm.cuh"

namespace fmmb {

__host__ __device__ inline int pad_ld(int n) { return n + 4; }  // n multiple of 8 -> 4 or 12 mod 16

// D[8x8] += A[8x4] . B[4x8] on the FP64 tensor cores
__device__ __forceinline__ void dmma(double (&d)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

// Warp tile: C[r0 + 8*rb + g][c0 + 8*cb*cstride + 2q + i] += sum_k A[.][k] * B[k][.]
// for rb < RB and the column blocks cb < CB that start below ncols
// (g = lane/4, q = lane%4; fragment layouts of mma.m8n8k4.f64).
// A: shared memory, row-major, stride lda.  B: global, row-major [K][ldb].
template <int RB, int CB>
__device__ __forceinline__ void warp_gemm(const double *A, int lda, const double *__restrict__ B,
                                          int ldb, int K, int r0, int c0, int cstride, int ncols,
                                          double (&acc)[RB][CB][2]) {
  const int lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
  const double *Ap = A + (r0 + g) * lda + q;
  const double *Bp = B + (size_t)q * ldb + c0 + g;
#pragma unroll 2
  for (int k = 0; k < K; k += 4) {
    double a[RB], b[CB];
#pragma unroll
    for (int rb = 0; rb < RB; ++rb) a[rb] = Ap[8 * rb * lda + k];
#pragma unroll
    for (int cb = 0; cb < CB; ++cb)
      b[cb] = (c0 + 8 * cb * cstride < ncols) ? __ldg(Bp + (size_t)k * ldb + 8 * cb * cstride) : 0.0;
#pragma unroll
    for (int rb = 0; rb < RB; ++rb)
#pragma unroll
      for (int cb = 0; cb < CB; ++cb)
        if (c0 + 8 * cb * cstride < ncols) dmma(acc[rb][cb], a[rb], b[cb]);
  }
}

template <int RB, int CB>
__device__ __forceinline__ void zero_acc(double (&acc)[RB][CB][2]) {
#pragma unroll
  for (int rb = 0; rb < RB; ++rb)
#pragma unroll
    for (int cb = 0; cb < CB; ++cb) acc[rb][cb][0] = acc[rb][cb][1] = 0.0;
}

// Check-to-equivalent on a 32-row tile: out = ((P . U) * sinv) . VH.
// P, T: shared [32][pad_ld(np)].  Row t goes to out_row[t] (global, np
// doubles) when out_row[t] is not null.  Starts and ends with a barrier-free
// read of P; the caller synchronises before.
__device__ inline void c2e_tile(const LevelOpsDev &op, int np, const double *P, double *T,
                         double *const *out_row) {
  const int ldp = pad_ld(np);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
  const int r0 = 8 * (warp & 3), c0 = 8 * (warp >> 2);
  double acc[1][4][2];
  zero_acc(acc);
  warp_gemm<1, 4>(P, ldp, op.u, np, np, r0, c0, 2, np, acc);
#pragma unroll
  for (int cb = 0; cb < 4; ++cb) {
    const int col = c0 + 16 * cb + 2 * q;
    if (col < np) {
      T[(r0 + g) * ldp + col] = acc[0][cb][0] * op.sinv[col];
      T[(r0 + g) * ldp + col + 1] = acc[0][cb][1] * op.sinv[col + 1];
    }
  }
  __syncthreads();
  zero_acc(acc);
  warp_gemm<1, 4>(T, ldp, op.vh, np, np, r0, c0, 2, np, acc);
  double *o = out_row[r0 + g];
  if (o) {
#pragma unroll
    for (int cb = 0; cb < 4; ++cb) {
      const int col = c0 + 16 * cb + 2 * q;
      if (col < np) *reinterpret_cast<double2 *>(o + col) = make_double2(acc[0][cb][0], acc[0][cb][1]);
    }
  }
}


}  // namespace fmmb
