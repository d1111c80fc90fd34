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
// A: shared memory, row-major, stride lda.  B: row-major [K][ldb], in global
// memory (SB = false) or staged in shared memory (SB = true).
template <int RB, int CB, bool SB = false>
__device__ __forceinline__ void warp_gemm(const double *A, int lda, const double *B, int ldb, int K,
                                          int r0, int c0, int cstride, int ncols,
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
    for (int cb = 0; cb < CB; ++cb) {
      const double *bp = Bp + (size_t)k * ldb + 8 * cb * cstride;
      b[cb] = (c0 + 8 * cb * cstride < ncols) ? (SB ? *bp : __ldg(bp)) : 0.0;
    }
#pragma unroll
    for (int rb = 0; rb < RB; ++rb)
#pragma unroll
      for (int cb = 0; cb < CB; ++cb)
        if (c0 + 8 * cb * cstride < ncols) dmma(acc[rb][cb], a[rb], b[cb]);
  }
}

// Asynchronous 16-byte global -> shared copy (cp.async, L2 only); complete
// after cp_async_wait_all() and, for other threads, a barrier.
__device__ __forceinline__ void cp_async16(void *smem_dst, const void *gsrc) {
  const unsigned int d = static_cast<unsigned int>(__cvta_generic_to_shared(smem_dst));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(d), "l"(gsrc) : "memory");
}

__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_all;\n" ::: "memory");
}

// Start copying a rows x cols row-major matrix (row stride cols) from global
// to shared memory with row stride ld; cols and ld are multiples of 16 bytes,
// both pointers 16-byte aligned.  Wait with cp_async_wait_all + barrier.
template <class T>
__device__ __forceinline__ void stage_rows(T *dst, int ld, const T *__restrict__ src, int rows,
                                           int cols) {
  constexpr int V = 16 / sizeof(T);
  const int cv = cols / V, n = rows * cv;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const int r = i / cv, c = i - r * cv;
    cp_async16(dst + (size_t)r * ld + c * V, src + (size_t)i * V);
  }
}

// Shared-memory row stride (in floats) for a B operand of the split-TF32
// warp GEMMs: the four k-rows a warp reads start in distinct bank groups.
__host__ __device__ inline int ldb_f(int cols) { return (cols % 16 == 8) ? cols : cols + 8; }

template <int RB, int CB>
__device__ __forceinline__ void zero_acc(double (&acc)[RB][CB][2]) {
#pragma unroll
  for (int rb = 0; rb < RB; ++rb)
#pragma unroll
    for (int cb = 0; cb < CB; ++cb) acc[rb][cb][0] = acc[rb][cb][1] = 0.0;
}

// Check-to-equivalent operators as a GEMM reads them: U and VH row-major
// with row stride ld, in global memory or staged in shared memory.
struct C2EView {
  const double *u, *sinv, *vh;
  int ld;
};

__device__ __forceinline__ C2EView c2e_global(const LevelOpsDev &op, int np) {
  return {op.u, op.sinv, op.vh, np};
}

// start staging a level's check-to-equivalent operators (U, 1/S, VH) in
// shared memory (asynchronous, see stage_rows): dst holds
// c2e_stage_doubles(np) doubles
__device__ __forceinline__ C2EView c2e_stage(const LevelOpsDev &op, int np, double *dst) {
  const int ld = pad_ld(np);
  double *u = dst, *vh = dst + np * ld, *si = dst + 2 * np * ld;
  stage_rows(u, ld, op.u, np, np);
  stage_rows(vh, ld, op.vh, np, np);
  stage_rows(si, np, op.sinv, 1, np);
  return {u, si, vh, ld};
}

__host__ __device__ inline int c2e_stage_doubles(int np) { return 2 * np * pad_ld(np) + np; }

// Check-to-equivalent on a 32-row tile: out = ((P . U) * sinv) . VH.
// P, T: shared [32][pad_ld(np)].  Row t goes to out_row[t] (np doubles) when
// out_row[t] is not null.  Starts and ends with a barrier-free read of P; the
// caller synchronises before.
template <bool SB>
__device__ inline void c2e_tile(const C2EView &op, int np, const double *P, double *T,
                                double *const *out_row) {
  const int ldp = pad_ld(np);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
  const int r0 = 8 * (warp & 3), c0 = 8 * (warp >> 2);
  double acc[1][4][2];
  zero_acc(acc);
  warp_gemm<1, 4, SB>(P, ldp, op.u, op.ld, np, r0, c0, 2, np, acc);
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
  warp_gemm<1, 4, SB>(T, ldp, op.vh, op.ld, np, r0, c0, 2, np, acc);
  double *o = out_row[r0 + g];
  if (o) {
#pragma unroll
    for (int cb = 0; cb < 4; ++cb) {
      const int col = c0 + 16 * cb + 2 * q;
      if (col < np) *reinterpret_cast<double2 *>(o + col) = make_double2(acc[0][cb][0], acc[0][cb][1]);
    }
  }
}

__device__ inline void c2e_tile(const LevelOpsDev &op, int np, const double *P, double *T,
                                double *const *out_row) {
  c2e_tile<false>(c2e_global(op, np), np, P, T, out_row);
}

// ---- GEMMs with the B operand streamed through shared memory ----
// B (row-major [K][ldb] in global memory, first ncols columns) is copied in
// chunks of GS_KC rows into a double buffer Bs of gemm_stage_doubles(ncols)
// doubles (row stride pad_ld(ncols)), the next chunk in flight while the
// warps multiply the current one: the k-loop reads shared memory only,
// where reading B from L2 inside it left each warp waiting on one L2 round
// trip per few k-steps.  Called by every thread of the block (barriers
// inside); ncols even, ldb and B 16-byte aligned, K a multiple of 4; no
// copies of the caller may be in flight (they would join the first group).
constexpr int GS_KC = 16;
__host__ __device__ inline int gemm_stage_doubles(int ncols) { return 2 * GS_KC * pad_ld(ncols); }

__device__ __forceinline__ void cp_async_commit_group() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait_group() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

template <int RB, int CB>
__device__ void warp_gemm_staged(const double *A, int lda, const double *__restrict__ B, int ldb,
                                 int K, int r0, int c0, int cstride, int ncols,
                                 double (&acc)[RB][CB][2], double *Bs) {
  const int lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
  const int ldbs = pad_ld(ncols), per_row = ncols / 2;
  const int nch = (K + GS_KC - 1) / GS_KC;
  auto stage = [&](int c) {
    const int k0 = c * GS_KC, rows = min(GS_KC, K - k0);
    double *dst = Bs + (c & 1) * GS_KC * ldbs;
    for (int i = threadIdx.x; i < rows * per_row; i += blockDim.x) {
      const int r = i / per_row, c2 = 2 * (i - r * per_row);
      cp_async16(dst + r * ldbs + c2, B + (size_t)(k0 + r) * ldb + c2);
    }
    cp_async_commit_group();
  };
  stage(0);
  const double *Ap = A + (r0 + g) * lda + q;
  for (int c = 0; c < nch; ++c) {
    if (c + 1 < nch) {
      stage(c + 1);
      cp_async_wait_group<1>();
    } else {
      cp_async_wait_group<0>();
    }
    __syncthreads();
    const double *Bp = Bs + (c & 1) * GS_KC * ldbs + q * ldbs + c0 + g;
    const int k0 = c * GS_KC, kn = min(GS_KC, K - k0);
#pragma unroll 4
    for (int k = 0; k < kn; k += 4) {
      double a[RB], b[CB];
#pragma unroll
      for (int rb = 0; rb < RB; ++rb) a[rb] = Ap[8 * rb * lda + k0 + k];
#pragma unroll
      for (int cb = 0; cb < CB; ++cb)
        b[cb] = (c0 + 8 * cb * cstride < ncols) ? Bp[k * ldbs + 8 * cb * cstride] : 0.0;
#pragma unroll
      for (int rb = 0; rb < RB; ++rb)
#pragma unroll
        for (int cb = 0; cb < CB; ++cb)
          if (c0 + 8 * cb * cstride < ncols) dmma(acc[rb][cb], a[rb], b[cb]);
    }
    __syncthreads();  // buffer c & 1 is refilled by the next iteration's copies
  }
}

// c2e_tile with U and VH streamed through Bs (gemm_stage_doubles(np))
__device__ inline void c2e_tile_staged(const LevelOpsDev &op, int np, const double *P, double *T,
                                       double *const *out_row, double *Bs) {
  const int ldp = pad_ld(np);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
  const int r0 = 8 * (warp & 3), c0 = 8 * (warp >> 2);
  double acc[1][4][2];
  zero_acc(acc);
  warp_gemm_staged<1, 4>(P, ldp, op.u, np, np, r0, c0, 2, np, acc, Bs);
#pragma unroll
  for (int cb = 0; cb < 4; ++cb) {
    const int col = c0 + 16 * cb + 2 * q;
    if (col < np) {
      T[(r0 + g) * ldp + col] = acc[0][cb][0] * __ldg(op.sinv + col);
      T[(r0 + g) * ldp + col + 1] = acc[0][cb][1] * __ldg(op.sinv + col + 1);
    }
  }
  __syncthreads();
  zero_acc(acc);
  warp_gemm_staged<1, 4>(T, ldp, op.vh, np, np, r0, c0, 2, np, acc, Bs);
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
