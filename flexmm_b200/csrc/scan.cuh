// Prefix sums of the tree build and the evaluation set-up (split counts,
// parent and node flags, targets per leaf, charges): one launch, the same
// result on every run.
//
// Tiles of SC_TILE consecutive elements (tile t on block t mod grid):
//   1. every block sums its tiles (each thread its SC_ITEMS items in order,
//      then the threads in a fixed order) into tsum[t] and, when the caller
//      uses the outputs as offsets, writes zeros over its tiles' outputs (a
//      valid fallback: 0 is in range); with one tile per block the tile
//      stays in registers for step 3;
//   2. a grid barrier; every block scans tsum over all tiles in a fixed
//      order (the same numbers on every block and every run) for its tiles'
//      prefixes;
//   3. each thread scans its items onto the prefix of its thread, warp and
//      tile and writes them.
// For floating point the grouping is fixed by the tile and thread layout,
// so results do not depend on timing.  A barrier wait that runs out sets
// *fail (if given) and leaves the fallback.  One tile runs as one block (no
// barrier).
#pragma once
#include "radix.cuh"

namespace fmmb {
namespace {

constexpr int SC_THREADS = 512;
constexpr int SC_ITEMS = 8;
constexpr int SC_TILE = SC_THREADS * SC_ITEMS;

// exclusive scan of one value per thread of the block; returns this
// thread's prefix, *total the block's sum (warp shuffles, then the warp
// totals in shared memory; fixed order)
template <class T>
__device__ T sc_block_exclusive(T v, T *total) {
  __shared__ T wsum[SC_THREADS / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  T incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const T u = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += u;
  }
  T ex = __shfl_up_sync(0xffffffffu, incl, 1);  // exclusive, not incl - v (exact for floats)
  if (lane == 0) ex = T(0);
  if (lane == 31) wsum[warp] = incl;
  __syncthreads();
  T before = T(0), all = T(0);
  for (int q = 0; q < SC_THREADS / 32; ++q) {
    if (q == warp) before = all;
    all += wsum[q];
  }
  __syncthreads();  // wsum reused by the next call
  *total = all;
  return before + ex;
}

template <class T, bool INCLUSIVE>
__global__ void __launch_bounds__(SC_THREADS, 2)
    k_scan(const T *__restrict__ in, T *out, int n, T *tsum, RadixSync *sync, int *fail,
           int zero_fallback) {
  // the tile, padded so that thread-blocked and coalesced accesses are both
  // free of bank conflicts
  constexpr int PAD = 128 / sizeof(T);
  __shared__ T stage[SC_TILE + SC_TILE / PAD];
  auto at = [](int k) { return k + k / PAD; };
  const int tiles = (n + SC_TILE - 1) / SC_TILE;
  const bool resident = gridDim.x > 1 && tiles <= (int)gridDim.x;  // phase 1's loads kept
  T v[SC_ITEMS];
  auto load = [&](int t) {
#pragma unroll
    for (int r = 0; r < SC_ITEMS; ++r) {
      const int i = t * SC_TILE + r * SC_THREADS + threadIdx.x;
      v[r] = i < n ? in[i] : T(0);
    }
  };
  // 1. tile sums (fixed order), optional zero fallback
  if (gridDim.x > 1) {
    for (int t = blockIdx.x; t < tiles; t += gridDim.x) {
      load(t);
      T s = T(0);
#pragma unroll
      for (int r = 0; r < SC_ITEMS; ++r) s += v[r];
      T total;
      sc_block_exclusive(s, &total);
      if (threadIdx.x == 0) tsum[t] = total;
      if (zero_fallback) {
#pragma unroll
        for (int r = 0; r < SC_ITEMS; ++r) {
          const int i = t * SC_TILE + r * SC_THREADS + threadIdx.x;
          if (i < n) out[i] = T(0);
        }
      }
    }
  }
  if (!grid_barrier(sync, fail)) return;
  // 2.-3. per tile: its prefix over the earlier tiles, then the items
  for (int t = blockIdx.x; t < tiles; t += gridDim.x) {
    T pre = T(0);
    if (gridDim.x > 1) {
      for (int c = 0; c * SC_THREADS < t; ++c) {  // tiles [0, t) in blocks of SC_THREADS
        const int j = c * SC_THREADS + threadIdx.x;
        T total;
        sc_block_exclusive(j < t ? __ldcg(&tsum[j]) : T(0), &total);
        pre += total;
      }
    }
    if (!resident) load(t);
#pragma unroll
    for (int r = 0; r < SC_ITEMS; ++r) stage[at(r * SC_THREADS + threadIdx.x)] = v[r];
    __syncthreads();
    T b[SC_ITEMS];
    T s = T(0);
#pragma unroll
    for (int r = 0; r < SC_ITEMS; ++r) {
      b[r] = stage[at(threadIdx.x * SC_ITEMS + r)];
      s += b[r];
    }
    T total;
    T run = pre + sc_block_exclusive(s, &total);
#pragma unroll
    for (int r = 0; r < SC_ITEMS; ++r) {
      if (INCLUSIVE) {
        run += b[r];
        b[r] = run;
      } else {
        const T x = b[r];
        b[r] = run;
        run += x;
      }
    }
#pragma unroll
    for (int r = 0; r < SC_ITEMS; ++r) stage[at(threadIdx.x * SC_ITEMS + r)] = b[r];
    __syncthreads();
#pragma unroll
    for (int r = 0; r < SC_ITEMS; ++r) {
      const int i = t * SC_TILE + r * SC_THREADS + threadIdx.x;
      if (i < n) out[i] = stage[at(r * SC_THREADS + threadIdx.x)];
    }
    __syncthreads();  // stage reused
  }
}

template <class T, bool INCLUSIVE>
int scan_grid(int64_t n) {
  static const int per_sm = [] {
    int b = 0;
    FMMB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k_scan<T, INCLUSIVE>, SC_THREADS, 0));
    return b;
  }();
  FMMB_CHECK(per_sm >= 1, ERR_CUDA, "scan kernel does not fit on an SM");
  const int64_t tiles = (n + SC_TILE - 1) / SC_TILE;
  if (tiles <= 1) return 1;
  int dev = 0, sms = 0;
  FMMB_CUDA(cudaGetDevice(&dev));
  FMMB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  return (int)std::min<int64_t>(tiles, (int64_t)sms * per_sm);
}

// scratch bytes of a scan of n elements
template <class T>
size_t scan_scratch_bytes(int64_t n) {
  return rs_round(sizeof(RadixSync)) + rs_round(sizeof(T) * (size_t)((n + SC_TILE - 1) / SC_TILE));
}

// out[i] = in[0] + ... + in[i - 1] (exclusive) or + in[i] (inclusive);
// in and out must not overlap
// zero_fallback: the outputs are offsets a later kernel writes through
// without a bounds check (on a failed barrier they are then 0, not garbage)
template <class T, bool INCLUSIVE>
void prefix_sum_run(const T *in, T *out, int64_t n, void *scratch, size_t bytes, int *fail,
                    bool zero_fallback, cudaStream_t s) {
  if (n <= 0) return;
  FMMB_CHECK(n < (int64_t(1) << 30), ERR_INVALID_ARGUMENT, "scan: more than 2^30 elements");
  FMMB_CHECK(bytes >= scan_scratch_bytes<T>(n), ERR_CAPACITY, "scan: scratch too small");
  RadixSync *sync = reinterpret_cast<RadixSync *>(scratch);
  T *tsum = reinterpret_cast<T *>(static_cast<unsigned char *>(scratch) + rs_round(sizeof(RadixSync)));
  const int g = scan_grid<T, INCLUSIVE>(n);
  int ni = (int)n, zf = zero_fallback ? 1 : 0;
  void *args[] = {(void *)&in, (void *)&out, (void *)&ni, (void *)&tsum, (void *)&sync,
                  (void *)&fail, (void *)&zf};
  if (g > 1) {
    FMMB_CUDA(cudaMemsetAsync(sync, 0, sizeof(RadixSync), s));
    FMMB_CUDA(cudaLaunchCooperativeKernel((const void *)k_scan<T, INCLUSIVE>, g, SC_THREADS, args,
                                          0, s));
  } else {
    FMMB_CUDA(cudaLaunchKernel((const void *)k_scan<T, INCLUSIVE>, 1, SC_THREADS, args, 0, s));
  }
}

template <class T, bool INCLUSIVE>
void prefix_sum(const T *in, T *out, int64_t n, int *fail, bool zero_fallback, cudaStream_t s) {
  if (n <= 0) return;
  const size_t bytes = scan_scratch_bytes<T>(n);
  DevBuf<unsigned char> tmp;
  tmp.alloc(bytes, s);
  prefix_sum_run<T, INCLUSIVE>(in, out, n, tmp.get(), bytes, fail, zero_fallback, s);
}

}  // namespace
}  // namespace fmmb
