// Stable LSD radix sort of the tree build (point keys, split boxes, parent
// boxes): all passes in one cooperative launch, in the manner of the
// single-sweep radix sort with decoupled look-back (Adinets and Merrill,
// "Onesweep", 2022), with a grid barrier between passes instead of one
// launch per pass.
//
//   0. Prepass: every block counts the digits of every pass over its tiles
//      (digit counts do not depend on the order) into ghist[pass][256];
//      a grid barrier; every block scans them into the digit bases.
//   Pass p (8-bit digit at bit begin_bit + 8 p), per tile of RS_TILE
//   consecutive elements (tile t on block t mod grid, in rounds):
//   1. each warp loads its RS_CPW chunks of 32 consecutive elements into
//      registers and ranks them: ballots on the digit's bits group the lanes
//      of one digit, a lane's rank is the lanes of its group below it plus the
//      warp's running count of that digit, and the group's leader advances
//      the count.  Warp, then chunk, then lane is the input order, so ranks
//      follow the input order (a stable pass);
//   2. per digit, the warps' counts become warp offsets, and the tile's
//      count is published in status[pass][tile][digit] as an aggregate;
//      the digit's thread then looks back over the earlier tiles, adding
//      aggregates until it meets an inclusive prefix, and publishes the
//      tile's own inclusive prefix (flag and value in one 32-bit word);
//   3. every element goes to digit base + earlier tiles + earlier warps +
//      its rank; the last pass writes through the emit functor.
//   A grid barrier separates passes (the next pass reads what other blocks
//   wrote; such reads go through L2, __ldcg).
// Every wait is bounded: a barrier or look-back wait that runs out sets
// *fail (if given; and sync->timeout for barriers) and the block stops
// waiting.  Before the prepass barrier each block has written a valid
// fallback into every output slot of its own tiles (the emit's init: the
// identity permutation), and no write leaves [0, n), so the outputs hold
// valid indices even then.  A single-block launch has no barriers.
//
// The first pass reads its keys through a source functor (stored keys, or
// point keys computed from the coordinates) and the last pass writes
// through an emit functor (stored keys / values, or the permutation with
// the sorted coordinates and keys of the points), so key computation and
// the keyed gather need no launches of their own.
#pragma once
#include <algorithm>
#include <cstdint>

#include "common.cuh"

namespace fmmb {
namespace {

constexpr int RS_THREADS = 512;
constexpr int RS_WARPS = RS_THREADS / 32;
constexpr int RS_CPW = 8;                          // chunks of 32 per warp and tile
constexpr int RS_TILE = RS_WARPS * RS_CPW * 32;    // elements per tile
constexpr int RS_PMAX = 8;                         // passes of a 64-bit key
constexpr unsigned int RS_BARRIER_TRIES = 1u << 22;
constexpr unsigned int RS_LOOKBACK_TRIES = 1u << 22;
constexpr int RS_LB = 16;                          // look-back reads in flight
constexpr unsigned int RS_AGG = 1u << 30, RS_INC = 2u << 30, RS_VAL = RS_AGG - 1;

struct RadixSync {  // zero before the launch
  unsigned int count;  // barrier arrivals so far
  int timeout, pad0, pad1;
};

struct RadixWork {
  RadixSync *sync;   // zero before the launch
  int *ghist;        // [passes][256], zero before the launch (follows sync)
  unsigned *status;  // [passes][tiles][256]
  int *fail;         // optional: set to 1 when a wait ran out
  // optional: the element count in device memory (written by an earlier
  // kernel), at most the launch's n, which then only sizes grid and scratch
  const unsigned long long *n_dev;
};

__host__ __device__ inline int64_t radix_tiles(int64_t n) { return (n + RS_TILE - 1) / RS_TILE; }

// bytes of RadixWork storage (sync, ghist, status) for n elements and `passes`
inline size_t radix_work_bytes(int64_t n, int passes) {
  return sizeof(RadixSync) + sizeof(int) * 256 * (size_t)passes +
         sizeof(unsigned) * 256 * (size_t)passes * (size_t)radix_tiles(n);
}

// Grid barrier on a counter that only grows: barrier k of the launch is
// passed once the count reaches (k + 1) * gridDim.x, so the last block to
// arrive has nothing to release (arrival and release are one atomic).
__device__ bool grid_barrier(RadixSync *sync, int *fail) {
  __shared__ int ok;
  __syncthreads();
  if (gridDim.x == 1) return true;
  if (threadIdx.x == 0) {
    unsigned int *cnt = &sync->count;
    unsigned int old;
    asm volatile("atom.add.acq_rel.gpu.global.u32 %0, [%1], 1;" : "=r"(old) : "l"(cnt) : "memory");
    const unsigned int target = (old / gridDim.x + 1) * gridDim.x;
    int good = 1;
    unsigned int tries = 0, cur = old + 1;
    while (cur < target) {
      if (++tries > RS_BARRIER_TRIES) {
        atomicExch(&sync->timeout, 1);
        if (fail) atomicExch(fail, 1);
        good = 0;
        break;
      }
      asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(cur) : "l"(cnt) : "memory");
    }
    ok = good;
  }
  __syncthreads();
  return ok;
}

__device__ __forceinline__ bool rs_grid_sync(const RadixWork &w) { return grid_barrier(w.sync, w.fail); }

// lanes of the warp holding the same 9-bit label as this lane: one ballot
// per bit (cheaper than match.any here)
__device__ __forceinline__ unsigned rs_peers(int d) {
  unsigned peers = 0xffffffffu;
#pragma unroll
  for (int b = 0; b < 9; ++b) {
    const bool bit = (d >> b) & 1;
    const unsigned bal = __ballot_sync(0xffffffffu, bit);
    peers &= bit ? bal : ~bal;
  }
  return peers;
}

__device__ __forceinline__ unsigned rs_load(const unsigned *p) {
  unsigned v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p));
  return v;
}
__device__ __forceinline__ void rs_store(unsigned *p, unsigned v) {
  asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v));
}

// ---- sources (first pass) ----
template <class K>
struct SrcKeys {  // stored keys; stored values, or the element index when vin is NULL
  const K *kin;
  const int *vin;
  __device__ K key(int i) const { return __ldg(kin + i); }
  __device__ int val(int i) const { return vin ? __ldg(vin + i) : int(i); }
};

// ---- emits (last pass) ----
struct NoPre {};

template <class K>
struct EmitPairs {  // kout / vout may be NULL (not written)
  using Pre = NoPre;
  K *kout;
  int *vout;
  __device__ void init(int i) const {
    if (vout) vout[i] = int(i);
  }
  __device__ Pre fetch(int) const { return Pre{}; }
  __device__ void operator()(int pos, K k, int v, Pre) const {
    if (kout) kout[pos] = k;
    if (vout) vout[pos] = v;
  }
};

template <class K, class Src, class Emit, bool VALS>
__global__ void __launch_bounds__(RS_THREADS, 2)
    k_radix_sort(Src src, Emit emit, int64_t n64, int begin_bit, int end_bit, K *kb0, int *vb0,
                 K *kb1, int *vb1, RadixWork w) {
  __shared__ int wcnt[RS_WARPS * 256];
  __shared__ int dbase[RS_PMAX * 256];
  __shared__ int tofs[256];    // global position of the tile's first element of each digit
  __shared__ int tstart[256];  // tile position of the tile's first element of each digit
  __shared__ int dsum[8];
  extern __shared__ __align__(16) unsigned char rs_stage[];  // the tile in sorted order
  K *sk = reinterpret_cast<K *>(rs_stage);
  int *sv = reinterpret_cast<int *>(rs_stage + RS_TILE * sizeof(K));
  // < 2^30 (checked by the host): element indices fit in int
  const int n = w.n_dev ? (int)min((unsigned long long)n64, __ldcg(w.n_dev)) : (int)n64;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  unsigned lt;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(lt));
  int *my = wcnt + warp * 256;
  const int passes = (end_bit - begin_bit + 7) / 8;
  const int tiles = (int)radix_tiles(n);
  auto digit_of = [&](K k, int p) -> int {
    const int shift = begin_bit + 8 * p, bits = min(8, end_bit - shift);
    return int(unsigned(k >> shift) & ((1u << bits) - 1u));
  };

  // 0. digit counts of every pass; status rows cleared; fallback outputs
  for (int i = threadIdx.x; i < passes * 256; i += RS_THREADS) dbase[i] = 0;
  __syncthreads();
  for (int t = blockIdx.x; t < tiles; t += gridDim.x) {
    K kk[RS_TILE / RS_THREADS];
#pragma unroll
    for (int r = 0; r < RS_TILE / RS_THREADS; ++r) {
      const int i = t * RS_TILE + r * RS_THREADS + threadIdx.x;
      kk[r] = i < n ? src.key(i) : K(0);
    }
#pragma unroll
    for (int r = 0; r < RS_TILE / RS_THREADS; ++r) {
      const int i = t * RS_TILE + r * RS_THREADS + threadIdx.x;
      if (i >= n) continue;
      for (int p = 0; p < passes; ++p) atomicAdd(&dbase[p * 256 + digit_of(kk[r], p)], 1);
      if (gridDim.x > 1) emit.init(i);
    }
    for (int j = threadIdx.x; j < passes * 256; j += RS_THREADS)
      w.status[((size_t)(j >> 8) * tiles + t) * 256 + (j & 255)] = 0;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < passes * 256; i += RS_THREADS)
    if (dbase[i]) atomicAdd(&w.ghist[i], dbase[i]);
  if (!rs_grid_sync(w)) return;
  for (int p = 0; p < passes; ++p) {  // digit bases: exclusive scans of the counts
    int ex = 0;
    if (threadIdx.x < 256) {
      const int v = __ldcg(&w.ghist[p * 256 + threadIdx.x]);
      int incl = v;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int u = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += u;
      }
      if (lane == 31) dsum[warp] = incl;
      ex = incl - v;
    }
    __syncthreads();
    if (threadIdx.x < 256) {
      for (int q = 0; q < warp; ++q) ex += dsum[q];
      dbase[p * 256 + threadIdx.x] = ex;
    }
    __syncthreads();
  }

  for (int p = 0; p < passes; ++p) {
    // pass p reads buffer (p - 1) & 1 and writes buffer p & 1
    const K *kin = (p & 1) ? kb0 : kb1;
    const int *vin = (p & 1) ? vb0 : vb1;
    K *kout = (p & 1) ? kb1 : kb0;
    int *vout = (p & 1) ? vb1 : vb0;
    const bool last = p == passes - 1;
    unsigned *status = w.status + (size_t)p * tiles * 256;
    for (int t = blockIdx.x; t < tiles; t += gridDim.x) {
      // 1. load and rank
      const int i0 = t * RS_TILE + warp * (RS_CPW * 32) + lane;
      K kk[RS_CPW];
      int vv[RS_CPW], rk[RS_CPW], dd[RS_CPW];
#pragma unroll
      for (int r = 0; r < RS_CPW; ++r) {
        const int i = i0 + r * 32;
        const bool ok = i < n;
        kk[r] = ok ? (p == 0 ? src.key(i) : __ldcg(kin + i)) : K(0);
        vv[r] = (VALS && ok) ? (p == 0 ? src.val(i) : __ldcg(vin + i)) : 0;
      }
      for (int d = lane; d < 256; d += 32) my[d] = 0;
      __syncwarp();
#pragma unroll
      for (int r = 0; r < RS_CPW; ++r) {
        const bool ok = i0 + r * 32 < n;
        const int d = ok ? digit_of(kk[r], p) : 256;  // lanes past n: a group of their own
        const unsigned peers = rs_peers(d);
        const int b = ok ? my[d] : 0;
        __syncwarp();
        if (ok && lane == __ffs(peers) - 1) my[d] = b + __popc(peers);
        __syncwarp();
        rk[r] = b + __popc(peers & lt);
        dd[r] = d;
      }
      __syncthreads();
      // 2. warp offsets; the tile's prefix over earlier tiles (look-back)
      if (threadIdx.x < 256) {
        const int d = threadIdx.x;
        int run = 0;
        for (int q = 0; q < RS_WARPS; ++q) {
          const int c = wcnt[q * 256 + d];
          wcnt[q * 256 + d] = run;
          run += c;
        }
        int ex = 0;
        if (t == 0) {
          rs_store(&status[d], RS_INC | unsigned(run));
        } else {
          rs_store(&status[t * 256 + d], RS_AGG | unsigned(run));
          // RS_LB earlier tiles per read (nearest first); an unpublished one
          // is read again; past tile 0 reads as an inclusive 0
          unsigned tries = 0;
          for (int j = t - 1; j >= 0;) {
            unsigned v[RS_LB];
#pragma unroll
            for (int q = 0; q < RS_LB; ++q)
              v[q] = j - q >= 0 ? rs_load(&status[(j - q) * 256 + d]) : RS_INC;
            int q = 0;
            bool done = false;
            for (; q < RS_LB; ++q) {
              if (v[q] == 0) break;
              ex += int(v[q] & RS_VAL);
              if (v[q] & RS_INC) {
                done = true;
                break;
              }
            }
            if (done) break;
            j -= q;
            if (q < RS_LB && ++tries > RS_LOOKBACK_TRIES) {  // never published: give up
              if (w.fail) atomicExch(w.fail, 1);
              break;
            }
          }
          rs_store(&status[t * 256 + d], RS_INC | unsigned(ex + run));
        }
        tofs[d] = dbase[p * 256 + d] + ex;
        // tile positions: exclusive scan of the tile's digit counts
        int incl = run;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int u = __shfl_up_sync(0xffffffffu, incl, o);
          if (lane >= o) incl += u;
        }
        if (lane == 31) dsum[warp] = incl;
        tstart[d] = incl - run;
      }
      __syncthreads();
      if (threadIdx.x < 256)
        for (int q = 0; q < warp; ++q) tstart[threadIdx.x] += dsum[q];
      __syncthreads();
      // 3. the tile in sorted order into shared memory, then out in runs of
      //    one digit (consecutive threads, consecutive positions)
#pragma unroll
      for (int r = 0; r < RS_CPW; ++r) {
        const int d = dd[r];
        if (d >= 256) continue;  // past n
        const int loc = tstart[d] + wcnt[warp * 256 + d] + rk[r];
        sk[loc] = kk[r];
        if (VALS) sv[loc] = vv[r];
      }
      __syncthreads();
      const int tn = min(RS_TILE, n - t * RS_TILE);
      for (int i = threadIdx.x; i < tn; i += RS_THREADS) {
        const K k = sk[i];
        const int v = VALS ? sv[i] : 0;
        const int d = digit_of(k, p);
        const int pos = tofs[d] + (i - tstart[d]);
        if (pos >= n) continue;  // (never: the offsets partition [0, n))
        if (last) {
          emit(pos, k, v, emit.fetch(v));
        } else {
          kout[pos] = k;
          if (VALS) vout[pos] = v;
        }
      }
      __syncthreads();  // wcnt, tofs, tstart and the stage reused by the next tile
    }
    if (!last && !rs_grid_sync(w)) return;
  }
}

// ---- host side ----
// Blocks of one sort launch: one per tile, at most the blocks that fit on
// the GPU at once (a cooperative launch); a single tile runs as one block
// (no barriers).
template <class K, bool VALS>
constexpr size_t radix_stage_bytes() {
  return RS_TILE * (sizeof(K) + (VALS ? sizeof(int) : 0));
}

template <class K, bool VALS, class Kern>
int radix_grid(Kern kern, int64_t n) {
  static const int per_sm = [&] {
    const size_t dyn = radix_stage_bytes<K, VALS>();
    FMMB_CUDA(cudaFuncSetAttribute((const void *)kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   (int)dyn));
    int b = 0;
    FMMB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, kern, RS_THREADS, dyn));
    return b;
  }();
  FMMB_CHECK(per_sm >= 1, ERR_CUDA, "radix sort kernel does not fit on an SM");
  const int64_t tiles = radix_tiles(n);
  if (tiles <= 1) return 1;
  int dev = 0, sms = 0;
  FMMB_CUDA(cudaGetDevice(&dev));
  FMMB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  return (int)std::min<int64_t>(tiles, (int64_t)sms * per_sm);
}

inline size_t rs_round(size_t b) { return (b + 255) & ~size_t(255); }

// Scratch bytes of a sort of n elements over `passes` passes.
template <class K, bool VALS>
size_t radix_scratch_bytes(int64_t n, int passes) {
  size_t b = 0;
  for (int k = 0; k < 2; ++k)
    if (passes >= 2 + k) b += rs_round(n * sizeof(K)) + (VALS ? rs_round(n * sizeof(int)) : 0);
  return b + rs_round(radix_work_bytes(n, passes));
}

// Sort n elements on bits [begin_bit, end_bit) with scratch of
// radix_scratch_bytes<K, VALS>(n, passes) bytes on g = radix_grid(...) blocks.
template <class K, bool VALS, class Src, class Emit>
void radix_sort_run(const Src &src, const Emit &emit, int64_t n, int begin_bit, int end_bit,
                    void *scratch, size_t bytes, int g, int *fail, cudaStream_t s,
                    const unsigned long long *n_dev = nullptr) {
  if (n <= 0) return;
  FMMB_CHECK(end_bit > begin_bit && end_bit <= int(8 * sizeof(K)) && n < (int64_t(1) << 30),
             ERR_INVALID_ARGUMENT, "radix sort: bad bit range or more than 2^30 elements");
  const int passes = (end_bit - begin_bit + 7) / 8;
  FMMB_CHECK((bytes >= radix_scratch_bytes<K, VALS>(n, passes)), ERR_CAPACITY,
             "radix sort: scratch too small");
  unsigned char *at = static_cast<unsigned char *>(scratch);
  K *kb[2] = {nullptr, nullptr};
  int *vb[2] = {nullptr, nullptr};
  for (int k = 0; k < 2; ++k)
    if (passes >= 2 + k) {
      kb[k] = reinterpret_cast<K *>(at);
      at += rs_round(n * sizeof(K));
      if (VALS) {
        vb[k] = reinterpret_cast<int *>(at);
        at += rs_round(n * sizeof(int));
      }
    }
  RadixWork w;
  w.sync = reinterpret_cast<RadixSync *>(at);
  w.ghist = reinterpret_cast<int *>(at + sizeof(RadixSync));
  w.status = reinterpret_cast<unsigned *>(at + sizeof(RadixSync) + sizeof(int) * 256 * passes);
  w.fail = fail;
  w.n_dev = n_dev;
  FMMB_CUDA(cudaMemsetAsync(w.sync, 0, sizeof(RadixSync) + sizeof(int) * 256 * passes, s));
  auto kern = k_radix_sort<K, Src, Emit, VALS>;
  void *args[] = {(void *)&src, (void *)&emit, (void *)&n, (void *)&begin_bit, (void *)&end_bit,
                  (void *)&kb[0], (void *)&vb[0], (void *)&kb[1], (void *)&vb[1], (void *)&w};
  const size_t dyn = radix_stage_bytes<K, VALS>();
  if (g > 1)
    FMMB_CUDA(cudaLaunchCooperativeKernel((const void *)kern, g, RS_THREADS, args, dyn, s));
  else
    FMMB_CUDA(cudaLaunchKernel((const void *)kern, 1, RS_THREADS, args, dyn, s));
}

// The same with scratch from the stream-ordered pool.
template <class K, bool VALS, class Src, class Emit>
void radix_sort(const Src &src, const Emit &emit, int64_t n, int begin_bit, int end_bit, int *fail,
                cudaStream_t s, const unsigned long long *n_dev = nullptr) {
  if (n <= 0) return;
  const int g = radix_grid<K, VALS>(k_radix_sort<K, Src, Emit, VALS>, n);
  const size_t bytes = radix_scratch_bytes<K, VALS>(n, (end_bit - begin_bit + 7) / 8);
  DevBuf<unsigned char> tmp;
  tmp.alloc(bytes, s);
  radix_sort_run<K, VALS>(src, emit, n, begin_bit, end_bit, tmp.get(), bytes, g, fail, s, n_dev);
}

}  // namespace
}  // namespace fmmb
