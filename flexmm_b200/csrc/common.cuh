// Shared definitions for the flexmm_b200 CUDA library (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string>
#include <vector>
#include <stdexcept>

namespace fmmb {

// Status codes returned by every C-ABI entry point (mirrored in include/flexmm_b200.h).
enum Status : int {
  OK = 0,
  ERR_INVALID_ARGUMENT = 1,
  ERR_CUDA = 2,
  ERR_TREE_TOO_DEEP = 3,
  ERR_NOT_READY = 4,
  ERR_UNSUPPORTED = 5,
  ERR_CAPACITY = 6,
};

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string &m) : std::runtime_error(m), code(c) {}
};

#define FMMB_CUDA(call)                                                                  \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess)                                                               \
      throw ::fmmb::Error(::fmmb::ERR_CUDA, std::string(#call) + ": " +                  \
                                                cudaGetErrorString(e_));                 \
  } while (0)

#define FMMB_CHECK(cond, code, msg)                                                      \
  do {                                                                                   \
    if (!(cond)) throw ::fmmb::Error((code), (msg));                                     \
  } while (0)

// Maximum number of quadrant digits in a point key.  A key holds the
// descent decisions of levels 0..MAXD-1, so trees have at most MAXD+1
// levels (0..MAXD).  Box codes pack (level << 58 | morton); bit 63 is free.
constexpr int MAXD = 29;
constexpr int LEVEL_SHIFT = 58;
constexpr uint64_t MORTON_MASK = (uint64_t(1) << LEVEL_SHIFT) - 1;
constexpr uint64_t XLIST_TAG = uint64_t(1) << 63;
constexpr uint64_t EMPTY_SLOT = ~uint64_t(0);

__host__ __device__ inline uint64_t box_code(int level, uint64_t morton) {
  return (uint64_t(level) << LEVEL_SHIFT) | morton;
}
__host__ __device__ inline int code_level(uint64_t c) { return int((c >> LEVEL_SHIFT) & 31); }
__host__ __device__ inline uint64_t code_morton(uint64_t c) { return c & MORTON_MASK; }

// interleaved morton: digit d = 2*xbit + ybit, most significant digit first
__host__ __device__ inline uint64_t morton_of(uint32_t ix, uint32_t iy, int level) {
  uint64_t m = 0;
  for (int l = level - 1; l >= 0; --l)
    m = (m << 2) | (uint64_t((ix >> l) & 1u) << 1) | uint64_t((iy >> l) & 1u);
  return m;
}
__host__ __device__ inline void morton_xy(uint64_t m, int level, uint32_t &ix, uint32_t &iy) {
  ix = 0;
  iy = 0;
  for (int l = level - 1; l >= 0; --l) {
    uint32_t d = uint32_t((m >> (2 * l)) & 3u);
    ix = (ix << 1) | (d >> 1);
    iy = (iy << 1) | (d & 1u);
  }
}

// Stream-ordered device buffer (cudaMallocAsync on the plan's stream; the
// device's default pool keeps freed blocks, so repeated plans reuse memory).
template <class T>
struct DevBuf {
  T *p = nullptr;
  size_t n = 0;
  cudaStream_t s = 0;
  DevBuf() = default;
  DevBuf(const DevBuf &) = delete;
  DevBuf &operator=(const DevBuf &) = delete;
  ~DevBuf() { release(); }
  void release() {
    if (p) cudaFreeAsync(p, s);
    p = nullptr;
    n = 0;
  }
  void alloc(size_t count, cudaStream_t stream) {
    if (count <= n && p) return;
    release();
    s = stream;
    n = count;
    if (count) FMMB_CUDA(cudaMallocAsync((void **)&p, count * sizeof(T), stream));
  }
  void zero(cudaStream_t stream) {
    if (n) FMMB_CUDA(cudaMemsetAsync(p, 0, n * sizeof(T), stream));
  }
  T *get() const { return p; }
};

// Programmatic dependent launch: a kernel launched by launch_pdl may start
// while the kernel before it in the stream is still running.  It must call
// pdl_wait() before it touches anything an earlier kernel writes (after that
// call every earlier kernel has completed and its writes are visible), and
// calls pdl_trigger() only after pdl_wait(), so the kernel after it cannot
// overtake the ones before it.  Without the launch attribute both are no-ops.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() {
  asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
}

template <typename... Params, typename... Args>
void launch_pdl(void (*kernel)(Params...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  FMMB_CUDA(cudaLaunchKernelEx(&cfg, kernel, static_cast<Params>(args)...));
}

// Raise a kernel's dynamic shared-memory limit to at least `bytes` on the
// current device.  The attribute is set once per (kernel, device) and size
// (later calls that need no more are no-ops), so launches inside a CUDA
// graph capture make no attribute calls once the kernel has run before.
void smem_limit_impl(const void *kernel, size_t bytes);
template <class F>
inline void smem_limit(F *kernel, size_t bytes) {
  smem_limit_impl(reinterpret_cast<const void *>(kernel), bytes);
}

// blocks for a persistent or grid-stride kernel over `units` work units (at
// most one block per unit): per_sm blocks per SM on a large problem, fewer
// on a small one (a batch of small problems then does not launch thousands
// of idle blocks per kernel)
inline int work_grid(int64_t units, int per_sm) {
  const int64_t cap = 148 * int64_t(per_sm);
  return int(units < 1 ? 1 : (units < cap ? units : cap));
}

inline int grid_for(int64_t n, int threads, int cap = 148 * 16) {
  int64_t g = (n + threads - 1) / threads;
  if (g < 1) g = 1;
  if (g > cap) g = cap;
  return int(g);
}

}  // namespace fmmb
