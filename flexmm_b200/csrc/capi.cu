// C-ABI entry points (include/flexmm_b200.h): operator sets, plans, passes.
#include <string.h>

#include <algorithm>
#include <cmath>

#include <map>
#include <atomic>
#include <mutex>

#include <memory>
#include <string>
#include <vector>

#include "../../include/flexmm_b200.h"
#include "fmm.cuh"
#include "timing.cuh"

using namespace fmmb;

namespace {
thread_local std::string g_last_error;

int fail(const Error &e) {
  g_last_error = e.what();
  return e.code;
}

template <class F>
int guarded(F &&f) {
  try {
    f();
    return FMM_OK;
  } catch (const Error &e) {
    return fail(e);
  } catch (const std::exception &e) {
    g_last_error = e.what();
    return FMM_ERR_INVALID_ARGUMENT;
  }
}

struct LevelEntry {
  DevBuf<double> buf;
  DevBuf<float> buf32;
  LevelOpsDev dev;
  DevBuf<LevelOpsDev> dev_copy;  // `dev` in device memory, gathered per plan by a kernel
  DevBuf<double> bb_m2l;  // black-box FMM: [np x 40 np], offset blocks side by side
  DevBuf<double> st;      // Stokes FMM: this width's operators (StokesArgs::Level layout)
  StokesArgs::Level st_lev{};
};

// round to TF32 (10 explicit mantissa bits), to nearest, ties away from zero
float tf32_rna(float x) {
  uint32_t u;
  memcpy(&u, &x, 4);
  if ((u & 0x7f800000u) != 0x7f800000u) u += 0x1000u;
  u &= 0xffffe000u;
  float r;
  memcpy(&r, &u, 4);
  return r;
}

int pad8(int n) { return (n + 7) & ~7; }

}  // namespace

void fmmb::smem_limit_impl(const void *kernel, size_t bytes) {
  static std::mutex mu;
  static std::map<std::pair<const void *, int>, size_t> done;
  int dev = 0;
  FMMB_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> g(mu);
  size_t &have = done[{kernel, dev}];
  if (have >= bytes) return;
  FMMB_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes)));
  have = bytes;
}

namespace {

// sqrt(x) e^x K_n(x), n = 0, 1, for x >= 1: trapezoidal rule on
// int_0^inf exp(-2x sinh^2(t/2)) cosh^n(t) dt (exponent without cancellation;
// step below the integrand's width 1/sqrt(x); summed from the small terms up)
double bessel_g_host(int n, double x) {
  const double h = std::min(1.0 / 16.0, 0.2 / std::sqrt(x));
  const int m = (int)std::ceil(std::acosh(1.0 + 60.0 / x) / h);
  double s = 0.0;
  for (int i = m; i >= 1; --i) {
    const double t = i * h, sh = std::sinh(0.5 * t);
    s += std::exp(-2.0 * x * sh * sh) * (n ? std::cosh(t) : 1.0);
  }
  s += 0.5;  // t = 0
  return std::sqrt(x) * h * s;
}

// Chebyshev coefficients of g_0, g_1 on the octaves [2^j, 2^(j+1)) (bessel.cuh)
const std::vector<double> &bessel_table_host() {
  static const std::vector<double> tab = [] {
    std::vector<double> t(BESSEL_TABLE_DOUBLES);
    const int N = BESSEL_NCHEB;
    for (int n = 0; n < 2; ++n)
      for (int j = 0; j < BESSEL_OCTAVES; ++j) {
        const double a = std::ldexp(1.0, j);
        double f[BESSEL_NCHEB];
        for (int k = 0; k < N; ++k)
          f[k] = bessel_g_host(n, 1.5 * a + 0.5 * a * std::cos(M_PI * (k + 0.5) / N));
        for (int i = 0; i < N; ++i) {
          double c = 0.0;
          for (int k = 0; k < N; ++k) c += f[k] * std::cos(M_PI * i * (k + 0.5) / N);
          t[(n * BESSEL_OCTAVES + j) * N + i] = (i == 0 ? 1.0 : 2.0) * c / N;
        }
      }
    return t;
  }();
  return tab;
}

// the Bessel tables on the current device (uploaded once per device, kept
// until exit)
const double *bessel_table_device() {
  static std::mutex mu;
  static std::map<int, double *> per_device;
  int dev = 0;
  FMMB_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> g(mu);
  auto it = per_device.find(dev);
  if (it != per_device.end()) return it->second;
  const std::vector<double> &h = bessel_table_host();
  double *d = nullptr;
  FMMB_CUDA(cudaMalloc((void **)&d, h.size() * sizeof(double)));
  FMMB_CUDA(cudaMemcpy(d, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice));
  per_device[dev] = d;
  return d;
}

// tabulated radial kernels registered by fmm_kernel_table_create: host
// coefficients plus their per-device copies (kept until exit)
struct RadialTable {
  int j0, noct, ncheb;
  std::vector<double> coef;
  std::map<int, double *> dev;
};
std::mutex g_tables_mu;
std::vector<std::unique_ptr<RadialTable>> g_tables;

bool kernel_known(int kernel_id) {
  return kernel_id == KERNEL_LAPLACE || kernel_id == KERNEL_MOD_HELMHOLTZ ||
         kernel_id == KERNEL_RADIAL_TABLE;
}

// a kernel's device parameters: the caller's values plus the tables it reads
KernelParams kernel_params(int kernel_id, const double *kparams) {
  KernelParams kp{};
  for (int i = 0; i < 4; ++i) kp.p[i] = kparams ? kparams[i] : 0.0;
  kp.table = nullptr;
  if (kernel_id == KERNEL_MOD_HELMHOLTZ) {
    FMMB_CHECK(kp.p[0] > 0.0, ERR_INVALID_ARGUMENT, "modified Helmholtz needs k = kparams[0] > 0");
    kp.table = bessel_table_device();
  }
  if (kernel_id == KERNEL_RADIAL_TABLE) {
    std::lock_guard<std::mutex> g(g_tables_mu);
    const int id = int(kp.p[0]);
    FMMB_CHECK(kp.p[0] == double(id) && id >= 0 && id < (int)g_tables.size() && g_tables[id],
               ERR_INVALID_ARGUMENT, "kparams[0] is not a table id from fmm_kernel_table_create");
    RadialTable &t = *g_tables[id];
    int dev = 0;
    FMMB_CUDA(cudaGetDevice(&dev));
    if (!t.dev.count(dev)) {
      double *d = nullptr;
      FMMB_CUDA(cudaMalloc((void **)&d, t.coef.size() * sizeof(double)));
      FMMB_CUDA(cudaMemcpy(d, t.coef.data(), t.coef.size() * sizeof(double), cudaMemcpyHostToDevice));
      t.dev[dev] = d;
    }
    kp.table = t.dev[dev];
    kp.p[1] = t.j0;
    kp.p[2] = t.noct;
    kp.p[3] = t.ncheb;
  }
  return kp;
}

bool kernel_scaled(int kernel_id) {
  switch (kernel_id) {
    case KERNEL_LAPLACE: return LaplaceF32::kScaled;
    default: return false;
  }
}

// kernels with an FP32 form for the mixed passes
bool kernel_mixed(int kernel_id) {
  return kernel_id == KERNEL_LAPLACE || kernel_id == KERNEL_MOD_HELMHOLTZ;
}

double kernel_offset(int kernel_id, const KernelParams &kp, double w) {
  switch (kernel_id) {
    case KERNEL_LAPLACE: return LaplaceF32::offset(w, kp);
    default: return 0.0;
  }
}

// Keep freed stream-ordered allocations in this process's default pool, so
// that plans created repeatedly reuse device memory instead of returning it
// to the driver at every synchronisation.
void retain_pool_memory() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return;
  static thread_local int done_for = -1;
  if (done_for == dev) return;
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
    uint64_t keep = ~uint64_t(0);
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    // headroom reserved once: plans built while earlier ones are still
    // queued (a host running steps ahead) then take memory the pool already
    // maps, instead of mapping more in the middle of a step (milliseconds)
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess) {
      const size_t want = std::min<size_t>(size_t(1) << 30, free_b / 8);
      void *p = nullptr;
      if (want > 0 && cudaMallocAsync(&p, want, 0) == cudaSuccess) {
        cudaFreeAsync(p, 0);
        cudaStreamSynchronize(0);
      }
    }
  }
  done_for = dev;
}
}  // namespace

constexpr int METHOD_KIFMM = 0, METHOD_BBFMM = 1, METHOD_STOKES = 2;

struct fmm_ops {
  int kernel_id;
  KernelParams kp;
  int neq, np;
  int method = METHOD_KIFMM;
  int p = 0;                  // black-box FMM: Chebyshev order
  DevBuf<double> bb_m2mc;     // black-box FMM: M2MC [np x 4np]
  DevBuf<double> bb_m2mct;    // and its transpose [4np x np]
  std::vector<std::unique_ptr<LevelEntry>> levels;
};

struct fmm_plan {
  fmm_ops *ops;
  cudaStream_t stream;
  TreeDev td;
  TreeHost th;
  std::vector<int> bound;  // per level: ops entry id or -1
  DevBuf<LevelOpsDev> ops_dev;
  DevBuf<double> tau_s, mult, ple, loc;
  DevBuf<float> mult32, loc32;  // mixed precision: FP32 expansions ...
  DevBuf<float> mult_tc;        // ... multipoles split TF32 hi / lo ...
  DevBuf<double> msum, lsum;    // ... and their FP64 component sums
  DevBuf<double> tsum;          // per node: FP64 sum of its charges
  DevBuf<int> err;              // set by kernels whose bounded waits ran out
  int precision = PREC_FP64;
  bool have_expansions = false;
  DevBuf<double> tau2_s, partial;  // Stokes FMM: sorted fy; partial multipoles
  int n_rhs = 1;                   // charge columns of the last build (multi-RHS)
  // split own-source evaluation (near field on a side stream, see SplitEval):
  // `ready` is recorded once a single-column KIFMM build has sorted its charges
  DevBuf<double> dvx, dvy;  // dipole sources: strength * normal, sorted (see PassArgs)
  bool has_dipoles = false;
  DevBuf<double> st_dip;    // Stokes stresslets: sigma_x, sigma_y, n_x, n_y, sorted ([4][n])
  bool has_st_dipoles = false;
  cudaStream_t side = nullptr;  // from the device's pool, not owned
  cudaEvent_t ev_ready = nullptr, ev_near = nullptr, ev_far = nullptr;
  bool ready_recorded = false;
  // mixed form: the split near field pauses during the M2L (SplitEval::hold)
  cudaEvent_t ev_m2l = nullptr;
  DevBuf<int> near_hold;
  bool hold_armed = false;
  ~fmm_plan() {
    for (cudaEvent_t e : {ev_ready, ev_near, ev_far, ev_m2l})
      if (e) cudaEventDestroy(e);
  }
};

namespace {
// Side streams for the split evaluation: a few non-blocking streams per
// device, handed to plans round-robin (created once, kept until exit).
constexpr int SIDE_STREAMS = 8;
constexpr int SIDE_MAX_DEVICES = 64;
std::mutex g_side_mu;
cudaStream_t g_side[SIDE_MAX_DEVICES][SIDE_STREAMS] = {};
int g_side_next[SIDE_MAX_DEVICES] = {};

cudaStream_t side_stream() {
  int dev = 0;
  FMMB_CUDA(cudaGetDevice(&dev));
  FMMB_CHECK(dev >= 0 && dev < SIDE_MAX_DEVICES, ERR_UNSUPPORTED, "device ordinal too large");
  std::lock_guard<std::mutex> g(g_side_mu);
  if (!g_side[dev][0])  // all at once: no plan after the first pays for a stream
    for (int k = 0; k < SIDE_STREAMS; ++k)
      FMMB_CUDA(cudaStreamCreateWithFlags(&g_side[dev][k], cudaStreamNonBlocking));
  return g_side[dev][g_side_next[dev]++ % SIDE_STREAMS];
}

// Whether own-source evaluation runs split (near field beside the level
// passes).  Measured at 1M clustered sources: the FP64 form gains ~0.6 ms
// (its level passes are DMMA tiles that share SMs well); the mixed form,
// whose near field pauses while the persistent tcgen05 M2L runs, gains
// ~0.03 ms (1.39 -> 1.36 ms).  On for both by default;
// FLEXMM_B200_SPLIT_EVAL=0 turns it off, =1 on.
std::atomic<int> g_split_mode{-2};  // -2: not yet read from the environment

bool split_enabled(int precision) {
  int mode = g_split_mode.load(std::memory_order_relaxed);
  if (mode == -2) {
    const char *e = getenv("FLEXMM_B200_SPLIT_EVAL");
    int env = e ? (e[0] == '0' ? 0 : 1) : -1;
    g_split_mode.compare_exchange_strong(mode, env);
    mode = g_split_mode.load(std::memory_order_relaxed);
  }
  (void)precision;  // the same default for both forms
  return mode < 0 || mode == 1;
}

// the plan's split-evaluation events (created on first use) and side stream
void split_prepare(fmm_plan *p) {
  if (!p->side) p->side = side_stream();
  for (cudaEvent_t *e : {&p->ev_ready, &p->ev_near, &p->ev_far, &p->ev_m2l})
    if (!*e) FMMB_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
}

// Zeroes up to 8 device buffers in one launch (instead of one memset each:
// at the start of build_expansions these sit between the tree and the first
// pass, where every launch's host and GPU overhead is on the critical path)
struct ZeroList {
  unsigned char *p[8];
  size_t bytes[8];
  int n;
};

__global__ void k_zero_buffers(ZeroList z) {
  const size_t tid = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  const size_t nthr = (size_t)gridDim.x * blockDim.x;
  for (int b = 0; b < z.n; ++b) {
    const size_t n16 = z.bytes[b] / 16;  // buffers are 16-byte aligned (checked by the host)
    uint4 *w = reinterpret_cast<uint4 *>(z.p[b]);
    for (size_t i = tid; i < n16; i += nthr) w[i] = make_uint4(0u, 0u, 0u, 0u);
    for (size_t i = 16 * n16 + tid; i < z.bytes[b]; i += nthr) z.p[b][i] = 0;
  }
}

class ZeroBatch {
 public:
  explicit ZeroBatch(cudaStream_t s) : s_(s) {}
  template <class T>
  ZeroBatch &add(DevBuf<T> &b) {
    if (!b.n) return *this;
    if (z_.n == 8 || (reinterpret_cast<uintptr_t>(b.get()) & 15)) {
      b.zero(s_);
      return *this;
    }
    z_.p[z_.n] = reinterpret_cast<unsigned char *>(b.get());
    z_.bytes[z_.n++] = b.n * sizeof(T);
    return *this;
  }
  void run() {
    if (!z_.n) return;
    size_t total = 0;
    for (int i = 0; i < z_.n; ++i) total += z_.bytes[i];
    int dev = 0, sms = 0;
    FMMB_CUDA(cudaGetDevice(&dev));
    FMMB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int blocks = (int)std::min<size_t>(size_t(sms) * 8, std::max<size_t>(1, total / 4096));
    k_zero_buffers<<<blocks, 256, 0, s_>>>(z_);
    FMMB_CUDA(cudaGetLastError());
    z_.n = 0;
  }

 private:
  cudaStream_t s_;
  ZeroList z_{};
};
}  // namespace

extern "C" {

const char *fmm_last_error(void) { return g_last_error.c_str(); }

int fmm_ops_create(int kernel_id, const double *kparams, int nequiv, fmm_ops **out) {
  return guarded([&] {
    FMMB_CHECK(out, ERR_INVALID_ARGUMENT, "out is NULL");
    FMMB_CHECK(kernel_known(kernel_id), ERR_UNSUPPORTED, "unknown kernel id");
    FMMB_CHECK(nequiv >= 1 && nequiv <= FMM_MAX_NEQUIV, ERR_INVALID_ARGUMENT,
               "nequiv must be in [1, 64]");
    const KernelParams kp = kernel_params(kernel_id, kparams);
    auto *o = new fmm_ops();
    o->kernel_id = kernel_id;
    o->kp = kp;
    o->neq = nequiv;
    o->np = pad8(nequiv);
    *out = o;
  });
}

int fmm_ops_add(fmm_ops *ops, const fmm_level_ops *lv, int *level_id) {
  return guarded([&] {
    FMMB_CHECK(ops && lv && level_id, ERR_INVALID_ARGUMENT, "NULL argument");
    FMMB_CHECK(ops->method == METHOD_KIFMM, ERR_INVALID_ARGUMENT,
               "black-box and Stokes operator sets take fmm_bb_ops_add / fmm_stokes_ops_add");
    const int n = ops->neq, np = ops->np;
    // host staging in the padded device layout
    std::vector<double> h;
    auto take = [&](size_t count) {
      size_t at = h.size();
      h.resize(at + ((count + 1) & ~size_t(1)), 0.0);  // keep 16-byte alignment
      return at;
    };
    const size_t o_lx = take(np), o_ly = take(np), o_u = take(size_t(np) * np), o_s = take(np),
                 o_vh = take(size_t(np) * np), o_m2mct = take(size_t(4) * np * np),
                 o_m2mc = take(size_t(4) * np * np);
    for (int k = 0; k < n; ++k) {
      h[o_lx + k] = lv->large_x[k];
      h[o_ly + k] = lv->large_y[k];
      h[o_s + k] = lv->c2e_sinv[k];
    }
    for (int i = 0; i < n; ++i)
      for (int k = 0; k < n; ++k) {
        h[o_u + size_t(i) * np + k] = lv->c2e_u[size_t(i) * n + k];
        h[o_vh + size_t(i) * np + k] = lv->c2e_vh[size_t(i) * n + k];
      }
    for (int i = 0; i < n; ++i)
      for (int c = 0; c < 4; ++c)
        for (int k = 0; k < n; ++k) {
          const double v = lv->m2mc[size_t(i) * 4 * n + c * n + k];
          h[o_m2mct + size_t(c * np + k) * np + i] = v;   // [4np x np]
          h[o_m2mc + size_t(i) * 4 * np + c * np + k] = v;  // [np x 4np]
        }
    size_t o_m2l[FMM_N_OFFSETS];
    int kind[FMM_N_OFFSETS], rp[FMM_N_OFFSETS];
    for (int o = 0; o < FMM_N_OFFSETS; ++o) {
      const int r = lv->m2l_rank[o];
      o_m2l[o] = 0;
      rp[o] = 0;
      if (r == 0) {
        kind[o] = M2L_NULL;
      } else if (r < 0) {
        kind[o] = M2L_DENSE;
        o_m2l[o] = take(size_t(np) * np);
        const double *a = lv->m2l_a[o];  // [n x n] (out i, in k); store D^T [k][i]
        for (int i = 0; i < n; ++i)
          for (int k = 0; k < n; ++k) h[o_m2l[o] + size_t(k) * np + i] = a[size_t(i) * n + k];
      } else {
        FMMB_CHECK(r <= n, ERR_INVALID_ARGUMENT, "M2L rank exceeds nequiv");
        kind[o] = M2L_SVD;
        const int p = pad8(r);
        rp[o] = p;
        o_m2l[o] = take(size_t(np) * p + size_t(p) * np);
        const double *m2 = lv->m2l_a[o];  // [n x r]
        const double *m1 = lv->m2l_b[o];  // [r x n]
        for (int q = 0; q < r; ++q)
          for (int k = 0; k < n; ++k) h[o_m2l[o] + size_t(k) * p + q] = m1[size_t(q) * n + k];
        const size_t base2 = o_m2l[o] + size_t(np) * p;
        for (int i = 0; i < n; ++i)
          for (int q = 0; q < r; ++q) h[base2 + size_t(q) * np + i] = m2[size_t(i) * r + q];
      }
    }
    // mixed precision: dense operators minus their mean, as TF32 hi + lo
    std::vector<float> f;
    auto takef = [&](size_t count) {
      size_t at = f.size();
      f.resize(at + ((count + 3) & ~size_t(3)), 0.f);  // 16-byte aligned blocks
      return at;
    };
    auto split = [&](double v, size_t hi_at, size_t lo_at) {
      const float hi = tf32_rna((float)v);
      f[hi_at] = hi;
      f[lo_at] = tf32_rna((float)(v - (double)hi));
    };
    // FP32 evaluations of scale-invariant kernels work in width units
    const bool scaled = kernel_scaled(ops->kernel_id);
    FMMB_CHECK(!scaled || lv->width > 0, ERR_INVALID_ARGUMENT, "level width must be positive");
    const double inv_w = scaled ? 1.0 / lv->width : 1.0;
    const size_t f_lx = takef(np), f_ly = takef(np);
    for (int k = 0; k < n; ++k) {
      f[f_lx + k] = (float)(lv->large_x[k] * inv_w);
      f[f_ly + k] = (float)(lv->large_y[k] * inv_w);
    }
    double c_m2m = 0.0;
    for (size_t i = 0; i < size_t(n) * 4 * n; ++i) c_m2m += lv->m2mc[i];
    c_m2m /= double(n) * 4 * n;
    const size_t f_m2mct_h = takef(size_t(4) * np * np), f_m2mct_l = takef(size_t(4) * np * np);
    const size_t f_m2mc_h = takef(size_t(4) * np * np), f_m2mc_l = takef(size_t(4) * np * np);
    for (int i = 0; i < n; ++i)
      for (int c = 0; c < 4; ++c)
        for (int k = 0; k < n; ++k) {
          const double v = lv->m2mc[size_t(i) * 4 * n + c * n + k] - c_m2m;
          const size_t t1 = size_t(c * np + k) * np + i, t2 = size_t(i) * 4 * np + c * np + k;
          split(v, f_m2mct_h + t1, f_m2mct_l + t1);
          split(v, f_m2mc_h + t2, f_m2mc_l + t2);
        }
    size_t f_m2l_h[FMM_N_OFFSETS], f_m2l_l[FMM_N_OFFSETS];
    size_t f_tc_h[FMM_N_OFFSETS], f_tc_l[FMM_N_OFFSETS];
    const int ntc = (np + 15) & ~15;  // tensor-core N: multiple of 16
    double c_m2l[FMM_N_OFFSETS];
    std::vector<double> dense(size_t(n) * n);
    for (int o = 0; o < FMM_N_OFFSETS; ++o) {
      const int r = lv->m2l_rank[o];
      c_m2l[o] = 0.0;
      f_m2l_h[o] = f_m2l_l[o] = f_tc_h[o] = f_tc_l[o] = 0;
      if (r == 0) continue;
      if (r < 0) {
        for (size_t i = 0; i < size_t(n) * n; ++i) dense[i] = lv->m2l_a[o][i];
      } else {  // the truncated operator M2 . M1, as the reference applies it
        for (int i = 0; i < n; ++i)
          for (int k = 0; k < n; ++k) {
            double acc = 0.0;
            for (int q = 0; q < r; ++q) acc += lv->m2l_a[o][size_t(i) * r + q] * lv->m2l_b[o][size_t(q) * n + k];
            dense[size_t(i) * n + k] = acc;
          }
      }
      double c = 0.0;
      for (size_t i = 0; i < size_t(n) * n; ++i) c += dense[i];
      c /= double(n) * n;
      c_m2l[o] = c;
      f_m2l_h[o] = takef(size_t(np) * np);
      f_m2l_l[o] = takef(size_t(np) * np);
      f_tc_h[o] = takef(size_t(ntc) * np);
      f_tc_l[o] = takef(size_t(ntc) * np);
      for (int i = 0; i < n; ++i)
        for (int k = 0; k < n; ++k) {
          const size_t t = size_t(k) * np + i;  // B layout [K = source comp][N = target comp]
          split(dense[size_t(i) * n + k] - c, f_m2l_h[o] + t, f_m2l_l[o] + t);
          const size_t u = size_t(i) * np + k;  // tcgen05 B: N x K, K-major
          split(dense[size_t(i) * n + k] - c, f_tc_h[o] + u, f_tc_l[o] + u);
        }
    }
    auto e = std::make_unique<LevelEntry>();
    e->buf32.alloc(f.size(), 0);
    FMMB_CUDA(cudaMemcpy(e->buf32.get(), f.data(), f.size() * sizeof(float), cudaMemcpyHostToDevice));
    {
      float *fb = e->buf32.get();
      e->dev.lx32 = fb + f_lx;
      e->dev.ly32 = fb + f_ly;
      e->dev.m2mct_hi = fb + f_m2mct_h;
      e->dev.m2mct_lo = fb + f_m2mct_l;
      e->dev.m2mc_hi = fb + f_m2mc_h;
      e->dev.m2mc_lo = fb + f_m2mc_l;
      e->dev.c_m2m = c_m2m;
      e->dev.inv_w = inv_w;
      e->dev.kofs = scaled ? kernel_offset(ops->kernel_id, ops->kp, lv->width) : 0.0;
      for (int o = 0; o < FMM_N_OFFSETS; ++o) {
        e->dev.m2l_hi[o] = lv->m2l_rank[o] == 0 ? nullptr : fb + f_m2l_h[o];
        e->dev.m2l_lo[o] = lv->m2l_rank[o] == 0 ? nullptr : fb + f_m2l_l[o];
        e->dev.m2l_tc_hi[o] = lv->m2l_rank[o] == 0 ? nullptr : fb + f_tc_h[o];
        e->dev.m2l_tc_lo[o] = lv->m2l_rank[o] == 0 ? nullptr : fb + f_tc_l[o];
        e->dev.c_m2l[o] = c_m2l[o];
      }
    }
    e->buf.alloc(h.size(), 0);
    FMMB_CUDA(cudaMemcpy(e->buf.get(), h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice));
    double *b = e->buf.get();
    e->dev.lx = b + o_lx;
    e->dev.ly = b + o_ly;
    e->dev.u = b + o_u;
    e->dev.sinv = b + o_s;
    e->dev.vh = b + o_vh;
    e->dev.m2mct = b + o_m2mct;
    e->dev.m2mc = b + o_m2mc;
    for (int o = 0; o < FMM_N_OFFSETS; ++o) {
      e->dev.m2l[o] = kind[o] == M2L_NULL ? nullptr : b + o_m2l[o];
      e->dev.kind[o] = kind[o];
      e->dev.rp[o] = rp[o];
    }
    e->dev_copy.alloc(1, 0);
    FMMB_CUDA(cudaMemcpy(e->dev_copy.get(), &e->dev, sizeof(LevelOpsDev), cudaMemcpyHostToDevice));
    ops->levels.push_back(std::move(e));
    *level_id = int(ops->levels.size()) - 1;
  });
}

int fmm_bb_ops_create(int kernel_id, const double *kparams, int p, const double *m2mc,
                      fmm_ops **out) {
  return guarded([&] {
    FMMB_CHECK(out && m2mc, ERR_INVALID_ARGUMENT, "NULL argument");
    FMMB_CHECK(kernel_known(kernel_id), ERR_UNSUPPORTED, "unknown kernel id");
    FMMB_CHECK(p >= 2 && p <= FMM_BB_MAX_P, ERR_INVALID_ARGUMENT, "p must be in [2, 16]");
    const KernelParams kp = kernel_params(kernel_id, kparams);
    const int n = p * p, np = pad8(n);
    std::vector<double> h(size_t(np) * 4 * np, 0.0);
    for (int i = 0; i < n; ++i)
      for (int c = 0; c < 4; ++c)
        for (int k = 0; k < n; ++k) h[size_t(i) * 4 * np + c * np + k] = m2mc[size_t(i) * 4 * n + c * n + k];
    auto o = std::make_unique<fmm_ops>();
    o->kernel_id = kernel_id;
    o->kp = kp;
    o->neq = n;
    o->np = np;
    o->method = METHOD_BBFMM;
    o->p = p;
    o->bb_m2mc.alloc(h.size(), 0);
    FMMB_CUDA(cudaMemcpy(o->bb_m2mc.get(), h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice));
    std::vector<double> ht(h.size(), 0.0);  // [4np x np]: the M2M row GEMM's operator
    for (int i = 0; i < np; ++i)
      for (int k = 0; k < 4 * np; ++k) ht[size_t(k) * np + i] = h[size_t(i) * 4 * np + k];
    o->bb_m2mct.alloc(ht.size(), 0);
    FMMB_CUDA(cudaMemcpy(o->bb_m2mct.get(), ht.data(), ht.size() * sizeof(double),
                         cudaMemcpyHostToDevice));
    *out = o.release();
  });
}

int fmm_bb_ops_add(fmm_ops *ops, const fmm_bb_level_ops *lv, int *level_id) {
  return guarded([&] {
    FMMB_CHECK(ops && lv && level_id && lv->m2l_rank, ERR_INVALID_ARGUMENT, "NULL argument");
    FMMB_CHECK(ops->method == METHOD_BBFMM, ERR_INVALID_ARGUMENT,
               "fmm_bb_ops_add needs a black-box operator set (fmm_bb_ops_create)");
    const int n = ops->neq, np = ops->np;
    const size_t ld = size_t(N_OFFSETS) * np;
    std::vector<double> h(size_t(np) * ld, 0.0);
    for (int o = 0; o < N_OFFSETS; ++o) {
      const int r = lv->m2l_rank[o];
      if (r == 0) continue;
      FMMB_CHECK(lv->m2l_a[o], ERR_INVALID_ARGUMENT, "missing M2L operator");
      // stored transposed, [40 np x np]: row o np + k holds column k of
      // offset o's operator (the M2L row GEMM's W)
      if (r < 0) {  // dense [n x n]
        for (int i = 0; i < n; ++i)
          for (int k = 0; k < n; ++k) h[(size_t(o) * np + k) * np + i] = lv->m2l_a[o][size_t(i) * n + k];
      } else {  // the truncated operator M2 . M1 ([n x r] . [r x n]), as the reference applies it
        FMMB_CHECK(r <= n && lv->m2l_b[o], ERR_INVALID_ARGUMENT, "bad M2L factors");
        for (int i = 0; i < n; ++i)
          for (int k = 0; k < n; ++k) {
            double acc = 0.0;
            for (int q = 0; q < r; ++q) acc += lv->m2l_a[o][size_t(i) * r + q] * lv->m2l_b[o][size_t(q) * n + k];
            h[(size_t(o) * np + k) * np + i] = acc;
          }
      }
    }
    auto e = std::make_unique<LevelEntry>();
    e->dev.inv_w = 1.0 / lv->width;
    e->bb_m2l.alloc(h.size(), 0);
    FMMB_CUDA(cudaMemcpy(e->bb_m2l.get(), h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice));
    ops->levels.push_back(std::move(e));
    *level_id = int(ops->levels.size()) - 1;
  });
}

int fmm_kernel_table_create(const double *coef, int j0, int n_octaves, int n_cheb, int *table_id) {
  return guarded([&] {
    FMMB_CHECK(coef && table_id, ERR_INVALID_ARGUMENT, "NULL argument");
    FMMB_CHECK(n_octaves >= 1 && n_octaves <= 2048 && n_cheb >= 1 && n_cheb <= 64, ERR_INVALID_ARGUMENT,
               "table size out of range");
    FMMB_CHECK(j0 >= -1000 && j0 + n_octaves <= 1000, ERR_INVALID_ARGUMENT, "octave range out of range");
    auto t = std::make_unique<RadialTable>();
    t->j0 = j0;
    t->noct = n_octaves;
    t->ncheb = n_cheb;
    t->coef.assign(coef, coef + size_t(n_octaves) * n_cheb);
    for (double v : t->coef) FMMB_CHECK(std::isfinite(v), ERR_INVALID_ARGUMENT, "non-finite coefficient");
    std::lock_guard<std::mutex> g(g_tables_mu);
    g_tables.push_back(std::move(t));
    *table_id = int(g_tables.size()) - 1;
  });
}

int fmm_stokes_ops_create(int nequiv, fmm_ops **out) {
  return guarded([&] {
    FMMB_CHECK(out, ERR_INVALID_ARGUMENT, "NULL argument");
    FMMB_CHECK(nequiv >= 1 && nequiv <= FMM_MAX_NEQUIV, ERR_INVALID_ARGUMENT, "nequiv must be in [1, 64]");
    auto o = std::make_unique<fmm_ops>();
    o->kernel_id = -1;
    o->kp = KernelParams{};
    o->neq = nequiv;
    o->np = pad8(2 * nequiv + 1);
    o->method = METHOD_STOKES;
    *out = o.release();
  });
}

int fmm_stokes_ops_add(fmm_ops *ops, const fmm_stokes_level_ops *lv, int *level_id) {
  return guarded([&] {
    FMMB_CHECK(ops && lv && level_id && lv->m2l_rank, ERR_INVALID_ARGUMENT, "NULL argument");
    FMMB_CHECK(ops->method == METHOD_STOKES, ERR_INVALID_ARGUMENT,
               "fmm_stokes_ops_add needs a Stokes operator set (fmm_stokes_ops_create)");
    const int neq = ops->neq, n1 = 2 * neq + 1, n2 = 2 * neq, np = ops->np;
    const size_t sq = size_t(np) * np, ld = size_t(N_OFFSETS) * np;
    std::vector<double> h;
    auto take = [&](size_t count) {
      size_t at = h.size();
      h.resize(at + ((count + 1) & ~size_t(1)), 0.0);  // 16-byte aligned blocks
      return at;
    };
    const size_t o_lx = take(neq), o_ly = take(neq);
    const size_t o_eu = take(sq), o_ev = take(sq), o_cu = take(sq), o_cv = take(sq);
    const size_t o_mm = take(4 * sq), o_ll = take(4 * sq), o_cat = take(size_t(np) * ld);
    for (int k = 0; k < neq; ++k) {
      h[o_lx + k] = lv->large_x[k];
      h[o_ly + k] = lv->large_y[k];
    }
    // x = (b . U) . (diag(1/S) VH); the C2E solve drops the extra unknown (column n2)
    auto solve = [&](const double *u, const double *sinv, const double *vh, size_t ou, size_t ov,
                     bool drop_extra) {
      for (int i = 0; i < n1; ++i)
        for (int j = 0; j < n1; ++j) {
          h[ou + size_t(i) * np + j] = u[size_t(i) * n1 + j];
          if (!(drop_extra && j == n2)) h[ov + size_t(i) * np + j] = sinv[i] * vh[size_t(i) * n1 + j];
        }
    };
    solve(lv->e2c_u, lv->e2c_sinv, lv->e2c_vh, o_eu, o_ev, false);
    solve(lv->c2e_u, lv->c2e_sinv, lv->c2e_vh, o_cu, o_cv, true);
    for (int i = 0; i < n1; ++i)
      for (int c = 0; c < 4; ++c)
        for (int k = 0; k < n2; ++k) {
          h[o_mm + size_t(c * np + k) * np + i] = lv->m2mc[size_t(i) * 4 * n2 + c * n2 + k];
          h[o_ll + size_t(k) * 4 * np + c * np + i] = lv->l2lc[size_t(c * n1 + i) * n2 + k];
        }
    for (int o = 0; o < N_OFFSETS; ++o) {
      const int r = lv->m2l_rank[o];
      if (r == 0) continue;
      FMMB_CHECK(lv->m2l_a[o], ERR_INVALID_ARGUMENT, "missing M2L operator");
      for (int i = 0; i < n1; ++i)
        for (int k = 0; k < n2; ++k) {
          double v;
          if (r < 0) {
            v = lv->m2l_a[o][size_t(i) * n2 + k];
          } else {  // M2 [n1 x r] . M1 [r x n2], the reference's truncated operator
            FMMB_CHECK(lv->m2l_b[o], ERR_INVALID_ARGUMENT, "bad M2L factors");
            v = 0.0;
            for (int q = 0; q < r; ++q) v += lv->m2l_a[o][size_t(i) * r + q] * lv->m2l_b[o][size_t(q) * n2 + k];
          }
          h[o_cat + (size_t(o) * np + k) * np + i] = v;  // transposed [40 np x np]
        }
    }
    auto e = std::make_unique<LevelEntry>();
    e->st.alloc(h.size(), 0);
    FMMB_CUDA(cudaMemcpy(e->st.get(), h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice));
    double *b = e->st.get();
    e->st_lev = StokesArgs::Level{b + o_lx, b + o_ly, b + o_eu, b + o_ev, b + o_cu,
                                  b + o_cv, b + o_mm, b + o_ll, b + o_cat};
    e->dev.inv_w = 1.0 / lv->width;
    ops->levels.push_back(std::move(e));
    *level_id = int(ops->levels.size()) - 1;
  });
}

int fmm_ops_destroy(fmm_ops *ops) {
  return guarded([&] {
    if (!ops) return;
    cudaDeviceSynchronize();
    delete ops;
  });
}

// the tree's host-side level offsets: build_tree returns before they arrive
static void tree_ready(fmm_plan *p) {
  if (p) finalize_tree(p->th);
}

int fmm_plan_create(fmm_ops *ops, const double *x, const double *y, int64_t n, int ncutoff,
                    const double *bbox, void *stream, fmm_plan **out) {
  return guarded([&] {
    FMMB_CHECK(ops && x && y && bbox && out, ERR_INVALID_ARGUMENT, "NULL argument");
    retain_pool_memory();
    auto p = std::make_unique<fmm_plan>();
    p->ops = ops;
    p->stream = (cudaStream_t)stream;
    {
      PhaseTimer timer(PH_TREE, p->stream);
      build_tree(p->td, p->th, x, y, n, ncutoff, bbox, p->stream);
    }
    p->bound.assign(p->th.L, -1);
    *out = p.release();
  });
}

int fmm_plan_info(fmm_plan *p, int *n_levels, double *widths, int *n_nodes) {
  return guarded([&] {
    FMMB_CHECK(p, ERR_INVALID_ARGUMENT, "plan is NULL");
    if (n_nodes) tree_ready(p);  // level counts need the finished tree; L and widths do not
    if (n_levels) *n_levels = p->th.L;
    for (int m = 0; m < p->th.L; ++m) {
      if (widths) widths[m] = p->th.width[m];
      if (n_nodes) n_nodes[m] = p->th.off[m + 1] - p->th.off[m];
    }
  });
}

int fmm_plan_set_precision(fmm_plan *p, int precision) {
  return guarded([&] {
    FMMB_CHECK(p, ERR_INVALID_ARGUMENT, "plan is NULL");
    FMMB_CHECK(precision == PREC_FP64 || precision == PREC_MIXED, ERR_INVALID_ARGUMENT,
               "precision must be FMM_PRECISION_FP64 or FMM_PRECISION_MIXED");
    FMMB_CHECK(precision == PREC_FP64 || kernel_mixed(p->ops->kernel_id), ERR_UNSUPPORTED,
               "the mixed form needs a kernel with an FP32 form (Laplace, modified Helmholtz)");
    FMMB_CHECK(precision == PREC_FP64 || p->ops->method == METHOD_KIFMM, ERR_UNSUPPORTED,
               "the black-box and Stokes FMMs have an FP64 form only");
    p->precision = precision;
    p->have_expansions = false;
  });
}

int fmm_plan_bind(fmm_plan *p, int level, int level_id) {
  return guarded([&] {
    FMMB_CHECK(p, ERR_INVALID_ARGUMENT, "plan is NULL");
    FMMB_CHECK(level >= 0 && level < p->th.L, ERR_INVALID_ARGUMENT, "level out of range");
    FMMB_CHECK(level_id >= 0 && level_id < (int)p->ops->levels.size(), ERR_INVALID_ARGUMENT,
               "unknown operator entry");
    p->bound[level] = level_id;
  });
}

int fmm_plan_bind_levels(fmm_plan *p, int n_levels, const int *level_ids) {
  return guarded([&] {
    FMMB_CHECK(p && (level_ids || n_levels == 0), ERR_INVALID_ARGUMENT, "NULL argument");
    FMMB_CHECK(n_levels >= 0 && n_levels <= p->th.L, ERR_INVALID_ARGUMENT, "level count out of range");
    for (int m = 0; m < n_levels; ++m)
      FMMB_CHECK(level_ids[m] >= -1 && level_ids[m] < (int)p->ops->levels.size(),
                 ERR_INVALID_ARGUMENT, "unknown operator entry");
    for (int m = 0; m < n_levels; ++m) p->bound[m] = level_ids[m];
  });
}

static PassArgs pass_args(fmm_plan *p) {
  PassArgs a;
  a.kernel_id = p->ops->kernel_id;
  a.kp = p->ops->kp;
  a.neq = p->ops->neq;
  a.np = p->ops->np;
  a.td = &p->td;
  a.th = &p->th;
  a.ops_dev = p->ops_dev.get();
  if (p->has_dipoles) {
    a.dvx = p->dvx.get();
    a.dvy = p->dvy.get();
  }
  return a;
}

__global__ void k_gather_dipoles(const double *__restrict__ str, const double *__restrict__ nx,
                                 const double *__restrict__ ny, const int *__restrict__ ordv,
                                 int64_t n, double *__restrict__ dvx, double *__restrict__ dvy) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int o = ordv[i];
    dvx[i] = str[o] * nx[o];
    dvy[i] = str[o] * ny[o];
  }
}

// The plan's per-level operator table, gathered on the device from the
// operator set's entries (no host copy: the launch arguments carry the
// entries' addresses)
struct LevelOpsSrc {
  const LevelOpsDev *p[FMM_MAX_LEVELS_DEV];
};
static_assert(sizeof(LevelOpsDev) % sizeof(int) == 0, "LevelOpsDev is copied as words");

__global__ void k_gather_level_ops(LevelOpsSrc src, LevelOpsDev *__restrict__ dst) {
  constexpr int NW = int(sizeof(LevelOpsDev) / sizeof(int));
  const int *from = reinterpret_cast<const int *>(src.p[blockIdx.x]);
  int *to = reinterpret_cast<int *>(dst + blockIdx.x);
  for (int i = threadIdx.x; i < NW; i += blockDim.x) to[i] = from ? from[i] : 0;
}

static void upload_level_ops(fmm_plan *p, cudaStream_t s) {
  const int L = p->th.L;
  FMMB_CHECK(L <= FMM_MAX_LEVELS_DEV, ERR_INVALID_ARGUMENT, "too many levels");
  p->ops_dev.alloc(L, s);
  LevelOpsSrc src{};
  for (int m = 0; m < L; ++m)
    if (p->bound[m] >= 0) src.p[m] = p->ops->levels[p->bound[m]]->dev_copy.get();
  k_gather_level_ops<<<L, 128, 0, s>>>(src, p->ops_dev.get());
  FMMB_CUDA(cudaGetLastError());
}

static StokesArgs stokes_args(fmm_plan *p, cudaStream_t) {
  StokesArgs a{};
  a.neq = p->ops->neq;
  a.np = p->ops->np;
  a.td = &p->td;
  a.th = &p->th;
  for (int m = 0; m < p->th.L && m < FMM_MAX_LEVELS_DEV; ++m)
    if (p->bound[m] >= 0) a.lev[m] = p->ops->levels[p->bound[m]]->st_lev;
  if (p->has_st_dipoles) {
    const size_t n = size_t(p->th.n_points);
    double *d = p->st_dip.get();
    a.sgx = d;
    a.sgy = d + n;
    a.dnx = d + 2 * n;
    a.dny = d + 3 * n;
  }
  return a;
}

static BBArgs bb_args(fmm_plan *p, cudaStream_t) {
  BBArgs b{};
  b.kernel_id = p->ops->kernel_id;
  b.kp = p->ops->kp;
  b.p = p->ops->p;
  b.np = p->ops->np;
  b.td = &p->td;
  b.th = &p->th;
  b.m2mc = p->ops->bb_m2mc.get();
  b.m2mct = p->ops->bb_m2mct.get();
  for (int m = 0; m < p->th.L && m < FMM_MAX_LEVELS_DEV; ++m)
    b.m2l_cat[m] = p->bound[m] >= 0 ? p->ops->levels[p->bound[m]]->bb_m2l.get() : nullptr;
  return b;
}

static void build_stokes(fmm_plan *p, const double *fx, const double *fy, const double *sgx,
                         const double *sgy, const double *nx, const double *ny, void *stream);

int fmm_build_expansions2(fmm_plan *p, const double *fx, const double *fy, void *stream) {
  return guarded([&] { build_stokes(p, fx, fy, nullptr, nullptr, nullptr, nullptr, stream); });
}

int fmm_build_expansions2_dipole(fmm_plan *p, const double *fx, const double *fy,
                                 const double *sigma_x, const double *sigma_y, const double *dip_nx,
                                 const double *dip_ny, void *stream) {
  return guarded([&] {
    FMMB_CHECK(sigma_x && sigma_y && dip_nx && dip_ny, ERR_INVALID_ARGUMENT, "NULL argument");
    build_stokes(p, fx, fy, sigma_x, sigma_y, dip_nx, dip_ny, stream);
  });
}

static void build_stokes(fmm_plan *p, const double *fx, const double *fy, const double *sgx,
                         const double *sgy, const double *nx, const double *ny, void *stream) {
  {
    tree_ready(p);
    FMMB_CHECK(p && fx && fy, ERR_INVALID_ARGUMENT, "NULL argument");
    FMMB_CHECK(p->ops->method == METHOD_STOKES, ERR_INVALID_ARGUMENT,
               "fmm_build_expansions2 takes Stokes plans (two force components)");
    cudaStream_t s = (cudaStream_t)stream;
    p->has_st_dipoles = sgx != nullptr;
    if (sgx) {  // stresslet strengths and normals in the tree's order
      const int64_t n = p->th.n_points;
      p->st_dip.alloc(4 * size_t(n), s);
      const double *src[4] = {sgx, sgy, nx, ny};
      for (int c = 0; c < 4; ++c) gather_sorted(src[c], p->td.ordv.get(), n, p->st_dip.get() + c * n, s);
    }
    const TreeHost &th = p->th;
    for (int m = 2; m < th.L; ++m)
      FMMB_CHECK(p->bound[m] >= 0, ERR_NOT_READY, "operators not bound for every level >= 2");
    const int np = p->ops->np;
    const int64_t total = th.n_total();
    StokesArgs a = stokes_args(p, s);
    p->tau_s.alloc(th.n_points, s);
    p->tau2_s.alloc(th.n_points, s);
    gather_sorted(fx, p->td.ordv.get(), th.n_points, p->tau_s.get(), s);
    gather_sorted(fy, p->td.ordv.get(), th.n_points, p->tau2_s.get(), s);
    for (DevBuf<double> *b : {&p->partial, &p->mult, &p->ple, &p->loc}) {
      b->alloc(total * np, s);
      b->zero(s);
    }
    run_stokes_upward(a, p->tau_s.get(), p->tau2_s.get(), p->partial.get(), p->mult.get(), s);
    run_stokes_downward(a, p->mult.get(), p->ple.get(), p->loc.get(), s);
    p->have_expansions = true;
  }
}

int fmm_build_expansions_multi(fmm_plan *p, const double *tau, int n_rhs, int64_t ld_tau,
                               void *stream) {
  return guarded([&] {
    tree_ready(p);
    FMMB_CHECK(p && tau, ERR_INVALID_ARGUMENT, "NULL argument");
    FMMB_CHECK(p->ops->method == METHOD_KIFMM && p->precision == PREC_FP64, ERR_UNSUPPORTED,
               "several charge columns: FP64 KIFMM plans");
    const TreeHost &th = p->th;
    FMMB_CHECK(n_rhs >= 1 && ld_tau >= th.n_points, ERR_INVALID_ARGUMENT, "bad n_rhs or ld_tau");
    cudaStream_t s = (cudaStream_t)stream;
    for (int m = 2; m < th.L; ++m)
      FMMB_CHECK(p->bound[m] >= 0, ERR_NOT_READY, "operators not bound for every level >= 2");
    const int np = p->ops->np;
    const int64_t total = th.n_total(), n = th.n_points, cs = total * np;
    upload_level_ops(p, s);
    p->has_dipoles = false;
    PassArgs a = pass_args(p);
    p->tau_s.alloc((size_t)n_rhs * n, s);
    p->mult.alloc((size_t)n_rhs * cs, s);
    p->ple.alloc((size_t)n_rhs * cs, s);
    p->loc.alloc((size_t)n_rhs * cs, s);
    p->mult.zero(s);
    p->ple.zero(s);
    p->loc.zero(s);
    for (int r = 0; r < n_rhs; ++r)
      gather_sorted(tau + (size_t)r * ld_tau, p->td.ordv.get(), n, p->tau_s.get() + (size_t)r * n, s);
    // every pass once per level for all columns (column = blockIdx.y)
    run_upward(a, p->tau_s.get(), p->mult.get(), s, n_rhs, n, cs);
    run_m2l(a, p->mult.get(), p->ple.get(), s, n_rhs, cs);
    run_downward(a, p->ple.get(), p->loc.get(), s, n_rhs, cs);
    p->n_rhs = n_rhs;
    p->ready_recorded = false;  // the split evaluation serves single-column builds
    p->have_expansions = true;
  });
}

int fmm_evaluate_multi(fmm_plan *p, const double *tx, const double *ty, int64_t m, int check,
                       double *out, int64_t ld_out, void *stream) {
  return guarded([&] {
    tree_ready(p);
    FMMB_CHECK(p, ERR_INVALID_ARGUMENT, "plan is NULL");
    FMMB_CHECK(p->have_expansions, ERR_NOT_READY, "build_expansions has not run");
    FMMB_CHECK(p->ops->method == METHOD_KIFMM && p->precision == PREC_FP64, ERR_UNSUPPORTED,
               "several charge columns: FP64 KIFMM plans");
    FMMB_CHECK(m >= 0 && ld_out >= m, ERR_INVALID_ARGUMENT, "bad target count or ld_out");
    if (m == 0) return;
    FMMB_CHECK(tx && ty && out, ERR_INVALID_ARGUMENT, "NULL argument");
    cudaStream_t s = (cudaStream_t)stream;
    PassArgs a = pass_args(p);
    a.ops_dev = p->ops_dev.get();
    DevBuf<uint64_t> tkeys;
    DevBuf<int> tperm;
    DevBuf<double> txs, tys;
    {
      PhaseTimer timer(PH_SORT_TGT, s);
      txs.alloc(m, s);
      tys.alloc(m, s);
      sort_points(tx, ty, m, p->th, tkeys, tperm, s, p->th.L > 1 ? p->th.L - 1 : 1, txs.get(),
                  tys.get(), p->td.sort_fail.get());
    }
    run_evaluate_multi(a, p->tau_s.get(), p->th.n_points, p->n_rhs, p->loc.get(),
                       (int64_t)p->th.n_total() * p->ops->np, txs.get(), tys.get(), tkeys.get(),
                       tperm.get(), m, check, out, ld_out, s);
  });
}

int fmm_evaluate_sources_multi(fmm_plan *p, int check, double *out, int64_t ld_out, void *stream) {
  return guarded([&] {
    tree_ready(p);
    FMMB_CHECK(p, ERR_INVALID_ARGUMENT, "plan is NULL");
    FMMB_CHECK(p->have_expansions, ERR_NOT_READY, "build_expansions has not run");
    FMMB_CHECK(p->ops->method == METHOD_KIFMM && p->precision == PREC_FP64, ERR_UNSUPPORTED,
               "several charge columns: FP64 KIFMM plans");
    FMMB_CHECK(out && ld_out >= p->th.n_points, ERR_INVALID_ARGUMENT, "NULL out or ld_out too small");
    cudaStream_t s = (cudaStream_t)stream;
    PassArgs a = pass_args(p);
    a.ops_dev = p->ops_dev.get();
    const TreeDev &td = p->td;
    run_evaluate_multi(a, p->tau_s.get(), p->th.n_points, p->n_rhs, p->loc.get(),
                       (int64_t)p->th.n_total() * p->ops->np, td.sx.get(), td.sy.get(),
                       td.pkeys.get(), td.ordv.get(), p->th.n_points, check, out, ld_out, s);
  });
}

int fmm_plan_create_local(fmm_ops *ops, const double *x, const double *y, int64_t n, int ncutoff,
                          double min_width, const double *bbox, void *stream, fmm_plan **out) {
  return guarded([&] {
    FMMB_CHECK(ops && x && y && bbox && out, ERR_INVALID_ARGUMENT, "NULL argument");
    FMMB_CHECK(ops->method == METHOD_KIFMM && ops->kernel_id >= 0, ERR_INVALID_ARGUMENT,
               "a local plan takes a kernel operator set (fmm_ops_create)");
    FMMB_CHECK(min_width >= 0.0, ERR_INVALID_ARGUMENT, "negative minimum width");
    // a box of level m (width w0 / 2^m, halved level by level as the
    // reference does) splits only while its width exceeds 2 min_width
    const double w0 = bbox[1] - bbox[0];
    int max_split = 0;
    for (double w = w0; max_split < 64 && w > 2.0 * min_width; w *= 0.5) ++max_split;
    retain_pool_memory();
    auto p = std::make_unique<fmm_plan>();
    p->ops = ops;
    p->stream = (cudaStream_t)stream;
    {
      PhaseTimer timer(PH_TREE, p->stream);
      build_tree(p->td, p->th, x, y, n, ncutoff, bbox, p->stream, max_split);
    }
    p->bound.assign(p->th.L, -1);
    *out = p.release();
  });
}

int fmm_local_evaluate(fmm_plan *p, const double *tau, const double *tx, const double *ty,
                       int64_t m, int check, const int64_t *src_cat, const int64_t *tgt_cat,
                       double *out, void *stream) {
  return guarded([&] {
    tree_ready(p);
    FMMB_CHECK(p && tau, ERR_INVALID_ARGUMENT, "NULL argument");
    FMMB_CHECK(p->ops->method == METHOD_KIFMM, ERR_INVALID_ARGUMENT, "not a local plan");
    FMMB_CHECK((src_cat == nullptr) == (tgt_cat == nullptr), ERR_INVALID_ARGUMENT,
               "source and target categories go together");
    FMMB_CHECK(m >= 0, ERR_INVALID_ARGUMENT, "negative target count");
    if (m == 0) return;
    FMMB_CHECK(tx && ty && out, ERR_INVALID_ARGUMENT, "NULL argument");
    FMMB_CHECK(m < (int64_t(1) << 31) - 1, ERR_INVALID_ARGUMENT, "more than 2^31-2 targets");
    cudaStream_t s = (cudaStream_t)stream;
    const int64_t n = p->th.n_points;
    p->tau_s.alloc(n, s);
    gather_sorted(tau, p->td.ordv.get(), n, p->tau_s.get(), s);
    DevBuf<int64_t> scat;
    if (src_cat) {
      scat.alloc(n, s);
      gather_sorted_i64(src_cat, p->td.ordv.get(), n, scat.get(), s);
    }
    PassArgs a = pass_args(p);
    DevBuf<uint64_t> tkeys;
    DevBuf<int> tperm;
    DevBuf<double> txs, tys;
    {
      PhaseTimer timer(PH_SORT_TGT, s);
      txs.alloc(m, s);
      tys.alloc(m, s);
      sort_points(tx, ty, m, p->th, tkeys, tperm, s, p->th.L > 1 ? p->th.L - 1 : 1, txs.get(),
                  tys.get(), p->td.sort_fail.get());
    }
    run_local_evaluate(a, p->tau_s.get(), txs.get(), tys.get(), tkeys.get(), tperm.get(), m,
                       check, src_cat ? scat.get() : nullptr, tgt_cat, out, s);
  });
}

static void build_expansions_impl(fmm_plan *p, const double *tau, void *stream);

int fmm_build_expansions(fmm_plan *p, const double *tau, void *stream) {
  return guarded([&] {
    tree_ready(p);
    FMMB_CHECK(p && tau, ERR_INVALID_ARGUMENT, "NULL argument");
    FMMB_CHECK(p->ops->method != METHOD_STOKES, ERR_INVALID_ARGUMENT,
               "Stokes plans take fmm_build_expansions2 (two force components)");
    p->has_dipoles = false;
    build_expansions_impl(p, tau, stream);
  });
}

int fmm_build_expansions_dipole(fmm_plan *p, const double *tau, const double *dip_str,
                                const double *dip_nx, const double *dip_ny, void *stream) {
  return guarded([&] {
    tree_ready(p);
    FMMB_CHECK(p && dip_str && dip_nx && dip_ny, ERR_INVALID_ARGUMENT, "NULL argument");
    FMMB_CHECK(p->ops->method == METHOD_KIFMM && p->ops->kernel_id == KERNEL_LAPLACE,
               ERR_UNSUPPORTED, "dipole sources: KIFMM plans of the Laplace kernel");
    FMMB_CHECK(p->precision == PREC_FP64, ERR_UNSUPPORTED, "dipole sources: FP64 form only");
    cudaStream_t s = (cudaStream_t)stream;
    const int64_t n = p->th.n_points;
    p->dvx.alloc(n, s);
    p->dvy.alloc(n, s);
    if (n > 0) {
      k_gather_dipoles<<<grid_for(n, 256), 256, 0, s>>>(dip_str, dip_nx, dip_ny,
                                                         p->td.ordv.get(), n, p->dvx.get(),
                                                         p->dvy.get());
      FMMB_CUDA(cudaGetLastError());
    }
    p->has_dipoles = true;
    build_expansions_impl(p, tau, stream);
  });
}

// the build itself (FP64 / mixed KIFMM or black-box), after the entry's checks;
// tau = NULL: zero charges
static void build_expansions_impl(fmm_plan *p, const double *tau, void *stream) {
  {
    p->n_rhs = 1;
    cudaStream_t s = (cudaStream_t)stream;
    const TreeHost &th = p->th;
    for (int m = 2; m < th.L; ++m)
      FMMB_CHECK(p->bound[m] >= 0, ERR_NOT_READY, "operators not bound for every level >= 2");
    const int np = p->ops->np;
    const int64_t total = th.n_total();
    if (p->ops->method == METHOD_BBFMM) {
      BBArgs b = bb_args(p, s);
      p->tau_s.alloc(th.n_points, s);
      gather_sorted(tau, p->td.ordv.get(), th.n_points, p->tau_s.get(), s);
      p->mult.alloc(total * np, s);
      p->ple.alloc(total * np, s);
      p->mult.zero(s);
      p->ple.zero(s);
      run_bb_upward(b, p->tau_s.get(), p->mult.get(), s);
      run_bb_downward(b, p->mult.get(), p->ple.get(), s);
      p->have_expansions = true;
      return;
    }
    std::unique_ptr<PhaseTimer> t_prep(new PhaseTimer(PH_PREP, s));
    upload_level_ops(p, s);
    split_prepare(p);
    p->ready_recorded = false;
    PassArgs a = pass_args(p);
    p->tau_s.alloc(th.n_points, s);
    if (tau)
      gather_sorted(tau, p->td.ordv.get(), th.n_points, p->tau_s.get(), s);
    else
      p->tau_s.zero(s);
    p->ple.alloc(total * np, s);
    if (p->precision == PREC_MIXED) {
      p->mult32.alloc(total * np, s);
      p->loc32.alloc(total * np, s);
      p->msum.alloc(total, s);
      p->lsum.alloc(total, s);
      p->mult_tc.alloc(total * 2 * np, s);
      // a split near field (if evaluation splits) runs beside the upward and
      // downward passes and pauses while the M2L runs: hold clear now, set
      // before the M2L; m2l_done recorded after it
      p->hold_armed = split_enabled(PREC_MIXED);
      if (p->hold_armed) p->near_hold.alloc(1, s);
      p->err.alloc(2, s);  // [0] error flag, [1] M2L tile counter
      ZeroBatch zb(s);
      zb.add(p->ple).add(p->mult32).add(p->mult_tc).add(p->loc32).add(p->msum).add(p->lsum).add(p->err);
      if (p->hold_armed) zb.add(p->near_hold);
      zb.run();
      p->tsum.alloc(total, s);
      node_charge_sums(a, p->tau_s.get(), p->tsum.get(), s);
      // sorted charges and box charge sums are all the near field reads
      FMMB_CUDA(cudaEventRecord(p->ev_ready, s));
      p->ready_recorded = true;
      t_prep.reset();
      run_upward_mixed(a, p->tau_s.get(), p->tsum.get(), p->mult32.get(), p->msum.get(),
                       p->mult_tc.get(), s);
      if (p->hold_armed) FMMB_CUDA(cudaMemsetAsync(p->near_hold.get(), 1, 1, s));
      run_m2l_mixed(a, p->mult32.get(), p->mult_tc.get(), p->msum.get(), p->ple.get(),
                    p->err.get(), s);
      if (p->hold_armed) FMMB_CUDA(cudaEventRecord(p->ev_m2l, s));
      run_downward_mixed(a, p->ple.get(), p->loc32.get(), p->lsum.get(), s);
    } else {
      p->mult.alloc(total * np, s);
      p->loc.alloc(total * np, s);
      ZeroBatch(s).add(p->ple).add(p->mult).add(p->loc).run();
      FMMB_CUDA(cudaEventRecord(p->ev_ready, s));  // sorted charges: all the near field reads
      p->ready_recorded = true;
      t_prep.reset();
      run_upward(a, p->tau_s.get(), p->mult.get(), s);
      run_m2l(a, p->mult.get(), p->ple.get(), s);
      run_downward(a, p->ple.get(), p->loc.get(), s);
    }
    p->have_expansions = true;
  }
}

namespace {
// outputs of an evaluator id (FMM_EVAL_*)
int evaluator_outputs(int evaluator) {
  FMMB_CHECK(evaluator == FMM_EVAL_POTENTIAL || evaluator == FMM_EVAL_GRADIENT ||
                 evaluator == FMM_EVAL_STOKES,
             ERR_INVALID_ARGUMENT, "evaluator must be one of FMM_EVAL_POTENTIAL, _GRADIENT, _STOKES");
  return evaluator == FMM_EVAL_POTENTIAL ? 1 : 3;
}

// a plan's method accepts the evaluator (Stokes plans: (u, v, p) only)
void check_evaluator(fmm_plan *p, int evaluator) {
  FMMB_CHECK(p, ERR_INVALID_ARGUMENT, "plan is NULL");
  const bool st = p->ops->method == METHOD_STOKES;
  FMMB_CHECK(st == (evaluator == FMM_EVAL_STOKES), ERR_INVALID_ARGUMENT,
             st ? "Stokes plans evaluate FMM_EVAL_STOKES (u, v, p)"
                : "FMM_EVAL_STOKES needs a Stokes plan");
}

void evaluate_points(fmm_plan *p, int nout, const double *tx, const double *ty, int64_t m,
                     int check, double *out, int64_t ld_out, cudaStream_t s) {
  FMMB_CHECK(p, ERR_INVALID_ARGUMENT, "plan is NULL");
  FMMB_CHECK(p->have_expansions, ERR_NOT_READY, "build_expansions has not run");
  FMMB_CHECK(m >= 0, ERR_INVALID_ARGUMENT, "negative target count");
  if (m == 0) return;
  FMMB_CHECK(tx && ty && out, ERR_INVALID_ARGUMENT, "NULL argument");
  FMMB_CHECK(m < (int64_t(1) << 31) - 1, ERR_INVALID_ARGUMENT, "more than 2^31-2 targets");
  FMMB_CHECK(nout == 1 || ld_out >= m, ERR_INVALID_ARGUMENT, "ld_out is smaller than the target count");
  PassArgs a = pass_args(p);
  DevBuf<uint64_t> tkeys;
  DevBuf<int> tperm;
  DevBuf<double> txs, tys;
  txs.alloc(m, s);
  tys.alloc(m, s);
  if (p->ops->method == METHOD_KIFMM) {
    // targets binned into their leaves (a descent along each key's digits and
    // a count per leaf) instead of sorted
    EvalItems it;
    {
      PhaseTimer timer(PH_SORT_TGT, s);
      tperm.alloc(m, s);
      eval_items_binned(a, tx, ty, m, it, txs.get(), tys.get(), tperm.get(), s);
    }
    if (p->precision == PREC_MIXED)
      run_evaluate_mixed(a, p->tau_s.get(), p->tsum.get(), p->loc32.get(), p->lsum.get(), txs.get(),
                         tys.get(), nullptr, tperm.get(), m, check, nout, out, ld_out, s, &it);
    else
      run_evaluate(a, p->tau_s.get(), p->loc.get(), txs.get(), tys.get(), nullptr, tperm.get(), m,
                   check, nout, out, ld_out, s, &it);
    return;
  }
  // evaluator ids carry the output count; Stokes plans produce (u, v, p)
  {
    PhaseTimer timer(PH_SORT_TGT, s);
    // leaves live on levels <= L-1: their first L-1 digits decide everything
    sort_points(tx, ty, m, p->th, tkeys, tperm, s, p->th.L > 1 ? p->th.L - 1 : 1, txs.get(),
                tys.get(), p->td.sort_fail.get());
  }
  if (p->ops->method == METHOD_STOKES)
    run_stokes_evaluate(stokes_args(p, s), p->tau_s.get(), p->tau2_s.get(), p->loc.get(), txs.get(),
                        tys.get(), tkeys.get(), tperm.get(), m, check, out, ld_out, s);
  else if (p->ops->method == METHOD_BBFMM)
    run_bb_evaluate(bb_args(p, s), p->tau_s.get(), p->ple.get(), txs.get(), tys.get(), tkeys.get(),
                    tperm.get(), m, check, nout, out, ld_out, s);
  else if (p->precision == PREC_MIXED)
    run_evaluate_mixed(a, p->tau_s.get(), p->tsum.get(), p->loc32.get(), p->lsum.get(), txs.get(),
                       tys.get(), tkeys.get(), tperm.get(), m, check, nout, out, ld_out, s);
  else
    run_evaluate(a, p->tau_s.get(), p->loc.get(), txs.get(), tys.get(), tkeys.get(), tperm.get(),
                 m, check, nout, out, ld_out, s);
}


void evaluate_own_sources(fmm_plan *p, int nout, int check, double *out, int64_t ld_out,
                          cudaStream_t s) {
  FMMB_CHECK(p, ERR_INVALID_ARGUMENT, "plan is NULL");
  FMMB_CHECK(p->have_expansions, ERR_NOT_READY, "build_expansions has not run");
  FMMB_CHECK(out, ERR_INVALID_ARGUMENT, "NULL argument");
  const TreeDev &td = p->td;
  const int64_t m = p->th.n_points;
  FMMB_CHECK(nout == 1 || ld_out >= m, ERR_INVALID_ARGUMENT, "ld_out is smaller than the source count");
  PassArgs a = pass_args(p);
  // the tree's sorted copy: keys sorted on at least their top L-1 digits,
  // which is all that leaf location reads
  if (p->ops->method == METHOD_STOKES)
    run_stokes_evaluate(stokes_args(p, s), p->tau_s.get(), p->tau2_s.get(), p->loc.get(),
                        td.sx.get(), td.sy.get(), td.pkeys.get(), td.ordv.get(), m, check, out,
                        ld_out, s);
  else if (p->ops->method == METHOD_BBFMM)
    run_bb_evaluate(bb_args(p, s), p->tau_s.get(), p->ple.get(), td.sx.get(), td.sy.get(),
                    td.pkeys.get(), td.ordv.get(), m, check, nout, out, ld_out, s);
  else if (nout == 1 && p->ready_recorded && p->n_rhs == 1 && split_enabled(p->precision)) {
    // near field on the side stream, started when the charges were sorted
    SplitEval se{p->side, p->ev_ready, p->ev_near, p->ev_far};
    if (p->precision == PREC_MIXED && p->hold_armed) {
      se.hold = p->near_hold.get();
      se.m2l_done = p->ev_m2l;
    }
    if (p->precision == PREC_MIXED)
      run_evaluate_sources_split_mixed(a, p->tau_s.get(), p->tsum.get(), p->loc32.get(),
                                       p->lsum.get(), check, out, s, se);
    else
      run_evaluate_sources_split(a, p->tau_s.get(), p->loc.get(), check, out, s, se);
  } else if (p->precision == PREC_MIXED)
    run_evaluate_mixed(a, p->tau_s.get(), p->tsum.get(), p->loc32.get(), p->lsum.get(),
                       td.sx.get(), td.sy.get(), td.pkeys.get(), td.ordv.get(), m, check, nout,
                       out, ld_out, s);
  else
    run_evaluate(a, p->tau_s.get(), p->loc.get(), td.sx.get(), td.sy.get(), td.pkeys.get(),
                 td.ordv.get(), m, check, nout, out, ld_out, s);
}
}  // namespace

int fmm_evaluate(fmm_plan *p, const double *tx, const double *ty, int64_t m, int check,
                 double *out, void *stream) {
  return guarded([&] {
    tree_ready(p);
    check_evaluator(p, FMM_EVAL_POTENTIAL);
    evaluate_points(p, 1, tx, ty, m, check, out, m, (cudaStream_t)stream);
  });
}

int fmm_evaluate_sources(fmm_plan *p, int check, double *out, void *stream) {
  return guarded([&] {
    tree_ready(p);
    check_evaluator(p, FMM_EVAL_POTENTIAL);
    evaluate_own_sources(p, 1, check, out, 0, (cudaStream_t)stream);
  });
}

int fmm_evaluate_outputs(fmm_plan *p, int evaluator, const double *tx, const double *ty,
                         int64_t m, int check, double *out, int64_t ld_out, void *stream) {
  return guarded([&] {
    tree_ready(p);
    const int nout = evaluator_outputs(evaluator);
    check_evaluator(p, evaluator);
    evaluate_points(p, nout, tx, ty, m, check, out, ld_out, (cudaStream_t)stream);
  });
}

int fmm_evaluate_sources_outputs(fmm_plan *p, int evaluator, int check, double *out,
                                 int64_t ld_out, void *stream) {
  return guarded([&] {
    tree_ready(p);
    const int nout = evaluator_outputs(evaluator);
    check_evaluator(p, evaluator);
    evaluate_own_sources(p, nout, check, out, ld_out, (cudaStream_t)stream);
  });
}

int fmm_plan_status(fmm_plan *p) {
  return guarded([&] {
    tree_ready(p);
    FMMB_CHECK(p, ERR_INVALID_ARGUMENT, "plan is NULL");
    FMMB_CUDA(cudaStreamSynchronize(p->stream));
    FMMB_CUDA(cudaGetLastError());
    if (p->err.get()) {
      int h = 0;
      FMMB_CUDA(cudaMemcpy(&h, p->err.get(), sizeof(int), cudaMemcpyDeviceToHost));
      FMMB_CHECK(h == 0, ERR_CUDA, "a tensor-core wait ran out of time; results are invalid");
    }
    if (p->td.sort_fail.get()) {
      int h = 0;
      FMMB_CUDA(cudaMemcpy(&h, p->td.sort_fail.get(), sizeof(int), cudaMemcpyDeviceToHost));
      FMMB_CHECK(h == 0, ERR_CUDA, "a radix sort's grid barrier wait ran out of time; results are invalid");
    }
  });
}

int fmm_plan_drop_expansions(fmm_plan *p) {
  return guarded([&] {
    FMMB_CHECK(p, ERR_INVALID_ARGUMENT, "plan is NULL");
    // device memory returns to the pool in the plan stream's order
    p->tau_s.release();
    p->tau2_s.release();
    p->mult.release();
    p->ple.release();
    p->loc.release();
    p->mult32.release();
    p->loc32.release();
    p->mult_tc.release();
    p->msum.release();
    p->lsum.release();
    p->tsum.release();
    p->partial.release();
    p->dvx.release();
    p->dvy.release();
    p->has_dipoles = false;
    p->st_dip.release();
    p->has_st_dipoles = false;
    p->have_expansions = false;
    p->ready_recorded = false;
  });
}

int fmm_plan_move_sources(fmm_plan *p, const double *x, const double *y, void *stream) {
  return guarded([&] {
    tree_ready(p);
    FMMB_CHECK(p, ERR_INVALID_ARGUMENT, "plan is NULL");
    const int64_t n = p->th.n_points;
    if (n == 0) return;
    FMMB_CHECK(x && y, ERR_INVALID_ARGUMENT, "NULL argument");
    cudaStream_t s = (cudaStream_t)stream;
    // the tree's sorted copy, in the tree's own order (sorted -> original)
    gather_sorted(x, p->td.ordv.get(), n, p->td.sx.get(), s);
    gather_sorted(y, p->td.ordv.get(), n, p->td.sy.get(), s);
    p->have_expansions = false;
    p->ready_recorded = false;
  });
}

int fmm_plan_destroy(fmm_plan *p) {
  // no host wait: the plan's device buffers go back to the pool with
  // cudaFreeAsync on the stream they were allocated on, after the work
  // already queued there
  return guarded([&] { delete p; });
}

int fmm_tree_export(fmm_plan *p, double *xmin, double *ymin, int *bot, int *top, int *parent,
                    int *child, uint8_t *flags, int *coll, int *il, int *ordv) {
  return guarded([&] {
    tree_ready(p);
    FMMB_CHECK(p, ERR_INVALID_ARGUMENT, "plan is NULL");
    const size_t T = p->th.n_total();
    cudaStream_t s = p->stream;
    auto cp = [&](void *dst, const void *src, size_t bytes) {
      if (dst && bytes) FMMB_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s));
    };
    cp(xmin, p->td.xmin.get(), T * sizeof(double));
    cp(ymin, p->td.ymin.get(), T * sizeof(double));
    cp(bot, p->td.bot.get(), T * sizeof(int));
    cp(top, p->td.top.get(), T * sizeof(int));
    cp(parent, p->td.parent.get(), T * sizeof(int));
    cp(child, p->td.child.get(), T * sizeof(int));
    cp(flags, p->td.flags.get(), T * sizeof(uint8_t));
    cp(coll, p->td.coll.get(), T * 9 * sizeof(int));
    cp(il, p->td.il.get(), T * N_OFFSETS * sizeof(int));
    cp(ordv, p->td.ordv.get(), size_t(p->th.n_points) * sizeof(int));
    FMMB_CUDA(cudaStreamSynchronize(s));
  });
}

int fmm_direct(int kernel_id, const double *kparams, const double *sx, const double *sy,
               const double *tau, int64_t ns, const double *tx, const double *ty, int64_t nt,
               int check, double *out, void *stream) {
  return guarded([&] {
    FMMB_CHECK(kernel_known(kernel_id), ERR_UNSUPPORTED, "unknown kernel id");
    FMMB_CHECK(ns >= 0 && nt >= 0, ERR_INVALID_ARGUMENT, "negative size");
    if (nt == 0) return;
    FMMB_CHECK(tx && ty && out && (ns == 0 || (sx && sy && tau)), ERR_INVALID_ARGUMENT,
               "NULL argument");
    const KernelParams kp = kernel_params(kernel_id, kparams);
    run_direct(kernel_id, kp, sx, sy, tau, ns, tx, ty, nt, check, out, (cudaStream_t)stream);
  });
}

int fmm_diag_log2(const double *x, int64_t n, double *out_table, double *out_library,
                  void *stream) {
  return guarded([&] {
    FMMB_CHECK(n >= 0, ERR_INVALID_ARGUMENT, "negative size");
    if (n == 0) return;
    FMMB_CHECK(x && out_table && out_library, ERR_INVALID_ARGUMENT, "NULL argument");
    run_diag_log2(x, n, out_table, out_library, (cudaStream_t)stream);
  });
}

int fmm_set_split_evaluation(int mode) {
  return guarded([&] {
    FMMB_CHECK(mode >= -1 && mode <= 1, ERR_INVALID_ARGUMENT, "mode must be -1, 0 or 1");
    if (mode == -1) {
      const char *e = getenv("FLEXMM_B200_SPLIT_EVAL");
      mode = e ? (e[0] == '0' ? 0 : 1) : -1;
    }
    g_split_mode.store(mode);
  });
}

int fmm_timing_enable(int on) {
  return guarded([&] {
    auto &R = TimingRegistry::get();
    std::lock_guard<std::mutex> g(R.mu);
    R.enabled = on != 0;
  });
}

int fmm_timing_read(double *ms, int64_t *launches) {
  return guarded([&] {
    auto &R = TimingRegistry::get();
    std::lock_guard<std::mutex> g(R.mu);
    for (int i = 0; i < FMM_N_PHASES; ++i) {
      if (ms) ms[i] = 0.0;
      if (launches) launches[i] = 0;
    }
    for (auto &r : R.recs) {
      FMMB_CUDA(cudaEventSynchronize(r.b));
      float t = 0.f;
      FMMB_CUDA(cudaEventElapsedTime(&t, r.a, r.b));
      if (ms) ms[r.phase] += t;
      if (launches) launches[r.phase] += 1;
      R.pool.push_back(r.a);
      R.pool.push_back(r.b);
    }
    R.recs.clear();
  });
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free evaluation.
//
// fmm_evaluate_noalloc does the work of fmm_evaluate without allocating
// device memory: its scratch (target keys and permutation, sorted target
// coordinates, per-node target ranges, sort and scan workspace) lives in the
// file-scope array below.  The array is part of the library image, so every
// GPU that loads the library holds it (NOALLOC_SCRATCH_BYTES) until the
// process exits.  Every call shares it and it keeps the last call's contents;
// nothing in it needs to start at zero (every scratch word is written before
// it is read).  Calls that overlap on the GPU (two streams, two threads) race
// on it and must be serialised by the caller.
namespace {
constexpr size_t NOALLOC_SCRATCH_BYTES = size_t(24) << 20;  // 24 MiB
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

// device address of the array, looked up once per device (with it current) by
// the first call on that device; that first call should come before any
// stream capture
constexpr int NOALLOC_MAX_DEVICES = 64;
std::mutex g_noalloc_mu;
void *g_noalloc_ptr[NOALLOC_MAX_DEVICES] = {};

void *noalloc_scratch_for_current_device() {
  int dev = 0;
  FMMB_CUDA(cudaGetDevice(&dev));
  FMMB_CHECK(dev >= 0 && dev < NOALLOC_MAX_DEVICES, ERR_UNSUPPORTED, "device ordinal too large");
  std::lock_guard<std::mutex> g(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void *ptr = nullptr;
    FMMB_CUDA(cudaGetSymbolAddress(&ptr, g_noalloc_scratch));
    g_noalloc_ptr[dev] = ptr;
  }
  return g_noalloc_ptr[dev];
}

size_t round256(size_t b) { return (b + 255) & ~size_t(255); }
}  // namespace

extern "C" int fmm_evaluate_noalloc(fmm_plan *p, const double *tx, const double *ty, int64_t m,
                                    int check, double *out, void *stream) {
  return guarded([&] {
    tree_ready(p);
    FMMB_CHECK(p, ERR_INVALID_ARGUMENT, "plan is NULL");
    FMMB_CHECK(p->have_expansions, ERR_NOT_READY, "build_expansions has not run");
    FMMB_CHECK(p->precision == PREC_FP64, ERR_UNSUPPORTED,
               "fmm_evaluate_noalloc evaluates FP64 plans only");
    FMMB_CHECK(p->ops->method == METHOD_KIFMM, ERR_UNSUPPORTED,
               "fmm_evaluate_noalloc evaluates KIFMM plans only");
    FMMB_CHECK(!p->has_dipoles, ERR_UNSUPPORTED,
               "fmm_evaluate_noalloc evaluates charge sources only (no dipoles)");
    FMMB_CHECK(m >= 0, ERR_INVALID_ARGUMENT, "negative target count");
    FMMB_CHECK(m <= FMM_NOALLOC_MAX_TARGETS, ERR_CAPACITY,
               "fmm_evaluate_noalloc: more than FMM_NOALLOC_MAX_TARGETS targets");
    const int total = p->th.n_total();
    FMMB_CHECK(total <= FMM_NOALLOC_MAX_NODES, ERR_CAPACITY,
               "fmm_evaluate_noalloc: tree has more than FMM_NOALLOC_MAX_NODES nodes");
    if (m == 0) return;
    FMMB_CHECK(tx && ty && out, ERR_INVALID_ARGUMENT, "NULL argument");
    cudaStream_t s = (cudaStream_t)stream;
    unsigned char *base = static_cast<unsigned char *>(noalloc_scratch_for_current_device());
    // carve the scratch
    const int digits = p->th.L > 1 ? p->th.L - 1 : 1;
    const size_t sort_bytes = round256(sort_points_scratch_bytes(m, digits));
    const size_t scan_bytes = round256(evaluate_scratch_bytes(total));
    size_t at = 0;
    auto carve = [&](size_t bytes) {
      unsigned char *q = base + at;
      at += round256(bytes);
      return q;
    };
    uint64_t *tkeys = (uint64_t *)carve(m * sizeof(uint64_t));
    int *tperm = (int *)carve(m * sizeof(int));
    double *txs = (double *)carve(m * sizeof(double));
    double *tys = (double *)carve(m * sizeof(double));
    int *tb = (int *)carve(total * sizeof(int));
    int *te = (int *)carve(total * sizeof(int));
    int *nch = (int *)carve(total * sizeof(int));
    int *choff = (int *)carve(total * sizeof(int));
    int4 *items = (int4 *)carve((total + m / EVAL_CHUNK + 1) * sizeof(int4));
    int *n_items = (int *)carve(sizeof(int));
    void *sort_tmp = carve(sort_bytes);
    void *scan_tmp = carve(scan_bytes);
    FMMB_CHECK(at <= NOALLOC_SCRATCH_BYTES, ERR_CAPACITY,
               "fmm_evaluate_noalloc: scratch needs exceed the static array");
    // the same passes as fmm_evaluate, on the static scratch
    PassArgs a;
    a.kernel_id = p->ops->kernel_id;
    a.kp = p->ops->kp;
    a.neq = p->ops->neq;
    a.np = p->ops->np;
    a.td = &p->td;
    a.th = &p->th;
    a.ops_dev = p->ops_dev.get();
    {
      PhaseTimer timer(PH_SORT_TGT, s);
      sort_points_scratch(tx, ty, m, p->th, digits, tkeys, tperm, txs, tys, sort_tmp, sort_bytes,
                          p->td.sort_fail.get(), s);
    }
    run_evaluate_scratch(a, p->tau_s.get(), p->loc.get(), txs, tys, tkeys, tperm, m, check, out, tb,
                         te, nch, choff, items, n_items, scan_tmp, scan_bytes, s);
  });
}
