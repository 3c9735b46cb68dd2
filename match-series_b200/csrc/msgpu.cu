// msgpu.cu -- C ABI and batch pipeline of the B200 registration path.
//
// Pipeline of msgpu_register_batch (one stage of series matching, all frames
// at once):
//   1. image preparation: exact saturated min/max by radix selection, clamp,
//      scale to [0,1] (registration.h:335-346, vec.h:864-871, 1084-1089)
//   2. image pyramid by RestrictOp<STD_QUOC_RESTRICT> (multilevelArray.h:94-110)
//   3. per level: ONE persistent launch (msgpu_level.cuh) solving every frame's
//      gradient flow, then prolongation of the displacements
//      (quocDescent.h:83-105, registration.h:510-521)
//   4. prolongation to the precision level (registration.h:462-467)
// and msgpu_warp_mean the warped-frame average (matchSeries.h:385-425).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <climits>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <atomic>
#include <string>
#include <thread>
#include <type_traits>
#include <vector>

#include "../../include/msgpu.h"
#include "msgpu_level.cuh"
#include "msgpu_series.cuh"
#include "msgpu_seismic.cuh"
#include "msgpu_unet.cuh"
#include "msgpu_tc.cuh"

using namespace msg;

struct msgpu_context {
  int device = 0;
  int sm_count = 0;
  std::string err;
  cudaStream_t stream = nullptr;
  // growable device buffers
  struct Buf { void* p = nullptr; size_t cap = 0; };
  Buf arena, shared_real, dscratch, small, phis_d, io[6], prof, sched, flags, nccbuf, ext, series, vals;
  int data_term = 0;           // data term of the single-operator entry points
  int sum_order = 0;           // order of the global sums of the single-operator entry points
  Buf xsum;                    // exact sums: per-instance term blocks and chunk summaries
  Buf xpart;                   // exact sums: per-tile bounds of the energy passes' sums
  bool certified = true;       // exact sums: certified control steps (kXsBufs term buffers)
  // CUDA graph of the last device batch call (msgpu_register_batch_device):
  // captured on the second call with the same parameters and buffers, then
  // replayed as one launch while they stay the same
  struct Graph {
    std::vector<unsigned char> key;
    int seen = 0;                // calls with this key so far
    cudaGraphExec_t exec = nullptr;
    int launches = 0;            // kernels in the graph
    unsigned long long epoch = 0;  // alloc_epoch when it was captured
  } graph;
  unsigned long long alloc_epoch = 0;   // counts reallocations of the context's buffers
  bool use_graphs = true;
  cudaStream_t graph_stream = nullptr;
  // scheduling of the level kernel per precision (FP32, FP64) and level;
  // zeros are the defaults (msgpu_autotune fills it)
  msgpu_level_tuning tuning[2][kMaxLevel + 1] = {};
  int* sched_error = nullptr;  // device flag of the level scheduler (in flags)
  // statistics of the last batch call
  bool profiling = false;
  msgpu_stats stats{};
  cudaEvent_t ev[32] = {};
  bool ev_ready = false;
  int last_grid = 0;        // CTAs of the last level launch
  // seismic line-shift solve: the spectral basis of its H1 metric
  int xs_nx = 0, xs_ny = 0;
  Buf xs_basis, xs_work;
  cudaStream_t xc_stream[4] = {nullptr, nullptr, nullptr, nullptr};   // capture streams of the findXShift graph
  bool xs_device_control = false;                             // findXShift as a device-controlled graph
  int warm_coarse_iters = 0;   // warm start: step limit below the stop level (0: maxGDIterations)
  // pass timeline of one level (profiling): the level, the capacity in
  // events, the buffer (events, then the count) and the events of the last
  // profiled call
  int trace_level = -1;
  unsigned trace_cap = 0;
  Buf trace;
  std::vector<unsigned long long> trace_host;
  std::vector<msgpu_context*> workers;   // contexts of the batch workers (own streams and buffers)
};

namespace {

constexpr int kAbiVersion = 8;
// default chunking of the level scheduler: a 24th of a pass, at most 16 tiles
constexpr int kChunkDiv = 24, kChunkMax = 16;

// Bounds of the device-side waits (global-timer nanoseconds), process-wide:
// a level-kernel worker waiting for work, a composition grid barrier.
// msgpu_set_wait_limits changes them (a diagnostic hook: shorter bounds make
// a wait run out on purpose, so that the error path can be checked).
std::atomic<unsigned long long> g_level_wait_ns{kMaxIdleNs};
std::atomic<unsigned long long> g_barrier_wait_ns{kExtBarrierNs};

int fail(msgpu_context* ctx, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (ctx) ctx->err = buf;
  return code;
}

#define CK(call)                                                                                  \
  do {                                                                                            \
    cudaError_t e_ = (call);                                                                      \
    if (e_ != cudaSuccess)                                                                        \
      return fail(ctx, MSGPU_ERR_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_),   \
                  __FILE__, __LINE__);                                                            \
  } while (0)

int ensure(msgpu_context* ctx, msgpu_context::Buf& b, size_t bytes) {
  if (b.cap >= bytes) return MSGPU_OK;
  ++ctx->alloc_epoch;   // a captured graph holding the old address is stale now
  if (b.p) CK(cudaFree(b.p));
  b.p = nullptr;
  b.cap = 0;
  CK(cudaMalloc(&b.p, bytes));
  b.cap = bytes;
  return MSGPU_OK;
}

__host__ __device__ inline int lvl_n(int l) { return (1 << l) + 1; }
__host__ __device__ inline size_t lvl_N(int l) { return (size_t)lvl_n(l) * lvl_n(l); }
inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// Q1 tables and assembled stiffness stencil per node class, computed in double
// the way the reference assembles StiffOp (FEOpInterface.h:65-88, 1362-1395).
// The values do not depend on the level: h enters only through exact powers of
// two that cancel between the gradients and the element volume.
bool g_tables_ready[64] = {false};

void host_basis_grad(int b, double x, double y, double h, double g[2]) {
  switch (b) {
    case 0: g[0] = (y - 1.0) / h; g[1] = (x - 1.0) / h; break;
    case 1: g[0] = (1.0 - y) / h; g[1] = (-x) / h; break;
    case 2: g[0] = (-y) / h; g[1] = (1.0 - x) / h; break;
    default: g[0] = y / h; g[1] = x / h; break;
  }
}
double host_basis_val(int b, double x, double y) {
  switch (b) {
    case 0: return (1.0 - x) * (1.0 - y);
    case 1: return x * (1.0 - y);
    case 2: return (1.0 - x) * y;
    default: return x * y;
  }
}

void host_fe_tables(FeTables& t) {
  const double g[2] = {0.2113248654051871, 0.7886751345948129};
  for (int i = 0, k = 0; i < 2; ++i)
    for (int j = 0; j < 2; ++j, ++k) { t.rc[k][0] = g[i]; t.rc[k][1] = g[j]; }
  const double h = 0.25, vol = h * h;
  double gq[4][4][2];
  for (int b = 0; b < 4; ++b)
    for (int q = 0; q < 4; ++q) {
      t.bq[b][q] = host_basis_val(b, t.rc[q][0], t.rc[q][1]);
      host_basis_grad(b, t.rc[q][0], t.rc[q][1], h, gq[b][q]);
    }
  t.w = 0.5 * 0.5;
  double L[4][4];
  for (int i = 0; i < 4; ++i) for (int j = 0; j < 4; ++j) L[i][j] = 0.;
  for (int q = 0; q < 4; ++q)
    for (int i = 0; i < 4; ++i)
      for (int j = i; j < 4; ++j) {
        double d = 0;
        d += gq[i][q][0] * gq[j][q][0];
        d += gq[i][q][1] * gq[j][q][1];
        L[i][j] += d * 1. * t.w;
      }
  for (int i = 0; i < 4; ++i)
    for (int j = i; j < 4; ++j) L[j][i] = L[i][j] = L[i][j] * vol;
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) t.lst[i][j] = L[i][j];
  // assemble on a 5x5 node grid in element order and read the 9 node classes
  const int n = 5;
  std::vector<double> st((size_t)n * n * 9, 0.0);
  for (int ey = 0; ey < n - 1; ++ey)
    for (int ex = 0; ex < n - 1; ++ex)
      for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) {
          const int gi = ex + ey * n + ((i & 1) ? 1 : 0) + ((i & 2) ? n : 0);
          const int gj = ex + ey * n + ((j & 1) ? 1 : 0) + ((j & 2) ? n : 0);
          const int dx = (gj % n) - (gi % n), dy = (gj / n) - (gi / n);
          st[(size_t)gi * 9 + (dy + 1) * 3 + (dx + 1)] += 1.0 * L[i][j];
        }
  const int rep[3] = {0, 2, 4};
  for (int cy = 0; cy < 3; ++cy)
    for (int cx = 0; cx < 3; ++cx) {
      const int node = rep[cx] + rep[cy] * n;
      for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 3; ++i) t.st[cx + 3 * cy][j][i] = st[(size_t)node * 9 + j * 3 + i];
    }
  // mass matrix (FELinScalarWeightedMassInterface::prepareLocalMatrix,
  // FEOpInterface.h:1445-1475) with element volume 1, same assembly
  double M[4][4];
  for (int i = 0; i < 4; ++i) for (int j = 0; j < 4; ++j) M[i][j] = 0.;
  for (int q = 0; q < 4; ++q)
    for (int i = 0; i < 4; ++i) {
      const double basisi = t.bq[i][q];
      for (int j = i; j < 4; ++j) M[i][j] += basisi * t.bq[j][q] * 1. * t.w;
    }
  for (int i = 0; i < 4; ++i)
    for (int j = i; j < 4; ++j) M[j][i] = M[i][j] = M[i][j] * 1.0;
  std::vector<double> ms((size_t)n * n * 9, 0.0);
  for (int ey = 0; ey < n - 1; ++ey)
    for (int ex = 0; ex < n - 1; ++ex)
      for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) {
          const int gi = ex + ey * n + ((i & 1) ? 1 : 0) + ((i & 2) ? n : 0);
          const int gj = ex + ey * n + ((j & 1) ? 1 : 0) + ((j & 2) ? n : 0);
          const int dx = (gj % n) - (gi % n), dy = (gj / n) - (gi / n);
          ms[(size_t)gi * 9 + (dy + 1) * 3 + (dx + 1)] += 1.0 * M[i][j];
        }
  for (int cy = 0; cy < 3; ++cy)
    for (int cx = 0; cx < 3; ++cx) {
      const int node = rep[cx] + rep[cy] * n;
      for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 3; ++i) t.ms[cx + 3 * cy][j][i] = ms[(size_t)node * 9 + j * 3 + i];
    }
}

int ensure_tables(msgpu_context* ctx) {
  int dev = 0;
  CK(cudaGetDevice(&dev));
  if (dev < 64 && g_tables_ready[dev]) return MSGPU_OK;
  FeTables t;
  host_fe_tables(t);
  CK(cudaMemcpyToSymbol(c_fe, &t, sizeof(t)));
  // a copy from pageable memory may return before it lands; the kernels that
  // read the tables run on non-blocking streams, which do not wait for it
  CK(cudaDeviceSynchronize());
  if (dev < 64) g_tables_ready[dev] = true;
  return MSGPU_OK;
}

// ---------------------------------------------------------------------------
// Kernels of the batch pipeline.

// Order-preserving 64-bit key of a double.
__device__ __forceinline__ unsigned long long dkey(double v) {
  const unsigned long long b = (unsigned long long)__double_as_longlong(v);
  return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double dkey_inv(unsigned long long k) {
  const unsigned long long b = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
  return __longlong_as_double((long long)b);
}

// Exact order statistics of every image (the entries a sort would put at
// positions rank_lo and rank_hi, vec.h:864-871) by MSD radix selection with
// 8-bit digits; one CTA per image, both ranks selected together.
constexpr int kSelThreads = 1024;
__global__ void __launch_bounds__(kSelThreads) k_select2(const double* __restrict__ img, size_t stride, int count,
                                                       int rank_lo, int rank_hi, double* out /* [2*i] */) {
  __shared__ unsigned int hist[2][256];
  __shared__ unsigned long long prefix[2];
  __shared__ int kk[2];
  const double* a = img + (size_t)blockIdx.x * stride;
  if (threadIdx.x == 0) {
    prefix[0] = prefix[1] = 0ull;
    kk[0] = rank_lo;
    kk[1] = rank_hi;
  }
  for (int pass = 0; pass < 8; ++pass) {
    const int shift = 56 - 8 * pass;
    for (int i = threadIdx.x; i < 512; i += kSelThreads) (&hist[0][0])[i] = 0u;
    __syncthreads();
    const unsigned long long mask = (pass == 0) ? 0ull : (~0ull << (shift + 8));
    const unsigned long long p0 = prefix[0], p1 = prefix[1];
    for (int i = threadIdx.x; i < count; i += kSelThreads) {
      const unsigned long long k = dkey(a[i]);
      const unsigned d = (unsigned)((k >> shift) & 0xffu);
      if ((k & mask) == p0) atomicAdd(&hist[0][d], 1u);
      if ((k & mask) == p1) atomicAdd(&hist[1][d], 1u);
    }
    __syncthreads();
    if (threadIdx.x < 2) {
      const int s = threadIdx.x;
      int k = kk[s];
      unsigned acc = 0;
      int b = 0;
      for (; b < 256; ++b) {
        if (acc + hist[s][b] > (unsigned)k) break;
        acc += hist[s][b];
      }
      kk[s] = k - (int)acc;
      prefix[s] |= ((unsigned long long)b) << shift;
    }
    __syncthreads();
  }
  if (threadIdx.x < 2) out[2 * blockIdx.x + threadIdx.x] = dkey_inv(prefix[threadIdx.x]);
}

// Sets *flag when an image holds NaN or Inf.  The reference sorts such an
// image for its saturated min/max (vec.h:864-871), whose result is then
// unspecified, so the synchronous entry points refuse it after the call.
__global__ void k_finite_check(const double* __restrict__ img, size_t stride, int count, int* flag) {
  const double* a = img + (size_t)blockIdx.y * stride;
  bool bad = false;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    const double v = a[i];
    bad |= !(fabs(v) <= 1.7976931348623157e308);
  }
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicOr(flag, 1);
}

// min and max of every image (deterministic: min/max are order independent).
__global__ void __launch_bounds__(1024) k_minmax(const double* __restrict__ img, size_t stride, int count,
                                                 double* out) {
  __shared__ double smn[32], smx[32];
  const double* a = img + (size_t)blockIdx.x * stride;
  double mn = INFINITY, mx = -INFINITY;
  for (int i = threadIdx.x; i < count; i += blockDim.x) {
    const double v = a[i];
    mn = fmin(mn, v);
    mx = fmax(mx, v);
  }
  for (int o = 16; o > 0; o >>= 1) {
    mn = fmin(mn, __shfl_xor_sync(0xffffffffu, mn, o));
    mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  }
  if ((threadIdx.x & 31) == 0) { smn[threadIdx.x >> 5] = mn; smx[threadIdx.x >> 5] = mx; }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) { mn = fmin(mn, smn[w]); mx = fmax(mx, smx[w]); }
    mn = fmin(mn, smn[0]);
    mx = fmax(mx, smx[0]);
    out[2 * blockIdx.x] = mn;
    out[2 * blockIdx.x + 1] = mx;
  }
}

// prepareMultilevelArray scaling (registration.h:335-346).
//   sat >= 0 : x = clamp(x, lo, hi); x += -lo; x /= (hi + -lo) unless 0
//   sat <  0 : if (mn < 0 || min_to_zero) x += -mn; x /= max unless 0
__global__ void k_normalize(double* img, size_t stride, int count, const double* mm, int sat_mode,
                            int min_to_zero) {
  const int b = blockIdx.y;
  double* a = img + (size_t)b * stride;
  const double lo = mm[2 * b], hi = mm[2 * b + 1];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    double v = a[i];
    if (sat_mode) {
      v = v < lo ? lo : (v > hi ? hi : v);
      const double s = -1 * lo;
      v += s;
      const double mx = hi + s;
      if (mx != 0) v /= mx;
    } else {
      double mx = hi;
      if (lo < 0. || min_to_zero) {
        v += -lo;
        mx = hi + -lo;
      }
      if (mx != 0.) v /= mx;
    }
    a[i] = v;
  }
}

// One restriction step for a batch of images: coarse[b] = R fine[b].
template <typename T>
__global__ void k_restrict(const T* __restrict__ fine, size_t fstride, T* coarse, size_t cstride, int fine_level) {
  const int fw = lvl_n(fine_level), cw = lvl_n(fine_level - 1);
  const T* f = fine + (size_t)blockIdx.y * fstride;
  T* c = coarse + (size_t)blockIdx.y * cstride;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < cw * cw; i += gridDim.x * blockDim.x) {
    c[i] = restrict_node<T>(i % cw, i / cw, cw, [&](int x, int y) { return f[(size_t)y * fw + x]; });
  }
}

template <typename T>
__global__ void k_prolong(const T* __restrict__ coarse, size_t cstride, T* fine, size_t fstride, int coarse_level) {
  const int cw = lvl_n(coarse_level), fw = lvl_n(coarse_level + 1);
  const T* c = coarse + (size_t)blockIdx.y * cstride;
  T* f = fine + (size_t)blockIdx.y * fstride;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < fw * fw; i += gridDim.x * blockDim.x) {
    f[i] = prolong_node<T>(i % fw, i / fw, [&](int x, int y) { return c[(size_t)y * cw + x]; });
  }
}

template <typename Src, typename Dst>
__global__ void k_convert(const Src* __restrict__ src, size_t sstride, Dst* dst, size_t dstride, size_t count) {
  const Src* s = src + (size_t)blockIdx.y * sstride;
  Dst* d = dst + (size_t)blockIdx.y * dstride;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x)
    d[i] = (Dst)s[i];
}

// Dense n x n images (batch) <-> pitched rows of pitch_of(n) elements.
template <typename Src, typename Dst>
__global__ void k_to_pitched(const Src* __restrict__ src, size_t sstride, Dst* dst, size_t dstride, int n) {
  const Src* s = src + (size_t)blockIdx.y * sstride;
  Dst* d = dst + (size_t)blockIdx.y * dstride;
  const int P = pitch_of(n);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n * n; i += gridDim.x * blockDim.x)
    d[(size_t)(i / n) * P + (i % n)] = (Dst)s[i];
}
template <typename Src, typename Dst>
__global__ void k_from_pitched(const Src* __restrict__ src, size_t sstride, Dst* dst, size_t dstride, int n) {
  const Src* s = src + (size_t)blockIdx.y * sstride;
  Dst* d = dst + (size_t)blockIdx.y * dstride;
  const int P = pitch_of(n);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n * n; i += gridDim.x * blockDim.x)
    d[i] = (Dst)s[(size_t)(i / n) * P + (i % n)];
}

// Displacement transfer to the next level for every instance: reads the
// buffer bin[i], writes buffer bin[i]^1 and records it in bout[i].
// mode 0: ProlongOp (prolongation.cpp:195-232); mode 1: 1-D resampling of the
// flattened node vector (vec.h:461-472, 565-570; registration.h:510-516).
template <typename Real>
__global__ void k_phi_up(Real* arena, size_t inst_stride, size_t off0, size_t off1, int coarse_level,
                         const int* bin, int* bout, int mode) {
  const int inst = blockIdx.y;
  const int b = bin[inst];
  Real* base = arena + (size_t)inst * inst_stride;
  const Real* src = base + (b ? off1 : off0);
  Real* dst = base + (b ? off0 : off1);
  const int cw = lvl_n(coarse_level), fw = lvl_n(coarse_level + 1);
  const int cP = pitch_of(cw), fP = pitch_of(fw);
  const size_t cs_src = comp_stride(coarse_level), cs_dst = comp_stride(coarse_level + 1);
  const int ns = cw * cw, nd = fw * fw;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nd; i += gridDim.x * blockDim.x) {
    const int x = i % fw, y = i / fw;
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      const Real* s = src + (size_t)c * cs_src;
      Real v;
      if (mode == 0) {
        v = prolong_node<Real>(x, y, [&](int X, int Y) { return s[(size_t)Y * cP + X]; });
      } else {
        // dense (flattened) node index of the coarse vector
        auto at = [&](int q) { return s[(size_t)(q / cw) * cP + (q % cw)]; };
        const double sc = (ns - 1) / (double)(nd - 1);
        const double pos = i * sc;
        const int p = (int)pos;
        const double pf = pos - p;
        v = (p == ns - 1) ? at(p) : (Real)((1 - pf) * (double)at(p) + pf * (double)at(p + 1));
      }
      dst[(size_t)c * cs_dst + (size_t)y * fP + x] = v;
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) bout[inst] = b ^ 1;
}

template <typename Real>
__global__ void k_set_buf(int* buf, int n, int v) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) buf[i] = v;
}

// normalizeImageForNCC of the reference image of a level by one CTA
// (registration.h:1932-1944): u = R - sum_i (M R)_i, var = sqrt(u . M u),
// out = u / var (u when var is within 1e-15 of 0).  Sums are deterministic
// (fixed thread assignment, warps reduced in order).
// One block per reference: block 0 normalises R0 into out0; with pairwise
// references block b > 0 normalises the template of instance b - 1 (at
// arena + (b-1)*inst_stride + off_T) into out0 + b*out_stride; with inst_ref
// (ragged batches) block b normalises R0 + inst_ref[b]*ref_stride.
template <typename Real>
__global__ void k_ncc_normalize(const Real* __restrict__ R0, const Real* __restrict__ arena, size_t inst_stride,
                                size_t off_T, int level, Real* out0, size_t out_stride,
                                const int* inst_ref = nullptr, size_t ref_stride = 0) {
  const Real* __restrict__ R = inst_ref ? R0 + (size_t)inst_ref[blockIdx.x] * ref_stride
                               : (blockIdx.x == 0 ? R0 : arena + (size_t)(blockIdx.x - 1) * inst_stride + off_T);
  Real* out = out0 + (size_t)blockIdx.x * out_stride;
  const int n = lvl_n(level), P = pitch_of(n), N = n * n;
  const Real h = (Real)(1.0 / (double)(n - 1)), hh = h * h;
  __shared__ double red[32];
  __shared__ double val;
  auto block_sum = [&](double v) -> double {
    v = warp_sum(v);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
      val = t;
    }
    __syncthreads();
    return val;
  };
  double acc = 0.0;
  for (int i = threadIdx.x; i < N; i += blockDim.x) {
    const int x = i % n, y = i / n;
    acc += (double)mass_row<Real>(x, y, n, hh, [&](int X, int Y) { return R[(size_t)Y * P + X]; });
  }
  const Real m = (Real)(-block_sum(acc));
  for (int i = threadIdx.x; i < N; i += blockDim.x) {
    const size_t g = (size_t)(i / n) * P + (i % n);
    Real u = R[g];
    u += m;
    out[g] = u;
  }
  __syncthreads();
  acc = 0.0;
  for (int i = threadIdx.x; i < N; i += blockDim.x) {
    const int x = i % n, y = i / n;
    const Real mu = mass_row<Real>(x, y, n, hh, [&](int X, int Y) { return out[(size_t)Y * P + X]; });
    acc += (double)(out[(size_t)y * P + x] * mu);
  }
  const double var = sqrt(block_sum(acc));
  if (!(fabs(var - 0.0) < 1e-15)) {
    const Real v = (Real)var;
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
      const size_t g = (size_t)(i / n) * P + (i % n);
      out[g] /= v;
    }
  }
}

// phi of every instance at the given level -> double output (F x 2 x N, dense).
template <typename Real>
__global__ void k_phi_out(const Real* arena, size_t inst_stride, size_t off0, size_t off1, int level,
                          const int* buf, double* out) {
  const int inst = blockIdx.y;
  const int n = lvl_n(level), P = pitch_of(n);
  const int N = n * n;
  const size_t cs = comp_stride(level);
  const Real* src = arena + (size_t)inst * inst_stride + (buf[inst] ? off1 : off0);
  double* o = out + (size_t)inst * 2 * N;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    const size_t g = (size_t)(i / n) * P + (i % n);
    o[i] = (double)src[g];
    o[N + i] = (double)src[cs + g];
  }
}

// Energy/steps outputs of the last level solve.
__global__ void k_collect(const double* e, const int* s, int num, double* e_out, int* s_out, int s_stride,
                          int s_col) {
  for (int i = threadIdx.x; i < num; i += blockDim.x) {
    if (e_out) e_out[i] = e[i];
    if (s_out) s_out[(size_t)i * s_stride + s_col] = s[i];
  }
}

// Warped-frame average: DeformImage with Inf extension per frame
// (deformations.h:62-101), mean over finite samples (matchSeries.h:410-425).
__global__ void k_warp_mean(const double* __restrict__ frames, const double* __restrict__ phis, int F, int level,
                            const double* last_mean, double* mean, double* count) {
  const int n = lvl_n(level);
  const int N = n * n;
  const double h = 1.0 / (double)(n - 1);
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < N; j += gridDim.x * blockDim.x) {
    const int x = j % n, y = j / n;
    double acc = 0;
    int k = 0;
    for (int f = 0; f < F; ++f) {
      const double* ph = phis + (size_t)f * 2 * N;
      const double d0 = x + ph[j] / h, d1 = y + ph[N + j] / h;
      bool in = true;
      if (d0 < 0. || d0 > (double)(n - 1) || isnan(d0)) in = false;
      if (d1 < 0. || d1 > (double)(n - 1) || isnan(d1)) in = false;
      const double v = in ? interp_d(frames + (size_t)f * N, n, d0, d1) : INFINITY;
      if (v != INFINITY) {
        acc += v;
        ++k;
      }
    }
    mean[j] = (k > 0) ? acc / k : *last_mean;
    count[j] = k;
  }
}

// The per-rank part of the average of a sharded stage: per pixel the sum of
// the finite warped samples of this rank's frames (in frame order) and their
// number, as k_warp_mean accumulates them (averageSeries, matchSeries.h:
// 410-425); the ranks' sums and counts are then added by one all-reduce.
__global__ void k_warp_sum(const double* __restrict__ frames, const double* __restrict__ phis, int F, int level,
                           double* sum, double* count) {
  const int n = lvl_n(level);
  const int N = n * n;
  const double h = 1.0 / (double)(n - 1);
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < N; j += gridDim.x * blockDim.x) {
    const int x = j % n, y = j / n;
    double acc = 0;
    int k = 0;
    for (int f = 0; f < F; ++f) {
      const double* ph = phis + (size_t)f * 2 * N;
      const double d0 = x + ph[j] / h, d1 = y + ph[N + j] / h;
      bool in = true;
      if (d0 < 0. || d0 > (double)(n - 1) || isnan(d0)) in = false;
      if (d1 < 0. || d1 > (double)(n - 1) || isnan(d1)) in = false;
      const double v = in ? interp_d(frames + (size_t)f * N, n, d0, d1) : INFINITY;
      if (v != INFINITY) {
        acc += v;
        ++k;
      }
    }
    sum[j] = acc;
    count[j] = k;
  }
}

// mean = sum / count where a pixel has samples, else *fill.
__global__ void k_mean_from_sums(const double* sum, const double* count, int N, const double* fill, double* mean) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < N; j += gridDim.x * blockDim.x) {
    const double k = count[j];
    mean[j] = (k > 0) ? sum[j] / k : *fill;
  }
}

__global__ void k_mean(const double* a, int N, double* out) {
  __shared__ double sm[32];
  double s = 0;
  for (int i = threadIdx.x; i < N; i += blockDim.x) s += a[i];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sm[w];
    *out = t / N;
  }
}

// ---------------------------------------------------------------------------
// Arena layout of one registration instance (elements of Real), sized for
// the precision level M.
struct Layout {
  size_t off_T[kMaxLevel + 1];
  size_t off_phi[2], off_d[2], off_s, off_de;
  size_t off_td;   // NCC only: deformed template at the nodes
  size_t off_nr;   // NCC with pairwise references only: the instance's normalised reference
  size_t off_x2[kMaxLevel + 1], off_x5[kMaxLevel + 1], off_b[kMaxLevel + 1];
  size_t stride;
};

Layout make_layout(int M, bool ncc = false, bool pairwise = false) {
  Layout L;
  size_t off = 0;
  const size_t a = 64;
  for (int l = 0; l <= M; ++l) { L.off_T[l] = off; off = align_up(off + comp_stride(l), a); }
  for (int l = M + 1; l <= kMaxLevel; ++l) L.off_T[l] = 0;
  const size_t two = 2 * comp_stride(M);
  for (int b = 0; b < 2; ++b) { L.off_phi[b] = off; off = align_up(off + two, a); }
  for (int b = 0; b < 2; ++b) { L.off_d[b] = off; off = align_up(off + two, a); }
  L.off_s = off; off = align_up(off + two, a);
  L.off_de = off; off = align_up(off + two, a);
  L.off_td = 0;
  if (ncc) { L.off_td = off; off = align_up(off + comp_stride(M), a); }
  L.off_nr = 0;
  if (ncc && pairwise) { L.off_nr = off; off = align_up(off + comp_stride(M), a); }
  for (int k = 0; k <= kMaxLevel; ++k) {
    if (k <= M) {
      L.off_x2[k] = off; off = align_up(off + 2 * comp_stride(k), a);
      L.off_x5[k] = off; off = align_up(off + 2 * comp_stride(k), a);
      L.off_b[k] = off; off = align_up(off + 2 * comp_stride(k), a);
    } else {
      L.off_x2[k] = L.off_x5[k] = L.off_b[k] = 0;
    }
  }
  L.stride = off;
  return L;
}

template <typename Real>
size_t level_smem_bytes(int lc) {
  return align_up(level_smem_elems(lc) * sizeof(Real), 128);
}

template <typename Real>
int pick_lc(int level) {
  return std::min(level, 5);
}

// Largest number of tiles of any pass of a level (the per-tile partial sums
// of one instance).
int level_max_tiles(int level) {
  const int e = lvl_n(level) - 1;
  const int el = std::max(1, e / TX) * std::max(1, e / TY);
  const int vt = std::max(1, e / VTX) * std::max(1, e / VTY);
  return std::max(el, vt);
}

// Scheduler state of a level launch: dispenser words, the finished counter,
// per-instance control blocks, per-tile partial sums.
size_t sched_bytes(int num_inst, int max_tiles) {
  return align_up(sizeof(unsigned long long) * kWordStride * (size_t)num_inst, 256) + 256 +
         align_up(sizeof(InstCtl) * (size_t)num_inst, 256) +
         align_up(sizeof(double) * kRedSlots * (size_t)max_tiles * num_inst, 256);
}

template <typename Real>
SchedPtrs<Real> carve_sched(void* mem, int num_inst, int max_tiles, size_t* zero_bytes) {
  unsigned char* p = (unsigned char*)mem;
  SchedPtrs<Real> sp;
  sp.words = (unsigned long long*)p;
  p += align_up(sizeof(unsigned long long) * kWordStride * (size_t)num_inst, 256);
  sp.finished = (int*)p;
  sp.error = nullptr;
  p += 256;
  *zero_bytes = (size_t)(p - (unsigned char*)mem);
  sp.ctl = (InstCtl*)p;
  p += align_up(sizeof(InstCtl) * (size_t)num_inst, 256);
  sp.partials = (double*)p;
  sp.max_tiles = max_tiles;
  return sp;
}

// Launches the level kernel as a cooperative grid (every CTA resident, two
// per SM where registers and shared memory allow); sched_mem holds
// sched_bytes(a.num_inst, level_max_tiles(a.level)) bytes.
// error_flag: device int, set by a worker that gave up waiting for work; it
// is cleared by the caller at the start of an API call, not per launch.
template <typename Real>
cudaError_t launch_level_core(LevelArgs<Real>& a, void* sched_mem, int* error_flag, int sms, cudaStream_t st,
                              int* grid_out, int want_per_sm = 0) {
  const int max_tiles = level_max_tiles(a.level);
  a.idle_ns = g_level_wait_ns.load();
  if (a.chunk_div <= 0) a.chunk_div = kChunkDiv;
  if (a.chunk_max <= 0) a.chunk_max = kChunkMax;
  size_t zb = 0;
  SchedPtrs<Real> sp = carve_sched<Real>(sched_mem, a.num_inst, max_tiles, &zb);
  sp.error = error_flag;
  cudaError_t e = cudaMemsetAsync(sched_mem, 0, zb, st);
  if (e != cudaSuccess) return e;
  const size_t smem = level_smem_bytes<Real>(a.lc);
  // the kernel variant that carries only the passes this launch runs
  void (*kern)(LevelArgs<Real>, SchedPtrs<Real>) =
      a.ncc ? level_kernel<Real, kKmAny> : (a.xs ? level_kernel<Real, kKmSsdExact> : level_kernel<Real, kKmSsd>);
  e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads, smem);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  if (want_per_sm > 0 && want_per_sm < per_sm) per_sm = want_per_sm;
  const int grid = per_sm * sms;
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.gridDim = dim3(grid, 1, 1);
  cfg.blockDim = dim3(kThreads, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if (grid_out) *grid_out = grid;
  return cudaLaunchKernelEx(&cfg, kern, a, sp);
}

template <typename Real>
int launch_level(msgpu_context* ctx, LevelArgs<Real>& a, cudaStream_t st) {
  int rc;
  if ((rc = ensure(ctx, ctx->sched, sched_bytes(a.num_inst, level_max_tiles(a.level))))) return rc;
  const msgpu_level_tuning& t = ctx->tuning[sizeof(Real) == 8 ? 1 : 0][a.level];
  a.chunk_div = t.chunk_div;
  a.chunk_max = t.chunk_max;
  CK(launch_level_core<Real>(a, ctx->sched.p, ctx->sched_error, ctx->sm_count, st, &ctx->last_grid,
                             t.ctas_per_sm));
  return MSGPU_OK;
}

// Pass timeline of a profiled level launch (msgpu_set_trace): the event
// buffer when the launch's level is the traced one, and the events copied
// to the host after it.
template <typename Real>
int trace_attach(msgpu_context* ctx, LevelArgs<Real>& a, cudaStream_t st) {
  if (!ctx->profiling || a.level != ctx->trace_level || ctx->trace_cap == 0) return MSGPU_OK;
  int rc;
  const size_t tb = sizeof(unsigned long long) * 2 * (size_t)ctx->trace_cap;
  if ((rc = ensure(ctx, ctx->trace, tb + 16))) return rc;
  a.tl = (unsigned long long*)ctx->trace.p;
  a.tl_n = (unsigned int*)((char*)ctx->trace.p + tb);
  a.tl_cap = ctx->trace_cap;
  CK(cudaMemsetAsync(a.tl_n, 0, 16, st));
  return MSGPU_OK;
}
template <typename Real>
int trace_collect(msgpu_context* ctx, const LevelArgs<Real>& a, cudaStream_t st) {
  if (!a.tl) return MSGPU_OK;
  unsigned cnt = 0;
  CK(cudaMemcpyAsync(&cnt, a.tl_n, sizeof(cnt), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  cnt = std::min(cnt, a.tl_cap);
  ctx->trace_host.resize(2 * (size_t)cnt);
  if (cnt) CK(cudaMemcpy(ctx->trace_host.data(), a.tl, sizeof(unsigned long long) * 2 * cnt, cudaMemcpyDeviceToHost));
  return MSGPU_OK;
}

// Exact sums of a level launch (FP64, SSD, sum order 0): per instance
// xs_bufs term buffers of XsLayout(n).stride doubles and (xs_bufs > 1) the
// per-tile bound sums of its energy passes.  kXsBufs buffers let a control
// step be taken on bounded sums while the values that may still need their
// ordered sums keep their terms (certified steps); one buffer (certified
// steps off, or more memory than kXsCertBytes) adds every pass's sums in order
// before its control step.  Otherwise the launch adds its sums in the fixed
// parallel order of the tile partials.
constexpr size_t kXsCertBytes = 32ull << 30;
template <typename Real>
int xs_attach(msgpu_context* ctx, LevelArgs<Real>& a, bool exact, int max_level, int num_inst) {
  a.xs = nullptr;
  a.xs_stride = 0;
  a.xs_bufs = 1;
  a.xpart = nullptr;
  a.xpart_stride = 0;
  if (!exact || !std::is_same<Real, double>::value || a.ncc) return MSGPU_OK;
  int rc;
  const size_t stride = XsLayout(lvl_n(max_level)).stride;
  const size_t xps = (size_t)level_max_tiles(max_level) * kXpSlots;
  int nb = ctx->certified ? kXsBufs : 1;
  if (nb > 1 && sizeof(double) * (stride * nb + xps) * (size_t)num_inst > kXsCertBytes) nb = 1;
  if ((rc = ensure(ctx, ctx->xsum, sizeof(double) * stride * nb * (size_t)num_inst))) return rc;
  if (nb > 1) {
    if ((rc = ensure(ctx, ctx->xpart, sizeof(double) * xps * (size_t)num_inst))) return rc;
    a.xpart = (double*)ctx->xpart.p;
    a.xpart_stride = (size_t)level_max_tiles(a.level) * kXpSlots;
  }
  a.xs = (double*)ctx->xsum.p;
  a.xs_stride = XsLayout(a.n).stride;
  a.xs_bufs = nb;
  return MSGPU_OK;
}

// Clears the error flags at the start of an API call: word 0 is set by a
// level-kernel worker that gave up waiting for work, word 1 by the
// composition kernel when a grid-barrier wait gave up.
int sched_error_reset(msgpu_context* ctx, cudaStream_t st) {
  int rc;
  if (!ctx->sched_error) {
    if ((rc = ensure(ctx, ctx->flags, 256))) return rc;
    ctx->sched_error = (int*)ctx->flags.p;
  }
  CK(cudaMemsetAsync(ctx->sched_error, 0, 4 * sizeof(int), st));
  return MSGPU_OK;
}

// After the call's work has completed: reports a kernel that gave up waiting
// and input images holding NaN or Inf (word 2, set by k_finite_check).
int sched_error_check(msgpu_context* ctx) {
  int h[4] = {0, 0, 0, 0};
  if (!ctx->sched_error) return MSGPU_OK;
  CK(cudaMemcpy(h, ctx->sched_error, sizeof(h), cudaMemcpyDeviceToHost));
  if (h[0] == 2) return fail(ctx, MSGPU_ERR_CUDA, "level kernel: exact-sum bookkeeping failed (no free term buffer)");
  if (h[0]) return fail(ctx, MSGPU_ERR_CUDA, "level kernel: a worker waited too long for work (scheduler stalled)");
  if (h[1]) return fail(ctx, MSGPU_ERR_CUDA, "composition: a grid-barrier wait timed out");
  if (h[2]) return fail(ctx, MSGPU_ERR_INVALID_ARG, "an input image holds a non-finite value (NaN or Inf)");
  if (h[3]) return fail(ctx, MSGPU_ERR_CUDA, "tensor-core convolution: a wait for the tensor core timed out");
  return MSGPU_OK;
}

// Upper bound on the CTAs of a level launch (for the per-CTA pass counters).
int max_level_grid(int sms) { return 4 * sms; }

// Image preparation of prepareMultilevelArray (registration.h:331-367) on
// nimg images already copied to their pyramid rows at the input level:
// exact saturated min/max by radix selection, clamp, scale to [0,1]
// (vec.h:864-871, 1084-1089), then RestrictOp<STD_QUOC_RESTRICT> down to
// level 0 (multilevelArray.h:94-110).  mm: 2 * nimg doubles of scratch.
int prepare_pyramid(msgpu_context* ctx, const msgpu_params& p, double* pyr, const std::vector<size_t>& poff,
                    size_t pstride, int nimg, double* mm, cudaStream_t st) {
  const int Lin = p.input_level;
  const size_t Nin = lvl_N(Lin);
  int& launches = ctx->stats.kernel_launches;
  if (ctx->sched_error) {
    k_finite_check<<<dim3((unsigned)std::min<size_t>(256, (Nin + 255) / 256), nimg), 256, 0, st>>>(
        pyr + poff[Lin], pstride, (int)Nin, ctx->sched_error + 2);
    ++launches;
  }
  if (!p.dont_normalize_input) {
    if (p.saturation_percent >= 0) {
      const int m1 = (int)Nin - 1;
      int il = (int)(p.saturation_percent / 200 * m1), ih = (int)((1 - p.saturation_percent / 200) * m1);
      il = std::min(std::max(il, 0), m1);
      ih = std::min(std::max(ih, 0), m1);
      k_select2<<<nimg, kSelThreads, 0, st>>>(pyr + poff[Lin], pstride, (int)Nin, il, ih, mm);
    } else {
      k_minmax<<<nimg, 1024, 0, st>>>(pyr + poff[Lin], pstride, (int)Nin, mm);
    }
    CK(cudaGetLastError());
    k_normalize<<<dim3((unsigned)std::min<size_t>(1024, (Nin + 255) / 256), nimg), 256, 0, st>>>(
        pyr + poff[Lin], pstride, (int)Nin, mm, p.saturation_percent >= 0 ? 1 : 0, p.normalize_min_to_zero);
    CK(cudaGetLastError());
    launches += 2;
  }
  for (int l = Lin; l >= 1; --l) {
    const size_t cN = lvl_N(l - 1);
    k_restrict<double><<<dim3((unsigned)std::min<size_t>(1024, (cN + 255) / 256), nimg), 256, 0, st>>>(
        pyr + poff[l], pstride, pyr + poff[l - 1], pstride, l);
    ++launches;
  }
  CK(cudaGetLastError());
  return MSGPU_OK;
}

// Pyramid rows of images at input level Lin: offsets of the levels (finest
// first) and the row stride, in doubles.
size_t pyramid_layout(int Lin, std::vector<size_t>& poff) {
  poff.assign(Lin + 1, 0);
  size_t pstride = 0;
  for (int l = Lin; l >= 0; --l) { poff[l] = pstride; pstride = align_up(pstride + lvl_N(l), 32); }
  return pstride;
}

// ---------------------------------------------------------------------------
struct BatchIO {
  const double* ref;        // device, input level
  const double* tmpl;       // device, F images at input level
  const double* init_phi;   // device, F x 2 x N_M or null
  double* phis_out;         // device, F x 2 x N_M
  double* energies_out;     // device or null
  int* steps_out;           // device or null
};

// Options of a batch beyond the parameter file.
struct BatchOpts {
  int pairwise = 0;      // template i > 0 is registered to template i - 1 (series matching, matchSeries.h:141-155)
  int lambda_stop = -1;  // level that lambdaFactor's exponent counts from (default: stop_level)
  int reset_error = 1;   // clear the error flags (0: a caller running several batches clears them once)
  msgpu_net* warm = nullptr;   // learned warm start: the network's prediction is the start-level displacement
  const double* e_target = nullptr;   // device, per frame: stop the stop-level solve at this energy (+ e_tol)
  double e_tol = 0.0;
  int max_iter_stop = 0;              // > 0: step limit of the stop level (with energy targets)
  int max_iter_below = 0;             // > 0: step limit of the levels below the stop level
};

int warm_start_phi(msgpu_net* net, const double* pyr, const std::vector<size_t>& poff, size_t pstride, int F,
                   cudaStream_t st, double** phi);

template <typename Real>
int run_batch(msgpu_context* ctx, const msgpu_params& p, int F, const BatchIO& io, cudaStream_t st,
              const BatchOpts& opt = BatchOpts()) {
  const int M = p.precision_level, Lin = p.input_level;
  const int start = p.start_level, stop = p.stop_level;
  const int lambda_stop = opt.lambda_stop >= 0 ? opt.lambda_stop : stop;
  const int nimg = F + 1;  // image 0 is the reference
  const size_t Nin = lvl_N(Lin);
  const bool ncc = p.data_term == 1;
  const bool pairwise = opt.pairwise != 0 && F > 1;
  const Layout L = make_layout(M, ncc, pairwise);
  int rc;
  if ((rc = ensure_tables(ctx))) return rc;
  if (opt.reset_error && (rc = sched_error_reset(ctx, st))) return rc;
  if (ncc && (rc = ensure(ctx, ctx->nccbuf, sizeof(Real) * (comp_stride(M) + 64)))) return rc;
  // --- double scratch: per image a pyramid from Lin down to 0
  std::vector<size_t> poff;
  const size_t pstride = pyramid_layout(Lin, poff);
  const int nlev_all = stop - start + 1;
  const size_t small_bytes = sizeof(double) * (2 * nimg + 2 * F + 64) + sizeof(int) * ((2 * nlev_all + 4) * F + 64);
  if ((rc = ensure(ctx, ctx->dscratch, sizeof(double) * pstride * nimg))) return rc;
  if ((rc = ensure(ctx, ctx->arena, sizeof(Real) * L.stride * F))) return rc;
  if ((rc = ensure(ctx, ctx->shared_real, sizeof(Real) * (L.off_T[M] + comp_stride(M) + 64)))) return rc;
  if ((rc = ensure(ctx, ctx->small, small_bytes))) return rc;
  double* pyr = (double*)ctx->dscratch.p;
  Real* arena = (Real*)ctx->arena.p;
  Real* Rpyr = (Real*)ctx->shared_real.p;
  double* mm = (double*)ctx->small.p;                 // 2 * nimg
  double* e_lvl = mm + 2 * nimg;                      // F
  int* ibase = (int*)(e_lvl + 2 * F + 64);
  int* bufA = ibase;                                  // F
  int* bufB = ibase + F;                              // F
  int* steps_all = ibase + 2 * F;                     // nlev x F
  int* evals_all = steps_all + (size_t)nlev_all * F;  // nlev x F
  int& launches = ctx->stats.kernel_launches;
  launches = 0;
  ctx->stats.num_levels = nlev_all;
  ctx->stats.first_level = start;
  if (ctx->profiling && !ctx->ev_ready) {
    for (int i = 0; i < 32; ++i) CK(cudaEventCreate(&ctx->ev[i]));
    ctx->ev_ready = true;
  }

  // 1. copy inputs into the pyramid scratch and prepare (normalise) them
  CK(cudaMemcpy2DAsync(pyr + poff[Lin], pstride * sizeof(double), io.ref, Nin * sizeof(double),
                       Nin * sizeof(double), 1, cudaMemcpyDeviceToDevice, st));
  CK(cudaMemcpy2DAsync(pyr + pstride + poff[Lin], pstride * sizeof(double), io.tmpl, Nin * sizeof(double),
                       Nin * sizeof(double), F, cudaMemcpyDeviceToDevice, st));
  if ((rc = prepare_pyramid(ctx, p, pyr, poff, pstride, nimg, mm, st))) return rc;
  // 2. Real copies of the levels 0..M
  CK(cudaGetLastError());
  for (int l = 0; l <= M; ++l) {
    const size_t Nl = lvl_N(l);
    const unsigned gx = (unsigned)std::min<size_t>(1024, (Nl + 255) / 256);
    k_to_pitched<double, Real><<<dim3(gx, 1), 256, 0, st>>>(pyr + poff[l], 0, Rpyr + L.off_T[l], 0, lvl_n(l));
    k_to_pitched<double, Real><<<dim3(gx, F), 256, 0, st>>>(pyr + pstride + poff[l], pstride, arena + L.off_T[l],
                                                             L.stride, lvl_n(l));
    launches += 2;
  }
  CK(cudaGetLastError());
  // 3. initial displacement at the start level (restricted from M), buffer 0
  k_set_buf<Real><<<1, 256, 0, st>>>(bufA, F, 0);
  ++launches;
  {
    const size_t Ns = lvl_N(start);
    if (opt.warm) {
      double* wphi;
      if ((rc = warm_start_phi(opt.warm, pyr, poff, pstride, F, st, &wphi))) return rc;
      for (int c = 0; c < 2; ++c)
        k_to_pitched<double, Real><<<dim3((unsigned)std::min<size_t>(1024, (Ns + 255) / 256), F), 256, 0, st>>>(
            wphi + (size_t)c * Ns, 2 * Ns, arena + L.off_phi[0] + (size_t)c * comp_stride(start), L.stride,
            lvl_n(start));
      launches += 2;
    } else if (io.init_phi) {
      // restrict the initial displacement in double inside the template pyramid scratch of level < M
      // storage: reuse the double scratch rows of the templates (already converted)
      double* tmp = pyr + pstride;  // F images, 2 components need 2F slots: use pairs of images
      for (int c = 0; c < 2; ++c) {
        const size_t NM = lvl_N(M);
        CK(cudaMemcpy2DAsync(tmp + poff[M], pstride * sizeof(double), io.init_phi + (size_t)c * NM,
                             2 * NM * sizeof(double), NM * sizeof(double), F, cudaMemcpyDeviceToDevice, st));
        for (int l = M; l > start; --l) {
          const size_t cN = lvl_N(l - 1);
          k_restrict<double><<<dim3((unsigned)std::min<size_t>(1024, (cN + 255) / 256), F), 256, 0, st>>>(
              tmp + poff[l], pstride, tmp + poff[l - 1], pstride, l);
        }
        k_to_pitched<double, Real><<<dim3((unsigned)std::min<size_t>(1024, (Ns + 255) / 256), F), 256, 0, st>>>(
            tmp + poff[start], pstride, arena + L.off_phi[0] + (size_t)c * comp_stride(start), L.stride,
            lvl_n(start));
      }
    } else {
      CK(cudaMemset2DAsync(arena + L.off_phi[0], L.stride * sizeof(Real), 0, 2 * comp_stride(start) * sizeof(Real),
                           F, st));
    }
  }
  CK(cudaGetLastError());
  // 4. level loop
  int* bin = bufA;
  int* bout = bufB;
  const int nlev = stop - start + 1;
  for (int l = start; l <= stop; ++l) {
    LevelArgs<Real> a;
    memset(&a, 0, sizeof(a));
    a.arena = arena;
    a.inst_stride = L.stride;
    a.R = Rpyr + L.off_T[l];
    a.r_prev = pairwise ? 1 : 0;
    if (ncc) {
      a.ncc = 1;
      a.normR = (const Real*)ctx->nccbuf.p;
      a.off_td = L.off_td;
      a.off_nr = L.off_nr;
      if (pairwise)
        k_ncc_normalize<Real><<<F, 1024, 0, st>>>(a.R, arena, L.stride, L.off_T[l], l, arena + L.off_nr, L.stride);
      else
        k_ncc_normalize<Real><<<1, 1024, 0, st>>>(a.R, arena, L.stride, L.off_T[l], l, (Real*)ctx->nccbuf.p, 0);
      ++launches;
    }
    a.off_T = L.off_T[l];
    a.off_phi[0] = L.off_phi[0];
    a.off_phi[1] = L.off_phi[1];
    a.off_d[0] = L.off_d[0];
    a.off_d[1] = L.off_d[1];
    a.off_s = L.off_s;
    a.off_de = L.off_de;
    for (int k = 0; k <= kMaxLevel; ++k) { a.off_x2[k] = L.off_x2[k]; a.off_x5[k] = L.off_x5[k]; a.off_b[k] = L.off_b[k]; }
    a.level = l;
    a.n = lvl_n(l);
    a.num_inst = F;
    a.lc = pick_lc<Real>(l);
    a.mode = MODE_SOLVE;
    a.lambda = std::pow(p.lambda_factor, (double)(lambda_stop - l)) * p.lambda;
    a.stop_eps = p.stop_epsilon;
    a.max_iter = p.max_gd_iterations;
    a.phi_in_dev = bin;
    a.out_energy = e_lvl;
    a.out_steps = steps_all + (size_t)(l - start) * F;
    a.out_evals = evals_all + (size_t)(l - start) * F;
    a.out_phi_buf = bin;   // the level kernel updates the buffer index in place
    if (l < stop && opt.max_iter_below > 0) a.max_iter = opt.max_iter_below;
    if (l == stop && opt.e_target) {
      a.e_target = opt.e_target;
      a.e_tol = opt.e_tol;
      if (opt.max_iter_stop > 0) a.max_iter = opt.max_iter_stop;
    }
    const size_t prof_n = (size_t)max_level_grid(ctx->sm_count) * kPassKinds;
    if (ctx->profiling) {
      if ((rc = ensure(ctx, ctx->prof, sizeof(unsigned long long) * (prof_n + 8) * nlev_all))) return rc;
      a.pass_cycles = (unsigned long long*)ctx->prof.p + prof_n * (l - start);
      a.xs_prof = (unsigned long long*)ctx->prof.p + prof_n * nlev_all + 8 * (l - start);
      CK(cudaMemsetAsync(a.pass_cycles, 0, sizeof(unsigned long long) * prof_n, st));
      CK(cudaMemsetAsync(a.xs_prof, 0, sizeof(unsigned long long) * 8, st));
      if ((rc = trace_attach<Real>(ctx, a, st))) return rc;
    }
    if ((rc = xs_attach<Real>(ctx, a, p.sum_order == 0, stop, F))) return rc;
    if (ctx->profiling && l - start < 16) CK(cudaEventRecord(ctx->ev[2 * (l - start)], st));
    if ((rc = launch_level<Real>(ctx, a, st))) return rc;
    if ((rc = trace_collect<Real>(ctx, a, st))) return rc;
    if (l - start < 16) ctx->stats.level_cluster[l - start] = ctx->last_grid;
    if (ctx->profiling && l - start < 16) CK(cudaEventRecord(ctx->ev[2 * (l - start) + 1], st));
    k_collect<<<1, 256, 0, st>>>(e_lvl, a.out_steps, F, (l == stop) ? io.energies_out : nullptr, io.steps_out,
                                 nlev, l - start);
    CK(cudaGetLastError());
    launches += 2;
    if (l < stop) {
      const size_t fw = lvl_N(l + 1);
      k_phi_up<Real><<<dim3((unsigned)std::min<size_t>(1024, (fw + 255) / 256), F), 256, 0, st>>>(
          arena, L.stride, L.off_phi[0], L.off_phi[1], l, bin, bout, p.resample_deformation ? 1 : 0);
      CK(cudaGetLastError());
      ++launches;
      std::swap(bin, bout);
    }
  }
  for (int l = stop; l < M; ++l) {
    const size_t fw = lvl_N(l + 1);
    k_phi_up<Real><<<dim3((unsigned)std::min<size_t>(1024, (fw + 255) / 256), F), 256, 0, st>>>(
        arena, L.stride, L.off_phi[0], L.off_phi[1], l, bin, bout, p.resample_deformation ? 1 : 0);
    CK(cudaGetLastError());
    ++launches;
    std::swap(bin, bout);
  }
  const int NM = (int)lvl_N(M);
  k_phi_out<Real><<<dim3((unsigned)std::min(1024, (NM + 255) / 256), F), 256, 0, st>>>(
      arena, L.stride, L.off_phi[0], L.off_phi[1], M, bin, io.phis_out);
  CK(cudaGetLastError());
  ++launches;
  if (ctx->profiling) {
    std::vector<int> hs((size_t)nlev_all * F), he((size_t)nlev_all * F);
    CK(cudaMemcpyAsync(hs.data(), steps_all, sizeof(int) * hs.size(), cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(he.data(), evals_all, sizeof(int) * he.size(), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    for (int k = 0; k < nlev_all && k < 16; ++k) {
      float ms = 0.f;
      CK(cudaEventElapsedTime(&ms, ctx->ev[2 * k], ctx->ev[2 * k + 1]));
      ctx->stats.level_ms[k] = ms;
      long long ss = 0, ee = 0;
      for (int f = 0; f < F; ++f) { ss += hs[(size_t)k * F + f]; ee += he[(size_t)k * F + f]; }
      ctx->stats.level_steps[k] = ss;
      ctx->stats.level_evals[k] = ee;
    }
    const size_t prof_n = (size_t)max_level_grid(ctx->sm_count) * kPassKinds;
    std::vector<unsigned long long> pc(prof_n);
    for (int k = 0; k < nlev_all && k < 16; ++k) {
      CK(cudaMemcpy(pc.data(), (unsigned long long*)ctx->prof.p + prof_n * k, sizeof(unsigned long long) * prof_n,
                    cudaMemcpyDeviceToHost));
      const int nctas = std::min<int>(ctx->stats.level_cluster[k], max_level_grid(ctx->sm_count));
      for (int q = 0; q < kPassKinds && q < 8; ++q) {
        unsigned long long sum = 0;
        for (int c = 0; c < nctas; ++c) sum += pc[(size_t)c * kPassKinds + q];
        const unsigned long long mx = nctas > 0 ? sum / (unsigned long long)nctas : 0ull;
        ctx->stats.level_pass_cycles[k][q] = (long long)mx;
      }
      unsigned long long xp[8];
      CK(cudaMemcpy(xp, (unsigned long long*)ctx->prof.p + prof_n * nlev_all + 8 * k, sizeof(xp),
                    cudaMemcpyDeviceToHost));
      for (int q = 0; q < 8; ++q) ctx->stats.level_xs[k][q] = (long long)xp[q];
    }
  }
  return MSGPU_OK;
}

// The exact sequential sum of the level solve (msgpu_xsum.cuh) on its own,
// for an n x n array of terms in row-major order (a node sum): the terms go
// to the term blocks with their chunk totals, then the three steps run as
// kernels of their own.
__global__ void k_xs_fill(const double* __restrict__ t, int n, XsSum s) {
  const XsGeom g(n);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n * n; i += gridDim.x * blockDim.x) {
    const int y = i / n, x = i - y * n;
    int tx = x / 64;
    if (tx > g.nx - 1) tx = g.nx - 1;
    int ty = y / 8;
    if (ty > g.ny - 1) ty = g.ny - 1;
    xs_block(s, ty * g.nx + tx)[xs_at(x - 64 * tx, y - 8 * ty)] = t[i];
  }
}
__global__ void k_xs_totals(const double* __restrict__ t, int n, XsSum s) {
  const XsGeom g(n);
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n * g.nx; j += gridDim.x * blockDim.x) {
    const int y = j / g.nx, tx = j - y * g.nx;
    const int x0 = 64 * tx, x1 = (tx == g.nx - 1) ? n : x0 + 64;
    double a = 0.0;
    for (int x = x0; x < x1; ++x) a += t[(size_t)y * n + x];
    s.tot[2 * j] = a;
    s.tot[2 * j + 1] = 0.0;
  }
}
__global__ void k_xs_predict(XsSum s, int n) {
  __shared__ double wtot[32];
  xs_predict(&s, 1, XsGeom(n), wtot, nullptr);
}
__global__ void k_xs_summaries(XsSum s, int n) {
  xs_summary_task([&](int) { return s; }, 1, XsGeom(n), (int)blockIdx.x);
}
__global__ void k_xs_walk(XsSum s, int n, double* out) {
  __shared__ double r[1];
  xs_walk(&s, 1, XsGeom(n), r, nullptr);
  if (threadIdx.x == 0) *out = r[0];
}

// One device batch through a CUDA graph.  The first call with a given set of
// parameters and buffers runs directly (and sizes every buffer); the second
// captures the same work on the context's capture stream and replays it; later
// calls with the same key replay the instantiated graph on the caller's
// stream as a single launch.  A capture that fails (an operation the graph
// cannot hold) turns graphs off for the context and the call runs directly.
int run_batch_graph(msgpu_context* ctx, const msgpu_params& p, int F, const BatchIO& io, cudaStream_t st) {
  auto direct = [&]() {
    return p.use_fp64 ? run_batch<double>(ctx, p, F, io, st) : run_batch<float>(ctx, p, F, io, st);
  };
  std::vector<unsigned char> key(sizeof(p) + sizeof(F) + sizeof(io));
  memcpy(key.data(), &p, sizeof(p));
  memcpy(key.data() + sizeof(p), &F, sizeof(F));
  memcpy(key.data() + sizeof(p) + sizeof(F), &io, sizeof(io));
  msgpu_context::Graph& g = ctx->graph;
  if (g.key != key || (g.exec && g.epoch != ctx->alloc_epoch)) {
    if (g.exec) cudaGraphExecDestroy(g.exec);
    g.exec = nullptr;
    g.key = key;
    g.seen = 0;
  }
  if (g.exec) {
    CK(cudaGraphLaunch(g.exec, st));
    ctx->stats.kernel_launches = g.launches;
    ctx->stats.graph_replayed = 1;
    return MSGPU_OK;
  }
  if (++g.seen < 2) return direct();
  if (!ctx->graph_stream) CK(cudaStreamCreateWithFlags(&ctx->graph_stream, cudaStreamNonBlocking));
  const unsigned long long epoch = ctx->alloc_epoch;
  CK(cudaStreamBeginCapture(ctx->graph_stream, cudaStreamCaptureModeThreadLocal));
  const int rc = p.use_fp64 ? run_batch<double>(ctx, p, F, io, ctx->graph_stream)
                            : run_batch<float>(ctx, p, F, io, ctx->graph_stream);
  cudaGraph_t graph = nullptr;
  const cudaError_t ce = cudaStreamEndCapture(ctx->graph_stream, &graph);
  cudaGraphExec_t exec = nullptr;
  // a buffer that grew during the capture (it must not: the first call sized
  // them) would leave the graph with a freed address
  const bool ok = rc == MSGPU_OK && ce == cudaSuccess && graph && epoch == ctx->alloc_epoch &&
                  cudaGraphInstantiate(&exec, graph, 0) == cudaSuccess;
  if (graph) cudaGraphDestroy(graph);
  if (!ok) {
    if (exec) cudaGraphExecDestroy(exec);
    cudaGetLastError();   // a refused capture leaves a sticky-free error state
    ctx->use_graphs = false;
    g.key.clear();
    return direct();
  }
  g.exec = exec;
  g.epoch = epoch;
  g.launches = ctx->stats.kernel_launches;
  CK(cudaGraphLaunch(g.exec, st));
  ctx->stats.graph_replayed = 1;
  return MSGPU_OK;
}

// ---------------------------------------------------------------------------
// Ragged batches: series of different sizes, each registered to its own
// reference, one level-kernel launch per level for all of them.

struct RaggedSeries {
  int level, F;            // precision = input = stop level of the series, templates
  const double* ref;       // device, (2^level+1)^2
  const double* tmpl;      // device, F images
  double* phis;            // device, F x 2 x N_level
  double* energies;        // device or null, F
};

// Normalisation and image pyramid of one series (reference + templates), as
// steps 1-2 of run_batch, into the arena slots starting at instance i0 and the
// reference slot at Rslot (layout L of the batch's largest level).
template <typename Real>
int prepare_series(msgpu_context* ctx, const msgpu_params& p, const RaggedSeries& S, const Layout& L, Real* arena,
                   size_t i0, Real* Rslot, double* pyr, size_t pstride, const std::vector<size_t>& poff,
                   double* mm, cudaStream_t st, int& launches) {
  const int Lin = S.level, F = S.F, nimg = F + 1;
  const size_t Nin = lvl_N(Lin);
  CK(cudaMemcpy2DAsync(pyr + poff[Lin], pstride * sizeof(double), S.ref, Nin * sizeof(double), Nin * sizeof(double),
                       1, cudaMemcpyDeviceToDevice, st));
  CK(cudaMemcpy2DAsync(pyr + pstride + poff[Lin], pstride * sizeof(double), S.tmpl, Nin * sizeof(double),
                       Nin * sizeof(double), F, cudaMemcpyDeviceToDevice, st));
  if (ctx->sched_error) {
    k_finite_check<<<dim3((unsigned)std::min<size_t>(256, (Nin + 255) / 256), nimg), 256, 0, st>>>(
        pyr + poff[Lin], pstride, (int)Nin, ctx->sched_error + 2);
    ++launches;
  }
  if (!p.dont_normalize_input) {
    if (p.saturation_percent >= 0) {
      const int m1 = (int)Nin - 1;
      int il = (int)(p.saturation_percent / 200 * m1), ih = (int)((1 - p.saturation_percent / 200) * m1);
      il = std::min(std::max(il, 0), m1);
      ih = std::min(std::max(ih, 0), m1);
      k_select2<<<nimg, kSelThreads, 0, st>>>(pyr + poff[Lin], pstride, (int)Nin, il, ih, mm);
    } else {
      k_minmax<<<nimg, 1024, 0, st>>>(pyr + poff[Lin], pstride, (int)Nin, mm);
    }
    k_normalize<<<dim3((unsigned)std::min<size_t>(1024, (Nin + 255) / 256), nimg), 256, 0, st>>>(
        pyr + poff[Lin], pstride, (int)Nin, mm, p.saturation_percent >= 0 ? 1 : 0, p.normalize_min_to_zero);
    launches += 2;
  }
  for (int l = Lin; l >= 1; --l) {
    const size_t cN = lvl_N(l - 1);
    k_restrict<double><<<dim3((unsigned)std::min<size_t>(1024, (cN + 255) / 256), nimg), 256, 0, st>>>(
        pyr + poff[l], pstride, pyr + poff[l - 1], pstride, l);
    ++launches;
  }
  for (int l = 0; l <= Lin; ++l) {
    const size_t Nl = lvl_N(l);
    const unsigned gx = (unsigned)std::min<size_t>(1024, (Nl + 255) / 256);
    k_to_pitched<double, Real><<<dim3(gx, 1), 256, 0, st>>>(pyr + poff[l], 0, Rslot + L.off_T[l], 0, lvl_n(l));
    k_to_pitched<double, Real><<<dim3(gx, F), 256, 0, st>>>(pyr + pstride + poff[l], pstride,
                                                             arena + i0 * L.stride + L.off_T[l], L.stride, lvl_n(l));
    launches += 2;
  }
  CK(cudaGetLastError());
  return MSGPU_OK;
}

template <typename Real>
int run_ragged(msgpu_context* ctx, const msgpu_params& p, std::vector<RaggedSeries> S, cudaStream_t st) {
  // largest series first: the instances still running at a level are a prefix
  std::stable_sort(S.begin(), S.end(), [](const RaggedSeries& a, const RaggedSeries& b) { return a.level > b.level; });
  const int ns = (int)S.size();
  const int Lmax = S[0].level, start = p.start_level;
  const bool ncc = p.data_term == 1;
  const Layout L = make_layout(Lmax, ncc, ncc);
  int Ftot = 0;
  std::vector<int> first(ns);
  for (int s = 0; s < ns; ++s) { first[s] = Ftot; Ftot += S[s].F; }
  int rc;
  if ((rc = ensure_tables(ctx))) return rc;
  if ((rc = sched_error_reset(ctx, st))) return rc;
  const size_t rstride = align_up(L.off_T[Lmax] + comp_stride(Lmax), 64);
  size_t pmax = 0;
  std::vector<std::vector<size_t>> poffs(ns);
  std::vector<size_t> pstrides(ns);
  for (int s = 0; s < ns; ++s) {
    poffs[s].assign(S[s].level + 1, 0);
    size_t ps = 0;
    for (int l = S[s].level; l >= 0; --l) { poffs[s][l] = ps; ps = align_up(ps + lvl_N(l), 32); }
    pstrides[s] = ps;
    pmax = std::max(pmax, ps * (size_t)(S[s].F + 1));
  }
  const int nlev = Lmax - start + 1;
  const size_t small_bytes = sizeof(double) * (2 * (size_t)(Ftot + ns + 1) + (size_t)Ftot * (nlev + 1) + 64) +
                             sizeof(int) * ((size_t)Ftot * 5 + 64);
  if ((rc = ensure(ctx, ctx->dscratch, sizeof(double) * pmax))) return rc;
  if ((rc = ensure(ctx, ctx->arena, sizeof(Real) * L.stride * Ftot))) return rc;
  if ((rc = ensure(ctx, ctx->shared_real, sizeof(Real) * rstride * ns))) return rc;
  if ((rc = ensure(ctx, ctx->small, small_bytes))) return rc;
  double* pyr = (double*)ctx->dscratch.p;
  Real* arena = (Real*)ctx->arena.p;
  Real* refs = (Real*)ctx->shared_real.p;
  double* mm = (double*)ctx->small.p;                       // 2 * (Fmax + 1)
  double* e_lvl = mm + 2 * (size_t)(Ftot + ns + 1);        // Ftot
  double* lam_all = e_lvl + Ftot;                           // nlev x Ftot
  int* ibase = (int*)(lam_all + (size_t)Ftot * nlev + 64);
  int* bufA = ibase;
  int* bufB = ibase + Ftot;
  int* steps = ibase + 2 * (size_t)Ftot;
  int* evals = ibase + 3 * (size_t)Ftot;
  int* inst_ref = ibase + 4 * (size_t)Ftot;
  int& launches = ctx->stats.kernel_launches;
  launches = 0;
  ctx->stats.num_levels = nlev;
  ctx->stats.first_level = start;
  // per-instance reference index and level weights
  std::vector<int> h_ref(Ftot);
  std::vector<double> h_lam((size_t)Ftot * nlev);
  for (int s = 0; s < ns; ++s)
    for (int f = 0; f < S[s].F; ++f) {
      h_ref[first[s] + f] = s;
      for (int l = start; l <= Lmax; ++l)
        h_lam[(size_t)(l - start) * Ftot + first[s] + f] =
            std::pow(p.lambda_factor, (double)(S[s].level - l)) * p.lambda;
    }
  CK(cudaMemcpyAsync(inst_ref, h_ref.data(), sizeof(int) * Ftot, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(lam_all, h_lam.data(), sizeof(double) * h_lam.size(), cudaMemcpyHostToDevice, st));
  // 1. every series' images
  for (int s = 0; s < ns; ++s)
    if ((rc = prepare_series<Real>(ctx, p, S[s], L, arena, (size_t)first[s], refs + (size_t)s * rstride, pyr,
                                   pstrides[s], poffs[s], mm, st, launches)))
      return rc;
  // 2. zero displacement at the start level
  k_set_buf<Real><<<1, 256, 0, st>>>(bufA, Ftot, 0);
  CK(cudaMemset2DAsync(arena + L.off_phi[0], L.stride * sizeof(Real), 0, 2 * comp_stride(start) * sizeof(Real), Ftot,
                       st));
  ++launches;
  // 3. level loop over the running prefix of instances
  int* bin = bufA;
  int* bout = bufB;
  for (int l = start; l <= Lmax; ++l) {
    int A = 0, Anext = 0;
    for (int s = 0; s < ns; ++s) {
      if (S[s].level >= l) A += S[s].F;
      if (S[s].level > l) Anext += S[s].F;
    }
    LevelArgs<Real> a;
    memset(&a, 0, sizeof(a));
    a.arena = arena;
    a.inst_stride = L.stride;
    a.R = refs + L.off_T[l];
    a.inst_ref = inst_ref;
    a.ref_stride = rstride;
    a.lambda = p.lambda;
    a.lambda_inst = lam_all + (size_t)(l - start) * Ftot;
    if (ncc) {
      a.ncc = 1;
      a.off_td = L.off_td;
      a.off_nr = L.off_nr;
      k_ncc_normalize<Real><<<A, 1024, 0, st>>>(refs + L.off_T[l], arena, L.stride, L.off_T[l], l, arena + L.off_nr,
                                               L.stride, inst_ref, rstride);
      ++launches;
    }
    a.off_T = L.off_T[l];
    a.off_phi[0] = L.off_phi[0];
    a.off_phi[1] = L.off_phi[1];
    a.off_d[0] = L.off_d[0];
    a.off_d[1] = L.off_d[1];
    a.off_s = L.off_s;
    a.off_de = L.off_de;
    for (int k = 0; k <= kMaxLevel; ++k) { a.off_x2[k] = L.off_x2[k]; a.off_x5[k] = L.off_x5[k]; a.off_b[k] = L.off_b[k]; }
    a.level = l;
    a.n = lvl_n(l);
    a.num_inst = A;
    a.lc = pick_lc<Real>(l);
    a.mode = MODE_SOLVE;
    a.stop_eps = p.stop_epsilon;
    a.max_iter = p.max_gd_iterations;
    a.phi_in_dev = bin;
    a.out_energy = e_lvl;
    a.out_steps = steps;
    a.out_evals = evals;
    a.out_phi_buf = bin;
    // sized for this level's grid and running instances (the term buffers
    // hold no state from one level to the next)
    if ((rc = xs_attach<Real>(ctx, a, p.sum_order == 0, l, A))) return rc;
    if ((rc = trace_attach<Real>(ctx, a, st))) return rc;
    if ((rc = launch_level<Real>(ctx, a, st))) return rc;
    if ((rc = trace_collect<Real>(ctx, a, st))) return rc;
    ++launches;
    // series finishing at this level: displacements and energies out
    for (int s = 0; s < ns; ++s) {
      if (S[s].level != l) continue;
      const int NM = (int)lvl_N(l);
      k_phi_out<Real><<<dim3((unsigned)std::min(1024, (NM + 255) / 256), S[s].F), 256, 0, st>>>(
          arena + (size_t)first[s] * L.stride, L.stride, L.off_phi[0], L.off_phi[1], l, bin + first[s], S[s].phis);
      ++launches;
      if (S[s].energies)
        CK(cudaMemcpyAsync(S[s].energies, e_lvl + first[s], sizeof(double) * S[s].F, cudaMemcpyDeviceToDevice, st));
    }
    CK(cudaGetLastError());
    if (Anext > 0) {
      const size_t fw = lvl_N(l + 1);
      k_phi_up<Real><<<dim3((unsigned)std::min<size_t>(1024, (fw + 255) / 256), Anext), 256, 0, st>>>(
          arena, L.stride, L.off_phi[0], L.off_phi[1], l, bin, bout, p.resample_deformation ? 1 : 0);
      CK(cudaGetLastError());
      ++launches;
      std::swap(bin, bout);
    }
  }
  return MSGPU_OK;
}

int check_params(msgpu_context* ctx, const msgpu_params* p) {
  if (!p) return fail(ctx, MSGPU_ERR_INVALID_ARG, "params is NULL");
  if (p->precision_level < 1 || p->precision_level > kMaxLevel)
    return fail(ctx, MSGPU_ERR_INVALID_ARG, "precisionLevel %d outside [1, %d]", p->precision_level, kMaxLevel);
  if (p->input_level < p->precision_level || p->input_level > kMaxLevel)
    return fail(ctx, MSGPU_ERR_SIZE,
                "Input data size too small. Note: Unless \"resizeInput\" is used, \"precisionLevel\" may not be "
                "bigger than the grid level of the input data.");
  if (p->start_level < 1 || p->stop_level > p->precision_level || p->start_level > p->stop_level)
    return fail(ctx, MSGPU_ERR_INVALID_ARG, "level range startLevel %d .. stopLevel %d invalid for precisionLevel %d",
                p->start_level, p->stop_level, p->precision_level);
  if (p->max_gd_iterations < 0) return fail(ctx, MSGPU_ERR_INVALID_ARG, "maxGDIterations < 0");
  if (p->data_term != 0 && p->data_term != 1)
    return fail(ctx, MSGPU_ERR_INVALID_ARG, "data_term %d: 0 (SSD) or 1 (NCC)", p->data_term);
  if (p->sum_order != 0 && p->sum_order != 1)
    return fail(ctx, MSGPU_ERR_INVALID_ARG, "sum_order %d: 0 (reference order) or 1 (parallel order)", p->sum_order);
  return MSGPU_OK;
}

int bind_device(msgpu_context* ctx) {
  CK(cudaSetDevice(ctx->device));
  return MSGPU_OK;
}

// ---------------------------------------------------------------------------
// Series pipeline: composition, median, the stage loop.

// Grid of the composition kernel (cooperative: every CTA resident).
int compose_grid(msgpu_context* ctx, int* grid) {
  int per_sm = 0;
  CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_extend_pcg, kExtThreads, 0));
  if (per_sm < 1) return fail(ctx, MSGPU_ERR_CUDA, "composition kernel does not fit on an SM");
  *grid = std::min(per_sm, 2) * ctx->sm_count;
  return MSGPU_OK;
}

// Doubles of the composition scratch before its counters: bc, g, hA, hB (2N
// each), two directions (4N), the per-CTA partials.
size_t compose_doubles(size_t N, int grid) { return 12 * N + (size_t)grid * 4; }

// ConcatAndSmoothlyExtendDeformations on device arrays (2N each); inout
// carries the solver's initial guess in.  The error flags must have been
// cleared by the API call (sched_error_reset).
int compose_device(msgpu_context* ctx, int level, const double* d1, const double* d2, double* inout,
                   cudaStream_t st) {
  const size_t N = lvl_N(level);
  int rc, grid = 0;
  if ((rc = ensure_tables(ctx))) return rc;
  if ((rc = compose_grid(ctx, &grid))) return rc;
  const size_t nd = compose_doubles(N, grid);
  const size_t bytes = sizeof(double) * nd + 64 + align_up(N, 256);
  if ((rc = ensure(ctx, ctx->ext, bytes))) return rc;
  double* base = (double*)ctx->ext.p;
  ExtArgs a;
  a.d1 = d1;
  a.d2 = d2;
  a.x = inout;
  a.bc = base;
  a.g = base + 2 * N;
  a.hA = base + 4 * N;
  a.hB = base + 6 * N;
  a.dbuf = base + 8 * N;
  a.partials = base + 12 * N;
  a.bar = (unsigned*)(base + nd);
  a.iters_out = (int*)(a.bar + 2);
  a.defined = (unsigned char*)(base + nd) + 64;
  a.error = ctx->sched_error + 1;
  a.level = level;
  a.bar_ns = g_barrier_wait_ns.load();
  CK(cudaMemsetAsync(a.bar, 0, 2 * sizeof(unsigned), st));
  k_compose_prep<<<(unsigned)std::min<size_t>(2048, (N + 255) / 256), 256, 0, st>>>(a);
  CK(cudaGetLastError());
  cudaLaunchConfig_t cfg = {};
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.gridDim = dim3(grid, 1, 1);
  cfg.blockDim = dim3(kExtThreads, 1, 1);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  CK(cudaLaunchKernelEx(&cfg, k_extend_pcg, a));
  ctx->stats.kernel_launches += 2;
  return MSGPU_OK;
}

// PCG steps per component of the last composition (after synchronising).
int compose_iterations(msgpu_context* ctx, int level, int it[2]) {
  int rc, grid = 0;
  if ((rc = compose_grid(ctx, &grid))) return rc;
  const size_t nd = compose_doubles(lvl_N(level), grid);
  CK(cudaMemcpy(it, (const unsigned char*)ctx->ext.p + sizeof(double) * nd + 2 * sizeof(unsigned), 2 * sizeof(int),
                cudaMemcpyDeviceToHost));
  return MSGPU_OK;
}

// Average and median of the warped frames (averageSeries, matchSeries.h:
// 385-445); the fill of pixels without samples is the mean of the last frame.
int average_median_device(msgpu_context* ctx, int level, const double* frames, const double* phis, int F,
                          double* avg, double* median, double* count, cudaStream_t st) {
  const size_t N = lvl_N(level);
  int rc;
  if ((rc = ensure(ctx, ctx->io[5], 64))) return rc;
  double* fill = (double*)ctx->io[5].p;
  k_mean<<<1, 1024, 0, st>>>(frames + (size_t)(F - 1) * N, (int)N, fill);
  ctx->stats.kernel_launches += 1;
  if (avg) {
    k_warp_mean<<<(unsigned)std::min<size_t>(2048, (N + 255) / 256), 256, 0, st>>>(frames, phis, F, level, fill,
                                                                                  avg, count);
    ctx->stats.kernel_launches += 1;
  }
  if (median) {
    if ((rc = ensure(ctx, ctx->vals, sizeof(double) * N * F))) return rc;
    double* vals = (double*)ctx->vals.p;
    k_warp_values<<<dim3((unsigned)std::min<size_t>(1024, (N + 255) / 256), F), 256, 0, st>>>(frames, phis, F,
                                                                                              level, vals);
    k_median<<<(unsigned)std::min<size_t>(2048, (N + 255) / 256), 256, 0, st>>>(vals, F, (int)N, fill, median);
    ctx->stats.kernel_launches += 2;
  }
  CK(cudaGetLastError());
  return MSGPU_OK;
}

// lambda of the extra stages: the parameter file value is replaced by the
// "%f" print of lambda * extraStagesLambdaFactor (matchSeries.h:1300).
double extra_stage_lambda(double lambda, double factor) {
  char buf[64];
  snprintf(buf, sizeof buf, "%f", lambda * factor);
  return strtod(buf, nullptr);
}

int check_series_params(msgpu_context* ctx, const msgpu_params* p, const msgpu_series_params* sp, int F) {
  int rc;
  if ((rc = check_params(ctx, p))) return rc;
  if (!sp) return fail(ctx, MSGPU_ERR_INVALID_ARG, "series params is NULL");
  if (F < 2) return fail(ctx, MSGPU_ERR_INVALID_ARG, "series matching needs at least 2 frames");
  if (p->input_level != p->precision_level)
    return fail(ctx, MSGPU_ERR_UNSUPPORTED, "series matching needs input_level == precision_level");
  if (p->stop_level != p->precision_level)
    return fail(ctx, MSGPU_ERR_UNSUPPORTED, "series matching needs stopLevel == precisionLevel");
  if (sp->num_extra_stages < 0) return fail(ctx, MSGPU_ERR_INVALID_ARG, "numExtraStages < 0");
  if (!sp->dont_accumulate_deformation &&
      (sp->refine_start_level < 1 || sp->refine_stop_level > p->precision_level ||
       sp->refine_start_level > sp->refine_stop_level))
    return fail(ctx, MSGPU_ERR_INVALID_ARG, "refineStartLevel %d .. refineStopLevel %d invalid for precisionLevel %d",
                sp->refine_start_level, sp->refine_stop_level, p->precision_level);
  return MSGPU_OK;
}

int series_num_energies(int F, int extra) { return (F - 1) + extra * F; }

// The stage loop of matchSeries<>() on device arrays (see msgpu.h).
template <typename Real>
int run_series(msgpu_context* ctx, const msgpu_params& p, const msgpu_series_params& sp, const double* frames,
               int F, double* phis_out, double* energies_out, double* avg_out, double* median_out,
               double* count_out, cudaStream_t st) {
  const int M = p.precision_level;
  const size_t N = lvl_N(M);
  const int stages = 1 + sp.num_extra_stages;
  int rc;
  // scratch: target N | acc 2N | tmp 2N | stage phis F*2N | energies | stage avg, median, count 3N
  const size_t ne = (size_t)series_num_energies(F, sp.num_extra_stages);
  const size_t need = sizeof(double) * (N + 4 * N + 2 * N * F + ne + 3 * N + 64);
  if ((rc = ensure(ctx, ctx->series, need))) return rc;
  double* target = (double*)ctx->series.p;
  double* acc = target + N;
  double* tmp = acc + 2 * N;
  double* sphis = tmp + 2 * N;
  double* en_scratch = sphis + 2 * N * F;
  double* savg = en_scratch + ne;
  double* smed = savg + N;
  double* scnt = smed + N;
  double* energies = energies_out ? energies_out : en_scratch;
  if ((rc = sched_error_reset(ctx, st))) return rc;
  int launches = 0;
  BatchOpts keep;
  keep.reset_error = 0;
  size_t eoff = 0;
  for (int s = 1; s <= stages; ++s) {
    msgpu_params ps = p;
    if (s > 1) ps.lambda = extra_stage_lambda(p.lambda, sp.extra_stages_lambda_factor);
    const int first = (s == 1) ? 1 : 0, m = F - first;
    const double* ref = (s == 1) ? frames : target;
    const double* tmpl = frames + (size_t)first * N;
    const bool last = (s == stages);
    double* phis = last ? phis_out : sphis;
    double* en = energies + eoff;
    if (sp.dont_accumulate_deformation) {
      BatchIO io{ref, tmpl, nullptr, phis, en, nullptr};
      if ((rc = run_batch<Real>(ctx, ps, m, io, st, keep))) return rc;
      launches += ctx->stats.kernel_launches;
    } else {
      BatchOpts pw = keep;
      pw.pairwise = 1;
      BatchIO io{ref, tmpl, nullptr, phis, en, nullptr};
      if ((rc = run_batch<Real>(ctx, ps, m, io, st, pw))) return rc;
      launches += ctx->stats.kernel_launches;
      CK(cudaMemsetAsync(acc, 0, sizeof(double) * 2 * N, st));
      msgpu_params pr = ps;
      pr.start_level = sp.refine_start_level;
      pr.stop_level = sp.refine_stop_level;
      BatchOpts rf = keep;
      rf.lambda_stop = ps.stop_level;
      for (int i = 0; i < m; ++i) {
        double* phi_i = phis + (size_t)2 * i * N;
        CK(cudaMemcpyAsync(tmp, acc, sizeof(double) * 2 * N, cudaMemcpyDeviceToDevice, st));
        ctx->stats.kernel_launches = 0;
        if ((rc = compose_device(ctx, M, phi_i, tmp, acc, st))) return rc;
        launches += ctx->stats.kernel_launches;
        if (i > 0) {
          BatchIO ri{ref, tmpl + (size_t)i * N, acc, acc, en + i, nullptr};
          if ((rc = run_batch<Real>(ctx, pr, 1, ri, st, rf))) return rc;
          launches += ctx->stats.kernel_launches;
          CK(cudaMemcpyAsync(phi_i, acc, sizeof(double) * 2 * N, cudaMemcpyDeviceToDevice, st));
        }
      }
    }
    ctx->stats.kernel_launches = 0;
    double* a_out = last ? avg_out : (sp.use_median_as_new_target ? nullptr : savg);
    double* m_out = last ? median_out : (sp.use_median_as_new_target ? smed : nullptr);
    if ((rc = average_median_device(ctx, M, tmpl, phis, m, a_out, m_out, last ? count_out : scnt, st)))
      return rc;
    launches += ctx->stats.kernel_launches;
    if (!last)
      CK(cudaMemcpyAsync(target, sp.use_median_as_new_target ? smed : savg, sizeof(double) * N,
                         cudaMemcpyDeviceToDevice, st));
    eoff += (size_t)m;
  }
  ctx->stats.kernel_launches = launches;
  return MSGPU_OK;
}

}  // namespace

// ===========================================================================
extern "C" {

void msgpu_params_default(msgpu_params* p) {
  if (!p) return;
  memset(p, 0, sizeof(*p));
  p->precision_level = 9;
  p->input_level = 9;
  p->start_level = 5;
  p->stop_level = 9;
  p->lambda = 0.1;
  p->lambda_factor = 1.0;
  p->max_gd_iterations = 30;
  p->stop_epsilon = 0.0;
  p->saturation_percent = 0.15;
  p->normalize_min_to_zero = 1;
  p->dont_normalize_input = 0;
  p->resample_deformation = 0;
  p->use_fp64 = 0;
}

int msgpu_abi_version(void) { return kAbiVersion; }

int msgpu_set_wait_limits(double level_wait_s, double barrier_wait_s) {
  if (std::isnan(level_wait_s) || std::isnan(barrier_wait_s)) return MSGPU_ERR_INVALID_ARG;
  auto ns = [](double s, unsigned long long dflt) {
    if (s <= 0) return dflt;
    const double v = s * 1e9;
    return v >= 1.8e19 ? dflt : (unsigned long long)v;
  };
  g_level_wait_ns.store(ns(level_wait_s, kMaxIdleNs));
  g_barrier_wait_ns.store(ns(barrier_wait_s, kExtBarrierNs));
  return MSGPU_OK;
}

int msgpu_get_tuning(const msgpu_context* ctx, int use_fp64, int level, msgpu_level_tuning* out) {
  if (!ctx || !out || level < 0 || level > kMaxLevel) return MSGPU_ERR_INVALID_ARG;
  *out = ctx->tuning[use_fp64 ? 1 : 0][level];
  return MSGPU_OK;
}

int msgpu_set_tuning(msgpu_context* ctx, int use_fp64, int level, const msgpu_level_tuning* t) {
  if (!ctx || !t || level < 0 || level > kMaxLevel) return MSGPU_ERR_INVALID_ARG;
  if (t->chunk_div < 0 || t->chunk_max < 0 || t->ctas_per_sm < 0)
    return fail(ctx, MSGPU_ERR_INVALID_ARG, "tuning values must be >= 0");
  ctx->tuning[use_fp64 ? 1 : 0][level] = *t;
  ctx->graph.key.clear();   // a captured graph holds the old launch settings
  return MSGPU_OK;
}

int msgpu_autotune_device(msgpu_context* ctx, const msgpu_params* p, const double* d_reference,
                          const double* d_templates, int num_templates, double* d_phis_scratch, void* stream) {
  if (!ctx) return MSGPU_ERR_INVALID_ARG;
  int rc;
  if ((rc = check_params(ctx, p))) return rc;
  if (num_templates < 1 || !d_reference || !d_templates || !d_phis_scratch)
    return fail(ctx, MSGPU_ERR_INVALID_ARG, "invalid autotune arguments");
  if (p->stop_level - p->start_level + 1 > 16) return fail(ctx, MSGPU_ERR_UNSUPPORTED, "more than 16 levels");
  if ((rc = bind_device(ctx))) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  const int fp = p->use_fp64 ? 1 : 0;
  const int divs[3] = {12, 24, 48}, maxs[3] = {8, 16, 32}, ctas[2] = {2, 1};
  const bool prof = ctx->profiling;
  ctx->profiling = true;
  msgpu_level_tuning best[kMaxLevel + 1];
  for (int l = 0; l <= kMaxLevel; ++l) best[l] = ctx->tuning[fp][l], best[l].ms = 1e30f;
  BatchIO io{d_reference, d_templates, nullptr, d_phis_scratch, nullptr, nullptr};
  for (int c = 0; c < 2 && rc == MSGPU_OK; ++c)
    for (int i = 0; i < 3 && rc == MSGPU_OK; ++i)
      for (int j = 0; j < 3 && rc == MSGPU_OK; ++j) {
        const msgpu_level_tuning cand = {divs[i], maxs[j], ctas[c], 0.f};
        for (int l = p->start_level; l <= p->stop_level; ++l) ctx->tuning[fp][l] = cand;
        rc = fp ? run_batch<double>(ctx, *p, num_templates, io, st) : run_batch<float>(ctx, *p, num_templates, io, st);
        if (rc) break;
        for (int l = p->start_level; l <= p->stop_level; ++l) {
          const float ms = ctx->stats.level_ms[l - p->start_level];
          if (ms < best[l].ms) best[l] = cand, best[l].ms = ms;
        }
      }
  ctx->profiling = prof;
  for (int l = p->start_level; l <= p->stop_level; ++l) ctx->tuning[fp][l] = best[l];
  ctx->graph.key.clear();
  if (rc) return rc;
  CK(cudaStreamSynchronize(st));
  return sched_error_check(ctx);
}

int msgpu_exact_sum_device(msgpu_context* ctx, int level, const double* d_terms, double* d_out, void* stream) {
  if (!ctx) return MSGPU_ERR_INVALID_ARG;
  if (level < 1 || level > kMaxLevel || !d_terms || !d_out)
    return fail(ctx, MSGPU_ERR_INVALID_ARG, "invalid exact_sum arguments");
  int rc;
  if ((rc = bind_device(ctx))) return rc;
  const int n = lvl_n(level);
  const XsLayout L(n);
  if ((rc = ensure(ctx, ctx->xsum, sizeof(double) * L.stride))) return rc;
  const XsSum s = xs_sum((double*)ctx->xsum.p, n, 0, false);
  cudaStream_t st = (cudaStream_t)stream;
  const XsGeom g(n);
  k_xs_fill<<<std::min(2048, (n * n + 255) / 256), 256, 0, st>>>(d_terms, n, s);
  k_xs_totals<<<std::min(2048, (n * g.nx + 255) / 256), 256, 0, st>>>(d_terms, n, s);
  k_xs_predict<<<1, 256, 0, st>>>(s, n);
  k_xs_summaries<<<xs_summary_tasks(1, n), 256, 0, st>>>(s, n);
  k_xs_walk<<<1, 32, 0, st>>>(s, n, d_out);
  CK(cudaGetLastError());
  ctx->stats.kernel_launches += 5;
  return MSGPU_OK;
}

int msgpu_set_graphs(msgpu_context* ctx, int on) {
  if (!ctx) return MSGPU_ERR_INVALID_ARG;
  ctx->use_graphs = on != 0;
  if (!ctx->use_graphs && ctx->graph.exec) {
    cudaGraphExecDestroy(ctx->graph.exec);
    ctx->graph.exec = nullptr;
  }
  ctx->graph.key.clear();
  ctx->graph.seen = 0;
  return MSGPU_OK;
}

int msgpu_set_sum_order(msgpu_context* ctx, int sum_order) {
  if (!ctx) return MSGPU_ERR_INVALID_ARG;
  if (sum_order != 0 && sum_order != 1) return fail(ctx, MSGPU_ERR_INVALID_ARG, "sum_order must be 0 or 1");
  ctx->sum_order = sum_order;
  return MSGPU_OK;
}

int msgpu_set_warm_schedule(msgpu_context* ctx, int coarse_iters) {
  if (!ctx) return MSGPU_ERR_INVALID_ARG;
  if (coarse_iters < 0) return fail(ctx, MSGPU_ERR_INVALID_ARG, "coarse_iters %d < 0", coarse_iters);
  ctx->warm_coarse_iters = coarse_iters;
  ++ctx->alloc_epoch;   // a captured graph holds the old step limits
  return MSGPU_OK;
}

int msgpu_set_seismic_device_control(msgpu_context* ctx, int on) {
  if (!ctx) return MSGPU_ERR_INVALID_ARG;
  ctx->xs_device_control = on != 0;
  return MSGPU_OK;
}

int msgpu_set_certified_steps(msgpu_context* ctx, int on) {
  if (!ctx) return MSGPU_ERR_INVALID_ARG;
  ctx->certified = on != 0;
  ++ctx->alloc_epoch;   // a captured graph holds the old launch arguments
  return MSGPU_OK;
}

int msgpu_set_data_term(msgpu_context* ctx, int data_term) {
  if (!ctx) return MSGPU_ERR_INVALID_ARG;
  if (data_term != 0 && data_term != 1)
    return fail(ctx, MSGPU_ERR_INVALID_ARG, "data_term %d: 0 (SSD) or 1 (NCC)", data_term);
  ctx->data_term = data_term;
  return MSGPU_OK;
}

int msgpu_create(int device, msgpu_context** out) {
  if (!out) return MSGPU_ERR_INVALID_ARG;
  *out = nullptr;
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count == 0) return MSGPU_ERR_CUDA;
  if (device < 0 || device >= count) return MSGPU_ERR_INVALID_ARG;
  msgpu_context* ctx = new msgpu_context();
  ctx->device = device;
  if (cudaSetDevice(device) != cudaSuccess ||
      cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, device) != cudaSuccess ||
      cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete ctx;
    return MSGPU_ERR_CUDA;
  }
  *out = ctx;
  return MSGPU_OK;
}

int msgpu_destroy(msgpu_context* ctx) {
  if (!ctx) return MSGPU_OK;
  cudaSetDevice(ctx->device);
  msgpu_context::Buf* bufs[] = {&ctx->arena, &ctx->shared_real, &ctx->dscratch, &ctx->small, &ctx->phis_d,
                                &ctx->io[0], &ctx->io[1],   &ctx->io[2],    &ctx->io[3], &ctx->io[4],
                                &ctx->io[5], &ctx->prof,    &ctx->sched,    &ctx->flags, &ctx->nccbuf,
                                &ctx->ext,   &ctx->series,  &ctx->vals,  &ctx->xs_basis, &ctx->xs_work,
                                &ctx->xsum,  &ctx->xpart};
  if (ctx->graph.exec) cudaGraphExecDestroy(ctx->graph.exec);
  for (auto& xs : ctx->xc_stream)
    if (xs) cudaStreamDestroy(xs);
  if (ctx->graph_stream) cudaStreamDestroy(ctx->graph_stream);
  for (auto* b : bufs)
    if (b->p) cudaFree(b->p);
  if (ctx->ev_ready)
    for (int i = 0; i < 32; ++i) cudaEventDestroy(ctx->ev[i]);
  for (msgpu_context* w : ctx->workers) msgpu_destroy(w);
  ctx->workers.clear();
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
  return MSGPU_OK;
}

const char* msgpu_last_error(const msgpu_context* ctx) { return ctx ? ctx->err.c_str() : "no context"; }

int msgpu_register_batch_device(msgpu_context* ctx, const msgpu_params* p, const double* d_reference,
                                const double* d_templates, int num_templates, const double* d_initial_phis,
                                double* d_phis_out, double* d_energies_out, int* d_steps_out, void* stream) {
  if (!ctx) return MSGPU_ERR_INVALID_ARG;
  int rc;
  if ((rc = check_params(ctx, p))) return rc;
  if (num_templates < 1) return fail(ctx, MSGPU_ERR_INVALID_ARG, "num_templates must be >= 1");
  if (!d_reference || !d_templates || !d_phis_out) return fail(ctx, MSGPU_ERR_INVALID_ARG, "null buffer");
  if ((rc = bind_device(ctx))) return rc;
  BatchIO io{d_reference, d_templates, d_initial_phis, d_phis_out, d_energies_out, d_steps_out};
  cudaStream_t st = (cudaStream_t)stream;
  ctx->stats.graph_replayed = 0;
  if (ctx->use_graphs && !ctx->profiling) return run_batch_graph(ctx, *p, num_templates, io, st);
  return p->use_fp64 ? run_batch<double>(ctx, *p, num_templates, io, st)
                     : run_batch<float>(ctx, *p, num_templates, io, st);
}

int msgpu_register_batch(msgpu_context* ctx, const msgpu_params* p, const double* reference,
                         const double* templates, int num_templates, const double* initial_phis,
                         double* phis_out, double* energies_out, int* steps_out) {
  if (!ctx) return MSGPU_ERR_INVALID_ARG;
  int rc;
  if ((rc = check_params(ctx, p))) return rc;
  if (num_templates < 1) return fail(ctx, MSGPU_ERR_INVALID_ARG, "num_templates must be >= 1");
  if (!reference || !templates || !phis_out) return fail(ctx, MSGPU_ERR_INVALID_ARG, "null buffer");
  if ((rc = bind_device(ctx))) return rc;
  const size_t Nin = lvl_N(p->input_level), NM = lvl_N(p->precision_level);
  const int F = num_templates;
  const int nlev = p->stop_level - p->start_level + 1;
  if ((rc = ensure(ctx, ctx->io[0], sizeof(double) * Nin))) return rc;
  if ((rc = ensure(ctx, ctx->io[1], sizeof(double) * Nin * F))) return rc;
  if ((rc = ensure(ctx, ctx->io[2], sizeof(double) * 2 * NM * F))) return rc;
  if ((rc = ensure(ctx, ctx->io[3], sizeof(double) * 2 * NM * F))) return rc;
  if ((rc = ensure(ctx, ctx->io[4], sizeof(double) * F + sizeof(int) * F * nlev + 64))) return rc;
  cudaStream_t st = ctx->stream;
  CK(cudaMemcpyAsync(ctx->io[0].p, reference, sizeof(double) * Nin, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(ctx->io[1].p, templates, sizeof(double) * Nin * F, cudaMemcpyHostToDevice, st));
  if (initial_phis)
    CK(cudaMemcpyAsync(ctx->io[2].p, initial_phis, sizeof(double) * 2 * NM * F, cudaMemcpyHostToDevice, st));
  double* d_e = (double*)ctx->io[4].p;
  int* d_s = (int*)(d_e + F);
  BatchIO io{(const double*)ctx->io[0].p, (const double*)ctx->io[1].p,
             initial_phis ? (const double*)ctx->io[2].p : nullptr, (double*)ctx->io[3].p, d_e, d_s};
  rc = p->use_fp64 ? run_batch<double>(ctx, *p, F, io, st) : run_batch<float>(ctx, *p, F, io, st);
  if (rc) return rc;
  CK(cudaMemcpyAsync(phis_out, ctx->io[3].p, sizeof(double) * 2 * NM * F, cudaMemcpyDeviceToHost, st));
  std::vector<double> e(F);
  std::vector<int> s((size_t)F * nlev);
  CK(cudaMemcpyAsync(e.data(), d_e, sizeof(double) * F, cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(s.data(), d_s, sizeof(int) * F * nlev, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  if ((rc = sched_error_check(ctx))) return rc;
  if (energies_out) memcpy(energies_out, e.data(), sizeof(double) * F);
  if (steps_out) memcpy(steps_out, s.data(), sizeof(int) * F * nlev);
  return MSGPU_OK;
}

int msgpu_warp_mean_device(msgpu_context* ctx, int level, const double* d_frames, const double* d_phis,
                           int num_frames, double* d_mean_out, double* d_count_out, void* stream) {
  if (!ctx) return MSGPU_ERR_INVALID_ARG;
  if (level < 1 || level > kMaxLevel || num_frames < 1 || !d_frames || !d_phis || !d_mean_out || !d_count_out)
    return fail(ctx, MSGPU_ERR_INVALID_ARG, "invalid warp_mean arguments");
  int rc;
  if ((rc = bind_device(ctx))) return rc;
  if ((rc = ensure(ctx, ctx->io[5], 64))) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  const int N = (int)lvl_N(level);
  k_mean<<<1, 1024, 0, st>>>(d_frames + (size_t)(num_frames - 1) * N, N, (double*)ctx->io[5].p);
  k_warp_mean<<<std::min(2048, (N + 255) / 256), 256, 0, st>>>(d_frames, d_phis, num_frames, level,
                                                               (const double*)ctx->io[5].p, d_mean_out,
                                                               d_count_out);
  CK(cudaGetLastError());
  ctx->stats.kernel_launches += 2;
  return MSGPU_OK;
}

int msgpu_warp_sum_device(msgpu_context* ctx, int level, const double* d_frames, const double* d_phis,
                          int num_frames, double* d_sum_out, double* d_count_out, double* d_last_mean_out,
                          void* stream) {
  if (!ctx) return MSGPU_ERR_INVALID_ARG;
  if (level < 1 || level > kMaxLevel || num_frames < 0 || (num_frames > 0 && (!d_frames || !d_phis)) ||
      !d_sum_out || !d_count_out)
    return fail(ctx, MSGPU_ERR_INVALID_ARG, "invalid warp_sum arguments");
  int rc;
  if ((rc = bind_device(ctx))) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  const int N = (int)lvl_N(level);
  if (num_frames > 0 && d_last_mean_out) {
    k_mean<<<1, 1024, 0, st>>>(d_frames + (size_t)(num_frames - 1) * N, N, d_last_mean_out);
    ++ctx->stats.kernel_launches;
  }
  k_warp_sum<<<std::min(2048, (N + 255) / 256), 256, 0, st>>>(d_frames, d_phis, num_frames, level, d_sum_out,
                                                              d_count_out);
  CK(cudaGetLastError());
  ++ctx->stats.kernel_launches;
  return MSGPU_OK;
}

int msgpu_mean_from_sums_device(msgpu_context* ctx, int level, const double* d_sum, const double* d_count,
                                const double* d_fill, double* d_mean_out, void* stream) {
  if (!ctx) return MSGPU_ERR_INVALID_ARG;
  if (level < 1 || level > kMaxLevel || !d_sum || !d_count || !d_fill || !d_mean_out)
    return fail(ctx, MSGPU_ERR_INVALID_ARG, "invalid mean_from_sums arguments");
  int rc;
  if ((rc = bind_device(ctx))) return rc;
  const int N = (int)lvl_N(level);
  k_mean_from_sums<<<std::min(2048, (N + 255) / 256), 256, 0, (cudaStream_t)stream>>>(d_sum, d_count, N, d_fill,
                                                                                       d_mean_out);
  CK(cudaGetLastError());
  ++ctx->stats.kernel_launches;
  return MSGPU_OK;
}

int msgpu_match_series_stage_device(msgpu_context* ctx, const msgpu_params* p, const double* d_reference,
                                    const double* d_templates, int num_templates, double* d_phis_out,
                                    double* d_energies_out, int* d_steps_out, double* d_mean_out,
                                    double* d_count_out, void* stream) {
  int rc = msgpu_register_batch_device(ctx, p, d_reference, d_templates, num_templates, nullptr, d_phis_out,
                                       d_energies_out, d_steps_out, stream);
  if (rc) return rc;
  if (p->input_level != p->precision_level)
    return fail(ctx, MSGPU_ERR_UNSUPPORTED, "the stage average needs input_level == precision_level");
  return msgpu_warp_mean_device(ctx, p->precision_level, d_templates, d_phis_out, num_templates, d_mean_out,
                                d_count_out, stream);
}

int msgpu_match_series_stage(msgpu_context* ctx, const msgpu_params* p, const double* reference,
                             const double* templates, int num_templates, double* phis_out, double* energies_out,
                             int* steps_out, double* mean_out, double* count_out) {
  if (!ctx) return MSGPU_ERR_INVALID_ARG;
  int rc;
  if ((rc = check_params(ctx, p))) return rc;
  if (num_templates < 1) return fail(ctx, MSGPU_ERR_INVALID_ARG, "num_templates must be >= 1");
  if (!reference || !templates || !phis_out || !mean_out || !count_out)
    return fail(ctx, MSGPU_ERR_INVALID_ARG, "null buffer");
  if (p->input_level != p->precision_level)
    return fail(ctx, MSGPU_ERR_UNSUPPORTED, "the stage average needs input_level == precision_level");
  if ((rc = bind_device(ctx))) return rc;
  const size_t N = lvl_N(p->precision_level);
  const int F = num_templates;
  const int nlev = p->stop_level - p->start_level + 1;
  if ((rc = ensure(ctx, ctx->io[0], sizeof(double) * N))) return rc;
  if ((rc = ensure(ctx, ctx->io[1], sizeof(double) * N * F))) return rc;
  if ((rc = ensure(ctx, ctx->io[3], sizeof(double) * (2 * N * F + 2 * N)))) return rc;
  if ((rc = ensure(ctx, ctx->io[4], sizeof(double) * F + sizeof(int) * F * nlev + 64))) return rc;
  cudaStream_t st = ctx->stream;
  CK(cudaMemcpyAsync(ctx->io[0].p, reference, sizeof(double) * N, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(ctx->io[1].p, templates, sizeof(double) * N * F, cudaMemcpyHostToDevice, st));
  double* d_phis = (double*)ctx->io[3].p;
  double* d_mean = d_phis + 2 * N * F;
  double* d_e = (double*)ctx->io[4].p;
  int* d_s = (int*)(d_e + F);
  if ((rc = msgpu_match_series_stage_device(ctx, p, (const double*)ctx->io[0].p, (const double*)ctx->io[1].p, F,
                                            d_phis, d_e, d_s, d_mean, d_mean + N, st)))
    return rc;
  CK(cudaMemcpyAsync(phis_out, d_phis, sizeof(double) * 2 * N * F, cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(mean_out, d_mean, sizeof(double) * N, cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(count_out, d_mean + N, sizeof(double) * N, cudaMemcpyDeviceToHost, st));
  std::vector<double> e(F);
  std::vector<int> s((size_t)F * nlev);
  CK(cudaMemcpyAsync(e.data(), d_e, sizeof(double) * F, cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(s.data(), d_s, sizeof(int) * F * nlev, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  if ((rc = sched_error_check(ctx))) return rc;
  if (energies_out) memcpy(energies_out, e.data(), sizeof(double) * F);
  if (steps_out) memcpy(steps_out, s.data(), sizeof(int) * F * nlev);
  return MSGPU_OK;
}

namespace {
int check_ragged(msgpu_context* ctx, const msgpu_params* p, const msgpu_series_desc* series, int num_series) {
  if (!p) return fail(ctx, MSGPU_ERR_INVALID_ARG, "params is NULL");
  if (!series || num_series < 1) return fail(ctx, MSGPU_ERR_INVALID_ARG, "no series");
  if (p->max_gd_iterations < 0) return fail(ctx, MSGPU_ERR_INVALID_ARG, "maxGDIterations < 0");
  if (p->data_term != 0 && p->data_term != 1)
    return fail(ctx, MSGPU_ERR_INVALID_ARG, "data_term %d: 0 (SSD) or 1 (NCC)", p->data_term);
  for (int s = 0; s < num_series; ++s) {
    const msgpu_series_desc& d = series[s];
    if (d.level < 1 || d.level > kMaxLevel || d.level < p->start_level || p->start_level < 1)
      return fail(ctx, MSGPU_ERR_INVALID_ARG, "series %d: level %d outside [startLevel %d, %d]", s, d.level,
                  p->start_level, kMaxLevel);
    if (d.num_templates < 1 || !d.reference || !d.templates || !d.phis_out)
      return fail(ctx, MSGPU_ERR_INVALID_ARG, "series %d: no templates or a null buffer", s);
  }
  return MSGPU_OK;
}
}  // namespace

int msgpu_register_ragged_device(msgpu_context* ctx, const msgpu_params* p, const msgpu_series_desc* series,
                                 int num_series, void* stream) {
  if (!ctx) return MSGPU_ERR_INVALID_ARG;
  int rc;
  if ((rc = check_ragged(ctx, p, series, num_series))) return rc;
  if ((rc = bind_device(ctx))) return rc;
  std::vector<RaggedSeries> S(num_series);
  for (int s = 0; s < num_series; ++s)
    S[s] = RaggedSeries{series[s].level, series[s].num_templates, series[s].reference, series[s].templates,
                        series[s].phis_out, series[s].energies_out};
  cudaStream_t st = (cudaStream_t)stream;
  return p->use_fp64 ? run_ragged<double>(ctx, *p, S, st) : run_ragged<float>(ctx, *p, S, st);
}

int msgpu_register_ragged(msgpu_context* ctx, const msgpu_params* p, const msgpu_series_desc* series,
                          int num_series) {
  if (!ctx) return MSGPU_ERR_INVALID_ARG;
  int rc;
  if ((rc = check_ragged(ctx, p, series, num_series))) return rc;
  if ((rc = bind_device(ctx))) return rc;
  size_t in = 0, out = 0;
  std::vector<size_t> ioff(num_series), ooff(num_series);
  for (int s = 0; s < num_series; ++s) {
    const size_t N = lvl_N(series[s].level);
    ioff[s] = in;
    ooff[s] = out;
    in += N * (1 + (size_t)series[s].num_templates);
    out += 2 * N * series[s].num_templates + series[s].num_templates;
  }
  if ((rc = ensure(ctx, ctx->io[1], sizeof(double) * in))) return rc;
  if ((rc = ensure(ctx, ctx->io[3], sizeof(double) * out))) return rc;
  cudaStream_t st = ctx->stream;
  double* din = (double*)ctx->io[1].p;
  double* dout = (double*)ctx->io[3].p;
  std::vector<RaggedSeries> S(num_series);
  for (int s = 0; s < num_series; ++s) {
    const msgpu_series_desc& d = series[s];
    const size_t N = lvl_N(d.level);
    CK(cudaMemcpyAsync(din + ioff[s], d.reference, sizeof(double) * N, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(din + ioff[s] + N, d.templates, sizeof(double) * N * d.num_templates, cudaMemcpyHostToDevice,
                       st));
    S[s] = RaggedSeries{d.level, d.num_templates, din + ioff[s], din + ioff[s] + N, dout + ooff[s],
                        dout + ooff[s] + 2 * N * d.num_templates};
  }
  if ((rc = p->use_fp64 ? run_ragged<double>(ctx, *p, S, st) : run_ragged<float>(ctx, *p, S, st))) return rc;
  for (int s = 0; s < num_series; ++s) {
    const msgpu_series_desc& d = series[s];
    const size_t N = lvl_N(d.level);
    CK(cudaMemcpyAsync(d.phis_out, dout + ooff[s], sizeof(double) * 2 * N * d.num_templates, cudaMemcpyDeviceToHost,
                       st));
    if (d.energies_out)
      CK(cudaMemcpyAsync(d.energies_out, dout + ooff[s] + 2 * N * d.num_templates, sizeof(double) * d.num_templates,
                         cudaMemcpyDeviceToHost, st));
  }
  CK(cudaStreamSynchronize(st));
  return sched_error_check(ctx);
}

namespace {
// The 1-D mass band of a line of n nodes, assembled in element order as
// MassOp<RectangularGridConfigurator<., QC_1D, Gauss 3>> does (h = 1/(n-1)).
LineTables host_line_tables(int n) {
  LineTables t;
  t.h = 1. / (double)(n - 1);
  t.g[0] = 0.2113248654051871;
  t.g[1] = 0.7886751345948129;
  for (int q = 0; q < 2; ++q) { t.bq[0][q] = 1. - t.g[q]; t.bq[1][q] = t.g[q]; }
  double M[2][2] = {{0., 0.}, {0., 0.}};
  for (int q = 0; q < 2; ++q)
    for (int i = 0; i < 2; ++i) {
      const double bi = t.bq[i][q];
      for (int j = i; j < 2; ++j) M[i][j] += bi * t.bq[j][q] * 1. * 0.5;
    }
  for (int i = 0; i < 2; ++i)
    for (int j = i; j < 2; ++j) M[j][i] = M[i][j] = M[i][j] * t.h;
  double band[4][3] = {};
  for (int e = 0; e < 3; ++e)
    for (int i = 0; i < 2; ++i)
      for (int j = 0; j < 2; ++j) band[e + i][j - i + 1] += 1.0 * M[i][j];
  t.d0 = band[0][1];
  t.u0 = band[0][2];
  t.l = band[1][0];
  t.d = band[1][1];
  t.u = band[1][2];
  t.ln = band[3][0];
  t.dn = band[3][1];
  return t;
}

// Nine-point rows of K = stiffX + yreg * stiffY (FEOpMixedDerivative) for
// h = 1/(max(nx,ny)-1), assembled on a 5 x 5 node patch in element order.
XRegTables host_xreg_tables(int nx, int ny, double yreg) {
  const double h = 1. / (double)((nx > ny ? nx : ny) - 1), vol = h * h;
  const double g[2] = {0.2113248654051871, 0.7886751345948129};
  double rc[4][2];
  for (int i = 0, k = 0; i < 2; ++i)
    for (int j = 0; j < 2; ++j, ++k) { rc[k][0] = g[i]; rc[k][1] = g[j]; }
  double gq[4][4][2];
  for (int b = 0; b < 4; ++b)
    for (int q = 0; q < 4; ++q) host_basis_grad(b, rc[q][0], rc[q][1], h, gq[b][q]);
  const int n = 5;
  std::vector<double> st((size_t)n * n * 9, 0.0);
  for (int pass = 0; pass < 2; ++pass) {
    const int sd = pass;
    const double factor = pass == 0 ? 1.0 : yreg;
    double L[4][4] = {};
    for (int q = 0; q < 4; ++q)
      for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) L[i][j] += 1. * gq[i][q][sd] * gq[j][q][sd] * 0.25;
    for (int i = 0; i < 4; ++i)
      for (int j = 0; j < 4; ++j) L[i][j] *= vol;
    for (int ey = 0; ey < n - 1; ++ey)
      for (int ex = 0; ex < n - 1; ++ex)
        for (int i = 0; i < 4; ++i)
          for (int j = 0; j < 4; ++j) {
            const int gi = ex + ey * n + ((i & 1) ? 1 : 0) + ((i & 2) ? n : 0);
            const int gj = ex + ey * n + ((j & 1) ? 1 : 0) + ((j & 2) ? n : 0);
            const int dx = (gj % n) - (gi % n), dy = (gj / n) - (gi / n);
            st[(size_t)gi * 9 + (dy + 1) * 3 + (dx + 1)] += factor * L[i][j];
          }
  }
  XRegTables tb;
  const int rep[3] = {0, 2, 4};
  for (int cy = 0; cy < 3; ++cy)
    for (int cx = 0; cx < 3; ++cx)
      for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 3; ++i) tb.st[cx + 3 * cy][j][i] = st[(size_t)(rep[cx] + rep[cy] * n) * 9 + j * 3 + i];
  return tb;
}

// The 25-point rows of laplaceWeight L M^-1 L + stiffX + yreg stiffY for
// h = 1/(max(nx,ny)-1), formed on a 5 x 5 node patch the way findXShift
// assembles them (matchSeries.h:828-838): L = StiffOp assembled element by
// element, M the lumped mass (LumpedMassOp, element-order sums, inverted),
// rows of L scaled by M^-1, the product added into entry (i, j) over k in
// increasing column order (aol::Matrix::addMatrixProduct, matrix.cpp:
// 414-429), scaled by laplaceWeight, then stiffX and yreg * stiffY added
// element by element.  Every row depends only on its node's class along x
// and y (first, second, interior, second last, last), so the patch's node
// c holds class c's row.  Needs nx, ny >= 5.
XLapTables host_xreg_lap_tables(int nx, int ny, double yreg, double w) {
  const double h = 1. / (double)((nx > ny ? nx : ny) - 1), vol = h * h;
  const double g[2] = {0.2113248654051871, 0.7886751345948129};
  double rc[4][2];
  for (int i = 0, k = 0; i < 2; ++i)
    for (int j = 0; j < 2; ++j, ++k) { rc[k][0] = g[i]; rc[k][1] = g[j]; }
  double gq[4][4][2], bq[4][4];
  for (int b = 0; b < 4; ++b)
    for (int q = 0; q < 4; ++q) {
      host_basis_grad(b, rc[q][0], rc[q][1], h, gq[b][q]);
      bq[b][q] = host_basis_val(b, rc[q][0], rc[q][1]);
    }
  const int n = 5, N = n * n;
  double Ls[4][4] = {};
  for (int q = 0; q < 4; ++q)
    for (int i = 0; i < 4; ++i)
      for (int j = i; j < 4; ++j) {
        double d = 0;
        d += gq[i][q][0] * gq[j][q][0];
        d += gq[i][q][1] * gq[j][q][1];
        Ls[i][j] += d * 1. * 0.25;
      }
  for (int i = 0; i < 4; ++i)
    for (int j = i; j < 4; ++j) Ls[j][i] = Ls[i][j] = Ls[i][j] * vol;
  double lmloc[4] = {0., 0., 0., 0.};
  for (int q = 0; q < 4; ++q)
    for (int i = 0; i < 4; ++i) lmloc[i] += 1. * bq[i][q] * 0.25;
  for (int i = 0; i < 4; ++i) lmloc[i] *= vol;
  std::vector<double> L((size_t)N * 9, 0.0), lm(N, 0.0), K((size_t)N * 25, 0.0);
  for (int ey = 0; ey < n - 1; ++ey)
    for (int ex = 0; ex < n - 1; ++ex)
      for (int i = 0; i < 4; ++i) {
        const int gi = ex + ey * n + ((i & 1) ? 1 : 0) + ((i & 2) ? n : 0);
        lm[gi] += lmloc[i];
        for (int j = 0; j < 4; ++j) {
          const int gj = ex + ey * n + ((j & 1) ? 1 : 0) + ((j & 2) ? n : 0);
          const int dx = (gj % n) - (gi % n), dy = (gj / n) - (gi / n);
          L[(size_t)gi * 9 + (dy + 1) * 3 + (dx + 1)] += Ls[i][j];
        }
      }
  for (int r = 0; r < N; ++r) {
    const int x = r % n, y = r / n;
    double* kr = K.data() + (size_t)r * 25;
    for (int a = -1; a <= 1; ++a)
      for (int b = -1; b <= 1; ++b) {
        const int X = x + b, Y = y + a;
        if (X < 0 || X >= n || Y < 0 || Y >= n) continue;
        const int k = X + Y * n;
        const double lik = L[(size_t)r * 9 + (a + 1) * 3 + (b + 1)];
        const double minv = 1. / lm[k];
        for (int c = -1; c <= 1; ++c)
          for (int d = -1; d <= 1; ++d) {
            const int X2 = X + d, Y2 = Y + c;
            if (X2 < 0 || X2 >= n || Y2 < 0 || Y2 >= n) continue;
            const double m2 = L[(size_t)k * 9 + (c + 1) * 3 + (d + 1)] * minv;
            kr[(a + c + 2) * 5 + (b + d + 2)] += lik * m2;
          }
      }
    for (int e = 0; e < 25; ++e) kr[e] *= w;
  }
  for (int pass = 0; pass < 2; ++pass) {
    const int sd = pass;
    const double factor = pass == 0 ? 1.0 : yreg;
    double Lm[4][4] = {};
    for (int q = 0; q < 4; ++q)
      for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) Lm[i][j] += 1. * gq[i][q][sd] * gq[j][q][sd] * 0.25;
    for (int i = 0; i < 4; ++i)
      for (int j = 0; j < 4; ++j) Lm[i][j] *= vol;
    for (int ey = 0; ey < n - 1; ++ey)
      for (int ex = 0; ex < n - 1; ++ex)
        for (int i = 0; i < 4; ++i)
          for (int j = 0; j < 4; ++j) {
            const int gi = ex + ey * n + ((i & 1) ? 1 : 0) + ((i & 2) ? n : 0);
            const int gj = ex + ey * n + ((j & 1) ? 1 : 0) + ((j & 2) ? n : 0);
            const int dx = (gj % n) - (gi % n), dy = (gj / n) - (gi / n);
            K[(size_t)gi * 25 + (dy + 2) * 5 + (dx + 2)] += factor * Lm[i][j];
          }
  }
  XLapTables tb;
  for (int cy = 0; cy < 5; ++cy)
    for (int cx = 0; cx < 5; ++cx)
      for (int e = 0; e < 25; ++e) tb.st[cx + 5 * cy][e] = K[(size_t)(cx + cy * n) * 25 + e];
  return tb;
}
}  // namespace

namespace {
// --- findXShift on the device ---------------------------------------------
// The inverse H1 metric (M + tau L)^{-1} on the nx x ny grid: M and L are
// Kronecker sums of the line operators (M = My (x) Mx, L = My (x) Kx + Ky (x)
// Mx for Q1 elements with tensor Gauss quadrature), so with the generalised
// eigenvectors of (K1, M1) -- the cosine modes v_k(i) = cos(k pi i/(n-1)),
// normalised to v^T M1 v = 1, eigenvalues 6/h^2 (1 - cos t_k)/(2 + cos t_k) --
// (M + tau L)^{-1} = V (1 + tau (lx_i + ly_j))^{-1} V^T: dense products
// (cuBLAS DGEMM) and a spectral scaling, the x products on the parity-folded
// halves of each column (k_xfold: even and odd modes separately, half the
// work of one full product each).  It is the exact
// inverse that the reference's CholeskyBasedInverseH1Metric computes by a
// sparse Cholesky factorisation, up to rounding.
void host_spectral_basis(int n, double h, double* V, double* lam) {
  const double pi = 3.14159265358979323846;
  const double m0 = h / 3.0, md = 2.0 * h / 3.0, mo = h / 6.0;   // line mass: ends, interior, off-diagonal
  std::vector<double> v(n);
  for (int k = 0; k < n; ++k) {
    const int per = 2 * (n - 1);
    for (int i = 0; i < n; ++i) v[i] = cos(pi * (double)(((long long)k * i) % per) / (double)(n - 1));
    double c = 0.0;
    for (int i = 0; i < n; ++i) {
      double mv = (i == 0 || i == n - 1) ? m0 * v[i] : md * v[i];
      if (i > 0) mv += mo * v[i - 1];
      if (i < n - 1) mv += mo * v[i + 1];
      c += v[i] * mv;
    }
    const double s = 1.0 / sqrt(c);
    for (int i = 0; i < n; ++i) V[i + (size_t)k * n] = v[i] * s;   // column k
    const double ct = cos(pi * (double)k / (double)(n - 1));
    lam[k] = 6.0 / (h * h) * (1.0 - ct) / (2.0 + ct);
  }
}

struct XsBufs {
  double *Ve, *Vo, *Vy, *lx, *ly;      // spectral basis: even and odd x modes on half the rows, y modes;
                                       // lx in the folded order (even modes, then odd modes)
  double *d, *og, *od, *de, *tx, *kphi, *t1, *t2, *nr, *part, *scal;
  unsigned* done;                      // line and regulariser counters of the fused totals
};

int xs_setup(msgpu_context* ctx, int nx, int ny, XsBufs& B, cudaStream_t st) {
  int rc;
  (void)st;
  const int ne = (nx + 1) / 2, no = nx / 2;
  const size_t nb = (size_t)ne * ne + (size_t)no * no + (size_t)ny * ny + nx + ny;
  if ((rc = ensure(ctx, ctx->xs_basis, sizeof(double) * nb))) return rc;
  B.Ve = (double*)ctx->xs_basis.p;
  B.Vo = B.Ve + (size_t)ne * ne;
  B.Vy = B.Vo + (size_t)no * no;
  B.lx = B.Vy + (size_t)ny * ny;
  B.ly = B.lx + nx;
  if (ctx->xs_nx != nx || ctx->xs_ny != ny) {
    const double h = 1. / (double)((nx > ny ? nx : ny) - 1);
    std::vector<double> vx((size_t)nx * nx), lxf(nx), hb(nb);
    host_spectral_basis(nx, h, vx.data(), lxf.data());
    double* Ve = hb.data();
    double* Vo = Ve + (size_t)ne * ne;
    for (int k = 0; k < ne; ++k)
      for (int i = 0; i < ne; ++i) Ve[i + (size_t)k * ne] = vx[i + (size_t)(2 * k) * nx];
    for (int k = 0; k < no; ++k)
      for (int i = 0; i < no; ++i) Vo[i + (size_t)k * no] = vx[i + (size_t)(2 * k + 1) * nx];
    double* Vy = Vo + (size_t)no * no;
    double* lx = Vy + (size_t)ny * ny;
    host_spectral_basis(ny, h, Vy, lx + nx);
    for (int r = 0; r < ne; ++r) lx[r] = lxf[2 * r];
    for (int r = 0; r < no; ++r) lx[ne + r] = lxf[2 * r + 1];
    CK(cudaMemcpyAsync(B.Ve, hb.data(), sizeof(double) * nb, cudaMemcpyHostToDevice, st));
    ctx->xs_nx = nx;
    ctx->xs_ny = ny;
  }
  const size_t N = (size_t)nx * ny;
  if ((rc = ensure(ctx, ctx->xs_work, sizeof(double) * (10 * N + 4096)))) return rc;
  double* w = (double*)ctx->xs_work.p;
  B.d = w; B.og = w + N; B.od = w + 2 * N; B.de = w + 3 * N; B.tx = w + 4 * N; B.kphi = w + 5 * N;
  B.t1 = w + 6 * N; B.t2 = w + 7 * N; B.nr = w + 8 * N; B.part = w + 9 * N; B.scal = B.part + 2048;
  B.done = (unsigned*)(B.scal + 64);
  CK(cudaMemsetAsync(B.done, 0, 2 * sizeof(unsigned), st));
  return MSGPU_OK;
}

// C = op(A) op(B), column-major, by k_dgemm (FP64 on the tensor pipe).
cudaError_t dgemm(cudaStream_t st, bool ta, bool tb, int M, int N, int K, const double* A, int lda,
                  const double* B, int ldb, double* C, int ldc) {
  const dim3 grid((unsigned)((M + kGemmBM - 1) / kGemmBM), (unsigned)((N + kGemmBN - 1) / kGemmBN));
  if (ta && tb) k_dgemm<true, true><<<grid, 256, 0, st>>>(M, N, K, A, lda, B, ldb, C, ldc);
  else if (ta) k_dgemm<true, false><<<grid, 256, 0, st>>>(M, N, K, A, lda, B, ldb, C, ldc);
  else if (tb) k_dgemm<false, true><<<grid, 256, 0, st>>>(M, N, K, A, lda, B, ldb, C, ldc);
  else k_dgemm<false, false><<<grid, 256, 0, st>>>(M, N, K, A, lda, B, ldb, C, ldc);
  return cudaGetLastError();
}

int xs_metric(msgpu_context* ctx, const XsBufs& B, int nx, int ny, double sigma, double* g, cudaStream_t st) {
  const double tau = 0.5 * (sigma * sigma);
  const int ne = (nx + 1) / 2, no = nx / 2;
  const int N = nx * ny;
  const int gb = std::min(2048, (N + 255) / 256);
  // column-major view: G is nx x ny (x fastest).  Analysis along x on the
  // parity-folded columns (even and odd modes), along y with Vy; scaling;
  // synthesis along y, then along x and unfolded.
  k_xfold<<<gb, 256, 0, st>>>(g, B.t1, nx, ny);
  CK(dgemm(st, true, false, ne, ny, ne, B.Ve, ne, B.t1, nx, B.t2, nx));
  CK(dgemm(st, true, false, no, ny, no, B.Vo, no, B.t1 + ne, nx, B.t2 + ne, nx));
  CK(dgemm(st, false, false, nx, ny, ny, B.t2, nx, B.Vy, ny, B.t1, nx));
  k_spectral_scale<<<gb, 256, 0, st>>>(B.t1, B.lx, B.ly, tau, nx, ny);
  CK(dgemm(st, false, true, nx, ny, ny, B.t1, nx, B.Vy, ny, B.t2, nx));
  CK(dgemm(st, false, false, ne, ny, ne, B.Ve, ne, B.t2, nx, B.t1, nx));
  CK(dgemm(st, false, false, no, ny, no, B.Vo, no, B.t2 + ne, nx, B.t1 + ne, nx));
  k_xunfold<<<gb, 256, 0, st>>>(B.t1, g, nx, ny);
  CK(cudaGetLastError());
  ctx->stats.kernel_launches += 9;
  return MSGPU_OK;
}

struct XsSolver {
  msgpu_context* ctx;
  XsBufs B;
  int nx, ny, N;
  const double *R, *T;
  double lambda, yreg;
  LineTables lt;
  XRegTables rt;
  double lapw = 0.;      // laplaceWeight (> 0: the Laplace-square regulariser)
  XLapTables lapt;
  cudaStream_t st;
  double rb_tau[2], rb_e[2];
  int rb_pos = 0, evals = 0;
  double e_at_pos = 0;
  int grid1() const { return std::min(2048, (N + 255) / 256); }

  int dot(const double* a, const double* b, double* out) {
    const int nb = std::min(1024, (N + 255) / 256);
    k_dot_part<<<nb, 256, 0, st>>>(a, b, N, B.part);
    k_sum_part<<<1, 256, 0, st>>>(B.part, nb, B.scal);
    CK(cudaMemcpyAsync(out, B.scal, sizeof(double), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    ctx->stats.kernel_launches += 2;
    return MSGPU_OK;
  }
  // data term and regulariser at p: energies into B.scal[1..2], derivative (if de) into de
  int parts(const double* p, double* de) {
    LineArgs a;
    memset(&a, 0, sizeof(a));
    a.nx = nx; a.ny = ny; a.img_stride = (size_t)N; a.R = R; a.T = T; a.phi = p;
    a.e_line = (double*)ctx->nccbuf.p; a.de = de; a.t = lt;
    a.nr_pre = B.nr; a.done = B.done; a.e_total = B.scal + 1;
    const size_t smem = sizeof(double) * 3 * (size_t)nx;
    k_lineshift<<<dim3(ny, 1), kLineThreads, smem, st>>>(a);
    const int nb = std::min(1024, (N + 255) / 256);
    if (lapw > 0)
      k_xshift_reg_lap<<<dim3(nb, 1), 256, 0, st>>>(lapt, nx, ny, (size_t)N, p, B.kphi, B.part, B.done + 1,
                                                    B.scal + 2);
    else
      k_xshift_reg<<<dim3(nb, 1), 256, 0, st>>>(rt, nx, ny, (size_t)N, p, B.kphi, B.part, B.done + 1, B.scal + 2);
    ctx->stats.kernel_launches += 2;
    CK(cudaGetLastError());
    return MSGPU_OK;
  }
  int energy(const double* p, double* e) {
    int rc;
    if ((rc = parts(p, nullptr))) return rc;
    double h[2];
    CK(cudaMemcpyAsync(h, B.scal + 1, sizeof(h), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    double v = 0.;
    v += h[0];
    v += lambda * h[1];
    *e = v;
    return MSGPU_OK;
  }
  int gradient(const double* p) {
    int rc;
    if ((rc = parts(p, B.de))) return rc;
    k_axpy<<<grid1(), 256, 0, st>>>(B.de, lambda, B.kphi, B.de, N);
    ctx->stats.kernel_launches += 1;
    return MSGPU_OK;
  }
  int eval(const double* p, const double* d, double tw, double* e) {
    if (tw == 0) { *e = e_at_pos; return MSGPU_OK; }
    k_axpy<<<grid1(), 256, 0, st>>>(p, tw, d, B.tx, N);
    ctx->stats.kernel_launches += 1;
    int rc;
    if ((rc = energy(B.tx, e))) return rc;
    rb_tau[rb_pos] = tw;
    rb_e[rb_pos] = *e;
    rb_pos ^= 1;
    evals++;
    return MSGPU_OK;
  }
  // getTimestepWidthWithArmijoLineSearch (ArmijoSearch.h:118-200)
  int armijo(const double* p, const double* d, double old_tau, double* out) {
    const double sg = 0.5, tau_min = std::pow(2., -30.), tau_max = std::pow(2., 25.);
    double tau = old_tau < tau_min ? tau_min : (old_tau > tau_max ? tau_max : old_tau);
    double f, fnew, Df;
    int rc;
    if ((rc = eval(p, d, 0., &f)) || (rc = eval(p, d, tau, &fnew)) || (rc = dot(B.de, d, &Df))) return rc;
    double G = (fnew - f) / (Df * tau);
    if (Df >= 0 || !std::isfinite(f)) { *out = 0; return MSGPU_OK; }
    if (G >= sg && f >= fnew) {
      do {
        tau *= 2.;
        if ((rc = eval(p, d, tau, &fnew))) return rc;
        G = (fnew - f) / (Df * tau);
      } while (G >= sg && f >= fnew && tau <= tau_max);
      tau *= 0.5;
    } else {
      do {
        if (tau > tau_min) tau *= 0.5;
        if ((rc = eval(p, d, tau, &fnew))) return rc;
        G = (fnew - f) / (Df * tau);
      } while ((!std::isfinite(fnew) || (G < sg || f < fnew)) && (tau > tau_min));
    }
    *out = (tau > tau_min) ? tau : 0.;
    return MSGPU_OK;
  }
};

// findXShift (matchSeries.h:805-865) with laplaceWeight <= 0: the descent
// control of GradientDescentWithAutomaticFilterWidth over H1GradientDescent
// (gradientDescent.h:295-464, 675-691) on the host, every vector operation on
// the device; phi (device, nx*ny) in/out.
int run_xshift(msgpu_context* ctx, int nx, int ny, const double* R, const double* T, double lambda, double yreg,
               double lapw,
               int max_iter, double* phi, double* energy_out, int* steps_out, cudaStream_t st) {
  XsSolver S;
  S.ctx = ctx; S.nx = nx; S.ny = ny; S.N = nx * ny; S.R = R; S.T = T; S.lambda = lambda; S.yreg = yreg; S.st = st;
  S.rb_tau[0] = S.rb_tau[1] = NAN;
  S.rb_e[0] = S.rb_e[1] = NAN;
  int rc;
  if ((rc = xs_setup(ctx, nx, ny, S.B, st))) return rc;
  if ((rc = ensure(ctx, ctx->nccbuf, sizeof(double) * (size_t)ny + 64))) return rc;
  S.lt = host_line_tables(nx);
  S.rt = host_xreg_tables(nx, ny, yreg);
  S.lapw = lapw;
  if (lapw > 0) S.lapt = host_xreg_lap_tables(nx, ny, yreg, lapw);
  CK(cudaFuncSetAttribute(k_lineshift, cudaFuncAttributeMaxDynamicSharedMemorySize,
                          (int)(sizeof(double) * 3 * (size_t)nx)));
  CK(cudaFuncSetAttribute(k_lineshift_prep_ref, cudaFuncAttributeMaxDynamicSharedMemorySize,
                          (int)(sizeof(double) * 3 * (size_t)nx)));
  const int N = S.N, g1 = S.grid1();
  const XsBufs& B = S.B;
  // the reference lines normalised once for the whole descent
  k_lineshift_prep_ref<<<dim3(ny, 1), kLineThreads, sizeof(double) * 3 * (size_t)nx, st>>>(R, nx, (size_t)N, S.lt,
                                                                                         B.nr);
  CK(cudaMemsetAsync(B.og, 0, sizeof(double) * N, st));
  CK(cudaMemsetAsync(B.od, 0, sizeof(double) * N, st));
  const double scale = (double)nx / (double)(nx > ny ? nx : ny);
  k_divide<<<g1, 256, 0, st>>>(phi, scale, N);
  double tau = 1.0, sigma = 1.0;
  const double stop_sigma = 0.0001, sigma_tol = 0.00001, stop_eps = 0.;
  double energy, energy_new;
  if ((rc = S.energy(phi, &energy))) return rc;
  energy_new = energy;
  int iter = 0;
  bool go = max_iter > 0;
  while (go) {
    iter++;
    energy = energy_new;
    S.e_at_pos = energy;
    S.evals = 0;
    if ((rc = S.gradient(phi))) return rc;
    k_mul<<<g1, 256, 0, st>>>(B.de, -1., B.d, N);
    if ((rc = xs_metric(ctx, B, nx, ny, sigma, B.d, st))) return rc;
    double beta = 0.;
    if ((iter - 1) % 10) {
      double a, b;
      if ((rc = S.dot(B.d, B.d, &a)) || (rc = S.dot(B.og, B.og, &b))) return rc;
      beta = a / b;
    }
    CK(cudaMemcpyAsync(B.og, B.d, sizeof(double) * N, cudaMemcpyDeviceToDevice, st));
    k_axpy<<<g1, 256, 0, st>>>(B.d, beta, B.od, B.d, N);
    CK(cudaMemcpyAsync(B.od, B.d, sizeof(double) * N, cudaMemcpyDeviceToDevice, st));
    if ((rc = S.armijo(phi, B.d, tau, &tau))) return rc;
    k_scale<<<g1, 256, 0, st>>>(B.d, tau, N);
    if (tau == 0) {
      CK(cudaMemcpyAsync(B.d, B.og, sizeof(double) * N, cudaMemcpyDeviceToDevice, st));
      CK(cudaMemsetAsync(B.od, 0, sizeof(double) * N, st));
      if ((rc = S.armijo(phi, B.d, tau, &tau))) return rc;
      k_scale<<<g1, 256, 0, st>>>(B.d, tau, N);
    }
    double enew = NAN;
    if (S.rb_tau[0] == tau) enew = S.rb_e[0];
    else if (S.rb_tau[1] == tau) enew = S.rb_e[1];
    else if (tau == 0) enew = energy;
    if (tau != 0) k_axpy<<<g1, 256, 0, st>>>(phi, 1.0, B.d, phi, N);
    ctx->stats.kernel_launches += 4;
    if (std::isnan(enew) && (rc = S.energy(phi, &enew))) return rc;
    energy_new = enew;
    go = ((energy - energy_new) > stop_eps) && (iter < max_iter);
    if ((0.5 * sigma > stop_sigma) && ((energy - energy_new) < sigma_tol)) {
      sigma *= 0.5;
      tau = 1.;
      go = (sigma > stop_sigma) && (iter < max_iter);
    }
  }
  k_scale<<<g1, 256, 0, st>>>(phi, scale, N);
  CK(cudaGetLastError());
  if (energy_out) *energy_out = energy_new;
  if (steps_out) *steps_out = iter;
  return MSGPU_OK;
}

// ---------------------------------------------------------------------------
// findXShift with the descent control on the device: the same steps as
// run_xshift, captured once into a CUDA graph whose loops and branches are
// conditional nodes (the outer step loop and each Armijo search as while
// nodes, the fallback attempt and the energy at the new position as if
// nodes).  One-thread control kernels take every decision from the sums the
// vector kernels leave on the device, in the same double arithmetic as the
// host control, and set the conditions; the vector kernels read their
// scalars (trial step, Fletcher-Reeves factor, filter width) from memory.
// A descent is one graph launch instead of ~4,000 launches and ~3,000 host
// round trips.  Measured on B200 (driver 580) it is the slower of the two:
// the nodes of conditional bodies cost ~7.7 us each, more than the host round
// trips they replace, so the host control stays the default.
struct XsCtl {
  double tau, sigma, energy, energy_new, f, fnew, Df, tau_ls, tw, result, beta, e_at_pos, enew;
  double rb_tau[2], rb_e[2];
  int rb_pos, iter, mode, go, ls_steps, guard;
};
constexpr double kXcTauMin = 9.313225746154785e-10;   // 2^-30 (ArmijoSearch.h:77)
constexpr double kXcTauMax = 33554432.0;              // 2^25  (ArmijoSearch.h:67)

__device__ __forceinline__ double xc_energy(const double* scal, double lambda) {
  double v = 0.;
  v += scal[1];
  v += lambda * scal[2];
  return v;
}
__global__ void k_xc_init(XsCtl* c, const double* scal, double lambda, int max_iter, cudaGraphConditionalHandle hgo) {
  c->tau = 1.0;
  c->sigma = 1.0;
  c->energy = c->energy_new = xc_energy(scal, lambda);
  c->rb_tau[0] = c->rb_tau[1] = __longlong_as_double(0x7ff8000000000000LL);
  c->rb_e[0] = c->rb_e[1] = __longlong_as_double(0x7ff8000000000000LL);
  c->rb_pos = 0;
  c->iter = 0;
  c->guard = 0;
  c->go = max_iter > 0;
  cudaGraphSetConditional(hgo, c->go ? 1u : 0u);
}
__global__ void k_xc_begin(XsCtl* c) {
  c->iter++;
  c->energy = c->energy_new;
  c->e_at_pos = c->energy;
}
// beta = |d|^2 / |og|^2 except every 10th step (scal[3], scal[4])
__global__ void k_xc_beta(XsCtl* c, const double* scal) {
  c->beta = ((c->iter - 1) % 10) ? scal[3] / scal[4] : 0.;
}
// Armijo: the starting step, f at the position, the first trial step
__global__ void k_xc_ls_init(XsCtl* c) {
  const double t = c->tau;
  c->tau_ls = t < kXcTauMin ? kXcTauMin : (t > kXcTauMax ? kXcTauMax : t);
  c->f = c->e_at_pos;
  c->tw = c->tau_ls;
}
// the energy at the trial point into the ring buffer
__global__ void k_xc_eval(XsCtl* c, const double* scal, double lambda) {
  c->fnew = xc_energy(scal, lambda);
  c->rb_tau[c->rb_pos] = c->tw;
  c->rb_e[c->rb_pos] = c->fnew;
  c->rb_pos ^= 1;
}
// after the first trial: Df = DE . d (scal[3]); doubling (mode 1), halving
// (mode 2) or done
__global__ void k_xc_ls_first(XsCtl* c, const double* scal, cudaGraphConditionalHandle hls) {
  const double sg = 0.5;
  c->Df = scal[3];
  const double f = c->f, fnew = c->fnew, Df = c->Df, tau = c->tau_ls;
  const double G = (fnew - f) / (Df * tau);
  unsigned go = 1;
  if (Df >= 0 || !isfinite(f)) {
    c->result = 0.;
    go = 0;
  } else if (G >= sg && f >= fnew) {
    c->mode = 1;
    c->tau_ls = tau * 2.;
    c->tw = c->tau_ls;
  } else {
    c->mode = 2;
    if (c->tau_ls > kXcTauMin) c->tau_ls *= 0.5;
    c->tw = c->tau_ls;
  }
  c->ls_steps = 0;
  cudaGraphSetConditional(hls, go);
}
__global__ void k_xc_ls_step(XsCtl* c, cudaGraphConditionalHandle hls) {
  const double sg = 0.5;
  const double f = c->f, fnew = c->fnew, Df = c->Df;
  double tau = c->tau_ls;
  const double G = (fnew - f) / (Df * tau);
  unsigned go = 1;
  if (c->mode == 1) {
    if (G >= sg && f >= fnew && tau <= kXcTauMax) {
      tau *= 2.;
    } else {
      tau *= 0.5;
      go = 0;
    }
  } else {
    if ((!isfinite(fnew) || (G < sg || f < fnew)) && (tau > kXcTauMin)) {
      if (tau > kXcTauMin) tau *= 0.5;
    } else {
      go = 0;
    }
  }
  c->tau_ls = tau;
  c->tw = tau;
  // the step range bounds a search to ~56 trials; a second bound guards the loop
  if (++c->ls_steps > 200) {
    c->guard = 1;
    go = 0;
  }
  if (!go) c->result = (tau > kXcTauMin) ? tau : 0.;
  cudaGraphSetConditional(hls, go);
}
// the search's result is the step; 0 -> the fallback attempt from the plain direction
__global__ void k_xc_after(XsCtl* c, cudaGraphConditionalHandle hfb) {
  c->tau = c->result;
  cudaGraphSetConditional(hfb, c->tau == 0 ? 1u : 0u);
}
__global__ void k_xc_after_fallback(XsCtl* c) { c->tau = c->result; }
// the energy at the new position from the ring buffer, or an evaluation there
__global__ void k_xc_ring(XsCtl* c, cudaGraphConditionalHandle hne) {
  double enew = __longlong_as_double(0x7ff8000000000000LL);
  if (c->rb_tau[0] == c->tau) enew = c->rb_e[0];
  else if (c->rb_tau[1] == c->tau) enew = c->rb_e[1];
  else if (c->tau == 0) enew = c->energy;
  c->enew = enew;
  cudaGraphSetConditional(hne, isnan(enew) ? 1u : 0u);
}
__global__ void k_xc_eval_pos(XsCtl* c, const double* scal, double lambda) { c->enew = xc_energy(scal, lambda); }
// stop rule and filter-width schedule (gradientDescent.h:416-439, 675-691)
__global__ void k_xc_end(XsCtl* c, int max_iter, cudaGraphConditionalHandle hgo) {
  const double stop_sigma = 0.0001, sigma_tol = 0.00001, stop_eps = 0.;
  c->energy_new = c->enew;
  bool go = ((c->energy - c->energy_new) > stop_eps) && (c->iter < max_iter);
  if ((0.5 * c->sigma > stop_sigma) && ((c->energy - c->energy_new) < sigma_tol)) {
    c->sigma *= 0.5;
    c->tau = 1.;
    go = (c->sigma > stop_sigma) && (c->iter < max_iter);
  }
  c->go = go;
  cudaGraphSetConditional(hgo, go ? 1u : 0u);
}

// Graph capture of the descent: conditional nodes appended to the capture
// of a stream, their bodies captured on further streams.
struct XsGraphBuilder {
  msgpu_context* ctx;
  XsSolver& S;
  XsCtl* c;
  int max_iter;
  cudaStream_t s[4];
  cudaError_t err = cudaSuccess;

  void check(cudaError_t e) {
    if (e != cudaSuccess && err == cudaSuccess) err = e;
  }
  cudaGraphConditionalHandle handle(cudaStream_t st) {
    cudaStreamCaptureStatus cs;
    cudaGraph_t g = nullptr;
    cudaGraphConditionalHandle h = 0;
    check(cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, nullptr, nullptr));
    if (err == cudaSuccess) check(cudaGraphConditionalHandleCreate(&h, g, 0, 0));
    return h;
  }
  cudaGraph_t cond(cudaStream_t st, cudaGraphConditionalHandle h, cudaGraphConditionalNodeType type) {
    cudaStreamCaptureStatus cs;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    check(cudaStreamGetCaptureInfo(st, &cs, nullptr, &g, &deps, &nd));
    if (err != cudaSuccess) return nullptr;
    cudaGraphNodeParams p = {cudaGraphNodeTypeConditional};
    p.conditional.handle = h;
    p.conditional.type = type;
    p.conditional.size = 1;
    cudaGraphNode_t node;
    check(cudaGraphAddNode(&node, g, deps, nd, &p));
    if (err != cudaSuccess) return nullptr;
    check(cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies));
    return p.conditional.phGraph_out[0];
  }
  // kernels of one energy evaluation at p: data term and regulariser into scal[1..2]
  void parts(cudaStream_t st, const double* p, double* de) {
    LineArgs a;
    memset(&a, 0, sizeof(a));
    a.nx = S.nx; a.ny = S.ny; a.img_stride = (size_t)S.N; a.R = S.R; a.T = S.T; a.phi = p;
    a.e_line = (double*)ctx->nccbuf.p; a.de = de; a.t = S.lt;
    a.nr_pre = S.B.nr; a.done = S.B.done; a.e_total = S.B.scal + 1;
    k_lineshift<<<dim3(S.ny, 1), kLineThreads, sizeof(double) * 3 * (size_t)S.nx, st>>>(a);
    const int nb = std::min(1024, (S.N + 255) / 256);
    if (S.lapw > 0)
      k_xshift_reg_lap<<<dim3(nb, 1), 256, 0, st>>>(S.lapt, S.nx, S.ny, (size_t)S.N, p, S.B.kphi, S.B.part,
                                                    S.B.done + 1, S.B.scal + 2);
    else
      k_xshift_reg<<<dim3(nb, 1), 256, 0, st>>>(S.rt, S.nx, S.ny, (size_t)S.N, p, S.B.kphi, S.B.part, S.B.done + 1,
                                                S.B.scal + 2);
    check(cudaGetLastError());
  }
  void dot(cudaStream_t st, const double* a, const double* b, double* out) {
    const int nb = std::min(1024, (S.N + 255) / 256);
    k_dot_part<<<nb, 256, 0, st>>>(a, b, S.N, S.B.part);
    k_sum_part<<<1, 256, 0, st>>>(S.B.part, nb, out);
    check(cudaGetLastError());
  }
  void metric(cudaStream_t st, double* g) {
    const XsBufs& B = S.B;
    const int nx = S.nx, ny = S.ny, ne = (nx + 1) / 2, no = nx / 2;
    const int gb = std::min(2048, (S.N + 255) / 256);
    k_xfold<<<gb, 256, 0, st>>>(g, B.t1, nx, ny);
    check(dgemm(st, true, false, ne, ny, ne, B.Ve, ne, B.t1, nx, B.t2, nx));
    check(dgemm(st, true, false, no, ny, no, B.Vo, no, B.t1 + ne, nx, B.t2 + ne, nx));
    check(dgemm(st, false, false, nx, ny, ny, B.t2, nx, B.Vy, ny, B.t1, nx));
    k_spectral_scale_dev<<<gb, 256, 0, st>>>(B.t1, B.lx, B.ly, &c->sigma, nx, ny);
    check(dgemm(st, false, true, nx, ny, ny, B.t1, nx, B.Vy, ny, B.t2, nx));
    check(dgemm(st, false, false, ne, ny, ne, B.Ve, ne, B.t2, nx, B.t1, nx));
    check(dgemm(st, false, false, no, ny, no, B.Vo, no, B.t2 + ne, nx, B.t1 + ne, nx));
    k_xunfold<<<gb, 256, 0, st>>>(B.t1, g, nx, ny);
    check(cudaGetLastError());
  }
  // the descent step loop's body, captured on s[1]
  void step_body(double* phi) {
    cudaStream_t st = s[1];
    const XsBufs& B = S.B;
    const int N = S.N, g1 = S.grid1();
    k_xc_begin<<<1, 1, 0, st>>>(c);
    parts(st, phi, B.de);
    k_axpy<<<g1, 256, 0, st>>>(B.de, S.lambda, B.kphi, B.de, N);
    k_mul<<<g1, 256, 0, st>>>(B.de, -1., B.d, N);
    metric(st, B.d);
    dot(st, B.d, B.d, B.scal + 3);
    dot(st, B.og, B.og, B.scal + 4);
    k_xc_beta<<<1, 1, 0, st>>>(c, B.scal);
    check(cudaMemcpyAsync(B.og, B.d, sizeof(double) * N, cudaMemcpyDeviceToDevice, st));
    k_axpy_dev<<<g1, 256, 0, st>>>(B.d, &c->beta, B.od, B.d, N);
    check(cudaMemcpyAsync(B.od, B.d, sizeof(double) * N, cudaMemcpyDeviceToDevice, st));
    check(cudaGetLastError());
    // the search on the step body's stream, its loop body on s[2]
    armijo_on(st, s[2], phi);
    const cudaGraphConditionalHandle hfb = handle(st);
    k_xc_after<<<1, 1, 0, st>>>(c, hfb);
    k_scale_dev<<<g1, 256, 0, st>>>(B.d, &c->tau, N);
    check(cudaGetLastError());
    cudaGraph_t fb = cond(st, hfb, cudaGraphCondTypeIf);
    if (err != cudaSuccess) return;
    {
      // fallback attempt: the plain direction, no memory of the old one
      cudaStream_t sf = s[2];
      check(cudaStreamBeginCaptureToGraph(sf, fb, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
      check(cudaMemcpyAsync(B.d, B.og, sizeof(double) * N, cudaMemcpyDeviceToDevice, sf));
      check(cudaMemsetAsync(B.od, 0, sizeof(double) * N, sf));
      armijo_on(sf, s[3], phi);
      k_xc_after_fallback<<<1, 1, 0, sf>>>(c);
      k_scale_dev<<<g1, 256, 0, sf>>>(B.d, &c->tau, N);
      check(cudaGetLastError());
      cudaGraph_t out = nullptr;
      check(cudaStreamEndCapture(sf, &out));
    }
    const cudaGraphConditionalHandle hne = handle(st);
    k_xc_ring<<<1, 1, 0, st>>>(c, hne);
    k_step_dev<<<g1, 256, 0, st>>>(phi, B.d, &c->tau, N);
    check(cudaGetLastError());
    cudaGraph_t ne = cond(st, hne, cudaGraphCondTypeIf);
    if (err != cudaSuccess) return;
    {
      cudaStream_t sn = s[2];
      check(cudaStreamBeginCaptureToGraph(sn, ne, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
      parts(sn, phi, nullptr);
      k_xc_eval_pos<<<1, 1, 0, sn>>>(c, B.scal, S.lambda);
      check(cudaGetLastError());
      cudaGraph_t out = nullptr;
      check(cudaStreamEndCapture(sn, &out));
    }
    const cudaGraphConditionalHandle hgo = go_handle;
    k_xc_end<<<1, 1, 0, st>>>(c, max_iter, hgo);
    check(cudaGetLastError());
  }
  cudaGraphConditionalHandle go_handle = 0;
  // one Armijo search captured on st, its loop body on sb
  void armijo_on(cudaStream_t st, cudaStream_t sb, double* phi) {
    const int g1 = S.grid1();
    k_xc_ls_init<<<1, 1, 0, st>>>(c);
    k_axpy_dev<<<g1, 256, 0, st>>>(phi, &c->tw, S.B.d, S.B.tx, S.N);
    parts(st, S.B.tx, nullptr);
    k_xc_eval<<<1, 1, 0, st>>>(c, S.B.scal, S.lambda);
    dot(st, S.B.de, S.B.d, S.B.scal + 3);
    const cudaGraphConditionalHandle hls = handle(st);
    k_xc_ls_first<<<1, 1, 0, st>>>(c, S.B.scal, hls);
    check(cudaGetLastError());
    cudaGraph_t body = cond(st, hls, cudaGraphCondTypeWhile);
    if (err != cudaSuccess) return;
    check(cudaStreamBeginCaptureToGraph(sb, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
    k_axpy_dev<<<g1, 256, 0, sb>>>(phi, &c->tw, S.B.d, S.B.tx, S.N);
    parts(sb, S.B.tx, nullptr);
    k_xc_eval<<<1, 1, 0, sb>>>(c, S.B.scal, S.lambda);
    k_xc_ls_step<<<1, 1, 0, sb>>>(c, hls);
    check(cudaGetLastError());
    cudaGraph_t out = nullptr;
    check(cudaStreamEndCapture(sb, &out));
  }
};

int run_xshift_graph(msgpu_context* ctx, int nx, int ny, const double* R, const double* T, double lambda, double yreg,
                     double lapw, int max_iter, double* phi, double* energy_out, int* steps_out, cudaStream_t st) {
  XsSolver S;
  S.ctx = ctx; S.nx = nx; S.ny = ny; S.N = nx * ny; S.R = R; S.T = T; S.lambda = lambda; S.yreg = yreg; S.st = st;
  int rc;
  if ((rc = xs_setup(ctx, nx, ny, S.B, st))) return rc;
  if ((rc = ensure(ctx, ctx->nccbuf, sizeof(double) * (size_t)ny + 64))) return rc;
  S.lt = host_line_tables(nx);
  S.rt = host_xreg_tables(nx, ny, yreg);
  S.lapw = lapw;
  if (lapw > 0) S.lapt = host_xreg_lap_tables(nx, ny, yreg, lapw);
  CK(cudaFuncSetAttribute(k_lineshift, cudaFuncAttributeMaxDynamicSharedMemorySize,
                          (int)(sizeof(double) * 3 * (size_t)nx)));
  CK(cudaFuncSetAttribute(k_lineshift_prep_ref, cudaFuncAttributeMaxDynamicSharedMemorySize,
                          (int)(sizeof(double) * 3 * (size_t)nx)));
  for (int k = 0; k < 4; ++k)
    if (!ctx->xc_stream[k]) CK(cudaStreamCreateWithFlags(&ctx->xc_stream[k], cudaStreamNonBlocking));
  XsCtl* c = reinterpret_cast<XsCtl*>(S.B.scal + 128);
  XsGraphBuilder gb{ctx, S, c, max_iter, {ctx->xc_stream[0], ctx->xc_stream[1], ctx->xc_stream[2], ctx->xc_stream[3]}};
  const int N = S.N, g1 = S.grid1();
  const XsBufs& B = S.B;
  const double scale = (double)nx / (double)(nx > ny ? nx : ny);
  cudaStream_t s0 = gb.s[0];
  CK(cudaStreamBeginCapture(s0, cudaStreamCaptureModeRelaxed));
  k_lineshift_prep_ref<<<dim3(ny, 1), kLineThreads, sizeof(double) * 3 * (size_t)nx, s0>>>(R, nx, (size_t)N, S.lt,
                                                                                         B.nr);
  gb.check(cudaMemsetAsync(B.og, 0, sizeof(double) * N, s0));
  gb.check(cudaMemsetAsync(B.od, 0, sizeof(double) * N, s0));
  k_divide<<<g1, 256, 0, s0>>>(phi, scale, N);
  gb.parts(s0, phi, nullptr);
  gb.go_handle = gb.handle(s0);
  k_xc_init<<<1, 1, 0, s0>>>(c, B.scal, lambda, max_iter, gb.go_handle);
  gb.check(cudaGetLastError());
  cudaGraph_t loop = gb.cond(s0, gb.go_handle, cudaGraphCondTypeWhile);
  if (gb.err == cudaSuccess) {
    gb.check(cudaStreamBeginCaptureToGraph(gb.s[1], loop, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
    gb.step_body(phi);
    cudaGraph_t out = nullptr;
    gb.check(cudaStreamEndCapture(gb.s[1], &out));
  }
  k_scale<<<g1, 256, 0, s0>>>(phi, scale, N);
  gb.check(cudaGetLastError());
  cudaGraph_t graph = nullptr;
  const cudaError_t ce = cudaStreamEndCapture(s0, &graph);
  if (gb.err == cudaSuccess) gb.check(ce);
  cudaGraphExec_t exec = nullptr;
  if (gb.err == cudaSuccess) gb.check(cudaGraphInstantiate(&exec, graph, 0));
  if (graph) cudaGraphDestroy(graph);
  if (gb.err != cudaSuccess) {
    if (exec) cudaGraphExecDestroy(exec);
    return fail(ctx, MSGPU_ERR_CUDA, "findXShift graph: %s", cudaGetErrorString(gb.err));
  }
  const cudaError_t le = cudaGraphLaunch(exec, st);
  double res[2];
  cudaError_t ce2 = le;
  if (ce2 == cudaSuccess) ce2 = cudaMemcpyAsync(res, &c->energy_new, sizeof(double), cudaMemcpyDeviceToHost, st);
  int it[2] = {0, 0};   // iter, guard
  if (ce2 == cudaSuccess) ce2 = cudaMemcpyAsync(it, &c->iter, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (ce2 == cudaSuccess) ce2 = cudaMemcpyAsync(it + 1, &c->guard, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (ce2 == cudaSuccess) ce2 = cudaStreamSynchronize(st);
  cudaGraphExecDestroy(exec);
  CK(ce2);
  if (it[1]) return fail(ctx, MSGPU_ERR_CUDA, "findXShift graph: a line search exceeded its trial bound");
  ctx->stats.kernel_launches += 1;
  if (energy_out) *energy_out = res[0];
  if (steps_out) *steps_out = it[0];
  return MSGPU_OK;
}
}  // namespace

namespace {
// findXShiftYConst (matchSeries.h:873-920): one shift per line v (ny),
// started from the line means of phix; four GridlessGradientDescent runs
// with Fletcher-Reeves NCG (GradientDescentBase::applySingle,
// gradientDescent.h:295-464: no smoothing, no filter widths, stop when the
// Armijo step is 0) against the template smoothed along x by boxes of 13, 9
// and 5 samples, then unsmoothed.  E(v) is the line-shift data term of the
// row-constant shift and DE its derivative summed along each line, both
// evaluated on the device (k_lineshift in row mode); the ny-long vector
// algebra and the descent control run on the host in double.
struct YcSolver {
  msgpu_context* ctx;
  int nx, ny;
  LineArgs a;
  double *vdev, *derow, *etot;
  cudaStream_t st;
  double rb_tau[2] = {NAN, NAN}, rb_e[2] = {NAN, NAN};
  int rb_pos = 0;
  double e_at_pos = 0;
  std::vector<double> tx;

  static double dotv(const double* x, const double* y, int n) {
    double r = 0;
    for (int i = 0; i < n; ++i) r += x[i] * y[i];
    return r;
  }
  int eval_device(const double* v, double* e, double* de) {
    CK(cudaMemcpyAsync(vdev, v, sizeof(double) * ny, cudaMemcpyHostToDevice, st));
    a.de_row = de ? derow : nullptr;
    k_lineshift<<<dim3(ny, 1), kLineThreads, sizeof(double) * 3 * (size_t)nx, st>>>(a);
    CK(cudaGetLastError());
    ++ctx->stats.kernel_launches;
    CK(cudaMemcpyAsync(e, etot, sizeof(double), cudaMemcpyDeviceToHost, st));
    if (de) CK(cudaMemcpyAsync(de, derow, sizeof(double) * ny, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return MSGPU_OK;
  }
  int eval(const double* p, const double* d, double tw, double* e) {
    if (tw == 0) { *e = e_at_pos; return MSGPU_OK; }
    for (int i = 0; i < ny; ++i) { tx[i] = p[i]; tx[i] += tw * d[i]; }
    int rc;
    if ((rc = eval_device(tx.data(), e, nullptr))) return rc;
    rb_tau[rb_pos] = tw;
    rb_e[rb_pos] = *e;
    rb_pos ^= 1;
    return MSGPU_OK;
  }
  // getTimestepWidthWithArmijoLineSearch (ArmijoSearch.h:118-200)
  int armijo(const double* p, const double* d, const double* DE, double old_tau, double* out) {
    const double sg = 0.5, tau_min = std::pow(2., -30.), tau_max = std::pow(2., 25.);
    double tau = old_tau < tau_min ? tau_min : (old_tau > tau_max ? tau_max : old_tau);
    double f, fnew;
    int rc;
    if ((rc = eval(p, d, 0., &f)) || (rc = eval(p, d, tau, &fnew))) return rc;
    const double Df = dotv(DE, d, ny);
    double G = (fnew - f) / (Df * tau);
    if (Df >= 0 || !std::isfinite(f)) { *out = 0; return MSGPU_OK; }
    if (G >= sg && f >= fnew) {
      do {
        tau *= 2.;
        if ((rc = eval(p, d, tau, &fnew))) return rc;
        G = (fnew - f) / (Df * tau);
      } while (G >= sg && f >= fnew && tau <= tau_max);
      tau *= 0.5;
    } else {
      do {
        if (tau > tau_min) tau *= 0.5;
        if ((rc = eval(p, d, tau, &fnew))) return rc;
        G = (fnew - f) / (Df * tau);
      } while ((!std::isfinite(fnew) || (G < sg || f < fnew)) && (tau > tau_min));
    }
    *out = (tau > tau_min) ? tau : 0.;
    return MSGPU_OK;
  }
};

int run_xshift_yconst(msgpu_context* ctx, int nx, int ny, const double* R, const double* T, int max_iter,
                      double* phix, double* energy_out, int* steps_out, cudaStream_t st) {
  const size_t N = (size_t)nx * ny;
  int rc;
  if ((rc = ensure(ctx, ctx->xs_work, sizeof(double) * (2 * N + 3 * (size_t)ny + 64)))) return rc;
  double* w = (double*)ctx->xs_work.p;
  double* Ts = w;
  double* nr = w + N;
  YcSolver S;
  S.ctx = ctx; S.nx = nx; S.ny = ny; S.st = st;
  S.vdev = w + 2 * N;
  S.derow = S.vdev + ny;
  double* eline = S.derow + ny;
  S.etot = eline + ny;
  unsigned* done = (unsigned*)(S.etot + 8);
  S.tx.assign(ny, 0.);
  CK(cudaMemsetAsync(done, 0, sizeof(unsigned), st));
  const LineTables lt = host_line_tables(nx);
  const size_t smem = sizeof(double) * 3 * (size_t)nx;
  CK(cudaFuncSetAttribute(k_lineshift, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  CK(cudaFuncSetAttribute(k_lineshift_prep_ref, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k_lineshift_prep_ref<<<dim3(ny, 1), kLineThreads, smem, st>>>(R, nx, N, lt, nr);
  memset(&S.a, 0, sizeof(S.a));
  S.a.nx = nx; S.a.ny = ny; S.a.img_stride = N; S.a.R = R; S.a.T = Ts; S.a.phi = S.vdev;
  S.a.e_line = eline; S.a.t = lt; S.a.nr_pre = nr; S.a.done = done; S.a.e_total = S.etot;
  S.a.phi_row = S.vdev;
  ++ctx->stats.kernel_launches;
  // the line means of phix (sumInXDirectionTo, then / numX)
  std::vector<double> ph(N), v(ny), d(ny), og(ny), od(ny), DE(ny);
  CK(cudaMemcpyAsync(ph.data(), phix, sizeof(double) * N, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  for (int y = 0; y < ny; ++y) {
    double sum = 0.;
    for (int x = 0; x < nx; ++x) sum += ph[(size_t)y * nx + x];
    v[y] = sum;
  }
  for (int y = 0; y < ny; ++y) v[y] /= (double)nx;
  double energy_new = INFINITY;
  int iter = 0;
  for (int round = 3; round >= 0; --round) {
    if (round > 0) {
      k_box_x<<<(unsigned)std::min<size_t>(2048, (N + 255) / 256), 256, 0, st>>>(T, nx, ny, 2 * round, Ts);
      ++ctx->stats.kernel_launches;
    } else {
      CK(cudaMemcpyAsync(Ts, T, sizeof(double) * N, cudaMemcpyDeviceToDevice, st));
    }
    S.rb_tau[0] = S.rb_tau[1] = NAN;
    S.rb_pos = 0;
    std::fill(og.begin(), og.end(), 0.);
    std::fill(od.begin(), od.end(), 0.);
    double tau = 1.0, energy;
    if ((rc = S.eval_device(v.data(), &energy, nullptr))) return rc;
    energy_new = energy;
    iter = 0;
    bool go = max_iter > 0;
    while (go) {
      iter++;
      energy = energy_new;
      S.e_at_pos = energy;
      double e_pos;
      if ((rc = S.eval_device(v.data(), &e_pos, DE.data()))) return rc;
      for (int i = 0; i < ny; ++i) d[i] = DE[i] * -1.;
      double beta = 0.;
      if ((iter - 1) % 10) beta = YcSolver::dotv(d.data(), d.data(), ny) / YcSolver::dotv(og.data(), og.data(), ny);
      og = d;
      for (int i = 0; i < ny; ++i) d[i] += beta * od[i];
      od = d;
      if ((rc = S.armijo(v.data(), d.data(), DE.data(), tau, &tau))) return rc;
      for (int i = 0; i < ny; ++i) d[i] *= tau;
      if (tau == 0) {
        d = og;
        std::fill(od.begin(), od.end(), 0.);
        if ((rc = S.armijo(v.data(), d.data(), DE.data(), tau, &tau))) return rc;
        for (int i = 0; i < ny; ++i) d[i] *= tau;
      }
      double enew = NAN;
      if (S.rb_tau[0] == tau) enew = S.rb_e[0];
      else if (S.rb_tau[1] == tau) enew = S.rb_e[1];
      else if (tau == 0) enew = energy;
      if (tau != 0)
        for (int i = 0; i < ny; ++i) v[i] += d[i];
      if (std::isnan(enew) && (rc = S.eval_device(v.data(), &enew, nullptr))) return rc;
      energy_new = enew;
      go = ((energy - energy_new) > 0.) && (iter < max_iter);
      if (tau == 0) go = false;
    }
  }
  for (int y = 0; y < ny; ++y)
    for (int x = 0; x < nx; ++x) ph[(size_t)y * nx + x] = v[y];
  CK(cudaMemcpyAsync(phix, ph.data(), sizeof(double) * N, cudaMemcpyHostToDevice, st));
  CK(cudaStreamSynchronize(st));
  if (energy_out) *energy_out = energy_new;
  if (steps_out) *steps_out = iter;
  return MSGPU_OK;
}
}  // namespace

int msgpu_find_xshift_yconst_device(msgpu_context* ctx, int nx, int ny, const double* d_R, const double* d_T,
                                    int max_iter, double* d_phix, double* energy_out, int* steps_out, void* stream) {
  if (!ctx) return MSGPU_ERR_INVALID_ARG;
  if (nx < 3 || ny < 1 || max_iter < 0 || !d_R || !d_T || !d_phix)
    return fail(ctx, MSGPU_ERR_INVALID_ARG, "invalid find_xshift_yconst arguments (lines of at least 3 samples)");
  if (sizeof(double) * 3 * (size_t)nx > 200 * 1024)
    return fail(ctx, MSGPU_ERR_SIZE, "lines of %d samples do not fit shared memory", nx);
  int rc;
  if ((rc = bind_device(ctx))) return rc;
  ctx->stats.kernel_launches = 0;
  return run_xshift_yconst(ctx, nx, ny, d_R, d_T, max_iter, d_phix, energy_out, steps_out, (cudaStream_t)stream);
}

int msgpu_find_xshift_yconst(msgpu_context* ctx, int nx, int ny, const double* R, const double* T, int max_iter,
                             double* phix, double* energy_out, int* steps_out) {
  if (!ctx) return MSGPU_ERR_INVALID_ARG;
  if (!R || !T || !phix) return fail(ctx, MSGPU_ERR_INVALID_ARG, "null buffer");
  int rc;
  if ((rc = bind_device(ctx))) return rc;
  const size_t N = (size_t)nx * ny;
  if ((rc = ensure(ctx, ctx->io[0], sizeof(double) * 3 * N))) return rc;
  double* dd = (double*)ctx->io[0].p;
  cudaStream_t st = ctx->stream;
  CK(cudaMemcpyAsync(dd, R, sizeof(double) * N, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(dd + N, T, sizeof(double) * N, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(dd + 2 * N, phix, sizeof(double) * N, cudaMemcpyHostToDevice, st));
  if ((rc = msgpu_find_xshift_yconst_device(ctx, nx, ny, dd, dd + N, max_iter, dd + 2 * N, energy_out, steps_out,
                                            st)))
    return rc;
  CK(cudaMemcpyAsync(phix, dd + 2 * N, sizeof(double) * N, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  return MSGPU_OK;
}

int msgpu_find_xshift_device(msgpu_context* ctx, int nx, int ny, const double* d_R, const double* d_T, double lambda,
                             double yreg, double laplace_weight, int max_iter, double* d_phix, double* energy_out,
                             int* steps_out, void* stream) {
  if (!ctx) return MSGPU_ERR_INVALID_ARG;
  if (nx < 3 || ny < 3 || max_iter < 0 || !d_R || !d_T || !d_phix)
    return fail(ctx, MSGPU_ERR_INVALID_ARG, "invalid find_xshift arguments (grids of at least 3 x 3 nodes)");
  if (!std::isfinite(laplace_weight) || (laplace_weight > 0 && (nx < 5 || ny < 5)))
    return fail(ctx, MSGPU_ERR_INVALID_ARG, "laplaceWeight %g: finite, and > 0 only on grids of at least 5 x 5 nodes",
                laplace_weight);
  if (sizeof(double) * 3 * (size_t)nx > 200 * 1024)
    return fail(ctx, MSGPU_ERR_SIZE, "lines of %d samples do not fit shared memory", nx);
  int rc;
  if ((rc = bind_device(ctx))) return rc;
  ctx->stats.kernel_launches = 0;
  if (ctx->xs_device_control)
    return run_xshift_graph(ctx, nx, ny, d_R, d_T, lambda, yreg, laplace_weight, max_iter, d_phix, energy_out,
                            steps_out, (cudaStream_t)stream);
  return run_xshift(ctx, nx, ny, d_R, d_T, lambda, yreg, laplace_weight, max_iter, d_phix, energy_out, steps_out,
                    (cudaStream_t)stream);
}

int msgpu_find_xshift(msgpu_context* ctx, int nx, int ny, const double* R, const double* T, double lambda,
                      double yreg, double laplace_weight, int max_iter, double* phix, double* energy_out,
                      int* steps_out) {
  if (!ctx) return MSGPU_ERR_INVALID_ARG;
  if (!R || !T || !phix) return fail(ctx, MSGPU_ERR_INVALID_ARG, "null buffer");
  int rc;
  if ((rc = bind_device(ctx))) return rc;
  const size_t N = (size_t)nx * ny;
  if ((rc = ensure(ctx, ctx->io[0], sizeof(double) * 3 * N))) return rc;
  double* d = (double*)ctx->io[0].p;
  cudaStream_t st = ctx->stream;
  CK(cudaMemcpyAsync(d, R, sizeof(double) * N, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(d + N, T, sizeof(double) * N, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(d + 2 * N, phix, sizeof(double) * N, cudaMemcpyHostToDevice, st));
  if ((rc = msgpu_find_xshift_device(ctx, nx, ny, d, d + N, lambda, yreg, laplace_weight, max_iter, d + 2 * N,
                                     energy_out, steps_out, st)))
    return rc;
  CK(cudaMemcpyAsync(phix, d + 2 * N, sizeof(double) * N, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  return MSGPU_OK;
}

int msgpu_find_xshift_batch(msgpu_context* ctx, int nx, int ny, int num_images, const double* R, int r_per_image,
                            const double* T, double lambda, double yreg, double laplace_weight, int max_iter,
                            double* phix, double* energies_out, int* steps_out, int workers) {
  if (!ctx) return MSGPU_ERR_INVALID_ARG;
  if (num_images < 1 || !R || !T || !phix) return fail(ctx, MSGPU_ERR_INVALID_ARG, "invalid find_xshift_batch arguments");
  int rc;
  if ((rc = bind_device(ctx))) return rc;
  const int nw = std::max(1, std::min(workers < 1 ? 4 : workers, num_images));
  while ((int)ctx->workers.size() < nw) {
    msgpu_context* w = nullptr;
    if ((rc = msgpu_create(ctx->device, &w))) return fail(ctx, rc, "cannot create a worker context");
    ctx->workers.push_back(w);
  }
  const size_t N = (size_t)nx * ny;
  std::atomic<int> next(0);
  std::vector<int> codes(nw, MSGPU_OK);
  std::vector<std::string> msgs(nw);
  auto work = [&](int wi) {
    msgpu_context* w = ctx->workers[wi];
    for (;;) {
      const int i = next.fetch_add(1);
      if (i >= num_images) break;
      double e = 0;
      int st = 0;
      const int c = msgpu_find_xshift(w, nx, ny, R + (r_per_image ? (size_t)i * N : 0), T + (size_t)i * N, lambda,
                                      yreg, laplace_weight, max_iter, phix + (size_t)i * N, &e, &st);
      if (c) {
        codes[wi] = c;
        msgs[wi] = w->err;
        next.store(num_images);
        break;
      }
      if (energies_out) energies_out[i] = e;
      if (steps_out) steps_out[i] = st;
    }
  };
  std::vector<std::thread> pool;
  for (int t = 1; t < nw; ++t) pool.emplace_back(work, t);
  work(0);
  for (auto& t : pool) t.join();
  int launches = 0;
  for (int t = 0; t < nw; ++t) launches += ctx->workers[t]->stats.kernel_launches;
  ctx->stats.kernel_launches = launches;
  for (int t = 0; t < nw; ++t)
    if (codes[t]) return fail(ctx, codes[t], "%s", msgs[t].c_str());
  return MSGPU_OK;
}

int msgpu_empty_lines_to_nan_device(msgpu_context* ctx, int nx, int ny, int num_images, double* d_img,
                                    int* replaced_out, void* stream) {
  if (!ctx) return MSGPU_ERR_INVALID_ARG;
  if (nx < 1 || ny < 1 || num_images < 1 || !d_img)
    return fail(ctx, MSGPU_ERR_INVALID_ARG, "invalid empty_lines_to_nan arguments");
  if ((size_t)ny * num_images > (size_t)INT_MAX)
    return fail(ctx, MSGPU_ERR_SIZE, "%d images of %d lines exceed the grid", num_images, ny);
  int rc;
  if ((rc = bind_device(ctx))) return rc;
  ctx->stats.kernel_launches = 0;
  cudaStream_t st = (cudaStream_t)stream;
  int* cnt = nullptr;
  if (replaced_out) {
    if ((rc = ensure(ctx, ctx->io[5], 64))) return rc;
    cnt = (int*)ctx->io[5].p;
    CK(cudaMemsetAsync(cnt, 0, sizeof(int), st));
  }
  msg::k_empty_lines_nan<<<ny * num_images, 256, 0, st>>>(d_img, nx, cnt);
  CK(cudaGetLastError());
  ctx->stats.kernel_launches = 1;
  if (replaced_out) {
    CK(cudaMemcpyAsync(replaced_out, cnt, sizeof(int), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
  }
  return MSGPU_OK;
}

int msgpu_remove_empty_lines_device(msgpu_context* ctx, int nx, int ny, const double* d_img, int keep_top_bottom,
                                    double* d_out, int* out_ny, void* stream) {
  if (!ctx) return MSGPU_ERR_INVALID_ARG;
  if (nx < 1 || ny < 1 || !d_img || !d_out || !out_ny || d_img == d_out)
    return fail(ctx, MSGPU_ERR_INVALID_ARG, "invalid remove_empty_lines arguments");
  int rc;
  if ((rc = bind_device(ctx))) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  if ((rc = ensure(ctx, ctx->io[5], sizeof(int) * 2 * (size_t)ny))) return rc;
  int* kept_d = (int*)ctx->io[5].p;
  int* map_d = kept_d + ny;
  msg::k_line_kept<<<ny, 256, 0, st>>>(d_img, nx, kept_d);
  CK(cudaGetLastError());
  std::vector<int> kept(ny), lines;
  CK(cudaMemcpyAsync(kept.data(), kept_d, sizeof(int) * ny, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  for (int y = 0; y < ny; ++y)
    if (kept[y]) lines.push_back(y);
  ctx->stats.kernel_launches = 1;
  if (lines.empty()) return fail(ctx, MSGPU_ERR_INVALID_ARG, "Input contains only empty lines");
  const int count = (int)lines.size(), first = lines.front(), last = lines.back();
  int top = 0, bottom = 0;
  if (keep_top_bottom) {
    if (count == 1)
      return fail(ctx, MSGPU_ERR_INVALID_ARG, "keeping the empty top and bottom blocks needs two non-empty lines");
    // aol::Rint (aol.h:422) of the mean distance of the non-empty lines
    const double d = (last - first) / (double)(count - 1);
    const int dist = d >= 0 ? (int)(d + 0.5) : (int)(d - 0.5);
    top = first / dist;
    bottom = (ny - 1 - last) / dist;
  }
  const int n = count + top + bottom;
  std::vector<int> map(n, -1);
  for (int k = 0; k < count; ++k) map[top + k] = lines[k];
  CK(cudaMemcpyAsync(map_d, map.data(), sizeof(int) * n, cudaMemcpyHostToDevice, st));
  msg::k_gather_lines<<<n, 256, 0, st>>>(d_img, nx, map_d, d_out);
  CK(cudaGetLastError());
  ctx->stats.kernel_launches = 2;
  CK(cudaStreamSynchronize(st));
  *out_ny = n;
  return MSGPU_OK;
}

int msgpu_remove_empty_lines(msgpu_context* ctx, int nx, int ny, const double* img, int keep_top_bottom, double* out,
                             int* out_ny) {
  if (!ctx) return MSGPU_ERR_INVALID_ARG;
  if (!img || !out || !out_ny) return fail(ctx, MSGPU_ERR_INVALID_ARG, "null buffer");
  if (nx < 1 || ny < 1) return fail(ctx, MSGPU_ERR_INVALID_ARG, "invalid remove_empty_lines arguments");
  int rc;
  if ((rc = bind_device(ctx))) return rc;
  const size_t N = (size_t)nx * ny;
  if ((rc = ensure(ctx, ctx->io[0], sizeof(double) * 2 * N))) return rc;
  double* d = (double*)ctx->io[0].p;
  cudaStream_t st = ctx->stream;
  CK(cudaMemcpyAsync(d, img, sizeof(double) * N, cudaMemcpyHostToDevice, st));
  if ((rc = msgpu_remove_empty_lines_device(ctx, nx, ny, d, keep_top_bottom, d + N, out_ny, st))) return rc;
  CK(cudaMemcpyAsync(out, d + N, sizeof(double) * nx * (size_t)*out_ny, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  return MSGPU_OK;
}

int msgpu_empty_lines_to_nan(msgpu_context* ctx, int nx, int ny, int num_images, double* img, int* replaced_out) {
  if (!ctx) return MSGPU_ERR_INVALID_ARG;
  if (!img) return fail(ctx, MSGPU_ERR_INVALID_ARG, "null buffer");
  if (nx < 1 || ny < 1 || num_images < 1)
    return fail(ctx, MSGPU_ERR_INVALID_ARG, "invalid empty_lines_to_nan arguments");
  int rc;
  if ((rc = bind_device(ctx))) return rc;
  const size_t N = (size_t)nx * ny * num_images;
  if ((rc = ensure(ctx, ctx->io[0], sizeof(double) * N))) return rc;
  double* d = (double*)ctx->io[0].p;
  cudaStream_t st = ctx->stream;
  CK(cudaMemcpyAsync(d, img, sizeof(double) * N, cudaMemcpyHostToDevice, st));
  if ((rc = msgpu_empty_lines_to_nan_device(ctx, nx, ny, num_images, d, replaced_out, st))) return rc;
  CK(cudaMemcpyAsync(img, d, sizeof(double) * N, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  return MSGPU_OK;
}

int msgpu_lineshift_energy_device(msgpu_context* ctx, int nx, int ny, int num_images, const double* d_R,
                                  const double* d_T, const double* d_phix, double* d_energy_out, double* d_de_out,
                                  void* stream) {
  if (!ctx) return MSGPU_ERR_INVALID_ARG;
  if (nx < 2 || ny < 1 || num_images < 1 || !d_R || !d_T || !d_phix || !d_energy_out)
    return fail(ctx, MSGPU_ERR_INVALID_ARG, "invalid lineshift arguments");
  const size_t smem = sizeof(double) * 3 * (size_t)nx;
  if (smem > 200 * 1024) return fail(ctx, MSGPU_ERR_SIZE, "lines of %d samples do not fit shared memory", nx);
  int rc;
  if ((rc = bind_device(ctx))) return rc;
  if ((rc = ensure(ctx, ctx->nccbuf, sizeof(double) * (size_t)ny * num_images + 64))) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  LineArgs a;
  memset(&a, 0, sizeof(a));
  a.nx = nx;
  a.ny = ny;
  a.img_stride = (size_t)nx * ny;
  a.R = d_R;
  a.T = d_T;
  a.phi = d_phix;
  a.e_line = (double*)ctx->nccbuf.p;
  a.de = d_de_out;
  a.t = host_line_tables(nx);
  CK(cudaFuncSetAttribute(k_lineshift, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k_lineshift<<<dim3(ny, num_images), kLineThreads, smem, st>>>(a);
  k_lineshift_total<<<num_images, 256, 0, st>>>(a.e_line, ny, d_energy_out);
  CK(cudaGetLastError());
  ctx->stats.kernel_launches = 2;
  return MSGPU_OK;
}

int msgpu_lineshift_energy(msgpu_context* ctx, int nx, int ny, const double* R, const double* T, const double* phix,
                           double* energy_out, double* de_out) {
  if (!ctx) return MSGPU_ERR_INVALID_ARG;
  if (nx < 2 || ny < 1 || !R || !T || !phix || !energy_out)
    return fail(ctx, MSGPU_ERR_INVALID_ARG, "invalid lineshift arguments");
  int rc;
  if ((rc = bind_device(ctx))) return rc;
  const size_t N = (size_t)nx * ny;
  if ((rc = ensure(ctx, ctx->io[0], sizeof(double) * (4 * N + 8)))) return rc;
  double* d = (double*)ctx->io[0].p;
  cudaStream_t st = ctx->stream;
  CK(cudaMemcpyAsync(d, R, sizeof(double) * N, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(d + N, T, sizeof(double) * N, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(d + 2 * N, phix, sizeof(double) * N, cudaMemcpyHostToDevice, st));
  if ((rc = msgpu_lineshift_energy_device(ctx, nx, ny, 1, d, d + N, d + 2 * N, d + 4 * N, de_out ? d + 3 * N : nullptr,
                                          st)))
    return rc;
  CK(cudaMemcpyAsync(energy_out, d + 4 * N, sizeof(double), cudaMemcpyDeviceToHost, st));
  if (de_out) CK(cudaMemcpyAsync(de_out, d + 3 * N, sizeof(double) * N, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  return MSGPU_OK;
}

int msgpu_xshift_reg_device(msgpu_context* ctx, int nx, int ny, int num_images, double yreg, double laplace_weight,
                            const double* d_phix, double* d_energy_out, double* d_kphi_out, void* stream) {
  if (!ctx) return MSGPU_ERR_INVALID_ARG;
  if (nx < 3 || ny < 3 || num_images < 1 || !d_phix || !d_energy_out || !d_kphi_out)
    return fail(ctx, MSGPU_ERR_INVALID_ARG, "invalid xshift_reg arguments (grids of at least 3 x 3 nodes)");
  if (!std::isfinite(laplace_weight) || (laplace_weight > 0 && (nx < 5 || ny < 5)))
    return fail(ctx, MSGPU_ERR_INVALID_ARG, "laplaceWeight %g: finite, and > 0 only on grids of at least 5 x 5 nodes",
                laplace_weight);
  int rc;
  if ((rc = bind_device(ctx))) return rc;
  const int N = nx * ny;
  const int nb = std::min(1024, (N + 255) / 256);
  if ((rc = ensure(ctx, ctx->vals, sizeof(double) * (size_t)nb * num_images + 64))) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  if (laplace_weight > 0)
    k_xshift_reg_lap<<<dim3(nb, num_images), 256, 0, st>>>(host_xreg_lap_tables(nx, ny, yreg, laplace_weight), nx, ny,
                                                           (size_t)N, d_phix, d_kphi_out, (double*)ctx->vals.p,
                                                           nullptr, nullptr);
  else
    k_xshift_reg<<<dim3(nb, num_images), 256, 0, st>>>(host_xreg_tables(nx, ny, yreg), nx, ny, (size_t)N, d_phix,
                                                       d_kphi_out, (double*)ctx->vals.p, nullptr, nullptr);
  k_xshift_reg_total<<<num_images, 256, 0, st>>>((const double*)ctx->vals.p, nb, d_energy_out);
  CK(cudaGetLastError());
  ctx->stats.kernel_launches = 2;
  return MSGPU_OK;
}

int msgpu_xshift_reg(msgpu_context* ctx, int nx, int ny, double yreg, double laplace_weight, const double* phix,
                     double* energy_out, double* kphi_out) {
  if (!ctx) return MSGPU_ERR_INVALID_ARG;
  if (!phix || !energy_out || !kphi_out) return fail(ctx, MSGPU_ERR_INVALID_ARG, "null buffer");
  int rc;
  if ((rc = bind_device(ctx))) return rc;
  const size_t N = (size_t)nx * ny;
  if ((rc = ensure(ctx, ctx->io[0], sizeof(double) * (2 * N + 8)))) return rc;
  double* d = (double*)ctx->io[0].p;
  cudaStream_t st = ctx->stream;
  CK(cudaMemcpyAsync(d, phix, sizeof(double) * N, cudaMemcpyHostToDevice, st));
  if ((rc = msgpu_xshift_reg_device(ctx, nx, ny, 1, yreg, laplace_weight, d, d + 2 * N, d + N, st))) return rc;
  CK(cudaMemcpyAsync(energy_out, d + 2 * N, sizeof(double), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(kphi_out, d + N, sizeof(double) * N, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  return MSGPU_OK;
}

void msgpu_series_params_default(const msgpu_params* p, msgpu_series_params* s) {
  if (!s) return;
  s->refine_start_level = p ? p->start_level : 1;
  s->refine_stop_level = p ? p->precision_level : 1;
  s->num_extra_stages = 0;
  s->extra_stages_lambda_factor = 1.0;
  s->use_median_as_new_target = 0;
  s->dont_accumulate_deformation = 0;
}

int msgpu_match_series_device(msgpu_context* ctx, const msgpu_params* p, const msgpu_series_params* s,
                              const double* d_frames, int num_frames, double* d_phis_out, double* d_energies_out,
                              double* d_average_out, double* d_median_out, double* d_count_out, void* stream) {
  if (!ctx) return MSGPU_ERR_INVALID_ARG;
  int rc;
  if ((rc = check_series_params(ctx, p, s, num_frames))) return rc;
  if (!d_frames || !d_phis_out || (d_average_out && !d_count_out))
    return fail(ctx, MSGPU_ERR_INVALID_ARG, "null buffer");
  if ((rc = bind_device(ctx))) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  return p->use_fp64 ? run_series<double>(ctx, *p, *s, d_frames, num_frames, d_phis_out, d_energies_out,
                                          d_average_out, d_median_out, d_count_out, st)
                     : run_series<float>(ctx, *p, *s, d_frames, num_frames, d_phis_out, d_energies_out,
                                         d_average_out, d_median_out, d_count_out, st);
}

int msgpu_match_series(msgpu_context* ctx, const msgpu_params* p, const msgpu_series_params* s,
                       const double* frames, int num_frames, double* phis_out, double* energies_out,
                       double* average_out, double* median_out, double* count_out) {
  if (!ctx) return MSGPU_ERR_INVALID_ARG;
  int rc;
  if ((rc = check_series_params(ctx, p, s, num_frames))) return rc;
  if (!frames || !phis_out || (average_out && !count_out)) return fail(ctx, MSGPU_ERR_INVALID_ARG, "null buffer");
  if ((rc = bind_device(ctx))) return rc;
  const size_t N = lvl_N(p->precision_level);
  const int F = num_frames;
  const int m = s->num_extra_stages > 0 ? F : F - 1;
  const size_t ne = (size_t)series_num_energies(F, s->num_extra_stages);
  if ((rc = ensure(ctx, ctx->io[1], sizeof(double) * N * F))) return rc;
  if ((rc = ensure(ctx, ctx->io[3], sizeof(double) * (2 * N * m + 3 * N + ne)))) return rc;
  cudaStream_t st = ctx->stream;
  CK(cudaMemcpyAsync(ctx->io[1].p, frames, sizeof(double) * N * F, cudaMemcpyHostToDevice, st));
  double* d_phis = (double*)ctx->io[3].p;
  double* d_avg = d_phis + 2 * N * m;
  double* d_med = d_avg + N;
  double* d_cnt = d_med + N;
  double* d_e = d_cnt + N;
  rc = p->use_fp64 ? run_series<double>(ctx, *p, *s, (const double*)ctx->io[1].p, F, d_phis, d_e,
                                        average_out ? d_avg : nullptr, median_out ? d_med : nullptr, d_cnt, st)
                   : run_series<float>(ctx, *p, *s, (const double*)ctx->io[1].p, F, d_phis, d_e,
                                       average_out ? d_avg : nullptr, median_out ? d_med : nullptr, d_cnt, st);
  if (rc) return rc;
  CK(cudaMemcpyAsync(phis_out, d_phis, sizeof(double) * 2 * N * m, cudaMemcpyDeviceToHost, st));
  if (average_out) {
    CK(cudaMemcpyAsync(average_out, d_avg, sizeof(double) * N, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(count_out, d_cnt, sizeof(double) * N, cudaMemcpyDeviceToHost, st));
  }
  if (median_out) CK(cudaMemcpyAsync(median_out, d_med, sizeof(double) * N, cudaMemcpyDeviceToHost, st));
  if (energies_out) CK(cudaMemcpyAsync(energies_out, d_e, sizeof(double) * ne, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  return sched_error_check(ctx);
}

int msgpu_compose_device(msgpu_context* ctx, int level, const double* d_d1, const double* d_d2, double* d_inout,
                         void* stream) {
  if (!ctx) return MSGPU_ERR_INVALID_ARG;
  if (level < 1 || level > kMaxLevel || !d_d1 || !d_d2 || !d_inout)
    return fail(ctx, MSGPU_ERR_INVALID_ARG, "invalid compose arguments");
  if (d_inout == d_d1 || d_inout == d_d2)
    return fail(ctx, MSGPU_ERR_INVALID_ARG, "compose: inout must not alias d1 or d2");
  int rc;
  if ((rc = bind_device(ctx))) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  if ((rc = sched_error_reset(ctx, st))) return rc;
  ctx->stats.kernel_launches = 0;
  return compose_device(ctx, level, d_d1, d_d2, d_inout, st);
}

int msgpu_compose(msgpu_context* ctx, int level, const double* d1, const double* d2, double* inout,
                  int* iterations_out) {
  if (!ctx) return MSGPU_ERR_INVALID_ARG;
  if (level < 1 || level > kMaxLevel || !d1 || !d2 || !inout)
    return fail(ctx, MSGPU_ERR_INVALID_ARG, "invalid compose arguments");
  int rc;
  if ((rc = bind_device(ctx))) return rc;
  const size_t N = lvl_N(level);
  if ((rc = ensure(ctx, ctx->io[0], sizeof(double) * 6 * N))) return rc;
  double* dd = (double*)ctx->io[0].p;
  cudaStream_t st = ctx->stream;
  CK(cudaMemcpyAsync(dd, d1, sizeof(double) * 2 * N, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(dd + 2 * N, d2, sizeof(double) * 2 * N, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(dd + 4 * N, inout, sizeof(double) * 2 * N, cudaMemcpyHostToDevice, st));
  if ((rc = sched_error_reset(ctx, st))) return rc;
  ctx->stats.kernel_launches = 0;
  if ((rc = compose_device(ctx, level, dd, dd + 2 * N, dd + 4 * N, st))) return rc;
  CK(cudaMemcpyAsync(inout, dd + 4 * N, sizeof(double) * 2 * N, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  if ((rc = sched_error_check(ctx))) return rc;
  if (iterations_out && (rc = compose_iterations(ctx, level, iterations_out))) return rc;
  return MSGPU_OK;
}

int msgpu_warp_median_device(msgpu_context* ctx, int level, const double* d_frames, const double* d_phis,
                             int num_frames, double* d_median_out, void* stream) {
  if (!ctx) return MSGPU_ERR_INVALID_ARG;
  if (level < 1 || level > kMaxLevel || num_frames < 1 || !d_frames || !d_phis || !d_median_out)
    return fail(ctx, MSGPU_ERR_INVALID_ARG, "invalid warp_median arguments");
  int rc;
  if ((rc = bind_device(ctx))) return rc;
  ctx->stats.kernel_launches = 0;
  return average_median_device(ctx, level, d_frames, d_phis, num_frames, nullptr, d_median_out, nullptr,
                               (cudaStream_t)stream);
}

int msgpu_warp_median(msgpu_context* ctx, int level, const double* frames, const double* phis, int num_frames,
                      double* median_out) {
  if (!ctx) return MSGPU_ERR_INVALID_ARG;
  if (level < 1 || level > kMaxLevel || num_frames < 1 || !frames || !phis || !median_out)
    return fail(ctx, MSGPU_ERR_INVALID_ARG, "invalid warp_median arguments");
  int rc;
  if ((rc = bind_device(ctx))) return rc;
  const size_t N = lvl_N(level);
  const int F = num_frames;
  if ((rc = ensure(ctx, ctx->io[0], sizeof(double) * N * F))) return rc;
  if ((rc = ensure(ctx, ctx->io[1], sizeof(double) * 2 * N * F))) return rc;
  if ((rc = ensure(ctx, ctx->io[2], sizeof(double) * N))) return rc;
  cudaStream_t st = ctx->stream;
  CK(cudaMemcpyAsync(ctx->io[0].p, frames, sizeof(double) * N * F, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(ctx->io[1].p, phis, sizeof(double) * 2 * N * F, cudaMemcpyHostToDevice, st));
  if ((rc = msgpu_warp_median_device(ctx, level, (const double*)ctx->io[0].p, (const double*)ctx->io[1].p, F,
                                     (double*)ctx->io[2].p, st)))
    return rc;
  CK(cudaMemcpyAsync(median_out, ctx->io[2].p, sizeof(double) * N, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  return MSGPU_OK;
}

int msgpu_set_profiling(msgpu_context* ctx, int on) {
  if (!ctx) return MSGPU_ERR_INVALID_ARG;
  ctx->profiling = (on != 0);
  return MSGPU_OK;
}

int msgpu_set_trace(msgpu_context* ctx, int level, unsigned int capacity) {
  if (!ctx || level > kMaxLevel || capacity > (1u << 26)) return MSGPU_ERR_INVALID_ARG;
  ctx->trace_level = level;
  ctx->trace_cap = level < 0 ? 0u : capacity;
  ctx->trace_host.clear();
  return MSGPU_OK;
}

long long msgpu_get_trace(const msgpu_context* ctx, unsigned long long* out, long long capacity) {
  if (!ctx || capacity < 0 || (capacity > 0 && !out)) return -1;
  const long long n = (long long)(ctx->trace_host.size() / 2);
  const long long m = std::min(n, capacity);
  if (m > 0) std::memcpy(out, ctx->trace_host.data(), sizeof(unsigned long long) * 2 * (size_t)m);
  return n;
}

int msgpu_get_stats(const msgpu_context* ctx, msgpu_stats* out) {
  if (!ctx || !out) return MSGPU_ERR_INVALID_ARG;
  *out = ctx->stats;
  return MSGPU_OK;
}

int msgpu_warp_mean(msgpu_context* ctx, int level, const double* frames, const double* phis, int num_frames,
                    double* mean_out, double* count_out) {
  if (!ctx) return MSGPU_ERR_INVALID_ARG;
  if (level < 1 || level > kMaxLevel || num_frames < 1 || !frames || !phis || !mean_out || !count_out)
    return fail(ctx, MSGPU_ERR_INVALID_ARG, "invalid warp_mean arguments");
  int rc;
  if ((rc = bind_device(ctx))) return rc;
  const size_t N = lvl_N(level);
  const int F = num_frames;
  if ((rc = ensure(ctx, ctx->io[0], sizeof(double) * N * F))) return rc;
  if ((rc = ensure(ctx, ctx->io[1], sizeof(double) * 2 * N * F))) return rc;
  if ((rc = ensure(ctx, ctx->io[2], sizeof(double) * 2 * N))) return rc;
  cudaStream_t st = ctx->stream;
  CK(cudaMemcpyAsync(ctx->io[0].p, frames, sizeof(double) * N * F, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(ctx->io[1].p, phis, sizeof(double) * 2 * N * F, cudaMemcpyHostToDevice, st));
  double* dm = (double*)ctx->io[2].p;
  if ((rc = msgpu_warp_mean_device(ctx, level, (const double*)ctx->io[0].p, (const double*)ctx->io[1].p, F, dm,
                                    dm + N, st)))
    return rc;
  CK(cudaMemcpyAsync(mean_out, dm, sizeof(double) * N, cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(count_out, dm + N, sizeof(double) * N, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  return MSGPU_OK;
}

}  // extern "C"

// --- single operators ------------------------------------------------------

namespace {
// Runs the level kernel for ONE instance at `level` in the given mode with
// R/T/phi (and for MODE_SMOOTH the vector in the DE slot) uploaded from host.
template <typename Real>
int single_level(msgpu_context* ctx, int level, int mode, const double* R, const double* T, const double* phix,
                 const double* phiy, const double* de_in, double lambda, int max_iter, double stop_eps,
                 double sigma, double* energy_out, int* steps_out, double* phix_out, double* phiy_out,
                 double* de_out, double* trace, int max_trace, double* elog_out = nullptr) {
  int rc;
  if ((rc = ensure_tables(ctx))) return rc;
  const bool ncc = ctx->data_term == 1 && mode != MODE_SMOOTH;
  const Layout L = make_layout(level, ncc);
  if (ncc && (rc = ensure(ctx, ctx->nccbuf, sizeof(Real) * (comp_stride(level) + 64)))) return rc;
  const size_t N = lvl_N(level);
  if ((rc = ensure(ctx, ctx->arena, sizeof(Real) * L.stride))) return rc;
  if ((rc = ensure(ctx, ctx->shared_real, sizeof(Real) * (comp_stride(level) + 64)))) return rc;
  if ((rc = ensure(ctx, ctx->io[0], sizeof(double) * 6 * N))) return rc;
  const size_t trace_n = (size_t)std::max(1, max_trace) * 4;
  const size_t elog_n = (size_t)(std::max(0, max_trace) + 1) * 3;
  if ((rc = ensure(ctx, ctx->small, sizeof(double) * (8 + trace_n + elog_n) + 64))) return rc;
  cudaStream_t st = ctx->stream;
  Real* arena = (Real*)ctx->arena.p;
  Real* Rd = (Real*)ctx->shared_real.p;
  double* h = (double*)ctx->io[0].p;
  double* sm = (double*)ctx->small.p;
  double* d_e = sm;
  int* d_i = (int*)(sm + 2);  // steps, buf
  double* d_trace = sm + 8;
  CK(cudaMemsetAsync(arena, 0, sizeof(Real) * L.stride, st));
  const double* srcs[5] = {R, T, phix, phiy, de_in};
  for (int k = 0; k < 5; ++k)
    if (srcs[k]) CK(cudaMemcpyAsync(h + k * N, srcs[k], sizeof(double) * N, cudaMemcpyHostToDevice, st));
  const unsigned gx = (unsigned)std::min<size_t>(1024, (N + 255) / 256);
  const int nl = lvl_n(level);
  const size_t cs = comp_stride(level);
  if (R) k_to_pitched<double, Real><<<gx, 256, 0, st>>>(h, 0, Rd, 0, nl);
  if (T) k_to_pitched<double, Real><<<gx, 256, 0, st>>>(h + N, 0, arena + L.off_T[level], 0, nl);
  if (phix) k_to_pitched<double, Real><<<gx, 256, 0, st>>>(h + 2 * N, 0, arena + L.off_phi[0], 0, nl);
  if (phiy) k_to_pitched<double, Real><<<gx, 256, 0, st>>>(h + 3 * N, 0, arena + L.off_phi[0] + cs, 0, nl);
  if (de_in) k_to_pitched<double, Real><<<gx, 256, 0, st>>>(h + 4 * N, 0, arena + L.off_de, 0, nl);
  k_set_buf<Real><<<1, 32, 0, st>>>(d_i + 1, 1, 0);
  CK(cudaGetLastError());
  LevelArgs<Real> a;
  memset(&a, 0, sizeof(a));
  a.arena = arena;
  a.inst_stride = L.stride;
  a.R = Rd;
  if (ncc) {
    a.ncc = 1;
    a.normR = (const Real*)ctx->nccbuf.p;
    a.off_td = L.off_td;
    k_ncc_normalize<Real><<<1, 1024, 0, st>>>(Rd, nullptr, 0, 0, level, (Real*)ctx->nccbuf.p, 0);
  }
  a.off_T = L.off_T[level];
  a.off_phi[0] = L.off_phi[0];
  a.off_phi[1] = L.off_phi[1];
  a.off_d[0] = L.off_d[0];
  a.off_d[1] = L.off_d[1];
  a.off_s = L.off_s;
  a.off_de = L.off_de;
  for (int k = 0; k <= kMaxLevel; ++k) { a.off_x2[k] = L.off_x2[k]; a.off_x5[k] = L.off_x5[k]; a.off_b[k] = L.off_b[k]; }
  a.level = level;
  a.n = lvl_n(level);
  a.num_inst = 1;
  a.lc = pick_lc<Real>(level);
  a.mode = mode;
  a.lambda = lambda;
  a.stop_eps = stop_eps;
  a.sigma_fixed = sigma;
  a.max_iter = max_iter;
  a.phi_in_dev = d_i + 1;
  a.out_energy = d_e;
  a.out_steps = d_i;
  a.out_phi_buf = d_i + 1;
  a.trace = trace ? d_trace : nullptr;
  a.max_trace = max_trace;
  a.elog = elog_out ? d_trace + trace_n : nullptr;
  if ((rc = xs_attach<Real>(ctx, a, ctx->sum_order == 0 && mode != MODE_SMOOTH, level, 1))) return rc;
  if ((rc = sched_error_reset(ctx, st))) return rc;
  if ((rc = launch_level<Real>(ctx, a, st))) return rc;
  CK(cudaGetLastError());
  // outputs
  int hi[2] = {0, 0};
  double he = 0;
  CK(cudaMemcpyAsync(&he, d_e, sizeof(double), cudaMemcpyDeviceToHost, st));
  CK(cudaMemcpyAsync(hi, d_i, sizeof(int) * 2, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  if ((rc = sched_error_check(ctx))) return rc;
  if (energy_out) *energy_out = he;
  if (steps_out) *steps_out = hi[0];
  auto fetch = [&](size_t off, double* dst) -> int {
    k_from_pitched<Real, double><<<gx, 256, 0, st>>>(arena + off, 0, h + 5 * N, 0, nl);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(dst, h + 5 * N, sizeof(double) * N, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    return MSGPU_OK;
  };
  if (mode == MODE_SMOOTH) {
    if ((rc = fetch(L.off_s, de_out))) return rc;
    return MSGPU_OK;
  }
  if (de_out) {
    if ((rc = fetch(L.off_de, de_out))) return rc;
    if ((rc = fetch(L.off_de + cs, de_out + N))) return rc;
  }
  const size_t phioff = hi[1] ? L.off_phi[1] : L.off_phi[0];
  if (phix_out && (rc = fetch(phioff, phix_out))) return rc;
  if (phiy_out && (rc = fetch(phioff + cs, phiy_out))) return rc;
  if (trace && max_trace > 0) {
    const int rows = std::min(hi[0], max_trace);
    CK(cudaMemcpy(trace, d_trace, sizeof(double) * 4 * rows, cudaMemcpyDeviceToHost));
  }
  if (elog_out) {
    const int rows = std::min(hi[0], max_trace) + 1;
    CK(cudaMemcpy(elog_out, d_trace + trace_n, sizeof(double) * 3 * rows, cudaMemcpyDeviceToHost));
  }
  return MSGPU_OK;
}
}  // namespace

extern "C" {

int msgpu_energy(msgpu_context* ctx, int level, const double* R, const double* T, const double* phix,
                 const double* phiy, double lambda, int use_fp64, double* energy_out, double* de_out) {
  if (!ctx) return MSGPU_ERR_INVALID_ARG;
  if (level < 1 || level > kMaxLevel || !R || !T || !phix || !phiy)
    return fail(ctx, MSGPU_ERR_INVALID_ARG, "invalid energy arguments");
  int rc;
  if ((rc = bind_device(ctx))) return rc;
  return use_fp64 ? single_level<double>(ctx, level, MODE_ENERGY, R, T, phix, phiy, nullptr, lambda, 0, 0, 0,
                                         energy_out, nullptr, nullptr, nullptr, de_out, nullptr, 0)
                  : single_level<float>(ctx, level, MODE_ENERGY, R, T, phix, phiy, nullptr, lambda, 0, 0, 0,
                                        energy_out, nullptr, nullptr, nullptr, de_out, nullptr, 0);
}

int msgpu_smooth(msgpu_context* ctx, int level, double sigma, int use_fp64, const double* in, double* out) {
  if (!ctx) return MSGPU_ERR_INVALID_ARG;
  if (level < 1 || level > kMaxLevel || !in || !out) return fail(ctx, MSGPU_ERR_INVALID_ARG, "invalid smooth arguments");
  int rc;
  if ((rc = bind_device(ctx))) return rc;
  // the V-cycle smooths -DE: place -in into the DE slot (exact negation)
  const size_t N = lvl_N(level);
  std::vector<double> neg(N);
  for (size_t i = 0; i < N; ++i) neg[i] = in[i] * -1.0;
  return use_fp64 ? single_level<double>(ctx, level, MODE_SMOOTH, nullptr, nullptr, nullptr, nullptr, neg.data(),
                                         1.0, 0, 0, sigma, nullptr, nullptr, nullptr, nullptr, out, nullptr, 0)
                  : single_level<float>(ctx, level, MODE_SMOOTH, nullptr, nullptr, nullptr, nullptr, neg.data(),
                                        1.0, 0, 0, sigma, nullptr, nullptr, nullptr, nullptr, out, nullptr, 0);
}

int msgpu_gd_level(msgpu_context* ctx, int level, const double* R, const double* T, double* phix, double* phiy,
                   double lambda, int max_iter, double stop_eps, int use_fp64, double* energy_out, int* steps_out,
                   double* trace, int max_trace) {
  if (!ctx) return MSGPU_ERR_INVALID_ARG;
  if (level < 1 || level > kMaxLevel || !R || !T || !phix || !phiy || max_iter < 0)
    return fail(ctx, MSGPU_ERR_INVALID_ARG, "invalid gd_level arguments");
  int rc;
  if ((rc = bind_device(ctx))) return rc;
  return use_fp64 ? single_level<double>(ctx, level, MODE_SOLVE, R, T, phix, phiy, nullptr, lambda, max_iter,
                                         stop_eps, 0, energy_out, steps_out, phix, phiy, nullptr, trace, max_trace)
                  : single_level<float>(ctx, level, MODE_SOLVE, R, T, phix, phiy, nullptr, lambda, max_iter,
                                        stop_eps, 0, energy_out, steps_out, phix, phiy, nullptr, trace, max_trace);
}

int msgpu_gd_level_log(msgpu_context* ctx, int level, const double* R, const double* T, double* phix,
                       double* phiy, double lambda, int max_iter, double stop_eps, int use_fp64, double* energy_out,
                       int* steps_out, double* energy_log, int max_rows) {
  if (!ctx) return MSGPU_ERR_INVALID_ARG;
  if (level < 1 || level > kMaxLevel || !R || !T || !phix || !phiy || max_iter < 0 || !energy_log || max_rows < 1)
    return fail(ctx, MSGPU_ERR_INVALID_ARG, "invalid gd_level_log arguments");
  int rc;
  if ((rc = bind_device(ctx))) return rc;
  const int mt = max_rows - 1;
  return use_fp64 ? single_level<double>(ctx, level, MODE_SOLVE, R, T, phix, phiy, nullptr, lambda, max_iter,
                                         stop_eps, 0, energy_out, steps_out, phix, phiy, nullptr, nullptr, mt,
                                         energy_log)
                  : single_level<float>(ctx, level, MODE_SOLVE, R, T, phix, phiy, nullptr, lambda, max_iter,
                                        stop_eps, 0, energy_out, steps_out, phix, phiy, nullptr, nullptr, mt,
                                        energy_log);
}

int msgpu_restrict(msgpu_context* ctx, int fine_level, const double* in, double* out) {
  if (!ctx) return MSGPU_ERR_INVALID_ARG;
  if (fine_level < 1 || fine_level > kMaxLevel || !in || !out)
    return fail(ctx, MSGPU_ERR_INVALID_ARG, "invalid restrict arguments");
  int rc;
  if ((rc = bind_device(ctx))) return rc;
  const size_t Nf = lvl_N(fine_level), Nc = lvl_N(fine_level - 1);
  if ((rc = ensure(ctx, ctx->io[0], sizeof(double) * (Nf + Nc)))) return rc;
  double* d = (double*)ctx->io[0].p;
  cudaStream_t st = ctx->stream;
  CK(cudaMemcpyAsync(d, in, sizeof(double) * Nf, cudaMemcpyHostToDevice, st));
  k_restrict<double><<<dim3((unsigned)std::min<size_t>(1024, (Nc + 255) / 256), 1), 256, 0, st>>>(d, 0, d + Nf, 0,
                                                                                                 fine_level);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(out, d + Nf, sizeof(double) * Nc, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  return MSGPU_OK;
}

int msgpu_prolong(msgpu_context* ctx, int coarse_level, const double* in, double* out) {
  if (!ctx) return MSGPU_ERR_INVALID_ARG;
  if (coarse_level < 0 || coarse_level >= kMaxLevel || !in || !out)
    return fail(ctx, MSGPU_ERR_INVALID_ARG, "invalid prolong arguments");
  int rc;
  if ((rc = bind_device(ctx))) return rc;
  const size_t Nc = lvl_N(coarse_level), Nf = lvl_N(coarse_level + 1);
  if ((rc = ensure(ctx, ctx->io[0], sizeof(double) * (Nf + Nc)))) return rc;
  double* d = (double*)ctx->io[0].p;
  cudaStream_t st = ctx->stream;
  CK(cudaMemcpyAsync(d, in, sizeof(double) * Nc, cudaMemcpyHostToDevice, st));
  k_prolong<double><<<dim3((unsigned)std::min<size_t>(1024, (Nf + 255) / 256), 1), 256, 0, st>>>(d, 0, d + Nc, 0,
                                                                                                coarse_level);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(out, d + Nc, sizeof(double) * Nf, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  return MSGPU_OK;
}

int msgpu_normalize(msgpu_context* ctx, const double* in, int count, double saturation_percent,
                    int normalize_min_to_zero, double* out) {
  if (!ctx) return MSGPU_ERR_INVALID_ARG;
  if (!in || !out || count < 1) return fail(ctx, MSGPU_ERR_INVALID_ARG, "invalid normalize arguments");
  int rc;
  if ((rc = bind_device(ctx))) return rc;
  if ((rc = ensure(ctx, ctx->io[0], sizeof(double) * (count + 8)))) return rc;
  double* d = (double*)ctx->io[0].p;
  double* mm = d + count;
  cudaStream_t st = ctx->stream;
  CK(cudaMemcpyAsync(d, in, sizeof(double) * count, cudaMemcpyHostToDevice, st));
  if (saturation_percent >= 0) {
    const int m1 = count - 1;
    int il = (int)(saturation_percent / 200 * m1), ih = (int)((1 - saturation_percent / 200) * m1);
    il = std::min(std::max(il, 0), m1);
    ih = std::min(std::max(ih, 0), m1);
    k_select2<<<1, kSelThreads, 0, st>>>(d, 0, count, il, ih, mm);
  } else {
    k_minmax<<<1, 1024, 0, st>>>(d, 0, count, mm);
  }
  k_normalize<<<dim3((unsigned)std::min(1024, (count + 255) / 256), 1), 256, 0, st>>>(
      d, 0, count, mm, saturation_percent >= 0 ? 1 : 0, normalize_min_to_zero);
  CK(cudaGetLastError());
  CK(cudaMemcpyAsync(out, d, sizeof(double) * count, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  return MSGPU_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Allocation-free level solve (msgpu_gd_level_noalloc).
//
// Some callers cannot allocate device memory: an application whose device
// memory is owned by its own pool allocator (which forbids other code from
// calling cudaMalloc / cudaFree behind its back, because those calls
// synchronise the device and fragment the pool), or a host that admits only
// code with a fixed, known device footprint.  For them this entry point runs
// the same level kernel as msgpu_gd_level with all of its scratch (the
// pitched copies of the images, the per-level arena of the gradient flow and
// the multigrid pyramid) carved out of one file-scope device array, so no
// device memory is allocated per call; the caller passes only inputs and
// outputs.
namespace {

// Size of the scratch array: enough for one level-8 solve (257^2 nodes) in
// FP64 (11.45 MB needed); every GPU that loads this library holds it until
// the process exits.
constexpr size_t kNoAllocScratchBytes = (size_t)12 << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

struct NoAllocDevice {
  bool ready = false;
  unsigned char* scratch = nullptr;  // device address of g_noalloc_scratch
  int sms = 0;
};
constexpr int kNoAllocMaxDevices = 64;
NoAllocDevice g_noalloc_dev[kNoAllocMaxDevices];
std::mutex g_noalloc_mu;

size_t noalloc_bytes_needed(int level, size_t real_bytes) {
  const Layout L = make_layout(level);
  return align_up(real_bytes * L.stride, 256) + align_up(real_bytes * (comp_stride(level) + 64), 256) + 256 +
         sched_bytes(1, level_max_tiles(level));
}

// Per-device set-up, run by the first call on a device with that device
// current: the device address of the scratch array, the finite-element
// tables in constant memory, the SM count.
int noalloc_setup(int dev, NoAllocDevice** out) {
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  NoAllocDevice& d = g_noalloc_dev[dev];
  if (!d.ready) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || p == nullptr) return MSGPU_ERR_CUDA;
    FeTables t;
    host_fe_tables(t);
    if (cudaMemcpyToSymbol(c_fe, &t, sizeof(t)) != cudaSuccess) return MSGPU_ERR_CUDA;
    // the upload must have landed before kernels on the caller's stream read it
    if (cudaDeviceSynchronize() != cudaSuccess) return MSGPU_ERR_CUDA;
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms < 1)
      return MSGPU_ERR_CUDA;
    d.scratch = (unsigned char*)p;
    d.sms = sms;
    d.ready = true;
  }
  *out = &d;
  return MSGPU_OK;
}

// Marks the outputs of a level solve whose scheduler gave up (error flag set).
__global__ void k_noalloc_status(const int* err, double* energy, int* steps) {
  if (threadIdx.x == 0 && *err) {
    *steps = -1;
    *energy = __longlong_as_double(0x7ff8000000000000ll);
  }
}

#define NA_CK(call)                                \
  do {                                             \
    if ((call) != cudaSuccess) return MSGPU_ERR_CUDA; \
  } while (0)

template <typename Real>
int noalloc_level(const NoAllocDevice& dv, int level, const double* d_R, const double* d_T, double* d_phi,
                  double lambda, int max_iter, double stop_eps, double* d_energy, int* d_steps, cudaStream_t st) {
  const Layout L = make_layout(level);
  const size_t cs = comp_stride(level);
  const size_t arena_b = align_up(sizeof(Real) * L.stride, 256);
  const size_t ref_b = align_up(sizeof(Real) * (cs + 64), 256);
  Real* arena = (Real*)dv.scratch;
  Real* Rd = (Real*)(dv.scratch + arena_b);
  double* e_slot = (double*)(dv.scratch + arena_b + ref_b);
  int* i_slot = (int*)(e_slot + 1);  // [0] steps, [1] buffer holding phi; e_slot[4]: scheduler error flag
  // The scratch keeps the previous call's contents: clear everything the
  // kernel reads before writing (as the allocating entry point does).
  NA_CK(cudaMemsetAsync(dv.scratch, 0, arena_b + ref_b + 256, st));
  const int nl = lvl_n(level);
  const size_t N = lvl_N(level);
  const unsigned gx = (unsigned)std::min<size_t>(1024, (N + 255) / 256);
  k_to_pitched<double, Real><<<gx, 256, 0, st>>>(d_R, 0, Rd, 0, nl);
  k_to_pitched<double, Real><<<gx, 256, 0, st>>>(d_T, 0, arena + L.off_T[level], 0, nl);
  k_to_pitched<double, Real><<<gx, 256, 0, st>>>(d_phi, 0, arena + L.off_phi[0], 0, nl);
  k_to_pitched<double, Real><<<gx, 256, 0, st>>>(d_phi + N, 0, arena + L.off_phi[0] + cs, 0, nl);
  NA_CK(cudaGetLastError());
  LevelArgs<Real> a;
  memset(&a, 0, sizeof(a));
  a.arena = arena;
  a.inst_stride = L.stride;
  a.R = Rd;
  a.off_T = L.off_T[level];
  a.off_phi[0] = L.off_phi[0];
  a.off_phi[1] = L.off_phi[1];
  a.off_d[0] = L.off_d[0];
  a.off_d[1] = L.off_d[1];
  a.off_s = L.off_s;
  a.off_de = L.off_de;
  for (int k = 0; k <= kMaxLevel; ++k) { a.off_x2[k] = L.off_x2[k]; a.off_x5[k] = L.off_x5[k]; a.off_b[k] = L.off_b[k]; }
  a.level = level;
  a.n = nl;
  a.num_inst = 1;
  a.lc = pick_lc<Real>(level);
  a.mode = MODE_SOLVE;
  a.lambda = lambda;
  a.stop_eps = stop_eps;
  a.sigma_fixed = 0;
  a.max_iter = max_iter;
  a.phi_in_dev = i_slot + 1;  // zeroed above: phi starts in buffer 0
  a.out_energy = d_energy ? d_energy : e_slot;
  a.out_steps = d_steps ? d_steps : i_slot;
  a.out_phi_buf = i_slot + 1;
  // the level kernel's scheduler state follows the other scratch
  unsigned char* sched = dv.scratch + arena_b + ref_b + 256;
  int* err = (int*)(e_slot + 4);
  NA_CK(launch_level_core<Real>(a, sched, err, dv.sms, st, nullptr));
  // result: [phi_x, phi_y] dense, from whichever buffer the solve ended in
  k_phi_out<Real><<<dim3(gx, 1), 256, 0, st>>>(arena, L.stride, L.off_phi[0], L.off_phi[1], level, i_slot + 1,
                                               d_phi);
  // a worker that gave up waiting leaves an unfinished solve: mark it in the
  // outputs (steps -1, energy NaN), since the call does not wait for the GPU
  k_noalloc_status<<<1, 32, 0, st>>>(err, a.out_energy, a.out_steps);
  NA_CK(cudaGetLastError());
  return MSGPU_OK;
}
#undef NA_CK

}  // namespace

extern "C" int msgpu_gd_level_noalloc(int level, const double* d_R, const double* d_T, double* d_phi,
                                      double lambda, int max_iter, double stop_eps, int use_fp64,
                                      double* d_energy_out, int* d_steps_out, void* stream) {
  if (level < 1 || level > kMaxLevel || !d_R || !d_T || !d_phi || max_iter < 0) return MSGPU_ERR_INVALID_ARG;
  if (noalloc_bytes_needed(level, use_fp64 ? sizeof(double) : sizeof(float)) > kNoAllocScratchBytes)
    return MSGPU_ERR_SIZE;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return MSGPU_ERR_CUDA;
  if (dev < 0 || dev >= kNoAllocMaxDevices) return MSGPU_ERR_UNSUPPORTED;
  NoAllocDevice* dv = nullptr;
  int rc = noalloc_setup(dev, &dv);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  return use_fp64 ? noalloc_level<double>(*dv, level, d_R, d_T, d_phi, lambda, max_iter, stop_eps, d_energy_out,
                                          d_steps_out, st)
                  : noalloc_level<float>(*dv, level, d_R, d_T, d_phi, lambda, max_iter, stop_eps, d_energy_out,
                                         d_steps_out, st);
}

// ---------------------------------------------------------------------------
// Learned warm start: the U-Net of msgpu_unet.cuh, its training step and its
// use as the start of the gradient flow.

namespace {
using msg::unet::bf16;

struct NetLayer {
  int cin, cout, stride, relu;
  int cin_pad, cout_pad;
  size_t w_off, b_off;     // in theta / grad (floats)
  size_t wf_off, wt_off;   // in the packed bf16 weights
};

// (cin, cout, stride, relu) of e0a e0b e1a e1b e2a e2b e3a e3b d2a d2b d1a d1b head
constexpr int kNetLayers = 13;
constexpr int kNetSpec[kNetLayers][4] = {{2, 16, 1, 1},   {16, 16, 1, 1},  {16, 32, 2, 1},   {32, 32, 1, 1},
                                         {32, 64, 2, 1},  {64, 64, 1, 1},  {64, 128, 2, 1},  {128, 128, 1, 1},
                                         {192, 64, 1, 1}, {64, 64, 1, 1},  {96, 32, 1, 1},   {32, 32, 1, 1},
                                         {32, 2, 1, 0}};
enum { E0A, E0B, E1A, E1B, E2A, E2B, E3A, E3B, D2A, D2B, D1A, D1B, HEAD };

inline int pad16(int c) { return (c + 15) / 16 * 16; }
// widest tile of 64, 32 or 16 channels that divides a padded channel count
inline int tile_of(int rows) { return rows % 64 == 0 ? 64 : (rows % 32 == 0 ? 32 : 16); }

// An NHWC bf16 tensor view: base (channel offset applied), image stride,
// nodes per side, elements per node.
struct View {
  bf16* p;
  size_t img;
  int n, cs;
  View ch(int c0) const { return View{p + c0, img, n, cs}; }
};
}  // namespace

struct msgpu_net {
  msgpu_context* ctx = nullptr;
  int level = 0;          // input grid 2^level + 1; output grid one level coarser
  int n[4] = {};          // nodes per side of the four grids
  NetLayer L[kNetLayers];
  size_t nparams = 0, npacked = 0;
  float *theta = nullptr, *grad = nullptr, *m = nullptr, *v = nullptr;
  bf16 *wf = nullptr, *wt = nullptr;
  long long step = 0;
  int batch = 0;                         // images the activation buffers hold
  msgpu_context::Buf act, part, small, phi, gather, phiall;
  // activations and their gradients (views into act)
  View x0, a0, a1, b0, cat1, c0, cat2, d0, d1, g0, g1, h0, h1;
  View dout, dh1, dh0, dcat1, dg1, dg0, dcat2, dd1, dd0, dc0, db0, da1, da0;
  float* out = nullptr;                  // head output, 2 floats per node of grid 1
  bool tcgen05 = true;                   // forward convolutions on tcgen05 (else mma.sync)
};

namespace {

#define NCK(call)                                                                                 \
  do {                                                                                            \
    cudaError_t e_ = (call);                                                                      \
    if (e_ != cudaSuccess)                                                                        \
      return fail(net->ctx, MSGPU_ERR_CUDA, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), \
                  __FILE__, __LINE__);                                                            \
  } while (0)

size_t net_param_count() {
  size_t n = 0;
  for (int i = 0; i < kNetLayers; ++i) n += (size_t)kNetSpec[i][1] * 9 * kNetSpec[i][0] + kNetSpec[i][1];
  return n;
}

int net_pack(msgpu_net* net, cudaStream_t st) {
  for (int i = 0; i < kNetLayers; ++i) {
    const NetLayer& l = net->L[i];
    const int n = l.cout_pad * 9 * l.cin_pad;
    msg::unet::k_pack_weights<<<std::min(1024, (n + 255) / 256), 256, 0, st>>>(
        net->theta + l.w_off, l.cout, l.cin, l.cout_pad, l.cin_pad, net->wf + l.wf_off, net->wt + l.wt_off);
  }
  NCK(cudaGetLastError());
  net->ctx->stats.kernel_launches += kNetLayers;
  return MSGPU_OK;
}

// Activation buffers for `batch` images.
int net_buffers(msgpu_net* net, int batch, cudaStream_t st) {
  if (batch <= net->batch) return MSGPU_OK;
  const size_t N[4] = {(size_t)net->n[0] * net->n[0], (size_t)net->n[1] * net->n[1], (size_t)net->n[2] * net->n[2],
                       (size_t)net->n[3] * net->n[3]};
  struct Spec { View* v; int g, c; };
  Spec specs[] = {{&net->x0, 0, 16},   {&net->a0, 0, 16},   {&net->a1, 0, 16},   {&net->b0, 1, 32},
                  {&net->cat1, 1, 96}, {&net->c0, 2, 64},   {&net->cat2, 2, 192}, {&net->d0, 3, 128},
                  {&net->d1, 3, 128},  {&net->g0, 2, 64},   {&net->g1, 2, 64},   {&net->h0, 1, 32},
                  {&net->h1, 1, 32},   {&net->dout, 1, 16}, {&net->dh1, 1, 32},  {&net->dh0, 1, 32},
                  {&net->dcat1, 1, 96}, {&net->dg1, 2, 64}, {&net->dg0, 2, 64},  {&net->dcat2, 2, 192},
                  {&net->dd1, 3, 128}, {&net->dd0, 3, 128}, {&net->dc0, 2, 64},  {&net->db0, 1, 32},
                  {&net->da1, 0, 16},  {&net->da0, 0, 16}};
  size_t total = 0;
  for (const Spec& s : specs) total += align_up(N[s.g] * s.c * batch, 128);
  const size_t out_floats = align_up(N[1] * 2 * batch, 64);
  int rc;
  if ((rc = ensure(net->ctx, net->act, total * sizeof(bf16) + out_floats * sizeof(float)))) return rc;
  bf16* p = (bf16*)net->act.p;
  for (const Spec& s : specs) {
    *s.v = View{p, N[s.g] * s.c, net->n[s.g], s.c};
    p += align_up(N[s.g] * s.c * batch, 128);
  }
  net->out = (float*)p;
  // zero once: padding channels of the input and of the loss gradient stay zero
  NCK(cudaMemsetAsync(net->act.p, 0, total * sizeof(bf16) + out_floats * sizeof(float), st));
  net->batch = batch;
  return MSGPU_OK;
}

// 16-channel outputs: 16 rows per block (four m16 tiles per warp), wider: 8 rows
template <int BN, int CIN>
void net_launch_halo(const msg::unet::ConvArgs& a, int images, int rows, cudaStream_t st) {
  namespace u = msg::unet;
  constexpr int MT = BN == 16 ? 4 : 2;
  const int ty = 4 * MT;
  const int tiles = ((a.out_n + ty - 1) / ty) * ((a.out_n + u::kHaloX - 1) / u::kHaloX);
  const dim3 grid((unsigned)(images * tiles), (unsigned)(rows / BN));
  u::k_conv_halo<BN, CIN, MT><<<grid, u::kThreads, u::conv_halo_smem_bytes<BN, CIN, MT>(), st>>>(a);
}

// shared-memory limits of the halo kernels (above the 48 KB default for the widest)
int net_kernel_attrs(msgpu_context* ctx) {
  namespace u = msg::unet;
  CK(cudaFuncSetAttribute(u::k_conv_halo<64, 32, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                          (int)u::conv_halo_smem_bytes<64, 32, 2>()));
  CK(cudaFuncSetAttribute(u::k_conv_halo<64, 16, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                          (int)u::conv_halo_smem_bytes<64, 16, 2>()));
  CK(cudaFuncSetAttribute(u::k_conv_halo<32, 32, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                          (int)u::conv_halo_smem_bytes<32, 32, 2>()));
  CK(cudaFuncSetAttribute(u::k_conv_tc<16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                          (int)u::conv_tc_smem_bytes<16>()));
  CK(cudaFuncSetAttribute(u::k_conv_tc<32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                          (int)u::conv_tc_smem_bytes<32>()));
  CK(cudaFuncSetAttribute(u::k_conv_tc<64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                          (int)u::conv_tc_smem_bytes<64>()));
  CK(cudaFuncSetAttribute(u::k_conv_tc<128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                          (int)u::conv_tc_smem_bytes<128>()));
  const int row_max = 200 * 1024;
  CK(cudaFuncSetAttribute(u::k_conv_row_tc<16, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, row_max));
  CK(cudaFuncSetAttribute(u::k_conv_row_tc<32, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, row_max));
  CK(cudaFuncSetAttribute(u::k_conv_row_tc<64, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, row_max));
  CK(cudaFuncSetAttribute(u::k_conv_row_tc<128, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, row_max));
  CK(cudaFuncSetAttribute(u::k_conv_row_tc<16, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, row_max));
  CK(cudaFuncSetAttribute(u::k_conv_row_tc<32, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, row_max));
  CK(cudaFuncSetAttribute(u::k_conv_row_tc<64, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, row_max));
  CK(cudaFuncSetAttribute(u::k_conv_row_tc<128, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, row_max));
  const int tma_max = 200 * 1024 + 1024 + 128;
  CK(cudaFuncSetAttribute(u::k_conv_row_tma<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, tma_max));
  CK(cudaFuncSetAttribute(u::k_conv_row_tma<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, tma_max));
  CK(cudaFuncSetAttribute(u::k_conv_row_tma<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, tma_max));
  CK(cudaFuncSetAttribute(u::k_conv_row_tma<128>, cudaFuncAttributeMaxDynamicSharedMemorySize, tma_max));
  return MSGPU_OK;
}

// The driver's tensor-map encoder, found through the runtime (no link
// dependency on the driver library); null when the driver does not offer it.
typedef CUresult (*TmapEncodeFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
TmapEncodeFn tmap_encoder() {
  static TmapEncodeFn fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<TmapEncodeFn>(p);
  }
  return fn;
}

// Stride-1 forward convolution on tcgen05 with TMA-fed operands: tensor maps
// over the input view (channels, x, y, image; out-of-grid boxes filled with
// zeros) and over the weight matrix (K, rows).  false: not launched (no
// encoder, or a map the encoder refuses).
template <int BN>
bool net_launch_row_tma(const msg::unet::ConvArgs& a, int rows, int sms, int* err, cudaStream_t st) {
  namespace u = msg::unet;
  const TmapEncodeFn enc = tmap_encoder();
  if (!enc) return false;
  int G = 0;
  for (int pass = 0; pass < 2 && !G; ++pass) {
    const size_t cap = pass == 0 ? 110 * 1024 : 200 * 1024;
    for (int g : {64, 48, 32, 16})
      if (a.cin % g == 0 && u::row_tma_smem(BN, g) <= cap) { G = g; break; }
  }
  if (!G) return false;
  const size_t smem = u::row_tma_smem(BN, G);
  const int R = u::row_tc_rows(BN);
  const int images = a.total / (a.out_n * a.out_n);
  CUtensorMap tin, tw;
  const cuuint64_t gd[4] = {(cuuint64_t)a.cin, (cuuint64_t)a.in_n, (cuuint64_t)a.in_n, (cuuint64_t)images};
  const cuuint64_t gs[3] = {(cuuint64_t)a.in_cs * 2, (cuuint64_t)a.in_n * a.in_cs * 2, (cuuint64_t)a.in_img * 2};
  const cuuint32_t box[4] = {8, 130, (cuuint32_t)(R + 2), 1};
  const cuuint32_t es[4] = {1, 1, 1, 1};
  if (enc(&tin, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, (void*)a.in, gd, gs, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
          CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) !=
      CUDA_SUCCESS)
    return false;
  const cuuint64_t K = (cuuint64_t)9 * a.cin;
  const cuuint64_t wd[2] = {K, (cuuint64_t)rows};
  const cuuint64_t ws[1] = {K * 2};
  const cuuint32_t wbox[2] = {8, (cuuint32_t)BN};
  const cuuint32_t wes[2] = {1, 1};
  if (enc(&tw, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, (void*)a.w, wd, ws, wbox, wes, CU_TENSOR_MAP_INTERLEAVE_NONE,
          CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) !=
      CUDA_SUCCESS)
    return false;
  const int per_sm = std::max(1, std::min((int)((227 * 1024) / (smem + 1024)), 512 / u::row_tma_cols<BN>()));
  const int segs = (a.out_n + u::kTcBM - 1) / u::kTcBM;
  const int tiles = images * ((a.out_n + R - 1) / R) * segs;
  const int ny = rows / BN;
  const int gx = std::max(1, std::min(tiles, (sms * per_sm + ny - 1) / ny));
  u::k_conv_row_tma<BN><<<dim3((unsigned)gx, (unsigned)ny), u::kRowTmaThreads, smem, st>>>(a, G, err, tin, tw);
  return true;
}

// Launches the row-tiled tensor-core convolution: the channel group G is the
// largest of 64, 48, 32, 16 dividing cin whose two shared-memory slots fit
// two CTAs per SM (else one); persistent CTAs over the row tiles.
template <int BN, int S>
void net_launch_row_tc(const msg::unet::ConvArgs& a, int rows, int sms, int* err, cudaStream_t st) {
  namespace u = msg::unet;
  int G = 16;
  size_t smem = u::row_tc_smem<BN, S>(16);
  for (int pass = 0; pass < 2; ++pass) {
    const size_t cap = pass == 0 ? 110 * 1024 : 200 * 1024;
    bool found = false;
    for (int g : {64, 48, 32, 16}) {
      if (a.cin % g || u::row_tc_smem<BN, S>(g) > cap) continue;
      G = g;
      smem = u::row_tc_smem<BN, S>(g);
      found = true;
      break;
    }
    if (found) break;
  }
  // CTAs per SM: by shared memory and by TMEM (512 columns)
  const int per_sm = std::max(1, std::min((int)((227 * 1024) / (smem + 1024)), 512 / u::row_tc_cols<BN>()));
  const int segs = (a.out_n + u::kTcBM - 1) / u::kTcBM;
  const int R = u::row_tc_rows(BN);
  const int tiles = (a.total / (a.out_n * a.out_n)) * ((a.out_n + R - 1) / R) * segs;
  const int ny = rows / BN;
  const int gx = std::max(1, std::min(tiles, (sms * per_sm + ny - 1) / ny));
  u::k_conv_row_tc<BN, S><<<dim3((unsigned)gx, (unsigned)ny), 128, smem, st>>>(a, G, err);
}

int net_conv_launch(msgpu_net* net, const msg::unet::ConvArgs& a, int rows, cudaStream_t st) {
  const int bn = tile_of(rows);
  // forward convolutions on tcgen05 where it measured faster (B200, 8 pairs
  // at 1025^2): stride 1 with 16 input channels, or with 64 and more input
  // channels and at most 64 output rows; stride 2, the 32-channel layers and
  // the 128-row layer (whose 129-node rows leave half of its second tile
  // empty) run on the mma.sync kernels below
  if (net->tcgen05 && a.mode == 0 && a.stride == 1 && (a.cin == 16 || (a.cin >= 64 && rows <= 64))) {
    namespace u = msg::unet;
    int rc;
    if (!net->ctx->sched_error && (rc = sched_error_reset(net->ctx, st))) return rc;
    const int tb = rows % 128 == 0 ? 128 : bn;
    int* err = net->ctx->sched_error + 3;
    const int sms = net->ctx->sm_count;
    bool tma = false;
    if (a.stride == 1) {
      if (tb == 128) tma = net_launch_row_tma<128>(a, rows, sms, err, st);
      else if (tb == 64) tma = net_launch_row_tma<64>(a, rows, sms, err, st);
      else if (tb == 32) tma = net_launch_row_tma<32>(a, rows, sms, err, st);
      else tma = net_launch_row_tma<16>(a, rows, sms, err, st);
    }
    if (tma) {
    } else if (a.stride == 1) {
      if (tb == 128) net_launch_row_tc<128, 1>(a, rows, sms, err, st);
      else if (tb == 64) net_launch_row_tc<64, 1>(a, rows, sms, err, st);
      else if (tb == 32) net_launch_row_tc<32, 1>(a, rows, sms, err, st);
      else net_launch_row_tc<16, 1>(a, rows, sms, err, st);
    } else if (a.stride == 2) {
      if (tb == 128) net_launch_row_tc<128, 2>(a, rows, sms, err, st);
      else if (tb == 64) net_launch_row_tc<64, 2>(a, rows, sms, err, st);
      else if (tb == 32) net_launch_row_tc<32, 2>(a, rows, sms, err, st);
      else net_launch_row_tc<16, 2>(a, rows, sms, err, st);
    } else {
      const dim3 grid((unsigned)((a.total + u::kTcBM - 1) / u::kTcBM), (unsigned)(rows / tb));
      if (tb == 128) u::k_conv_tc<128><<<grid, 128, u::conv_tc_smem_bytes<128>(), st>>>(a, err);
      else if (tb == 64) u::k_conv_tc<64><<<grid, 128, u::conv_tc_smem_bytes<64>(), st>>>(a, err);
      else if (tb == 32) u::k_conv_tc<32><<<grid, 128, u::conv_tc_smem_bytes<32>(), st>>>(a, err);
      else u::k_conv_tc<16><<<grid, 128, u::conv_tc_smem_bytes<16>(), st>>>(a, err);
    }
    NCK(cudaGetLastError());
    ++net->ctx->stats.kernel_launches;
    return MSGPU_OK;
  }
  if (a.stride == 1 && (a.cin == 16 || a.cin == 32)) {
    // narrow stride-1 layers: every input node fetched once through a halo tile
    const int images = a.total / (a.out_n * a.out_n);
    if (a.cin == 16) {
      if (bn == 64) net_launch_halo<64, 16>(a, images, rows, st);
      else if (bn == 32) net_launch_halo<32, 16>(a, images, rows, st);
      else net_launch_halo<16, 16>(a, images, rows, st);
    } else {
      if (bn == 64) net_launch_halo<64, 32>(a, images, rows, st);
      else if (bn == 32) net_launch_halo<32, 32>(a, images, rows, st);
      else net_launch_halo<16, 32>(a, images, rows, st);
    }
    NCK(cudaGetLastError());
    ++net->ctx->stats.kernel_launches;
    return MSGPU_OK;
  }
  namespace u = msg::unet;
  const dim3 grid((unsigned)((a.total + u::kConvBM - 1) / u::kConvBM), (unsigned)(rows / bn));
  if (bn == 64) u::k_conv<64><<<grid, u::kThreads, u::conv_smem_bytes<64>(), st>>>(a);
  else if (bn == 32) u::k_conv<32><<<grid, u::kThreads, u::conv_smem_bytes<32>(), st>>>(a);
  else u::k_conv<16><<<grid, u::kThreads, u::conv_smem_bytes<16>(), st>>>(a);
  NCK(cudaGetLastError());
  ++net->ctx->stats.kernel_launches;
  return MSGPU_OK;
}

// forward convolution of layer i: in -> out (bf16 view, or the float head output)
int net_fwd(msgpu_net* net, int i, const View& in, const View* out, int B, cudaStream_t st) {
  const NetLayer& l = net->L[i];
  msg::unet::ConvArgs a;
  memset(&a, 0, sizeof(a));
  a.in = in.p; a.in_img = in.img; a.in_n = in.n; a.in_cs = in.cs; a.cin = l.cin_pad;
  a.w = net->wf + l.wf_off;
  a.bias = net->theta + l.b_off;
  const int on = (in.n - 1) / l.stride + 1;
  if (out) {
    a.out = out->p; a.out_img = out->img; a.out_n = out->n; a.out_cs = out->cs;
  } else {
    a.out = net->out; a.out_img = (size_t)on * on * 2; a.out_n = on; a.out_cs = 2; a.out_f32 = 1;
  }
  a.cout = l.cout;
  a.mode = 0; a.stride = l.stride; a.relu = l.relu;
  a.total = B * on * on;
  return net_conv_launch(net, a, l.cout_pad, st);
}

// data gradient of layer i: dy (at its output) -> dx (at its input), times the
// ReLU mask of the input activation; accumulate adds dx's current value first
int net_bwd_data(msgpu_net* net, int i, const View& dy, const View& dx, const View& mask, int accumulate, int B,
                 cudaStream_t st) {
  const NetLayer& l = net->L[i];
  msg::unet::ConvArgs a;
  memset(&a, 0, sizeof(a));
  a.in = dy.p; a.in_img = dy.img; a.in_n = dy.n; a.in_cs = dy.cs; a.cin = l.cout_pad;
  a.w = net->wt + l.wt_off;
  a.out = dx.p; a.out_img = dx.img; a.out_n = dx.n; a.out_cs = dx.cs; a.cout = l.cin;
  a.mode = 1; a.stride = l.stride; a.accumulate = accumulate;
  a.mask = mask.p; a.mask_img = mask.img; a.mask_cs = mask.cs;
  a.total = B * dx.n * dx.n;
  return net_conv_launch(net, a, l.cin_pad, st);
}

// weight and bias gradients of layer i from its input activation and the gradient at its output
int net_bwd_weights(msgpu_net* net, int i, const View& in, const View& dy, int B, cudaStream_t st) {
  const NetLayer& l = net->L[i];
  const int K = 9 * l.cin_pad;
  const int bm = tile_of(l.cout_pad);
  const int xt = (K + 63) / 64, yt = l.cout_pad / bm;
  const int total = B * dy.n * dy.n;
  int chunks = std::max(1, (4 * net->ctx->sm_count + xt * yt - 1) / (xt * yt));
  chunks = std::min(chunks, std::max(1, total / 256));
  const int chunk = ((total + chunks - 1) / chunks + msg::unet::kBK - 1) / msg::unet::kBK * msg::unet::kBK;
  chunks = (total + chunk - 1) / chunk;
  const size_t need = (size_t)chunks * l.cout_pad * (K + 1);
  int rc;
  if ((rc = ensure(net->ctx, net->part, need * sizeof(float)))) return rc;
  float* part = (float*)net->part.p;
  float* bpart = part + (size_t)chunks * l.cout_pad * K;
  msg::unet::WgradArgs a;
  a.in = in.p; a.in_img = in.img; a.in_n = in.n; a.in_cs = in.cs; a.cin = l.cin_pad;
  a.dy = dy.p; a.dy_img = dy.img; a.dy_n = dy.n; a.dy_cs = dy.cs; a.cout_pad = l.cout_pad;
  a.stride = l.stride; a.part = part; a.bpart = bpart; a.total = total; a.chunk = chunk;
  const dim3 grid((unsigned)xt, (unsigned)yt, (unsigned)chunks);
  if (bm == 64) msg::unet::k_wgrad<64><<<grid, msg::unet::kThreads, 0, st>>>(a);
  else if (bm == 32) msg::unet::k_wgrad<32><<<grid, msg::unet::kThreads, 0, st>>>(a);
  else msg::unet::k_wgrad<16><<<grid, msg::unet::kThreads, 0, st>>>(a);
  const int nw = l.cout * 9 * l.cin;
  msg::unet::k_wgrad_reduce<<<std::min(1024, (nw + 255) / 256), 256, 0, st>>>(part, chunks, l.cout, l.cout_pad, l.cin,
                                                                              l.cin_pad, net->grad + l.w_off);
  msg::unet::k_bgrad_reduce<<<1, 128, 0, st>>>(bpart, chunks, l.cout, l.cout_pad, net->grad + l.b_off);
  NCK(cudaGetLastError());
  net->ctx->stats.kernel_launches += 3;
  return MSGPU_OK;
}

int net_up(msgpu_net* net, const View& src, const View& dst, int C, int B, cudaStream_t st) {
  const size_t total = (size_t)B * dst.n * dst.n * (C / 8);
  msg::unet::k_up<<<(unsigned)std::min<size_t>(4096, (total + 255) / 256), 256, 0, st>>>(
      src.p, src.img, src.n, src.cs, dst.p, dst.img, dst.cs, C, B);
  NCK(cudaGetLastError());
  ++net->ctx->stats.kernel_launches;
  return MSGPU_OK;
}

int net_up_back(msgpu_net* net, const View& df, const View& dc, const View& mask, int C, int B, cudaStream_t st) {
  const size_t total = (size_t)B * dc.n * dc.n * (C / 8);
  msg::unet::k_up_back<<<(unsigned)std::min<size_t>(4096, (total + 255) / 256), 256, 0, st>>>(
      df.p, df.img, df.n, df.cs, dc.p, dc.img, dc.cs, mask.p, mask.img, mask.cs, C, B);
  NCK(cudaGetLastError());
  ++net->ctx->stats.kernel_launches;
  return MSGPU_OK;
}

// Forward pass on the packed input x0 of B images; output in net->out.
int net_forward(msgpu_net* net, int B, cudaStream_t st) {
  int rc;
  msgpu_net& n = *net;
  if ((rc = net_fwd(net, E0A, n.x0, &n.a0, B, st)) || (rc = net_fwd(net, E0B, n.a0, &n.a1, B, st)) ||
      (rc = net_fwd(net, E1A, n.a1, &n.b0, B, st))) return rc;
  const View s1 = n.cat1.ch(0), up1 = n.cat1.ch(32), s2 = n.cat2.ch(0), up2 = n.cat2.ch(64);
  if ((rc = net_fwd(net, E1B, n.b0, &s1, B, st)) || (rc = net_fwd(net, E2A, s1, &n.c0, B, st)) ||
      (rc = net_fwd(net, E2B, n.c0, &s2, B, st)) || (rc = net_fwd(net, E3A, s2, &n.d0, B, st)) ||
      (rc = net_fwd(net, E3B, n.d0, &n.d1, B, st)) || (rc = net_up(net, n.d1, up2, 128, B, st)) ||
      (rc = net_fwd(net, D2A, n.cat2, &n.g0, B, st)) || (rc = net_fwd(net, D2B, n.g0, &n.g1, B, st)) ||
      (rc = net_up(net, n.g1, up1, 64, B, st)) || (rc = net_fwd(net, D1A, n.cat1, &n.h0, B, st)) ||
      (rc = net_fwd(net, D1B, n.h0, &n.h1, B, st)) || (rc = net_fwd(net, HEAD, n.h1, nullptr, B, st)))
    return rc;
  return MSGPU_OK;
}

// Backward pass from net->dout: every parameter gradient into net->grad.
int net_backward(msgpu_net* net, int B, cudaStream_t st) {
  int rc;
  msgpu_net& n = *net;
  const View none{nullptr, 0, 0, 0};
  const View s1 = n.cat1.ch(0), s2 = n.cat2.ch(0);
  const View ds1 = n.dcat1.ch(0), dup1 = n.dcat1.ch(32), ds2 = n.dcat2.ch(0), dup2 = n.dcat2.ch(64);
  if ((rc = net_bwd_weights(net, HEAD, n.h1, n.dout, B, st)) ||
      (rc = net_bwd_data(net, HEAD, n.dout, n.dh1, n.h1, 0, B, st)) ||
      (rc = net_bwd_weights(net, D1B, n.h0, n.dh1, B, st)) ||
      (rc = net_bwd_data(net, D1B, n.dh1, n.dh0, n.h0, 0, B, st)) ||
      (rc = net_bwd_weights(net, D1A, n.cat1, n.dh0, B, st)) ||
      (rc = net_bwd_data(net, D1A, n.dh0, n.dcat1, none, 0, B, st)) ||
      (rc = net_up_back(net, dup1, n.dg1, n.g1, 64, B, st)) ||
      (rc = net_bwd_weights(net, D2B, n.g0, n.dg1, B, st)) ||
      (rc = net_bwd_data(net, D2B, n.dg1, n.dg0, n.g0, 0, B, st)) ||
      (rc = net_bwd_weights(net, D2A, n.cat2, n.dg0, B, st)) ||
      (rc = net_bwd_data(net, D2A, n.dg0, n.dcat2, none, 0, B, st)) ||
      (rc = net_up_back(net, dup2, n.dd1, n.d1, 128, B, st)) ||
      (rc = net_bwd_weights(net, E3B, n.d0, n.dd1, B, st)) ||
      (rc = net_bwd_data(net, E3B, n.dd1, n.dd0, n.d0, 0, B, st)) ||
      (rc = net_bwd_weights(net, E3A, s2, n.dd0, B, st)) ||
      (rc = net_bwd_data(net, E3A, n.dd0, ds2, s2, 1, B, st)) ||
      (rc = net_bwd_weights(net, E2B, n.c0, ds2, B, st)) ||
      (rc = net_bwd_data(net, E2B, ds2, n.dc0, n.c0, 0, B, st)) ||
      (rc = net_bwd_weights(net, E2A, s1, n.dc0, B, st)) ||
      (rc = net_bwd_data(net, E2A, n.dc0, ds1, s1, 1, B, st)) ||
      (rc = net_bwd_weights(net, E1B, n.b0, ds1, B, st)) ||
      (rc = net_bwd_data(net, E1B, ds1, n.db0, n.b0, 0, B, st)) ||
      (rc = net_bwd_weights(net, E1A, n.a1, n.db0, B, st)) ||
      (rc = net_bwd_data(net, E1A, n.db0, n.da1, n.a1, 0, B, st)) ||
      (rc = net_bwd_weights(net, E0B, n.a0, n.da1, B, st)) ||
      (rc = net_bwd_data(net, E0B, n.da1, n.da0, n.a0, 0, B, st)) ||
      (rc = net_bwd_weights(net, E0A, n.x0, n.da0, B, st)))
    return rc;
  return MSGPU_OK;
}

int net_input(msgpu_net* net, const double* R, size_t r_stride, const double* T, size_t t_stride, int B,
              cudaStream_t st) {
  int rc;
  // the kernels index nodes of the whole batch with 32-bit integers
  if ((double)B * net->n[0] * net->n[0] * 16.0 > 2147483647.0)
    return fail(net->ctx, MSGPU_ERR_SIZE, "a batch of %d images of %d^2 nodes is too large for one network pass", B,
                net->n[0]);
  if ((rc = net_buffers(net, B, st))) return rc;
  const size_t total = (size_t)B * net->n[0] * net->n[0];
  msg::unet::k_pack_input<<<(unsigned)std::min<size_t>(4096, (total + 255) / 256), 256, 0, st>>>(
      R, r_stride, T, t_stride, net->n[0] * net->n[0], B, net->x0.p);
  NCK(cudaGetLastError());
  ++net->ctx->stats.kernel_launches;
  return MSGPU_OK;
}

// Loss of the head output against target displacements (B x 2 x N1, domain
// units) into net->small (float at offset 0), its gradient into dout.
int net_loss(msgpu_net* net, const double* target, int B, cudaStream_t st) {
  int rc;
  if ((rc = ensure(net->ctx, net->small, sizeof(float) * 1024))) return rc;
  float* s = (float*)net->small.p;
  const int N1 = net->n[1] * net->n[1];
  const int blocks = std::min(512, (B * N1 + 255) / 256);
  msg::unet::k_mse<<<blocks, 256, 0, st>>>(net->out, target, (double)(net->n[1] - 1), N1, B, net->dout.p, s + 8);
  msg::unet::k_loss_total<<<1, 32, 0, st>>>(s + 8, blocks, s);
  NCK(cudaGetLastError());
  net->ctx->stats.kernel_launches += 2;
  return MSGPU_OK;
}

int net_adam(msgpu_net* net, float lr, cudaStream_t st) {
  net->step++;
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.f - powf(b1, (float)net->step), c2 = 1.f - powf(b2, (float)net->step);
  const int n = (int)net->nparams;
  msg::unet::k_adam<<<std::min(2048, (n + 255) / 256), 256, 0, st>>>(net->theta, net->grad, net->m, net->v, n, lr, b1,
                                                                    b2, 1e-8f, c1, c2);
  NCK(cudaGetLastError());
  ++net->ctx->stats.kernel_launches;
  return net_pack(net, st);
}

// Prediction into the net's phi buffer (B x 2 x N1 doubles, domain units).
int net_predict(msgpu_net* net, const double* R, size_t r_stride, const double* T, size_t t_stride, int B,
                cudaStream_t st, double** phi_out) {
  int rc;
  if ((rc = net_input(net, R, r_stride, T, t_stride, B, st)) || (rc = net_forward(net, B, st))) return rc;
  const int N1 = net->n[1] * net->n[1];
  if ((rc = ensure(net->ctx, net->phi, sizeof(double) * 2 * (size_t)N1 * B))) return rc;
  double* phi = (double*)net->phi.p;
  msg::unet::k_out_to_phi<<<(unsigned)std::min(4096, (B * N1 + 255) / 256), 256, 0, st>>>(
      net->out, 1.0 / (double)(net->n[1] - 1), N1, B, phi);
  NCK(cudaGetLastError());
  ++net->ctx->stats.kernel_launches;
  *phi_out = phi;
  return MSGPU_OK;
}

// He-normal initialisation (deterministic for a seed), biases zero, the head scaled by 0.1.
void net_init_host(const msgpu_net* net, unsigned long long seed, std::vector<float>& th) {
  th.assign(net->nparams, 0.f);
  unsigned long long s = seed * 0x9E3779B97F4A7C15ull + 1;
  auto next = [&]() {   // splitmix64
    unsigned long long z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  };
  auto unif = [&]() { return ((next() >> 11) + 0.5) * (1.0 / 9007199254740992.0); };
  for (int i = 0; i < kNetLayers; ++i) {
    const NetLayer& l = net->L[i];
    const double sd = std::sqrt(2.0 / (9.0 * l.cin)) * (i == HEAD ? 0.1 : 1.0);
    const size_t nw = (size_t)l.cout * 9 * l.cin;
    for (size_t k = 0; k < nw; ++k) {   // Box-Muller
      const double u1 = unif(), u2 = unif();
      th[l.w_off + k] = (float)(sd * std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2));
    }
  }
}

int net_set_params_dev(msgpu_net* net, const float* host) {
  const cudaStream_t st = net->ctx->stream;
  NCK(cudaMemcpyAsync(net->theta, host, sizeof(float) * net->nparams, cudaMemcpyHostToDevice, st));
  NCK(cudaMemsetAsync(net->m, 0, sizeof(float) * net->nparams, st));
  NCK(cudaMemsetAsync(net->v, 0, sizeof(float) * net->nparams, st));
  net->step = 0;
  int rc;
  if ((rc = net_pack(net, net->ctx->stream))) return rc;
  NCK(cudaStreamSynchronize(net->ctx->stream));
  return MSGPU_OK;
}

// The network's start displacement for F templates from their prepared
// pyramids (reference row 0, templates rows 1..F): F x 2 x N doubles at the
// network's output level, in the net's phi buffer.
int warm_start_phi(msgpu_net* net, const double* pyr, const std::vector<size_t>& poff, size_t pstride, int F,
                   cudaStream_t st, double** phi) {
  const int l0 = net->level;
  const size_t N1 = (size_t)net->n[1] * net->n[1];
  int rc;
  if ((rc = ensure(net->ctx, net->phiall, sizeof(double) * 2 * N1 * F))) return rc;
  double* all = (double*)net->phiall.p;
  // at most 64 frames per network pass (activation memory and 32-bit node indices)
  for (int f0 = 0; f0 < F; f0 += 64) {
    const int m = std::min(64, F - f0);
    double* part;
    if ((rc = net_predict(net, pyr + poff[l0], 0, pyr + (size_t)(1 + f0) * pstride + poff[l0], pstride, m, st, &part)))
      return rc;
    NCK(cudaMemcpyAsync(all + 2 * N1 * f0, part, sizeof(double) * 2 * N1 * m, cudaMemcpyDeviceToDevice, st));
  }
  *phi = all;
  return MSGPU_OK;
}

// msgpu_register_batch_warm_device; warm_used (host, nullable).
template <typename Real>
int warm_batch(msgpu_context* ctx, const msgpu_params& p, msgpu_net* net, const double* d_ref, const double* d_tmpl,
               int F, const double* d_plain_e, double rel_tol, double* d_phis, double* d_e_out, int* d_s_out,
               int* warm_used, cudaStream_t st) {
  const int ws = net->level - 1;
  msgpu_params pw = p;
  pw.start_level = ws;
  const int nlev = p.stop_level - p.start_level + 1, nw = p.stop_level - ws + 1;
  const size_t NM = lvl_N(p.precision_level), Nin = lvl_N(p.input_level);
  int rc;
  if ((rc = ensure(ctx, ctx->io[5], sizeof(double) * F + sizeof(int) * (size_t)F * nw + 64))) return rc;
  double* e = (double*)ctx->io[5].p;
  int* s = (int*)(e + F);
  BatchIO io{d_ref, d_tmpl, nullptr, d_phis, e, s};
  BatchOpts opt;
  opt.warm = net;
  // to the stated energy tolerance: with the plain method's energies the
  // warm-started solve of the stop level ends as soon as it is within rel_tol
  // of them
  opt.e_target = d_plain_e;
  opt.e_tol = rel_tol;
  // a warm-started frame may need more steps than the plain schedule to
  // reach its target: the stop level runs until it does, at most twice
  // maxGDIterations steps (a frame that does not is registered again)
  opt.max_iter_stop = d_plain_e ? 2 * p.max_gd_iterations : 0;
  // the levels between the network's output and the stop level start near
  // their solution: optionally fewer steps there (msgpu_set_warm_schedule)
  opt.max_iter_below = ctx->warm_coarse_iters;
  if ((rc = run_batch<Real>(ctx, pw, F, io, st, opt))) return rc;
  if (d_e_out) CK(cudaMemcpyAsync(d_e_out, e, sizeof(double) * F, cudaMemcpyDeviceToDevice, st));
  if (d_s_out) {
    CK(cudaMemsetAsync(d_s_out, 0, sizeof(int) * (size_t)F * nlev, st));
    CK(cudaMemcpy2DAsync(d_s_out + (ws - p.start_level), sizeof(int) * nlev, s, sizeof(int) * nw, sizeof(int) * nw, F,
                         cudaMemcpyDeviceToDevice, st));
  }
  std::vector<int> used(F, 1);
  if (d_plain_e) {
    // the plain method's energies judge the warm start: worse by more than
    // rel_tol -> the frame is registered again from the plain start
    std::vector<double> he(F), hp(F);
    CK(cudaMemcpyAsync(he.data(), e, sizeof(double) * F, cudaMemcpyDeviceToHost, st));
    CK(cudaMemcpyAsync(hp.data(), d_plain_e, sizeof(double) * F, cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    std::vector<int> bad;
    for (int f = 0; f < F; ++f)
      if (!(he[f] <= hp[f] + rel_tol * std::fabs(hp[f]))) {
        bad.push_back(f);
        used[f] = 0;
      }
    const int G = (int)bad.size();
    if (G) {
      const size_t need = sizeof(double) * ((size_t)G * (Nin + 2 * NM) + G) + sizeof(int) * (size_t)G * nlev + 64;
      if ((rc = ensure(ctx, net->gather, need))) return rc;
      double* tm = (double*)net->gather.p;
      double* ph = tm + (size_t)G * Nin;
      double* e2 = ph + 2 * NM * G;
      int* s2 = (int*)(e2 + G);
      for (int g = 0; g < G; ++g)
        CK(cudaMemcpyAsync(tm + g * Nin, d_tmpl + (size_t)bad[g] * Nin, sizeof(double) * Nin,
                           cudaMemcpyDeviceToDevice, st));
      BatchIO io2{d_ref, tm, nullptr, ph, e2, s2};
      if ((rc = run_batch<Real>(ctx, p, G, io2, st))) return rc;
      for (int g = 0; g < G; ++g) {
        const int f = bad[g];
        CK(cudaMemcpyAsync(d_phis + 2 * NM * f, ph + 2 * NM * g, sizeof(double) * 2 * NM, cudaMemcpyDeviceToDevice,
                           st));
        if (d_e_out) CK(cudaMemcpyAsync(d_e_out + f, e2 + g, sizeof(double), cudaMemcpyDeviceToDevice, st));
        if (d_s_out)
          CK(cudaMemcpyAsync(d_s_out + (size_t)f * nlev, s2 + (size_t)g * nlev, sizeof(int) * nlev,
                             cudaMemcpyDeviceToDevice, st));
      }
    }
  }
  if (warm_used) std::copy(used.begin(), used.end(), warm_used);
  return MSGPU_OK;
}

int check_warm(msgpu_context* ctx, const msgpu_params* p, msgpu_net* net) {
  int rc;
  if ((rc = check_params(ctx, p))) return rc;
  if (!net || net->ctx != ctx) return fail(ctx, MSGPU_ERR_INVALID_ARG, "the network belongs to another context");
  const int ws = net->level - 1;
  if (net->level > p->input_level || ws < p->start_level || ws > p->stop_level)
    return fail(ctx, MSGPU_ERR_INVALID_ARG,
                "network input level %d: needs inputLevel >= %d and startLevel <= %d <= stopLevel", net->level,
                net->level, ws);
  return MSGPU_OK;
}
}  // namespace

extern "C" {

long long msgpu_net_num_params(void) { return (long long)net_param_count(); }

int msgpu_net_create(msgpu_context* ctx, int input_level, unsigned long long seed, msgpu_net** out) {
  if (!ctx || !out) return MSGPU_ERR_INVALID_ARG;
  *out = nullptr;
  if (input_level < 4 || input_level > 11)
    return fail(ctx, MSGPU_ERR_INVALID_ARG, "network input level %d: 4..11 (three stride-2 levels below it)",
                input_level);
  int rc;
  if ((rc = bind_device(ctx))) return rc;
  if ((rc = net_kernel_attrs(ctx))) return rc;
  msgpu_net* net = new msgpu_net();
  net->ctx = ctx;
  net->level = input_level;
  for (int g = 0; g < 4; ++g) net->n[g] = (1 << (input_level - g)) + 1;
  size_t off = 0, pk = 0;
  for (int i = 0; i < kNetLayers; ++i) {
    NetLayer& l = net->L[i];
    l.cin = kNetSpec[i][0]; l.cout = kNetSpec[i][1]; l.stride = kNetSpec[i][2]; l.relu = kNetSpec[i][3];
    l.cin_pad = pad16(l.cin); l.cout_pad = pad16(l.cout);
    l.w_off = off; off += (size_t)l.cout * 9 * l.cin;
    l.b_off = off; off += l.cout;
    l.wf_off = pk; l.wt_off = pk; pk += align_up((size_t)l.cout_pad * 9 * l.cin_pad, 64);
  }
  net->nparams = off;
  net->npacked = pk;
  cudaError_t e = cudaMalloc(&net->theta, sizeof(float) * 4 * off);
  if (e == cudaSuccess) e = cudaMalloc(&net->wf, sizeof(bf16) * 2 * pk);
  if (e != cudaSuccess) {
    cudaFree(net->theta);
    delete net;
    return fail(ctx, MSGPU_ERR_CUDA, "network allocation failed: %s", cudaGetErrorString(e));
  }
  net->grad = net->theta + off; net->m = net->grad + off; net->v = net->m + off;
  net->wt = net->wf + pk;
  std::vector<float> th;
  net_init_host(net, seed, th);
  if ((rc = net_set_params_dev(net, th.data()))) {
    cudaFree(net->theta); cudaFree(net->wf);
    delete net;
    return rc;
  }
  *out = net;
  return MSGPU_OK;
}

int msgpu_net_destroy(msgpu_net* net) {
  if (!net) return MSGPU_OK;
  cudaSetDevice(net->ctx->device);
  cudaFree(net->theta);
  cudaFree(net->wf);
  for (msgpu_context::Buf* b : {&net->act, &net->part, &net->small, &net->phi, &net->gather, &net->phiall})
    if (b->p) cudaFree(b->p);
  delete net;
  return MSGPU_OK;
}

int msgpu_net_input_level(const msgpu_net* net) { return net ? net->level : -1; }

int msgpu_net_set_tensor_cores(msgpu_net* net, int tcgen05) {
  if (!net) return MSGPU_ERR_INVALID_ARG;
  net->tcgen05 = tcgen05 != 0;
  return MSGPU_OK;
}

int msgpu_net_get_params(msgpu_net* net, float* out) {
  if (!net || !out) return MSGPU_ERR_INVALID_ARG;
  int rc;
  if ((rc = bind_device(net->ctx))) return rc;
  NCK(cudaDeviceSynchronize());   // training steps may have run on any stream
  NCK(cudaMemcpy(out, net->theta, sizeof(float) * net->nparams, cudaMemcpyDeviceToHost));
  return MSGPU_OK;
}

int msgpu_net_set_params(msgpu_net* net, const float* in) {
  if (!net || !in) return MSGPU_ERR_INVALID_ARG;
  int rc;
  if ((rc = bind_device(net->ctx))) return rc;
  return net_set_params_dev(net, in);
}

int msgpu_net_save(msgpu_net* net, const char* path) {
  if (!net || !path) return MSGPU_ERR_INVALID_ARG;
  std::vector<float> th(net->nparams);
  int rc;
  if ((rc = msgpu_net_get_params(net, th.data()))) return rc;
  FILE* f = fopen(path, "wb");
  if (!f) return fail(net->ctx, MSGPU_ERR_INVALID_ARG, "Could not open %s for writing", path);
  const char magic[8] = {'M', 'S', 'G', 'P', 'U', 'N', 'E', 'T'};
  const int hdr[2] = {1, (int)net->nparams};
  bool ok = fwrite(magic, 1, 8, f) == 8 && fwrite(hdr, sizeof(int), 2, f) == 2 &&
            fwrite(th.data(), sizeof(float), th.size(), f) == th.size();
  ok = (fclose(f) == 0) && ok;
  return ok ? MSGPU_OK : fail(net->ctx, MSGPU_ERR_INVALID_ARG, "writing %s failed", path);
}

int msgpu_net_load(msgpu_net* net, const char* path) {
  if (!net || !path) return MSGPU_ERR_INVALID_ARG;
  FILE* f = fopen(path, "rb");
  if (!f) return fail(net->ctx, MSGPU_ERR_INVALID_ARG, "Could not open %s", path);
  char magic[8];
  int hdr[2] = {0, 0};
  std::vector<float> th(net->nparams);
  const bool ok = fread(magic, 1, 8, f) == 8 && !memcmp(magic, "MSGPUNET", 8) && fread(hdr, sizeof(int), 2, f) == 2 &&
                  hdr[0] == 1 && hdr[1] == (int)net->nparams &&
                  fread(th.data(), sizeof(float), th.size(), f) == th.size();
  fclose(f);
  if (!ok) return fail(net->ctx, MSGPU_ERR_SIZE, "%s is not a network file of %zu parameters", path, net->nparams);
  return msgpu_net_set_params(net, th.data());
}

int msgpu_net_predict_device(msgpu_net* net, const double* d_R, long long r_stride, const double* d_T, int batch,
                             double* d_phi_out, void* stream) {
  if (!net || !d_R || !d_T || !d_phi_out || batch < 1 || r_stride < 0) return MSGPU_ERR_INVALID_ARG;
  int rc;
  if ((rc = bind_device(net->ctx))) return rc;
  net->ctx->stats.kernel_launches = 0;
  const cudaStream_t st = (cudaStream_t)stream;
  const size_t N0 = (size_t)net->n[0] * net->n[0], N1 = (size_t)net->n[1] * net->n[1];
  double* phi;
  if ((rc = net_predict(net, d_R, (size_t)r_stride, d_T, N0, batch, st, &phi))) return rc;
  NCK(cudaMemcpyAsync(d_phi_out, phi, sizeof(double) * 2 * N1 * batch, cudaMemcpyDeviceToDevice, st));
  return MSGPU_OK;
}

int msgpu_net_train_step_device(msgpu_net* net, const double* d_R, long long r_stride, const double* d_T,
                                const double* d_phi_target, int batch, float lr, float* loss_out, void* stream) {
  if (!net || !d_R || !d_T || !d_phi_target || batch < 1 || r_stride < 0 || !(lr >= 0))
    return MSGPU_ERR_INVALID_ARG;
  int rc;
  if ((rc = bind_device(net->ctx))) return rc;
  net->ctx->stats.kernel_launches = 0;
  const cudaStream_t st = (cudaStream_t)stream;
  const size_t N0 = (size_t)net->n[0] * net->n[0];
  if ((rc = net_input(net, d_R, (size_t)r_stride, d_T, N0, batch, st)) || (rc = net_forward(net, batch, st)) ||
      (rc = net_loss(net, d_phi_target, batch, st)) || (rc = net_backward(net, batch, st)) ||
      (rc = net_adam(net, lr, st)))
    return rc;
  if (loss_out) {
    NCK(cudaMemcpyAsync(loss_out, net->small.p, sizeof(float), cudaMemcpyDeviceToHost, st));
    NCK(cudaStreamSynchronize(st));
  }
  return MSGPU_OK;
}

int msgpu_net_loss_grad(msgpu_net* net, const double* R, const double* T, const double* phi_target, int batch,
                        float* loss_out, double* phi_out, float* grad_out) {
  if (!net || !R || !T || !phi_target || batch < 1) return MSGPU_ERR_INVALID_ARG;
  int rc;
  if ((rc = bind_device(net->ctx))) return rc;
  msgpu_context* ctx = net->ctx;
  const cudaStream_t st = ctx->stream;
  const size_t N0 = (size_t)net->n[0] * net->n[0], N1 = (size_t)net->n[1] * net->n[1];
  if ((rc = sched_error_reset(ctx, st))) return rc;
  if ((rc = ensure(ctx, ctx->io[0], sizeof(double) * (2 * N0 + 2 * N1) * batch))) return rc;
  double* d = (double*)ctx->io[0].p;
  CK(cudaMemcpyAsync(d, R, sizeof(double) * N0 * batch, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(d + N0 * batch, T, sizeof(double) * N0 * batch, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(d + 2 * N0 * batch, phi_target, sizeof(double) * 2 * N1 * batch, cudaMemcpyHostToDevice, st));
  double* phi;
  if ((rc = net_predict(net, d, N0, d + N0 * batch, N0, batch, st, &phi)) ||
      (rc = net_loss(net, d + 2 * N0 * batch, batch, st)) || (rc = net_backward(net, batch, st)))
    return rc;
  if (loss_out) CK(cudaMemcpyAsync(loss_out, net->small.p, sizeof(float), cudaMemcpyDeviceToHost, st));
  if (phi_out) CK(cudaMemcpyAsync(phi_out, phi, sizeof(double) * 2 * N1 * batch, cudaMemcpyDeviceToHost, st));
  if (grad_out) CK(cudaMemcpyAsync(grad_out, net->grad, sizeof(float) * net->nparams, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  return sched_error_check(ctx);
}

int msgpu_prepare_images_device(msgpu_context* ctx, const msgpu_params* p, const double* d_images, int count,
                                int level, double* d_out, void* stream) {
  if (!ctx) return MSGPU_ERR_INVALID_ARG;
  if (!p || !d_images || !d_out || count < 1) return fail(ctx, MSGPU_ERR_INVALID_ARG, "invalid prepare arguments");
  if (p->input_level < 1 || p->input_level > 12 || level < 0 || level > p->input_level)
    return fail(ctx, MSGPU_ERR_INVALID_ARG, "level %d outside 0..input_level %d", level, p->input_level);
  int rc;
  if ((rc = bind_device(ctx))) return rc;
  ctx->stats.kernel_launches = 0;
  const cudaStream_t st = (cudaStream_t)stream;
  std::vector<size_t> poff;
  const size_t pstride = pyramid_layout(p->input_level, poff);
  const size_t Nin = lvl_N(p->input_level), Nl = lvl_N(level);
  if ((rc = ensure(ctx, ctx->dscratch, sizeof(double) * pstride * count)) ||
      (rc = ensure(ctx, ctx->small, sizeof(double) * (2 * (size_t)count + 64))))
    return rc;
  double* pyr = (double*)ctx->dscratch.p;
  CK(cudaMemcpy2DAsync(pyr + poff[p->input_level], pstride * sizeof(double), d_images, Nin * sizeof(double),
                       Nin * sizeof(double), count, cudaMemcpyDeviceToDevice, st));
  if ((rc = prepare_pyramid(ctx, *p, pyr, poff, pstride, count, (double*)ctx->small.p, st))) return rc;
  CK(cudaMemcpy2DAsync(d_out, Nl * sizeof(double), pyr + poff[level], pstride * sizeof(double), Nl * sizeof(double),
                       count, cudaMemcpyDeviceToDevice, st));
  return MSGPU_OK;
}

int msgpu_register_batch_warm_device(msgpu_context* ctx, const msgpu_params* p, msgpu_net* net,
                                     const double* d_reference, const double* d_templates, int num_templates,
                                     const double* d_plain_energies, double rel_tol, double* d_phis_out,
                                     double* d_energies_out, int* d_steps_out, int* warm_used_out, void* stream) {
  if (!ctx) return MSGPU_ERR_INVALID_ARG;
  int rc;
  if ((rc = check_warm(ctx, p, net))) return rc;
  if (num_templates < 1) return fail(ctx, MSGPU_ERR_INVALID_ARG, "num_templates must be >= 1");
  if (!d_reference || !d_templates || !d_phis_out) return fail(ctx, MSGPU_ERR_INVALID_ARG, "null buffer");
  if ((rc = bind_device(ctx))) return rc;
  const cudaStream_t st = (cudaStream_t)stream;
  return p->use_fp64 ? warm_batch<double>(ctx, *p, net, d_reference, d_templates, num_templates, d_plain_energies,
                                          rel_tol, d_phis_out, d_energies_out, d_steps_out, warm_used_out, st)
                     : warm_batch<float>(ctx, *p, net, d_reference, d_templates, num_templates, d_plain_energies,
                                         rel_tol, d_phis_out, d_energies_out, d_steps_out, warm_used_out, st);
}

int msgpu_register_batch_warm(msgpu_context* ctx, const msgpu_params* p, msgpu_net* net, const double* reference,
                              const double* templates, int num_templates, const double* plain_energies,
                              double rel_tol, double* phis_out, double* energies_out, int* steps_out,
                              int* warm_used_out) {
  if (!ctx) return MSGPU_ERR_INVALID_ARG;
  int rc;
  if ((rc = check_warm(ctx, p, net))) return rc;
  if (num_templates < 1) return fail(ctx, MSGPU_ERR_INVALID_ARG, "num_templates must be >= 1");
  if (!reference || !templates || !phis_out) return fail(ctx, MSGPU_ERR_INVALID_ARG, "null buffer");
  if ((rc = bind_device(ctx))) return rc;
  const size_t Nin = lvl_N(p->input_level), NM = lvl_N(p->precision_level);
  const int F = num_templates;
  const int nlev = p->stop_level - p->start_level + 1;
  if ((rc = ensure(ctx, ctx->io[0], sizeof(double) * Nin)) || (rc = ensure(ctx, ctx->io[1], sizeof(double) * Nin * F)) ||
      (rc = ensure(ctx, ctx->io[3], sizeof(double) * 2 * NM * F)) ||
      (rc = ensure(ctx, ctx->io[4], sizeof(double) * 2 * F + sizeof(int) * F * nlev + 64)))
    return rc;
  const cudaStream_t st = ctx->stream;
  double* d_e = (double*)ctx->io[4].p;
  double* d_pe = d_e + F;
  int* d_s = (int*)(d_pe + F);
  CK(cudaMemcpyAsync(ctx->io[0].p, reference, sizeof(double) * Nin, cudaMemcpyHostToDevice, st));
  CK(cudaMemcpyAsync(ctx->io[1].p, templates, sizeof(double) * Nin * F, cudaMemcpyHostToDevice, st));
  if (plain_energies) CK(cudaMemcpyAsync(d_pe, plain_energies, sizeof(double) * F, cudaMemcpyHostToDevice, st));
  rc = p->use_fp64 ? warm_batch<double>(ctx, *p, net, (const double*)ctx->io[0].p, (const double*)ctx->io[1].p, F,
                                        plain_energies ? d_pe : nullptr, rel_tol, (double*)ctx->io[3].p, d_e, d_s,
                                        warm_used_out, st)
                   : warm_batch<float>(ctx, *p, net, (const double*)ctx->io[0].p, (const double*)ctx->io[1].p, F,
                                       plain_energies ? d_pe : nullptr, rel_tol, (double*)ctx->io[3].p, d_e, d_s,
                                       warm_used_out, st);
  if (rc) return rc;
  CK(cudaMemcpyAsync(phis_out, ctx->io[3].p, sizeof(double) * 2 * NM * F, cudaMemcpyDeviceToHost, st));
  if (energies_out) CK(cudaMemcpyAsync(energies_out, d_e, sizeof(double) * F, cudaMemcpyDeviceToHost, st));
  if (steps_out) CK(cudaMemcpyAsync(steps_out, d_s, sizeof(int) * F * nlev, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  return sched_error_check(ctx);
}

}  // extern "C"
