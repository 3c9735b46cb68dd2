// msgpu_series.cuh -- device kernels of the series pipeline around the level
// solves: composition of displacements with harmonic extension
// (ConcatAndSmoothlyExtendDeformations, deformations.h:498-520 and
// SmoothlyExtendImage, deformations.h:364-410) and the median of warped frames
// (averageSeries, matchSeries.h:442; MultiVector::getMedianVecOverComponents,
// multiVector.cpp:99-117).
//
// The extension solves, per component, the stiffness system whose rows and
// columns of the nodes where x + d2(x) stays inside the domain ("defined"
// nodes) are replaced by the identity, with the reference's PCGInverse
// (solver.h:264-358: diagonal preconditioner |1/diag|, stop when g.g < 1e-16,
// at most 1000 steps).  Both components run in one cooperative persistent
// kernel with two grid barriers per step; every CTA reduces the per-CTA
// partial sums in the same fixed order, so all CTAs hold bit-identical step
// sizes.  The new search direction d = d*beta - h of a step is not stored
// before the next stiffness product: each tile recomputes it on its halo from
// the previous direction and h, which yields the same bits as its owner.
#pragma once

#include "msgpu_level.cuh"

namespace msg {

constexpr int kExtThreads = 256;
constexpr int kExtTX = 32, kExtTY = 8;                        // tile of nodes, one node per thread
constexpr int kExtWX = kExtTX + 2, kExtWY = kExtTY + 2;       // with its one-node halo
constexpr int kExtWin = kExtWX * kExtWY;
constexpr int kExtMaxIter = 1000;
constexpr double kExtEps = 1e-16;
constexpr unsigned long long kExtBarrierNs = 2000000000ull;   // default bound of one grid-barrier wait

// Scratch of one composition (doubles unless noted), N = nodes of the level.
struct ExtArgs {
  const double* d1;        // 2N: [x | y] displacement applied second
  const double* d2;        // 2N: displacement applied first
  double* x;               // 2N: initial guess in, composition out
  double* bc;              // 2N: composed values at defined nodes, 0 elsewhere
  unsigned char* defined;  // N
  double* g;               // 2N: residual A x - b
  double* hA;              // 2N: preconditioned residual g * dinv
  double* hB;              // 2N: A d
  double* dbuf;            // 2 x 2N: search directions of odd / even steps
  double* partials;        // gridDim.x x 4
  unsigned* bar;           // [count, generation], zero at launch
  int* error;              // set when a barrier wait gave up
  int* iters_out;          // 2: PCG steps per component
  int level;
  unsigned long long bar_ns;  // bound of one grid-barrier wait (global-timer nanoseconds)
};

// DeformImage with an extension image of NaN (deformations.h:225-253), then
// + d2 (ConcatDeformations, deformations.h:498-510); a node is defined when
// the composed value is not NaN.
__global__ void k_compose_prep(ExtArgs a) {
  const int n = (1 << a.level) + 1, N = n * n;
  const double h = 1.0 / (double)(n - 1);
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < N; j += gridDim.x * blockDim.x) {
    const int x = j % n, y = j / n;
    const double ds0 = x + a.d2[j] / h, ds1 = y + a.d2[N + j] / h;
    const bool in = !(ds0 < 0. || ds0 > (double)(n - 1) || ds1 < 0. || ds1 > (double)(n - 1));
    double r0 = in ? interp_d(a.d1, n, ds0, ds1) : NAN;
    double r1 = in ? interp_d(a.d1 + N, n, ds0, ds1) : NAN;
    r0 += a.d2[j];
    r1 += a.d2[N + j];
    const bool def = !isnan(r0);
    a.defined[j] = def ? 1 : 0;
    a.bc[j] = def ? r0 : 0.;
    a.bc[N + j] = def ? r1 : 0.;
  }
}

// Grid-wide barrier with a bounded wait: returns false (and sets *error) when
// the other CTAs did not arrive within limit_ns or another CTA gave up.
__device__ __forceinline__ bool ext_grid_sync(unsigned* bar, int* error, unsigned long long limit_ns) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned* vgen = bar + 1;
    const unsigned gen = *vgen;
    __threadfence();
    const unsigned arrived = atomicAdd(bar, 1u) + 1u;
    int good = 1;
    if (arrived == gridDim.x) {
      atomicExch(bar, 0u);
      __threadfence();
      atomicAdd(bar + 1, 1u);
    } else {
      const unsigned long long t0 = global_ns();
      while (*vgen == gen) {
        if (*(volatile int*)error || global_ns() - t0 > limit_ns) {
          atomicExch(error, 1);
          good = 0;
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
    ok = good && (*(volatile int*)error == 0);
  }
  __syncthreads();
  return ok != 0;
}

// Sum over the block in a fixed order; the result is valid in every thread.
__device__ __forceinline__ void ext_block_sum(double v[4], double (*wbuf)[4]) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    double t = v[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
    if (lane == 0) wbuf[wid][k] = t;
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    double t = 0.0;
    for (int w = 0; w < kExtThreads / 32; ++w) t += wbuf[w][k];
    v[k] = t;
  }
  __syncthreads();
}

// Sum of the per-CTA partials (cnt of the 4 slots) in a fixed order: lane l
// adds CTAs l, l+32, ... in turn, then every thread adds the 32 lane sums in
// order, so that every CTA obtains the same bits.
__device__ __forceinline__ void ext_grid_total(const double* partials, int cnt, double out[4], double (*wbuf)[4]) {
  if (threadIdx.x < 32) {
    double t[4] = {0.0, 0.0, 0.0, 0.0};
    for (int c = threadIdx.x; c < (int)gridDim.x; c += 32)
      for (int k = 0; k < cnt; ++k) t[k] += __ldcg(partials + (size_t)c * 4 + k);
    for (int k = 0; k < cnt; ++k) wbuf[threadIdx.x][k] = t[k];
  }
  __syncthreads();
  for (int k = 0; k < cnt; ++k) {
    double s = 0.0;
    for (int l = 0; l < 32; ++l) s += wbuf[l][k];
    out[k] = s;
  }
  __syncthreads();
}

// StiffOp ONTHEFLY row at node (x,y) (LocalAssemblyHelper::doMultiplyOnTheFly,
// FEOpInterface.h:136-157): elements in x-fastest order, within an element the
// columns j = 0..3, accumulated one product at a time.
__device__ __forceinline__ double stiff_onthefly_row(const double* __restrict__ u, int n, int x, int y) {
  double s = 0.0;
#pragma unroll
  for (int ey = y - 1; ey <= y; ++ey) {
    if (ey < 0 || ey >= n - 1) continue;
#pragma unroll
    for (int ex = x - 1; ex <= x; ++ex) {
      if (ex < 0 || ex >= n - 1) continue;
      const int i = (x - ex) + 2 * (y - ey);
#pragma unroll
      for (int j = 0; j < 4; ++j) s += c_fe.lst[i][j] * u[(ex + (j & 1)) + (size_t)(ey + (j >> 1)) * n];
    }
  }
  return s;
}

// Row of the masked stiffness matrix applied to u (stiff_row's order; the
// entries coupling to a defined node are 0, a defined node's row is the
// identity).  get(X, Y) and def(X, Y) read u and the mask.
template <typename Get, typename Def>
__device__ __forceinline__ double masked_row(int x, int y, int n, Get get, Def def) {
  if (def(x, y)) return get(x, y);
  const int cls = node_class(x, n) + 3 * node_class(y, n);
  double d = 0.0;
#pragma unroll
  for (int j = -1; j <= 1; ++j)
#pragma unroll
    for (int i = -1; i <= 1; ++i) {
      const int X = x + i, Y = y + j;
      if (X >= 0 && X < n && Y >= 0 && Y < n) d += (def(X, Y) ? 0.0 : c_fe.st[cls][j + 1][i + 1]) * get(X, Y);
    }
  return d;
}

__device__ __forceinline__ double ext_dinv(int x, int y, int n, bool def) {
  if (def) return 1.0;
  const double a = c_fe.st[node_class(x, n) + 3 * node_class(y, n)][1][1];
  return fabs(1.0 / a);
}

// PCGInverse::apply (solver.h:264-358) for both components at once.  Every
// phase visits the nodes in the same order (tile t on CTA t mod grid, one
// node per thread), so that sums of equal products come out equal.
__global__ void __launch_bounds__(kExtThreads) k_extend_pcg(ExtArgs a) {
  __shared__ double s_d[2][kExtWin];
  __shared__ unsigned char s_m[kExtWin];
  __shared__ double wbuf[32][4];
  const int n = (1 << a.level) + 1, N = n * n;
  const int tx = threadIdx.x % kExtTX, ty = threadIdx.x / kExtTX;
  const int ntx = (n + kExtTX - 1) / kExtTX, nty = (n + kExtTY - 1) / kExtTY, ntiles = ntx * nty;
  auto defined = [&](int X, int Y) { return a.defined[X + (size_t)Y * n] != 0; };

  // --- b, then g = A x - b, h = g * dinv, d = 0 - h; partials g.h and g.g
  double part[4] = {0.0, 0.0, 0.0, 0.0};
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int x = (t % ntx) * kExtTX + tx, y = (t / ntx) * kExtTY + ty;
    if (x >= n || y >= n) continue;
    const size_t j = x + (size_t)y * n;
    const bool def = a.defined[j] != 0;
    const double di = ext_dinv(x, y, n, def);
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      const double* bc = a.bc + (size_t)c * N;
      const double* xc = a.x + (size_t)c * N;
      double b = stiff_onthefly_row(bc, n, x, y);
      b *= -1.;
      if (def) b = bc[j];
      const double hx = masked_row(x, y, n, [&](int X, int Y) { return xc[X + (size_t)Y * n]; }, defined);
      double g = hx;
      g -= b;
      const double h = g * di;
      double d = 0.0;
      d -= h;
      a.g[(size_t)c * N + j] = g;
      a.hA[(size_t)c * N + j] = h;
      a.dbuf[(size_t)2 * N + (size_t)c * N + j] = d;  // direction of step 1 (odd slot)
      part[c] += g * h;
      part[2 + c] += g * g;
    }
  }
  ext_block_sum(part, wbuf);
  if (threadIdx.x == 0)
    for (int k = 0; k < 4; ++k) __stcg(a.partials + (size_t)blockIdx.x * 4 + k, part[k]);
  if (!ext_grid_sync(a.bar, a.error, a.bar_ns)) return;
  double tot[4];
  ext_grid_total(a.partials, 4, tot, wbuf);
  double an[2] = {tot[0], tot[1]}, spn[2] = {tot[2], tot[3]}, q[2] = {0.0, 0.0};
  int it[2] = {0, 0};
  bool act[2];
  for (int c = 0; c < 2; ++c) act[c] = !(spn[c] < kExtEps) && it[c] < kExtMaxIter && !isnan(spn[c]);

  for (int k = 1; act[0] || act[1]; ++k) {
    for (int c = 0; c < 2; ++c)
      if (act[c]) ++it[c];
    double* dk = a.dbuf + (size_t)(k & 1) * 2 * N;             // direction of this step
    const double* dp = a.dbuf + (size_t)((k - 1) & 1) * 2 * N;  // of the previous step
    // --- phase A: d = d * beta - h (from step 2 on), h = A d; partial d.h
    double pa[4] = {0.0, 0.0, 0.0, 0.0};
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
      const int x0 = (t % ntx) * kExtTX, y0 = (t / ntx) * kExtTY;
      for (int w = threadIdx.x; w < kExtWin; w += kExtThreads) {
        const int X = x0 - 1 + w % kExtWX, Y = y0 - 1 + w / kExtWX;
        const bool in = X >= 0 && X < n && Y >= 0 && Y < n;
        const size_t gi = in ? X + (size_t)Y * n : 0;
        s_m[w] = in ? a.defined[gi] : 1;
#pragma unroll
        for (int c = 0; c < 2; ++c) {
          double v = 0.0;
          if (in && act[c]) {
            if (k == 1) {
              v = __ldcg(dk + (size_t)c * N + gi);
            } else {
              v = __ldcg(dp + (size_t)c * N + gi);
              v *= q[c];
              v -= __ldcg(a.hA + (size_t)c * N + gi);
            }
          }
          s_d[c][w] = v;
        }
      }
      __syncthreads();
      const int x = x0 + tx, y = y0 + ty;
      if (x < n && y < n) {
        const size_t gi = x + (size_t)y * n;
        auto def = [&](int X, int Y) { return s_m[(X - x0 + 1) + (Y - y0 + 1) * kExtWX] != 0; };
#pragma unroll
        for (int c = 0; c < 2; ++c) {
          if (!act[c]) continue;
          const double* sd = s_d[c];
          const double dv = sd[(tx + 1) + (ty + 1) * kExtWX];
          const double hv =
              masked_row(x, y, n, [&](int X, int Y) { return sd[(X - x0 + 1) + (Y - y0 + 1) * kExtWX]; }, def);
          if (k > 1) __stcg(dk + (size_t)c * N + gi, dv);
          __stcg(a.hB + (size_t)c * N + gi, hv);
          pa[c] += dv * hv;
        }
      }
      __syncthreads();
    }
    ext_block_sum(pa, wbuf);
    if (threadIdx.x == 0)
      for (int c = 0; c < 2; ++c) __stcg(a.partials + (size_t)blockIdx.x * 4 + c, pa[c]);
    if (!ext_grid_sync(a.bar, a.error, a.bar_ns)) return;
    ext_grid_total(a.partials, 2, tot, wbuf);
    double alpha[2];
    for (int c = 0; c < 2; ++c) alpha[c] = an[c] / tot[c];
    // --- phase B: x += d alpha, g += h alpha, h = g * dinv; partials g.h, g.g
    double pb[4] = {0.0, 0.0, 0.0, 0.0};
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
      const int x = (t % ntx) * kExtTX + tx, y = (t / ntx) * kExtTY + ty;
      if (x >= n || y >= n) continue;
      const size_t j = x + (size_t)y * n;
      const double di = ext_dinv(x, y, n, a.defined[j] != 0);
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        if (!act[c]) continue;
        const size_t gi = (size_t)c * N + j;
        double xv = __ldcg(a.x + gi), gv = __ldcg(a.g + gi);
        xv += __ldcg(dk + gi) * alpha[c];
        gv += __ldcg(a.hB + gi) * alpha[c];
        const double hv = gv * di;
        __stcg(a.x + gi, xv);
        __stcg(a.g + gi, gv);
        __stcg(a.hA + gi, hv);
        pb[c] += gv * hv;
        pb[2 + c] += gv * gv;
      }
    }
    ext_block_sum(pb, wbuf);
    if (threadIdx.x == 0)
      for (int k2 = 0; k2 < 4; ++k2) __stcg(a.partials + (size_t)blockIdx.x * 4 + k2, pb[k2]);
    if (!ext_grid_sync(a.bar, a.error, a.bar_ns)) return;
    ext_grid_total(a.partials, 4, tot, wbuf);
    for (int c = 0; c < 2; ++c) {
      if (!act[c]) continue;
      q[c] = tot[c] / an[c];
      an[c] = tot[c];
      spn[c] = tot[2 + c];
      act[c] = !(spn[c] < kExtEps) && it[c] < kExtMaxIter && !isnan(spn[c]);
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0 && a.iters_out) {
    a.iters_out[0] = it[0];
    a.iters_out[1] = it[1];
  }
}

// Warped frames with Inf extension into vals (F x N), as for the average.
__global__ void k_warp_values(const double* __restrict__ frames, const double* __restrict__ phis, int F, int level,
                              double* vals) {
  const int n = (1 << level) + 1, N = n * n;
  const double h = 1.0 / (double)(n - 1);
  const int f = blockIdx.y;
  const double* ph = phis + (size_t)f * 2 * N;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < N; j += gridDim.x * blockDim.x) {
    const int x = j % n, y = j / n;
    const double d0 = x + ph[j] / h, d1 = y + ph[N + j] / h;
    bool in = true;
    if (d0 < 0. || d0 > (double)(n - 1) || isnan(d0)) in = false;
    if (d1 < 0. || d1 > (double)(n - 1) || isnan(d1)) in = false;
    vals[(size_t)f * N + j] = in ? interp_d(frames + (size_t)f * N, n, d0, d1) : INFINITY;
  }
}

// Per pixel: the finite samples are moved to the front of the pixel's column
// of vals (stride N) and sorted there by insertion; the median is the middle
// sample, or the mean of the two middle ones (Vector::getMedianValue), and
// *fill where no sample is finite.
__global__ void k_median(double* vals, int F, int N, const double* fill, double* median) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < N; j += gridDim.x * blockDim.x) {
    double* v = vals + j;
    int k = 0;
    for (int f = 0; f < F; ++f) {
      const double s = v[(size_t)f * N];
      if (s != INFINITY) {
        int p = k++;
        while (p > 0 && v[(size_t)(p - 1) * N] > s) {
          v[(size_t)p * N] = v[(size_t)(p - 1) * N];
          --p;
        }
        v[(size_t)p * N] = s;
      }
    }
    if (k == 0) median[j] = *fill;
    else if (k & 1) median[j] = v[(size_t)(k / 2) * N];
    else median[j] = (v[(size_t)(k / 2 - 1) * N] + v[(size_t)(k / 2) * N]) / 2;
  }
}

}  // namespace msg
