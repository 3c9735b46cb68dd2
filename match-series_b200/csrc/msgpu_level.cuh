// msgpu_level.cuh -- the per-level solve as ONE persistent launch.
//
// Each registration instance (a template frame registered to the reference on
// one level of the multilevel pyramid) is owned by one thread-block cluster.
// The CTAs of the cluster split every data-parallel pass over the level's
// nodes/elements, synchronise with the hardware cluster barrier, and reduce
// their partial sums through distributed shared memory in a fixed rank order,
// so every CTA holds identical scalars and takes identical control decisions.
// The whole gradient flow of the level -- H1 metric V-cycle, Fletcher-Reeves
// NCG, Armijo line search, filter-width (sigma) schedule and stopping rule --
// runs on the device without host round trips:
//   GradientDescentBase::applySingle            gradientDescent.h:295-464
//   calcTaudAndDescentDir                       gradientDescent.h:200-236
//   GradientDescentWithAutomaticFilterWidth     gradientDescent.h:675-691
//   getTimestepWidthWithArmijoLineSearch        ArmijoSearch.h:118-200
//   LinearSmoothOp::apply / MDMultigrid::solve  linearSmoothOp.cpp:451-612
// Control flow is bounded: the step loop by max_iter, each line search by the
// tau range [2^-30, 2^25].  No CTA waits on anything but the cluster barrier.
#pragma once

#include <cooperative_groups.h>

#include "msgpu_fe.cuh"

namespace msg {

namespace cg = cooperative_groups;

constexpr int kThreads = 256;
constexpr int kMaxLevel = 12;
constexpr int kRedSlots = 4;   // partial sums reduced per pass

// Launch modes of the level kernel.
enum LevelMode : int {
  MODE_SOLVE = 0,   // full gradient flow on the level
  MODE_ENERGY = 1,  // E(phi) and DE(phi) only (parity entry point)
  MODE_SMOOTH = 2,  // one H1 V-cycle of the DE buffer's negation (parity)
};

template <typename Real>
struct LevelArgs {
  Real* arena;              // per-instance arenas, instance i at arena + i*inst_stride
  size_t inst_stride;
  const Real* R;            // reference image on this level (shared by all instances)
  size_t off_T;             // template image on this level
  size_t off_phi[2];        // displacement ping-pong buffers (2 components each)
  size_t off_d[2];          // descent-direction ping-pong buffers (2 components each)
  size_t off_s;             // smoothed negative gradient (2 components)
  size_t off_de;            // DE = E'[phi] (2 components)
  size_t off_x2[kMaxLevel + 1];  // V-cycle: x after pre-smoothing, per level (2 comps)
  size_t off_x5[kMaxLevel + 1];  // V-cycle: final x per level (2 comps)
  size_t off_b[kMaxLevel + 1];   // V-cycle: right-hand side per level (2 comps)
  int level, n, num_inst, lc;    // lc: levels <= lc are smoothed by CTA 0 in shared memory
  int mode;
  double lambda, stop_eps, sigma_fixed;
  int max_iter;
  const int* phi_in_dev;    // per instance: buffer holding the input displacement
  double* out_energy;       // per instance
  int* out_steps;           // per instance
  int* out_evals;           // per instance: energy evaluations of the line searches (nullable)
  int* out_phi_buf;         // per instance: buffer holding the result
  double* trace;            // optional: per instance max_trace rows of (energy, tau, sigma, evals)
  int max_trace;
};

// ---------------------------------------------------------------------------
// Cluster-wide deterministic reduction of kRedSlots doubles.
struct RedShared {
  double warp[kThreads / 32][kRedSlots];
  double slot[2][kRedSlots];  // double-buffered per-CTA partials read through DSMEM
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Returns the cluster totals in out[] (identical in every thread of every CTA).
__device__ __forceinline__ void cluster_reduce(cg::cluster_group& cluster, RedShared& rs, int& parity,
                                               const double part[kRedSlots], double out[kRedSlots]) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < kRedSlots; ++k) {
    const double v = warp_sum(part[k]);
    if (lane == 0) rs.warp[wid][k] = v;
  }
  __syncthreads();
  if (threadIdx.x < kRedSlots) {
    double s = 0.0;
#pragma unroll
    for (int w = 0; w < kThreads / 32; ++w) s += rs.warp[w][threadIdx.x];
    rs.slot[parity][threadIdx.x] = s;
  }
  __threadfence();
  cluster.sync();
  const unsigned G = cluster.num_blocks();
#pragma unroll
  for (int k = 0; k < kRedSlots; ++k) out[k] = 0.0;
  for (unsigned r = 0; r < G; ++r) {
    const double* remote = cluster.map_shared_rank(&rs.slot[parity][0], r);
#pragma unroll
    for (int k = 0; k < kRedSlots; ++k) out[k] += remote[k];
  }
  parity ^= 1;
}

__device__ __forceinline__ void cluster_barrier(cg::cluster_group& cluster) {
  __threadfence();
  cluster.sync();
}

// ---------------------------------------------------------------------------
template <typename Real>
struct Inst {
  Real* base;
  const Real* R;
  const Real* T;
  int n;
  Real h;
  __device__ Real* arr(size_t off) const { return base + off; }
};

// Energy pass over the elements owned by this CTA.
//   kind 0: E_data at phi (no direction)            -> part[0]
//            plus A = phi . L phi at owned nodes     -> part[1]
//   kind 1: E_data at phi + tau d                   -> part[0]
//   kind 2: NCG materialisation d = s + beta od (or d = s when od_zero),
//           E_data at phi + tau d                   -> part[0]
//           Df = DE . d, B = phi . L d, C = d . L d -> part[1..3]
template <typename Real>
__device__ void pass_energy(const Inst<Real>& I, int kind, Real tau, Real beta, bool od_zero,
                            const Real* __restrict__ phx, const Real* __restrict__ phy,
                            const Real* dx, const Real* dy,        // kind 1: d; kind 2: od
                            const Real* sx, const Real* sy,        // kind 2: s
                            Real* wdx, Real* wdy,                  // kind 2: output d
                            const Real* dex, const Real* dey,      // kind 2: DE
                            int rank, int G, double part[kRedSlots]) {
  const int n = I.n, ne = n - 1;
  const long total = (long)ne * ne;
  auto dval = [&](const Real* a, const Real* s, int idx) -> Real {
    // direction value at node idx for the current kind
    if (kind == 1) return a[idx];
    if (od_zero) return s[idx];
    return s[idx] + beta * a[idx];
  };
  for (long e = (long)rank * kThreads + threadIdx.x; e < total; e += (long)G * kThreads) {
    const int ex = (int)(e % ne), ey = (int)(e / ne);
    const int i0 = ey * n + ex;
    const int idx[4] = {i0, i0 + 1, i0 + n, i0 + n + 1};
    Real px[4], py[4], r[4];
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      r[b] = __ldg(I.R + idx[b]);
      if (kind == 0) {
        px[b] = phx[idx[b]];
        py[b] = phy[idx[b]];
      } else {
        // newPosition = phi + tau * d (gradientDescent.h:176-178)
        Real vx = phx[idx[b]], vy = phy[idx[b]];
        vx += tau * dval(dx, sx, idx[b]);
        vy += tau * dval(dy, sy, idx[b]);
        px[b] = vx;
        py[b] = vy;
      }
    }
    part[0] += (double)element_ssd(I.T, n, I.h, ex, ey, px, py, r);

    if (kind == 0 || kind == 2) {
      // nodes owned by this element: its lower-left node, plus the last
      // column / row of nodes for the elements on the upper boundaries.
      int own[4];
      int nown = 0;
      own[nown++] = i0;
      if (ex == ne - 1) own[nown++] = i0 + 1;
      if (ey == ne - 1) own[nown++] = i0 + n;
      if (ex == ne - 1 && ey == ne - 1) own[nown++] = i0 + n + 1;
      for (int k = 0; k < nown; ++k) {
        const int id = own[k];
        const int x = id % n, y = id / n;
        if (kind == 0) {
          const Real lx = stiff_row<Real>(x, y, n, [&](int X, int Y) { return phx[Y * n + X]; });
          const Real ly = stiff_row<Real>(x, y, n, [&](int X, int Y) { return phy[Y * n + X]; });
          part[1] += (double)phx[id] * (double)lx + (double)phy[id] * (double)ly;
        } else {
          const Real ddx = dval(dx, sx, id), ddy = dval(dy, sy, id);
          wdx[id] = ddx;
          wdy[id] = ddy;
          const Real lx = stiff_row<Real>(x, y, n, [&](int X, int Y) { return dval(dx, sx, Y * n + X); });
          const Real ly = stiff_row<Real>(x, y, n, [&](int X, int Y) { return dval(dy, sy, Y * n + X); });
          part[1] += (double)dex[id] * (double)ddx + (double)dey[id] * (double)ddy;
          part[2] += (double)phx[id] * (double)lx + (double)phy[id] * (double)ly;
          part[3] += (double)ddx * (double)lx + (double)ddy * (double)ly;
        }
      }
    }
  }
}

// Gradient pass: applies the pending update phi_new = phi + tau_p d (or copies
// phi when no step is pending), evaluates DE(phi_new) = SSDForce + lambda L phi
// (LinCombOp, registration.h:977-982) and A = phi_new . L phi_new -> part[1].
// Node tiles of 32 x 8 with the element contributions staged in shared memory;
// node sums are accumulated in the reference's element order (x fastest).
constexpr int GTX = 32, GTY = 8;
template <typename Real>
struct GradShared {
  Real pw[2][GTY + 2][GTX + 2];   // phi_new window, nodes [x0-1, x0+GTX] x [y0-1, y0+GTY]
  Real rw[GTY + 2][GTX + 2];      // reference window
  Real c[GTY + 1][GTX + 1][4][2]; // element contributions, elements [x0-1, x0+GTX) x [y0-1, y0+GTY)
};

template <typename Real>
__device__ void pass_gradient(const Inst<Real>& I, GradShared<Real>& S, bool step, Real tau_p,
                              const Real* phx, const Real* phy, const Real* dx, const Real* dy,
                              Real* nphx, Real* nphy, Real* dex, Real* dey, double lambda,
                              int rank, int G, double part[kRedSlots]) {
  const int n = I.n, ne = n - 1;
  const int tx_n = (n + GTX - 1) / GTX, ty_n = (n + GTY - 1) / GTY;
  const int tiles = tx_n * ty_n;
  const Real lam = (Real)lambda;
  for (int t = rank; t < tiles; t += G) {
    const int x0 = (t % tx_n) * GTX, y0 = (t / tx_n) * GTY;
    // 1. windows of phi_new and R
    for (int k = threadIdx.x; k < (GTY + 2) * (GTX + 2); k += kThreads) {
      const int wx = k % (GTX + 2), wy = k / (GTX + 2);
      const int x = x0 - 1 + wx, y = y0 - 1 + wy;
      Real vx = Real(0), vy = Real(0), rv = Real(0);
      if (x >= 0 && x < n && y >= 0 && y < n) {
        const int id = y * n + x;
        vx = phx[id];
        vy = phy[id];
        if (step) {  // Dest += tau * d (gradientDescent.h:385-387, descentDir *= tau)
          vx += tau_p * dx[id];
          vy += tau_p * dy[id];
        }
        rv = __ldg(I.R + id);
      }
      S.pw[0][wy][wx] = vx;
      S.pw[1][wy][wx] = vy;
      S.rw[wy][wx] = rv;
    }
    __syncthreads();
    // 2. element contributions
    for (int k = threadIdx.x; k < (GTY + 1) * (GTX + 1); k += kThreads) {
      const int cx = k % (GTX + 1), cy = k / (GTX + 1);
      const int ex = x0 - 1 + cx, ey = y0 - 1 + cy;
      if (ex < 0 || ey < 0 || ex >= ne || ey >= ne) continue;
      Real px[4], py[4], r[4];
      // window coordinates of node (ex, ey) are (cx, cy)
      px[0] = S.pw[0][cy][cx];     py[0] = S.pw[1][cy][cx];     r[0] = S.rw[cy][cx];
      px[1] = S.pw[0][cy][cx + 1]; py[1] = S.pw[1][cy][cx + 1]; r[1] = S.rw[cy][cx + 1];
      px[2] = S.pw[0][cy + 1][cx]; py[2] = S.pw[1][cy + 1][cx]; r[2] = S.rw[cy + 1][cx];
      px[3] = S.pw[0][cy + 1][cx + 1]; py[3] = S.pw[1][cy + 1][cx + 1]; r[3] = S.rw[cy + 1][cx + 1];
      element_force(I.T, n, I.h, ex, ey, px, py, r, S.c[cy][cx]);
    }
    __syncthreads();
    // 3. node sums, stiffness, outputs
    {
      const int lx = threadIdx.x % GTX, ly = threadIdx.x / GTX;
      const int x = x0 + lx, y = y0 + ly;
      if (x < n && y < n) {
        // window/contribution index of element (x-1+a, y-1+b) is (lx+a, ly+b)
        Real fx = Real(0), fy = Real(0);
        if (x - 1 >= 0 && y - 1 >= 0) { fx += S.c[ly][lx][3][0];     fy += S.c[ly][lx][3][1]; }
        if (x < ne && y - 1 >= 0)     { fx += S.c[ly][lx + 1][2][0]; fy += S.c[ly][lx + 1][2][1]; }
        if (x - 1 >= 0 && y < ne)     { fx += S.c[ly + 1][lx][1][0]; fy += S.c[ly + 1][lx][1][1]; }
        if (x < ne && y < ne)         { fx += S.c[ly + 1][lx + 1][0][0]; fy += S.c[ly + 1][lx + 1][0][1]; }
        const Real Lx = stiff_row<Real>(x, y, n, [&](int X, int Y) { return S.pw[0][Y - y0 + 1][X - x0 + 1]; });
        const Real Ly = stiff_row<Real>(x, y, n, [&](int X, int Y) { return S.pw[1][Y - y0 + 1][X - x0 + 1]; });
        const Real gx = (lambda != 1.0) ? fx + lam * Lx : fx + Lx;
        const Real gy = (lambda != 1.0) ? fy + lam * Ly : fy + Ly;
        const int id = y * n + x;
        dex[id] = gx;
        dey[id] = gy;
        const Real vx = S.pw[0][ly + 1][lx + 1], vy = S.pw[1][ly + 1][lx + 1];
        nphx[id] = vx;
        nphy[id] = vy;
        part[1] += (double)vx * (double)Lx + (double)vy * (double)Ly;
      }
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Multigrid V-cycle passes on the levels above lc (cluster passes).
constexpr int VTX = 32, VTY = 16;
template <typename Real>
struct DownShared {
  Real rhs[2][VTY + 6][VTX + 6];  // halo 3
  Real x1[2][VTY + 6][VTX + 6];   // halo 3
  Real x2[2][VTY + 4][VTX + 4];   // halo 2
  Real r[2][VTY + 2][VTX + 2];    // halo 1
};
template <typename Real>
struct UpShared {
  Real rhs[2][VTY + 4][VTX + 4];  // halo 2
  Real x3[2][VTY + 4][VTX + 4];   // halo 2
  Real x4[2][VTY + 2][VTX + 2];   // halo 1
};

// Pre-smoothing (2 Jacobi sweeps from x = 0), residual and restriction
// (MDMultigrid::solve steps 1-3, linearSmoothOp.cpp:465-477).
// rhs of level k: -DE on the finest level (negate), else b[k].
template <typename Real>
__device__ void pass_down(int k, int n, const Real* rhsx, const Real* rhsy, bool negate, Real* x2x, Real* x2y,
                          Real* bcx, Real* bcy, Real hsq, Real diag, DownShared<Real>& S, int rank, int G) {
  const int cw = (n >> 1) + 1;
  const int tx_n = (n + VTX - 1) / VTX, ty_n = (n + VTY - 1) / VTY;
  const int tiles = tx_n * ty_n;
  for (int t = rank; t < tiles; t += G) {
    const int x0 = (t % tx_n) * VTX, y0 = (t / tx_n) * VTY;
    // rhs and x1 = 0 + (rhs - A 0)/diag on halo 3
    for (int q = threadIdx.x; q < (VTY + 6) * (VTX + 6); q += kThreads) {
      const int wx = q % (VTX + 6), wy = q / (VTX + 6);
      const int x = x0 - 3 + wx, y = y0 - 3 + wy;
      Real a = Real(0), b = Real(0);
      if (x >= 0 && x < n && y >= 0 && y < n) {
        const int id = y * n + x;
        a = rhsx[id];
        b = rhsy[id];
        if (negate) { a = a * Real(-1); b = b * Real(-1); }
      }
      S.rhs[0][wy][wx] = a;
      S.rhs[1][wy][wx] = b;
      S.x1[0][wy][wx] = jacobi_update(Real(0), a, Real(0), diag);
      S.x1[1][wy][wx] = jacobi_update(Real(0), b, Real(0), diag);
    }
    __syncthreads();
    // x2 on halo 2
    for (int q = threadIdx.x; q < (VTY + 4) * (VTX + 4); q += kThreads) {
      const int wx = q % (VTX + 4), wy = q / (VTX + 4);
      const int x = x0 - 2 + wx, y = y0 - 2 + wy;
      if (x < 0 || x >= n || y < 0 || y >= n) continue;
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        auto A = [&](int X, int Y) { return S.x1[c][Y - y0 + 3][X - x0 + 3]; };
        const Real ax = heat_row<Real>(x, y, n, hsq, A);
        S.x2[c][wy][wx] = jacobi_update(S.x1[c][wy + 1][wx + 1], S.rhs[c][wy + 1][wx + 1], ax, diag);
      }
    }
    __syncthreads();
    // residual on halo 1, and x2 out for owned nodes
    for (int q = threadIdx.x; q < (VTY + 2) * (VTX + 2); q += kThreads) {
      const int wx = q % (VTX + 2), wy = q / (VTX + 2);
      const int x = x0 - 1 + wx, y = y0 - 1 + wy;
      if (x < 0 || x >= n || y < 0 || y >= n) continue;
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        auto A = [&](int X, int Y) { return S.x2[c][Y - y0 + 2][X - x0 + 2]; };
        const Real ax = heat_row<Real>(x, y, n, hsq, A);
        S.r[c][wy][wx] = S.rhs[c][wy + 2][wx + 2] - ax;
      }
      if (wx >= 1 && wx <= VTX && wy >= 1 && wy <= VTY) {
        const int id = y * n + x;
        x2x[id] = S.x2[0][wy + 1][wx + 1];
        x2y[id] = S.x2[1][wy + 1][wx + 1];
      }
    }
    __syncthreads();
    // restriction of the residual to the coarse nodes centred in this tile
    for (int q = threadIdx.x; q < (VTY / 2) * (VTX / 2); q += kThreads) {
      const int X = (x0 >> 1) + q % (VTX / 2), Y = (y0 >> 1) + q / (VTX / 2);
      if (X >= cw || Y >= cw) continue;
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        auto F = [&](int x, int y) { return S.r[c][y - y0 + 1][x - x0 + 1]; };
        const Real v = restrict_node<Real>(X, Y, cw, F);
        (c == 0 ? bcx : bcy)[Y * cw + X] = v;
      }
    }
    __syncthreads();
  }
}

// Correction and post-smoothing (MDMultigrid::solve steps 5-6,
// linearSmoothOp.cpp:483-493): x3 = x2 + P x_coarse, then 2 Jacobi sweeps.
// With want_norm, accumulates |x5|^2 into part[0].
template <typename Real>
__device__ void pass_up(int k, int n, const Real* rhsx, const Real* rhsy, bool negate, const Real* x2x,
                        const Real* x2y, const Real* xcx, const Real* xcy, Real* ox, Real* oy, Real hsq,
                        Real diag, UpShared<Real>& S, int rank, int G, bool want_norm, double part[kRedSlots]) {
  const int cw = (n >> 1) + 1;
  const int tx_n = (n + VTX - 1) / VTX, ty_n = (n + VTY - 1) / VTY;
  const int tiles = tx_n * ty_n;
  for (int t = rank; t < tiles; t += G) {
    const int x0 = (t % tx_n) * VTX, y0 = (t / tx_n) * VTY;
    for (int q = threadIdx.x; q < (VTY + 4) * (VTX + 4); q += kThreads) {
      const int wx = q % (VTX + 4), wy = q / (VTX + 4);
      const int x = x0 - 2 + wx, y = y0 - 2 + wy;
      Real a = Real(0), b = Real(0), u = Real(0), v = Real(0);
      if (x >= 0 && x < n && y >= 0 && y < n) {
        const int id = y * n + x;
        a = rhsx[id];
        b = rhsy[id];
        if (negate) { a = a * Real(-1); b = b * Real(-1); }
        const Real px = prolong_node<Real>(x, y, [&](int X, int Y) { return xcx[Y * cw + X]; });
        const Real py = prolong_node<Real>(x, y, [&](int X, int Y) { return xcy[Y * cw + X]; });
        u = x2x[id] + px;
        v = x2y[id] + py;
      }
      S.rhs[0][wy][wx] = a;
      S.rhs[1][wy][wx] = b;
      S.x3[0][wy][wx] = u;
      S.x3[1][wy][wx] = v;
    }
    __syncthreads();
    for (int q = threadIdx.x; q < (VTY + 2) * (VTX + 2); q += kThreads) {
      const int wx = q % (VTX + 2), wy = q / (VTX + 2);
      const int x = x0 - 1 + wx, y = y0 - 1 + wy;
      if (x < 0 || x >= n || y < 0 || y >= n) continue;
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        auto A = [&](int X, int Y) { return S.x3[c][Y - y0 + 2][X - x0 + 2]; };
        const Real ax = heat_row<Real>(x, y, n, hsq, A);
        S.x4[c][wy][wx] = jacobi_update(S.x3[c][wy + 1][wx + 1], S.rhs[c][wy + 1][wx + 1], ax, diag);
      }
    }
    __syncthreads();
    for (int q = threadIdx.x; q < VTY * VTX; q += kThreads) {
      const int wx = q % VTX, wy = q / VTX;
      const int x = x0 + wx, y = y0 + wy;
      if (x >= n || y >= n) continue;
      Real out[2];
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        auto A = [&](int X, int Y) { return S.x4[c][Y - y0 + 1][X - x0 + 1]; };
        const Real ax = heat_row<Real>(x, y, n, hsq, A);
        out[c] = jacobi_update(S.x4[c][wy + 1][wx + 1], S.rhs[c][wy + 2][wx + 2], ax, diag);
      }
      const int id = y * n + x;
      ox[id] = out[0];
      oy[id] = out[1];
      if (want_norm) part[0] += (double)out[0] * (double)out[0] + (double)out[1] * (double)out[1];
    }
    __syncthreads();
  }
}

// Coarse part of the V-cycle, levels lc..0, by one CTA in shared memory
// (MDMultigrid::solve recursion including the 100 sweeps on level 0).
// Layout per level k: x[c], b[c], tmp[c], each (2^k+1)^2.
template <typename Real>
__device__ __forceinline__ size_t coarse_level_offset(int k) {
  size_t off = 0;
  for (int j = 0; j < k; ++j) {
    const size_t w = (size_t)(1 << j) + 1;
    off += 6 * w * w;
  }
  return off;
}

template <typename Real>
__device__ void coarse_vcycle(int lc, double tau, Real* sm, const Real* bx, const Real* by, bool negate,
                              Real* outx, Real* outy, bool want_norm, double part[kRedSlots]) {
  auto X = [&](int k, int c) { const size_t w = (size_t)(1 << k) + 1; return sm + coarse_level_offset<Real>(k) + (size_t)c * w * w; };
  auto B = [&](int k, int c) { const size_t w = (size_t)(1 << k) + 1; return sm + coarse_level_offset<Real>(k) + (size_t)(2 + c) * w * w; };
  auto TMP = [&](int k, int c) { const size_t w = (size_t)(1 << k) + 1; return sm + coarse_level_offset<Real>(k) + (size_t)(4 + c) * w * w; };
  {
    const int w = (1 << lc) + 1;
    for (int i = threadIdx.x; i < w * w; i += kThreads) {
      Real a = bx[i], b = by[i];
      if (negate) { a = a * Real(-1); b = b * Real(-1); }
      B(lc, 0)[i] = a;
      B(lc, 1)[i] = b;
      X(lc, 0)[i] = Real(0);
      X(lc, 1)[i] = Real(0);
    }
    __syncthreads();
  }
  auto jacobi_sweep = [&](int k) {
    const int w = (1 << k) + 1;
    const Real hsq = (Real)(tau * (double)((w - 1) * (w - 1)));
    const Real diag = (Real)(1 + 4 * tau * (double)((w - 1) * (w - 1)));
    for (int i = threadIdx.x; i < 2 * w * w; i += kThreads) {
      const int c = i / (w * w), id = i % (w * w);
      const Real* xs = X(k, c);
      TMP(k, c)[id] = heat_row<Real>(id % w, id / w, w, hsq, [&](int a, int b) { return xs[b * w + a]; });
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 2 * w * w; i += kThreads) {
      const int c = i / (w * w), id = i % (w * w);
      X(k, c)[id] = jacobi_update(X(k, c)[id], B(k, c)[id], TMP(k, c)[id], diag);
    }
    __syncthreads();
  };
  // descend
  for (int k = lc; k >= 1; --k) {
    const int w = (1 << k) + 1, cw = (1 << (k - 1)) + 1;
    const Real hsq = (Real)(tau * (double)((w - 1) * (w - 1)));
    jacobi_sweep(k);
    jacobi_sweep(k);
    for (int i = threadIdx.x; i < 2 * w * w; i += kThreads) {
      const int c = i / (w * w), id = i % (w * w);
      const Real* xs = X(k, c);
      const Real ax = heat_row<Real>(id % w, id / w, w, hsq, [&](int a, int b) { return xs[b * w + a]; });
      TMP(k, c)[id] = B(k, c)[id] - ax;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 2 * cw * cw; i += kThreads) {
      const int c = i / (cw * cw), id = i % (cw * cw);
      const Real* rs = TMP(k, c);
      B(k - 1, c)[id] = restrict_node<Real>(id % cw, id / cw, cw, [&](int a, int b) { return rs[b * w + a]; });
      X(k - 1, c)[id] = Real(0);
    }
    __syncthreads();
  }
  // level 0: 100 sweeps by one warp (2 components x 4 nodes)
  if (threadIdx.x < 32) {
    const double hsq0 = tau * 1.0, diag0 = 1 + 4 * tau * 1.0;
    const Real hsq = (Real)hsq0, diag = (Real)diag0;
    const int c = (threadIdx.x >> 2) & 1, id = threadIdx.x & 3;
    for (int it = 0; it < 100; ++it) {
      Real ax = Real(0);
      if (threadIdx.x < 8) {
        const Real* xs = X(0, c);
        ax = heat_row<Real>(id & 1, id >> 1, 2, hsq, [&](int a, int b) { return xs[b * 2 + a]; });
      }
      __syncwarp();
      if (threadIdx.x < 8) X(0, c)[id] = jacobi_update(X(0, c)[id], B(0, c)[id], ax, diag);
      __syncwarp();
    }
  }
  __syncthreads();
  // ascend
  for (int k = 1; k <= lc; ++k) {
    const int w = (1 << k) + 1, cw = (1 << (k - 1)) + 1;
    for (int i = threadIdx.x; i < 2 * w * w; i += kThreads) {
      const int c = i / (w * w), id = i % (w * w);
      const Real* xc = X(k - 1, c);
      const Real p = prolong_node<Real>(id % w, id / w, [&](int a, int b) { return xc[b * cw + a]; });
      X(k, c)[id] += p;
    }
    __syncthreads();
    jacobi_sweep(k);
    jacobi_sweep(k);
  }
  {
    const int w = (1 << lc) + 1;
    for (int i = threadIdx.x; i < w * w; i += kThreads) {
      const Real a = X(lc, 0)[i], b = X(lc, 1)[i];
      outx[i] = a;
      outy[i] = b;
      if (want_norm) part[0] += (double)a * (double)a + (double)b * (double)b;
    }
  }
}

template <typename Real>
__host__ __device__ inline size_t coarse_smem_elems(int lc) {
  size_t off = 0;
  for (int j = 0; j <= lc; ++j) {
    const size_t w = (size_t)(1 << j) + 1;
    off += 6 * w * w;
  }
  return off;
}

// Full V-cycle on the current level: rhs = -DE (finest), output s.
// Returns |s|^2 (cluster total) in norm_out.
template <typename Real>
__device__ void vcycle(cg::cluster_group& cluster, RedShared& rs, int& parity, const LevelArgs<Real>& a,
                       const Inst<Real>& I, double tau, void* smem, int rank, int G, double& norm_out) {
  const int L = a.level;
  const Real* dex = I.arr(a.off_de);
  const Real* dey = dex + (size_t)I.n * I.n;
  Real* sx = I.arr(a.off_s);
  Real* sy = sx + (size_t)I.n * I.n;
  double part[kRedSlots] = {0, 0, 0, 0}, tot[kRedSlots];
  // descend through the cluster-pass levels
  for (int k = L; k > a.lc; --k) {
    const int w = (1 << k) + 1, cw = (1 << (k - 1)) + 1;
    const Real hsq = (Real)(tau * (double)((w - 1) * (w - 1)));
    const Real diag = (Real)(1 + 4 * tau * (double)((w - 1) * (w - 1)));
    const Real* rx = (k == L) ? dex : I.arr(a.off_b[k]);
    const Real* ry = rx + (size_t)w * w;
    Real* x2 = I.arr(a.off_x2[k]);
    Real* bc = I.arr(a.off_b[k - 1]);
    pass_down<Real>(k, w, rx, ry, k == L, x2, x2 + (size_t)w * w, bc, bc + (size_t)cw * cw, hsq, diag,
                    *reinterpret_cast<DownShared<Real>*>(smem), rank, G);
    cluster_barrier(cluster);
  }
  // coarse levels by CTA 0
  if (rank == 0) {
    const int lc = a.lc;
    const int w = (1 << lc) + 1;
    const Real* bx = (L == lc) ? dex : I.arr(a.off_b[lc]);
    Real* out = (L == lc) ? sx : I.arr(a.off_x5[lc]);
    coarse_vcycle<Real>(lc, tau, reinterpret_cast<Real*>(smem), bx, bx + (size_t)w * w, L == lc, out,
                        out + (size_t)w * w, L == lc, part);
  }
  if (L == a.lc) {
    cluster_reduce(cluster, rs, parity, part, tot);
    norm_out = tot[0];
    return;
  }
  cluster_barrier(cluster);
  // ascend
  for (int k = a.lc + 1; k <= L; ++k) {
    const int w = (1 << k) + 1, cw = (1 << (k - 1)) + 1;
    const Real hsq = (Real)(tau * (double)((w - 1) * (w - 1)));
    const Real diag = (Real)(1 + 4 * tau * (double)((w - 1) * (w - 1)));
    const Real* rx = (k == L) ? dex : I.arr(a.off_b[k]);
    const Real* x2 = I.arr(a.off_x2[k]);
    const Real* xc = I.arr(a.off_x5[k - 1]);
    Real* o = (k == L) ? sx : I.arr(a.off_x5[k]);
    pass_up<Real>(k, w, rx, rx + (size_t)w * w, k == L, x2, x2 + (size_t)w * w, xc, xc + (size_t)cw * cw, o,
                  o + (size_t)w * w, hsq, diag, *reinterpret_cast<UpShared<Real>*>(smem), rank, G, k == L, part);
    if (k < L) cluster_barrier(cluster);
  }
  cluster_reduce(cluster, rs, parity, part, tot);
  norm_out = tot[0];
}

__device__ __forceinline__ bool finite_d(double x) { return !isnan(x) && !isinf(x); }

// ---------------------------------------------------------------------------
template <typename Real>
__global__ void __launch_bounds__(kThreads) level_kernel(LevelArgs<Real> a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ RedShared rs;
  cg::cluster_group cluster = cg::this_cluster();
  const int G = (int)cluster.num_blocks();
  const int rank = (int)cluster.block_rank();
  const int cid = blockIdx.x / G;
  const int nclusters = gridDim.x / G;
  int parity = 0;
  const int n = a.n;
  const size_t N = (size_t)n * n;
  const double lam = a.lambda;

  for (int inst = cid; inst < a.num_inst; inst += nclusters) {
    Inst<Real> I;
    I.base = a.arena + (size_t)inst * a.inst_stride;
    I.R = a.R;
    I.T = I.base + a.off_T;
    I.n = n;
    I.h = (Real)(1.0 / (double)(n - 1));
    Real* de = I.arr(a.off_de);
    Real* s = I.arr(a.off_s);
    int cur = a.phi_in_dev ? a.phi_in_dev[inst] : 0;  // buffer holding phi
    int dcur = 0;         // buffer holding the current direction d (written by the NCG pass)
    double part[kRedSlots], tot[kRedSlots];

    auto reset = [&]() {
#pragma unroll
      for (int k = 0; k < kRedSlots; ++k) part[k] = 0.0;
    };
    Real* phi = I.arr(a.off_phi[cur]);

    if (a.mode == MODE_SMOOTH) {
      double nrm;
      vcycle<Real>(cluster, rs, parity, a, I, (double)(0.5f * (a.sigma_fixed * a.sigma_fixed)), smem_raw, rank, G, nrm);
      cluster_barrier(cluster);
      continue;
    }

    // initial energy E(phi) = E_data + lambda * 1/2 phi.L phi   (gradientDescent.h:306)
    reset();
    pass_energy<Real>(I, 0, Real(0), Real(0), false, phi, phi + N, nullptr, nullptr, nullptr, nullptr, nullptr,
                      nullptr, nullptr, nullptr, rank, G, part);
    cluster_reduce(cluster, rs, parity, part, tot);
    double A = tot[1];
    auto energy_of = [&](double edata, double ereg) {
      double e = 0.0;
      e += edata;
      if (lam != 1.0) e += lam * ereg; else e += ereg;
      return e;
    };
    double energy = energy_of(tot[0], 0.5 * A);
    double energy_new = energy;

    if (a.mode == MODE_ENERGY) {
      reset();
      pass_gradient<Real>(I, *reinterpret_cast<GradShared<Real>*>(smem_raw), false, Real(0), phi, phi + N,
                          nullptr, nullptr, I.arr(a.off_phi[cur ^ 1]), I.arr(a.off_phi[cur ^ 1]) + N, de, de + N,
                          lam, rank, G, part);
      cluster_barrier(cluster);
      if (rank == 0 && threadIdx.x == 0) {
        a.out_energy[inst] = energy;
        a.out_steps[inst] = 0;
        a.out_phi_buf[inst] = cur;
      }
      continue;
    }

    double tau = 1.0, sigma = 1.0;
    const double tau_min = 9.313225746154785e-10;  // 2^-30 (ArmijoSearch.h:77)
    const double tau_max = 33554432.0;             // 2^25  (ArmijoSearch.h:67)
    const double stop_sigma = 0.0001, sigma_tol = 0.00001;
    double og2 = 0.0;           // |OldGradient|^2
    bool od_zero = true;        // OldDirection is zero (start, or after the NCG fallback)
    double rb_tau[2] = {nan(""), nan("")}, rb_e[2] = {0, 0};
    int rb_pos = 0;
    bool pending = false;       // a step tau_p * d[dcur] still has to be added to phi
    double tau_p = 0.0;
    int iter = 0;
    int total_evals = 0;

    if (a.max_iter > 0) {
      bool go;
      do {
        iter++;
        energy = energy_new;
        const double f = energy;
        const double sigma_used = sigma;
        int evals = 0;
        // DE at the current position; applies the pending update (ping-pong phi)
        reset();
        {
          Real* nphi = I.arr(a.off_phi[cur ^ 1]);
          const Real* dd = I.arr(a.off_d[dcur]);
          pass_gradient<Real>(I, *reinterpret_cast<GradShared<Real>*>(smem_raw), pending, (Real)tau_p, phi,
                              phi + N, dd, dd + N, nphi, nphi + N, de, de + N, lam, rank, G, part);
          cur ^= 1;
          phi = nphi;
          pending = false;
        }
        cluster_reduce(cluster, rs, parity, part, tot);
        A = tot[1];
        // H1 smoothing of -DE (the descent direction's metric)
        double s2;
        vcycle<Real>(cluster, rs, parity, a, I, (double)(0.5f * (sigma * sigma)), smem_raw, rank, G, s2);
        // Fletcher-Reeves (gradientDescent.h:221-226)
        const double beta = ((iter - 1) % 10) ? (s2 / og2) : 0.0;
        og2 = s2;

        // Armijo line search with the NCG direction, then the NCG fallback
        double Bd = 0.0, Cd = 0.0;
        auto eval_at = [&](double tt) {
          // energy at phi + tt d; E_reg by the exact quadratic expansion in tt
          reset();
          const Real* dd = I.arr(a.off_d[dcur]);
          pass_energy<Real>(I, 1, (Real)tt, Real(0), false, phi, phi + N, dd, dd + N, nullptr, nullptr, nullptr,
                            nullptr, nullptr, nullptr, rank, G, part);
          cluster_reduce(cluster, rs, parity, part, tot);
          const double e = energy_of(tot[0], 0.5 * ((A + 2.0 * tt * Bd) + tt * tt * Cd));
          rb_tau[rb_pos] = tt;
          rb_e[rb_pos] = e;
          rb_pos ^= 1;
          evals++;
          return e;
        };
        double acc_tau = 0.0;
        for (int attempt = 0; attempt < 2; ++attempt) {
          const bool fallback = (attempt == 1);
          const int dn = dcur ^ 1;   // buffer receiving the new direction
          Real* wd = I.arr(a.off_d[dn]);
          const Real* od = I.arr(a.off_d[dcur]);
          double t = (attempt == 0) ? tau : 0.0;
          t = t < tau_min ? tau_min : (t > tau_max ? tau_max : t);
          // first trial fused with the direction materialisation
          reset();
          pass_energy<Real>(I, 2, (Real)t, (Real)beta, fallback || od_zero, phi, phi + N, od, od + N, s, s + N, wd,
                            wd + N, de, de + N, rank, G, part);
          cluster_reduce(cluster, rs, parity, part, tot);
          dcur = dn;
          const double Df = tot[1];
          Bd = tot[2];
          Cd = tot[3];
          double fnew = energy_of(tot[0], 0.5 * ((A + 2.0 * t * Bd) + t * t * Cd));
          rb_tau[rb_pos] = t;
          rb_e[rb_pos] = fnew;
          rb_pos ^= 1;
          evals++;
          double G_ = (fnew - f) / (Df * t);
          double res;
          if (Df >= 0) {
            res = 0.0;
          } else if (!finite_d(f)) {
            res = 0.0;
          } else {
            if (G_ >= 0.5 && f >= fnew) {
              do {
                t *= 2.;
                fnew = eval_at(t);
                G_ = (fnew - f) / (Df * t);
              } while (G_ >= 0.5 && f >= fnew && t <= tau_max);
              t *= 0.5;
            } else {
              do {
                if (t > tau_min) t *= 0.5;
                fnew = eval_at(t);
                G_ = (fnew - f) / (Df * t);
              } while ((!finite_d(fnew) || (G_ < 0.5 || f < fnew)) && (t > tau_min));
            }
            res = (t > tau_min) ? t : 0.0;
          }
          acc_tau = res;
          od_zero = fallback;
          if (res != 0.0) break;
        }
        tau = acc_tau;
        // energy at the new position (gradientDescent.h:365-395)
        double en = nan("");
        if (rb_tau[0] == tau) en = rb_e[0];
        else if (rb_tau[1] == tau) en = rb_e[1];
        else if (tau == 0) en = energy;
        if (isnan(en) && tau != 0) en = eval_at(tau);
        if (tau != 0) {
          pending = true;
          tau_p = tau;
        }
        energy_new = en;
        total_evals += evals;
        if (a.trace && rank == 0 && threadIdx.x == 0 && iter <= a.max_trace) {
          double* tr = a.trace + ((size_t)inst * a.max_trace + (iter - 1)) * 4;
          tr[0] = energy_new;
          tr[1] = tau;
          tr[2] = sigma_used;
          tr[3] = evals;
        }
        go = ((energy - energy_new) > a.stop_eps) && (iter < a.max_iter);
        if ((0.5 * sigma > stop_sigma) && ((energy - energy_new) < sigma_tol)) {
          sigma *= 0.5;
          tau = 1.;
          go = (sigma > stop_sigma) && (iter < a.max_iter);
        }
      } while (go);
    }
    // flush the last accepted step into phi
    if (pending) {
      Real* nphi = I.arr(a.off_phi[cur ^ 1]);
      const Real* dd = I.arr(a.off_d[dcur]);
      const Real tp = (Real)tau_p;
      for (size_t i = (size_t)rank * kThreads + threadIdx.x; i < N; i += (size_t)G * kThreads) {
        Real vx = phi[i], vy = phi[N + i];
        vx += tp * dd[i];
        vy += tp * dd[N + i];
        nphi[i] = vx;
        nphi[N + i] = vy;
      }
      cur ^= 1;
    }
    cluster_barrier(cluster);
    if (rank == 0 && threadIdx.x == 0) {
      a.out_energy[inst] = energy_new;
      a.out_steps[inst] = iter;
      a.out_phi_buf[inst] = cur;
      if (a.out_evals) a.out_evals[inst] = total_evals;
    }
  }
}

}  // namespace msg
