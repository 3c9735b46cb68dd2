// msgpu_level.cuh -- the per-level solve as ONE persistent launch.
//
// Each registration instance (a template frame registered to the reference on
// one level of the multilevel pyramid) runs the whole gradient flow of the
// level -- H1 metric V-cycle, Fletcher-Reeves NCG, Armijo line search,
// filter-width (sigma) schedule and stopping rule -- on the device without
// host round trips:
//   GradientDescentBase::applySingle            gradientDescent.h:295-464
//   calcTaudAndDescentDir                       gradientDescent.h:200-236
//   GradientDescentWithAutomaticFilterWidth     gradientDescent.h:675-691
//   getTimestepWidthWithArmijoLineSearch        ArmijoSearch.h:118-200
//   LinearSmoothOp::apply / MDMultigrid::solve  linearSmoothOp.cpp:451-612
// Every data-parallel pass of an instance is cut into node tiles, and one
// persistent grid of CTAs (two per SM) executes the tiles of all instances
// through a task scheduler (end of this file): tiles are handed out in
// chunks, every tile stores its partial sums, and whoever completes the last
// chunk of a pass adds them in tile order and takes the instance's next
// control decision.  Control flow is bounded: the step
// loop by max_iter, each line search by the tau range [2^-30, 2^25], every
// wait for work by an iteration limit.
//
// Every pass is a double-buffered tile pipeline: while a CTA computes one
// 64 x 4 node tile from shared memory, cp.async streams the windows (tile plus
// halo) of the next tile from HBM/L2 into the other buffer.  Rows are pitched
// to a multiple of 4 elements so that every window row is a sequence of
// aligned 16-byte chunks.
#pragma once

#include "msgpu_fe.cuh"
#include "msgpu_xsum.cuh"

namespace msg {

constexpr int kThreads = 256;
constexpr int kMaxLevel = 12;
constexpr int kRedSlots = 4;   // partial sums reduced per pass
// Certified control steps with exact sums: term buffers per instance, and per
// tile of an energy pass the sums and the magnitude sums of its 5 term sets.
constexpr int kXsBufs = 6;
constexpr int kXpSlots = 10;

// Node tiles: [x0, x0+TX) x [y0, y0+TY); the last tile of a row/column also
// owns the final node (n-1 = 2^l is a multiple of the tile size for l >= 6).
constexpr int TX = 64, TY = 8;
// Windows of the element passes: nodes [x0-4, x0+68) x [y0-1, y0+6).
constexpr int EWX = 72, EWY = TY + 3, EWIN = EWX * EWY;
// Multigrid passes use taller tiles of VTX x VTY nodes (halo 3 around them):
// windows of nodes [x0-4, x0+36) x [y0-3, y0+20).
constexpr int VTX = 32, VTY = 16;
constexpr int VWX = 40, VWY = 23, VWIN = VWX * VWY;
// Coarse window of the correction pass: coarse nodes [x0/2-4, x0/2+20) x [y0/2-2, y0/2+11).
constexpr int CWX = 24, CWY = 13, CWIN = CWX * CWY;
// Element contributions of the gradient pass: elements [x0-1, x0+65) x [y0-1, y0+5).
constexpr int GCX = 66, GCY = TY + 2;

// Launch modes of the level kernel.
enum LevelMode : int {
  MODE_SOLVE = 0,   // full gradient flow on the level
  MODE_ENERGY = 1,  // E(phi) and DE(phi) only (parity entry point)
  MODE_SMOOTH = 2,  // one H1 V-cycle of the DE buffer's negation (parity)
};

__host__ __device__ inline int pitch_of(int n) { return (n + 3) & ~3; }

template <typename Real>
struct LevelArgs {
  Real* arena;              // per-instance arenas, instance i at arena + i*inst_stride
  size_t inst_stride;
  const Real* R;            // reference image on this level (shared by all instances), pitched
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
  // optional energy log of the reference's per-level file (energy_%02d.txt,
  // gradientDescent.h:254-272): per instance max_trace + 1 rows of
  // (iteration - 1, lambda * E_reg at the new position, energy), the
  // first row (-1) for the initial position
  double* elog;
  unsigned long long* pass_cycles;  // optional: per CTA kPassKinds clock64 totals
  // normalized cross-correlation data term (ncc != 0)
  int ncc;
  const Real* normR;        // normalised reference on this level, pitched (shared)
  size_t off_td;            // per instance: deformed template at the nodes (1 component)
  // r_prev != 0: instance i > 0 is registered to the template of instance
  // i - 1 (the pairwise step of series matching) instead of R; with NCC each
  // instance then reads its own normalised reference at off_nr.
  int r_prev;
  size_t off_nr;
  // ragged batches (series of different sizes in one launch): inst_ref != 0
  // gives each instance the reference of its series, R + inst_ref[i] *
  // ref_stride, and (with NCC) its own normalised reference at off_nr;
  // lambda_inst != 0 its own regularisation weight.
  const int* inst_ref;
  size_t ref_stride;
  const double* lambda_inst;
  // bound of one wait for work, in nanoseconds of the global timer; a worker
  // that waits longer sets the error flag and every worker returns
  unsigned long long idle_ns;
  // exact sums (FP64, SSD): every global sum in the reference's sequential
  // order (msgpu_xsum.cuh); per-instance regions of xs_stride doubles, or null
  double* xs;
  size_t xs_stride;
  // certified control steps: xs_bufs term buffers of xs_stride doubles per
  // instance (<= 1: one, and every pass's sums are added in order before its
  // control step); xpart (nullable): per instance xpart_stride doubles, per
  // tile of an energy pass kXpSlots sums (the 5 sums, their magnitude sums)
  int xs_bufs;
  double* xpart;
  size_t xpart_stride;
  // energy targets (nullable, per instance): the solve stops as soon as its
  // energy is <= e_target + e_tol |e_target| (registration to a stated
  // energy tolerance; no counterpart in the reference's stop rules)
  const double* e_target;
  double e_tol;
  // scheduling (tuned per level, results do not depend on them): a pass is
  // handed out in chunks of ntiles / chunk_div tiles, at most chunk_max
  int chunk_div, chunk_max;
  // optional profile of the exact sums: calls, cycles of their three steps,
  // chunks walked, chunks added term by term
  unsigned long long* xs_prof;
  // optional pass timeline (profiling): up to tl_cap events of two words
  // (global timer in ns; the packed event, trace_ev), their count at tl_n
  unsigned long long* tl;
  unsigned int* tl_n;
  unsigned int tl_cap;
};

// Events of the pass timeline: a pass published (instance, kind), a pass
// completed (its last chunk done: instance, kind), a wait for work of one
// CTA that lasted 500 ns or more (its length), an ordered walk (its length),
// an open control step that has a term buffer's sums added in order
// (instance, buffer, the kind of the pass whose step is open).
constexpr unsigned kEvPublish = 1, kEvComplete = 2, kEvIdle = 3, kEvWalk = 4, kEvResolve = 5;
__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
template <typename Real>
__device__ __forceinline__ void trace_ev(const LevelArgs<Real>& a, unsigned long long t, unsigned ev,
                                         unsigned value) {
  if (!a.tl) return;
  const unsigned i = atomicAdd(a.tl_n, 1u);
  if (i < a.tl_cap) {
    a.tl[2 * (size_t)i] = t;
    a.tl[2 * (size_t)i + 1] = ((unsigned long long)((ev << 24) | blockIdx.x) << 32) | value;
  }
}

// A 2-component array of level k occupies 2 * comp_stride(k) elements.
__host__ __device__ inline size_t comp_stride(int level) {
  const size_t n = (size_t)(1 << level) + 1;
  return n * (size_t)pitch_of((int)n);
}

// Pass kinds of the per-pass cycle counters.
enum PassKind : int { PK_ENERGY0 = 0, PK_GRAD, PK_VDOWN, PK_VCOARSE, PK_VUP, PK_NCG, PK_ENERGY, PK_REDUCE, kPassKinds };

#define MSG_TIMED(pt, kind, ...) \
  do {                                \
    (pt).start();                     \
    __VA_ARGS__;                      \
    (pt).stop(kind);                  \
  } while (0)

struct PassTimer {
  unsigned long long* acc;
  long long t0;
  __device__ void start() { if (acc) t0 = clock64(); }
  __device__ void stop(int kind) {
    if (acc && threadIdx.x == 0) acc[kind] += (unsigned long long)(clock64() - t0);
  }
};

// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// ---------------------------------------------------------------------------
// Asynchronous window copies (cp.async, 16-byte chunks, zero fill outside).
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, bool valid) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  const int sz = valid ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(sz) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Copies nodes [wx0, wx0+WW) x [wy0, wy0+WH) of a pitched array (rows of P
// elements, P a multiple of 4) into sm (row stride WW).  wx0 and WW are
// multiples of 4, so every chunk is either fully inside a row (possibly in
// its padding, which is never read) or fully outside and zero-filled.
template <typename Real>
__device__ __forceinline__ void load_window(Real* sm, const Real* g, int n, int P, int wx0, int wy0, int WW,
                                            int WH) {
  constexpr int C = 16 / (int)sizeof(Real);
  const int cpr = WW / C;
  for (int i = threadIdx.x; i < cpr * WH; i += kThreads) {
    const int cx = i % cpr, wy = i / cpr;
    const int x = wx0 + cx * C, y = wy0 + wy;
    const bool ok = (y >= 0 && y < n && x >= 0 && x < P);
    const Real* src = ok ? g + (size_t)y * P + x : g;
    cp_async16(sm + wy * WW + cx * C, src, ok);
  }
}

// Tile geometry of a level with n nodes per side and tiles of tx x ty nodes;
// the last tile of a row/column also owns the final node.
struct Tiles {
  int n, tw, th, nx, ny;
  __device__ Tiles(int n_, int tw_ = TX, int th_ = TY) : n(n_), tw(tw_), th(th_) {
    nx = (n - 1) / tw;
    if (nx < 1) nx = 1;
    ny = (n - 1) / th;
    if (ny < 1) ny = 1;
  }
  __device__ int count() const { return nx * ny; }
  __device__ void rect(int t, int& x0, int& x1, int& y0, int& y1) const {
    const int tx = t % nx, ty = t / nx;
    x0 = tx * tw;
    y0 = ty * th;
    x1 = (tx == nx - 1) ? n : x0 + tw;
    y1 = (ty == ny - 1) ? n : y0 + th;
  }
};

// Runs f(x, y) over [0, w) x [0, h) with the CTA's threads laid out as LX x
// (kThreads/LX) lanes (no integer division in the index math).
template <int LX, class F>
__device__ __forceinline__ void for_2d(int w, int h, F&& f) {
  constexpr int LY = kThreads / LX;
  const int lx = threadIdx.x % LX, ly = threadIdx.x / LX;
  for (int y = ly; y < h; y += LY)
    for (int x = lx; x < w; x += LX) f(x, y);
}

// Runs f(x, y) over [0, w) x [0, h), the w*h points spread evenly over the
// CTA's threads.  The row index is a multiply-high by m = floor((2^32-1)/w)+1:
// with m*w = 2^32 + e, 0 <= e < w, the product i*m/2^32 exceeds i/w by less
// than i/2^32 < 1/w for i*w < 2^32, so it floors to i/w exactly.
template <class F>
__device__ __forceinline__ void for_rect(int w, int h, F&& f) {
  const unsigned m = 0xFFFFFFFFu / (unsigned)w + 1u;
  for (int i = threadIdx.x; i < w * h; i += kThreads) {
    const int y = (w == 1) ? i : (int)__umulhi((unsigned)i, m);
    f(i - y * w, y);
  }
}
// Same over two components stacked in y: f(c, x, y) for c in {0, 1}.
template <class F>
__device__ __forceinline__ void for_rect2(int w, int h, F&& f) {
  for_rect(w, 2 * h, [&](int x, int yy) {
    const int c = yy >= h;
    f(c, x, yy - c * h);
  });
}

// ---------------------------------------------------------------------------
template <typename Real>
struct Inst {
  Real* base;
  const Real* R;
  const Real* T;
  const Real* normR;
  double lambda;
  int n, P;
  Real h;
  __device__ Real* arr(size_t off) const { return base + off; }
};

// Energy pass.
//   kind 0: E_data at phi (no direction)            -> part[0]
//            A = phi . L phi over the owned nodes    -> part[1]
//   kind 1: E_data at phi + tau d                   -> part[0]
//   kind 2: NCG materialisation d = s + beta od (d = s when od_zero),
//           E_data at phi + tau d                   -> part[0]
//           Df = DE . d, B = phi . L d, C = d . L d -> part[1..3]
// Windows (EWX x EWY, origin (x0-4, y0-1)) per stage, in this order:
//   kind 0: phx phy R ; kind 1: phx phy dx dy R ; kind 2: phx phy sx sy odx ody R
// (kind 2 reads DE, needed at the owned nodes only, straight from L2).
// Variants of the level kernel, compiled separately so that each carries
// only the passes it runs (registers are allocated for the whole kernel):
// every pass kind (NCC data term, or any mode), the SSD data term in the
// parallel sum order, and the SSD data term with exact sums.
constexpr int kKmAny = 0, kKmSsd = 1, kKmSsdExact = 2;

template <typename Real, int KM = kKmAny>
struct EnergyPass {
  Inst<Real> I;
  int kind;
  Real tau, beta;
  bool od_zero;
  const Real *phx, *phy, *dx, *dy, *sx, *sy, *dex, *dey;
  Real *wdx, *wdy;
  Real* sm;
  int nwin;
  double* part;
  Tiles tl;
  double* xs;   // exact sums: the pass's term buffer (Real = double), or null
  double* xp;   // certified control steps: the instance's per-tile sums, or null
  double (*xpw)[kXpSlots];   // with xp: per warp, the sums of its rows (shared)

  __device__ EnergyPass(const Inst<Real>& I_, int kind_, Real tau_, Real beta_, bool odz, const Real* phx_,
                        const Real* phy_, const Real* dx_, const Real* dy_, const Real* sx_, const Real* sy_,
                        const Real* dex_, const Real* dey_, Real* wdx_, Real* wdy_, Real* sm_, double* part_,
                        double* xs_ = nullptr, double* xp_ = nullptr, double (*xpw_)[kXpSlots] = nullptr)
      : I(I_), kind(kind_), tau(tau_), beta(beta_), od_zero(odz), phx(phx_), phy(phy_), dx(dx_), dy(dy_),
        sx(sx_), sy(sy_), dex(dex_), dey(dey_), wdx(wdx_), wdy(wdy_), sm(sm_), part(part_), tl(I_.n), xs(xs_),
        xp(xp_), xpw(xpw_) {
    nwin = (kind == 0) ? 3 : (kind == 1 ? 5 : 7);
  }
  __device__ Real* win(int stage, int k) const { return sm + ((size_t)stage * nwin + k) * EWIN; }

  __device__ void issue(int t, int stage) {
    int x0, x1, y0, y1;
    tl.rect(t, x0, x1, y0, y1);
    const int wx0 = x0 - 4, wy0 = y0 - 1, n = I.n, P = I.P;
    int k = 0;
    load_window(win(stage, k++), phx, n, P, wx0, wy0, EWX, EWY);
    load_window(win(stage, k++), phy, n, P, wx0, wy0, EWX, EWY);
    if (kind == 1) {
      load_window(win(stage, k++), dx, n, P, wx0, wy0, EWX, EWY);
      load_window(win(stage, k++), dy, n, P, wx0, wy0, EWX, EWY);
    } else if (kind == 2) {
      load_window(win(stage, k++), sx, n, P, wx0, wy0, EWX, EWY);
      load_window(win(stage, k++), sy, n, P, wx0, wy0, EWX, EWY);
      if (!od_zero) {
        load_window(win(stage, k), dx, n, P, wx0, wy0, EWX, EWY);
        load_window(win(stage, k + 1), dy, n, P, wx0, wy0, EWX, EWY);
      }
      k += 2;
    }
    load_window(win(stage, k), I.R, n, P, wx0, wy0, EWX, EWY);
  }

  // Exact-sum variant: the terms of E_data (per element), of phi . L phi at
  // the evaluated position (per node and component) and, for the NCG pass,
  // of DE . d go to the instance's term blocks in the reference's order
  // (msgpu_xsum.cuh); the completing CTA adds them exactly.  The evaluated
  // position newPosition = phi + tau d (gradientDescent.h:176-178) is formed
  // on the whole window first, and E_reg = 1/2 (p_x . L p_x + p_y . L p_y)
  // is evaluated there as DisplacementLengthEnergy does (hyperelastic.h:
  // 178-183), not by the quadratic expansion of the fast path.  With xp the
  // tile also adds up, per warp and term set, the sum of its terms and of
  // their magnitudes (any order: they only bound the ordered sums); the
  // task loop stores the tile's totals after its reduction barrier.
  __device__ void compute_exact(int t, int stage) {
    int x0, x1, y0, y1;
    tl.rect(t, x0, x1, y0, y1);
    const int n = I.n;
    const int wid = threadIdx.x >> 5;
    if (xp && (threadIdx.x & 31) == 0) {
#pragma unroll
      for (int k = 0; k < kXpSlots; ++k) xpw[wid][k] = 0.0;
    }
    Real* Wpx = win(stage, 0);
    Real* Wpy = win(stage, 1);
    const Real* Wr = win(stage, nwin - 1);
    Real* Wa = (kind != 0) ? win(stage, 2) : nullptr;
    Real* Wb = (kind != 0) ? win(stage, 3) : nullptr;
    const Real* Wox = (kind == 2) ? win(stage, 4) : nullptr;
    const Real* Woy = (kind == 2) ? win(stage, 5) : nullptr;
    if (kind != 0) {
      for (int i = threadIdx.x; i < EWIN; i += kThreads) {
        Real ddx = Wa[i], ddy = Wb[i];
        if (kind == 2 && !od_zero) {
          // d = s + beta od (gradientDescent.h:221-229)
          ddx = ddx + beta * Wox[i];
          ddy = ddy + beta * Woy[i];
          Wa[i] = ddx;
          Wb[i] = ddy;
        }
        Real vx = Wpx[i], vy = Wpy[i];
        vx += tau * ddx;
        vy += tau * ddy;
        Wpx[i] = vx;
        Wpy[i] = vy;
      }
      __syncthreads();
    }
    auto at = [&](int x, int y) { return (y - (y0 - 1)) * EWX + (x - (x0 - 4)); };
    const XsGeom g(n);
    const int tx = t % g.nx;
    const int lx = threadIdx.x & 63, ly = threadIdx.x >> 6, half = lx >> 5, lane = threadIdx.x & 31;
    // elements owned by the tile: E_data terms.  A tile has at most 64
    // element columns and 8 element rows, so a thread owns column lx of rows
    // ly and ly + 4; both elements are evaluated together (independent
    // chains), then summed row by row as one row at a time would be.
    {
      const XsSum s0 = xs_sum(xs, n, 0, true);
      double* B0 = xs_block(s0, t);
      const int ex1 = (x1 < n - 1) ? x1 : n - 1, ey1 = (y1 < n - 1) ? y1 : n - 1;
      const int ew = ex1 - x0, eh = ey1 - y0;
      const bool ein = lx < ew;
      auto elem = [&](int ix, int iy) -> double {
        const int ex = x0 + ix, ey = y0 + iy;
        const int c0 = at(ex, ey);
        const int idx[4] = {c0, c0 + 1, c0 + EWX, c0 + EWX + 1};
        Real px[4], py[4], r[4];
#pragma unroll
        for (int b = 0; b < 4; ++b) {
          r[b] = Wr[idx[b]];
          px[b] = Wpx[idx[b]];
          py[b] = Wpy[idx[b]];
        }
        return (double)element_ssd(I.T, n, I.P, I.h, ex, ey, px, py, r);
      };
      // the SSD element integrals are >= 0 (or NaN), so the sum of their
      // magnitudes is the sum itself, added in the same order
      auto row_done = [&](int iy, double acc) {
        acc = warp_sum(acc);
        if (lane == 0) s0.tot[((y0 + iy) * g.nx + tx) * 2 + half] = acc;
        if (xp && lane == 0) {
          xpw[wid][0] += acc;
          xpw[wid][5] += acc;
        }
      };
      if (ly < eh) {
        const int iy = ly, iy2 = ly + 4;
        const bool two = iy2 < eh;
        double acc = 0.0, acc2 = 0.0;
        if (ein) {
          const double v = elem(lx, iy);
          const double v2 = elem(lx, two ? iy2 : iy);
          B0[xs_at(lx, iy)] = v;
          acc += v;
          if (two) {
            B0[xs_at(lx, iy2)] = v2;
            acc2 += v2;
          }
        }
        row_done(iy, acc);
        if (two) row_done(iy2, acc2);
      }
    }
    // owned nodes: p . L p per component; NCG also DE . d and the direction
    {
      const XsSum s1 = xs_sum(xs, n, 1, false), s2 = xs_sum(xs, n, 2, false);
      const XsSum s3 = xs_sum(xs, n, 3, false), s4 = xs_sum(xs, n, 4, false);
      double* B1 = xs_block(s1, t);
      double* B2 = xs_block(s2, t);
      double* B3 = xs_block(s3, t);
      double* B4 = xs_block(s4, t);
      const int nw = x1 - x0, nh = y1 - y0;
      for (int iy = ly; iy < nh; iy += kThreads / 64) {
        double a1 = 0.0, a2 = 0.0, a3 = 0.0, a4 = 0.0;
        double m1 = 0.0, m2 = 0.0, m3 = 0.0, m4 = 0.0;
        for (int ix = lx; ix < nw; ix += 64) {
          const int x = x0 + ix, y = y0 + iy;
          const int c = at(x, y);
          const Real lx_ = stiff_row<Real>(x, y, n, [&](int X, int Y) { return Wpx[at(X, Y)]; });
          const Real ly_ = stiff_row<Real>(x, y, n, [&](int X, int Y) { return Wpy[at(X, Y)]; });
          const double t1 = (double)(Wpx[c] * lx_), t2 = (double)(Wpy[c] * ly_);
          B1[xs_at(ix, iy)] = t1;
          B2[xs_at(ix, iy)] = t2;
          a1 += t1;
          a2 += t2;
          m1 += fabs(t1);
          m2 += fabs(t2);
          if (kind == 2) {
            const Real ddx = Wa[c], ddy = Wb[c];
            const size_t gg = (size_t)y * I.P + x;
            wdx[gg] = ddx;
            wdy[gg] = ddy;
            const double t3 = (double)(__ldcg(dex + gg) * ddx), t4 = (double)(__ldcg(dey + gg) * ddy);
            B3[xs_at(ix, iy)] = t3;
            B4[xs_at(ix, iy)] = t4;
            a3 += t3;
            a4 += t4;
            m3 += fabs(t3);
            m4 += fabs(t4);
          }
        }
        a1 = warp_sum(a1);
        a2 = warp_sum(a2);
        if (kind == 2) {
          a3 = warp_sum(a3);
          a4 = warp_sum(a4);
        }
        if (lane == 0) {
          const int j2 = ((y0 + iy) * g.nx + tx) * 2 + half;
          s1.tot[j2] = a1;
          s2.tot[j2] = a2;
          if (kind == 2) {
            s3.tot[j2] = a3;
            s4.tot[j2] = a4;
          }
        }
        if (xp) {
          m1 = warp_sum(m1);
          m2 = warp_sum(m2);
          if (kind == 2) {
            m3 = warp_sum(m3);
            m4 = warp_sum(m4);
          }
          if (lane == 0) {
            xpw[wid][1] += a1;
            xpw[wid][2] += a2;
            xpw[wid][6] += m1;
            xpw[wid][7] += m2;
            if (kind == 2) {
              xpw[wid][3] += a3;
              xpw[wid][4] += a4;
              xpw[wid][8] += m3;
              xpw[wid][9] += m4;
            }
          }
        }
      }
    }
  }

  __device__ void compute(int t, int stage) {
    if constexpr (KM == kKmSsdExact) {
      compute_exact(t, stage);
      return;
    } else {
      if (KM == kKmAny && xs) {
        compute_exact(t, stage);
        return;
      }
      compute_parallel(t, stage);
    }
  }

  __device__ void compute_parallel(int t, int stage) {
    int x0, x1, y0, y1;
    tl.rect(t, x0, x1, y0, y1);
    const int n = I.n;
    const Real* Wpx = win(stage, 0);
    const Real* Wpy = win(stage, 1);
    const Real* Wr = win(stage, nwin - 1);
    const Real* Wa = (kind != 0) ? win(stage, 2) : nullptr;   // d (kind 1) or s (kind 2)
    const Real* Wb = (kind != 0) ? win(stage, 3) : nullptr;
    const Real* Wox = (kind == 2) ? win(stage, 4) : nullptr;  // od
    const Real* Woy = (kind == 2) ? win(stage, 5) : nullptr;
    auto at = [&](int x, int y) { return (y - (y0 - 1)) * EWX + (x - (x0 - 4)); };
    // direction at a window position
    auto dirx = [&](int i) -> Real {
      if (kind == 1) return Wa[i];
      if (od_zero) return Wa[i];
      return Wa[i] + beta * Wox[i];
    };
    auto diry = [&](int i) -> Real {
      if (kind == 1) return Wb[i];
      if (od_zero) return Wb[i];
      return Wb[i] + beta * Woy[i];
    };
    // elements owned by the tile (at most 64 columns and 8 rows): a thread
    // owns column lx of rows ly and ly + 4, evaluated together and added in
    // that order
    const int ex1 = (x1 < n - 1) ? x1 : n - 1, ey1 = (y1 < n - 1) ? y1 : n - 1;
    const int ew = ex1 - x0, eh = ey1 - y0;
    auto elem = [&](int ix, int iy) -> double {
      const int ex = x0 + ix, ey = y0 + iy;
      const int c0 = at(ex, ey);
      const int idx[4] = {c0, c0 + 1, c0 + EWX, c0 + EWX + 1};
      Real px[4], py[4], r[4];
#pragma unroll
      for (int b = 0; b < 4; ++b) {
        r[b] = Wr[idx[b]];
        if (kind == 0) {
          px[b] = Wpx[idx[b]];
          py[b] = Wpy[idx[b]];
        } else {
          // newPosition = phi + tau * d (gradientDescent.h:176-178)
          Real vx = Wpx[idx[b]], vy = Wpy[idx[b]];
          vx += tau * dirx(idx[b]);
          vy += tau * diry(idx[b]);
          px[b] = vx;
          py[b] = vy;
        }
      }
      return (double)element_ssd(I.T, n, I.P, I.h, ex, ey, px, py, r);
    };
    {
      const int lx = threadIdx.x & 63, ly = threadIdx.x >> 6;
      if (lx < ew && ly < eh) {
        const bool two = ly + 4 < eh;
        const double v = elem(lx, ly);
        const double v2 = elem(lx, two ? ly + 4 : ly);
        part[0] += v;
        if (two) part[0] += v2;
      }
    }
    if (kind == 1) return;
    // owned nodes
    const int nw = x1 - x0, nh = y1 - y0;
    for_2d<64>(nw, nh, [&](int ix, int iy) {
      const int x = x0 + ix, y = y0 + iy;
      const int c = at(x, y);
      if (kind == 0) {
        const Real lx = stiff_row<Real>(x, y, n, [&](int X, int Y) { return Wpx[at(X, Y)]; });
        const Real ly = stiff_row<Real>(x, y, n, [&](int X, int Y) { return Wpy[at(X, Y)]; });
        part[1] += (double)Wpx[c] * (double)lx + (double)Wpy[c] * (double)ly;
      } else {
        const Real ddx = dirx(c), ddy = diry(c);
        const size_t g = (size_t)y * I.P + x;
        wdx[g] = ddx;
        wdy[g] = ddy;
        const Real lx = stiff_row<Real>(x, y, n, [&](int X, int Y) { return dirx(at(X, Y)); });
        const Real ly = stiff_row<Real>(x, y, n, [&](int X, int Y) { return diry(at(X, Y)); });
        part[1] += (double)__ldcg(dex + g) * (double)ddx + (double)__ldcg(dey + g) * (double)ddy;
        part[2] += (double)Wpx[c] * (double)lx + (double)Wpy[c] * (double)ly;
        part[3] += (double)ddx * (double)lx + (double)ddy * (double)ly;
      }
    });
  }
};

// Gradient pass: applies the pending update phi_new = phi + tau_p d (or keeps
// phi), evaluates DE(phi_new) = SSDForce + lambda L phi_new (LinCombOp,
// registration.h:977-982) and A = phi_new . L phi_new -> part[1].  Element
// contributions are staged in shared memory and summed per node in the
// reference's element order (x fastest).
// Windows (EWX x EWY, origin (x0-4, y0-1)): phx phy dx dy R; plus GCY x GCX x 8
// contributions.
template <typename Real>
struct GradPass {
  Inst<Real> I;
  bool step;
  Real tau_p;
  double lambda;
  const Real *phx, *phy, *dx, *dy;
  Real *nphx, *nphy, *dex, *dey;
  Real* sm;
  double* part;
  Tiles tl;
  static constexpr int kWin = 5;

  __device__ GradPass(const Inst<Real>& I_, bool step_, Real tau_p_, double lam, const Real* phx_, const Real* phy_,
                      const Real* dx_, const Real* dy_, Real* nphx_, Real* nphy_, Real* dex_, Real* dey_, Real* sm_,
                      double* part_)
      : I(I_), step(step_), tau_p(tau_p_), lambda(lam), phx(phx_), phy(phy_), dx(dx_), dy(dy_), nphx(nphx_),
        nphy(nphy_), dex(dex_), dey(dey_), sm(sm_), part(part_), tl(I_.n) {}
  __device__ Real* win(int stage, int k) const { return sm + ((size_t)stage * kWin + k) * EWIN; }
  __device__ Real* contrib() const { return sm + (size_t)2 * kWin * EWIN; }

  __device__ void issue(int t, int stage) {
    int x0, x1, y0, y1;
    tl.rect(t, x0, x1, y0, y1);
    const int wx0 = x0 - 4, wy0 = y0 - 1, n = I.n, P = I.P;
    load_window(win(stage, 0), phx, n, P, wx0, wy0, EWX, EWY);
    load_window(win(stage, 1), phy, n, P, wx0, wy0, EWX, EWY);
    if (step) {
      load_window(win(stage, 2), dx, n, P, wx0, wy0, EWX, EWY);
      load_window(win(stage, 3), dy, n, P, wx0, wy0, EWX, EWY);
    }
    load_window(win(stage, 4), I.R, n, P, wx0, wy0, EWX, EWY);
  }

  __device__ void compute(int t, int stage) {
    int x0, x1, y0, y1;
    tl.rect(t, x0, x1, y0, y1);
    const int n = I.n, ne = n - 1;
    Real* Wpx = win(stage, 0);
    Real* Wpy = win(stage, 1);
    const Real* Wdx = win(stage, 2);
    const Real* Wdy = win(stage, 3);
    const Real* Wr = win(stage, 4);
    auto at = [&](int x, int y) { return (y - (y0 - 1)) * EWX + (x - (x0 - 4)); };
    // 1. phi_new in the windows: Dest += tau * d (gradientDescent.h:385-387)
    if (step) {
      for (int i = threadIdx.x; i < EWIN; i += kThreads) {
        Real vx = Wpx[i], vy = Wpy[i];
        vx += tau_p * Wdx[i];
        vy += tau_p * Wdy[i];
        Wpx[i] = vx;
        Wpy[i] = vy;
      }
      __syncthreads();
    }
    // 2. element contributions, elements [x0-1, x1) x [y0-1, y1) that exist
    Real* C = contrib();
    const int cw = (x1 < ne ? x1 : ne) - (x0 - 1), ch = (y1 < ne ? y1 : ne) - (y0 - 1);
    for_rect(cw, ch, [&](int ix, int iy) {
      const int ex = x0 - 1 + ix, ey = y0 - 1 + iy;
      if (ex < 0 || ey < 0) return;
      const int c0 = at(ex, ey);
      const int idx[4] = {c0, c0 + 1, c0 + EWX, c0 + EWX + 1};
      Real px[4], py[4], r[4];
#pragma unroll
      for (int b = 0; b < 4; ++b) {
        px[b] = Wpx[idx[b]];
        py[b] = Wpy[idx[b]];
        r[b] = Wr[idx[b]];
      }
      Real out[4][2];
      element_force(I.T, n, I.P, I.h, ex, ey, px, py, r, out);
      Real* cc = C + ((size_t)(ey - (y0 - 1)) * GCX + (ex - (x0 - 1))) * 8;
#pragma unroll
      for (int b = 0; b < 4; ++b) {
        cc[2 * b] = out[b][0];
        cc[2 * b + 1] = out[b][1];
      }
    });
    __syncthreads();
    // 3. node sums in element order, stiffness, outputs
    const Real lam = (Real)lambda;
    const int nw = x1 - x0, nh = y1 - y0;
    for_2d<64>(nw, nh, [&](int ix, int iy) {
      const int x = x0 + ix, y = y0 + iy;
      auto cc = [&](int ex, int ey, int b, int comp) {
        return C[((size_t)(ey - (y0 - 1)) * GCX + (ex - (x0 - 1))) * 8 + 2 * b + comp];
      };
      Real fx = Real(0), fy = Real(0);
      if (x - 1 >= 0 && y - 1 >= 0) { fx += cc(x - 1, y - 1, 3, 0); fy += cc(x - 1, y - 1, 3, 1); }
      if (x < ne && y - 1 >= 0)     { fx += cc(x, y - 1, 2, 0);     fy += cc(x, y - 1, 2, 1); }
      if (x - 1 >= 0 && y < ne)     { fx += cc(x - 1, y, 1, 0);     fy += cc(x - 1, y, 1, 1); }
      if (x < ne && y < ne)         { fx += cc(x, y, 0, 0);         fy += cc(x, y, 0, 1); }
      const Real Lx = stiff_row<Real>(x, y, n, [&](int X, int Y) { return Wpx[at(X, Y)]; });
      const Real Ly = stiff_row<Real>(x, y, n, [&](int X, int Y) { return Wpy[at(X, Y)]; });
      const Real gx = (lambda != 1.0) ? fx + lam * Lx : fx + Lx;
      const Real gy = (lambda != 1.0) ? fy + lam * Ly : fy + Ly;
      const size_t g = (size_t)y * I.P + x;
      dex[g] = gx;
      dey[g] = gy;
      const Real vx = Wpx[at(x, y)], vy = Wpy[at(x, y)];
      nphx[g] = vx;
      nphy[g] = vy;
      part[1] += (double)vx * (double)Lx + (double)vy * (double)Ly;
    });
  }
};

// ---------------------------------------------------------------------------
// Normalized cross-correlation data term (NormalizedCrossCorrelationEnergy,
// registration.h:1909-1983).  One energy evaluation is three passes, each
// followed by a global sum:
//   sub 1: Td = FastDeformImage(T, p) at the nodes, sum_i (M Td)_i   (mean)
//   sub 2: u = Td - mean,                     sum_i u_i (M u)_i      (var^2)
//   sub 3: normT = u / var,                   sum_i (M normT)_i normR_i
// and E_ncc = -(last sum) (normalizeImageForNCC, computeEnergy,
// registration.h:1932-1962).  The position p of sub 1 depends on the purpose:
//   E0:   p = phi; also A = phi . L phi                     -> part[1]
//   GRAD: p = phi + tau_p d (pending step), written to nphi
//   TRIAL: p = phi + tau d
//   NCG:  d = s + beta od materialised (written), p = phi + tau d,
//         Df = DE . d, B = phi . L d, C = d . L d           -> part[1..3]
// Windows (EWX x EWY, origin (x0-4, y0-1)) per stage: sub 1 as the energy
// passes (phx phy [dx dy | sx sy odx ody]); sub 2: Td; sub 3: Td normR.
// Work window: Td (sub 1) or u / normT (subs 2, 3).
enum NccMode : int { NM_E0 = 0, NM_GRAD, NM_TRIAL, NM_NCG };

template <typename Real>
struct NccPass {
  Inst<Real> I;
  int sub, mode;
  Real tau, beta;
  double mean, var;
  bool od_zero, step;
  const Real *phx, *phy, *dx, *dy, *sx, *sy, *dex, *dey, *normR;
  Real *wdx, *wdy, *nphx, *nphy, *td;
  Real* sm;
  int nwin;
  double* part;
  Tiles tl;

  __device__ NccPass(const Inst<Real>& I_, int sub_, int mode_, Real tau_, Real beta_, double mean_, double var_,
                     bool odz, bool step_, const Real* phx_, const Real* phy_, const Real* dx_, const Real* dy_,
                     const Real* sx_, const Real* sy_, const Real* dex_, const Real* dey_, const Real* normR_,
                     Real* wdx_, Real* wdy_, Real* nphx_, Real* nphy_, Real* td_, Real* sm_, double* part_)
      : I(I_), sub(sub_), mode(mode_), tau(tau_), beta(beta_), mean(mean_), var(var_), od_zero(odz), step(step_),
        phx(phx_), phy(phy_), dx(dx_), dy(dy_), sx(sx_), sy(sy_), dex(dex_), dey(dey_), normR(normR_), wdx(wdx_),
        wdy(wdy_), nphx(nphx_), nphy(nphy_), td(td_), sm(sm_), part(part_), tl(I_.n) {
    if (sub == 1) nwin = (mode == NM_NCG) ? 6 : ((mode == NM_TRIAL || (mode == NM_GRAD && step)) ? 4 : 2);
    else nwin = (sub == 2) ? 1 : 2;
  }
  __device__ Real* win(int stage, int k) const { return sm + ((size_t)stage * nwin + k) * EWIN; }
  __device__ Real* work() const { return sm + (size_t)2 * nwin * EWIN; }

  __device__ void issue(int t, int stage) {
    int x0, x1, y0, y1;
    tl.rect(t, x0, x1, y0, y1);
    const int wx0 = x0 - 4, wy0 = y0 - 1, n = I.n, P = I.P;
    if (sub == 1) {
      load_window(win(stage, 0), phx, n, P, wx0, wy0, EWX, EWY);
      load_window(win(stage, 1), phy, n, P, wx0, wy0, EWX, EWY);
      if (mode == NM_TRIAL || (mode == NM_GRAD && step)) {
        load_window(win(stage, 2), dx, n, P, wx0, wy0, EWX, EWY);
        load_window(win(stage, 3), dy, n, P, wx0, wy0, EWX, EWY);
      } else if (mode == NM_NCG) {
        load_window(win(stage, 2), sx, n, P, wx0, wy0, EWX, EWY);
        load_window(win(stage, 3), sy, n, P, wx0, wy0, EWX, EWY);
        if (!od_zero) {
          load_window(win(stage, 4), dx, n, P, wx0, wy0, EWX, EWY);
          load_window(win(stage, 5), dy, n, P, wx0, wy0, EWX, EWY);
        }
      }
    } else {
      load_window(win(stage, 0), td, n, P, wx0, wy0, EWX, EWY);
      if (sub == 3) load_window(win(stage, 1), normR, n, P, wx0, wy0, EWX, EWY);
    }
  }

  __device__ void compute(int t, int stage) {
    int x0, x1, y0, y1;
    tl.rect(t, x0, x1, y0, y1);
    const int n = I.n, P = I.P;
    const Real hh = I.h * I.h, inv_h = Real(n - 1);
    auto at = [&](int x, int y) { return (y - (y0 - 1)) * EWX + (x - (x0 - 4)); };
    Real* W = work();
    // nodes of the tile and a one-node halo (the mass stencil's support)
    const int hx0 = max(x0 - 1, 0), hx1 = min(x1 + 1, n), hy0 = max(y0 - 1, 0), hy1 = min(y1 + 1, n);
    if (sub == 1) {
      const Real* Wpx = win(stage, 0);
      const Real* Wpy = win(stage, 1);
      const Real* Wa = (nwin >= 4) ? win(stage, 2) : nullptr;
      const Real* Wb = (nwin >= 4) ? win(stage, 3) : nullptr;
      const Real* Wox = (mode == NM_NCG) ? win(stage, 4) : nullptr;
      const Real* Woy = (mode == NM_NCG) ? win(stage, 5) : nullptr;
      const bool moves = (mode == NM_TRIAL || mode == NM_NCG || (mode == NM_GRAD && step));
      auto dirx = [&](int i) -> Real {
        if (mode != NM_NCG || od_zero) return Wa[i];
        return Wa[i] + beta * Wox[i];
      };
      auto diry = [&](int i) -> Real {
        if (mode != NM_NCG || od_zero) return Wb[i];
        return Wb[i] + beta * Woy[i];
      };
      for_rect(hx1 - hx0, hy1 - hy0, [&](int ix, int iy) {
        const int x = hx0 + ix, y = hy0 + iy;
        const int c = at(x, y);
        Real vx = Wpx[c], vy = Wpy[c];
        if (moves) {
          // newPosition = phi + tau * d (gradientDescent.h:176-178, 385-387)
          vx += tau * dirx(c);
          vy += tau * diry(c);
        }
        W[c] = fast_deform_node(I.T, n, P, x, y, vx, vy, inv_h);
        if (x >= x0 && x < x1 && y >= y0 && y < y1) {
          const size_t g = (size_t)y * P + x;
          td[g] = W[c];
          if (mode == NM_GRAD) {
            nphx[g] = vx;
            nphy[g] = vy;
          }
        }
      });
      __syncthreads();
      for_2d<64>(x1 - x0, y1 - y0, [&](int ix, int iy) {
        const int x = x0 + ix, y = y0 + iy;
        const int c = at(x, y);
        part[0] += (double)mass_row<Real>(x, y, n, hh, [&](int X, int Y) { return W[at(X, Y)]; });
        if (mode == NM_E0) {
          const Real lx = stiff_row<Real>(x, y, n, [&](int X, int Y) { return Wpx[at(X, Y)]; });
          const Real ly = stiff_row<Real>(x, y, n, [&](int X, int Y) { return Wpy[at(X, Y)]; });
          part[1] += (double)Wpx[c] * (double)lx + (double)Wpy[c] * (double)ly;
        } else if (mode == NM_NCG) {
          const Real ddx = dirx(c), ddy = diry(c);
          const size_t g = (size_t)y * P + x;
          wdx[g] = ddx;
          wdy[g] = ddy;
          const Real lx = stiff_row<Real>(x, y, n, [&](int X, int Y) { return dirx(at(X, Y)); });
          const Real ly = stiff_row<Real>(x, y, n, [&](int X, int Y) { return diry(at(X, Y)); });
          part[1] += (double)__ldcg(dex + g) * (double)ddx + (double)__ldcg(dey + g) * (double)ddy;
          part[2] += (double)Wpx[c] * (double)lx + (double)Wpy[c] * (double)ly;
          part[3] += (double)ddx * (double)lx + (double)ddy * (double)ly;
        }
      });
      return;
    }
    // subs 2 and 3: u = Td + (-mean) (addToAll), normT = u / var
    const Real* Wt = win(stage, 0);
    const Real m = (Real)(-mean), vr = (Real)var;
    const bool divide = !(fabs(var - 0.0) < 1e-15);  // aol::appeqAbsolute (aol.h:791-794)
    for_rect(hx1 - hx0, hy1 - hy0, [&](int ix, int iy) {
      const int c = at(hx0 + ix, hy0 + iy);
      Real u = Wt[c];
      u += m;
      if (sub == 3 && divide) u /= vr;
      W[c] = u;
    });
    __syncthreads();
    const Real* Wr = (sub == 3) ? win(stage, 1) : nullptr;
    for_2d<64>(x1 - x0, y1 - y0, [&](int ix, int iy) {
      const int x = x0 + ix, y = y0 + iy;
      const int c = at(x, y);
      const Real mu = mass_row<Real>(x, y, n, hh, [&](int X, int Y) { return W[at(X, Y)]; });
      if (sub == 2) part[0] += (double)(W[c] * mu);
      else part[0] += (double)(mu * Wr[c]);
    });
  }
};

// Variation of the NCC energy at phi (applyDerivative, registration.h:
// 1972-1983): temp = (normR + E normT) / var, CrossCorrelationForce with
// temp as the weight (registration.h:1828-1862), plus lambda L phi; the
// force contributions are staged per element and summed per node in the
// reference's element order (as the SSD gradient pass).  A = phi . L phi ->
// part[1].  Windows per stage: phx phy Td normR; work: temp window and
// GCY x GCX x 8 contributions.
template <typename Real>
struct NccForcePass {
  Inst<Real> I;
  double lambda, mean, var, energy;
  const Real *phx, *phy, *td, *normR;
  Real *dex, *dey;
  Real* sm;
  double* part;
  Tiles tl;
  static constexpr int kWin = 4;

  __device__ NccForcePass(const Inst<Real>& I_, double lam, double mean_, double var_, double e_, const Real* phx_,
                          const Real* phy_, const Real* td_, const Real* normR_, Real* dex_, Real* dey_, Real* sm_,
                          double* part_)
      : I(I_), lambda(lam), mean(mean_), var(var_), energy(e_), phx(phx_), phy(phy_), td(td_), normR(normR_),
        dex(dex_), dey(dey_), sm(sm_), part(part_), tl(I_.n) {}
  __device__ Real* win(int stage, int k) const { return sm + ((size_t)stage * kWin + k) * EWIN; }
  __device__ Real* tmpw() const { return sm + (size_t)2 * kWin * EWIN; }
  __device__ Real* contrib() const { return sm + (size_t)(2 * kWin + 1) * EWIN; }

  __device__ void issue(int t, int stage) {
    int x0, x1, y0, y1;
    tl.rect(t, x0, x1, y0, y1);
    const int wx0 = x0 - 4, wy0 = y0 - 1, n = I.n, P = I.P;
    load_window(win(stage, 0), phx, n, P, wx0, wy0, EWX, EWY);
    load_window(win(stage, 1), phy, n, P, wx0, wy0, EWX, EWY);
    load_window(win(stage, 2), td, n, P, wx0, wy0, EWX, EWY);
    load_window(win(stage, 3), normR, n, P, wx0, wy0, EWX, EWY);
  }

  __device__ void compute(int t, int stage) {
    int x0, x1, y0, y1;
    tl.rect(t, x0, x1, y0, y1);
    const int n = I.n, ne = n - 1;
    const Real* Wpx = win(stage, 0);
    const Real* Wpy = win(stage, 1);
    const Real* Wt = win(stage, 2);
    const Real* Wr = win(stage, 3);
    Real* Wm = tmpw();
    auto at = [&](int x, int y) { return (y - (y0 - 1)) * EWX + (x - (x0 - 4)); };
    // 1. temp on the nodes of the elements [x0-1, x1) x [y0-1, y1)
    {
      const Real m = (Real)(-mean), vr = (Real)var, e = (Real)energy;
      const bool divide = !(fabs(var - 0.0) < 1e-15);
      const int hx0 = max(x0 - 1, 0), hx1 = min(x1 + 1, n), hy0 = max(y0 - 1, 0), hy1 = min(y1 + 1, n);
      for_rect(hx1 - hx0, hy1 - hy0, [&](int ix, int iy) {
        const int c = at(hx0 + ix, hy0 + iy);
        Real nt = Wt[c];
        nt += m;
        if (divide) nt /= vr;
        Real v = Wr[c];
        v += nt * e;                 // addMultiple (vec.cpp:768-777)
        if (divide) v /= vr;
        Wm[c] = v;
      });
    }
    __syncthreads();
    // 2. element contributions
    Real* C = contrib();
    const int cw = (x1 < ne ? x1 : ne) - (x0 - 1), ch = (y1 < ne ? y1 : ne) - (y0 - 1);
    for_rect(cw, ch, [&](int ix, int iy) {
      const int ex = x0 - 1 + ix, ey = y0 - 1 + iy;
      if (ex < 0 || ey < 0) return;
      const int c0 = at(ex, ey);
      const int idx[4] = {c0, c0 + 1, c0 + EWX, c0 + EWX + 1};
      Real px[4], py[4], tm[4];
#pragma unroll
      for (int b = 0; b < 4; ++b) {
        px[b] = Wpx[idx[b]];
        py[b] = Wpy[idx[b]];
        tm[b] = Wm[idx[b]];
      }
      Real out[4][2];
      element_ncc_force(I.T, n, I.P, I.h, ex, ey, px, py, tm, out);
      Real* cc = C + ((size_t)(ey - (y0 - 1)) * GCX + (ex - (x0 - 1))) * 8;
#pragma unroll
      for (int b = 0; b < 4; ++b) {
        cc[2 * b] = out[b][0];
        cc[2 * b + 1] = out[b][1];
      }
    });
    __syncthreads();
    // 3. node sums in element order, stiffness, outputs
    const Real lam = (Real)lambda;
    for_2d<64>(x1 - x0, y1 - y0, [&](int ix, int iy) {
      const int x = x0 + ix, y = y0 + iy;
      auto cc = [&](int ex, int ey, int b, int comp) {
        return C[((size_t)(ey - (y0 - 1)) * GCX + (ex - (x0 - 1))) * 8 + 2 * b + comp];
      };
      Real fx = Real(0), fy = Real(0);
      if (x - 1 >= 0 && y - 1 >= 0) { fx += cc(x - 1, y - 1, 3, 0); fy += cc(x - 1, y - 1, 3, 1); }
      if (x < ne && y - 1 >= 0)     { fx += cc(x, y - 1, 2, 0);     fy += cc(x, y - 1, 2, 1); }
      if (x - 1 >= 0 && y < ne)     { fx += cc(x - 1, y, 1, 0);     fy += cc(x - 1, y, 1, 1); }
      if (x < ne && y < ne)         { fx += cc(x, y, 0, 0);         fy += cc(x, y, 0, 1); }
      const Real Lx = stiff_row<Real>(x, y, n, [&](int X, int Y) { return Wpx[at(X, Y)]; });
      const Real Ly = stiff_row<Real>(x, y, n, [&](int X, int Y) { return Wpy[at(X, Y)]; });
      const Real gx = (lambda != 1.0) ? fx + lam * Lx : fx + Lx;
      const Real gy = (lambda != 1.0) ? fy + lam * Ly : fy + Ly;
      const size_t g = (size_t)y * I.P + x;
      dex[g] = gx;
      dey[g] = gy;
      part[1] += (double)Wpx[at(x, y)] * (double)Lx + (double)Wpy[at(x, y)] * (double)Ly;
    });
  }
};

// ---------------------------------------------------------------------------
// Multigrid V-cycle passes on the levels above lc (tiled passes).

// Pre-smoothing (2 Jacobi sweeps from x = 0), residual and restriction
// (MDMultigrid::solve steps 1-3, linearSmoothOp.cpp:465-477).
// rhs = sgn * window (sgn = -1 turns DE into the descent direction).
// Staged windows (VWX x VWY, origin (x0-4, y0-3)): rhs_x rhs_y; work: x2[2] r[2] x1[2].
template <typename Real>
struct DownPass {
  int n, P, cw, cP;
  const Real *rx, *ry;
  Real sgn;
  Real *x2x, *x2y, *bcx, *bcy;
  Real hsq, diag;
  Real* sm;
  Tiles tl;
  __device__ DownPass(int n_, const Real* rx_, const Real* ry_, Real sgn_, Real* x2x_, Real* x2y_, Real* bcx_,
                      Real* bcy_, Real hsq_, Real diag_, Real* sm_)
      : n(n_), P(pitch_of(n_)), cw((n_ >> 1) + 1), cP(pitch_of((n_ >> 1) + 1)), rx(rx_), ry(ry_), sgn(sgn_),
        x2x(x2x_), x2y(x2y_), bcx(bcx_), bcy(bcy_), hsq(hsq_), diag(diag_), sm(sm_), tl(n_, VTX, VTY) {}
  __device__ Real* rhs(int stage, int c) const { return sm + ((size_t)stage * 2 + c) * VWIN; }
  __device__ Real* work(int k, int c) const { return sm + ((size_t)4 + 2 * k + c) * VWIN; }

  __device__ void issue(int t, int stage) {
    int x0, x1, y0, y1;
    tl.rect(t, x0, x1, y0, y1);
    load_window(rhs(stage, 0), rx, n, P, x0 - 4, y0 - 3, VWX, VWY);
    load_window(rhs(stage, 1), ry, n, P, x0 - 4, y0 - 3, VWX, VWY);
  }

  __device__ void compute(int t, int stage) {
    int x0, x1, y0, y1;
    tl.rect(t, x0, x1, y0, y1);
    auto at = [&](int x, int y) { return (y - (y0 - 3)) * VWX + (x - (x0 - 4)); };
    // rhs sign and x1 = 0 + (rhs - A 0)/diag on the whole window (one division per node)
    for (int i = threadIdx.x; i < 2 * VWIN; i += kThreads) {
      const int c = i / VWIN, j = i % VWIN;
      const Real r = rhs(stage, c)[j] * sgn;
      rhs(stage, c)[j] = r;
      work(2, c)[j] = jacobi_update(Real(0), r, Real(0), diag);
    }
    __syncthreads();
    // x2 on nodes [x0-2, x1+2) x [y0-2, y1+2)
    {
      const int ax0 = max(x0 - 2, 0), ax1 = min(x1 + 2, n), ay0 = max(y0 - 2, 0), ay1 = min(y1 + 2, n);
      const int w = ax1 - ax0, h = ay1 - ay0;
      for_rect2(w, h, [&](int c, int ix, int iy) {
        const int x = ax0 + ix, y = ay0 + iy;
        const Real* X1 = work(2, c);
        const Real ax = heat_row<Real>(x, y, n, hsq, [&](int a, int b) { return X1[at(a, b)]; });
        work(0, c)[at(x, y)] = jacobi_update(X1[at(x, y)], rhs(stage, c)[at(x, y)], ax, diag);
      });
    }
    __syncthreads();
    // residual on nodes [x0-1, x1+1) x [y0-1, y1+1); x2 out for owned nodes
    {
      const int ax0 = max(x0 - 1, 0), ax1 = min(x1 + 1, n), ay0 = max(y0 - 1, 0), ay1 = min(y1 + 1, n);
      const int w = ax1 - ax0, h = ay1 - ay0;
      for_rect2(w, h, [&](int c, int ix, int iy) {
        const int x = ax0 + ix, y = ay0 + iy;
        const Real* X2 = work(0, c);
        const Real ax = heat_row<Real>(x, y, n, hsq, [&](int a, int b) { return X2[at(a, b)]; });
        work(1, c)[at(x, y)] = rhs(stage, c)[at(x, y)] - ax;
        if (x >= x0 && x < x1 && y >= y0 && y < y1) (c == 0 ? x2x : x2y)[(size_t)y * P + x] = X2[at(x, y)];
      });
    }
    __syncthreads();
    // restriction to the coarse nodes centred in the tile
    {
      const int X0 = x0 >> 1, X1 = (x1 + 1) >> 1, Y0 = y0 >> 1, Y1 = (y1 + 1) >> 1;
      const int w = X1 - X0, h = Y1 - Y0;
      for_rect2(w, h, [&](int c, int ix, int iy) {
        const int X = X0 + ix, Y = Y0 + iy;
        const Real* Rs = work(1, c);
        const Real v = restrict_node<Real>(X, Y, cw, [&](int x, int y) { return Rs[at(x, y)]; });
        (c == 0 ? bcx : bcy)[(size_t)Y * cP + X] = v;
      });
    }
  }
};

// Correction and post-smoothing (MDMultigrid::solve steps 5-6,
// linearSmoothOp.cpp:483-493): x3 = x2 + P x_coarse, then 2 Jacobi sweeps.
// Staged windows: rhs_x rhs_y x2_x x2_y (VWX x VWY, origin (x0-4, y0-3)) and
// xc_x xc_y (CWX x CWY, origin (x0/2-4, y0/2-2)); work: x4[2].  x0/2 is a
// multiple of 16, so the coarse window starts on a 16-byte boundary.
template <typename Real>
struct UpPass {
  int n, P, cw, cP;
  const Real *rx, *ry, *x2x, *x2y, *xcx, *xcy;
  Real sgn;
  Real *ox, *oy;
  Real hsq, diag;
  Real* sm;
  bool want_norm;
  double* part;
  Tiles tl;
  double* xs;   // exact sums of |s|^2 (want_norm, Real = double), or null
  static constexpr size_t kStage = 4 * VWIN + 2 * CWIN;
  __device__ UpPass(int n_, const Real* rx_, const Real* ry_, Real sgn_, const Real* x2x_, const Real* x2y_,
                    const Real* xcx_, const Real* xcy_, Real* ox_, Real* oy_, Real hsq_, Real diag_, Real* sm_,
                    bool wn, double* part_, double* xs_ = nullptr)
      : n(n_), P(pitch_of(n_)), cw((n_ >> 1) + 1), cP(pitch_of((n_ >> 1) + 1)), rx(rx_), ry(ry_), x2x(x2x_),
        x2y(x2y_), xcx(xcx_), xcy(xcy_), sgn(sgn_), ox(ox_), oy(oy_), hsq(hsq_), diag(diag_), sm(sm_),
        want_norm(wn), part(part_), tl(n_, VTX, VTY), xs(xs_) {}
  __device__ Real* rhs(int stage, int c) const { return sm + stage * kStage + (size_t)c * VWIN; }
  __device__ Real* x2(int stage, int c) const { return sm + stage * kStage + (size_t)(2 + c) * VWIN; }
  __device__ Real* xc(int stage, int c) const { return sm + stage * kStage + 4 * VWIN + (size_t)c * CWIN; }
  __device__ Real* x4(int c) const { return sm + 2 * kStage + (size_t)c * VWIN; }

  __device__ void issue(int t, int stage) {
    int x0, x1, y0, y1;
    tl.rect(t, x0, x1, y0, y1);
    load_window(rhs(stage, 0), rx, n, P, x0 - 4, y0 - 3, VWX, VWY);
    load_window(rhs(stage, 1), ry, n, P, x0 - 4, y0 - 3, VWX, VWY);
    load_window(x2(stage, 0), x2x, n, P, x0 - 4, y0 - 3, VWX, VWY);
    load_window(x2(stage, 1), x2y, n, P, x0 - 4, y0 - 3, VWX, VWY);
    load_window(xc(stage, 0), xcx, cw, cP, (x0 >> 1) - 4, (y0 >> 1) - 2, CWX, CWY);
    load_window(xc(stage, 1), xcy, cw, cP, (x0 >> 1) - 4, (y0 >> 1) - 2, CWX, CWY);
  }

  __device__ void compute(int t, int stage) {
    int x0, x1, y0, y1;
    tl.rect(t, x0, x1, y0, y1);
    auto at = [&](int x, int y) { return (y - (y0 - 3)) * VWX + (x - (x0 - 4)); };
    auto atc = [&](int X, int Y) { return (Y - ((y0 >> 1) - 2)) * CWX + (X - ((x0 >> 1) - 4)); };
    // x3 = x2 + P xc in place on nodes [x0-2, x1+2) x [y0-2, y1+2)
    {
      const int ax0 = max(x0 - 2, 0), ax1 = min(x1 + 2, n), ay0 = max(y0 - 2, 0), ay1 = min(y1 + 2, n);
      const int w = ax1 - ax0, h = ay1 - ay0;
      for_rect2(w, h, [&](int c, int ix, int iy) {
        const int x = ax0 + ix, y = ay0 + iy;
        const Real* XC = xc(stage, c);
        const Real p = prolong_node<Real>(x, y, [&](int X, int Y) { return XC[atc(X, Y)]; });
        x2(stage, c)[at(x, y)] = x2(stage, c)[at(x, y)] + p;
      });
    }
    __syncthreads();
    // x4 on nodes [x0-1, x1+1) x [y0-1, y1+1)
    {
      const int ax0 = max(x0 - 1, 0), ax1 = min(x1 + 1, n), ay0 = max(y0 - 1, 0), ay1 = min(y1 + 1, n);
      const int w = ax1 - ax0, h = ay1 - ay0;
      for_rect2(w, h, [&](int c, int ix, int iy) {
        const int x = ax0 + ix, y = ay0 + iy;
        const Real* X3 = x2(stage, c);
        const Real ax = heat_row<Real>(x, y, n, hsq, [&](int a, int b) { return X3[at(a, b)]; });
        x4(c)[at(x, y)] = jacobi_update(X3[at(x, y)], rhs(stage, c)[at(x, y)] * sgn, ax, diag);
      });
    }
    __syncthreads();
    // x5 on the owned nodes
    if (xs && want_norm) {
      // the smoothed direction s and the terms s_c * s_c of |s|^2 = s_x . s_x +
      // s_y . s_y (gradientDescent.h:221-226), node sums of the element-pass
      // geometry: a 32-wide tile is one half of a 64-wide chunk
      const int w = x1 - x0, h = y1 - y0;
      const XsGeom g(n);
      const XsSum s0 = xs_sum(xs, n, 0, false), s1 = xs_sum(xs, n, 1, false);
      const int txE = x0 / 64, kb = x0 - txE * 64, half = (x0 >> 5) & 1;
      const bool whole = (tl.nx == 1);   // this tile covers its chunk: no second half
      const int lx = threadIdx.x & 31, ly = threadIdx.x >> 5;
      for (int iy = ly; iy < h; iy += kThreads / 32) {
        const int y = y0 + iy;
        int tyE = y / 8;
        if (tyE > g.ny - 1) tyE = g.ny - 1;
        const int r = y - tyE * 8;
        double* B0 = xs_block(s0, tyE * g.nx + txE);
        double* B1 = xs_block(s1, tyE * g.nx + txE);
        double a0 = 0.0, a1 = 0.0;
        for (int ix = lx; ix < w; ix += 32) {
          const int x = x0 + ix;
          Real o[2];
#pragma unroll
          for (int c = 0; c < 2; ++c) {
            const Real* X4 = x4(c);
            const Real ax = heat_row<Real>(x, y, n, hsq, [&](int a, int b) { return X4[at(a, b)]; });
            o[c] = jacobi_update(X4[at(x, y)], rhs(stage, c)[at(x, y)] * sgn, ax, diag);
          }
          const size_t gg = (size_t)y * P + x;
          ox[gg] = o[0];
          oy[gg] = o[1];
          const double t0 = (double)(o[0] * o[0]), t1 = (double)(o[1] * o[1]);
          B0[xs_at(kb + ix, r)] = t0;
          B1[xs_at(kb + ix, r)] = t1;
          a0 += t0;
          a1 += t1;
        }
        a0 = warp_sum(a0);
        a1 = warp_sum(a1);
        if (lx == 0) {
          const int j = y * g.nx + txE;
          s0.tot[2 * j + half] = a0;
          s1.tot[2 * j + half] = a1;
          if (whole) {
            s0.tot[2 * j + 1] = 0.0;
            s1.tot[2 * j + 1] = 0.0;
          }
        }
      }
    } else {
      const int w = x1 - x0, h = y1 - y0;
      for_rect(w, h, [&](int ix, int iy) {
        const int x = x0 + ix, y = y0 + iy;
        Real o[2];
#pragma unroll
        for (int c = 0; c < 2; ++c) {
          const Real* X4 = x4(c);
          const Real ax = heat_row<Real>(x, y, n, hsq, [&](int a, int b) { return X4[at(a, b)]; });
          o[c] = jacobi_update(X4[at(x, y)], rhs(stage, c)[at(x, y)] * sgn, ax, diag);
        }
        const size_t g = (size_t)y * P + x;
        ox[g] = o[0];
        oy[g] = o[1];
        if (want_norm) part[0] += (double)o[0] * (double)o[0] + (double)o[1] * (double)o[1];
      });
    }
  }
};

// Coarse part of the V-cycle, levels lc..0, by one CTA in shared memory
// (MDMultigrid::solve recursion including the 100 sweeps on level 0,
// linearSmoothOp.cpp:451-494, 556-580).
// Layout per level k (dense, width w = 2^k+1): slots 0/1 hold the iterate
// (ping-pong), slot 2 the right-hand side, each with two components.
// The offset of level k is sum_{j<k} 6 (2^j+1)^2 = 2(4^k-1) + 12(2^k-1) + 6k.
__host__ __device__ inline size_t coarse_level_offset(int k) {
  return (size_t)2 * ((1u << (2 * k)) - 1u) + (size_t)12 * ((1u << k) - 1u) + (size_t)6 * k;
}
__host__ __device__ inline size_t coarse_smem_elems(int lc) { return coarse_level_offset(lc + 1); }

template <typename Real>
struct Coarse {
  Real* sm;
  double tau;
  unsigned cur = 0;  // bit k: slot holding the iterate of level k
  __device__ Real* S(int k, int slot, int c) const {
    const int w = (1 << k) + 1;
    return sm + coarse_level_offset(k) + (size_t)(2 * slot + c) * (size_t)(w * w);
  }
  __device__ int slot(int k) const { return (int)((cur >> k) & 1u); }
  __device__ Real hsq(int k) const {
    const int w = (1 << k) + 1;
    return (Real)(tau * (double)((w - 1) * (w - 1)));
  }
  __device__ Real diag(int k) const {
    const int w = (1 << k) + 1;
    return (Real)(1 + 4 * tau * (double)((w - 1) * (w - 1)));
  }

  // One Jacobi sweep (HeatMultigrid::jacobi) on level k; the items are
  // (component, node) pairs, components stacked in y.
  __device__ void sweep(int k) {
    const int w = (1 << k) + 1, s = slot(k);
    const Real h2 = hsq(k), dg = diag(k);
    for_rect(w, 2 * w, [&](int x, int yy) {
      const int c = yy >= w, y = yy - c * w, id = y * w + x;
      const Real* xs = S(k, s, c);
      const Real a = heat_row<Real>(x, y, w, h2, [&](int i, int j) { return xs[j * w + i]; });
      S(k, s ^ 1, c)[id] = jacobi_update(xs[id], S(k, 2, c)[id], a, dg);
    });
    cur ^= 1u << k;
    __syncthreads();
  }

  // Second pre-sweep, residual, restriction to level k-1 and (k-1 >= 1) the
  // first pre-sweep of level k-1 from x = 0, where A 0 is exactly +0.
  __device__ void down(int k) {
    sweep(k);
    const int w = (1 << k) + 1, cw = (1 << (k - 1)) + 1, s = slot(k);
    const Real h2 = hsq(k);
    for_rect(w, 2 * w, [&](int x, int yy) {
      const int c = yy >= w, y = yy - c * w, id = y * w + x;
      const Real* xs = S(k, s, c);
      const Real a = heat_row<Real>(x, y, w, h2, [&](int i, int j) { return xs[j * w + i]; });
      S(k, s ^ 1, c)[id] = S(k, 2, c)[id] - a;
    });
    __syncthreads();
    const Real cdg = diag(k - 1);
    const bool first_sweep = (k - 1 >= 1);
    for_rect(cw, 2 * cw, [&](int X, int YY) {
      const int c = YY >= cw, Y = YY - c * cw, id = Y * cw + X;
      const Real* rs = S(k, s ^ 1, c);
      const Real v = restrict_node<Real>(X, Y, cw, [&](int i, int j) { return rs[j * w + i]; });
      S(k - 1, 2, c)[id] = v;
      if (first_sweep) S(k - 1, 0, c)[id] = jacobi_update(Real(0), v, Real(0), cdg);
    });
    cur &= ~(1u << (k - 1));  // level k-1 iterate in slot 0
    __syncthreads();
  }

  // Correction x3 = x2 + P x_coarse, then the two post-sweeps.
  __device__ void up(int k) {
    const int w = (1 << k) + 1, cw = (1 << (k - 1)) + 1, s = slot(k), sc = slot(k - 1);
    for_rect(w, 2 * w, [&](int x, int yy) {
      const int c = yy >= w, y = yy - c * w, id = y * w + x;
      const Real* xc = S(k - 1, sc, c);
      const Real p = prolong_node<Real>(x, y, [&](int X, int Y) { return xc[Y * cw + X]; });
      S(k, s, c)[id] += p;
    });
    __syncthreads();
    sweep(k);
    sweep(k);
  }

  // Level 0 (2 x 2 nodes, all corners): 100 sweeps from x = 0 by the first 8
  // lanes (component x node), the iterate in registers, neighbours by shuffle.
  __device__ void bottom() {
    if (threadIdx.x < 32) {
      const int lane = threadIdx.x, c = (lane >> 2) & 1, i = lane & 3, x = i & 1, y = i >> 1;
      const Real h2 = hsq(0), dg = diag(0);
      const Real bv = (lane < 8) ? S(0, 2, c)[i] : Real(0);
      Real xv = Real(0);
      for (int it = 0; it < 100; ++it) {
        const Real nx = __shfl_xor_sync(0xffffffffu, xv, 1);  // node (x^1, y)
        const Real ny = __shfl_xor_sync(0xffffffffu, xv, 2);  // node (x, y^1)
        const Real a = heat_row<Real>(x, y, 2, h2, [&](int p, int q) { return (p != x) ? nx : ((q != y) ? ny : xv); });
        xv = jacobi_update(xv, bv, a, dg);
      }
      if (lane < 8) S(0, slot(0), c)[i] = xv;
    }
    __syncthreads();
  }
};

template <typename Real>
__device__ void coarse_vcycle(int lc, double tau, Real* sm, const Real* bx, const Real* by, Real sgn, Real* outx,
                              Real* outy, bool want_norm, double part[kRedSlots], double* xs = nullptr) {
  Coarse<Real> C{sm, tau};
  const int wl = (1 << lc) + 1, Pl = pitch_of(wl);
  {
    // right-hand side and the first pre-sweep from x = 0 on level lc
    const Real dg = C.diag(lc);
    for_rect(wl, 2 * wl, [&](int x, int yy) {
      const int c = yy >= wl, y = yy - c * wl, id = y * wl + x;
      const Real r = (c ? by : bx)[(size_t)y * Pl + x] * sgn;
      C.S(lc, 2, c)[id] = r;
      C.S(lc, 0, c)[id] = jacobi_update(Real(0), r, Real(0), dg);
    });
    __syncthreads();
  }
  for (int k = lc; k >= 1; --k) C.down(k);
  C.bottom();
  for (int k = 1; k <= lc; ++k) C.up(k);
  const Real *s0 = C.S(lc, C.slot(lc), 0), *s1 = C.S(lc, C.slot(lc), 1);
  if (xs && want_norm) {
    // exact sums of |s|^2 in the element-pass geometry (one chunk per row)
    const XsGeom g(wl);
    const XsSum q0 = xs_sum(xs, wl, 0, false), q1 = xs_sum(xs, wl, 1, false);
    const int lx = threadIdx.x & 63, ly = threadIdx.x >> 6, half = lx >> 5;
    for (int y = ly; y < wl; y += kThreads / 64) {
      int ty = y / 8;
      if (ty > g.ny - 1) ty = g.ny - 1;
      const int r = y - ty * 8;
      double* B0 = xs_block(q0, ty * g.nx);
      double* B1 = xs_block(q1, ty * g.nx);
      double a0 = 0.0, a1 = 0.0;
      for (int x = lx; x < wl; x += 64) {
        const int id = y * wl + x;
        const Real a = s0[id], b = s1[id];
        const size_t gg = (size_t)y * Pl + x;
        outx[gg] = a;
        outy[gg] = b;
        const double t0 = (double)(a * a), t1 = (double)(b * b);
        B0[xs_at(x, r)] = t0;
        B1[xs_at(x, r)] = t1;
        a0 += t0;
        a1 += t1;
      }
      a0 = warp_sum(a0);
      a1 = warp_sum(a1);
      if ((threadIdx.x & 31) == 0) {
        q0.tot[2 * y * g.nx + half] = a0;
        q1.tot[2 * y * g.nx + half] = a1;
      }
    }
    return;
  }
  for_rect(wl, wl, [&](int x, int y) {
    const int id = y * wl + x;
    const Real a = s0[id], b = s1[id];
    const size_t g = (size_t)y * Pl + x;
    outx[g] = a;
    outy[g] = b;
    if (want_norm) part[0] += (double)a * (double)a + (double)b * (double)b;
  });
}

// Dynamic shared memory of the level kernel (elements of Real).
__host__ __device__ inline size_t level_smem_elems(int lc) {
  size_t e = (size_t)2 * 7 * EWIN;                               // energy, kind 2
  const size_t g = (size_t)2 * 5 * EWIN + (size_t)GCX * GCY * 8;  // gradient
  const size_t d = (size_t)2 * 2 * VWIN + (size_t)6 * VWIN;      // down
  const size_t u = (size_t)2 * (4 * VWIN + 2 * CWIN) + 2 * VWIN;  // up
  const size_t c = coarse_smem_elems(lc);
  const size_t n1 = (size_t)(2 * 6 + 1) * EWIN;                       // NCC energy, NCG purpose
  const size_t nf = (size_t)(2 * 4 + 1) * EWIN + (size_t)GCX * GCY * 8; // NCC variation
  if (n1 > e) e = n1;
  if (nf > e) e = nf;
  if (g > e) e = g;
  if (d > e) e = d;
  if (u > e) e = u;
  if (c > e) e = c;
  return e;
}

__device__ __forceinline__ bool finite_d(double x) { return !isnan(x) && !isinf(x); }

// ---------------------------------------------------------------------------
// Bounded values.  With exact sums a pass's sum in the reference's sequential
// order Q differs from any other order's sum P of the same N terms by at most
// 2 gamma_{N-1} sum |t| (both lie within gamma_{N-1} sum |t| of the real sum;
// recursive summation bound, Higham, Accuracy and Stability of Numerical
// Algorithms, 2nd ed., eq. 4.4), so Q is known to lie in an interval before
// the ordered sum is formed.  Rounding to nearest is monotone, so an
// expression of additions, subtractions, scalings and divisions (denominator
// of fixed sign) evaluated on the ends of its operands' intervals bounds its
// value on the exact operands; a comparison that the bounds settle is the
// comparison of the exact values.  ex: the value is known exactly (lo = hi).
// m: the term buffers (bit per buffer) whose bounded sums the interval was
// evaluated from (0 for an exact value).
struct Iv {
  double lo, hi;
  int ex;
  int m;
};
__device__ __forceinline__ Iv ivx(double x) { return Iv{x, x, 1, 0}; }
__device__ __forceinline__ Iv iv_unknown(int m) {
  const double q = __longlong_as_double(0x7ff8000000000000ll);
  return Iv{q, q, 0, m};
}
__device__ __forceinline__ Iv iv_add(Iv a, Iv b) {
  if (a.ex && b.ex) return ivx(a.lo + b.lo);
  return Iv{a.lo + b.lo, a.hi + b.hi, 0, a.m | b.m};
}
__device__ __forceinline__ Iv iv_sub(Iv a, Iv b) {
  if (a.ex && b.ex) return ivx(a.lo - b.lo);
  return Iv{a.lo - b.hi, a.hi - b.lo, 0, a.m | b.m};
}
__device__ __forceinline__ Iv iv_scale(Iv a, double s) {
  if (a.ex) return ivx(a.lo * s);
  return s >= 0.0 ? Iv{a.lo * s, a.hi * s, 0, a.m} : Iv{a.hi * s, a.lo * s, 0, a.m};
}
__device__ __forceinline__ Iv iv_div(Iv a, Iv b) {
  if (a.ex && b.ex) return ivx(a.lo / b.lo);
  if (!(b.lo > 0.0 || b.hi < 0.0)) return iv_unknown(a.m | b.m);
  const double c1 = a.lo / b.lo, c2 = a.lo / b.hi, c3 = a.hi / b.lo, c4 = a.hi / b.hi;
  if (isnan(c1) || isnan(c2) || isnan(c3) || isnan(c4)) return iv_unknown(a.m | b.m);
  return Iv{fmin(fmin(c1, c2), fmin(c3, c4)), fmax(fmax(c1, c2), fmax(c3, c4)), 0, a.m | b.m};
}
// E_reg = 1/2 (0 + s1 + s2) and Df = 0 + s3 + s4 from a pass's sums
__device__ __forceinline__ Iv xs_ereg(Iv s1, Iv s2) { return iv_scale(iv_add(iv_add(ivx(0.0), s1), s2), 0.5); }
__device__ __forceinline__ Iv xs_df(Iv s3, Iv s4) { return iv_add(iv_add(ivx(0.0), s3), s4); }
// E = (0 + E_data) + lambda E_reg, as the energy passes' totals combine
__device__ __forceinline__ Iv xs_energy(Iv edata, Iv ereg, double lam) {
  Iv e = ivx(0.0);
  e = iv_add(e, edata);
  if (lam != 1.0) e = iv_add(e, iv_scale(ereg, lam)); else e = iv_add(e, ereg);
  return e;
}

// A value of the descent state; while it is not exact it was evaluated from
// the bounded sums of term buffer buf (which then stays untouched) by kind.
enum XvKind : int { XK_NONE = 0, XK_ENERGY, XK_EREG, XK_DF };
struct XV {
  Iv v;
  int buf, kind;
};
__device__ __forceinline__ XV xv_exact(double x) { return XV{ivx(x), -1, XK_NONE}; }

// Sums of a term buffer's pass: state 0 being written, 1 bounded (or not
// known: NaN bounds), 2 exact; ns sums.
struct XsBufState {
  double lo[5], hi[5];
  int state, ns;
};

// ---------------------------------------------------------------------------
// Persistent task scheduler of the level kernel.
//
// A level solve of one instance is a chain of passes (initial energy,
// gradient, V-cycle down per level, coarse V-cycle, V-cycle up per level,
// NCG + first Armijo trial, further trials, final flush).  Every pass is cut
// into tiles.  All CTAs of the launch pull chunks of tiles from whichever
// instance has a published pass with chunks left; every tile stores its own
// partial sums, and the CTA that completes the last chunk of a pass adds them
// in tile order (so every total is independent of which CTA did what and of
// the chunking), runs the instance's descent control
// (gradientDescent.h / ArmijoSearch.h) and publishes the next pass.  No CTA
// ever waits for a particular other CTA, so uneven SM sharing, slow tiles and
// the single-CTA coarse V-cycle of one instance are hidden by the work of the
// others.
//
// Tiles are handed out in chunks of consecutive tiles.  Dispenser word per
// instance: [63:40] priority (an estimate of the instance's work left;
// workers take the highest first), [39:20] chunks of the pass, [19:0] next
// chunk.  A worker reads the word and only when chunks are left takes one
// with an atomic increment; an increment that arrives after the next pass was
// published takes a valid chunk of that pass, whose descriptor was written
// (and fenced) before the word.  Every wait for work is bounded; a worker
// that gives up sets the error flag and all workers return.
enum TaskKind : int {
  TK_E0 = 0, TK_GRAD, TK_VDOWN, TK_COARSE, TK_VUP, TK_NCG, TK_TRIAL, TK_FLUSH,
  TK_N1, TK_N2, TK_N3, TK_NF,   // NCC data term: energy subs 1-3, variation
  TK_XSUM,                      // exact sums: chunk summaries of the pass it stands for (purpose)
  TK_DONE
};
__device__ __forceinline__ int task_pass_kind(int kind) {
  switch (kind) {
    case TK_E0: return PK_ENERGY0;
    case TK_GRAD: return PK_GRAD;
    case TK_VDOWN: return PK_VDOWN;
    case TK_COARSE: return PK_VCOARSE;
    case TK_VUP: return PK_VUP;
    case TK_NCG: return PK_NCG;
    case TK_NF: return PK_GRAD;
    case TK_XSUM: return PK_REDUCE;
    default: return PK_ENERGY;
  }
}
constexpr int PF_STEP = 1;     // GRAD / FLUSH: add tau_p * d[dcur] to phi[cur]
constexpr int PF_ODZERO = 2;   // NCG: the old direction is zero (d = s)

struct PassDesc {
  int kind, k, cur, dcur, dn, flags;
  int ntiles, chunk;   // tiles of the pass, tiles per dispensed chunk
  int purpose;   // NCC energy subs, TK_XSUM: the pass they stand for (TK_E0, TK_GRAD, TK_TRIAL, TK_NCG, ...)
  int xn;        // TK_XSUM: exact sums of the buffer it adds
  int xbuf;      // exact sums: the pass's term buffer (TK_XSUM: of the pass it stands for)
  int xres;      // TK_XSUM: the term buffer whose sums it adds
  double t;      // trial step (NCG, TRIAL) or pending step (GRAD, FLUSH)
  double beta;   // Fletcher-Reeves factor (NCG)
  double vtau;   // tau of the V-cycle passes
  double mean, var, e;   // NCC: mass mean and norm of the deformed template, NCC energy
};

// Descent state of one instance; written only by the CTA completing a pass.
struct InstCtl {
  PassDesc desc;
  int done;            // tiles of the current pass completed
  int ls;              // TRIAL role: 0 doubling, 1 halving, 2 energy at the accepted step
  int iter, evals, total_evals, attempt, rb_pos, pending, od_zero, cur, dcur;
  double sigma, sigma_used, tau, og2, A, Bd, Cd, t, beta, tau_p;
  XV energy, energy_new, f, Df;
  XV last_ereg;        // E_reg of the last energy evaluation
  XV ereg_pos;         // E_reg at the current position (the energy log)
  XV rb_r[2];          // E_reg of the ring buffer's evaluations
  XV rb_e[2];
  double rb_tau[2];
  double n1[kRedSlots];      // NCC: totals of energy sub 1 (mean, then A or Df B C)
  XsBufState bs[kXsBufs];    // exact sums: the term buffers' sums
};
constexpr int kCtlWords = (int)((sizeof(InstCtl) + 7) / 8);
constexpr int kWordStride = 16;  // dispenser words 128 bytes apart

// A dispenser word: the pass's priority (bits 40-63), its chunks (20-39) and
// the chunks handed out (0-19).
__host__ __device__ inline unsigned long long pack_word(unsigned long long prio, int ntiles, int next) {
  return ((prio & 0xFFFFFFull) << 40) | ((unsigned long long)(ntiles & 0xFFFFF) << 20) | (unsigned long long)(next & 0xFFFFF);
}

template <typename Real>
struct SchedPtrs {
  InstCtl* ctl;                 // num_inst
  unsigned long long* words;    // num_inst * kWordStride
  double* partials;             // num_inst * max_tiles * kRedSlots
  int* finished;                // instances finished
  int* error;                   // non-zero: a worker gave up waiting
  int max_tiles;
};

template <typename Real>
__device__ __forceinline__ Inst<Real> make_inst(const LevelArgs<Real>& a, int inst) {
  Inst<Real> I;
  I.base = a.arena + (size_t)inst * a.inst_stride;
  if (a.inst_ref) I.R = a.R + (size_t)a.inst_ref[inst] * a.ref_stride;
  else I.R = (a.r_prev && inst > 0) ? a.arena + (size_t)(inst - 1) * a.inst_stride + a.off_T : a.R;
  I.T = I.base + a.off_T;
  I.normR = (a.r_prev || a.inst_ref) ? I.base + a.off_nr : a.normR;
  I.lambda = a.lambda_inst ? a.lambda_inst[inst] : a.lambda;
  I.n = a.n;
  I.P = pitch_of(a.n);
  I.h = (Real)(1.0 / (double)(a.n - 1));
  return I;
}

// The exact sums of a pass of kind `kind` for instance inst: slot 0 is the
// element sum E_data for the energy passes, every other slot a node sum.
template <typename Real>
__device__ __forceinline__ double* xs_buffer(const LevelArgs<Real>& a, int inst, int buf) {
  return a.xs + ((size_t)inst * (a.xs_bufs > 1 ? a.xs_bufs : 1) + buf) * a.xs_stride;
}
template <typename Real>
__device__ __forceinline__ void xs_pass_sums(const LevelArgs<Real>& a, int inst, int kind, int ns, int buf,
                                             XsSum* out) {
  double* base = xs_buffer(a, inst, buf);
  const bool energy = (kind == TK_E0 || kind == TK_TRIAL || kind == TK_NCG);
  for (int k = 0; k < ns; ++k) out[k] = xs_sum(base, a.n, k, energy && k == 0);
}

__device__ __forceinline__ int pass_tiles(int kind, int k, int level, int n, int xn) {
  switch (kind) {
    case TK_XSUM: return xs_summary_tasks(xn, n);
    case TK_VDOWN:
    case TK_VUP: {
      const int w = (1 << k) + 1;
      int nx = (w - 1) / VTX, ny = (w - 1) / VTY;
      return (nx < 1 ? 1 : nx) * (ny < 1 ? 1 : ny);
    }
    case TK_COARSE: return 1;
    default: {
      int nx = (n - 1) / TX, ny = (n - 1) / TY;
      return (nx < 1 ? 1 : nx) * (ny < 1 ? 1 : ny);
    }
  }
}

// Tiles per dispensed chunk: large enough that taking a chunk (a few L2
// round trips) is small against its work -- about a 24th of the pass, at
// most 16 tiles -- but no larger than the pass's tiles times the instances
// still running spread over the grid, so that the pass of a lone instance
// still spreads over every CTA.  Every tile stores its own partial sums and
// a pass adds them in tile order, so the chunking never changes a result.
__device__ __forceinline__ int chunk_tiles(int ntiles, int active, int div, int cmax) {
  int c = ntiles / div;
  c = c < 1 ? 1 : (c > cmax ? cmax : c);
  const long long work = (long long)ntiles * (active < 1 ? 1 : active);
  const int spread = (int)((work + gridDim.x - 1) / gridDim.x);
  return spread < c ? (spread < 1 ? 1 : spread) : c;
}

// Tiles of one pass: issue(t, stage) starts the window copies, compute(t,
// stage) does the work and accumulates part[].
template <typename Real, int KM = kKmAny>
struct TaskRunner {
  const LevelArgs<Real>& a;
  Real* smem;
  double (*xpw)[kXpSlots];   // shared: per-warp bound sums of an energy tile
  __device__ TaskRunner(const LevelArgs<Real>& a_, Real* sm, double (*xpw_)[kXpSlots])
      : a(a_), smem(sm), xpw(xpw_) {}
  // exact sums in this launch (the host launches kKmSsdExact exactly when
  // a.xs is set and the data term is SSD, kKmSsd when a.xs is null)
  __device__ bool xs_on() const { return KM == kKmSsdExact ? true : (KM == kKmSsd ? false : a.xs != nullptr); }

  template <class F>
  __device__ void with_pass(int inst, const PassDesc& d, double* part, F&& f) const {
    const Inst<Real> I = make_inst(a, inst);
    const int L = a.level;
    const size_t cs = comp_stride(L);
    Real* phi = I.arr(a.off_phi[d.cur]);
    Real* de = I.arr(a.off_de);
    Real* s = I.arr(a.off_s);
    double* xs = xs_on() ? xs_buffer(a, inst, d.xbuf) : nullptr;
    double* xp = (xs_on() && a.xpart) ? a.xpart + (size_t)inst * a.xpart_stride : nullptr;
    switch (d.kind) {
      case TK_E0: {
        EnergyPass<Real, KM> ps(I, 0, Real(0), Real(0), false, phi, phi + cs, nullptr, nullptr, nullptr, nullptr, nullptr,
                            nullptr, nullptr, nullptr, smem, part, xs, xp, xpw);
        f(ps);
        break;
      }
      case TK_TRIAL: {
        const Real* dd = I.arr(a.off_d[d.dcur]);
        EnergyPass<Real, KM> ps(I, 1, (Real)d.t, Real(0), false, phi, phi + cs, dd, dd + cs, nullptr, nullptr, nullptr,
                            nullptr, nullptr, nullptr, smem, part, xs, xp, xpw);
        f(ps);
        break;
      }
      case TK_NCG: {
        const Real* od = I.arr(a.off_d[d.dcur]);
        Real* wd = I.arr(a.off_d[d.dn]);
        EnergyPass<Real, KM> ps(I, 2, (Real)d.t, (Real)d.beta, (d.flags & PF_ODZERO) != 0, phi, phi + cs, od, od + cs, s,
                            s + cs, de, de + cs, wd, wd + cs, smem, part, xs, xp, xpw);
        f(ps);
        break;
      }
      case TK_GRAD: {
        Real* nphi = I.arr(a.off_phi[d.cur ^ 1]);
        const Real* dd = I.arr(a.off_d[d.dcur]);
        GradPass<Real> ps(I, (d.flags & PF_STEP) != 0, (Real)d.t, I.lambda, phi, phi + cs, dd, dd + cs, nphi,
                          nphi + cs, de, de + cs, smem, part);
        f(ps);
        break;
      }
      case TK_N1:
      case TK_N2:
      case TK_N3:
        if constexpr (KM == kKmAny) {   // the NCC passes exist in this variant only
          const int sub = (d.kind == TK_N1) ? 1 : (d.kind == TK_N2 ? 2 : 3);
          const int mode = (d.purpose == TK_GRAD) ? NM_GRAD
                           : (d.purpose == TK_TRIAL ? NM_TRIAL : (d.purpose == TK_NCG ? NM_NCG : NM_E0));
          const Real* dd = I.arr(a.off_d[d.dcur]);
          Real* wd = I.arr(a.off_d[d.dn]);
          Real* nphi = I.arr(a.off_phi[d.cur ^ 1]);
          Real* td = I.arr(a.off_td);
          const bool step = (d.flags & PF_STEP) != 0, odz = (d.flags & PF_ODZERO) != 0;
          NccPass<Real> ps(I, sub, mode, (Real)d.t, (Real)d.beta, d.mean, d.var, odz, step, phi, phi + cs, dd,
                           dd + cs, s, s + cs, de, de + cs, I.normR, wd, wd + cs, nphi, nphi + cs, td, smem, part);
          f(ps);
        }
        break;
      case TK_NF:
        if constexpr (KM == kKmAny) {
          Real* nphi = I.arr(a.off_phi[d.cur ^ 1]);
          NccForcePass<Real> ps(I, I.lambda, d.mean, d.var, d.e, nphi, nphi + cs, I.arr(a.off_td), I.normR, de,
                                de + cs, smem, part);
          f(ps);
        }
        break;
      case TK_VDOWN: {
        const int k = d.k, w = (1 << k) + 1;
        const Real hsq = (Real)(d.vtau * (double)((w - 1) * (w - 1)));
        const Real diag = (Real)(1 + 4 * d.vtau * (double)((w - 1) * (w - 1)));
        const Real* rx = (k == L) ? de : I.arr(a.off_b[k]);
        const Real* ry = (k == L) ? de + cs : rx + comp_stride(k);
        Real* x2 = I.arr(a.off_x2[k]);
        Real* bc = I.arr(a.off_b[k - 1]);
        DownPass<Real> ps(w, rx, ry, (k == L) ? Real(-1) : Real(1), x2, x2 + comp_stride(k), bc,
                          bc + comp_stride(k - 1), hsq, diag, smem);
        f(ps);
        break;
      }
      case TK_VUP: {
        const int k = d.k, w = (1 << k) + 1;
        const Real hsq = (Real)(d.vtau * (double)((w - 1) * (w - 1)));
        const Real diag = (Real)(1 + 4 * d.vtau * (double)((w - 1) * (w - 1)));
        const Real* rx = (k == L) ? de : I.arr(a.off_b[k]);
        const Real* ry = (k == L) ? de + cs : rx + comp_stride(k);
        const Real* x2 = I.arr(a.off_x2[k]);
        const Real* xc = I.arr(a.off_x5[k - 1]);
        Real* o = (k == L) ? s : I.arr(a.off_x5[k]);
        Real* oy = (k == L) ? s + cs : o + comp_stride(k);
        UpPass<Real> ps(w, rx, ry, (k == L) ? Real(-1) : Real(1), x2, x2 + comp_stride(k), xc,
                        xc + comp_stride(k - 1), o, oy, hsq, diag, smem, k == L, part,
                        (k == L && a.mode != MODE_SMOOTH) ? xs : nullptr);
        f(ps);
        break;
      }
      default: break;
    }
  }

  __device__ void issue(int inst, const PassDesc& d, int tile, int stage) const {
    if (d.kind == TK_COARSE || d.kind == TK_FLUSH || d.kind == TK_XSUM) return;  // these read global memory directly
    double dummy[kRedSlots];
    with_pass(inst, d, dummy, [&](auto& ps) { ps.issue(tile, stage); });
  }

  __device__ void compute(int inst, const PassDesc& d, int tile, int stage, double* part) const {
    if (KM != kKmSsd && d.kind == TK_XSUM) {
      // chunk and group summaries of the task tile's tile rows (all sums in turn)
      const bool energy = (d.purpose == TK_E0 || d.purpose == TK_TRIAL || d.purpose == TK_NCG);
      double* base = xs_buffer(a, inst, d.xres);
      const int n = a.n;
      xs_summary_task([&](int k) { return xs_sum(base, n, k, energy && k == 0); }, d.xn, XsGeom(n), tile);
      return;
    }
    if (d.kind == TK_COARSE) {
      const Inst<Real> I = make_inst(a, inst);
      const int L = a.level, lc = a.lc;
      const size_t cs = comp_stride(L);
      Real* de = I.arr(a.off_de);
      Real* s = I.arr(a.off_s);
      const Real* bx = (L == lc) ? de : I.arr(a.off_b[lc]);
      const Real* by = (L == lc) ? de + cs : bx + comp_stride(lc);
      Real* out = (L == lc) ? s : I.arr(a.off_x5[lc]);
      Real* outy = (L == lc) ? s + cs : out + comp_stride(lc);
      double* xs = (xs_on() && L == lc && a.mode != MODE_SMOOTH) ? xs_buffer(a, inst, d.xbuf) : nullptr;
      coarse_vcycle<Real>(lc, d.vtau, smem, bx, by, (L == lc) ? Real(-1) : Real(1), out, outy, L == lc, part, xs);
      return;
    }
    if (d.kind == TK_FLUSH) {
      // phi[cur^1] = phi[cur] + tau_p d[dcur] on the tile's nodes (gradientDescent.h:385-387)
      const Inst<Real> I = make_inst(a, inst);
      const size_t cs = comp_stride(a.level);
      const Real* phi = I.arr(a.off_phi[d.cur]);
      Real* nphi = I.arr(a.off_phi[d.cur ^ 1]);
      const Real* dd = I.arr(a.off_d[d.dcur]);
      const Real tp = (Real)d.t;
      Tiles tl(a.n);
      int x0, x1, y0, y1;
      tl.rect(tile, x0, x1, y0, y1);
      for_rect(x1 - x0, y1 - y0, [&](int ix, int iy) {
        const size_t g = (size_t)(y0 + iy) * I.P + (x0 + ix);
        Real vx = __ldcg(phi + g), vy = __ldcg(phi + cs + g);
        vx += tp * __ldcg(dd + g);
        vy += tp * __ldcg(dd + cs + g);
        nphi[g] = vx;
        nphi[cs + g] = vy;
      });
      return;
    }
    with_pass(inst, d, part, [&](auto& ps) { ps.compute(tile, stage); });
  }
};

// Deterministic CTA sum of kRedSlots per-thread values (warp butterflies,
// then the warps in order); the result is in out[] for every thread.
__device__ __forceinline__ void block_sum(const double part[kRedSlots], double (*wbuf)[kRedSlots],
                                          double* out) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < kRedSlots; ++k) {
    const double v = warp_sum(part[k]);
    if (lane == 0) wbuf[wid][k] = v;
  }
  __syncthreads();
  if (threadIdx.x < kRedSlots) {
    double s = 0.0;
#pragma unroll
    for (int w = 0; w < kThreads / 32; ++w) s += wbuf[w][threadIdx.x];
    out[threadIdx.x] = s;
  }
  __syncthreads();
}

// Descent control of one instance after a completed pass (run by one thread
// on a private copy of the state).  tot[] are the pass's totals; with exact
// sums xr[] are the pass's sums in the reference's order, each known exactly
// or (certified step) only within rigorous bounds.  Fills c.desc with the
// next pass; kind TK_DONE when the level solve is finished.  Returns false
// when a bounded value left a decision open (or a result to be written, or
// an operand of arithmetic, is not exact yet): the caller then discards c
// and has the sums added in order first.
// Follows GradientDescentBase::applySingle with the automatic filter width
// (gradientDescent.h:295-464, 675-691), Fletcher-Reeves NCG
// (gradientDescent.h:200-236) and ArmijoLineSearchUsingOp
// (ArmijoSearch.h:118-200).
template <typename Real>
__device__ bool advance(const LevelArgs<Real>& a, int inst, InstCtl& c, const double* tot, const Iv* xr,
                        int* open_bufs = nullptr) {
  const double lam = a.lambda_inst ? a.lambda_inst[inst] : a.lambda;
  const double tau_min = 9.313225746154785e-10;  // 2^-30 (ArmijoSearch.h:77)
  const double tau_max = 33554432.0;             // 2^25  (ArmijoSearch.h:67)
  const double stop_sigma = 0.0001, sigma_tol = 0.00001;
  const int L = a.level, lc = a.lc;
  PassDesc& d = c.desc;
  const int xb = d.xbuf;   // term buffer of the completed pass
  bool open = false;       // a decision the bounds do not settle
  // open_bufs: the term buffers the open decisions were evaluated from
  if (open_bufs) *open_bufs = 0;
  auto mark = [&](int m) {
    open = true;
    if (open_bufs) *open_bufs |= m;
  };
  // comparisons: exact operands compare as doubles; bounded ones decide
  // when the intervals do, else the step stays open
  auto ge = [&](Iv x, Iv y) {
    if (x.ex && y.ex) return x.lo >= y.lo;
    if (x.lo >= y.hi) return true;
    if (x.hi < y.lo) return false;
    mark(x.m | y.m);
    return false;
  };
  auto lt = [&](Iv x, Iv y) {
    if (x.ex && y.ex) return x.lo < y.lo;
    if (x.hi < y.lo) return true;
    if (x.lo >= y.hi) return false;
    mark(x.m | y.m);
    return false;
  };
  auto gt = [&](Iv x, Iv y) {
    if (x.ex && y.ex) return x.lo > y.lo;
    if (x.lo > y.hi) return true;
    if (x.hi <= y.lo) return false;
    mark(x.m | y.m);
    return false;
  };
  auto le = [&](Iv x, Iv y) {
    if (x.ex && y.ex) return x.lo <= y.lo;
    if (x.hi <= y.lo) return true;
    if (x.lo > y.hi) return false;
    mark(x.m | y.m);
    return false;
  };
  auto finite = [&](Iv x) {
    if (x.ex) return finite_d(x.lo);
    if (finite_d(x.lo) && finite_d(x.hi)) return true;
    mark(x.m);
    return true;
  };
  auto is_nan = [&](Iv x) {
    if (x.ex) return (bool)isnan(x.lo);
    if (isnan(x.lo) || isnan(x.hi)) mark(x.m);
    return false;
  };
  auto need = [&](Iv x) {   // a value written out or used in arithmetic
    if (!x.ex) mark(x.m);
    return (bool)x.ex;
  };
  // a value of the state evaluated from this pass's sums
  auto val = [&](Iv v, int kind) { return XV{v, (xr && !v.ex) ? xb : -1, kind}; };
  auto energy_of = [&](Iv edata, Iv ereg) { return xs_energy(edata, ereg, lam); };
  auto quad = [&](double tt) { return 0.5 * ((c.A + 2.0 * tt * c.Bd) + tt * tt * c.Cd); };
  auto target_met = [&](Iv en) {
    if (!a.e_target) return false;
    const double tg = a.e_target[inst];
    return le(en, ivx(tg + a.e_tol * fabs(tg)));
  };
  // exact sums (xr): E_reg = 1/2 (0 + p_x . L p_x + p_y . L p_y), the order of
  // DisplacementLengthEnergy::apply (hyperelastic.h:178-183)
  auto ereg_exact = [&]() { return xs_ereg(xr[1], xr[2]); };
  // the next pass is an energy-type pass: with the NCC data term it starts
  // with energy sub 1 and remembers what it stands for
  auto to = [&](int kind) {
    if (a.ncc) {
      d.purpose = kind;
      d.kind = TK_N1;
    } else {
      d.kind = kind;
    }
  };
  auto start_vcycle = [&](double vtau) {
    d.vtau = vtau;
    if (L > lc) { d.kind = TK_VDOWN; d.k = L; } else { d.kind = TK_COARSE; d.k = lc; }
  };
  auto start_iteration = [&]() {
    c.iter++;
    c.energy = c.energy_new;
    c.f = c.energy;
    c.sigma_used = c.sigma;
    c.evals = 0;
    to(TK_GRAD);
    d.cur = c.cur;
    d.dcur = c.dcur;
    d.flags = c.pending ? PF_STEP : 0;
    d.t = c.tau_p;
  };
  auto finish = [&]() {
    if (c.pending) {
      d.kind = TK_FLUSH;
      d.cur = c.cur;
      d.dcur = c.dcur;
      d.t = c.tau_p;
      d.flags = PF_STEP;
    } else {
      d.kind = TK_DONE;
    }
  };
  auto start_attempt = [&]() {
    const bool fallback = (c.attempt == 1);
    double t = (c.attempt == 0) ? c.tau : 0.0;
    t = t < tau_min ? tau_min : (t > tau_max ? tau_max : t);
    c.t = t;
    to(TK_NCG);
    d.cur = c.cur;
    d.dcur = c.dcur;
    d.dn = c.dcur ^ 1;
    d.t = t;
    d.beta = c.beta;
    d.flags = (fallback || c.od_zero) ? PF_ODZERO : 0;
  };
  auto trial = [&](double t, int role) {
    c.t = t;
    c.ls = role;
    to(TK_TRIAL);
    d.cur = c.cur;
    d.dcur = c.dcur;
    d.t = t;
  };
  auto push_ring = [&](double t, XV e) {
    c.rb_tau[c.rb_pos] = t;
    c.rb_e[c.rb_pos] = e;
    c.rb_r[c.rb_pos] = c.last_ereg;
    c.rb_pos ^= 1;
    c.evals++;
  };
  // the reference's energy log holds lambda * E_reg at the new position
  // (with a log file it evaluates the energy there again, gradientDescent.h:
  // 364-369, and writes the last evaluation's components)
  auto log_row = [&](int row, Iv en) {
    if (a.elog && row <= a.max_trace) {
      if (!need(en) || !need(c.ereg_pos.v)) return;
      double* lg = a.elog + ((size_t)inst * (a.max_trace + 1) + row) * 3;
      lg[0] = (double)(row - 1);
      lg[1] = lam * c.ereg_pos.v.lo;
      lg[2] = en.lo;
    }
  };
  auto end_iteration = [&](XV en, XV er) {
    c.ereg_pos = er;
    if (c.tau != 0) {
      c.pending = 1;
      c.tau_p = c.tau;
    }
    c.energy_new = en;
    c.total_evals += c.evals;
    log_row(c.iter, en.v);
    if (a.trace && c.iter <= a.max_trace && need(c.energy_new.v)) {
      double* tr = a.trace + ((size_t)inst * a.max_trace + (c.iter - 1)) * 4;
      tr[0] = c.energy_new.v.lo;
      tr[1] = c.tau;
      tr[2] = c.sigma_used;
      tr[3] = c.evals;
    }
    const Iv dec = iv_sub(c.energy.v, c.energy_new.v);
    bool go = (c.iter < a.max_iter) && gt(dec, ivx(a.stop_eps));
    if ((0.5 * c.sigma > stop_sigma) && lt(dec, ivx(sigma_tol))) {
      c.sigma *= 0.5;
      c.tau = 1.;
      go = (c.sigma > stop_sigma) && (c.iter < a.max_iter);
    }
    if (target_met(c.energy_new.v)) go = false;
    if (go) start_iteration(); else finish();
  };
  auto step_done = [&](double acc_tau) {
    c.tau = acc_tau;
    // energy at the new position (gradientDescent.h:365-395)
    XV en = c.energy, er = c.ereg_pos;
    bool found = false;
    if (c.rb_tau[0] == c.tau) { en = c.rb_e[0]; er = c.rb_r[0]; found = true; }
    else if (c.rb_tau[1] == c.tau) { en = c.rb_e[1]; er = c.rb_r[1]; found = true; }
    else if (c.tau == 0) { en = c.energy; found = true; }
    if ((!found || is_nan(en.v)) && c.tau != 0) {
      trial(c.tau, 2);
      return;
    }
    end_iteration(en, er);
  };
  auto attempt_done = [&](double res) {
    const bool fallback = (c.attempt == 1);
    c.od_zero = fallback ? 1 : 0;
    if (res != 0.0 || fallback) {
      step_done(res);
    } else {
      c.attempt = 1;
      start_attempt();
    }
  };

  // NCC energy subs: chain them, then continue as the pass they stand for
  double nt[kRedSlots];
  switch (d.kind) {
    case TK_N1:
#pragma unroll
      for (int k = 0; k < kRedSlots; ++k) c.n1[k] = tot[k];
      d.mean = tot[0];
      d.kind = TK_N2;
      return true;
    case TK_N2:
      d.var = sqrt(tot[0]);
      d.kind = TK_N3;
      return true;
    case TK_N3:
      d.e = -(tot[0]);
      if (d.purpose == TK_GRAD) {
        d.kind = TK_NF;
        return true;
      }
      nt[0] = d.e;
#pragma unroll
      for (int k = 1; k < kRedSlots; ++k) nt[k] = c.n1[k];
      tot = nt;
      d.kind = d.purpose;
      break;
    case TK_NF:
      d.kind = TK_GRAD;
      break;
    default: break;
  }

  switch (d.kind) {
    case TK_E0: {
      c.A = tot[1];
      c.last_ereg = xr ? val(ereg_exact(), XK_EREG) : val(ivx(0.5 * c.A), XK_EREG);
      c.energy = val(energy_of(xr ? xr[0] : ivx(tot[0]), c.last_ereg.v), XK_ENERGY);
      c.energy_new = c.energy;
      c.ereg_pos = c.last_ereg;
      log_row(0, c.energy.v);
      if (a.mode == MODE_ENERGY) {
        to(TK_GRAD);
        d.cur = c.cur;
        d.dcur = c.dcur;
        d.flags = 0;
        d.t = 0;
      } else if (a.max_iter > 0 && !target_met(c.energy.v)) {
        start_iteration();
      } else {
        d.kind = TK_DONE;
      }
      break;
    }
    case TK_GRAD: {
      if (a.mode == MODE_ENERGY) {
        d.kind = TK_DONE;
        break;
      }
      c.A = tot[1];
      c.cur ^= 1;
      c.pending = 0;
      start_vcycle((double)(0.5f * (c.sigma * c.sigma)));
      break;
    }
    case TK_VDOWN: {
      if (d.k - 1 > lc) d.k -= 1; else { d.kind = TK_COARSE; d.k = lc; }
      break;
    }
    case TK_COARSE:
    case TK_VUP: {
      const bool top = (d.kind == TK_COARSE) ? (L == lc) : (d.k == L);
      if (!top) {
        d.k = (d.kind == TK_COARSE) ? lc + 1 : d.k + 1;
        d.kind = TK_VUP;
        break;
      }
      if (a.mode == MODE_SMOOTH) {
        d.kind = TK_DONE;
        break;
      }
      double s2 = tot[0];
      if (xr) {   // 0 + s_x . s_x + s_y . s_y in the reference's order
        if (!need(xr[0]) || !need(xr[1])) return false;
        s2 = 0.0;
        s2 += xr[0].lo;
        s2 += xr[1].lo;
      }
      c.beta = ((c.iter - 1) % 10) ? (s2 / c.og2) : 0.0;
      c.og2 = s2;
      c.attempt = 0;
      start_attempt();
      break;
    }
    case TK_NCG: {
      c.dcur = d.dn;
      c.Df = val(ivx(tot[1]), XK_DF);
      c.Bd = tot[2];
      c.Cd = tot[3];
      if (xr) c.Df = val(xs_df(xr[3], xr[4]), XK_DF);   // 0 + DE_x . d_x + DE_y . d_y (ArmijoSearch.h:129-131)
      const double t = c.t;
      const Iv f = c.f.v, Df = c.Df.v;
      c.last_ereg = xr ? val(ereg_exact(), XK_EREG) : val(ivx(quad(t)), XK_EREG);
      const Iv fnew = energy_of(xr ? xr[0] : ivx(tot[0]), c.last_ereg.v);
      push_ring(t, val(fnew, XK_ENERGY));
      const Iv G = iv_div(iv_sub(fnew, f), iv_scale(Df, t));
      if (ge(Df, ivx(0.0)) || !finite(f)) {
        attempt_done(0.0);
      } else if (ge(G, ivx(0.5)) && ge(f, fnew)) {
        trial(t * 2., 0);
      } else {
        trial((t > tau_min) ? t * 0.5 : t, 1);
      }
      break;
    }
    case TK_TRIAL: {
      const double t = c.t;
      const Iv f = c.f.v;
      c.last_ereg = xr ? val(ereg_exact(), XK_EREG) : val(ivx(quad(t)), XK_EREG);
      const Iv fnew = energy_of(xr ? xr[0] : ivx(tot[0]), c.last_ereg.v);
      const XV fv = val(fnew, XK_ENERGY);
      push_ring(t, fv);
      if (c.ls == 2) {
        end_iteration(fv, c.last_ereg);
        break;
      }
      const Iv G = iv_div(iv_sub(fnew, f), iv_scale(c.Df.v, t));
      if (c.ls == 0) {
        if (ge(G, ivx(0.5)) && ge(f, fnew) && t <= tau_max) {
          trial(t * 2., 0);
        } else {
          const double tt = t * 0.5;
          attempt_done((tt > tau_min) ? tt : 0.0);
        }
      } else {
        if ((!finite(fnew) || (lt(G, ivx(0.5)) || lt(f, fnew))) && (t > tau_min)) {
          trial((t > tau_min) ? t * 0.5 : t, 1);
        } else {
          attempt_done((t > tau_min) ? t : 0.0);
        }
      }
      break;
    }
    case TK_FLUSH: {
      c.cur ^= 1;
      c.pending = 0;
      d.kind = TK_DONE;
      break;
    }
    default: d.kind = TK_DONE; break;
  }
  // the energy the solve reports is written out when it ends (after a flush
  // of the pending step, or after the gradient in energy mode)
  if ((d.kind == TK_DONE || d.kind == TK_FLUSH || (a.mode == MODE_ENERGY && d.kind == TK_GRAD)) &&
      a.mode != MODE_SMOOTH)
    need(c.energy_new.v);
  return !open;
}

__device__ __forceinline__ void init_ctl_state(InstCtl& c, int cur) {
  memset(&c, 0, sizeof(c));
  c.cur = cur;
  c.dcur = 0;
  c.tau = 1.0;
  c.sigma = 1.0;
  c.og2 = 0.0;
  c.od_zero = 1;
  c.rb_tau[0] = c.rb_tau[1] = nan("");
  c.energy = c.energy_new = c.f = c.Df = xv_exact(0.0);
  c.last_ereg = c.ereg_pos = xv_exact(0.0);
  c.rb_r[0] = c.rb_r[1] = c.rb_e[0] = c.rb_e[1] = xv_exact(0.0);
}

__device__ __forceinline__ void ctl_load(InstCtl& dst, const InstCtl* src) {
  const unsigned long long* s = reinterpret_cast<const unsigned long long*>(src);
  unsigned long long* d = reinterpret_cast<unsigned long long*>(&dst);
  for (int i = 0; i < kCtlWords; ++i) d[i] = __ldcg(s + i);
}
__device__ __forceinline__ void ctl_store(InstCtl* dst, const InstCtl& src) {
  const unsigned long long* s = reinterpret_cast<const unsigned long long*>(&src);
  unsigned long long* d = reinterpret_cast<unsigned long long*>(dst);
  for (int i = 0; i < kCtlWords; ++i) __stcg(d + i, s[i]);
}

// Exact sums a completed pass leaves to add (0: none): the energy passes
// E_data and p . L p per component, the NCG pass also DE . d per component,
// the top of the V-cycle |s|^2 per component.
template <typename Real>
__device__ __forceinline__ int xs_count(const LevelArgs<Real>& a, const PassDesc& d) {
  if (a.mode == MODE_SMOOTH) return 0;
  switch (d.kind) {
    case TK_E0:
    case TK_TRIAL: return 3;
    case TK_NCG: return 5;
    case TK_VUP: return d.k == a.level ? 2 : 0;
    case TK_COARSE: return a.level == a.lc ? 2 : 0;
    default: return 0;
  }
}

__device__ __forceinline__ bool is_energy_kind(int kind) {
  return kind == TK_E0 || kind == TK_TRIAL || kind == TK_NCG;
}

// Bounds of the ordered sum Q of at most N terms from another order's sum P
// and the sum A of the terms' magnitudes, both rounded themselves:
// |Q - P| <= 2 gamma_{N-1} A_true and A_true <= A / (1 - gamma_{N-1}); the
// factor 3 N u (u = 2^-53) and the term 2^-50 |P| also cover the rounding of
// the bounds.  Non-finite or huge inputs give no bounds (NaN).
__device__ __forceinline__ void xs_bounds(double P, double A, double N, double& lo, double& hi) {
  if (!(A < 1e300) || !(fabs(P) < 1e300)) {
    lo = hi = __longlong_as_double(0x7ff8000000000000ll);
    return;
  }
  const double B = A * (3.0 * N * 1.1102230246251565e-16) + fabs(P) * 8.881784197001252e-16;
  lo = P - B;
  hi = P + B;
}

// Term buffers the state holds: those of its values that are not exact yet.
__device__ __forceinline__ unsigned xs_held(const InstCtl& c) {
  unsigned m = 0;
  auto hold = [&](const XV& x) {
    if (!x.v.ex && x.buf >= 0) m |= 1u << x.buf;
  };
  hold(c.energy);
  hold(c.energy_new);
  hold(c.f);
  hold(c.Df);
  hold(c.last_ereg);
  hold(c.ereg_pos);
  hold(c.rb_r[0]);
  hold(c.rb_r[1]);
  hold(c.rb_e[0]);
  hold(c.rb_e[1]);
  return m;
}

// Buffer b's sums added in order (out[]): they are exact from now on, and so
// are the values evaluated from them (the control step's expressions again,
// on the exact sums); a summary pass's pending control step is taken again.
template <typename Real>
__device__ void xs_settle(const LevelArgs<Real>& a, int inst, InstCtl& c, int b, const double* out) {
  XsBufState& B = c.bs[b];
  for (int k = 0; k < B.ns; ++k) B.lo[k] = B.hi[k] = out[k];
  B.state = 2;
  const double lam = a.lambda_inst ? a.lambda_inst[inst] : a.lambda;
  Iv sv[5];
  for (int k = 0; k < 5; ++k) sv[k] = ivx(k < B.ns ? B.lo[k] : 0.0);
  auto upd = [&](XV& x) {
    if (x.v.ex || x.buf != b) return;
    if (x.kind == XK_EREG) x.v = xs_ereg(sv[1], sv[2]);
    else if (x.kind == XK_DF) x.v = xs_df(sv[3], sv[4]);
    else if (x.kind == XK_ENERGY) x.v = xs_energy(sv[0], xs_ereg(sv[1], sv[2]), lam);
    x.buf = -1;
  };
  upd(c.energy);
  upd(c.energy_new);
  upd(c.f);
  upd(c.Df);
  upd(c.last_ereg);
  upd(c.ereg_pos);
  upd(c.rb_r[0]);
  upd(c.rb_r[1]);
  upd(c.rb_e[0]);
  upd(c.rb_e[1]);
  if (c.desc.kind == TK_XSUM) c.desc.kind = c.desc.purpose;
}

// The buffer whose ordered sums an open control step needs next: the
// completed pass's own, then those of the state's bounded values.
// why: 0 for the pass's own buffer, else 1 + the position of the value in
// the order below (energy_new, energy, f, Df, the ring's energies, E_reg at
// the position, the last E_reg, the ring's E_reg).
__device__ __forceinline__ int xs_next_resolve(const InstCtl& c, int& why) {
  const int xb = c.desc.xbuf;
  why = 0;
  if (xb >= 0 && c.bs[xb].state != 2) return xb;
  const XV* order[10] = {&c.energy_new, &c.energy,    &c.f,       &c.Df,      &c.rb_e[0],
                         &c.rb_e[1],    &c.ereg_pos,  &c.last_ereg, &c.rb_r[0], &c.rb_r[1]};
  for (int i = 0; i < 10; ++i) {
    const XV& x = *order[i];
    if (!x.v.ex && x.buf >= 0 && c.bs[x.buf].state != 2) {
      why = i + 1;
      return x.buf;
    }
  }
  return -1;
}

// The control step after a completed pass (thread 0; c is the CTA's copy).
// With exact sums it is taken on the pass's sums as far as they are known:
// bounded sums settle most steps (certified step); a step they leave open is
// undone, and c then describes the summary pass that adds the needed
// buffer's sums in order, whose index is returned (-1: step taken).  With a
// single term buffer every pass's sums are added in order before its step.
template <typename Real>
__device__ int control_step(const LevelArgs<Real>& a, const SchedPtrs<Real>& sp, int inst, InstCtl& c,
                            const double* tot, bool xsums) {
  if (!xsums) {   // cannot be open: the values it writes out were exact before
    if (!advance(a, inst, c, tot, nullptr)) atomicExch(sp.error, 2);
    return -1;
  }
  const XsBufState& B = c.bs[c.desc.xbuf];
  int obufs = 0;   // buffers the open decisions were evaluated from
  if (a.xs_bufs > 1 || B.state == 2) {
    const bool bounded = B.state != 2;
    ctl_store(sp.ctl + inst, c);   // the state before the step
    Iv xr[5];
    for (int k = 0; k < 5; ++k) xr[k] = bounded ? Iv{B.lo[k], B.hi[k], 0, 1 << c.desc.xbuf} : ivx(B.lo[k]);
    if (advance(a, inst, c, tot, xr, &obufs)) {
      if (bounded && a.xs_prof) atomicAdd(a.xs_prof + 2, 1ull);
      return -1;
    }
    ctl_load(c, sp.ctl + inst);
  }
  // the buffer to add in order: one the open decisions were evaluated from
  // (the pass's own first), else the first bounded one in a fixed order
  int why = 0, rb = -1;
  for (int q = -1; q < kXsBufs && rb < 0; ++q) {
    const int b = q < 0 ? c.desc.xbuf : q;
    if (b >= 0 && ((obufs >> b) & 1) && c.bs[b].state != 2) {
      rb = b;
      why = 11;
    }
  }
  if (rb < 0) rb = xs_next_resolve(c, why);
  if (rb < 0) {   // cannot happen: a step on exact values is never open
    atomicExch(sp.error, 2);
    c.desc.kind = TK_DONE;
    return -1;
  }
  c.desc.purpose = c.desc.kind;
  c.desc.kind = TK_XSUM;
  c.desc.xres = rb;
  c.desc.xn = c.bs[rb].ns;
  trace_ev(a, global_ns(), kEvResolve,
           ((unsigned)inst << 16) | ((unsigned)rb << 12) | ((unsigned)why << 8) | (unsigned)c.desc.purpose);
  return rb;
}

// Publishes the instance's next pass (thread 0 of the completing CTA), or
// writes its results and counts it finished.
template <typename Real>
__device__ void publish(const LevelArgs<Real>& a, const SchedPtrs<Real>& sp, int inst, InstCtl& c) {
  unsigned long long* word = sp.words + (size_t)inst * kWordStride;
  // priority of the pass: an estimate of the instance's work left, the
  // gradient steps it has left at most times (3 + its energy evaluations per
  // step so far; the other passes of a step cost about three evaluations),
  // so that workers serve the instances furthest behind first and the
  // batch's solves end close together (results do not depend on it)
  const long long left = a.max_iter > c.iter ? (long long)(a.max_iter - c.iter) : 0ll;
  const long long rate = 48 + (16ll * c.total_evals) / (c.iter > 0 ? c.iter : 1);
  const unsigned long long prio = (unsigned long long)min(left * rate, 0xFFFFFFll);
  if (c.desc.kind == TK_DONE) {
    if (a.mode != MODE_SMOOTH) {
      a.out_energy[inst] = c.energy_new.v.lo;
      a.out_steps[inst] = c.iter;
      a.out_phi_buf[inst] = c.cur;
      if (a.out_evals) a.out_evals[inst] = c.total_evals;
    }
    c.done = 0;
    ctl_store(sp.ctl + inst, c);
    __threadfence();
    atomicExch(word, pack_word(prio, 0, 0));
    atomicAdd(sp.finished, 1);
    trace_ev(a, global_ns(), kEvPublish, ((unsigned)inst << 8) | (unsigned)TK_DONE);
    return;
  }
  // a pass with exact sums writes its terms to a buffer no bounded value holds
  if (a.xs && c.desc.kind != TK_XSUM) {
    const int nxs = xs_count(a, c.desc);
    if (nxs) {
      int b = 0;
      if (a.xs_bufs > 1) {
        const unsigned held = xs_held(c);
        b = -1;
        for (int q = 0; q < a.xs_bufs && q < kXsBufs; ++q)
          if (!(held & (1u << q))) { b = q; break; }
        if (b < 0) {   // cannot happen: at most 5 values are bounded at a time
          atomicExch(sp.error, 2);
          b = 0;
        }
      }
      c.desc.xbuf = b;
      c.bs[b].state = 0;
      c.bs[b].ns = nxs;
    }
  }
  c.desc.ntiles = pass_tiles(c.desc.kind, c.desc.k, a.level, a.n, c.desc.xn);
  c.desc.chunk = chunk_tiles(c.desc.ntiles, a.num_inst - *(volatile int*)sp.finished, a.chunk_div, a.chunk_max);
  const int nchunks = (c.desc.ntiles + c.desc.chunk - 1) / c.desc.chunk;
  c.done = 0;
  ctl_store(sp.ctl + inst, c);
  __threadfence();
  atomicExch(word, pack_word(prio, nchunks, 0));
  trace_ev(a, global_ns(), kEvPublish, ((unsigned)inst << 8) | (unsigned)c.desc.kind);
}

// Two passes whose tiles use the same shared-memory layout (so the first
// tile of one can be prefetched while the other computes).
__device__ __forceinline__ bool same_layout(const PassDesc& a, const PassDesc& b) {
  if (a.kind != b.kind || a.kind == TK_COARSE || a.kind == TK_FLUSH || a.kind == TK_XSUM) return false;
  if (a.kind == TK_N1) return a.purpose == b.purpose && a.flags == b.flags;
  return true;
}

struct TaskSlot {
  int inst, chunk, nchunks;   // chunk index of the pass, chunks of the pass
  PassDesc desc;
};

// One scan over the instances by the first warp (every lane of it calls this):
// each lane reads the dispenser words of its instances, and the lanes that
// see chunks left try to take one, in order from `start`.  Returns the same
// value in every lane; on success the task is in t (written by one lane).
template <typename Real>
__device__ bool try_take(const LevelArgs<Real>& a, const SchedPtrs<Real>& sp, int start, TaskSlot& t) {
  const int lane = threadIdx.x & 31;
  for (int base = 0; base < a.num_inst; base += 32) {
    const bool valid = base + lane < a.num_inst;
    const int inst = valid ? (start + base + lane) % a.num_inst : 0;
    unsigned long long* word = sp.words + (size_t)inst * kWordStride;
    bool avail = false;
    unsigned prio = 0;
    if (valid) {
      const unsigned long long w = __ldcg(word);
      avail = (int)(w & 0xFFFFF) < (int)((w >> 20) & 0xFFFFF);
      prio = (unsigned)(w >> 40);
    }
    unsigned mask = __ballot_sync(0xffffffffu, avail);
    while (mask) {
      // the first lane (from start) among those of the highest priority
      const unsigned top = __reduce_max_sync(0xffffffffu, ((mask >> lane) & 1u) ? prio : 0u);
      const int src = __ffs(__ballot_sync(0xffffffffu, ((mask >> lane) & 1u) && prio == top)) - 1;
      mask &= ~(1u << src);
      int got = 0;
      if (lane == src) {
        const unsigned long long old = atomicAdd(word, 1ull);
        const int chunk = (int)(old & 0xFFFFF), nchunks = (int)((old >> 20) & 0xFFFFF);
        if (chunk < nchunks) {
          __threadfence();
          t.inst = inst;
          t.chunk = chunk;
          t.nchunks = nchunks;
          const unsigned long long* src_d = reinterpret_cast<const unsigned long long*>(&sp.ctl[inst].desc);
          unsigned long long* dst = reinterpret_cast<unsigned long long*>(&t.desc);
#pragma unroll
          for (int i = 0; i < (int)(sizeof(PassDesc) / 8); ++i) dst[i] = __ldcg(src_d + i);
          got = 1;
        }
      }
      if (__shfl_sync(0xffffffffu, got, src)) return true;
    }
  }
  return false;
}

// Default bound on one wait for work (nanoseconds of the global timer, see
// LevelArgs::idle_ns); beyond it the worker sets the error flag and every
// worker returns.
constexpr unsigned long long kMaxIdleNs = 4000000000ull;

template <typename Real, int KM>
__global__ void __launch_bounds__(kThreads, 2) level_kernel(LevelArgs<Real> a, SchedPtrs<Real> sp) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  Real* smem = reinterpret_cast<Real*>(smem_raw);
  __shared__ double wbuf[kThreads / 32][kRedSlots];
  __shared__ double tot[kRedSlots];
  __shared__ TaskSlot slot[2];
  __shared__ int flag_wait, flag_next, flag_last;
  __shared__ InstCtl cs;
  __shared__ XsSum xss[kXsSlots];
  __shared__ double xres[kXsSlots], xwtot[kThreads / 32];
  __shared__ double xsp[12];   // bounds of a pass's sums: term sums, magnitude sums
  __shared__ int xact;         // buffer whose ordered sums the control step needs, or -1
  PassTimer pt{a.pass_cycles ? a.pass_cycles + (size_t)blockIdx.x * kPassKinds : nullptr, 0};
  __shared__ double xpw[kThreads / 32][kXpSlots];
  const TaskRunner<Real, KM> run(a, smem, xpw);
  const bool xs_on = run.xs_on();

  // publish the first pass of the instances this CTA owns
  if (threadIdx.x == 0) {
    for (int inst = blockIdx.x; inst < a.num_inst; inst += gridDim.x) {
      init_ctl_state(cs, a.phi_in_dev ? a.phi_in_dev[inst] : 0);
      if (a.mode == MODE_SMOOTH) {
        cs.desc.vtau = (double)(0.5f * (a.sigma_fixed * a.sigma_fixed));
        if (a.level > a.lc) { cs.desc.kind = TK_VDOWN; cs.desc.k = a.level; }
        else { cs.desc.kind = TK_COARSE; cs.desc.k = a.lc; }
      } else if (a.ncc) {
        cs.desc.kind = TK_N1;
        cs.desc.purpose = TK_E0;
      } else {
        cs.desc.kind = TK_E0;
      }
      cs.desc.cur = cs.cur;
      publish(a, sp, inst, cs);
    }
  }

  int cur_slot = 0, stage = 0;
  bool have = false;
  int last_inst = (a.num_inst > 0) ? (int)(blockIdx.x % (unsigned)a.num_inst) : 0;
  for (;;) {
    if (!have) {
      // wait for work (bounded)
      pt.start();
      if (threadIdx.x < 32) {
        int code = 0;
        const unsigned long long t_begin = global_ns();
        for (;;) {
          if (try_take(a, sp, last_inst, slot[cur_slot])) { code = 1; break; }
          int stop = 0;
          if (threadIdx.x == 0) {
            if (*(volatile int*)sp.error || *(volatile int*)sp.finished >= a.num_inst) stop = 2;
            else if (global_ns() - t_begin > a.idle_ns) {
              atomicExch(sp.error, 1);
              stop = 2;
            }
          }
          stop = __shfl_sync(0xffffffffu, stop, 0);
          if (stop) { code = stop; break; }
          __nanosleep(64);
        }
        if (threadIdx.x == 0) {
          flag_wait = code;
          if (a.tl && code == 1) {
            const unsigned long long w = global_ns() - t_begin;
            if (w >= 500) trace_ev(a, t_begin, kEvIdle, (unsigned)(w < 0xffffffffull ? w : 0xffffffffull));
          }
        }
      }
      __syncthreads();
      pt.stop(PK_REDUCE);
      if (flag_wait != 1) break;
      {
        const TaskSlot& f = slot[cur_slot];
        run.issue(f.inst, f.desc, f.chunk * f.desc.chunk, stage);
      }
      cp_async_commit();
      have = true;
    }
    const TaskSlot t = slot[cur_slot];
    const int tb = t.chunk * t.desc.chunk;
    const int te = min(tb + t.desc.chunk, t.desc.ntiles);
    TaskSlot nt;
    bool nh = false, pre = false;
    double part[kRedSlots] = {0.0, 0.0, 0.0, 0.0};
    pt.start();
    for (int tile = tb; tile < te; ++tile) {
      if (tile + 1 < te) {
        run.issue(t.inst, t.desc, tile + 1, stage ^ 1);
      } else {
        // last tile of the chunk: take the next chunk now (without waiting)
        // and prefetch its first tile when it uses the same layout
        if (threadIdx.x < 32) {
          const bool got = try_take(a, sp, t.inst, slot[cur_slot ^ 1]);
          if (threadIdx.x == 0) flag_next = got ? 1 : 0;
        }
        __syncthreads();
        nh = (flag_next == 1);
        if (nh) nt = slot[cur_slot ^ 1];
        pre = nh && same_layout(nt.desc, t.desc);
        if (pre) run.issue(nt.inst, nt.desc, nt.chunk * nt.desc.chunk, stage ^ 1);
      }
      cp_async_commit();
      cp_async_wait<1>();
      __syncthreads();
      run.compute(t.inst, t.desc, tile, stage, part);
      // the tile's partial sums, reduced in a fixed order and stored per tile
      block_sum(part, wbuf, tot);
      if (threadIdx.x == 0) {
        double* pp = sp.partials + ((size_t)t.inst * sp.max_tiles + tile) * kRedSlots;
#pragma unroll
        for (int k = 0; k < kRedSlots; ++k) __stcg(pp + k, tot[k]);
      }
      // an energy tile with bounds: its per-warp sums (written before the
      // reduction's barriers) into the tile's bound sums
      if (xs_on && a.xpart && is_energy_kind(t.desc.kind) && threadIdx.x < kXpSlots) {
        double v = 0.0;
#pragma unroll
        for (int w = 0; w < kThreads / 32; ++w) v += xpw[w][threadIdx.x];
        __stcg(a.xpart + (size_t)t.inst * a.xpart_stride + (size_t)tile * kXpSlots + threadIdx.x, v);
      }
#pragma unroll
      for (int k = 0; k < kRedSlots; ++k) part[k] = 0.0;
      stage ^= 1;
    }
    pt.stop(task_pass_kind(t.desc.kind));
    pt.start();
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) {
      const int dn = atomicAdd(&sp.ctl[t.inst].done, 1);
      flag_last = (dn == t.nchunks - 1) ? 1 : 0;
      __threadfence();
    }
    __syncthreads();
    if (flag_last) {
      // this CTA completed the pass: totals in tile order, then the control step
      if (threadIdx.x == 0) trace_ev(a, global_ns(), kEvComplete, ((unsigned)t.inst << 8) | (unsigned)t.desc.kind);
      double acc[kRedSlots] = {0.0, 0.0, 0.0, 0.0};
      const double* pp = sp.partials + (size_t)t.inst * sp.max_tiles * kRedSlots;
      for (int i = threadIdx.x; i < t.desc.ntiles; i += kThreads) {
#pragma unroll
        for (int k = 0; k < kRedSlots; ++k) acc[k] += __ldcg(pp + (size_t)i * kRedSlots + k);
      }
      block_sum(acc, wbuf, tot);
      const XsGeom xg(a.n);
      const bool xdone = xs_on && (t.desc.kind == TK_XSUM);
      const int nxs = (xs_on && !xdone) ? xs_count(a, t.desc) : 0;
      // an energy pass with bounds: the sums of its terms and magnitudes
      const bool cert = nxs && a.xpart && is_energy_kind(t.desc.kind);
      if (cert) {
        const double* xp = a.xpart + (size_t)t.inst * a.xpart_stride;
        for (int h = 0; h < kXpSlots; h += kRedSlots) {
          double v[kRedSlots] = {0.0, 0.0, 0.0, 0.0};
          for (int i = threadIdx.x; i < t.desc.ntiles; i += kThreads) {
#pragma unroll
            for (int k = 0; k < kRedSlots; ++k)
              if (h + k < kXpSlots) v[k] += __ldcg(xp + (size_t)i * kXpSlots + h + k);
          }
          block_sum(v, wbuf, xsp + h);
        }
      }
      // a summary pass completed: its buffer's sums in the reference's order
      if (xdone) {
        if (threadIdx.x == 0) xs_pass_sums(a, t.inst, t.desc.purpose, t.desc.xn, t.desc.xres, xss);
        __syncthreads();
        const unsigned long long tw = global_ns();
        xs_walk(xss, t.desc.xn, xg, xres, a.xs_prof);
        if (threadIdx.x == 0) trace_ev(a, tw, kEvWalk, (unsigned)(global_ns() - tw));
      }
      // the control step; when it needs a buffer's ordered sums first, the
      // predictions for them here and a summary pass over the grid (small
      // levels: the summaries and the walk right here, then the step again)
      for (bool first = true;; first = false) {
        if (threadIdx.x == 0) {
          if (first) {
            ctl_load(cs, sp.ctl + t.inst);
            if (xdone) {
              xs_settle(a, t.inst, cs, t.desc.xres, xres);
            } else if (nxs) {
              XsBufState& B = cs.bs[cs.desc.xbuf];
              B.ns = nxs;
              B.state = 1;
              const double N = (double)a.n * (double)a.n;
              for (int k = 0; k < nxs; ++k) {
                if (cert) xs_bounds(xsp[k], xsp[5 + k], N, B.lo[k], B.hi[k]);
                else B.lo[k] = B.hi[k] = __longlong_as_double(0x7ff8000000000000ll);
              }
            }
          }
          xact = control_step(a, sp, t.inst, cs, tot, xdone || nxs > 0);
        }
        __syncthreads();
        const int rb = xact;
        if (rb < 0) break;
        const int ns = cs.desc.xn;
        if (threadIdx.x == 0) xs_pass_sums(a, t.inst, cs.desc.purpose, ns, rb, xss);
        __syncthreads();
        xs_predict(xss, ns, xg, xwtot, a.xs_prof);
        const int ntask = xs_summary_tasks(ns, a.n);
        if (ntask > 6) break;   // summary pass published below
        for (int task = 0; task < ntask; ++task) xs_summary_task([&](int k) { return xss[k]; }, ns, xg, task);
        const unsigned long long tw = global_ns();
        xs_walk(xss, ns, xg, xres, a.xs_prof);
        if (threadIdx.x == 0) trace_ev(a, tw, kEvWalk, (unsigned)(global_ns() - tw));
        if (threadIdx.x == 0) xs_settle(a, t.inst, cs, rb, xres);
      }
      if (threadIdx.x == 0) publish(a, sp, t.inst, cs);
      __syncthreads();
    }
    pt.stop(PK_REDUCE);
    last_inst = t.inst;
    if (nh) {
      cur_slot ^= 1;
      if (!pre) {
        cp_async_wait<0>();
        __syncthreads();
        run.issue(nt.inst, nt.desc, nt.chunk * nt.desc.chunk, stage);
        cp_async_commit();
      }
    } else {
      have = false;
      cp_async_wait<0>();
      __syncthreads();
    }
  }
  cp_async_wait<0>();
}

}  // namespace msg
