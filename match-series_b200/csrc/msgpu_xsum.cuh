// msgpu_xsum.cuh -- the reference's sequential FP64 sums, reproduced bit for
// bit by a parallel computation.
//
// The reference adds every global sum of a level solve one term after the
// other in a fixed order: the SSD energy over the elements, x fastest
// (`res += a`, FEOpInterface.h:2600-2612), and every dot product over the
// nodes (`r += a[i] * b[i]`, aol::Vector).  The gradient flow decides its
// steps by comparing such sums (ArmijoSearch.h:118-200, gradientDescent.h:
// 416-439), and these decisions are discontinuous, so a sum that differs in
// its last bit can send the whole registration down another path.  Here
// every such sum gives exactly the reference's double:
//
// Let S be a partial sum with binade exponent E (ulp u = 2^E, so S = m u with
// 2^52 <= |m| < 2^53).  While the exact values S + p stay strictly inside
// that binade, round-to-nearest-even gives fl(S + p) = (m + c) u with
// c = rint(p / u), unless p / u lies exactly halfway between two integers
// (a tie), where the result is the even one of the two neighbours of m + p/u.
// So a run of terms whose partial sums stay in one binade is an integer sum
// of c's, which does not depend on the order of evaluation.
//
// The terms are cut into chunks (one tile row of 64 items; the order of the
// chunks is the reference's order).  For each chunk the kernel predicts the
// binade in which the running sum enters it (from an approximate prefix sum
// of chunk totals), and computes at that exponent: the sum of the c's, the
// smallest and largest partial sum, and the tie bookkeeping (after a first
// tie the running mantissa is even, so later ties are decided inside the
// chunk; the first tie is decided by the parity of the mantissa at the
// chunk start, known only when the chunk is reached).  One warp then walks
// the chunks in order, 32 at a time: a prefix sum over the lanes gives the
// mantissa at every chunk start, and a chunk whose partial sums leave
// [2^52 + 1, 2^53 - 1] (they cross a binade), whose predicted exponent is
// wrong, or whose running sum is zero is added term by term instead.  The
// result is exact whatever the prediction; predictions only change how many
// chunks take the slow path.
//
// Layout of one sum's terms: one block per tile of the pass (tile t of a grid
// of nx x ny tiles of TX x TY items), block = (TX + 1) x (TY + 1) doubles,
// term (k, r) (item x0 + k of row y0 + r) at k * (TY + 1) + r.  Every tile
// also writes two partial totals per (row, tile) chunk (the two warps of a
// row of 64), added to predict the binades.
#pragma once

#include <cuda_runtime.h>

namespace msg {

constexpr int kXsSlots = 5;           // sums of one pass at most (NCG: E_data, 2 x E_reg, 2 x Df)
constexpr int kXsBR = 9;              // rows per block: TY + 1 (the last tile row owns the final node row)
constexpr int kXsBK = 65;             // items per block row: TX + 1
constexpr int kXsBlock = kXsBR * kXsBK;

// Geometry of a level's sums: element-pass tiles of 64 x 8 items.
struct XsGeom {
  int n;        // nodes per side
  int nx, ny;   // tiles per row / column
  int nch;      // chunks of a node sum (n rows x nx); element sums have (n-1) x nx
  __host__ __device__ explicit XsGeom(int n_) : n(n_) {
    nx = (n - 1) / 64;
    if (nx < 1) nx = 1;
    ny = (n - 1) / 8;
    if (ny < 1) ny = 1;
    nch = n * nx;
  }
  __host__ __device__ size_t slot_terms() const { return (size_t)nx * ny * kXsBlock; }
};

// Per-instance region of the exact sums, in doubles: kXsSlots term arrays,
// the chunk totals (2 per chunk), and the chunk summaries (struct of arrays).
struct XsLayout {
  size_t terms, tot, X, R, mnB, mxB, mnA, mxA, ef, stride;
  __host__ __device__ explicit XsLayout(int n) {
    const XsGeom g(n);
    const size_t nc = (size_t)g.nch, a = 32;
    auto up = [&](size_t v) { return (v + a - 1) / a * a; };
    size_t o = 0;
    terms = o; o += up(kXsSlots * g.slot_terms());
    tot = o;   o += up(kXsSlots * 2 * nc);
    X = o;     o += up(kXsSlots * nc);
    R = o;     o += up(kXsSlots * nc);
    mnB = o;   o += up(kXsSlots * nc);
    mxB = o;   o += up(kXsSlots * nc);
    mnA = o;   o += up(kXsSlots * nc);
    mxA = o;   o += up(kXsSlots * nc);
    ef = o;    o += up((kXsSlots * nc + 1) / 2);   // ints
    stride = o;
  }
};

// One sum: its terms, chunk totals and summaries inside an instance region.
struct XsSum {
  double* terms;
  double* tot;
  long long *X, *R, *mnB, *mxB, *mnA, *mxA;
  int* ef;
  int rows, items;   // rows of items and items per row: n (node sums) or n - 1 (element sums)
};

__host__ __device__ inline XsSum xs_sum(double* base, int n, int slot, bool elements) {
  const XsGeom g(n);
  const XsLayout L(n);
  const size_t nc = (size_t)g.nch;
  XsSum s;
  s.terms = base + L.terms + slot * g.slot_terms();
  s.tot = base + L.tot + slot * 2 * nc;
  s.X = reinterpret_cast<long long*>(base + L.X) + slot * nc;
  s.R = reinterpret_cast<long long*>(base + L.R) + slot * nc;
  s.mnB = reinterpret_cast<long long*>(base + L.mnB) + slot * nc;
  s.mxB = reinterpret_cast<long long*>(base + L.mxB) + slot * nc;
  s.mnA = reinterpret_cast<long long*>(base + L.mnA) + slot * nc;
  s.mxA = reinterpret_cast<long long*>(base + L.mxA) + slot * nc;
  s.ef = reinterpret_cast<int*>(base + L.ef) + slot * nc;
  s.rows = elements ? n - 1 : n;
  s.items = elements ? n - 1 : n;
  return s;
}

// Block of tile t and the place of item (k, r) in it.
__device__ __forceinline__ double* xs_block(const XsSum& s, int tile) { return s.terms + (size_t)tile * kXsBlock; }
__device__ __forceinline__ int xs_at(int k, int r) { return k * kXsBR + r; }

// ---------------------------------------------------------------------------
// Exponent arithmetic.  A finite normal double S = m 2^E with 2^52 <= |m| <
// 2^53 (E the exponent of its ulp); exponents are kept within +-1000 so that
// 2^E and 2^-E are normal doubles.
__device__ __forceinline__ double xs_pow2(int e) { return __longlong_as_double((long long)(e + 1023) << 52); }

__device__ __forceinline__ bool xs_split(double S, int& E, long long& m) {
  const unsigned long long b = (unsigned long long)__double_as_longlong(S);
  const int ex = (int)((b >> 52) & 0x7ff);
  if (ex == 0 || ex == 0x7ff) return false;   // zero, subnormal, Inf, NaN
  E = ex - 1075;
  if (E < -1000 || E > 1000) return false;
  const long long mant = (long long)((b & 0xFFFFFFFFFFFFFull) | 0x10000000000000ull);
  m = (b >> 63) ? -mant : mant;
  return true;
}

// Packed exponent and flags of a chunk summary: bit 0 valid, bit 1 tie.
constexpr int kXsValid = 1, kXsTie = 2;
__device__ __forceinline__ int xs_pack(int E, int flags) { return ((E + 2048) << 2) | flags; }
__device__ __forceinline__ int xs_exp(int ef) { return (ef >> 2) - 2048; }
constexpr int kXsNoExp = 0;   // no prediction: xs_exp gives -2048, never a valid exponent

// Summary of one chunk (len terms at p[0], p[step], ...) for a running sum
// entering it with ulp exponent E (packed in ef; kXsNoExp: none).
//   no tie : X = sum of c, mnB/mxB = min/max partial sums (relative)
//   tie    : first tie at k1: X = c-sum before k1 + floor(p_k1/u); the
//            mantissa there is m + X + ((m + X) & 1), even; R = c-sum after
//            it with the later ties decided (parity of R so far), mnB/mxB
//            over the items before k1, mnA/mxA over the partial sums from k1.
__device__ __forceinline__ void xs_summarise(const double* p, int step, int len, int ef, long long& X,
                                             long long& R, long long& mnB, long long& mxB, long long& mnA,
                                             long long& mxA, int& out_ef) {
  const int E = xs_exp(ef);
  X = R = mnA = mxA = 0;
  mnB = mxB = 0;
  if (E < -1000 || E > 1000) { out_ef = xs_pack(E < -2000 ? -2000 : E, 0); return; }
  const double sc = xs_pow2(-E);
  long long P = 0, r = 0, lo = 0x7fffffffffffffffll, hi = -0x7fffffffffffffffll - 1;
  long long loA = 0, hiA = 0;
  bool tie = false, ok = true;
  for (int k0 = 0; k0 < len; k0 += 8) {
    double v[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = (k0 + i < len) ? __ldcg(p + (size_t)(k0 + i) * step) : 0.0;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      if (k0 + i >= len) break;
      const double q = v[i] * sc;
      if (!(fabs(q) < 36028797018963968.0)) {   // |q| < 2^55 (NaN and Inf fail too)
        ok = false;
        continue;
      }
      long long c = __double2ll_rn(q);
      const double d = q - (double)c;   // exact
      if (fabs(d) == 0.5) {
        const long long fl = (d > 0) ? c : c - 1;
        if (!tie) {
          tie = true;
          X = P + fl;
          continue;
        }
        c = fl + ((r + fl) & 1);
      }
      if (!tie) {
        P += c;
        lo = P < lo ? P : lo;
        hi = P > hi ? P : hi;
      } else {
        r += c;
        loA = r < loA ? r : loA;
        hiA = r > hiA ? r : hiA;
      }
    }
  }
  if (!tie) X = P;
  if (lo > hi) lo = hi = 0;   // no item before the first tie
  R = r;
  mnB = lo;
  mxB = hi;
  mnA = loA;
  mxA = hiA;
  out_ef = xs_pack(E, (ok ? kXsValid : 0) | (tie ? kXsTie : 0));
}

// Chunk j of a sum: its tile, row within the tile and length.
__device__ __forceinline__ void xs_chunk(const XsSum& s, const XsGeom& g, int j, int& tile, int& r, int& len) {
  const int y = j / g.nx, tx = j - y * g.nx;
  int ty = y / 8;
  if (ty > g.ny - 1) ty = g.ny - 1;
  r = y - ty * 8;
  tile = ty * g.nx + tx;
  const int x0 = tx * 64;
  len = (tx == g.nx - 1) ? s.items - x0 : 64;
}

__device__ __forceinline__ bool xs_in_range(long long v, bool neg) {
  constexpr long long lo = (1ll << 52) + 1, hi = (1ll << 53) - 1;
  return neg ? (v >= -hi && v <= -lo) : (v >= lo && v <= hi);
}

// S + t_0 + ... + t_{cnt-1} in sequence, the terms one per lane (lane k holds
// t_k), by the warp: at the exponent of the exact running sum every lane
// converts its term to units of the ulp, a prefix sum over the lanes gives
// the running mantissa after every term, and the run stops at the first term
// whose sum leaves the binade or is a tie (or whose running sum cannot be
// split); that one term is added in floating point, and the walk goes on
// from the next term.  Every lane returns the same value.
__device__ __forceinline__ double xs_add_lanes(double S, double v, int cnt) {
  const int lane = threadIdx.x & 31;
  int pos = 0;
  while (pos < cnt) {
    int E;
    long long m;
    if (!xs_split(S, E, m)) {
      S = __dadd_rn(S, __shfl_sync(0xffffffffu, v, pos));
      ++pos;
      continue;
    }
    const bool act = lane >= pos && lane < cnt;
    const double q = v * xs_pow2(-E);
    bool ok = act && fabs(q) < 36028797018963968.0;
    long long c = 0;
    if (ok) {
      c = __double2ll_rn(q);
      ok = fabs(q - (double)c) != 0.5;
    }
    unsigned long long inc = act ? (unsigned long long)c : 0ull;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned long long t = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += t;
    }
    const long long mi = m + (long long)inc;   // mantissa after this lane's term
    const bool good = ok && xs_in_range(mi, m < 0);
    const unsigned bad = __ballot_sync(0xffffffffu, act && !good);
    const int first = bad ? __ffs(bad) - 1 : cnt;
    if (first > pos) S = (double)__shfl_sync(0xffffffffu, mi, first - 1) * xs_pow2(E);
    if (first < cnt) {
      S = __dadd_rn(S, __shfl_sync(0xffffffffu, v, first));
      if (first == pos) {
        // no run at all: the sum changes binade term after term here, so
        // the rest of the segment goes one addition after the other
        for (int k = first + 1; k < cnt; ++k) S = __dadd_rn(S, __shfl_sync(0xffffffffu, v, k));
        return S;
      }
      pos = first + 1;
    } else {
      pos = cnt;
    }
  }
  return S;
}

// S + t_0 + ... + t_{cnt-1} one addition after the other (lane k holds t_k);
// the shuffles do not depend on S, so they are issued ahead of the additions.
__device__ __forceinline__ double xs_add_seq(double S, double v, int cnt) {
#pragma unroll
  for (int k0 = 0; k0 < 32; k0 += 8) {
    if (k0 >= cnt) break;
    double t[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) t[i] = __shfl_sync(0xffffffffu, v, k0 + i);
#pragma unroll
    for (int i = 0; i < 8; ++i)
      if (k0 + i < cnt) S = __dadd_rn(S, t[i]);
  }
  return S;
}

// One segment of up to 32 terms: where the terms are not small against the
// running sum (its binade would change at many of them) one addition after
// the other, else the binade runs of xs_add_lanes.
__device__ __forceinline__ double xs_add_segment(double S, double v, int cnt) {
  const int lane = threadIdx.x & 31;
  double a = lane < cnt ? fabs(v) : 0.0;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
  if (!(a < fabs(S) * 0.015625)) return xs_add_seq(S, v, cnt);   // also for S = 0 and non-finite values
  return xs_add_lanes(S, v, cnt);
}

// The terms of chunk j, lane k holding terms k, k + 32 and k + 64.
struct XsChunkTerms {
  double v0, v1, v2;
  int len;
};
__device__ __forceinline__ XsChunkTerms xs_load_chunk(const XsSum& s, const XsGeom& g, int j) {
  const int lane = threadIdx.x & 31;
  int tile, r, len;
  xs_chunk(s, g, j, tile, r, len);
  const double* p = xs_block(s, tile) + r;
  XsChunkTerms c;
  c.len = len;
  c.v0 = (lane < len) ? __ldcg(p + xs_at(lane, 0)) : 0.0;
  c.v1 = (lane + 32 < len) ? __ldcg(p + xs_at(lane + 32, 0)) : 0.0;
  c.v2 = (lane + 64 < len) ? __ldcg(p + xs_at(lane + 64, 0)) : 0.0;
  return c;
}

// fl(... fl(fl(S + p_0) + p_1) ... + p_{len-1}) for a chunk's terms, by the
// warp in segments of 32 terms (every lane returns the same value).
__device__ __forceinline__ double xs_add_terms(double S, const XsChunkTerms& c) {
  S = xs_add_segment(S, c.v0, c.len < 32 ? c.len : 32);
  if (c.len > 32) S = xs_add_segment(S, c.v1, c.len < 64 ? c.len - 32 : 32);
  if (c.len > 64) S = xs_add_seq(S, c.v2, c.len - 64);
  return S;
}
__device__ __forceinline__ double xs_add_chunk(const XsSum& s, const XsGeom& g, int j, double S) {
  return xs_add_terms(S, xs_load_chunk(s, g, j));
}

// The sequential sum 0 + t_0 + t_1 + ... of one sum, by one warp (every lane
// returns it).  Needs the summaries of every chunk.
__device__ double xs_drive(const XsSum& s, const XsGeom& g, unsigned long long* prof) {
  unsigned long long slow = 0, slow_cycles = 0;
  const long long t_start = clock64();
  const int lane = threadIdx.x & 31;
  const unsigned lt_mask = (1u << lane) - 1u;   // lanes below this one
  const int nch = s.rows * g.nx;
  double S = 0.0;
  int j = 0;
  // the records of the next window are loaded while the current one is walked
  auto load = [&](int jn, int& ef, long long& X, long long& lo, long long& hi, long long& R, long long& loA,
                  long long& hiA) {
    const bool in = jn < nch;
    ef = in ? __ldcg(s.ef + jn) : 0;
    X = in ? __ldcg(s.X + jn) : 0;
    lo = in ? __ldcg(s.mnB + jn) : 0;
    hi = in ? __ldcg(s.mxB + jn) : 0;
    R = in ? __ldcg(s.R + jn) : 0;
    loA = in ? __ldcg(s.mnA + jn) : 0;
    hiA = in ? __ldcg(s.mxA + jn) : 0;
  };
  int nef;
  long long nX, nlo, nhi, nR, nloA, nhiA;
  load(lane, nef, nX, nlo, nhi, nR, nloA, nhiA);
  for (int jb = 0; jb < nch; jb += 32) {
    const bool in = jb + lane < nch;
    const int ef = nef;
    const long long X = nX, lo = nlo, hi = nhi, R = nR, loA = nloA, hiA = nhiA;
    load(jb + lane + 32, nef, nX, nlo, nhi, nR, nloA, nhiA);
    // chunks where the predicted binade of the next chunk differs (the sum
    // crosses a binade inside) or without a usable summary: added term by
    // term, so their terms are fetched ahead, the first one now
    const int efn = __shfl_down_sync(0xffffffffu, ef, 1);
    const unsigned slowm =
        __ballot_sync(0xffffffffu, in && (!(ef & kXsValid) || (lane < 31 && jb + lane + 1 < nch &&
                                                                   xs_exp(efn) != xs_exp(ef))));
    auto next_slow = [&](int from) -> int {
      const unsigned m = from >= 32 ? 0u : (slowm & ~((1u << from) - 1u));
      return m ? __ffs(m) - 1 : -1;
    };
    int pf = next_slow(j - jb);
    XsChunkTerms pt;
    if (pf >= 0) pt = xs_load_chunk(s, g, jb + pf);
    while (j < jb + 32 && j < nch) {
      if (isnan(S)) return S;
      int E;
      long long m;
      if (!xs_split(S, E, m)) {
        const long long ts = clock64();
        if (j - jb == pf) {
          S = xs_add_terms(S, pt);
          pf = next_slow(pf + 1);
          if (pf >= 0) pt = xs_load_chunk(s, g, jb + pf);
        } else {
          S = xs_add_chunk(s, g, j, S);
        }
        slow_cycles += (unsigned long long)(clock64() - ts);
        ++slow;
        ++j;
        continue;
      }
      const bool neg = m < 0;
      const int o = j - jb;
      const bool act = lane >= o && in;
      const bool use = act && (ef & kXsValid) && xs_exp(ef) == E;
      const bool tie = use && (ef & kXsTie);
      // parity of the mantissa entering every lane's chunk: after a tie chunk
      // it is the parity of that chunk's R (its mantissa at the first tie is
      // even), before any tie the parity of m; the chunks in between add X
      const unsigned ties = __ballot_sync(0xffffffffu, tie);
      const unsigned odd = __ballot_sync(0xffffffffu, use && !tie && (X & 1));
      const unsigned tb = ties & lt_mask;
      const int t = tb ? 31 - __clz(tb) : -1;   // last tie chunk below this lane
      const long long Rt = __shfl_sync(0xffffffffu, R, t < 0 ? 0 : t);
      const unsigned between = lt_mask & (t < 0 ? ~((1u << o) - 1u) : ~((2u << t) - 1u));
      const int par_in = ((t < 0 ? (int)(m & 1) : (int)(Rt & 1)) + __popc(odd & between)) & 1;
      const long long b = (long long)((par_in + (int)(X & 1)) & 1);
      const long long delta = use ? (tie ? X + b + R : X) : 0;
      // exclusive prefix of the chunk deltas over the lanes
      unsigned long long inc = (unsigned long long)delta;
#pragma unroll
      for (int o2 = 1; o2 < 32; o2 <<= 1) {
        const unsigned long long tt = __shfl_up_sync(0xffffffffu, inc, o2);
        if (lane >= o2) inc += tt;
      }
      const long long mi = m + (long long)(inc - (unsigned long long)delta);
      bool good = use && xs_in_range(mi + lo, neg) && xs_in_range(mi + hi, neg);
      if (tie) {
        const long long m1 = mi + X + b;
        good = good && xs_in_range(m1 + loA, neg) && xs_in_range(m1 + hiA, neg);
      }
      const unsigned bad = __ballot_sync(0xffffffffu, act && !good);
      const int last = (nch - jb < 32 ? nch - jb : 32);   // lanes with a chunk
      const int first = bad ? __ffs(bad) - 1 : last;
      // mantissa at the start of chunk jb + first
      const long long mf = __shfl_sync(0xffffffffu, mi + delta, (first > 0 ? first : 1) - 1);
      if (first > o) S = (double)mf * xs_pow2(E);
      j = jb + first;
      if (j < jb + 32 && j < nch) {
        // chunk j interrupts the run (its sums leave the binade, or it has no
        // summary at this exponent): added term by term
        const long long ts = clock64();
        if (first == pf) {
          S = xs_add_terms(S, pt);
          pf = next_slow(pf + 1);
          if (pf >= 0) pt = xs_load_chunk(s, g, jb + pf);
        } else {
          S = xs_add_chunk(s, g, j, S);
          if (pf >= 0 && pf < first) {   // the fetched chunk was passed by the run
            pf = next_slow(first + 1);
            if (pf >= 0) pt = xs_load_chunk(s, g, jb + pf);
          }
        }
        slow_cycles += (unsigned long long)(clock64() - ts);
        ++slow;
        ++j;
      }
    }
  }
  if (prof && (threadIdx.x & 31) == 0) {
    atomicAdd(prof + 4, (unsigned long long)nch);
    atomicAdd(prof + 5, slow);
    atomicAdd(prof + 6, slow_cycles);
    atomicAdd(prof + 7, (unsigned long long)(clock64() - t_start));
  }
  return S;
}

// Block-wide exclusive prefix sum of one double per thread (256 threads);
// the order of the additions does not matter here (predictions only).
__device__ __forceinline__ double xs_block_excl(double v, double* wtot /* [8] shared */) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  double inc = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const double t = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += t;
  }
  if (lane == 31) wtot[w] = inc;
  __syncthreads();
  double base = 0.0;
  for (int k = 0; k < w; ++k) base += wtot[k];
  __syncthreads();
  return base + inc - v;
}

// The exact sums of a completed pass in three steps.  1 (xs_predict, the
// CTA that completed the pass): the predicted binade at every chunk start.
// 2 (xs_summary_row, a pass of its own spread over the grid): the chunk
// summaries at the predicted exponents, one chunk per thread.  3 (xs_walk,
// the CTA that completed step 2): one warp per sum walks its chunks in order.
constexpr int kXsTilesPerTask = 256 / kXsBR;   // term blocks per task tile of step 2 (9 rows each)

// Profile counters (nullable): [0] passes, [1..3] cycles of the steps,
// [4] chunks walked, [5] chunks added term by term.
__device__ __noinline__ void xs_predict(const XsSum* sums, int ns, const XsGeom& g, double* wtot /* shared [8] */,
                           unsigned long long* prof) {
  const long long t0 = clock64();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int k = 0; k < ns; ++k) {
    const XsSum& s = sums[k];
    const int nch = s.rows * g.nx;
    // warp w takes the contiguous range [c0, c1) in rounds of 32 chunks,
    // lane l chunk c0 + 32 i + l (coalesced loads of the two partial totals)
    const int per = ((nch + nw - 1) / nw + 31) & ~31;
    const int c0 = warp * per, c1 = min(c0 + per, nch);
    double loc = 0.0;
    const double2* tot2 = reinterpret_cast<const double2*>(s.tot);
    for (int c = c0 + lane; c < c1; c += 128) {
      double2 tt[4];
#pragma unroll
      for (int u = 0; u < 4; ++u)
        tt[u] = (c + 32 * u < c1) ? __ldcg(tot2 + c + 32 * u) : make_double2(0.0, 0.0);
#pragma unroll
      for (int u = 0; u < 4; ++u) loc += tt[u].x + tt[u].y;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) loc += __shfl_xor_sync(0xffffffffu, loc, o);
    if (lane == 0) wtot[warp] = loc;
    __syncthreads();
    double run = 0.0;
    for (int w = 0; w < warp; ++w) run += wtot[w];
    __syncthreads();
    double2 nxt = (c0 + lane < c1) ? __ldcg(tot2 + c0 + lane) : make_double2(0.0, 0.0);
    for (int cb = c0; cb < c1; cb += 32) {
      const int c = cb + lane;
      const double2 tt = nxt;
      nxt = (c + 32 < c1) ? __ldcg(tot2 + c + 32) : make_double2(0.0, 0.0);
      const double v = tt.x + tt.y;
      double inc = v;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const double u = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += u;
      }
      const double start = run + (inc - v);   // estimated running sum at the chunk start
      int E;
      long long m;
      if (c < c1) __stcg(s.ef + c, xs_split(start, E, m) ? xs_pack(E, 0) : kXsNoExp);
      run += __shfl_sync(0xffffffffu, inc, 31);
    }
  }
  __threadfence();
  __syncthreads();
  if (prof && threadIdx.x == 0) {
    atomicAdd(prof + 0, 1ull);
    atomicAdd(prof + 1, (unsigned long long)(clock64() - t0));
  }
}

// Step 2: the summary of chunk row r of term block t of sum s (one thread).
__device__ __noinline__ void xs_summary_row(const XsSum& s, const XsGeom& g, int t, int r) {
  const int ty = t / g.nx, tx = t - ty * g.nx;
  const int rows_t = (ty == g.ny - 1) ? s.rows - ty * 8 : 8;
  if (r >= rows_t) return;
  const int y = ty * 8 + r;
  const int x0 = tx * 64;
  const int len = (tx == g.nx - 1) ? s.items - x0 : 64;
  const int j = y * g.nx + tx;
  long long X, R, lo, hi, loA, hiA;
  int ef;
  xs_summarise(xs_block(s, t) + r, kXsBR, len, __ldcg(s.ef + j), X, R, lo, hi, loA, hiA, ef);
  __stcg(s.X + j, X);
  __stcg(s.R + j, R);
  __stcg(s.mnB + j, lo);
  __stcg(s.mxB + j, hi);
  __stcg(s.mnA + j, loA);
  __stcg(s.mxA + j, hiA);
  __stcg(s.ef + j, ef);
}

// Task tiles of the summary pass.
__host__ __device__ inline int xs_summary_tasks(int ns, int n) {
  const XsGeom g(n);
  return (ns * g.nx * g.ny + kXsTilesPerTask - 1) / kXsTilesPerTask;
}

// Step 3: out[k] = the sequential sum k (one warp per sum).
__device__ __noinline__ void xs_walk(const XsSum* sums, int ns, const XsGeom& g, double* out /* shared [ns] */,
                        unsigned long long* prof) {
  const long long t0 = clock64();
  const int warp = threadIdx.x >> 5;
  if (warp < ns) {
    const double v = xs_drive(sums[warp], g, prof);
    if ((threadIdx.x & 31) == 0) out[warp] = v;
  }
  __syncthreads();
  if (prof && threadIdx.x == 0) atomicAdd(prof + 3, (unsigned long long)(clock64() - t0));
}

}  // namespace msg
