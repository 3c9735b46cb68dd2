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
// of nx x ny tiles of TX x TY items), block = (TY + 1) rows of TX + 2 doubles
// (TX + 1 items, padded to 16 bytes), term (k, r) (item x0 + k of row y0 + r)
// at r * (TX + 2) + k: the tiles store their terms with coalesced writes.  Every tile
// also writes two partial totals per (row, tile) chunk (the two warps of a
// row of 64), added to predict the binades.
#pragma once

#include <cuda_runtime.h>

namespace msg {

constexpr int kXsSlots = 5;           // sums of one pass at most (NCG: E_data, 2 x E_reg, 2 x Df)
constexpr int kXsBR = 9;              // rows per block: TY + 1 (the last tile row owns the final node row)
constexpr int kXsBK = 66;             // doubles per block row: TX + 1 items, padded to 16 bytes
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
  size_t terms, tot, X, R, mnB, mxB, mnA, mxA, ef, gX, gmn, gmx, gef, stride;
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
    const size_t ng = (size_t)g.ny;
    gX = o;    o += up(kXsSlots * ng);
    gmn = o;   o += up(kXsSlots * ng);
    gmx = o;   o += up(kXsSlots * ng);
    gef = o;   o += up((kXsSlots * ng + 1) / 2);   // ints
    stride = o;
  }
};

// One sum: its terms, chunk totals and summaries inside an instance region.
struct XsSum {
  double* terms;
  double* tot;
  long long *X, *R, *mnB, *mxB, *mnA, *mxA;
  int* ef;
  long long *gX, *gmn, *gmx;   // group summaries (one group per tile row)
  int* gef;
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
  const size_t ng = (size_t)g.ny;
  s.gX = reinterpret_cast<long long*>(base + L.gX) + slot * ng;
  s.gmn = reinterpret_cast<long long*>(base + L.gmn) + slot * ng;
  s.gmx = reinterpret_cast<long long*>(base + L.gmx) + slot * ng;
  s.gef = reinterpret_cast<int*>(base + L.gef) + slot * ng;
  s.rows = elements ? n - 1 : n;
  s.items = elements ? n - 1 : n;
  return s;
}

// Block of tile t and the place of item (k, r) in it.
__device__ __forceinline__ double* xs_block(const XsSum& s, int tile) { return s.terms + (size_t)tile * kXsBlock; }
__host__ __device__ __forceinline__ int xs_at(int k, int r) { return r * kXsBK + k; }

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

// Packed exponent and flags of a chunk summary: bit 0 valid, bit 1 tie,
// bit 2 zero: every term of the chunk (group) is +0 or -0.
constexpr int kXsValid = 1, kXsTie = 2, kXsZero = 4;
__device__ __forceinline__ int xs_pack(int E, int flags) { return ((E + 2048) << 3) | flags; }
__device__ __forceinline__ int xs_exp(int ef) { return (ef >> 3) - 2048; }
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
  if (E < -1000 || E > 1000) {
    bool zero = true;
    for (int k = 0; k < len; ++k) zero = zero && __ldcg(p + (size_t)k * step) == 0.0;
    out_ef = xs_pack(E < -2000 ? -2000 : E, zero ? kXsZero : 0);
    return;
  }
  const double sc = xs_pow2(-E);
  long long P = 0, r = 0, lo = 0x7fffffffffffffffll, hi = -0x7fffffffffffffffll - 1;
  long long loA = 0, hiA = 0;
  bool tie = false, ok = true, zero = true;
  for (int k0 = 0; k0 < len; k0 += 8) {
    double v[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = (k0 + i < len) ? __ldcg(p + (size_t)(k0 + i) * step) : 0.0;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      if (k0 + i >= len) break;
      zero = zero && v[i] == 0.0;
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
  out_ef = xs_pack(E, (ok ? kXsValid : 0) | (tie ? kXsTie : 0) | (zero ? kXsZero : 0));
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

// The terms of chunk j, lane k holding terms k, k + 32 and k + 64.
struct XsChunkTerms {
  double v0, v1, v2;
  int len;
};
__device__ __forceinline__ XsChunkTerms xs_load_chunk(const XsSum& s, const XsGeom& g, int j) {
  const int lane = threadIdx.x & 31;
  int tile, r, len;
  xs_chunk(s, g, j, tile, r, len);
  const double* p = xs_block(s, tile) + xs_at(0, r);
  XsChunkTerms c;
  c.len = len;
  c.v0 = (lane < len) ? __ldcg(p + lane) : 0.0;
  c.v1 = (lane + 32 < len) ? __ldcg(p + lane + 32) : 0.0;
  c.v2 = (lane + 64 < len) ? __ldcg(p + lane + 64) : 0.0;
  return c;
}

// S + t_0 + ... + t_{cnt-1} in sequence for up to 64 terms (lane k holds t_k
// in va and t_{32+k} in vb), by the warp: at the exponent of the exact
// running sum every lane converts its terms to units of the ulp, a prefix
// sum over the lanes gives the running mantissa after every term, and the
// run stops at the first term whose sum leaves the binade or is a tie (or
// whose running sum cannot be split); that one term is added in floating
// point, and the walk goes on from the next term.  Both halves are
// converted and prefix-summed at once, so a run that stays in one binade
// costs one pass over all 64 terms, and a run that crosses a binade once
// costs two.  After two passes in a row that make no progress the rest goes
// one addition after the other.
__device__ __forceinline__ double xs_add_lanes64(double S, double va, double vb, int cnt) {
  const int lane = threadIdx.x & 31;
  auto term = [&](int t) { return __shfl_sync(0xffffffffu, t < 32 ? va : vb, t & 31); };
  int pos = 0, stalls = 0;
  while (pos < cnt) {
    int E;
    long long m;
    if (!xs_split(S, E, m)) {
      S = __dadd_rn(S, term(pos));
      ++pos;
      continue;
    }
    const double sc = xs_pow2(-E);
    const bool actA = lane >= pos && lane < cnt, actB = lane + 32 >= pos && lane + 32 < cnt;
    const double qa = va * sc, qb = vb * sc;
    bool okA = actA && fabs(qa) < 36028797018963968.0, okB = actB && fabs(qb) < 36028797018963968.0;
    long long ca = 0, cb = 0;
    if (okA) {
      ca = __double2ll_rn(qa);
      okA = fabs(qa - (double)ca) != 0.5;
    }
    if (okB) {
      cb = __double2ll_rn(qb);
      okB = fabs(qb - (double)cb) != 0.5;
    }
    unsigned long long ia = actA ? (unsigned long long)ca : 0ull, ib = actB ? (unsigned long long)cb : 0ull;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned long long ta = __shfl_up_sync(0xffffffffu, ia, o);
      const unsigned long long tb = __shfl_up_sync(0xffffffffu, ib, o);
      if (lane >= o) {
        ia += ta;
        ib += tb;
      }
    }
    const unsigned long long totA = __shfl_sync(0xffffffffu, ia, 31);
    const long long miA = m + (long long)ia, miB = m + (long long)(totA + ib);   // mantissas after the terms
    const bool neg = m < 0;
    const unsigned badA = __ballot_sync(0xffffffffu, actA && !(okA && xs_in_range(miA, neg)));
    const unsigned badB = __ballot_sync(0xffffffffu, actB && !(okB && xs_in_range(miB, neg)));
    const int first = badA ? __ffs(badA) - 1 : (badB ? 32 + __ffs(badB) - 1 : cnt);
    if (first > pos) {
      const int t = first - 1;
      S = (double)__shfl_sync(0xffffffffu, t < 32 ? miA : miB, t & 31) * xs_pow2(E);
    }
    if (first >= cnt) break;
    S = __dadd_rn(S, term(first));
    if (first == pos && ++stalls >= 2) {   // the sum changes binade term after term here
      for (int t = first + 1; t < cnt; ++t) S = __dadd_rn(S, term(t));
      return S;
    }
    if (first > pos) stalls = 0;
    pos = first + 1;
  }
  return S;
}

// fl(... fl(fl(S + p_0) + p_1) ... + p_{len-1}) for a chunk's terms, by the
// warp (every lane returns the same value): where the terms are small
// against the running sum (its binade changes at few of them) in binade
// runs of up to 64 terms, else one addition after the other.
__device__ __forceinline__ double xs_add_terms(double S, const XsChunkTerms& c) {
  const int lane = threadIdx.x & 31;
  const int n64 = c.len < 64 ? c.len : 64;
  double a = (lane < n64 ? fabs(c.v0) : 0.0) + (lane + 32 < n64 ? fabs(c.v1) : 0.0);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
  if (a < fabs(S) * 0.015625) {   // false for S = 0 and non-finite values
    S = xs_add_lanes64(S, c.v0, c.v1, n64);
  } else {
    S = xs_add_seq(S, c.v0, c.len < 32 ? c.len : 32);
    if (c.len > 32) S = xs_add_seq(S, c.v1, c.len < 64 ? c.len - 32 : 32);
  }
  if (c.len > 64) S = xs_add_seq(S, c.v2, c.len - 64);
  return S;
}
__device__ __forceinline__ double xs_add_chunk(const XsSum& s, const XsGeom& g, int j, double S) {
  return xs_add_terms(S, xs_load_chunk(s, g, j));
}

// Walk counters of one warp: chunks added term by term and their cycles.
struct XsWalkCount {
  unsigned long long chunks, slow, slow_cycles;
};

// S + the terms of chunks [j0, j1) of one sum in order, by one warp (every
// lane returns it), from the chunk summaries: 32 chunks at a time.
__device__ double xs_walk_chunks(const XsSum& s, const XsGeom& g, int j0, int j1, double S, XsWalkCount& wc) {
  unsigned long long slow = 0, slow_cycles = 0;
  const int lane = threadIdx.x & 31;
  const unsigned lt_mask = (1u << lane) - 1u;   // lanes below this one
  const int nch = j1;
  int j = j0;
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
  load(j0 + lane, nef, nX, nlo, nhi, nR, nloA, nhiA);
  for (int jb = j0; jb < nch && !isnan(S); jb += 32) {
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
      if (isnan(S)) break;
      int E;
      long long m;
      if (!xs_split(S, E, m)) {
        // +0 plus a chunk of zeros stays +0
        if (__double_as_longlong(S) == 0 && (__shfl_sync(0xffffffffu, ef, j - jb) & kXsZero)) {
          ++j;
          continue;
        }
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
  wc.chunks += (unsigned long long)(j1 - j0);
  wc.slow += slow;
  wc.slow_cycles += slow_cycles;
  return S;
}


// Chunk group ty of a sum: the chunks of tile row ty (rows [8 ty, 8 ty + 8),
// the last group to the last row), a contiguous run of the walk order.
__device__ __forceinline__ void xs_group_range(const XsSum& s, const XsGeom& g, int ty, int& j0, int& j1) {
  j0 = ty * 8 * g.nx;
  j1 = ((ty == g.ny - 1) ? s.rows : ty * 8 + 8) * g.nx;
}

// Summary of chunk group ty (one warp): when every chunk of it has a summary
// at the first chunk's exponent, without a tie and with moderate sizes, the
// sum of their c's (gX) and the smallest and largest partial sum relative to
// the group start (gmn, gmx); else the group is marked without one (the walk
// then takes its chunks).  Sizes below 2^53 per chunk keep the int64 sums
// exact; a usable run never needs more (its partial sums span < 2^52).
__device__ void xs_group_summary(const XsSum& s, const XsGeom& g, int ty) {
  const int lane = threadIdx.x & 31;
  int j0, j1;
  xs_group_range(s, g, ty, j0, j1);
  const int ef0 = __ldcg(s.ef + j0);
  const long long lim = 1ll << 53;
  long long carry = 0, mn = 0x7fffffffffffffffll, mx = -0x7fffffffffffffffll - 1;
  bool ok = (ef0 & kXsValid) && !(ef0 & kXsTie);
  bool zero = true;
  for (int jb = j0; jb < j1; jb += 32) {
    const int j = jb + lane;
    zero = zero && __all_sync(0xffffffffu, j >= j1 || (__ldcg(s.ef + j) & kXsZero));
  }
  for (int jb = j0; jb < j1 && ok; jb += 32) {
    const int j = jb + lane;
    const bool in = j < j1;
    const int ef = in ? __ldcg(s.ef + j) : ef0;
    const long long X = in ? __ldcg(s.X + j) : 0;
    const long long lo = in ? __ldcg(s.mnB + j) : 0, hi = in ? __ldcg(s.mxB + j) : 0;
    const bool bad = in && (!(ef & kXsValid) || (ef & kXsTie) || xs_exp(ef) != xs_exp(ef0) || X >= lim ||
                            X <= -lim || lo >= lim || lo <= -lim || hi >= lim || hi <= -lim);
    if (__any_sync(0xffffffffu, bad)) {
      ok = false;
      break;
    }
    long long inc = X;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const long long t = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += t;
    }
    const long long P = carry + inc - X;   // partial c-sum at this chunk's start
    long long a = in ? P + lo : 0x7fffffffffffffffll, b = in ? P + hi : -0x7fffffffffffffffll - 1;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const long long ta = __shfl_xor_sync(0xffffffffu, a, o), tb = __shfl_xor_sync(0xffffffffu, b, o);
      a = ta < a ? ta : a;
      b = tb > b ? tb : b;
    }
    mn = a < mn ? a : mn;
    mx = b > mx ? b : mx;
    carry += __shfl_sync(0xffffffffu, inc, 31);
  }
  if (lane == 0) {
    __stcg(s.gX + ty, carry);
    __stcg(s.gmn + ty, mn);
    __stcg(s.gmx + ty, mx);
    __stcg(s.gef + ty, xs_pack(xs_exp(ef0), (ok ? kXsValid : 0) | (zero ? kXsZero : 0)));
  }
}

// The sequential sum 0 + t_0 + t_1 + ... of one sum, by one warp (every lane
// returns it): 32 chunk groups at a time from their summaries (a prefix sum
// over the lanes gives the mantissa at every group start), a group without
// a usable summary or whose partial sums leave the binade by its chunks
// (xs_walk_chunks).  Needs the summaries of every chunk and group.
__device__ double xs_drive(const XsSum& s, const XsGeom& g, unsigned long long* prof) {
  const long long t_start = clock64();
  XsWalkCount wc{0, 0, 0};
  const int lane = threadIdx.x & 31;
  const int ng = g.ny;
  double S = 0.0;
  int q = 0;
  auto load = [&](int qn, int& ef, long long& X, long long& lo, long long& hi) {
    const bool in = qn < ng;
    ef = in ? __ldcg(s.gef + qn) : 0;
    X = in ? __ldcg(s.gX + qn) : 0;
    lo = in ? __ldcg(s.gmn + qn) : 0;
    hi = in ? __ldcg(s.gmx + qn) : 0;
  };
  int nef;
  long long nX, nlo, nhi;
  load(lane, nef, nX, nlo, nhi);
  for (int qb = 0; qb < ng && !isnan(S); qb += 32) {
    const bool in = qb + lane < ng;
    const int ef = nef;
    const long long X = nX, lo = nlo, hi = nhi;
    load(qb + lane + 32, nef, nX, nlo, nhi);
    while (q < qb + 32 && q < ng) {
      if (isnan(S)) break;
      int E;
      long long m;
      int first = q - qb;
      // +0 plus a group of zeros stays +0
      if (__double_as_longlong(S) == 0 && (__shfl_sync(0xffffffffu, ef, q - qb) & kXsZero)) {
        ++q;
        continue;
      }
      if (xs_split(S, E, m)) {
        const bool neg = m < 0;
        const int o = q - qb;
        const bool act = lane >= o && in;
        const bool use = act && (ef & kXsValid) && xs_exp(ef) == E;
        const unsigned long long delta = use ? (unsigned long long)X : 0ull;
        unsigned long long inc = delta;
#pragma unroll
        for (int o2 = 1; o2 < 32; o2 <<= 1) {
          const unsigned long long tt = __shfl_up_sync(0xffffffffu, inc, o2);
          if (lane >= o2) inc += tt;
        }
        const long long mi = m + (long long)(inc - delta);   // mantissa at this group's start
        const bool good = use && xs_in_range(mi + lo, neg) && xs_in_range(mi + hi, neg);
        const unsigned bad = __ballot_sync(0xffffffffu, act && !good);
        const int last = (ng - qb < 32 ? ng - qb : 32);
        first = bad ? __ffs(bad) - 1 : last;
        const long long mf = __shfl_sync(0xffffffffu, mi + (long long)delta, (first > 0 ? first : 1) - 1);
        if (first > o) S = (double)mf * xs_pow2(E);
      }
      q = qb + first;
      if (q < qb + 32 && q < ng) {
        int j0, j1;
        xs_group_range(s, g, q, j0, j1);
        S = xs_walk_chunks(s, g, j0, j1, S, wc);
        ++q;
      }
    }
  }
  if (prof && lane == 0) {
    atomicAdd(prof + 4, wc.chunks);
    atomicAdd(prof + 5, wc.slow);
    atomicAdd(prof + 6, wc.slow_cycles);
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
  xs_summarise(xs_block(s, t) + xs_at(0, r), 1, len, __ldcg(s.ef + j), X, R, lo, hi, loA, hiA, ef);
  __stcg(s.X + j, X);
  __stcg(s.R + j, R);
  __stcg(s.mnB + j, lo);
  __stcg(s.mxB + j, hi);
  __stcg(s.mnA + j, loA);
  __stcg(s.mxA + j, hiA);
  __stcg(s.ef + j, ef);
}

// Tile rows of chunk summaries per task tile of the summary pass (every
// thread one chunk row of a term block, nx blocks per tile row), and the task
// tiles of ns sums.
__host__ __device__ inline int xs_rows_per_task(const XsGeom& g) {
  const int r = 256 / (g.nx * kXsBR);
  return r < 1 ? 1 : r;
}
__host__ __device__ inline int xs_summary_tasks(int ns, int n) {
  const XsGeom g(n);
  const int rt = xs_rows_per_task(g);
  return (ns * g.ny + rt - 1) / rt;
}

// Step 2, task tile `task` (the whole CTA of 256 threads, every thread
// calls): the chunk summaries of its tile rows (groups), then the group
// summaries, one warp per group.  sum(k) gives sum k of the pass.
template <class SumOf>
__device__ void xs_summary_task(SumOf&& sum, int ns, const XsGeom& g, int task) {
  const int rt = xs_rows_per_task(g);
  const int q0 = task * rt;
  int nq = ns * g.ny - q0;
  nq = nq < rt ? nq : rt;
  const int per = g.nx * kXsBR;
  for (int job = threadIdx.x; job < nq * per; job += blockDim.x) {
    const int q = q0 + job / per, rem = job - (job / per) * per;
    const int k = q / g.ny, ty = q - k * g.ny;
    xs_summary_row(sum(k), g, ty * g.nx + rem / kXsBR, rem % kXsBR);
  }
  __threadfence();
  __syncthreads();
  for (int w = threadIdx.x >> 5; w < nq; w += blockDim.x >> 5) {
    const int q = q0 + w, k = q / g.ny;
    xs_group_summary(sum(k), g, q - k * g.ny);
  }
  __threadfence();
  __syncthreads();
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
