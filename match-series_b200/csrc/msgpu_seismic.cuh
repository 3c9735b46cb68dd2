// msgpu_seismic.cuh -- the energy of the seismic line-shift model
// (matchSeismicSeries): the data term FELineShiftRegisEnergy
// (registration.h:2137-2193), a 1-D normalized cross-correlation per image
// line under a shift of the line along x, and the anisotropic regulariser of
// findXShift (matchSeries.h:819-845), K = stiffX + yRegFactor * stiffY.
//
// k_lineshift: one CTA per line (blockIdx.x) and image (blockIdx.y); the
// line's reference, deformed template and work vectors live in shared memory.
// The three global sums of a line (mass-weighted mean, norm, correlation) are
// fixed-order block reductions; everything else follows the reference's
// arithmetic step by step (the 1-D mass band assembled on the host in element
// order, FastDeformImage with Vector::interpolate, CrossCorrelationForce at the
// two Gauss points of each element, node sums in element order).
#pragma once

#include "msgpu_level.cuh"

namespace msg {

constexpr int kLineThreads = 256;

// Assembled 1-D mass band (DiagBandMatrix<.,1,1>) of a line of n nodes:
// row 0 (d0, u0), interior rows (l, d, u), row n-1 (ln, dn); Gauss points
// and basis values; h = 1/(n-1).
struct LineTables {
  double d0, u0, l, d, u, ln, dn;
  double h;
  double g[2];
  double bq[2][2];
};

struct LineArgs {
  int nx, ny;
  size_t img_stride;           // elements between images
  const double* R;
  const double* T;
  const double* phi;
  double* e_line;              // ny per image
  double* de;                  // nullable: nx*ny per image
  LineTables t;
  const double* nr_pre;        // nullable: the reference lines already normalised (k_lineshift_prep_ref)
  const double* phi_row;       // nullable: one shift per line (phi = phi_row[y] on the whole line)
  double* de_row;              // nullable (with phi_row): the derivative summed along each line, in x order
  unsigned* done;              // nullable: per-image line counter; the last line's CTA writes the total
  double* e_total;             // one per image (with done): mean of the line energies in line order
};

__device__ __forceinline__ double line_block_sum(double v, double* red) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  __syncthreads();
  if (lane == 0) red[wid] = v;
  __syncthreads();
  double s = 0.0;
  for (int w = 0; w < kLineThreads / 32; ++w) s += red[w];
  return s;
}

__device__ __forceinline__ double line_mass_row(const LineTables& t, const double* u, int i, int n) {
  double r = 0.;
  if (i == 0) {
    r += t.d0 * u[0];
    r += t.u0 * u[1];
  } else if (i == n - 1) {
    r += t.ln * u[n - 2];
    r += t.dn * u[n - 1];
  } else {
    r += t.l * u[i - 1];
    r += t.d * u[i];
    r += t.u * u[i + 1];
  }
  return r;
}

// normalizeImageForNCC on a line in shared memory: v <- (v - mean)/norm,
// returns the norm (tmp: scratch of n).
__device__ double line_normalize(const LineTables& t, double* v, double* tmp, int n, double* red) {
  double part = 0.0;
  for (int i = threadIdx.x; i < n; i += kLineThreads) part += line_mass_row(t, v, i, n);
  const double mean = line_block_sum(part, red);
  for (int i = threadIdx.x; i < n; i += kLineThreads) v[i] += -mean;
  __syncthreads();
  part = 0.0;
  for (int i = threadIdx.x; i < n; i += kLineThreads) part += v[i] * line_mass_row(t, v, i, n);
  const double var = sqrt(line_block_sum(part, red));
  if (!(fabs(var - 0.) < 1e-15))
    for (int i = threadIdx.x; i < n; i += kLineThreads) v[i] /= var;
  __syncthreads();
  (void)tmp;
  return var;
}

// With a.done: the CTA of the image's last finished line adds the line
// energies in line order (no CTA waits for another: a counter decides who
// is last) and resets the counter for the next launch.
// buf: the CTA's line buffer (cap doubles), free again at this point.
__device__ __forceinline__ void line_total(const LineArgs& a, double* buf, int cap) {
  if (!a.done) return;
  __shared__ int last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = (atomicAdd(a.done + blockIdx.y, 1u) == (unsigned)a.ny - 1) ? 1 : 0;
  __syncthreads();
  if (!last) return;
  __threadfence();
  const double* e = a.e_line + (size_t)blockIdx.y * a.ny;
  double s = 0.;
  for (int y0 = 0; y0 < a.ny; y0 += cap) {
    const int m = min(cap, a.ny - y0);
    for (int i = threadIdx.x; i < m; i += kLineThreads) buf[i] = __ldcg(e + y0 + i);
    __syncthreads();
    if (threadIdx.x == 0)
      for (int i = 0; i < m; ++i) s += buf[i];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    a.e_total[blockIdx.y] = s / a.ny;
    a.done[blockIdx.y] = 0u;
  }
}

// The reference lines normalised once (normalizeImageForNCC of
// registration.h:2137-2193 on each line; R does not change during a
// descent), for k_lineshift's nr_pre.
__global__ void __launch_bounds__(kLineThreads) k_lineshift_prep_ref(const double* R, int nx, size_t img_stride,
                                                                    LineTables t, double* nr_out) {
  extern __shared__ double lsm[];
  __shared__ double red[kLineThreads / 32];
  const int n = nx;
  const size_t base = (size_t)blockIdx.y * img_stride + (size_t)blockIdx.x * n;
  double* nr = lsm;
  double* tmp = lsm + n;
  if (isnan(R[base])) {
    for (int i = threadIdx.x; i < n; i += kLineThreads) nr_out[base + i] = R[base + i];
    return;
  }
  for (int i = threadIdx.x; i < n; i += kLineThreads) nr[i] = R[base + i];
  __syncthreads();
  line_normalize(t, nr, tmp, n, red);
  for (int i = threadIdx.x; i < n; i += kLineThreads) nr_out[base + i] = nr[i];
}

__global__ void __launch_bounds__(kLineThreads) k_lineshift(LineArgs a) {
  extern __shared__ double lsm[];
  __shared__ double red[kLineThreads / 32];
  const int n = a.nx, y = blockIdx.x;
  const size_t base = (size_t)blockIdx.y * a.img_stride + (size_t)y * n;
  const double* R = a.R + base;
  const double* T = a.T + base;
  const double* phi = a.phi_row ? nullptr : a.phi + base;
  const double prow = a.phi_row ? a.phi_row[(size_t)blockIdx.y * a.ny + y] : 0.0;
  double* nr = lsm;            // normalised reference line
  double* nt = lsm + n;        // deformed, then normalised template line
  double* tmp = lsm + 2 * n;   // (M nt), then the force weights
  const LineTables& t = a.t;
  if (isnan(R[0]) || isnan(T[0])) {
    if (threadIdx.x == 0) a.e_line[(size_t)blockIdx.y * a.ny + y] = 0.0;
    if (a.de)
      for (int i = threadIdx.x; i < n; i += kLineThreads) a.de[base + i] = 0.0;
    if (a.de_row && threadIdx.x == 0) a.de_row[(size_t)blockIdx.y * a.ny + y] = 0.0;
    line_total(a, lsm, 3 * n);
    return;
  }
  for (int i = threadIdx.x; i < n; i += kLineThreads) {
    nr[i] = a.nr_pre ? a.nr_pre[base + i] : R[i];
    // doFastDeformImage<., QC_1D> (deformations.h:111-137), Vector::interpolate (vec.h:461-472)
    double ds = i + (phi ? phi[i] : prow) / t.h;
    ds = ds < 0. ? 0. : (ds > (double)(n - 1) ? (double)(n - 1) : ds);
    const int p = (int)ds;
    const double pf = ds - p;
    nt[i] = (p == n - 1) ? T[p] : (1 - pf) * T[p] + pf * T[p + 1];
  }
  __syncthreads();
  if (!a.nr_pre) line_normalize(t, nr, tmp, n, red);
  const double var = line_normalize(t, nt, tmp, n, red);
  double part = 0.0;
  for (int i = threadIdx.x; i < n; i += kLineThreads) part += line_mass_row(t, nt, i, n) * nr[i];
  const double energy = -line_block_sum(part, red);
  if (threadIdx.x == 0) a.e_line[(size_t)blockIdx.y * a.ny + y] = energy;
  if (!a.de && !a.de_row) {
    line_total(a, lsm, 3 * n);
    return;
  }
  // VariationOfNormalizedCrossCorrelationEnergy: temp = (normR + normT * E) / var
  for (int i = threadIdx.x; i < n; i += kLineThreads) {
    double v = nr[i];
    v += nt[i] * energy;
    if (!(fabs(var - 0.) < 1e-15)) v /= var;
    tmp[i] = v;
  }
  __syncthreads();
  // CrossCorrelationForce per element at its two Gauss points; node i takes
  // element i-1 (as its right node) first, then element i (as its left node)
  auto elem = [&](int e, int b) -> double {
    double nl[2];
#pragma unroll
    for (int q = 0; q < 2; ++q) {
      double off = 0.;
      off += (phi ? phi[e] : prow) * t.bq[0][q];
      off += (phi ? phi[e + 1] : prow) * t.bq[1][q];
      const double tc = ((double)e + t.g[q]) + off / t.h;
      int el = (short)tc;
      double loc = tc - el;
      if (el == n - 1 && loc == 0) { el = n - 2; loc = 1; }
      if (tc < 0. || el < 0 || el >= n - 1) { nl[q] = 0.; continue; }
      double gr = 0.;
      double v = -1. / t.h;
      v *= T[el];
      gr += v;
      v = 1. / t.h;
      v *= T[el + 1];
      gr += v;
      double tq = 0.;
      tq += tmp[e] * t.bq[0][q];
      tq += tmp[e + 1] * t.bq[1][q];
      nl[q] = gr * -tq;
    }
    double acc = 0.;
#pragma unroll
    for (int q = 0; q < 2; ++q) acc += nl[q] * (t.bq[b][q] * 0.5);
    return t.h * acc;
  };
  for (int i = threadIdx.x; i < n; i += kLineThreads) {
    double d = 0.;
    if (i > 0) d += elem(i - 1, 1);
    if (i < n - 1) d += elem(i, 0);
    d /= a.ny;
    if (a.de) a.de[base + i] = d;
    if (a.de_row) nr[i] = d;   // nr is free once tmp holds the force weights
  }
  if (a.de_row) {
    // ScalarArray<QC_2D>::sumInXDirectionTo (scalarArray.h:1395-1402): from 0, in x order
    __syncthreads();
    if (threadIdx.x == 0) {
      double sum = 0.;
      for (int i = 0; i < n; ++i) sum += nr[i];
      a.de_row[(size_t)blockIdx.y * a.ny + y] = sum;
    }
  }
  line_total(a, lsm, 3 * n);
}

// Sum of the line energies in line order, divided by the line count: one
// block per image stages the lines in shared memory (coalesced), one thread
// adds them in order.
__global__ void __launch_bounds__(256) k_lineshift_total(const double* e_line, int ny, double* out) {
  __shared__ double buf[1024];
  const double* e = e_line + (size_t)blockIdx.x * ny;
  double s = 0.;
  for (int y0 = 0; y0 < ny; y0 += 1024) {
    const int m = min(1024, ny - y0);
    for (int i = threadIdx.x; i < m; i += blockDim.x) buf[i] = e[y0 + i];
    __syncthreads();
    if (threadIdx.x == 0)
      for (int i = 0; i < m; ++i) s += buf[i];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[blockIdx.x] = s / ny;
}

// Sum of n values in a fixed order for a block of 256 threads: strided
// per-thread sums, a shuffle tree per warp, the eight warps in order
// (thread 0 holds the result).
__device__ __forceinline__ double block_fixed_sum(const double* v, int n, double* red) {
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += 256) s += v[i];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < 8; ++w) t += red[w];
  return t;
}

// findXShift's regulariser: K phi with the assembled nine-point rows of the
// nine node classes (first / interior / last along x and y), and the partial
// sums of phi . K phi per block for E = 1/2 phi.K phi.
struct XRegTables {
  double st[9][3][3];
};

// With done (one counter per image): the CTA that finishes an image's last
// block sums its partials like k_xshift_reg_total (E = 1/2 phi.K phi into
// e_total) and resets the counter.
__global__ void __launch_bounds__(256) k_xshift_reg(XRegTables tb, int nx, int ny, size_t img_stride,
                                                    const double* phi, double* kphi, double* part,
                                                    unsigned* done, double* e_total) {
  __shared__ double red[8];
  const double* p = phi + (size_t)blockIdx.y * img_stride;
  double* k = kphi + (size_t)blockIdx.y * img_stride;
  const int N = nx * ny;
  double acc = 0.0;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < N; r += gridDim.x * blockDim.x) {
    const int x = r % nx, y = r / nx;
    const int cls = (x == 0 ? 0 : (x == nx - 1 ? 2 : 1)) + 3 * (y == 0 ? 0 : (y == ny - 1 ? 2 : 1));
    double d = 0.;
#pragma unroll
    for (int j = -1; j <= 1; ++j)
#pragma unroll
      for (int i = -1; i <= 1; ++i) {
        const int X = x + i, Y = y + j;
        if (X >= 0 && X < nx && Y >= 0 && Y < ny) d += tb.st[cls][j + 1][i + 1] * p[X + (size_t)Y * nx];
      }
    k[r] = d;
    acc += d * p[r];
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < 8; ++w) s += red[w];
    part[(size_t)blockIdx.y * gridDim.x + blockIdx.x] = s;
  }
  if (!done) return;
  __shared__ int last;
  __shared__ double red2[8];
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = (atomicAdd(done + blockIdx.y, 1u) == gridDim.x - 1) ? 1 : 0;
  __syncthreads();
  if (!last) return;
  __threadfence();
  const double* pp = part + (size_t)blockIdx.y * gridDim.x;
  double v = 0.0;
  for (int i = threadIdx.x; i < (int)gridDim.x; i += 256) v += __ldcg(pp + i);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red2[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < 8; ++w) t += red2[w];
    e_total[blockIdx.y] = 0.5 * t;
    done[blockIdx.y] = 0u;
  }
}

// E = 1/2 phi.K phi from the block partials, one block (256 threads) per image
__global__ void __launch_bounds__(256) k_xshift_reg_total(const double* part, int nblocks, double* out) {
  __shared__ double red[8];
  const double s = block_fixed_sum(part + (size_t)blockIdx.x * nblocks, nblocks, red);
  if (threadIdx.x == 0) out[blockIdx.x] = 0.5 * s;
}

// findXShift's regulariser with laplaceWeight > 0 (matchSeries.h:828-838):
// the 25-point rows of laplaceWeight L M^-1 L + stiffX + yRegFactor stiffY
// for the 25 node classes (first, second, interior, second last, last along
// x and y), applied in column order (the reference's CSR rows are sorted by
// column, i.e. by offset (dy, dx)); partial sums of phi . K phi per block,
// the image's total by the last block as in k_xshift_reg.
struct XLapTables {
  double st[25][25];   // [class cx + 5 cy][(dy + 2) * 5 + (dx + 2)]
};

__device__ __forceinline__ int lap_class(int x, int n) {
  return x == 0 ? 0 : (x == 1 ? 1 : (x == n - 1 ? 4 : (x == n - 2 ? 3 : 2)));
}

__global__ void __launch_bounds__(256) k_xshift_reg_lap(XLapTables tb, int nx, int ny, size_t img_stride,
                                                        const double* phi, double* kphi, double* part,
                                                        unsigned* done, double* e_total) {
  __shared__ double red[8];
  const double* p = phi + (size_t)blockIdx.y * img_stride;
  double* k = kphi + (size_t)blockIdx.y * img_stride;
  const int N = nx * ny;
  double acc = 0.0;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < N; r += gridDim.x * blockDim.x) {
    const int x = r % nx, y = r / nx;
    const double* row = tb.st[lap_class(x, nx) + 5 * lap_class(y, ny)];
    double d = 0.;
#pragma unroll
    for (int j = -2; j <= 2; ++j)
#pragma unroll
      for (int i = -2; i <= 2; ++i) {
        const int X = x + i, Y = y + j;
        if (X >= 0 && X < nx && Y >= 0 && Y < ny) d += row[(j + 2) * 5 + (i + 2)] * p[X + (size_t)Y * nx];
      }
    k[r] = d;
    acc += d * p[r];
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < 8; ++w) s += red[w];
    part[(size_t)blockIdx.y * gridDim.x + blockIdx.x] = s;
  }
  if (!done) return;
  __shared__ int last;
  __shared__ double red2[8];
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = (atomicAdd(done + blockIdx.y, 1u) == gridDim.x - 1) ? 1 : 0;
  __syncthreads();
  if (!last) return;
  __threadfence();
  const double* pp = part + (size_t)blockIdx.y * gridDim.x;
  double v = 0.0;
  for (int i = threadIdx.x; i < (int)gridDim.x; i += 256) v += __ldcg(pp + i);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red2[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < 8; ++w) t += red2[w];
    e_total[blockIdx.y] = 0.5 * t;
    done[blockIdx.y] = 0u;
  }
}

// The template smoothed along x for findXShiftYConst (matchSeries.h:886-896):
// ScalarArray<QC_2D>::applyLinearFilterTo with a (2o+1) x (2o+1) kernel whose
// middle row is 1/(2o+1) and the other rows 0 (scalarArray.cpp:936-965: the
// whole window in row order, periodic outside the array, so the zero rows
// still carry a NaN or Inf of their pixels).
__global__ void k_box_x(const double* T, int nx, int ny, int o, double* out) {
  const double k = 1. / (double)(2 * o + 1);
  const int N = nx * ny;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < N; r += gridDim.x * blockDim.x) {
    const int x = r % nx, y = r / nx;
    double val = 0.0;
    for (int oy = -o; oy <= o; ++oy) {
      int Y = y + oy;
      if (Y < 0) Y += ny; else if (Y > ny - 1) Y = Y % ny;
      for (int ox = -o; ox <= o; ++ox) {
        int X = x + ox;
        if (X < 0) X += nx; else if (X > nx - 1) X = X % nx;
        val += (oy == 0 ? k : 0.0) * T[(size_t)Y * nx + X];
      }
    }
    out[r] = val;
  }
}

// --- vector kernels of the seismic descent ----------------------------------
// out[i] = a[i] + s * b[i]  (also the in-place updates, with out == a)
// replaceEmptyLinesWithNaN (matchSeismicSeries.h:141-157): a line whose
// squared norm is 0 becomes quiet NaNs.  The norm of the reference is a sum of
// rounded squares, which are never negative, so it is 0 exactly when every
// square rounds to 0, whatever the order of the additions (a NaN sample makes
// it NaN and keeps the line): one block per line tests each square.
__global__ void __launch_bounds__(256) k_empty_lines_nan(double* img, int nx, int* replaced) {
  double* line = img + (size_t)blockIdx.x * nx;
  int nonzero = 0;
  for (int i = threadIdx.x; i < nx; i += 256) {
    const double v = line[i];
    nonzero |= !(v * v == 0.0);
  }
  if (__syncthreads_or(nonzero)) return;
  for (int i = threadIdx.x; i < nx; i += 256) line[i] = __longlong_as_double(0x7ff8000000000000LL);
  if (threadIdx.x == 0 && replaced) atomicAdd(replaced, 1);
}

// removeEmptyLinesFromImage (matchSeismicSeries.h:101-136), first pass: a
// line is kept unless its squared norm is 0 (every square rounds to 0, see
// k_empty_lines_nan) or it holds NaNs only; one block per line.
__global__ void __launch_bounds__(256) k_line_kept(const double* img, int nx, int* kept) {
  const double* line = img + (size_t)blockIdx.x * nx;
  int nonzero = 0, number = 0;
  for (int i = threadIdx.x; i < nx; i += 256) {
    const double v = line[i];
    nonzero |= !(v * v == 0.0);
    number |= !isnan(v);
  }
  const int nz = __syncthreads_or(nonzero);
  const int nn = __syncthreads_or(number);
  if (threadIdx.x == 0) kept[blockIdx.x] = nz && nn;
}

// Second pass: output line y copies source line map[y], or is zero for -1.
__global__ void __launch_bounds__(256) k_gather_lines(const double* img, int nx, const int* map, double* out) {
  const int src = map[blockIdx.x];
  double* o = out + (size_t)blockIdx.x * nx;
  for (int i = threadIdx.x; i < nx; i += 256) o[i] = src >= 0 ? img[(size_t)src * nx + i] : 0.0;
}

__global__ void k_axpy(const double* a, double s, const double* b, double* out, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double v = a[i];
    v += s * b[i];
    out[i] = v;
  }
}
__global__ void k_scale(double* a, double s, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) a[i] *= s;
}
__global__ void k_divide(double* a, double s, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) a[i] /= s;
}
__global__ void k_mul(const double* a, double s, double* out, int n) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = a[i] * s;
}
// Parity fold of the H1 metric's x transform: the cosine modes satisfy
// v_k(nx-1-i) = (-1)^k v_k(i), so the transform of column j splits into the
// even modes applied to S_i = g_i + g_(nx-1-i) (S_mid = g_mid for odd nx) and
// the odd modes applied to A_i = g_i - g_(nx-1-i): two products of half size.
// f (nx x ny, column-major, leading dimension nx): rows 0..ne-1 = S, rows
// ne..nx-1 = A.
__global__ void k_xfold(const double* g, double* f, int nx, int ny) {
  const int ne = (nx + 1) / 2, no = nx / 2;
  const int total = nx * ny;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
    const int j = t / nx, r = t - j * nx;
    const double* c = g + (size_t)j * nx;
    double v;
    if (r < ne) v = (r < no) ? c[r] + c[nx - 1 - r] : c[r];
    else v = c[r - ne] - c[nx - 1 - (r - ne)];
    f[(size_t)j * nx + r] = v;
  }
}
// Inverse of the fold after the synthesis products: rows 0..ne-1 hold the
// even-mode sums E, rows ne..nx-1 the odd-mode sums O; g_i = E_i + O_i,
// g_(nx-1-i) = E_i - O_i, g_mid = E_mid.
__global__ void k_xunfold(const double* f, double* g, int nx, int ny) {
  const int ne = (nx + 1) / 2, no = nx / 2;
  const int total = nx * ny;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < total; t += gridDim.x * blockDim.x) {
    const int j = t / nx, i = t - j * nx;
    const double* c = f + (size_t)j * nx;
    double v;
    if (i < no) v = c[i] + c[ne + i];
    else if (i >= ne) v = c[nx - 1 - i] - c[ne + (nx - 1 - i)];
    else v = c[i];
    g[(size_t)j * nx + i] = v;
  }
}

// a[i] * b[i] summed per block in a fixed order (partials, then k_sum_part)
__global__ void __launch_bounds__(256) k_dot_part(const double* a, const double* b, int n, double* part) {
  __shared__ double red[8];
  double acc = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) acc += a[i] * b[i];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int w = 0; w < 8; ++w) s += red[w];
    part[blockIdx.x] = s;
  }
}
__global__ void __launch_bounds__(256) k_sum_part(const double* part, int n, double* out) {
  __shared__ double red[8];
  const double s = block_fixed_sum(part, n, red);
  if (threadIdx.x == 0) *out = s;
}
// Spectral scaling of the H1 metric: z[y][x] /= 1 + tau (lx[x] + ly[y])
// Vector kernels whose scalar lives on the device (the descent control of
// findXShift as a graph with device-side conditions): the same arithmetic as
// k_axpy / k_scale with the scalar read from memory.
__global__ void k_axpy_dev(const double* a, const double* s, const double* b, double* out, int n) {
  const double sv = *s;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double v = a[i];
    v += sv * b[i];
    out[i] = v;
  }
}
__global__ void k_scale_dev(double* a, const double* s, int n) {
  const double sv = *s;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) a[i] *= sv;
}
// phi += d when the accepted step *tau is not 0
__global__ void k_step_dev(double* phi, const double* d, const double* tau, int n) {
  if (*tau == 0) return;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    double v = phi[i];
    v += 1.0 * d[i];
    phi[i] = v;
  }
}
// the spectral scaling with tau = sigma^2 / 2 from the device's sigma
__global__ void k_spectral_scale_dev(double* z, const double* lx, const double* ly, const double* sigma, int nx,
                                     int ny) {
  const double sg = *sigma;
  const double tau = 0.5 * (sg * sg);
  const int N = nx * ny;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    const int x = i % nx, y = i / nx;
    z[i] /= 1.0 + tau * (lx[x] + ly[y]);
  }
}

__global__ void k_spectral_scale(double* z, const double* lx, const double* ly, double tau, int nx, int ny) {
  const int N = nx * ny;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
    const int x = i % nx, y = i / nx;
    z[i] /= 1.0 + tau * (lx[x] + ly[y]);
  }
}

// ---------------------------------------------------------------------------
// Dense FP64 products of the H1 metric's cosine-basis transforms, on the
// tensor pipe: C = op(A) op(B), column-major (the layout of the transforms:
// an nx x ny image with x fastest is an nx x ny column-major matrix), op a
// transpose when TA / TB.  A 64 x 64 tile of C per CTA (256 threads, 8 warps
// of 32 x 16), k in steps of 16 through shared memory, each warp issuing
// mma.sync m8n8k4 FP64 (DMMA) on fragments read from shared memory.
constexpr int kGemmBM = 64, kGemmBN = 64, kGemmBK = 16, kGemmPad = 2;

__device__ __forceinline__ void dmma_8x8x4(double& c0, double& c1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(c0), "+d"(c1)
               : "d"(a), "d"(b));
}

template <bool TA, bool TB>
__global__ void __launch_bounds__(256) k_dgemm(int M, int N, int K, const double* __restrict__ A, int lda,
                                              const double* __restrict__ B, int ldb, double* __restrict__ C,
                                              int ldc) {
  __shared__ double As[kGemmBK][kGemmBM + kGemmPad];   // As[k][m] = op(A)(m, k)
  __shared__ double Bs[kGemmBK][kGemmBN + kGemmPad];   // Bs[k][n] = op(B)(k, n)
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int bm = blockIdx.x * kGemmBM, bn = blockIdx.y * kGemmBN;
  const int wm = (warp & 1) * 32, wn = (warp >> 1) * 16;
  double acc[4][2][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
  for (int k0 = 0; k0 < K; k0 += kGemmBK) {
    // op(A) tile (64 x 16) and op(B) tile (16 x 64), zero outside the matrices
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int i = tid + 256 * r;
      int m, k;
      if (TA) { k = i % kGemmBK; m = i / kGemmBK; } else { m = i % kGemmBM; k = i / kGemmBM; }
      const int gm = bm + m, gk = k0 + k;
      double v = 0.0;
      if (gm < M && gk < K) v = TA ? A[gk + (size_t)gm * lda] : A[gm + (size_t)gk * lda];
      As[k][m] = v;
      int n;
      if (TB) { n = i % kGemmBN; k = i / kGemmBN; } else { k = i % kGemmBK; n = i / kGemmBK; }
      const int gn = bn + n, gk2 = k0 + k;
      double w = 0.0;
      if (gn < N && gk2 < K) w = TB ? B[gn + (size_t)gk2 * ldb] : B[gk2 + (size_t)gn * ldb];
      Bs[k][n] = w;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kGemmBK; kk += 4) {
      double a[4], b[2];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = As[kk + (lane & 3)][wm + 8 * i + (lane >> 2)];
#pragma unroll
      for (int j = 0; j < 2; ++j) b[j] = Bs[kk + (lane & 3)][wn + 8 * j + (lane >> 2)];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 2; ++j) dmma_8x8x4(acc[i][j][0], acc[i][j][1], a[i], b[j]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int m = bm + wm + 8 * i + (lane >> 2), n = bn + wn + 8 * j + (lane & 3) * 2 + e;
        if (m < M && n < N) C[m + (size_t)n * ldc] = acc[i][j][e];
      }
}

}  // namespace msg
