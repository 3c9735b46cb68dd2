// msgpu_fe.cuh -- device building blocks of the registration path on the
// uniform 2^l+1 grid: Q1 quadrature, the clipped warp of a quadrature point,
// the SSD integrand and its variation, the assembled Q1 stiffness stencil,
// and the finite-difference heat operator / transfer stencils of the
// multigrid smoother.
//
// Every function states the reference code it follows.  Floating-point
// operations are written in the reference's order so that the FP64
// instantiation reproduces the reference to rounding; the FP32 instantiation
// uses the same formulas in single precision.
#pragma once

#include <cuda_runtime.h>
#include <float.h>
#include <stdint.h>

namespace msg {

// Quadrature and stiffness tables, computed on the host in double exactly like
// BaseFunctionSetMultiLin<double,QC_2D,GaussQuadrature<double,QC_2D,3>>
// (baseFunctionSet.h:58-65, 128-195; Quadrature2D baseFunctionSet.h:1443-1454)
// and the assembled StiffOp (FEOpInterface.h:1362-1395, 65-88).
struct FeTables {
  double rc[4][2];      // reference coordinates of quadrature point q
  double bq[4][4];      // basis b at quadrature point q
  double w;             // quadrature weight (0.25)
  // Assembled stiffness stencil per node class: class = cx + 3*cy with
  // c = 0 (first node), 1 (interior), 2 (last node) along each axis;
  // entry [class][j+1][i+1] couples node (x,y) with (x+i, y+j).
  double st[9][3][3];
  // Assembled Q1 mass stencil (MassOp ASSEMBLED, FEOpInterface.h:2382-2394,
  // local matrix 1445-1475) for element volume 1; the stencil of a level is
  // this times h^2, an exact power-of-two scaling.
  double ms[9][3][3];
  // Local Q1 stiffness matrix of one element (FELinScalarWeightedStiffInterface::
  // prepareLocalMatrix, FEOpInterface.h:1362-1395), local node i = x + 2y.
  double lst[4][4];
};

__constant__ FeTables c_fe;

template <typename Real> struct RealTraits;
template <> struct RealTraits<float> {
  static __device__ __forceinline__ float eps() { return FLT_EPSILON; }
};
template <> struct RealTraits<double> {
  static __device__ __forceinline__ double eps() { return DBL_EPSILON; }
};

__device__ __forceinline__ int node_class(int x, int n) { return x == 0 ? 0 : (x == n - 1 ? 2 : 1); }

// DiscreteFunctionDefault::evaluateAtQuadPoint (discreteFunction.h:239-246)
// on the four nodal values v[b] of an element.  The reference starts the sum
// at 0.; starting at the first product differs only in the sign of an exact
// zero, which no later operation of the path can observe.
template <typename Real>
__device__ __forceinline__ Real at_quad(const Real v[4], int q) {
  Real w = v[0] * Real(c_fe.bq[0][q]);
  w += v[1] * Real(c_fe.bq[1][q]);
  w += v[2] * Real(c_fe.bq[2][q]);
  w += v[3] * Real(c_fe.bq[3][q]);
  return w;
}

// Result of transformAndClipCoord + getLocalCoordsRegularRectangularGrid
// (deformations.h:765-817, configurators.h:34-51).
template <typename Real>
struct Warped {
  int ex, ey;          // element of the warped point
  Real lx, ly;         // local coordinates in that element
  bool inx, iny;       // coordinate within [0, width) on each axis
};

template <typename Real>
__device__ __forceinline__ void clip_axis(Real coord, int n, Real h, int& el, Real& loc, bool& inside) {
  // width = (int)((n-1) * h) is exactly 1 on every dyadic level.
  (void)h;
  inside = true;
  if (coord < Real(0)) {
    coord = Real(0);
    inside = false;
  } else if (coord >= Real(1)) {
    coord = Real(1) - RealTraits<Real>::eps();
    inside = false;
  }
  // coord / h with h = 2^-l, written as the exactly equal product with 2^l.
  // After clipping sc < n-1, so the reference's "exactly on the right
  // boundary" adjustment (configurators.h:40-44) cannot apply.
  const Real sc = coord * Real(n - 1);
  const int e = (short)sc;
  el = e;
  loc = sc - Real(e);
}

template <typename Real>
__device__ __forceinline__ Warped<Real> warp_quad_point(int ex, int ey, int q, Real offx, Real offy, int n, Real h) {
  Real cx = (Real(ex) + Real(c_fe.rc[q][0])) * h;
  Real cy = (Real(ey) + Real(c_fe.rc[q][1])) * h;
  cx += offx;
  cy += offy;
  Warped<Real> w;
  clip_axis(cx, n, h, w.ex, w.lx, w.inx);
  clip_axis(cy, n, h, w.ey, w.ly, w.iny);
  return w;
}

// DiscreteFunctionDefault::evaluate (discreteFunction.h:230-237) with the Q1
// basis (baseFunctionSet.h:141-144) on the 4 texels t[0..3] of the element.
template <typename Real>
__device__ __forceinline__ Real q1_value(const Real t[4], Real x, Real y) {
  Real w = t[0] * ((Real(1) - x) * (Real(1) - y));
  w += t[1] * (x * (Real(1) - y));
  w += t[2] * ((Real(1) - x) * y);
  w += t[3] * (x * y);
  return w;
}

// DiscreteFunctionDefault::evaluateGradient (discreteFunction.h:259-269),
// basis derivatives baseFunctionSet.h:131-139, divided by h.  h = 2^-l, so the
// division is the exactly equal product with inv_h = 2^l.
template <typename Real>
__device__ __forceinline__ void q1_grad(const Real t[4], Real x, Real y, Real inv_h, Real& gx, Real& gy) {
  Real vx, vy;
  vx = (y - Real(1)) * inv_h; vy = (x - Real(1)) * inv_h; vx *= t[0]; vy *= t[0]; gx = vx; gy = vy;
  vx = (Real(1) - y) * inv_h; vy = (-x) * inv_h;          vx *= t[1]; vy *= t[1]; gx += vx; gy += vy;
  vx = (-y) * inv_h;          vy = (Real(1) - x) * inv_h; vx *= t[2]; vy *= t[2]; gx += vx; gy += vy;
  vx = y * inv_h;             vy = x * inv_h;             vx *= t[3]; vy *= t[3]; gx += vx; gy += vy;
}

// The 4 texels of element (ex, ey) of an image with row pitch P.
template <typename Real>
__device__ __forceinline__ void load_texels(const Real* __restrict__ T, int P, int ex, int ey, Real t[4]) {
  const Real* p = T + (size_t)ey * P + ex;
  t[0] = __ldg(p);
  t[1] = __ldg(p + 1);
  t[2] = __ldg(p + P);
  t[3] = __ldg(p + P + 1);
}

// SSDEnergy integrand summed over the element's 4 quadrature points and
// multiplied by the element volume (registration.h:1606-1615,
// FEOpInterface.h:2598-2610).  p[c][b] are the nodal displacements of
// component c, r[b] the nodal reference values.
template <typename Real>
__device__ __forceinline__ Real element_ssd(const Real* __restrict__ T, int n, int P, Real h, int ex, int ey,
                                            const Real px[4], const Real py[4], const Real r[4]) {
  Real a;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const Real ox = at_quad(px, q);
    const Real oy = at_quad(py, q);
    const Warped<Real> w = warp_quad_point(ex, ey, q, ox, oy, n, h);
    Real t[4];
    load_texels(T, P, w.ex, w.ey, t);
    const Real tv = q1_value(t, w.lx, w.ly);
    const Real rv = at_quad(r, q);
    const Real d = tv - rv;
    const Real v = (Real(0.5) * (d * d)) * Real(c_fe.w);
    if (q == 0) a = v; else a += v;   // the integrand is >= 0: no signed-zero difference
  }
  a *= h * h;
  return a;
}

// SSDForce nonlinearity at the 4 quadrature points and its integration
// against the 4 basis functions (registration.h:1648-1666,
// FEOpInterface.h:1821-1848): out[b][c] = vol * sum_q nl[q][c] * bq[b][q] * w.
template <typename Real>
__device__ __forceinline__ void element_force(const Real* __restrict__ T, int n, int P, Real h, int ex, int ey,
                                              const Real px[4], const Real py[4], const Real r[4],
                                              Real out[4][2]) {
  Real nl[4][2];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const Real ox = at_quad(px, q);
    const Real oy = at_quad(py, q);
    const Warped<Real> w = warp_quad_point(ex, ey, q, ox, oy, n, h);
    Real t[4];
    load_texels(T, P, w.ex, w.ey, t);
    const Real td = q1_value(t, w.lx, w.ly);
    const Real rv = at_quad(r, q);
    Real gx, gy;
    q1_grad(t, w.lx, w.ly, Real(n - 1), gx, gy);
    nl[q][0] = w.inx ? gx * (td - rv) : Real(0);
    nl[q][1] = w.iny ? gy * (td - rv) : Real(0);
  }
  const Real vol = h * h;
#pragma unroll
  for (int b = 0; b < 4; ++b) {
    Real a0 = Real(0), a1 = Real(0);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const Real f = Real(c_fe.bq[b][q]) * Real(c_fe.w);
      a0 += nl[q][0] * f;
      a1 += nl[q][1] * f;
    }
    out[b][0] = vol * a0;
    out[b][1] = vol * a1;
  }
}

// Assembled stiffness row at node (x,y) applied to u (fastUniformGridMatrix.h:
// 259-279 order: rows j = -1..1, columns i = -1..1).  get(X, Y) reads u.
template <typename Real, typename Get>
__device__ __forceinline__ Real stiff_row(int x, int y, int n, Get get) {
  Real d = Real(0);
  if (x > 0 && x < n - 1 && y > 0 && y < n - 1) {
    // interior node: all nine entries of its class, in the same order (the
    // coefficients are the same for every interior node)
#pragma unroll
    for (int j = -1; j <= 1; ++j)
#pragma unroll
      for (int i = -1; i <= 1; ++i) d += Real(c_fe.st[4][j + 1][i + 1]) * get(x + i, y + j);
    return d;
  }
  const int cls = node_class(x, n) + 3 * node_class(y, n);
#pragma unroll
  for (int j = -1; j <= 1; ++j)
#pragma unroll
    for (int i = -1; i <= 1; ++i) {
      const int X = x + i, Y = y + j;
      if (X >= 0 && X < n && Y >= 0 && Y < n) d += Real(c_fe.st[cls][j + 1][i + 1]) * get(X, Y);
    }
  return d;
}

// Assembled mass row at node (x,y) applied to u, same order as stiff_row;
// hh = h^2.
template <typename Real, typename Get>
__device__ __forceinline__ Real mass_row(int x, int y, int n, Real hh, Get get) {
  Real d = Real(0);
  if (x > 0 && x < n - 1 && y > 0 && y < n - 1) {   // interior node, as in stiff_row
#pragma unroll
    for (int j = -1; j <= 1; ++j)
#pragma unroll
      for (int i = -1; i <= 1; ++i) d += (Real(c_fe.ms[4][j + 1][i + 1]) * hh) * get(x + i, y + j);
    return d;
  }
  const int cls = node_class(x, n) + 3 * node_class(y, n);
#pragma unroll
  for (int j = -1; j <= 1; ++j)
#pragma unroll
    for (int i = -1; i <= 1; ++i) {
      const int X = x + i, Y = y + j;
      if (X >= 0 && X < n && Y >= 0 && Y < n) d += (Real(c_fe.ms[cls][j + 1][i + 1]) * hh) * get(X, Y);
    }
  return d;
}

// FastDeformImage at node (x,y) (deformations.h:138-159): position
// x + phi/h clamped to the grid, then ScalarArray::interpolate
// (scalarArray.h:499-525) of the pitched image T.  inv_h = 2^l makes the
// division by h an exact product.
template <typename Real>
__device__ __forceinline__ Real fast_deform_node(const Real* __restrict__ T, int n, int P, int x, int y, Real px,
                                                 Real py, Real inv_h) {
  const Real hi = Real(n - 1);
  Real X = Real(x) + px * inv_h, Y = Real(y) + py * inv_h;
  X = X < Real(0) ? Real(0) : (X > hi ? hi : X);
  Y = Y < Real(0) ? Real(0) : (Y > hi ? hi : Y);
  int xL = (int)X, yL = (int)Y;
  if (X >= hi) xL = n - 2;
  if (Y >= hi) yL = n - 2;
  X -= Real(xL);
  Y -= Real(yL);
  const Real* p = T + (size_t)yL * P + xL;
  const Real v0 = __ldg(p), v1 = __ldg(p + 1);
  if (Y == Real(0)) return (Real(1) - X) * v0 + X * v1;
  const Real v2 = __ldg(p + P), v3 = __ldg(p + P + 1);
  return (Real(1) - X) * (Real(1) - Y) * v0 + X * (Real(1) - Y) * v1 + (Real(1) - X) * Y * v2 + X * Y * v3;
}

// transformCoord<ConfiguratorType, false> (deformations.h:622-668) of
// quadrature point q of element (ex,ey): grid coordinates El + RefCoord +
// offset / h without clipping; false when the point leaves the grid.
template <typename Real>
__device__ __forceinline__ bool transform_noclip_axis(Real coord, Real off, int n, Real inv_h, int& el, Real& loc) {
  const Real tc = coord + off * inv_h;
  int e = (short)tc;
  Real l = tc - Real(e);
  if (e == n - 1 && l == Real(0)) {
    e = n - 2;
    l = Real(1);
  }
  el = e;
  loc = l;
  return !(tc < Real(0) || e < 0 || e >= n - 1);
}

// CrossCorrelationForce nonlinearity at the 4 quadrature points and its
// integration against the 4 basis functions (registration.h:1849-1861,
// FEOpInterface.h:1821-1848): out[b][c] = vol * sum_q nl[q][c] * bq[b][q] * w
// with nl = -temp(x_q) * grad T(transformed x_q), 0 outside the grid.
template <typename Real>
__device__ __forceinline__ void element_ncc_force(const Real* __restrict__ T, int n, int P, Real h, int ex, int ey,
                                                  const Real px[4], const Real py[4], const Real tmp[4],
                                                  Real out[4][2]) {
  Real nl[4][2];
  const Real inv_h = Real(n - 1);
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const Real ox = at_quad(px, q);
    const Real oy = at_quad(py, q);
    int elx, ely;
    Real lx, ly;
    const bool inx = transform_noclip_axis(Real(ex) + Real(c_fe.rc[q][0]), ox, n, inv_h, elx, lx);
    const bool iny = inx && transform_noclip_axis(Real(ey) + Real(c_fe.rc[q][1]), oy, n, inv_h, ely, ly);
    if (!iny) {
      nl[q][0] = Real(0);
      nl[q][1] = Real(0);
      continue;
    }
    Real t[4];
    load_texels(T, P, elx, ely, t);
    Real gx, gy;
    q1_grad(t, lx, ly, inv_h, gx, gy);
    const Real f = -at_quad(tmp, q);
    nl[q][0] = gx * f;
    nl[q][1] = gy * f;
  }
  const Real vol = h * h;
#pragma unroll
  for (int b = 0; b < 4; ++b) {
    Real a0 = Real(0), a1 = Real(0);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const Real f = Real(c_fe.bq[b][q]) * Real(c_fe.w);
      a0 += nl[q][0] * f;
      a1 += nl[q][1] * f;
    }
    out[b][0] = vol * a0;
    out[b][1] = vol * a1;
  }
}

// HeatEquation2DFD::apply at one node (linearSmoothOp.cpp:61-146):
// (I + tau (w-1)^2 L_FD) with the reference's boundary rows.  hsq = tau (w-1)^2.
template <typename Real, typename Get>
__device__ __forceinline__ Real heat_row(int X, int Y, int w, Real hsq, Get A) {
  const int e = w - 1;
  const Real c = A(X, Y);
  const Real a = c * Real(4);
  Real b;
  const bool bx = (X == 0 || X == e), by = (Y == 0 || Y == e);
  if (bx && by) {  // corner
    const int ox = (X == 0) ? 1 : -1, oy = (Y == 0) ? 1 : -1;
    b = -A(X + ox, Y) - A(X, Y + oy);
    return c + hsq * (a + Real(2) * b);
  }
  if (by) {  // edge parallel to the x axis (Y == 0 or Y == e)
    const int oy = (Y == 0) ? 1 : -1;
    b = Real(-2) * (A(X, Y + oy));
    b -= A(X + 1, Y);
    b -= A(X - 1, Y);
    return c + hsq * (a + b);
  }
  if (bx) {  // edge parallel to the y axis (X == 0 or X == e)
    const int ox = (X == 0) ? 1 : -1;
    b = Real(-2) * (A(X + ox, Y));
    b -= A(X, Y + 1);
    b -= A(X, Y - 1);
    return c + hsq * (a + b);
  }
  b = Real(0);
  b -= A(X + 1, Y);
  b -= A(X - 1, Y);
  b -= A(X, Y + 1);
  b -= A(X, Y - 1);
  return c + hsq * (a + b);
}

// One damped-Jacobi update with relax 1 (linearSmoothOp.cpp:556-580).
template <typename Real>
__device__ __forceinline__ Real jacobi_update(Real x, Real rhs, Real Ax, Real diag) {
  const Real v = rhs - Ax;
  return x + Real(1) * v / diag;
}

// RestrictOp<STD_QUOC_RESTRICT> value of coarse node (X,Y) (restriction.cpp:
// 397-470), accumulated in the reference's loop order.  F(x, y) reads the
// fine array; cw is the coarse width.
template <typename Real, typename Get>
__device__ __forceinline__ Real restrict_node(int X, int Y, int cw, Get F) {
  Real c = F(2 * X, 2 * Y) / Real(4);
  // diagonal fine nodes, loop X' outer, Y' inner
  if (X - 1 >= 0 && Y - 1 >= 0) c += F(2 * (X - 1) + 1, 2 * (Y - 1) + 1) / Real(16);
  if (X - 1 >= 0 && Y < cw - 1) c += F(2 * (X - 1) + 1, 2 * Y + 1) / Real(16);
  if (X < cw - 1 && Y - 1 >= 0) c += F(2 * X + 1, 2 * (Y - 1) + 1) / Real(16);
  if (X < cw - 1 && Y < cw - 1) c += F(2 * X + 1, 2 * Y + 1) / Real(16);
  // x-edge midpoints
  if (X - 1 >= 0) c += F(2 * (X - 1) + 1, 2 * Y) / Real(8);
  if (X < cw - 1) c += F(2 * X + 1, 2 * Y) / Real(8);
  // y-edge midpoints
  if (Y - 1 >= 0) c += F(2 * X, 2 * (Y - 1) + 1) / Real(8);
  if (Y < cw - 1) c += F(2 * X, 2 * Y + 1) / Real(8);
  const bool bx = (X == 0 || X == cw - 1), by = (Y == 0 || Y == cw - 1);
  if (bx && by) c = Real(16) * (c / Real(9));
  else if (bx || by) c = Real(4) * (c / Real(3));
  return c;
}

// ProlongOp::std_mg_prolongate value at fine node (x,y) (prolongation.cpp:
// 195-232).  C(X, Y) reads the coarse array.
template <typename Real, typename Get>
__device__ __forceinline__ Real prolong_node(int x, int y, Get C) {
  const int X = x >> 1, Y = y >> 1;
  auto even_row = [&](int yy) -> Real {  // value on an even fine row 2*yy
    if ((x & 1) == 0) return C(X, yy);
    return (C(X, yy) + C(X + 1, yy)) / Real(2);
  };
  if ((y & 1) == 0) return even_row(Y);
  return (even_row(Y) + even_row(Y + 1)) / Real(2);
}

// ScalarArray<QC_2D>::interpolate (scalarArray.h:499-525).
__device__ __forceinline__ double interp_d(const double* img, int n, double X, double Y) {
  int xL = (int)X, yL = (int)Y;
  if (X >= (double)(n - 1)) xL = n - 2;
  if (Y >= (double)(n - 1)) yL = n - 2;
  if (X < 0.) xL = 0;
  if (Y < 0.) yL = 0;
  X -= xL;
  Y -= yL;
  const int xU = xL + 1, yU = yL + 1;
  const double v0 = img[xL + (size_t)yL * n], v1 = img[xU + (size_t)yL * n];
  if (Y == 0) return (1 - X) * v0 + X * v1;
  const double v2 = img[xL + (size_t)yU * n], v3 = img[xU + (size_t)yU * n];
  return (1 - X) * (1 - Y) * v0 + X * (1 - Y) * v1 + (1 - X) * Y * v2 + X * Y * v3;
}

}  // namespace msg
