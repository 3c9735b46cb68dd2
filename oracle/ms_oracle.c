/*
 * ms_oracle.c -- FP64 CPU restatement of the matchSeries registration path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA path, never the product.
 * Each function follows the reference file:line given beside it, including
 * the order of floating-point operations where that order is observable in
 * FP64 (sums are accumulated in the reference's loop order), so that the
 * restatement agrees with the reference's own templates to rounding.
 */
#include "ms_oracle.h"

#include <float.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* 1-D Gauss points of GaussQuadrature<double,QC_1D,3> (baseFunctionSet.h:1538-1545) */
#define GP0 0.2113248654051871
#define GP1 0.7886751345948129

static int lvl_n(int level) { return (1 << level) + 1; }
static double lvl_h(int level) { return 1.0 / (double)(1 << level); }
static double sqr(double x) { return x * x; }

/* Quadrature tables of BaseFunctionSetMultiLin<double,QC_2D,Gauss3>
 * (baseFunctionSet.h:58-65, 128-195, Quadrature2D 1443-1454).            */
typedef struct {
  double rc[4][2];       /* reference coordinates of the 4 quad points   */
  double bq[4][4];       /* basis value  [basis][quad]                   */
  double gq[4][4][2];    /* basis gradient / h [basis][quad][comp]       */
  double w;              /* quad weight (0.5 * 0.5)                      */
} quad_t;

static void basis_grad(int b, double x, double y, double h, double g[2]) {
  switch (b) {
    case 0: g[0] = (y - 1.0) / h; g[1] = (x - 1.0) / h; break;
    case 1: g[0] = (1.0 - y) / h; g[1] = (-x) / h; break;
    case 2: g[0] = (-y) / h; g[1] = (1.0 - x) / h; break;
    default: g[0] = y / h; g[1] = x / h; break;
  }
}

static double basis_val(int b, double x, double y) {
  switch (b) {
    case 0: return (1.0 - x) * (1.0 - y);
    case 1: return x * (1.0 - y);
    case 2: return (1.0 - x) * y;
    default: return x * y;
  }
}

static void quad_init(quad_t* Q, double h) {
  const double g[2] = {GP0, GP1};
  for (int i = 0, k = 0; i < 2; ++i)
    for (int j = 0; j < 2; ++j, ++k) { Q->rc[k][0] = g[i]; Q->rc[k][1] = g[j]; }
  for (int b = 0; b < 4; ++b)
    for (int q = 0; q < 4; ++q) {
      Q->bq[b][q] = basis_val(b, Q->rc[q][0], Q->rc[q][1]);
      basis_grad(b, Q->rc[q][0], Q->rc[q][1], h, Q->gq[b][q]);
    }
  Q->w = 0.5 * 0.5;
}

/* global node index of local dof b of element (ex, ey) (indexMapper.h:410-414) */
static int dof(int n, int ex, int ey, int b) {
  return ex + ey * n + ((b & 1) ? 1 : 0) + ((b & 2) ? n : 0);
}

/* DiscreteFunctionDefault::evaluateAtQuadPoint (discreteFunction.h:239-246) */
static double eval_at_quad(const quad_t* Q, const double* f, int n, int ex, int ey, int q) {
  double w = 0.;
  for (int b = 0; b < 4; ++b) w += f[dof(n, ex, ey, b)] * Q->bq[b][q];
  return w;
}

/* DiscreteFunctionDefault::evaluate (discreteFunction.h:230-237) */
static double eval_local(const double* f, int n, int ex, int ey, double x, double y) {
  double w = 0.;
  for (int b = 0; b < 4; ++b) w += f[dof(n, ex, ey, b)] * basis_val(b, x, y);
  return w;
}

/* DiscreteFunctionDefault::evaluateGradient (discreteFunction.h:259-269) */
static void eval_grad_local(const double* f, int n, int ex, int ey, double x, double y,
                            double h, double g[2]) {
  g[0] = 0.; g[1] = 0.;
  for (int b = 0; b < 4; ++b) {
    double v[2];
    basis_grad(b, x, y, h, v);
    const double d = f[dof(n, ex, ey, b)];
    v[0] *= d; v[1] *= d;
    g[0] += v[0]; g[1] += v[1];
  }
}

/* transformAndClipCoord (deformations.h:765-817) followed by
 * getLocalCoordsRegularRectangularGrid (configurators.h:34-51).            */
typedef struct { int el[2]; double loc[2]; int within[2]; } tcoord_t;

static void transform_and_clip(const quad_t* Q, int n, double h, int ex, int ey, int q,
                               double off_x, double off_y, tcoord_t* t) {
  double coord[2];
  coord[0] = ((double)ex + Q->rc[q][0]) * h;
  coord[1] = ((double)ey + Q->rc[q][1]) * h;
  coord[0] += off_x;
  coord[1] += off_y;
  for (int c = 0; c < 2; ++c) {
    const int width = (int)((double)(n - 1) * h);
    t->within[c] = 1;
    if (coord[c] < 0.) {
      coord[c] = 0.;
      t->within[c] = 0;
    } else if (coord[c] >= width) {
      coord[c] = width - DBL_EPSILON;
      t->within[c] = 0;
    }
    const double sc = coord[c] / h;
    int e = (short)sc;
    double l = sc - e;
    if (e == n - 1 && fabs(l - 0.) < 1e-15) { e = n - 2; l = 1; }
    t->el[c] = e;
    t->loc[c] = l;
  }
}

/* ---------------------------------------------------------------------- */

double msor_ssd_energy(int level, const double* R, const double* T,
                       const double* phix, const double* phiy) {
  const int n = lvl_n(level);
  const double h = lvl_h(level);
  const double vol = sqr(h);
  quad_t Q;
  quad_init(&Q, h);
  double res = 0.;
  for (int ey = 0; ey < n - 1; ++ey)
    for (int ex = 0; ex < n - 1; ++ex) {
      double a = 0.;
      for (int q = 0; q < 4; ++q) {
        const double ox = eval_at_quad(&Q, phix, n, ex, ey, q);
        const double oy = eval_at_quad(&Q, phiy, n, ex, ey, q);
        tcoord_t t;
        transform_and_clip(&Q, n, h, ex, ey, q, ox, oy, &t);
        const double tv = eval_local(T, n, t.el[0], t.el[1], t.loc[0], t.loc[1]);
        const double rv = eval_at_quad(&Q, R, n, ex, ey, q);
        a += (0.5 * sqr(tv - rv)) * Q.w;
      }
      a *= vol;
      res += a;
    }
  return 0. + res;
}

void msor_ssd_force(int level, const double* R, const double* T,
                    const double* phix, const double* phiy, double* gx, double* gy) {
  const int n = lvl_n(level);
  const double h = lvl_h(level);
  const double vol = sqr(h);
  quad_t Q;
  quad_init(&Q, h);
  memset(gx, 0, sizeof(double) * n * n);
  memset(gy, 0, sizeof(double) * n * n);
  for (int ey = 0; ey < n - 1; ++ey)
    for (int ex = 0; ex < n - 1; ++ex) {
      double nl[4][2];
      for (int q = 0; q < 4; ++q) {
        const double ox = eval_at_quad(&Q, phix, n, ex, ey, q);
        const double oy = eval_at_quad(&Q, phiy, n, ex, ey, q);
        tcoord_t t;
        transform_and_clip(&Q, n, h, ex, ey, q, ox, oy, &t);
        const double td = eval_local(T, n, t.el[0], t.el[1], t.loc[0], t.loc[1]);
        const double rv = eval_at_quad(&Q, R, n, ex, ey, q);
        eval_grad_local(T, n, t.el[0], t.el[1], t.loc[0], t.loc[1], h, nl[q]);
        for (int c = 0; c < 2; ++c) nl[q][c] = t.within[c] ? nl[q][c] * (td - rv) : 0;
      }
      for (int b = 0; b < 4; ++b) {
        double a0 = 0., a1 = 0.;
        for (int q = 0; q < 4; ++q) {
          const double f = Q.bq[b][q] * Q.w;
          a0 += nl[q][0] * f;
          a1 += nl[q][1] * f;
        }
        const int g = dof(n, ex, ey, b);
        gx[g] += vol * a0;
        gy[g] += vol * a1;
      }
    }
}

/* Assembled Q1 stiffness in the 3x3-per-row layout of FastUniformGridMatrix
 * (fastUniformGridMatrix.h:313-470): local matrix by quadrature
 * (FEOpInterface.h:1362-1395), added once per entry in element order
 * (LocalAssemblyHelper<QUOC_GRID_INDEX_MODE>::doLocalAssembly,
 * FEOpInterface.h:65-88).                                                 */
static double* stiff_build(int level) {
  const int n = lvl_n(level);
  const double h = lvl_h(level);
  const double vol = sqr(h);
  quad_t Q;
  quad_init(&Q, h);
  double L[4][4];
  for (int i = 0; i < 4; ++i) for (int j = 0; j < 4; ++j) L[i][j] = 0.;
  for (int q = 0; q < 4; ++q) {
    const double coeff = 1.;
    for (int i = 0; i < 4; ++i)
      for (int j = i; j < 4; ++j) {
        double dot = 0;
        dot += Q.gq[i][q][0] * Q.gq[j][q][0];
        dot += Q.gq[i][q][1] * Q.gq[j][q][1];
        L[i][j] += dot * coeff * Q.w;
      }
  }
  for (int i = 0; i < 4; ++i)
    for (int j = i; j < 4; ++j) L[j][i] = L[i][j] = L[i][j] * vol;
  double* st = (double*)calloc((size_t)n * n * 9, sizeof(double));
  for (int ey = 0; ey < n - 1; ++ey)
    for (int ex = 0; ex < n - 1; ++ex)
      for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) {
          const int gi = dof(n, ex, ey, i), gj = dof(n, ex, ey, j);
          const int dx = (gj % n) - (gi % n), dy = (gj / n) - (gi / n);
          double* e = &st[(size_t)gi * 9 + (dy + 1) * 3 + (dx + 1)];
          *e += 1.0 * L[i][j];
        }
  return st;
}

static void stiff_apply_with(const double* st, int level, const double* u, double* Lu) {
  const int n = lvl_n(level);
  for (int r = 0; r < n * n; ++r) {
    const int x = r % n, y = r / n;
    double d = 0.;
    for (int j = -1; j <= 1; ++j)
      for (int i = -1; i <= 1; ++i) {
        const int X = x + i, Y = y + j;
        if (X >= 0 && X < n && Y >= 0 && Y < n)
          d += st[(size_t)r * 9 + (j + 1) * 3 + (i + 1)] * u[X + Y * n];
      }
    Lu[r] = d;
  }
}

void msor_stiff_apply(int level, const double* u, double* Lu) {
  double* st = stiff_build(level);
  stiff_apply_with(st, level, u, Lu);
  free(st);
}

static double dot(const double* a, const double* b, int N) {
  double r = 0;
  for (int i = 0; i < N; ++i) r += a[i] * b[i];
  return r;
}

/* data term of a level solve: SSD, or NCC with its precomputed parts */
typedef struct dterm_s {
  int ncc;           /* 0: SSD, 1: NCC                                   */
  double* M;         /* mass matrix (NCC)                                */
  double* normR;     /* normalised reference (NCC)                       */
} dterm_t;
static double ncc_energy_with(const dterm_t* D, int level, const double* T, const double* phix,
                              const double* phiy, double* var_out, double* normT_out);
static void ncc_variation_with(const dterm_t* D, int level, const double* T, const double* phix,
                               const double* phiy, double* gx, double* gy);
static double interp(const double* img, int n, double X, double Y);
static void dterm_init(dterm_t* D, int ncc, int level, const double* R);
static void dterm_free(dterm_t* D);

/* DisplacementLengthEnergy::apply (hyperelastic.h:178-183) */
static double reg_energy_with(const double* st, int level, const double* phix, const double* phiy) {
  const int n = lvl_n(level), N = n * n;
  double* tmp = (double*)malloc(sizeof(double) * N * 2);
  stiff_apply_with(st, level, phix, tmp);
  stiff_apply_with(st, level, phiy, tmp + N);
  double d = 0;
  d += dot(phix, tmp, N);
  d += dot(phiy, tmp + N, N);
  free(tmp);
  return 0.5 * d;
}

static double energy_with(const double* st, const dterm_t* D, int level, const double* R, const double* T,
                          const double* phix, const double* phiy, double lambda, double* ereg) {
  double e = 0.;
  if (D && D->ncc) e += ncc_energy_with(D, level, T, phix, phiy, NULL, NULL);
  else e += msor_ssd_energy(level, R, T, phix, phiy);
  const double r = reg_energy_with(st, level, phix, phiy);
  if (ereg) *ereg = r;
  if (lambda != 1.0) e += lambda * r; else e += r;
  return e;
}

double msor_energy(int level, const double* R, const double* T, const double* phix,
                   const double* phiy, double lambda, double* ereg) {
  double* st = stiff_build(level);
  const double e = energy_with(st, NULL, level, R, T, phix, phiy, lambda, ereg);
  free(st);
  return e;
}

double msor_energy_dt(int data_term, int level, const double* R, const double* T, const double* phix,
                      const double* phiy, double lambda, double* ereg) {
  double* st = stiff_build(level);
  dterm_t D;
  dterm_init(&D, data_term, level, R);
  const double e = energy_with(st, &D, level, R, T, phix, phiy, lambda, ereg);
  dterm_free(&D);
  free(st);
  return e;
}

static void denergy_with(const double* st, const dterm_t* D, int level, const double* R, const double* T,
                         const double* phix, const double* phiy, double lambda,
                         double* gx, double* gy) {
  const int n = lvl_n(level), N = n * n;
  if (D && D->ncc) ncc_variation_with(D, level, T, phix, phiy, gx, gy);
  else msor_ssd_force(level, R, T, phix, phiy, gx, gy);
  double* tmp = (double*)malloc(sizeof(double) * N);
  stiff_apply_with(st, level, phix, tmp);
  for (int i = 0; i < N; ++i) gx[i] += (lambda != 1.0) ? lambda * tmp[i] : tmp[i];
  stiff_apply_with(st, level, phiy, tmp);
  for (int i = 0; i < N; ++i) gy[i] += (lambda != 1.0) ? lambda * tmp[i] : tmp[i];
  free(tmp);
}

void msor_denergy(int level, const double* R, const double* T, const double* phix,
                  const double* phiy, double lambda, double* gx, double* gy) {
  double* st = stiff_build(level);
  denergy_with(st, NULL, level, R, T, phix, phiy, lambda, gx, gy);
  free(st);
}

void msor_denergy_dt(int data_term, int level, const double* R, const double* T, const double* phix,
                     const double* phiy, double lambda, double* gx, double* gy) {
  double* st = stiff_build(level);
  dterm_t D;
  dterm_init(&D, data_term, level, R);
  denergy_with(st, &D, level, R, T, phix, phiy, lambda, gx, gy);
  dterm_free(&D);
  free(st);
}

/* --- normalized cross-correlation data term (registration.h:1828-2018) ---- */

/* Assembled Q1 mass matrix (MassOp ASSEMBLED, FEOpInterface.h:2382-2394):
 * local matrix by quadrature (FELinScalarWeightedMassInterface::
 * prepareLocalMatrix, FEOpInterface.h:1445-1475) in the layout and
 * assembly order of the stiffness matrix above.                             */
static double* mass_build(int level) {
  const int n = lvl_n(level);
  const double h = lvl_h(level);
  const double vol = sqr(h);
  quad_t Q;
  quad_init(&Q, h);
  double L[4][4];
  for (int i = 0; i < 4; ++i) for (int j = 0; j < 4; ++j) L[i][j] = 0.;
  for (int q = 0; q < 4; ++q) {
    const double coeff = 1.;
    for (int i = 0; i < 4; ++i) {
      const double basisi = Q.bq[i][q];
      for (int j = i; j < 4; ++j) L[i][j] += basisi * Q.bq[j][q] * coeff * Q.w;
    }
  }
  for (int i = 0; i < 4; ++i)
    for (int j = i; j < 4; ++j) L[j][i] = L[i][j] = L[i][j] * vol;
  double* st = (double*)calloc((size_t)n * n * 9, sizeof(double));
  for (int ey = 0; ey < n - 1; ++ey)
    for (int ex = 0; ex < n - 1; ++ex)
      for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) {
          const int gi = dof(n, ex, ey, i), gj = dof(n, ex, ey, j);
          const int dx = (gj % n) - (gi % n), dy = (gj / n) - (gi / n);
          double* e = &st[(size_t)gi * 9 + (dy + 1) * 3 + (dx + 1)];
          *e += 1.0 * L[i][j];
        }
  return st;
}

void msor_mass_apply(int level, const double* u, double* Mu) {
  double* m = mass_build(level);
  stiff_apply_with(m, level, u, Mu);
  free(m);
}

/* NormalizedCrossCorrelationEnergy::normalizeImageForNCC (registration.h:
 * 1932-1944): subtract the mass-weighted mean, divide by the mass-weighted
 * norm; returns that norm.                                                 */
static double ncc_normalize(const double* M, int level, const double* img, double* out) {
  const int n = lvl_n(level), N = n * n;
  double* temp = (double*)malloc(sizeof(double) * N);
  stiff_apply_with(M, level, img, temp);
  double mean = 0.;                          /* Vector::sum (vec.cpp:847-860) */
  for (int i = 0; i < N; ++i) mean += temp[i];
  for (int i = 0; i < N; ++i) { out[i] = img[i]; out[i] += -mean; }   /* addToAll */
  stiff_apply_with(M, level, out, temp);
  const double var = sqrt(dot(out, temp, N));
  if (!(fabs(var - 0.) < 1e-15))             /* aol::appeqAbsolute, aol.h:791-794 */
    for (int i = 0; i < N; ++i) out[i] /= var;
  free(temp);
  return var;
}

/* FastDeformImage, 2-D (deformations.h:138-159): nodal positions clamped to
 * the grid, bilinear ScalarArray::interpolate.                             */
static void fast_deform(int level, const double* img, const double* phix, const double* phiy, double* out) {
  const int n = lvl_n(level);
  const double h = lvl_h(level);
  for (int j = 0; j < n; ++j)
    for (int i = 0; i < n; ++i) {
      const int index = i + j * n;
      double ds0 = i + phix[index] / h, ds1 = j + phiy[index] / h;
      const double hi = (double)(n - 1);
      ds0 = ds0 < 0. ? 0. : (ds0 > hi ? hi : ds0);            /* aol::Clamp */
      ds1 = ds1 < 0. ? 0. : (ds1 > hi ? hi : ds1);
      out[index] = interp(img, n, ds0, ds1);
    }
}


static void dterm_init(dterm_t* D, int ncc, int level, const double* R) {
  D->ncc = ncc;
  D->M = NULL;
  D->normR = NULL;
  if (ncc) {
    const int n = lvl_n(level);
    D->M = mass_build(level);
    D->normR = (double*)malloc(sizeof(double) * n * n);
    ncc_normalize(D->M, level, R, D->normR);
  }
}

static void dterm_free(dterm_t* D) {
  free(D->M);
  free(D->normR);
}

/* NormalizedCrossCorrelationEnergy::computeEnergy (registration.h:1950-1962);
 * var_out / normT_out (nullable) receive the norm and the normalised
 * deformed template.                                                       */
static double ncc_energy_with(const dterm_t* D, int level, const double* T, const double* phix,
                              const double* phiy, double* var_out, double* normT_out) {
  const int n = lvl_n(level), N = n * n;
  double* deformedT = (double*)malloc(sizeof(double) * N);
  double* normT = (double*)malloc(sizeof(double) * N);
  fast_deform(level, T, phix, phiy, deformedT);
  const double var = ncc_normalize(D->M, level, deformedT, normT);
  stiff_apply_with(D->M, level, normT, deformedT);
  const double e = -(dot(deformedT, D->normR, N));
  if (var_out) *var_out = var;
  if (normT_out) memcpy(normT_out, normT, sizeof(double) * N);
  free(deformedT);
  free(normT);
  return e;
}

double msor_ncc_energy(int level, const double* R, const double* T, const double* phix, const double* phiy) {
  dterm_t D;
  dterm_init(&D, 1, level, R);
  const double e = ncc_energy_with(&D, level, T, phix, phiy, NULL, NULL);
  dterm_free(&D);
  return e;
}

/* transformCoord<ConfiguratorType, false> (deformations.h:622-668): grid
 * coordinates El + RefCoord + Offset / H, no clipping; 0 when the point
 * leaves the grid.                                                         */
static int transform_noclip(const quad_t* Q, int n, double h, int ex, int ey, int q, double off_x,
                            double off_y, tcoord_t* t) {
  const double coord[2] = {(double)ex + Q->rc[q][0], (double)ey + Q->rc[q][1]};
  const double off[2] = {off_x, off_y};
  for (int c = 0; c < 2; ++c) {
    const double tc = coord[c] + off[c] / h;
    int e = (short)tc;
    double l = tc - e;
    if (e == n - 1 && l == 0) { e = n - 2; l = 1; }
    if (tc < 0. || e < 0 || e >= n - 1) return 0;
    t->el[c] = e;
    t->loc[c] = l;
    t->within[c] = 1;
  }
  return 1;
}

/* NormalizedCrossCorrelationEnergy::applyDerivative (registration.h:1972-1983)
 * with CrossCorrelationForce (registration.h:1828-1862) integrated like
 * FENonlinVectorOpInterface::applyAdd (FEOpInterface.h:1803-1852).          */
static void ncc_variation_with(const dterm_t* D, int level, const double* T, const double* phix,
                               const double* phiy, double* gx, double* gy) {
  const int n = lvl_n(level), N = n * n;
  const double h = lvl_h(level);
  const double vol = sqr(h);
  double var;
  double* normT = (double*)malloc(sizeof(double) * N);
  double* temp = (double*)malloc(sizeof(double) * N);
  const double energy = ncc_energy_with(D, level, T, phix, phiy, &var, normT);
  for (int i = 0; i < N; ++i) temp[i] = D->normR[i];
  for (int i = 0; i < N; ++i) temp[i] += normT[i] * energy;          /* addMultiple */
  if (!(fabs(var - 0.) < 1e-15))
    for (int i = 0; i < N; ++i) temp[i] /= var;
  quad_t Q;
  quad_init(&Q, h);
  memset(gx, 0, sizeof(double) * N);
  memset(gy, 0, sizeof(double) * N);
  for (int ey = 0; ey < n - 1; ++ey)
    for (int ex = 0; ex < n - 1; ++ex) {
      double nl[4][2];
      for (int q = 0; q < 4; ++q) {
        const double ox = eval_at_quad(&Q, phix, n, ex, ey, q);
        const double oy = eval_at_quad(&Q, phiy, n, ex, ey, q);
        tcoord_t t;
        if (!transform_noclip(&Q, n, h, ex, ey, q, ox, oy, &t)) {
          nl[q][0] = 0.;
          nl[q][1] = 0.;
          continue;
        }
        eval_grad_local(T, n, t.el[0], t.el[1], t.loc[0], t.loc[1], h, nl[q]);
        const double f = -eval_at_quad(&Q, temp, n, ex, ey, q);
        nl[q][0] *= f;
        nl[q][1] *= f;
      }
      for (int b = 0; b < 4; ++b) {
        double a0 = 0., a1 = 0.;
        for (int q = 0; q < 4; ++q) {
          const double f = Q.bq[b][q] * Q.w;
          a0 += nl[q][0] * f;
          a1 += nl[q][1] * f;
        }
        const int g = dof(n, ex, ey, b);
        gx[g] += vol * a0;
        gy[g] += vol * a1;
      }
    }
  free(normT);
  free(temp);
}

void msor_ncc_variation(int level, const double* R, const double* T, const double* phix, const double* phiy,
                        double* gx, double* gy) {
  dterm_t D;
  dterm_init(&D, 1, level, R);
  ncc_variation_with(&D, level, T, phix, phiy, gx, gy);
  dterm_free(&D);
}

/* --- multigrid heat smoother (linearSmoothOp.cpp) --------------------- */

/* HeatEquation2DFD::apply (linearSmoothOp.cpp:61-146) */
static void heat_apply(int level, double tau, const double* A, double* D) {
  const int w = lvl_n(level);
  const double hsq = tau * (double)((w - 1) * (w - 1));
#define AG(X, Y) A[(X) + (Y) * w]
#define DS(X, Y, V) D[(X) + (Y) * w] = (V)
  for (int X = 1; X < w - 1; ++X)
    for (int Y = 1; Y < w - 1; ++Y) {
      const double a = AG(X, Y) * 4;
      double b = 0.0;
      b -= AG(X + 1, Y);
      b -= AG(X - 1, Y);
      b -= AG(X, Y + 1);
      b -= AG(X, Y - 1);
      DS(X, Y, AG(X, Y) + hsq * (a + b));
    }
  const int e = w - 1;
  const int cs[4][2] = {{0, 0}, {e, 0}, {0, e}, {e, e}};
  const int co[4][2] = {{1, 1}, {-1, 1}, {1, -1}, {-1, -1}};
  for (int i = 0; i < 4; ++i) {
    const int cx = cs[i][0], cy = cs[i][1];
    const double a = AG(cx, cy) * 4;
    const double b = -AG(cx + co[i][0], cy) - AG(cx, cy + co[i][1]);
    DS(cx, cy, AG(cx, cy) + hsq * (a + 2 * b));
  }
  for (int X = 1; X < w - 1; ++X) {
    double a = AG(X, e) * 4;
    double b = -2 * (AG(X, e - 1));
    b -= AG(X + 1, e);
    b -= AG(X - 1, e);
    DS(X, e, AG(X, e) + hsq * (a + b));
    a = AG(X, 0) * 4;
    b = -2 * (AG(X, 1));
    b -= AG(X + 1, 0);
    b -= AG(X - 1, 0);
    DS(X, 0, AG(X, 0) + hsq * (a + b));
  }
  for (int X = 1; X < w - 1; ++X) {
    double a = AG(e, X) * 4;
    double b = -2 * (AG(e - 1, X));
    b -= AG(e, X + 1);
    b -= AG(e, X - 1);
    DS(e, X, AG(e, X) + hsq * (a + b));
    a = AG(0, X) * 4;
    b = -2 * (AG(1, X));
    b -= AG(0, X + 1);
    b -= AG(0, X - 1);
    DS(0, X, AG(0, X) + hsq * (a + b));
  }
#undef AG
#undef DS
}

/* HeatMultigrid::jacobi (linearSmoothOp.cpp:556-580) */
static void jacobi(int level, double tau, double* X, const double* rhs, double* dummy) {
  const int w = lvl_n(level);
  const double diag = 1 + 4 * tau * (double)((w - 1) * (w - 1));
  const double relax = 1.0;
  heat_apply(level, tau, X, dummy);
  for (int l = 0; l < w * w; ++l) {
    const double v = rhs[l] - dummy[l];
    X[l] += relax * v / diag;
  }
}

typedef struct { double* x[16]; double* rhs[16]; double* dummy[16]; double* res[16]; } mg_t;

/* MDMultigrid::solve (linearSmoothOp.cpp:451-494) */
static void mg_solve(mg_t* M, int level, double tau) {
  const int w = lvl_n(level);
  if (level == 0) {
    for (int i = 0; i < 100; ++i) jacobi(level, tau, M->x[level], M->rhs[level], M->dummy[level]);
    return;
  }
  for (int i = 0; i < 2; ++i) jacobi(level, tau, M->x[level], M->rhs[level], M->dummy[level]);
  heat_apply(level, tau, M->x[level], M->dummy[level]);
  for (int l = 0; l < w * w; ++l) M->res[level][l] = M->rhs[level][l] - M->dummy[level][l];
  msor_restrict(level, M->res[level], M->rhs[level - 1]);
  const int wc = lvl_n(level - 1);
  memset(M->x[level - 1], 0, sizeof(double) * wc * wc);
  mg_solve(M, level - 1, tau);
  msor_prolong(level - 1, M->x[level - 1], M->dummy[level]);
  for (int l = 0; l < w * w; ++l) M->x[level][l] += M->dummy[level][l];
  for (int i = 0; i < 2; ++i) jacobi(level, tau, M->x[level], M->rhs[level], M->dummy[level]);
}

void msor_smooth_tau(int level, double tau, const double* in, double* out) {
  mg_t M = {{0}, {0}, {0}, {0}};
  for (int l = 0; l <= level; ++l) {
    const int w = lvl_n(l);
    M.x[l] = (double*)calloc((size_t)w * w, sizeof(double));
    M.rhs[l] = (double*)calloc((size_t)w * w, sizeof(double));
    M.dummy[l] = (double*)calloc((size_t)w * w, sizeof(double));
    M.res[l] = (double*)calloc((size_t)w * w, sizeof(double));
  }
  const int w = lvl_n(level);
  memcpy(M.rhs[level], in, sizeof(double) * w * w);
  mg_solve(&M, level, tau);
  memcpy(out, M.x[level], sizeof(double) * w * w);
  for (int l = 0; l <= level; ++l) { free(M.x[l]); free(M.rhs[l]); free(M.dummy[l]); free(M.res[l]); }
}

/* LinearSmoothOp::setSigma: tau = 0.5f * sigma^2 (linearSmoothOp.h:50-52) */
void msor_smooth(int level, double sigma, const double* in, double* out) {
  msor_smooth_tau(level, 0.5f * sqr(sigma), in, out);
}

/* --- level transfer ----------------------------------------------------- */

void msor_restrict(int fine_level, const double* fine, double* coarse) {
  const int cw = lvl_n(fine_level - 1), fw = lvl_n(fine_level);
#define F(X, Y) fine[(X) + (Y) * fw]
#define C(X, Y) coarse[(X) + (Y) * cw]
  for (int X = 0; X < cw; ++X)
    for (int Y = 0; Y < cw; ++Y) C(X, Y) = F(2 * X, 2 * Y) / 4;
  for (int X = 0; X < cw - 1; ++X)
    for (int Y = 0; Y < cw - 1; ++Y) {
      const double v = F(2 * X + 1, 2 * Y + 1) / 16;
      C(X, Y) += v; C(X + 1, Y) += v; C(X, Y + 1) += v; C(X + 1, Y + 1) += v;
    }
  for (int X = 0; X < cw - 1; ++X)
    for (int Y = 0; Y < cw; ++Y) {
      const double v = F(2 * X + 1, 2 * Y) / 8;
      C(X, Y) += v; C(X + 1, Y) += v;
    }
  for (int X = 0; X < cw; ++X)
    for (int Y = 0; Y < cw - 1; ++Y) {
      const double v = F(2 * X, 2 * Y + 1) / 8;
      C(X, Y + 1) += v; C(X, Y) += v;
    }
  for (int X = 1; X < cw - 1; ++X) {
    C(X, 0) = 4 * (C(X, 0) / 3);
    C(X, cw - 1) = 4 * (C(X, cw - 1) / 3);
    C(0, X) = 4 * (C(0, X) / 3);
    C(cw - 1, X) = 4 * (C(cw - 1, X) / 3);
  }
  C(0, 0) = 16 * (C(0, 0) / 9);
  C(cw - 1, 0) = 16 * (C(cw - 1, 0) / 9);
  C(0, cw - 1) = 16 * (C(0, cw - 1) / 9);
  C(cw - 1, cw - 1) = 16 * (C(cw - 1, cw - 1) / 9);
#undef F
#undef C
}

void msor_prolong(int coarse_level, const double* coarse, double* fine) {
  const int cw = lvl_n(coarse_level) - 1, fw = lvl_n(coarse_level + 1);
  int cc = 0, fc = 0;
  for (int y = 0; y <= cw; ++y) {
    double u = coarse[cc++];
    for (int x = 0; x < cw; ++x) {
      const double w = coarse[cc++];
      fine[fc++] = u;
      fine[fc++] = (u + w) / 2;
      u = w;
    }
    fine[fc++] = u;
    fc += fw;
  }
  fc = fw;
  int tc = 0;
  cc = fw << 1;
  for (int y = 0; y < cw; ++y) {
    for (int x = 0; x < fw; ++x) fine[fc++] = (fine[tc++] + fine[cc++]) / 2;
    fc += fw; tc += fw; cc += fw;
  }
}

/* ScalarArray<QC_2D>::interpolate (scalarArray.h:499-525) */
static double interp(const double* img, int n, double X, double Y) {
  int xL = (int)X, yL = (int)Y;
  if (X >= (double)(n - 1)) xL = n - 2;
  if (Y >= (double)(n - 1)) yL = n - 2;
  if (X < 0.) xL = 0;
  if (Y < 0.) yL = 0;
  X -= xL;
  Y -= yL;
  const int xU = xL + 1, yU = yL + 1;
  const double v0 = img[xL + yL * n], v1 = img[xU + yL * n], v2 = img[xL + yU * n], v3 = img[xU + yU * n];
  if (Y == 0) return (1 - X) * v0 + X * v1;
  return (1 - X) * (1 - Y) * v0 + X * (1 - Y) * v1 + (1 - X) * Y * v2 + X * Y * v3;
}

void msor_resample(int src_level, const double* src, int dst_level, double* dst) {
  const int ns = lvl_n(src_level), nd = lvl_n(dst_level);
  const long double hx = (long double)(ns - 1) / (nd - 1);
  for (int y = 0; y < nd; ++y)
    for (int x = 0; x < nd; ++x) {
      const double sx = (double)(x * hx), sy = (double)(y * hx);
      dst[x + y * nd] = interp(src, ns, sx, sy);
    }
}

void msor_deform_image(int level, const double* img, const double* phix, const double* phiy,
                       double ext_value, double* out) {
  const int n = lvl_n(level);
  const double h = lvl_h(level);
  for (int y = 0; y < n; ++y)
    for (int x = 0; x < n; ++x) {
      const int i = x + y * n;
      const double ds0 = x + phix[i] / h, ds1 = y + phiy[i] / h;
      int inside = 1;
      if (ds0 < 0. || ds0 > (double)(n - 1) || isnan(ds0)) inside = 0;
      if (ds1 < 0. || ds1 > (double)(n - 1) || isnan(ds1)) inside = 0;
      out[i] = inside ? interp(img, n, ds0, ds1) : ext_value;
    }
}

static int cmp_double(const void* a, const void* b) {
  const double x = *(const double*)a, y = *(const double*)b;
  return (x < y) ? -1 : (x > y) ? 1 : 0;
}

void msor_normalize(double* img, int count, double sat, int min_to_zero) {
  if (sat >= 0) {
    double* tmp = (double*)malloc(sizeof(double) * count);
    memcpy(tmp, img, sizeof(double) * count);
    qsort(tmp, count, sizeof(double), cmp_double);
    const int m1 = count - 1;
    int il = (int)(sat / 200 * m1), ih = (int)((1 - sat / 200) * m1);
    il = il < 0 ? 0 : (il > m1 ? m1 : il);
    ih = ih < 0 ? 0 : (ih > m1 ? m1 : ih);
    const double lo = tmp[il], hi = tmp[ih];
    free(tmp);
    for (int i = 0; i < count; ++i) img[i] = img[i] < lo ? lo : (img[i] > hi ? hi : img[i]);
    double mn = img[0];
    for (int i = 1; i < count; ++i) if (img[i] < mn) mn = img[i];
    const double s = -1 * mn;
    for (int i = 0; i < count; ++i) img[i] += s;
    double mx = img[0];
    for (int i = 1; i < count; ++i) if (img[i] > mx) mx = img[i];
    if (mx != 0) for (int i = 0; i < count; ++i) img[i] /= mx;
  } else {
    double mn = img[0];
    for (int i = 1; i < count; ++i) if (img[i] < mn) mn = img[i];
    if (mn < 0. || min_to_zero) for (int i = 0; i < count; ++i) img[i] += -mn;
    double mx = img[0];
    for (int i = 1; i < count; ++i) if (img[i] > mx) mx = img[i];
    if (mx != 0.) for (int i = 0; i < count; ++i) img[i] /= mx;
  }
}

/* --- gradient flow ------------------------------------------------------ */

typedef struct {
  int level, N;
  const double *R, *T;
  const double* st;
  double lambda;
  const dterm_t* D;
  /* ring buffer of the last two Armijo evaluations (gradientDescent.h:56-59) */
  double rb_tau[2], rb_e[2];
  int rb_pos;
  int evals;
  double e_at_pos;
  double *tx, *ty;  /* scratch position */
} gd_ctx;

/* ArmijoLineSearchHelpFunction_evaluate (gradientDescent.h:168-187) */
static double armijo_eval(gd_ctx* C, const double* px, const double* py, const double* dx,
                          const double* dy, double tw) {
  if (tw == 0) return C->e_at_pos;
  for (int i = 0; i < C->N; ++i) { C->tx[i] = px[i]; C->tx[i] += tw * dx[i]; }
  for (int i = 0; i < C->N; ++i) { C->ty[i] = py[i]; C->ty[i] += tw * dy[i]; }
  const double e = energy_with(C->st, C->D, C->level, C->R, C->T, C->tx, C->ty, C->lambda, NULL);
  C->rb_tau[C->rb_pos] = tw;
  C->rb_e[C->rb_pos] = e;
  C->rb_pos ^= 1;
  C->evals++;
  return e;
}

static int finite(double x) { return !isnan(x) && !isinf(x); }

/* getTimestepWidthWithArmijoLineSearch (ArmijoSearch.h:118-200) */
static double armijo(gd_ctx* C, const double* px, const double* py, const double* dx,
                     const double* dy, const double* DEx, const double* DEy, double old_tau) {
  const double sigma = 0.5, tau_min = pow(2., -30.), tau_max = pow(2., 25.);
  double tau = old_tau < tau_min ? tau_min : (old_tau > tau_max ? tau_max : old_tau);
  const double f = armijo_eval(C, px, py, dx, dy, 0.);
  double fnew = armijo_eval(C, px, py, dx, dy, tau);
  double Df = 0;
  Df += dot(DEx, dx, C->N);
  Df += dot(DEy, dy, C->N);
  double G = (fnew - f) / (Df * tau);
  if (Df >= 0) return 0;
  if (!finite(f)) return 0;
  if (G >= sigma && f >= fnew) {
    do {
      tau *= 2.;
      fnew = armijo_eval(C, px, py, dx, dy, tau);
      G = (fnew - f) / (Df * tau);
    } while (G >= sigma && f >= fnew && tau <= tau_max);
    tau *= 0.5;
  } else {
    do {
      if (tau > tau_min) tau *= 0.5;
      fnew = armijo_eval(C, px, py, dx, dy, tau);
      G = (fnew - f) / (Df * tau);
    } while ((!finite(fnew) || (G < sigma || f < fnew)) && (tau > tau_min));
  }
  return (tau > tau_min) ? tau : 0.;
}

int msor_gd_level(int level, const double* R, const double* T, double* phix, double* phiy,
                  double lambda, int max_iter, double stop_eps, double* energy_out,
                  msor_step* trace, int trace_cap) {
  return msor_gd_level_dt(0, level, R, T, phix, phiy, lambda, max_iter, stop_eps, energy_out, trace, trace_cap);
}

int msor_gd_level_dt(int data_term, int level, const double* R, const double* T, double* phix, double* phiy,
                     double lambda, int max_iter, double stop_eps, double* energy_out,
                     msor_step* trace, int trace_cap) {
  const int n = lvl_n(level), N = n * n;
  double* st = stiff_build(level);
  dterm_t D;
  dterm_init(&D, data_term, level, R);
  gd_ctx C;
  memset(&C, 0, sizeof(C));
  C.level = level; C.N = N; C.R = R; C.T = T; C.st = st; C.lambda = lambda; C.D = &D;
  C.rb_tau[0] = C.rb_tau[1] = NAN;
  double* buf = (double*)calloc((size_t)N * 12, sizeof(double));
  double *dx = buf, *dy = buf + N;            /* descent direction           */
  double *ogx = buf + 2 * N, *ogy = buf + 3 * N; /* OldGradient              */
  double *odx = buf + 4 * N, *ody = buf + 5 * N; /* OldDirection             */
  double *DEx = buf + 6 * N, *DEy = buf + 7 * N; /* cached DE                */
  C.tx = buf + 8 * N; C.ty = buf + 9 * N;
  double *sx = buf + 10 * N, *sy = buf + 11 * N;

  double tau = 1.0;              /* startTau (registration.h:52) */
  double sigma = 1.0;            /* GradientDescentWithAutomaticFilterWidth (gradientDescent.h:688) */
  const double stop_sigma = 0.0001, sigma_tol = 0.00001;
  double energy = energy_with(st, &D, level, R, T, phix, phiy, lambda, NULL);
  double energy_new = energy;
  int iter = 0, n_trace = 0;
  if (max_iter <= 0) {
    if (energy_out) *energy_out = energy_new;
    free(buf); free(st); dterm_free(&D);
    return 0;
  }
  int go;
  do {
    iter++;
    energy = energy_new;
    C.e_at_pos = energy;
    C.evals = 0;
    const double sigma_used = sigma;
    /* calcTaudAndDescentDir (gradientDescent.h:200-236) */
    denergy_with(st, &D, level, R, T, phix, phiy, lambda, DEx, DEy);
    for (int i = 0; i < N; ++i) { dx[i] = DEx[i] * -1.; dy[i] = DEy[i] * -1.; }
    msor_smooth(level, sigma, dx, sx); memcpy(dx, sx, sizeof(double) * N);
    msor_smooth(level, sigma, dy, sy); memcpy(dy, sy, sizeof(double) * N);
    double beta = 0.;
    if ((iter - 1) % 10) {
      double a = 0, b = 0;
      a += dot(dx, dx, N); a += dot(dy, dy, N);
      b += dot(ogx, ogx, N); b += dot(ogy, ogy, N);
      beta = a / b;
    }
    memcpy(ogx, dx, sizeof(double) * N); memcpy(ogy, dy, sizeof(double) * N);
    for (int i = 0; i < N; ++i) { dx[i] += beta * odx[i]; dy[i] += beta * ody[i]; }
    memcpy(odx, dx, sizeof(double) * N); memcpy(ody, dy, sizeof(double) * N);
    tau = armijo(&C, phix, phiy, dx, dy, DEx, DEy, tau);
    for (int i = 0; i < N; ++i) { dx[i] *= tau; dy[i] *= tau; }
    if (tau == 0) {
      memcpy(dx, ogx, sizeof(double) * N); memcpy(dy, ogy, sizeof(double) * N);
      memset(odx, 0, sizeof(double) * N); memset(ody, 0, sizeof(double) * N);
      tau = armijo(&C, phix, phiy, dx, dy, DEx, DEy, tau);
      for (int i = 0; i < N; ++i) { dx[i] *= tau; dy[i] *= tau; }
    }
    /* energy at the new position (gradientDescent.h:356-395) */
    double enew = NAN;
    if (C.rb_tau[0] == tau) enew = C.rb_e[0];
    else if (C.rb_tau[1] == tau) enew = C.rb_e[1];
    else if (tau == 0) enew = energy;
    if (tau != 0) {
      for (int i = 0; i < N; ++i) { phix[i] += dx[i]; phiy[i] += dy[i]; }
    }
    if (isnan(enew)) enew = energy_with(st, &D, level, R, T, phix, phiy, lambda, NULL);
    energy_new = enew;
    if (trace && n_trace < trace_cap) {
      trace[n_trace].iter = iter; trace[n_trace].energy = energy_new; trace[n_trace].tau = tau;
      trace[n_trace].sigma = sigma_used; trace[n_trace].evals = C.evals; n_trace++;
    }
    /* stopping and filter-width schedule (gradientDescent.h:416-439) */
    go = ((energy - energy_new) > stop_eps) && (iter < max_iter);
    if ((0.5 * sigma > stop_sigma) && ((energy - energy_new) < sigma_tol)) {
      sigma *= 0.5;
      tau = 1.;
      go = (sigma > stop_sigma) && (iter < max_iter);
    }
  } while (go);
  if (energy_out) *energy_out = energy_new;
  free(buf);
  free(st);
  dterm_free(&D);
  return iter;
}

/* --- multilevel driver ------------------------------------------------- */

/* The displacement components of the multilevel descent are qc::Array
 * (aol::Vector) objects, so resampleInsteadOfProlongateDeformation resamples
 * the flattened node vector linearly in 1-D: aol::Vector::resampleFrom and
 * aol::Vector::interpolate (vec.h:461-472, 565-570), as called from
 * RegistrationMultilevelDescentInterface::prolongate (registration.h:510-521). */
static void resample_flat(const double* src, int ns, double* dst, int nd) {
  const double s = (ns - 1) / (double)(nd - 1);
  for (int i = 0; i < nd; ++i) {
    const double pos = i * s;
    const int p = (int)pos;
    const double pf = pos - p;
    dst[i] = (p == ns - 1) ? src[p] : (1 - pf) * src[p] + pf * src[p + 1];
  }
}

static void phi_up(int level, int resample, double* const* Px, double* const* Py) {
  if (resample) {
    const int ns = lvl_n(level) * lvl_n(level), nd = lvl_n(level + 1) * lvl_n(level + 1);
    resample_flat(Px[level], ns, Px[level + 1], nd);
    resample_flat(Py[level], ns, Py[level + 1], nd);
  } else {
    msor_prolong(level, Px[level], Px[level + 1]);
    msor_prolong(level, Py[level], Py[level + 1]);
  }
}

double msor_register(int max_level, int start_level, int stop_level, const double* R,
                     const double* T, double* phix, double* phiy, double lambda,
                     double lambda_factor, int max_iter, double stop_eps, int resample_phi,
                     int* steps_per_level) {
  return msor_register_dt(0, max_level, start_level, stop_level, R, T, phix, phiy, lambda, lambda_factor,
                          max_iter, stop_eps, resample_phi, steps_per_level);
}

static double register_core(int data_term, int max_level, int start_level, int stop_level, int lambda_stop,
                            const double* R, const double* T, double* phix, double* phiy, double lambda,
                            double lambda_factor, int max_iter, double stop_eps, int resample_phi,
                            int* steps_per_level);

double msor_register_dt(int data_term, int max_level, int start_level, int stop_level, const double* R,
                        const double* T, double* phix, double* phiy, double lambda,
                        double lambda_factor, int max_iter, double stop_eps, int resample_phi,
                        int* steps_per_level) {
  return register_core(data_term, max_level, start_level, stop_level, stop_level, R, T, phix, phiy, lambda,
                       lambda_factor, max_iter, stop_eps, resample_phi, steps_per_level);
}

/* lambda_stop: the parameter file's stopLevel, which the level weights
 * lambda * lambdaFactor^(stopLevel - level) refer to also when a solve runs
 * on other levels (the refinement of series matching).                     */
static double register_core(int data_term, int max_level, int start_level, int stop_level, int lambda_stop,
                            const double* R, const double* T, double* phix, double* phiy, double lambda,
                            double lambda_factor, int max_iter, double stop_eps, int resample_phi,
                            int* steps_per_level) {
  double *Rl[16] = {0}, *Tl[16] = {0}, *Px[16] = {0}, *Py[16] = {0};
  for (int l = 0; l <= max_level; ++l) {
    const int n = lvl_n(l);
    Rl[l] = (double*)calloc((size_t)n * n, sizeof(double));
    Tl[l] = (double*)calloc((size_t)n * n, sizeof(double));
    Px[l] = (double*)calloc((size_t)n * n, sizeof(double));
    Py[l] = (double*)calloc((size_t)n * n, sizeof(double));
  }
  const int nm = lvl_n(max_level);
  memcpy(Rl[max_level], R, sizeof(double) * nm * nm);
  memcpy(Tl[max_level], T, sizeof(double) * nm * nm);
  memcpy(Px[max_level], phix, sizeof(double) * nm * nm);
  memcpy(Py[max_level], phiy, sizeof(double) * nm * nm);
  /* MultilevelArray::levRestrict (multilevelArray.h:94-110) */
  for (int l = max_level; l > 0; --l) {
    msor_restrict(l, Rl[l], Rl[l - 1]);
    msor_restrict(l, Tl[l], Tl[l - 1]);
    msor_restrict(l, Px[l], Px[l - 1]);
    msor_restrict(l, Py[l], Py[l - 1]);
  }
  double energy = NAN;
  int cur = start_level;
  if (start_level <= stop_level) {
    for (int level = start_level; level <= stop_level; ++level) {
      /* getRegularizationWeight (registration.h:523-526) */
      const double lam = (double)pow(lambda_factor, lambda_stop - level) * lambda;
      const int steps = msor_gd_level_dt(data_term, level, Rl[level], Tl[level], Px[level], Py[level], lam,
                                         max_iter, stop_eps, &energy, NULL, 0);
      if (steps_per_level) steps_per_level[level - start_level] = steps;
      if (level < stop_level) {
        phi_up(level, resample_phi, Px, Py);
        cur = level + 1;
      }
    }
  }
  for (; cur < max_level; ++cur) phi_up(cur, resample_phi, Px, Py);
  memcpy(phix, Px[max_level], sizeof(double) * nm * nm);
  memcpy(phiy, Py[max_level], sizeof(double) * nm * nm);
  for (int l = 0; l <= max_level; ++l) { free(Rl[l]); free(Tl[l]); free(Px[l]); free(Py[l]); }
  return energy;
}

/* --- composition of displacements (series matching) ---------------------- */

/* StiffOp ONTHEFLY apply: Dest = 0, then per element (x fastest) and local
 * row i, column j: Dest[g_i] += L[i][j] * Arg[g_j]
 * (LocalAssemblyHelper::doMultiplyOnTheFly, FEOpInterface.h:136-157).      */
static void stiff_apply_onthefly(int level, const double* u, double* out) {
  const int n = lvl_n(level);
  const double h = lvl_h(level);
  const double vol = sqr(h);
  quad_t Q;
  quad_init(&Q, h);
  double L[4][4];
  for (int i = 0; i < 4; ++i) for (int j = 0; j < 4; ++j) L[i][j] = 0.;
  for (int q = 0; q < 4; ++q)
    for (int i = 0; i < 4; ++i)
      for (int j = i; j < 4; ++j) {
        double d = 0;
        d += Q.gq[i][q][0] * Q.gq[j][q][0];
        d += Q.gq[i][q][1] * Q.gq[j][q][1];
        L[i][j] += d * 1. * Q.w;
      }
  for (int i = 0; i < 4; ++i)
    for (int j = i; j < 4; ++j) L[j][i] = L[i][j] = L[i][j] * vol;
  memset(out, 0, sizeof(double) * n * n);
  for (int ey = 0; ey < n - 1; ++ey)
    for (int ex = 0; ex < n - 1; ++ex)
      for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) out[dof(n, ex, ey, i)] += L[i][j] * u[dof(n, ex, ey, j)];
}

/* Masked system matrix of SmoothlyExtendImage (deformations.h:364-410):
 * the assembled stiffness without the rows and columns of defined nodes,
 * whose diagonal is 1 (LocalAssemblyHelper::doLocalAssemblyDirichlet,
 * FEOpInterface.h:92-128).                                                  */
static double* masked_stiff_build(int level, const unsigned char* defined) {
  const int n = lvl_n(level);
  double* full = stiff_build(level);
  double* m = (double*)calloc((size_t)n * n * 9, sizeof(double));
  /* the same element-order sums as the unmasked assembly, restricted to
   * undefined rows and columns: an entry is either its full value or 0     */
  for (int r = 0; r < n * n; ++r) {
    if (defined[r]) { m[(size_t)r * 9 + 4] = 0. + 1.; continue; }
    const int x = r % n, y = r / n;
    for (int j = -1; j <= 1; ++j)
      for (int i = -1; i <= 1; ++i) {
        const int X = x + i, Y = y + j;
        if (X < 0 || X >= n || Y < 0 || Y >= n) continue;
        if (!defined[X + Y * n]) m[(size_t)r * 9 + (j + 1) * 3 + (i + 1)] = full[(size_t)r * 9 + (j + 1) * 3 + (i + 1)];
      }
  }
  free(full);
  return m;
}

/* PCGInverse::apply with the diagonal preconditioner |1/diag|
 * (solver.h:264-358, matrix.h:1256-1269, 1199-1210), absolute stopping
 * g.g < eps (solverInfo.h:162-192), at most max_iter steps.              */
static int pcg(const double* A, int level, const double* b, double* x, double eps, int max_iter) {
  const int n = lvl_n(level), N = n * n;
  double* g = (double*)calloc(N, sizeof(double));
  double* d = (double*)calloc(N, sizeof(double));
  double* h = (double*)calloc(N, sizeof(double));
  double* dinv = (double*)malloc(sizeof(double) * N);
  for (int i = 0; i < N; ++i) {
    const double a = A[(size_t)i * 9 + 4];
    dinv[i] = (a != 0.) ? fabs(1. / a) : 1.;
  }
  stiff_apply_with(A, level, x, h);
  for (int i = 0; i < N; ++i) { g[i] = h[i]; g[i] -= b[i]; }
  for (int i = 0; i < N; ++i) h[i] = g[i] * dinv[i];
  double spn = dot(g, g, N);
  for (int i = 0; i < N; ++i) d[i] -= h[i];
  int it = 0;
  while (!(spn < eps) && it < max_iter && !isnan(spn)) {
    ++it;
    const double alpha_numer = dot(g, h, N), beta_denom = alpha_numer;
    stiff_apply_with(A, level, d, h);
    const double alpha_denom = dot(d, h, N);
    for (int i = 0; i < N; ++i) x[i] += d[i] * (alpha_numer / alpha_denom);
    for (int i = 0; i < N; ++i) g[i] += h[i] * (alpha_numer / alpha_denom);
    for (int i = 0; i < N; ++i) h[i] = g[i] * dinv[i];
    const double beta_numer = dot(g, h, N);
    for (int i = 0; i < N; ++i) d[i] *= (beta_numer / beta_denom);
    for (int i = 0; i < N; ++i) d[i] -= h[i];
    spn = dot(g, g, N);
  }
  free(g); free(d); free(h); free(dinv);
  return it;
}

/* ConcatAndSmoothlyExtendDeformations (deformations.h:498-520):
 * identity + out = (identity + D1) o (identity + D2), extended where
 * x + D2(x) leaves the domain by the discrete harmonic extension of
 * SmoothlyExtendImage.  outx/outy hold the solver's initial guess on entry
 * (the previous content of the destination in the reference).              */
int msor_compose(int level, const double* d1x, const double* d1y, const double* d2x, const double* d2y,
                 double* outx, double* outy) {
  const int n = lvl_n(level), N = n * n;
  const double h = lvl_h(level);
  double* res[2];
  res[0] = (double*)malloc(sizeof(double) * N);
  res[1] = (double*)malloc(sizeof(double) * N);
  const double* d1[2] = {d1x, d1y};
  const double* d2[2] = {d2x, d2y};
  /* DeformImage with an extension image of NaN (deformations.h:225-253) */
  for (int c = 0; c < 2; ++c)
    for (int y = 0; y < n; ++y)
      for (int x = 0; x < n; ++x) {
        const int i = x + y * n;
        const double ds0 = x + d2x[i] / h, ds1 = y + d2y[i] / h;
        const int in = !(ds0 < 0. || ds0 > (double)(n - 1) || ds1 < 0. || ds1 > (double)(n - 1));
        res[c][i] = in ? interp(d1[c], n, ds0, ds1) : NAN;
      }
  for (int c = 0; c < 2; ++c)
    for (int i = 0; i < N; ++i) res[c][i] += d2[c][i];
  unsigned char* defined = (unsigned char*)malloc(N);
  for (int i = 0; i < N; ++i) defined[i] = !isnan(res[0][i]);
  /* SmoothlyExtendImage (deformations.h:364-410) */
  double* A = masked_stiff_build(level, defined);
  double* bc = (double*)malloc(sizeof(double) * N);
  double* rhs = (double*)malloc(sizeof(double) * N);
  double* out[2] = {outx, outy};
  int iters = 0;
  for (int c = 0; c < 2; ++c) {
    for (int i = 0; i < N; ++i) bc[i] = defined[i] ? res[c][i] : 0.;
    stiff_apply_onthefly(level, bc, rhs);
    for (int i = 0; i < N; ++i) rhs[i] *= -1.;
    for (int i = 0; i < N; ++i) if (defined[i]) rhs[i] = bc[i];
    iters += pcg(A, level, rhs, out[c], 1e-16, 1000);
  }
  free(A); free(bc); free(rhs); free(defined); free(res[0]); free(res[1]);
  return iters;
}

/* MultiVector::getMedianVecOverComponents (multiVector.cpp:99-117) of the
 * warped frames (DeformImage with Inf extension), Vector::getMedianValue
 * (vec.cpp:933-949); pixels without samples take fill.                     */
static int cmp_d(const void* a, const void* b) {
  const double x = *(const double*)a, y = *(const double*)b;
  return (x < y) ? -1 : (x > y) ? 1 : 0;
}

void msor_warp_median(int level, int F, const double* frames, const double* phis, double fill, double* median) {
  const int n = lvl_n(level), N = n * n;
  double* def = (double*)malloc(sizeof(double) * (size_t)N * F);
  for (int f = 0; f < F; ++f)
    msor_deform_image(level, frames + (size_t)f * N, phis + (size_t)2 * f * N,
                      phis + (size_t)(2 * f + 1) * N, INFINITY, def + (size_t)f * N);
  double* tmp = (double*)malloc(sizeof(double) * F);
  for (int j = 0; j < N; ++j) {
    int k = 0;
    for (int f = 0; f < F; ++f) {
      const double v = def[(size_t)f * N + j];
      if (v != INFINITY) tmp[k++] = v;
    }
    if (k == 0) { median[j] = fill; continue; }
    qsort(tmp, k, sizeof(double), cmp_d);
    median[j] = (k % 2 == 1) ? tmp[k / 2] : (tmp[k / 2 - 1] + tmp[k / 2]) / 2;
  }
  free(tmp);
  free(def);
}

void msor_warp_mean(int level, int F, const double* frames, const double* phis, double* mean,
                    double* count) {
  const int n = lvl_n(level), N = n * n;
  double* def = (double*)malloc(sizeof(double) * (size_t)N * F);
  for (int f = 0; f < F; ++f)
    msor_deform_image(level, frames + (size_t)f * N, phis + (size_t)2 * f * N,
                      phis + (size_t)(2 * f + 1) * N, INFINITY, def + (size_t)f * N);
  double last_mean = 0;
  for (int i = 0; i < N; ++i) last_mean += frames[(size_t)(F - 1) * N + i];
  last_mean /= N;
  for (int j = 0; j < N; ++j) {
    double a = 0;
    int k = 0;
    for (int f = 0; f < F; ++f) {
      const double v = def[(size_t)f * N + j];
      if (v != INFINITY) { a += v; ++k; }
    }
    mean[j] = (k > 0) ? a / k : last_mean;
    count[j] = k;
  }
  free(def);
}

/* --- the series pipeline --------------------------------------------------- */

/* The stage loop of matchSeries<>() (matchSeries.h:1250-1320) with its
 * default options, each stage SeriesMatching::matchSeries with accumulated
 * deformations (matchSeries.h:87-265) followed by averageSeries
 * (matchSeries.h:353-445):
 *   stage 1: reference frame 0, templates 1..F-1; stage s > 1: reference the
 *   average (median with use_median) of stage s-1, templates 0..F-1, lambda
 *   the "%f" print of lambda * extra_lambda_factor (matchSeries.h:1300).
 *   Per template i: registration to the previous template (to the reference
 *   for i = 0) from zero; acc = compose(current, acc); for i > 0 refinement
 *   of acc against the stage reference on refine_start..refine_stop.
 * The images are prepared by msor_normalize(sat, min_to_zero) like the
 * reference's loadRefOrTemplate; the average and median warp the raw frames.
 * Outputs of the last stage: phis (m x 2 x N, m = F-1 without extra stages,
 * else F), avg, median, count (N each); energies (nullable) receives, per
 * stage, m energies (the pairwise one for i = 0, the refined one after).    */
void msor_match_series(int data_term, int level, int start, int stop, double lambda, double lambda_factor,
                       int max_iter, double stop_eps, double sat, int min_to_zero, int refine_start,
                       int refine_stop, int extra_stages, double extra_lambda_factor, int use_median, int F,
                       const double* frames, double* phis, double* avg, double* median, double* count,
                       double* energies) {
  const int n = lvl_n(level), N = n * n;
  double* target = (double*)malloc(sizeof(double) * N);
  double* R = (double*)malloc(sizeof(double) * N);
  double* Rprev = (double*)malloc(sizeof(double) * N);
  double* T = (double*)malloc(sizeof(double) * N);
  double* cur = (double*)malloc(sizeof(double) * 2 * N);
  double* acc = (double*)malloc(sizeof(double) * 2 * N);
  double* tmp = (double*)malloc(sizeof(double) * 2 * N);
  memcpy(target, frames, sizeof(double) * N);
  int eoff = 0;
  for (int stage = 1; stage <= 1 + extra_stages; ++stage) {
    double lam = lambda;
    if (stage > 1) {
      char buf[64];
      snprintf(buf, sizeof buf, "%f", lambda * extra_lambda_factor);
      lam = atof(buf);
    }
    const int first = (stage == 1) ? 1 : 0, m = F - first;
    memcpy(R, target, sizeof(double) * N);
    msor_normalize(R, N, sat, min_to_zero);
    memcpy(Rprev, R, sizeof(double) * N);
    memset(acc, 0, sizeof(double) * 2 * N);
    for (int i = 0; i < m; ++i) {
      memcpy(T, frames + (size_t)(first + i) * N, sizeof(double) * N);
      msor_normalize(T, N, sat, min_to_zero);
      memset(cur, 0, sizeof(double) * 2 * N);
      double e = register_core(data_term, level, start, stop, stop, Rprev, T, cur, cur + N, lam, lambda_factor,
                               max_iter, stop_eps, 0, NULL);
      memcpy(tmp, acc, sizeof(double) * 2 * N);
      msor_compose(level, cur, cur + N, tmp, tmp + N, acc, acc + N);
      if (i > 0)
        e = register_core(data_term, level, refine_start, refine_stop, stop, R, T, acc, acc + N, lam,
                          lambda_factor, max_iter, stop_eps, 0, NULL);
      memcpy(phis + (size_t)2 * i * N, (i == 0) ? cur : acc, sizeof(double) * 2 * N);
      if (energies) energies[eoff + i] = e;
      memcpy(Rprev, T, sizeof(double) * N);
    }
    eoff += m;
    msor_warp_mean(level, m, frames + (size_t)first * N, phis, avg, count);
    double last_mean = 0;
    for (int j = 0; j < N; ++j) last_mean += frames[(size_t)(F - 1) * N + j];
    last_mean /= N;
    msor_warp_median(level, m, frames + (size_t)first * N, phis, last_mean, median);
    memcpy(target, use_median ? median : avg, sizeof(double) * N);
  }
  free(target); free(R); free(Rprev); free(T); free(cur); free(acc); free(tmp);
}

/* --- the seismic line-shift data term --------------------------------------- */
/* FELineShiftRegisEnergy (registration.h:2137-2193): per line y of an nx x ny
 * image, the 1-D NormalizedCrossCorrelationEnergy (registration.h:1909-1983)
 * of the reference line and the template line under the line's displacement,
 * on RectangularGridConfigurator<double, QC_1D, Gauss 3> (configurators.h:
 * 746-820): nodes 0..nx-1, h = 1/(nx-1), two Gauss points, assembled 1-D
 * mass matrix (DiagBandMatrix<.,1,1>, diagBandMatrix.cpp:123-160).  Lines
 * whose first reference or template value is NaN are skipped; the energy is
 * the sum over lines divided by ny, the derivative of each line too.      */
typedef struct {
  int n;
  double h, vol;
  double bq[2][2];   /* basis b at Gauss point q */
  double band[0];
} line1d_t;

static line1d_t* line1d_new(int n) {
  line1d_t* L = (line1d_t*)calloc(1, sizeof(line1d_t) + sizeof(double) * 3 * (size_t)n);
  L->n = n;
  L->h = 1. / (double)(n - 1);
  L->vol = L->h;
  const double g[2] = {GP0, GP1};
  for (int q = 0; q < 2; ++q) { L->bq[0][q] = 1. - g[q]; L->bq[1][q] = g[q]; }
  double M[2][2] = {{0., 0.}, {0., 0.}};
  for (int q = 0; q < 2; ++q)
    for (int i = 0; i < 2; ++i) {
      const double bi = L->bq[i][q];
      for (int j = i; j < 2; ++j) M[i][j] += bi * L->bq[j][q] * 1. * 0.5;
    }
  for (int i = 0; i < 2; ++i)
    for (int j = i; j < 2; ++j) M[j][i] = M[i][j] = M[i][j] * L->vol;
  for (int e = 0; e < n - 1; ++e)
    for (int i = 0; i < 2; ++i)
      for (int j = 0; j < 2; ++j) L->band[(size_t)(e + i) * 3 + (j - i + 1)] += 1.0 * M[i][j];
  return L;
}

static void line1d_mass(const line1d_t* L, const double* u, double* out) {
  const int n = L->n;
  for (int i = 0; i < n; ++i) {
    double r = 0.;
    for (int j = (i > 0 ? i - 1 : 0); j <= (i < n - 1 ? i + 1 : n - 1); ++j) r += L->band[(size_t)i * 3 + (j - i + 1)] * u[j];
    out[i] = r;
  }
}

static double line1d_normalize(const line1d_t* L, const double* img, double* out, double* tmp) {
  const int n = L->n;
  line1d_mass(L, img, tmp);
  double mean = 0.;
  for (int i = 0; i < n; ++i) mean += tmp[i];
  for (int i = 0; i < n; ++i) { out[i] = img[i]; out[i] += -mean; }
  line1d_mass(L, out, tmp);
  const double var = sqrt(dot(out, tmp, n));
  if (!(fabs(var - 0.) < 1e-15))
    for (int i = 0; i < n; ++i) out[i] /= var;
  return var;
}

/* doFastDeformImage<., QC_1D> (deformations.h:111-137) with
 * Vector::interpolate (vec.h:461-472) */
static void line1d_deform(const line1d_t* L, const double* img, const double* phi, double* out) {
  const int n = L->n;
  for (int i = 0; i < n; ++i) {
    double ds = i + phi[i] / L->h;
    ds = ds < 0. ? 0. : (ds > (double)(n - 1) ? (double)(n - 1) : ds);
    const int p = (int)ds;
    const double pf = ds - p;
    out[i] = (p == n - 1) ? img[p] : (1 - pf) * img[p] + pf * img[p + 1];
  }
}

static double line1d_energy(const line1d_t* L, const double* normR, const double* T, const double* phi, double* var,
                            double* normT, double* w1, double* w2) {
  const int n = L->n;
  line1d_deform(L, T, phi, w1);
  *var = line1d_normalize(L, w1, normT, w2);
  line1d_mass(L, normT, w1);
  return -dot(w1, normR, n);
}

/* VariationOfNormalizedCrossCorrelationEnergy::apply on one line: the energy,
 * then CrossCorrelationForce (registration.h:1828-1862) integrated like
 * FENonlinVectorOpInterface::applyAdd (FEOpInterface.h:1803-1852). */
static void line1d_variation(const line1d_t* L, const double* normR, const double* T, const double* phi, double* dy,
                             double* w1, double* w2, double* normT, double* temp) {
  const int n = L->n;
  double var;
  const double energy = line1d_energy(L, normR, T, phi, &var, normT, w1, w2);
  for (int i = 0; i < n; ++i) temp[i] = normR[i];
  for (int i = 0; i < n; ++i) temp[i] += normT[i] * energy;
  if (!(fabs(var - 0.) < 1e-15))
    for (int i = 0; i < n; ++i) temp[i] /= var;
  const double g[2] = {GP0, GP1};
  for (int i = 0; i < n; ++i) dy[i] = 0.;
  for (int e = 0; e < n - 1; ++e) {
    double nl[2];
    for (int q = 0; q < 2; ++q) {
      double off = 0.;
      off += phi[e] * L->bq[0][q];
      off += phi[e + 1] * L->bq[1][q];
      const double tc = ((double)e + g[q]) + off / L->h;
      int el = (short)tc;
      double loc = tc - el;
      if (el == n - 1 && loc == 0) { el = n - 2; loc = 1; }
      if (tc < 0. || el < 0 || el >= n - 1) { nl[q] = 0.; continue; }
      double gr = 0.;
      double v = -1. / L->h;
      v *= T[el];
      gr += v;
      v = 1. / L->h;
      v *= T[el + 1];
      gr += v;
      double tq = 0.;
      tq += temp[e] * L->bq[0][q];
      tq += temp[e + 1] * L->bq[1][q];
      nl[q] = gr * -tq;
    }
    for (int b = 0; b < 2; ++b) {
      double a = 0.;
      for (int q = 0; q < 2; ++q) a += nl[q] * (L->bq[b][q] * 0.5);
      dy[e + b] += L->vol * a;
    }
  }
}

double msor_lineshift(int nx, int ny, const double* R, const double* T, const double* phix, double* de) {
  line1d_t* L = line1d_new(nx);
  double* normR = (double*)malloc(sizeof(double) * nx);
  double* w1 = (double*)malloc(sizeof(double) * nx);
  double* w2 = (double*)malloc(sizeof(double) * nx);
  double* w3 = (double*)malloc(sizeof(double) * nx);
  double* w4 = (double*)malloc(sizeof(double) * nx);
  double e = 0.;
  if (de) memset(de, 0, sizeof(double) * (size_t)nx * ny);
  for (int y = 0; y < ny; ++y) {
    const double* r = R + (size_t)y * nx;
    const double* t = T + (size_t)y * nx;
    const double* p = phix + (size_t)y * nx;
    if (isnan(r[0]) || isnan(t[0])) continue;
    line1d_normalize(L, r, normR, w1);
    double var;
    e += line1d_energy(L, normR, t, p, &var, w3, w1, w2);
    if (de) {
      double* dy = de + (size_t)y * nx;
      line1d_variation(L, normR, t, p, dy, w1, w2, w3, w4);
      for (int i = 0; i < nx; ++i) dy[i] /= ny;
    }
  }
  e /= ny;
  free(L); free(normR); free(w1); free(w2); free(w3); free(w4);
  return e;
}

/* The regulariser of findXShift for laplaceWeight <= 0 (matchSeries.h:
 * 819-845): K = stiffX + yRegFactor * stiffY, FEOpMixedDerivative
 * (FEOpInterface.h:1075-1135) with local matrices
 * L[i][j] += 1 * g_i[s] * g_j[t] * w, times vol = h^2, assembled element by
 * element into the nine-point band matrix (stiffX first, then stiffY with the
 * factor), on the nx x ny rectangular grid with h = 1/(max(nx,ny)-1);
 * E = 1/2 phi.(K phi) (QuadraticFormOp, op.h:1410-1429).  Returns E, Kphi out. */
double msor_xshift_reg(int nx, int ny, double yreg, const double* phi, double* kphi) {
  const double h = 1. / (double)((nx > ny ? nx : ny) - 1);
  const double vol = sqr(h);
  quad_t Q;
  quad_init(&Q, h);
  double* st = (double*)calloc((size_t)nx * ny * 9, sizeof(double));
  for (int pass = 0; pass < 2; ++pass) {
    const int s = pass;  /* stiffX: s = t = 0; stiffY: s = t = 1 */
    const double factor = pass == 0 ? 1.0 : yreg;
    double L[4][4];
    for (int i = 0; i < 4; ++i) for (int j = 0; j < 4; ++j) L[i][j] = 0.;
    for (int q = 0; q < 4; ++q)
      for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) L[i][j] += 1. * Q.gq[i][q][s] * Q.gq[j][q][s] * Q.w;
    for (int i = 0; i < 4; ++i) for (int j = 0; j < 4; ++j) L[i][j] *= vol;
    for (int ey = 0; ey < ny - 1; ++ey)
      for (int ex = 0; ex < nx - 1; ++ex)
        for (int i = 0; i < 4; ++i)
          for (int j = 0; j < 4; ++j) {
            const int gi = ex + ey * nx + ((i & 1) ? 1 : 0) + ((i & 2) ? nx : 0);
            const int gj = ex + ey * nx + ((j & 1) ? 1 : 0) + ((j & 2) ? nx : 0);
            const int dx = (gj % nx) - (gi % nx), dy = (gj / nx) - (gi / nx);
            st[(size_t)gi * 9 + (dy + 1) * 3 + (dx + 1)] += factor * L[i][j];
          }
  }
  for (int r = 0; r < nx * ny; ++r) {
    const int x = r % nx, y = r / nx;
    double d = 0.;
    for (int j = -1; j <= 1; ++j)
      for (int i = -1; i <= 1; ++i) {
        const int X = x + i, Y = y + j;
        if (X >= 0 && X < nx && Y >= 0 && Y < ny) d += st[(size_t)r * 9 + (j + 1) * 3 + (i + 1)] * phi[X + Y * nx];
      }
    kphi[r] = d;
  }
  free(st);
  return 0.5 * dot(kphi, phi, nx * ny);
}

/* The regulariser of findXShift for laplaceWeight > 0 (matchSeries.h:828-838):
 * K = w L M^{-1} L + stiffX + yRegFactor stiffY with L the assembled Q1
 * stiffness (StiffOp) and M the lumped mass (LumpedMassOp, inverted), the
 * product formed as qc::assembleLaplaceSquareRegMatrix does
 * (hyperelastic.h:234-251: rows of L scaled by M^{-1}, then
 * aol::Matrix::addMatrixProduct, matrix.cpp:414-429, which adds
 * L[i][k] * (M^{-1}L)[k][j] into entry (i, j) for k in increasing column
 * order of row i -- aol::SparseRow keeps its entries sorted), scaled by w,
 * then stiffX and yRegFactor * stiffY added element by element; applied as
 * the column-sorted CSR_Matrix (sparseMatrices.h CSRMatrix::apply: a
 * row's sum from 0 in column order).  25-point rows (offsets -2..2).
 * Returns E = 1/2 phi.(K phi), K phi out.                                  */
double msor_xshift_reg_laplace(int nx, int ny, double yreg, double w, const double* phi, double* kphi) {
  const int N = nx * ny;
  const double h = 1. / (double)((nx > ny ? nx : ny) - 1), vol = sqr(h);
  quad_t Q;
  quad_init(&Q, h);
  /* L: rect_system's stiffness pass alone (StiffOp = FELinScalarWeightedStiffInterface, coefficient 1) */
  double Ls[4][4];
  for (int i = 0; i < 4; ++i) for (int j = 0; j < 4; ++j) Ls[i][j] = 0.;
  for (int q = 0; q < 4; ++q)
    for (int i = 0; i < 4; ++i)
      for (int j = i; j < 4; ++j) {
        double d = 0;
        d += Q.gq[i][q][0] * Q.gq[j][q][0];
        d += Q.gq[i][q][1] * Q.gq[j][q][1];
        Ls[i][j] += d * 1. * Q.w;
      }
  for (int i = 0; i < 4; ++i)
    for (int j = i; j < 4; ++j) Ls[j][i] = Ls[i][j] = Ls[i][j] * vol;
  double* L = (double*)calloc((size_t)N * 9, sizeof(double));
  double* lm = (double*)calloc((size_t)N, sizeof(double));
  double lmloc[4] = {0., 0., 0., 0.};
  for (int q = 0; q < 4; ++q)
    for (int i = 0; i < 4; ++i) lmloc[i] += 1. * Q.bq[i][q] * Q.w;
  for (int i = 0; i < 4; ++i) lmloc[i] *= vol;
  for (int ey = 0; ey < ny - 1; ++ey)
    for (int ex = 0; ex < nx - 1; ++ex)
      for (int i = 0; i < 4; ++i) {
        const int gi = ex + ey * nx + ((i & 1) ? 1 : 0) + ((i & 2) ? nx : 0);
        lm[gi] += lmloc[i];
        for (int j = 0; j < 4; ++j) {
          const int gj = ex + ey * nx + ((j & 1) ? 1 : 0) + ((j & 2) ? nx : 0);
          const int dx = (gj % nx) - (gi % nx), dy = (gj / nx) - (gi / nx);
          L[(size_t)gi * 9 + (dy + 1) * 3 + (dx + 1)] += Ls[i][j];
        }
      }
  /* K = w (L M^{-1} L) as 25-point rows, accumulated in increasing k */
  double* K = (double*)calloc((size_t)N * 25, sizeof(double));
  for (int r = 0; r < N; ++r) {
    const int x = r % nx, y = r / nx;
    double* kr = K + (size_t)r * 25;
    for (int a = -1; a <= 1; ++a)
      for (int b = -1; b <= 1; ++b) {
        const int X = x + b, Y = y + a;
        if (X < 0 || X >= nx || Y < 0 || Y >= ny) continue;
        const int k = X + Y * nx;
        const double lik = L[(size_t)r * 9 + (a + 1) * 3 + (b + 1)];
        const double minv = 1. / lm[k];
        for (int c = -1; c <= 1; ++c)
          for (int d = -1; d <= 1; ++d) {
            const int X2 = X + d, Y2 = Y + c;
            if (X2 < 0 || X2 >= nx || Y2 < 0 || Y2 >= ny) continue;
            const double m2 = L[(size_t)k * 9 + (c + 1) * 3 + (d + 1)] * minv;
            kr[(a + c + 2) * 5 + (b + d + 2)] += lik * m2;
          }
      }
    for (int e = 0; e < 25; ++e) kr[e] *= w;
  }
  /* + stiffX + yRegFactor stiffY, element by element (FEOpMixedDerivative) */
  for (int pass = 0; pass < 2; ++pass) {
    const int sd = pass;
    const double factor = pass == 0 ? 1.0 : yreg;
    double Lm[4][4];
    for (int i = 0; i < 4; ++i) for (int j = 0; j < 4; ++j) Lm[i][j] = 0.;
    for (int q = 0; q < 4; ++q)
      for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) Lm[i][j] += 1. * Q.gq[i][q][sd] * Q.gq[j][q][sd] * Q.w;
    for (int i = 0; i < 4; ++i) for (int j = 0; j < 4; ++j) Lm[i][j] *= vol;
    for (int ey = 0; ey < ny - 1; ++ey)
      for (int ex = 0; ex < nx - 1; ++ex)
        for (int i = 0; i < 4; ++i)
          for (int j = 0; j < 4; ++j) {
            const int gi = ex + ey * nx + ((i & 1) ? 1 : 0) + ((i & 2) ? nx : 0);
            const int gj = ex + ey * nx + ((j & 1) ? 1 : 0) + ((j & 2) ? nx : 0);
            const int dx = (gj % nx) - (gi % nx), dy = (gj / nx) - (gi / nx);
            K[(size_t)gi * 25 + (dy + 2) * 5 + (dx + 2)] += factor * Lm[i][j];
          }
  }
  for (int r = 0; r < N; ++r) {
    const int x = r % nx, y = r / nx;
    double sum = 0.;
    for (int a = -2; a <= 2; ++a)
      for (int b = -2; b <= 2; ++b) {
        const int X = x + b, Y = y + a;
        if (X < 0 || X >= nx || Y < 0 || Y >= ny) continue;
        sum += K[(size_t)r * 25 + (a + 2) * 5 + (b + 2)] * phi[X + Y * nx];
      }
    kphi[r] = sum;
  }
  free(L); free(lm); free(K);
  return 0.5 * dot(kphi, phi, N);
}

/* --- the seismic solve: findXShift (matchSeries.h:805-865) -------------------- */
/* Nine-point rows of an assembled Q1 operator on the nx x ny rectangular grid
 * (h = 1/(max(nx,ny)-1)): mass (FELinScalarWeightedMassInterface) with factor
 * fm, then stiffness (FELinScalarWeightedStiffInterface) with factor fs, each
 * assembled element by element (InverseH1MetricBase::assembleSystemMatrix,
 * linearSmoothOp.h:295-299).                                                */
static double* rect_system(int nx, int ny, double fm, double fs) {
  const double h = 1. / (double)((nx > ny ? nx : ny) - 1), vol = sqr(h);
  quad_t Q;
  quad_init(&Q, h);
  double Mm[4][4], Ls[4][4];
  for (int i = 0; i < 4; ++i) for (int j = 0; j < 4; ++j) { Mm[i][j] = 0.; Ls[i][j] = 0.; }
  for (int q = 0; q < 4; ++q)
    for (int i = 0; i < 4; ++i) {
      const double bi = Q.bq[i][q];
      for (int j = i; j < 4; ++j) {
        Mm[i][j] += bi * Q.bq[j][q] * 1. * Q.w;
        double d = 0;
        d += Q.gq[i][q][0] * Q.gq[j][q][0];
        d += Q.gq[i][q][1] * Q.gq[j][q][1];
        Ls[i][j] += d * 1. * Q.w;
      }
    }
  for (int i = 0; i < 4; ++i)
    for (int j = i; j < 4; ++j) { Mm[j][i] = Mm[i][j] = Mm[i][j] * vol; Ls[j][i] = Ls[i][j] = Ls[i][j] * vol; }
  double* st = (double*)calloc((size_t)nx * ny * 9, sizeof(double));
  for (int pass = 0; pass < 2; ++pass) {
    if (pass == 1 && fs == 0.) break;
    for (int ey = 0; ey < ny - 1; ++ey)
      for (int ex = 0; ex < nx - 1; ++ex)
        for (int i = 0; i < 4; ++i)
          for (int j = 0; j < 4; ++j) {
            const int gi = ex + ey * nx + ((i & 1) ? 1 : 0) + ((i & 2) ? nx : 0);
            const int gj = ex + ey * nx + ((j & 1) ? 1 : 0) + ((j & 2) ? nx : 0);
            const int dx = (gj % nx) - (gi % nx), dy = (gj / nx) - (gi / nx);
            st[(size_t)gi * 9 + (dy + 1) * 3 + (dx + 1)] += pass == 0 ? fm * Mm[i][j] : fs * Ls[i][j];
          }
  }
  return st;
}

static void rect_apply(const double* st, int nx, int ny, const double* u, double* out) {
  for (int r = 0; r < nx * ny; ++r) {
    const int x = r % nx, y = r / nx;
    double d = 0.;
    for (int j = -1; j <= 1; ++j)
      for (int i = -1; i <= 1; ++i) {
        const int X = x + i, Y = y + j;
        if (X >= 0 && X < nx && Y >= 0 && Y < ny) d += st[(size_t)r * 9 + (j + 1) * 3 + (i + 1)] * u[X + Y * nx];
      }
    out[r] = d;
  }
}

/* M + tau L with tau = 0.5 sigma^2 (InverseH1MetricBase::setSigma) applied to x */
void msor_h1sys_apply(int nx, int ny, double sigma, const double* x, double* y) {
  double* st = rect_system(nx, ny, 1.0, (double)(0.5f * sqr(sigma)));
  rect_apply(st, nx, ny, x, y);
  free(st);
}

/* Band Cholesky of a nine-point SPD matrix (half-bandwidth nx + 1): the
 * exact solve that CholeskyBasedInverseH1Metric (linearSmoothOp.h:345-378)
 * obtains from SuiteSparse's CHOLMOD, which the reference does not vendor. */
typedef struct { int N, b; double* L; } band_chol_t;

static band_chol_t band_chol(const double* st, int nx, int ny) {
  band_chol_t C;
  C.N = nx * ny;
  C.b = nx + 1;
  const int b = C.b;
  C.L = (double*)calloc((size_t)C.N * (b + 1), sizeof(double));  /* L[i*(b+1) + k] = A(i, i-k) */
  for (int r = 0; r < C.N; ++r) {
    const int x = r % nx, y = r / nx;
    for (int j = -1; j <= 1; ++j)
      for (int i = -1; i <= 1; ++i) {
        const int X = x + i, Y = y + j;
        if (X < 0 || X >= nx || Y < 0 || Y >= ny) continue;
        const int c = X + Y * nx;
        if (c <= r) C.L[(size_t)r * (b + 1) + (r - c)] = st[(size_t)r * 9 + (j + 1) * 3 + (i + 1)];
      }
  }
  for (int i = 0; i < C.N; ++i) {
    for (int k = (i - b > 0 ? i - b : 0); k < i; ++k) {
      double s = C.L[(size_t)i * (b + 1) + (i - k)];
      for (int m = (i - b > k - b ? i - b : k - b); m < k; ++m)
        if (m >= 0) s -= C.L[(size_t)i * (b + 1) + (i - m)] * C.L[(size_t)k * (b + 1) + (k - m)];
      C.L[(size_t)i * (b + 1) + (i - k)] = s / C.L[(size_t)k * (b + 1)];
    }
    double s = C.L[(size_t)i * (b + 1)];
    for (int m = (i - b > 0 ? i - b : 0); m < i; ++m) s -= sqr(C.L[(size_t)i * (b + 1) + (i - m)]);
    C.L[(size_t)i * (b + 1)] = sqrt(s);
  }
  return C;
}

static void band_chol_solve(const band_chol_t* C, double* x) {
  const int N = C->N, b = C->b;
  for (int i = 0; i < N; ++i) {
    double s = x[i];
    for (int m = (i - b > 0 ? i - b : 0); m < i; ++m) s -= C->L[(size_t)i * (b + 1) + (i - m)] * x[m];
    x[i] = s / C->L[(size_t)i * (b + 1)];
  }
  for (int i = N - 1; i >= 0; --i) {
    double s = x[i];
    for (int m = i + 1; m <= (i + b < N - 1 ? i + b : N - 1); ++m) s -= C->L[(size_t)m * (b + 1) + (m - i)] * x[m];
    x[i] = s / C->L[(size_t)i * (b + 1)];
  }
}

/* (M + 0.5 sigma^2 L)^{-1} x in place */
void msor_h1_metric(int nx, int ny, double sigma, double* x) {
  double* st = rect_system(nx, ny, 1.0, (double)(0.5f * sqr(sigma)));
  band_chol_t C = band_chol(st, nx, ny);
  band_chol_solve(&C, x);
  free(C.L);
  free(st);
}

typedef struct {
  int nx, ny, N;
  const double *R, *T;
  double lambda, yreg, lapw;   /* lapw: laplaceWeight (> 0: the Laplace-square regulariser) */
  double rb_tau[2], rb_e[2];
  int rb_pos, evals;
  double e_at_pos;
  double *tx, *w;
  int yconst;                  /* findXShiftYConst: the unknown is one shift per line (N = ny) */
  double *full, *defull;       /* nx*ny scratch of the row-constant mode */
} xs_ctx;

/* qc::ScalarArray<QC_2D>::setInXDirectionFrom (scalarArray.h:1409-1416) */
static void yc_expand(const xs_ctx* C, const double* v) {
  for (int y = 0; y < C->ny; ++y)
    for (int x = 0; x < C->nx; ++x) C->full[(size_t)y * C->nx + x] = v[y];
}

static double xs_reg(xs_ctx* C, const double* phi) {
  return C->lapw > 0 ? msor_xshift_reg_laplace(C->nx, C->ny, C->yreg, C->lapw, phi, C->w)
                     : msor_xshift_reg(C->nx, C->ny, C->yreg, phi, C->w);
}

/* E = EData + lambda * ERegStiff (LinCombOp, matchSeries.h:847-850) */
static double xs_energy(xs_ctx* C, const double* phi) {
  if (C->yconst) {   /* PixelWiseToRowWiseOp::apply (quocOps.h:195-199): the data term alone */
    yc_expand(C, phi);
    return msor_lineshift(C->nx, C->ny, C->R, C->T, C->full, NULL);
  }
  double e = 0.;
  e += msor_lineshift(C->nx, C->ny, C->R, C->T, phi, NULL);
  e += C->lambda * xs_reg(C, phi);
  return e;
}

/* DE = DEData + lambda * K phi */
static void xs_gradient(xs_ctx* C, const double* phi, double* de) {
  if (C->yconst) {   /* PixelWiseToRowWiseOp::applyDerivative: row sums (sumInXDirectionTo, scalarArray.h:1395-1402) */
    yc_expand(C, phi);
    msor_lineshift(C->nx, C->ny, C->R, C->T, C->full, C->defull);
    for (int y = 0; y < C->ny; ++y) {
      double sum = 0.;
      for (int x = 0; x < C->nx; ++x) sum += C->defull[(size_t)y * C->nx + x];
      de[y] = sum;
    }
    return;
  }
  msor_lineshift(C->nx, C->ny, C->R, C->T, phi, de);
  xs_reg(C, phi);
  for (int i = 0; i < C->N; ++i) de[i] += C->lambda * C->w[i];
}

static double xs_eval(xs_ctx* C, const double* p, const double* d, double tw) {
  if (tw == 0) return C->e_at_pos;
  for (int i = 0; i < C->N; ++i) { C->tx[i] = p[i]; C->tx[i] += tw * d[i]; }
  const double e = xs_energy(C, C->tx);
  C->rb_tau[C->rb_pos] = tw;
  C->rb_e[C->rb_pos] = e;
  C->rb_pos ^= 1;
  C->evals++;
  return e;
}

static double xs_armijo(xs_ctx* C, const double* p, const double* d, const double* DE, double old_tau) {
  const double sigma = 0.5, tau_min = pow(2., -30.), tau_max = pow(2., 25.);
  double tau = old_tau < tau_min ? tau_min : (old_tau > tau_max ? tau_max : old_tau);
  const double f = xs_eval(C, p, d, 0.);
  double fnew = xs_eval(C, p, d, tau);
  const double Df = dot(DE, d, C->N);
  double G = (fnew - f) / (Df * tau);
  if (Df >= 0) return 0;
  if (!finite(f)) return 0;
  if (G >= sigma && f >= fnew) {
    do {
      tau *= 2.;
      fnew = xs_eval(C, p, d, tau);
      G = (fnew - f) / (Df * tau);
    } while (G >= sigma && f >= fnew && tau <= tau_max);
    tau *= 0.5;
  } else {
    do {
      if (tau > tau_min) tau *= 0.5;
      fnew = xs_eval(C, p, d, tau);
      G = (fnew - f) / (Df * tau);
    } while ((!finite(fnew) || (G < sigma || f < fnew)) && (tau > tau_min));
  }
  return (tau > tau_min) ? tau : 0.;
}

/* The template smoothed along x for findXShiftYConst: Template.applyLinearFilterTo
 * with a (4i+1) x (4i+1) kernel whose middle row is 1/(4i+1) and the other
 * rows 0 (ScalarArray<QC_2D>::getConvolveValue, scalarArray.cpp:936-965: the
 * whole window in row order, periodic outside the array, so the zero rows
 * still carry a NaN of their pixels).                                      */
void msor_box_x(const double* T, int nx, int ny, int i, double* out) {
  const int o = 2 * i;
  const double k = 1. / (double)(2 * o + 1);
  for (int y = 0; y < ny; ++y)
    for (int x = 0; x < nx; ++x) {
      double val = 0.0;
      for (int oy = -o; oy <= o; ++oy)
        for (int ox = -o; ox <= o; ++ox) {
          int X = x + ox, Y = y + oy;
          if (X < 0) X += nx; else if (X > nx - 1) X = X % nx;
          if (Y < 0) Y += ny; else if (Y > ny - 1) Y = Y % ny;
          val += (oy == 0 ? k : 0.0) * T[(size_t)Y * nx + X];
        }
      out[(size_t)y * nx + x] = val;
    }
}

/* replaceEmptyLinesWithNaN (matchSeismicSeries.h:141-157): a line whose
 * squared norm (Vector::normSqr, the sum of the squares in index order) is 0
 * is overwritten by quiet NaNs.  A NaN sample makes the norm NaN, so such a
 * line is kept.                                                            */
int msor_empty_lines_to_nan(double* img, int nx, int ny) {
  int replaced = 0;
  for (int y = 0; y < ny; ++y) {
    double* line = img + (size_t)y * nx;
    double s = 0.0;
    for (int x = 0; x < nx; ++x) s += line[x] * line[x];
    if (s == 0.0) {
      for (int x = 0; x < nx; ++x) line[x] = NAN;
      ++replaced;
    }
  }
  return replaced;
}

/* removeEmptyLinesFromImage (matchSeismicSeries.h:101-136): a line is empty
 * when its squared norm is 0 or it holds NaNs only.  The kept top and bottom
 * blocks count the empty lines there in units of the mean distance of the
 * non-empty lines, rounded by aol::Rint (aol.h:422).  The reference divides
 * by that distance, which is 0 for a single non-empty line: -2 here.      */
int msor_remove_empty_lines(const double* img, int nx, int ny, int keep_top_bottom, double* out) {
  int count = 0, first = -1, last = -1;
  for (int y = 0; y < ny; ++y) {
    const double* line = img + (size_t)y * nx;
    double s = 0.0;
    int non_nan = 0;
    for (int x = 0; x < nx; ++x) {
      s += line[x] * line[x];
      if (!isnan(line[x])) ++non_nan;
    }
    if (s == 0.0 || non_nan == 0) continue;
    if (first < 0) first = y;
    last = y;
    ++count;
  }
  if (count == 0) return -1;
  int top = 0, bottom = 0;
  if (keep_top_bottom) {
    if (count == 1) return -2;
    const double d = (last - first) / (double)(count - 1);
    const int dist = d >= 0 ? (int)(d + 0.5) : (int)(d - 0.5);
    top = first / dist;
    bottom = (ny - 1 - last) / dist;
  }
  const int out_ny = count + top + bottom;
  memset(out, 0, sizeof(double) * (size_t)nx * out_ny);
  int k = top;
  for (int y = 0; y < ny; ++y) {
    const double* line = img + (size_t)y * nx;
    double s = 0.0;
    int non_nan = 0;
    for (int x = 0; x < nx; ++x) {
      s += line[x] * line[x];
      if (!isnan(line[x])) ++non_nan;
    }
    if (s == 0.0 || non_nan == 0) continue;
    memcpy(out + (size_t)k * nx, line, sizeof(double) * nx);
    ++k;
  }
  return out_ny;
}

/* findXShiftYConst (matchSeries.h:873-920): one shift per line, started from
 * the line means of phix; four descents (GridlessGradientDescent with
 * Fletcher-Reeves NCG: GradientDescentBase::applySingle, gradientDescent.h:
 * 295-464, without smoothing or filter widths, stopping when the Armijo step
 * is 0) against the template smoothed along x by boxes of 13, 9 and 5
 * samples and then unsmoothed; E = the line-shift data term of the
 * row-constant shift, DE its derivative summed along each line.  phix
 * (nx*ny) in/out; returns the steps of the last descent.                  */
int msor_xshift_yconst(int nx, int ny, const double* R, const double* T, int max_iter, double* phix,
                       double* energy_out) {
  const int N = nx * ny;
  xs_ctx C;
  memset(&C, 0, sizeof(C));
  C.nx = nx; C.ny = ny; C.N = ny; C.R = R; C.yconst = 1;
  double* big = (double*)calloc((size_t)N * 3, sizeof(double));
  double* Ts = big;
  C.full = big + N; C.defull = big + 2 * N;
  double* buf = (double*)calloc((size_t)ny * 7, sizeof(double));
  double *v = buf, *d = buf + ny, *og = buf + 2 * ny, *od = buf + 3 * ny, *DE = buf + 4 * ny;
  C.tx = buf + 5 * ny; C.w = buf + 6 * ny;
  for (int y = 0; y < ny; ++y) {
    double sum = 0.;
    for (int x = 0; x < nx; ++x) sum += phix[(size_t)y * nx + x];
    v[y] = sum;
  }
  for (int y = 0; y < ny; ++y) v[y] /= (double)nx;
  double energy_new = INFINITY;
  int iter = 0;
  for (int round = 3; round >= 0; --round) {
    if (round > 0) msor_box_x(T, nx, ny, round, Ts);
    else memcpy(Ts, T, sizeof(double) * N);
    C.T = Ts;
    C.rb_tau[0] = C.rb_tau[1] = NAN;
    C.rb_pos = 0;
    memset(og, 0, sizeof(double) * ny);
    memset(od, 0, sizeof(double) * ny);
    double tau = 1.0;
    double energy = xs_energy(&C, v);
    energy_new = energy;
    iter = 0;
    int go = max_iter > 0;
    while (go) {
      iter++;
      energy = energy_new;
      C.e_at_pos = energy;
      C.evals = 0;
      xs_gradient(&C, v, DE);
      for (int i = 0; i < ny; ++i) d[i] = DE[i] * -1.;
      double beta = 0.;
      if ((iter - 1) % 10) beta = dot(d, d, ny) / dot(og, og, ny);
      memcpy(og, d, sizeof(double) * ny);
      for (int i = 0; i < ny; ++i) d[i] += beta * od[i];
      memcpy(od, d, sizeof(double) * ny);
      tau = xs_armijo(&C, v, d, DE, tau);
      for (int i = 0; i < ny; ++i) d[i] *= tau;
      if (tau == 0) {
        memcpy(d, og, sizeof(double) * ny);
        memset(od, 0, sizeof(double) * ny);
        tau = xs_armijo(&C, v, d, DE, tau);
        for (int i = 0; i < ny; ++i) d[i] *= tau;
      }
      double enew = NAN;
      if (C.rb_tau[0] == tau) enew = C.rb_e[0];
      else if (C.rb_tau[1] == tau) enew = C.rb_e[1];
      else if (tau == 0) enew = energy;
      if (tau != 0)
        for (int i = 0; i < ny; ++i) v[i] += d[i];
      if (isnan(enew)) enew = xs_energy(&C, v);
      energy_new = enew;
      go = ((energy - energy_new) > 0.) && (iter < max_iter);
      if (tau == 0) go = 0;
    }
  }
  for (int y = 0; y < ny; ++y)
    for (int x = 0; x < nx; ++x) phix[(size_t)y * nx + x] = v[y];
  if (energy_out) *energy_out = energy_new;
  free(big);
  free(buf);
  return iter;
}

/* findXShift with laplaceWeight <= 0: GradientDescentWithAutomaticFilterWidth
 * over H1GradientDescent with the exact inverse H1 metric, Fletcher-Reeves
 * NCG, Armijo (the control of gradientDescent.h:295-464, 675-691 and
 * ArmijoSearch.h:118-200, as in msor_gd_level_dt, on one component); phix is
 * scaled by nx/max(nx,ny) around the descent (matchSeries.h:860-864).
 * Returns the steps; *energy_out the energy at the end.                    */
int msor_xshift(int nx, int ny, const double* R, const double* T, double lambda, double yreg, double laplace_weight,
                int max_iter, double* phix, double* energy_out, msor_step* trace, int trace_cap) {
  const int N = nx * ny;
  xs_ctx C;
  memset(&C, 0, sizeof(C));
  C.nx = nx; C.ny = ny; C.N = N; C.R = R; C.T = T; C.lambda = lambda; C.yreg = yreg; C.lapw = laplace_weight;
  C.rb_tau[0] = C.rb_tau[1] = NAN;
  double* buf = (double*)calloc((size_t)N * 6, sizeof(double));
  double *d = buf, *og = buf + N, *od = buf + 2 * N, *DE = buf + 3 * N;
  C.tx = buf + 4 * N; C.w = buf + 5 * N;
  const double scale = (double)nx / (double)(nx > ny ? nx : ny);
  for (int i = 0; i < N; ++i) phix[i] /= scale;
  double tau = 1.0, sigma = 1.0;
  const double stop_sigma = 0.0001, sigma_tol = 0.00001, stop_eps = 0.;
  band_chol_t chol = {0, 0, NULL};
  double chol_sigma = 0.;
  double energy = xs_energy(&C, phix), energy_new = energy;
  int iter = 0, n_trace = 0, go = max_iter > 0;
  while (go) {
    iter++;
    energy = energy_new;
    C.e_at_pos = energy;
    C.evals = 0;
    const double sigma_used = sigma;
    xs_gradient(&C, phix, DE);
    for (int i = 0; i < N; ++i) d[i] = DE[i] * -1.;
    /* the factorisation is redone only when the filter width changes
     * (InverseH1MetricBase::setTau, linearSmoothOp.h:283-288) */
    if (!chol.L || chol_sigma != sigma) {
      free(chol.L);
      double* sys = rect_system(nx, ny, 1.0, (double)(0.5f * sqr(sigma)));
      chol = band_chol(sys, nx, ny);
      free(sys);
      chol_sigma = sigma;
    }
    band_chol_solve(&chol, d);
    double beta = 0.;
    if ((iter - 1) % 10) beta = dot(d, d, N) / dot(og, og, N);
    memcpy(og, d, sizeof(double) * N);
    for (int i = 0; i < N; ++i) d[i] += beta * od[i];
    memcpy(od, d, sizeof(double) * N);
    tau = xs_armijo(&C, phix, d, DE, tau);
    for (int i = 0; i < N; ++i) d[i] *= tau;
    if (tau == 0) {
      memcpy(d, og, sizeof(double) * N);
      memset(od, 0, sizeof(double) * N);
      tau = xs_armijo(&C, phix, d, DE, tau);
      for (int i = 0; i < N; ++i) d[i] *= tau;
    }
    double enew = NAN;
    if (C.rb_tau[0] == tau) enew = C.rb_e[0];
    else if (C.rb_tau[1] == tau) enew = C.rb_e[1];
    else if (tau == 0) enew = energy;
    if (tau != 0)
      for (int i = 0; i < N; ++i) phix[i] += d[i];
    if (isnan(enew)) enew = xs_energy(&C, phix);
    energy_new = enew;
    if (trace && n_trace < trace_cap) {
      trace[n_trace].iter = iter; trace[n_trace].energy = energy_new; trace[n_trace].tau = tau;
      trace[n_trace].sigma = sigma_used; trace[n_trace].evals = C.evals; n_trace++;
    }
    go = ((energy - energy_new) > stop_eps) && (iter < max_iter);
    if ((0.5 * sigma > stop_sigma) && ((energy - energy_new) < sigma_tol)) {
      sigma *= 0.5;
      tau = 1.;
      go = (sigma > stop_sigma) && (iter < max_iter);
    }
  }
  for (int i = 0; i < N; ++i) phix[i] *= scale;
  if (energy_out) *energy_out = energy_new;
  free(chol.L);
  free(buf);
  return iter;
}
