/*
 * ms_oracle.h -- FP64 CPU restatement of matchSeries' SSD + Dirichlet H1
 * gradient-flow registration on the uniform 2^l+1 grid.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker that the CUDA path
 * is compared against (tests, the smoke check and the CPU-baseline leg of the
 * benchmark).  The product path never links or calls it.
 *
 * Parity status: pinned.  Every entry point below is compared against the
 * reference's own templates (compiled from the quocmesh sources by
 * oracle/Makefile.ref into oracle/_ref/ms_ref) on the golden fixtures under
 * tests/golden/.
 *
 * Conventions (shared with the reference):
 *   level l  ->  n = 2^l + 1 nodes per side, h = 1 / 2^l, N = n*n nodes.
 *   Node (x, y) is stored at index x + y*n (x fastest, quoc ILex order).
 *   Displacements are in domain units: a pixel shift equals phi / h.
 */
#ifndef MS_ORACLE_H
#define MS_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* One gradient-flow step as logged by the oracle's level solve. */
typedef struct {
  int    iter;        /* 1-based step number                              */
  double energy;      /* energy after the step (E_data + lambda * E_reg)  */
  double tau;         /* accepted Armijo step (0 = step rejected)        */
  double sigma;       /* filter width used for this step's H1 smoothing  */
  int    evals;       /* energy evaluations spent in the line search(es) */
} msor_step;

/* --- single operators -------------------------------------------------- */
/* SSDEnergy::apply  (registration.h:1584-1616, FEOpInterface.h:2586-2613) */
double msor_ssd_energy(int level, const double* R, const double* T,
                       const double* phix, const double* phiy);
/* SSDForce::apply   (registration.h:1623-1667, FEOpInterface.h:1803-1852) */
void   msor_ssd_force(int level, const double* R, const double* T,
                      const double* phix, const double* phiy,
                      double* gx, double* gy);
/* StiffOp ASSEMBLED apply, one component (FEOpInterface.h:2333-2347)      */
void   msor_stiff_apply(int level, const double* u, double* Lu);
/* E = SSD + lambda * 1/2 sum_c phi_c . L phi_c ; returns E, E_reg in *ereg */
double msor_energy(int level, const double* R, const double* T,
                   const double* phix, const double* phiy, double lambda,
                   double* ereg);
/* DE = SSDForce + lambda * L phi  (LinCombOp, registration.h:977-982)      */
void   msor_denergy(int level, const double* R, const double* T,
                    const double* phix, const double* phiy, double lambda,
                    double* gx, double* gy);
/* LinearSmoothOp::apply with tau = sigma^2/2 (linearSmoothOp.cpp:591-612)  */
void   msor_smooth(int level, double sigma, const double* in, double* out);
/* same, with tau given directly (used by the image pre-smoothing)          */
void   msor_smooth_tau(int level, double tau, const double* in, double* out);
/* RestrictOp<STD_QUOC_RESTRICT> (restriction.cpp:397-470)                 */
void   msor_restrict(int fine_level, const double* fine, double* coarse);
/* ProlongOp::std_mg_prolongate (prolongation.cpp:195-232)                  */
void   msor_prolong(int coarse_level, const double* coarse, double* fine);
/* ScalarArray::resampleFrom, bilinear (scalarArray.h:310-333,1052-1059)    */
void   msor_resample(int src_level, const double* src, int dst_level, double* dst);
/* DeformImage with constant extension (deformations.h:62-101)             */
void   msor_deform_image(int level, const double* img, const double* phix,
                         const double* phiy, double ext_value, double* out);
/* saturated min/max + clamp + scaleValuesTo01 (registration.h:331-346,
 * vec.h:864-871,1084-1089).  sat_percent < 0 selects the branch without
 * enhanceContrastSaturationPercentage (min -> 0 if normalize_min_to_zero or
 * min < 0, then divide by max).                                            */
void   msor_normalize(double* img, int count, double sat_percent,
                      int normalize_min_to_zero);

/* --- solvers ----------------------------------------------------------- */
/* GradientDescentWithAutomaticFilterWidth<H1GradientDescent>::applySingle
 * with Armijo + Fletcher-Reeves NCG (gradientDescent.h:295-464,
 * ArmijoSearch.h:118-200).  phi is updated in place.  Returns the number of
 * steps; *energy_out receives the energy at the final position.
 * trace (may be NULL) receives at most trace_cap steps.                   */
int    msor_gd_level(int level, const double* R, const double* T,
                     double* phix, double* phiy, double lambda, int max_iter,
                     double stop_eps, double* energy_out,
                     msor_step* trace, int trace_cap);

/* RegistrationMultilevelDescentInterface::solveAndProlongToMaxDepth
 * (registration.h:462-467, quocDescent.h:83-105): R/T are the prepared
 * full-resolution images at max_level; they are restricted down, phi (at
 * max_level, in/out) is restricted down to start_level, the levels
 * start..stop are solved, phi is prolongated up to max_level (with
 * resample_phi: resampled as the flattened node vector, which is what the
 * reference's qc::Array components do).  Returns the energy of the last level solve.
 * steps_per_level (may be NULL) gets stop-start+1 entries.                */
double msor_register(int max_level, int start_level, int stop_level,
                     const double* R, const double* T,
                     double* phix, double* phiy,
                     double lambda, double lambda_factor, int max_iter,
                     double stop_eps, int resample_phi, int* steps_per_level);

/* Mean of the frames warped by their displacements with Inf extension and a
 * per-pixel count of finite samples (matchSeries.h:385-425).  frames and
 * phis are F consecutive images (phis: phix0, phiy0, phix1, ...).  Pixels
 * without any sample take the mean of the last frame.                     */
void   msor_warp_mean(int level, int num_frames, const double* frames,
                      const double* phis, double* mean, double* count);

/* --- normalized cross-correlation data term ------------------------------
 * data_term 0 = SSD (the functions above), 1 = NCC:
 * NormalizedCrossCorrelationEnergy / VariationOfNormalizedCrossCorrelationEnergy
 * (registration.h:1909-2018) with the same Dirichlet regulariser.          */
/* MassOp ASSEMBLED apply (FEOpInterface.h:2382-2394, 1445-1475)             */
void   msor_mass_apply(int level, const double* u, double* Mu);
/* the NCC energy alone (computeEnergy, registration.h:1950-1962)           */
double msor_ncc_energy(int level, const double* R, const double* T,
                       const double* phix, const double* phiy);
/* its variation alone (applyDerivative, registration.h:1972-1983)          */
void   msor_ncc_variation(int level, const double* R, const double* T,
                          const double* phix, const double* phiy, double* gx, double* gy);
double msor_energy_dt(int data_term, int level, const double* R, const double* T,
                      const double* phix, const double* phiy, double lambda, double* ereg);
void   msor_denergy_dt(int data_term, int level, const double* R, const double* T,
                       const double* phix, const double* phiy, double lambda,
                       double* gx, double* gy);
int    msor_gd_level_dt(int data_term, int level, const double* R, const double* T,
                        double* phix, double* phiy, double lambda, int max_iter,
                        double stop_eps, double* energy_out, msor_step* trace, int trace_cap);
double msor_register_dt(int data_term, int max_level, int start_level, int stop_level,
                        const double* R, const double* T, double* phix, double* phiy,
                        double lambda, double lambda_factor, int max_iter, double stop_eps,
                        int resample_phi, int* steps_per_level);

/* --- series matching helpers -------------------------------------------- */
/* ConcatAndSmoothlyExtendDeformations (deformations.h:498-520): out = the
 * displacement of (id + d1) o (id + d2), harmonically extended where
 * x + d2(x) leaves the domain; outx/outy carry the PCG's initial guess in.
 * Returns the PCG iterations of both components.                          */
int    msor_compose(int level, const double* d1x, const double* d1y, const double* d2x,
                    const double* d2y, double* outx, double* outy);
/* median of the warped frames over the finite samples (averageSeries,
 * matchSeries.h:442; multiVector.cpp:99-117), fill where none            */
void   msor_warp_median(int level, int F, const double* frames, const double* phis, double fill,
                        double* median);
/* The seismic model's line-shift data term (FELineShiftRegisEnergy,
 * registration.h:2137-2193): the mean over the ny lines of the 1-D NCC energy
 * of each reference line against its template line shifted by phix along x
 * (units of the line grid, h = 1/(nx-1)); de (nullable) its derivative.    */
double msor_lineshift(int nx, int ny, const double* R, const double* T, const double* phix, double* de);
/* findXShift's regulariser (laplaceWeight <= 0): K = stiffX + yreg * stiffY
 * on the nx x ny grid; returns 1/2 phi.K phi, K phi into kphi.             */
double msor_xshift_reg(int nx, int ny, double yreg, const double* phi, double* kphi);
/* findXShift's regulariser with laplaceWeight w > 0: w L M^{-1} L + stiffX + yreg stiffY */
double msor_xshift_reg_laplace(int nx, int ny, double yreg, double w, const double* phi, double* kphi);
/* (M + tau L) x with tau = 0.5 sigma^2 on the nx x ny rectangular grid
 * (InverseH1MetricBase's system matrix), and its exact inverse in place.   */
void   msor_h1sys_apply(int nx, int ny, double sigma, const double* x, double* y);
void   msor_h1_metric(int nx, int ny, double sigma, double* x);
/* findXShift (matchSeries.h:805-865) with the exact H1 metric; laplace_weight
 * > 0 selects the Laplace-square regulariser: phix (nx*ny) in/out; returns
 * the steps.                                                               */
int    msor_xshift(int nx, int ny, const double* R, const double* T, double lambda, double yreg,
                   double laplace_weight, int max_iter, double* phix, double* energy_out, msor_step* trace,
                   int trace_cap);
/* findXShiftYConst (matchSeries.h:873-920): one shift per line; phix in/out */
int    msor_xshift_yconst(int nx, int ny, const double* R, const double* T, int max_iter, double* phix,
                          double* energy_out);
void   msor_box_x(const double* T, int nx, int ny, int i, double* out);
/* replaceEmptyLinesWithNaN (matchSeismicSeries.h:141-157) on ny lines of nx
 * samples, in place; returns the number of lines replaced                 */
int    msor_empty_lines_to_nan(double* img, int nx, int ny);
/* removeEmptyLinesFromImage (matchSeismicSeries.h:101-136): out (ny lines
 * at most) gets the non-empty lines, with keep_top_bottom the empty blocks at
 * the top and bottom as zero lines; returns its line count, -1 when every
 * line is empty, -2 when keep_top_bottom meets a single non-empty line     */
int    msor_remove_empty_lines(const double* img, int nx, int ny, int keep_top_bottom, double* out);
/* matchSeries<>() with accumulated deformations, refinement and extra stages
 * (matchSeries.h:87-265, 353-445, 1250-1320); see ms_oracle.c.             */
void   msor_match_series(int data_term, int level, int start, int stop, double lambda,
                         double lambda_factor, int max_iter, double stop_eps, double sat,
                         int min_to_zero, int refine_start, int refine_stop, int extra_stages,
                         double extra_lambda_factor, int use_median, int F, const double* frames,
                         double* phis, double* avg, double* median, double* count,
                         double* energies);

#ifdef __cplusplus
}
#endif
#endif
