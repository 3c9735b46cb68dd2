/*
 * msgpu.h -- C ABI of the B200 implementation of matchSeries' multilevel
 * SSD + Dirichlet H1 gradient-flow registration and warped-frame average.
 *
 * Plain pointers and sizes only.  Every function returns an msgpu_status;
 * on failure msgpu_last_error() gives the message (the reference throws
 * aol::Exception with file and line; a C++ adapter rethrows this text).
 * A context is bound to one CUDA device and is not shared between threads.
 * Host-pointer entry points are synchronous.  They refuse input images that
 * hold NaN or Inf with MSGPU_ERR_INVALID_ARG (the reference's saturated
 * min/max sorts the image, and with NaN the order is unspecified); with the
 * device entry points such results are unspecified.  Images are (2^l+1)^2 float64
 * arrays, x fastest (quoc ILex order); displacements are in domain units
 * (pixel shift = phi * 2^l) and stored as [phi_x, phi_y] per frame.
 */
#ifndef MSGPU_H
#define MSGPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  MSGPU_OK = 0,
  MSGPU_ERR_INVALID_ARG = 1,   /* null pointer, bad level range, ...        */
  MSGPU_ERR_SIZE = 2,          /* input size does not match the grid        */
  MSGPU_ERR_CUDA = 3,          /* CUDA runtime or launch failure            */
  MSGPU_ERR_UNSUPPORTED = 4    /* option not provided by this build         */
} msgpu_status;

typedef struct msgpu_context msgpu_context;

/* Scheduling of the level kernel on one level (no counterpart in the
 * reference).  The results do not depend on it: every tile keeps its own
 * partial sums and a pass adds them in a fixed order.                      */
typedef struct {
  int chunk_div;     /* a pass is handed out in chunks of ntiles / chunk_div
                        tiles (0: default 24)                                */
  int chunk_max;     /* at most chunk_max tiles per chunk (0: default 16)    */
  int ctas_per_sm;   /* CTAs of the persistent grid per SM (0: as many as
                        fit, which is 2)                                    */
  float ms;          /* msgpu_autotune_device: the level's measured time    */
} msgpu_level_tuning;

/* The parameter-file keys of the registration path (names as in the
 * reference's .par files; see msgpu_params_default for the defaults).       */
typedef struct {
  int precision_level;         /* precisionLevel: images are (2^l+1)^2      */
  int input_level;             /* level of the input images (>= precision)  */
  int start_level;             /* startLevel                                 */
  int stop_level;              /* stopLevel                                  */
  double lambda;               /* lambda                                     */
  double lambda_factor;        /* lambdaFactor (1 when absent)               */
  int max_gd_iterations;       /* maxGDIterations                            */
  double stop_epsilon;         /* stopEpsilon (0 when absent)                */
  double saturation_percent;   /* enhanceContrastSaturationPercentage; <0 = absent */
  int normalize_min_to_zero;   /* normalizeMinToZero                         */
  int dont_normalize_input;    /* dontNormalizeInputImages                   */
  int resample_deformation;    /* resampleInsteadOfProlongateDeformation     */
  int use_fp64;                /* 0: FP32 bulk + FP64 reductions; 1: FP64   */
  int data_term;               /* deformationModel's data term: 0 SSD
                                  (SSDRegistrationConfigurator), 1 normalized
                                  cross-correlation (NCCRegistrationConfigurator,
                                  registration.h:1766-1780, 1909-2018)        */
  int sum_order;               /* order of the global FP64 sums of a level
                                  solve (no parameter-file key; the reference
                                  has only its own order): 0 (default) the
                                  reference's sequential order, every sum the
                                  reference's double bit for bit, so the
                                  gradient flow takes the reference's steps;
                                  1 a fixed parallel order (deterministic, a
                                  little faster, sums within rounding of the
                                  reference's).  Applies with use_fp64 = 1
                                  and data_term = 0; otherwise the parallel
                                  order is used.                            */
} msgpu_params;

void msgpu_params_default(msgpu_params* p);
int  msgpu_abi_version(void);

/* Bounds of the device-side waits, in seconds, for every context of the
 * process (no counterpart in the reference, which has no device waits):
 * level_wait_s bounds one wait of a level-kernel worker for work (default
 * 4 s), barrier_wait_s one grid-barrier wait of the composition kernel
 * (default 2 s); a value <= 0 restores the default.  A kernel whose wait runs
 * out sets an error flag and returns; the synchronous entry points then
 * report MSGPU_ERR_CUDA and the context stays usable.  A diagnostic hook:
 * shorter bounds make the waits run out on purpose, so that these error
 * paths can be checked without a stuck kernel.                             */
int  msgpu_set_wait_limits(double level_wait_s, double barrier_wait_s);

int  msgpu_create(int device, msgpu_context** out);
/* Data term (0 SSD, 1 NCC) of the single-operator entry points msgpu_energy
 * and msgpu_gd_level of this context; the batch entry points take it from
 * msgpu_params.data_term.                                                  */
int  msgpu_set_data_term(msgpu_context* ctx, int data_term);
/* Order of the global sums (msgpu_params.sum_order) of the single-operator
 * entry points msgpu_energy and msgpu_gd_level of this context (default 0). */
int  msgpu_set_sum_order(msgpu_context* ctx, int sum_order);
/* Certified control steps with sum order 0 (default on).  A pass's sums in
 * the reference's order differ from its parallel sums by at most
 * 2 gamma_{N-1} sum |t| (N terms t); the level kernel takes each control
 * decision (Armijo tests, stop rule, sigma schedule) on these bounds when
 * they settle it, and adds the sums in order only where a decision stays
 * open, where a value is written out (energies, logs) or enters arithmetic
 * (the Fletcher-Reeves factor).  The results are those of the ordered sums
 * either way; on costs six term buffers per instance of a level launch
 * (at most 32 GiB per launch, beyond that one).  Off: every pass's sums
 * are added in order.                                                      */
int  msgpu_set_certified_steps(msgpu_context* ctx, int on);
/* findXShift's descent control (msgpu_find_xshift{,_device,_batch}) on the
 * device (1): the descent is captured once into a CUDA graph whose step loop
 * and Armijo searches are conditional while nodes and whose fallback attempt
 * and energy re-evaluation are conditional if nodes, the decisions taken by
 * one-thread kernels from the sums on the device -- one graph launch per
 * descent.  0 (default): the same control on the host, measured faster on
 * B200.  The two take the same decisions in the same double arithmetic:
 * identical results.                                                       */
int  msgpu_set_seismic_device_control(msgpu_context* ctx, int on);
/* Warm-started batches (msgpu_register_batch_warm{,_device}): the step limit
 * of the levels between the network's output level and the stop level
 * (0, the default: maxGDIterations).  They start near their solution; the
 * stop level still runs to the stated energy tolerance.                    */
int  msgpu_set_warm_schedule(msgpu_context* ctx, int coarse_iters);
int  msgpu_destroy(msgpu_context* ctx);
const char* msgpu_last_error(const msgpu_context* ctx);

/* One stage of series matching against a fixed reference: every template is
 * prepared like the reference image (prepareMultilevelArray,
 * registration.h:331-367), registered from initial_phis (NULL = zero,
 * setTransformationToZero registration.h:570-574) by
 * solveAndProlongToMaxDepth (registration.h:462-467), and returned at the
 * precision level.  Replaces the per-frame loop of SeriesMatching::matchSeries
 * (matchSeries.h:141-155, 223-245) for all frames of the stage at once.
 *   reference  : (2^input_level+1)^2 doubles
 *   templates  : num_templates such images
 *   phis_out   : num_templates * 2 * (2^precision_level+1)^2 doubles
 *   energies_out (nullable): energy of the last level solve per template
 *                (getEnergyOfLastSolution, registration.h:1117-1119)
 *   steps_out  (nullable): num_templates * (stop-start+1) gradient steps     */
int msgpu_register_batch(msgpu_context* ctx, const msgpu_params* p, const double* reference,
                         const double* templates, int num_templates, const double* initial_phis,
                         double* phis_out, double* energies_out, int* steps_out);

/* Same with device pointers, enqueued on the CUDA stream `stream`
 * (a cudaStream_t; NULL = legacy default stream); returns after enqueueing.
 * energies_out/steps_out are device pointers too (nullable).               */
int msgpu_register_batch_device(msgpu_context* ctx, const msgpu_params* p, const double* d_reference,
                                const double* d_templates, int num_templates, const double* d_initial_phis,
                                double* d_phis_out, double* d_energies_out, int* d_steps_out,
                                void* stream);

/* averageSeries (matchSeries.h:385-425): each frame is warped by its
 * displacement with DeformImage and Inf extension (deformations.h:62-101,
 * registration.h:595-610); mean over the finite samples per pixel, pixels
 * without samples take the last frame's mean; count = number of samples.   */
int msgpu_warp_mean(msgpu_context* ctx, int level, const double* frames, const double* phis,
                    int num_frames, double* mean_out, double* count_out);
int msgpu_warp_mean_device(msgpu_context* ctx, int level, const double* d_frames, const double* d_phis,
                           int num_frames, double* d_mean_out, double* d_count_out, void* stream);

/* The average of a stage whose frames are sharded over several GPUs (no
 * single counterpart in the reference, which averages in one process):
 * msgpu_warp_sum_device gives, for this rank's frames, the per-pixel sum of
 * the finite warped samples and their number (averageSeries,
 * matchSeries.h:410-425) and, when d_last_mean_out is not NULL, the mean of
 * its last frame (the fill of pixels without samples when this rank holds
 * the series' last frame); the caller adds the ranks' sums and counts (one
 * all-reduce, e.g. NCCL) and msgpu_mean_from_sums_device divides:
 * mean = sum / count, or *d_fill where count is 0.  The result equals
 * msgpu_warp_mean over all frames up to the order of the per-pixel sums.   */
int msgpu_warp_sum_device(msgpu_context* ctx, int level, const double* d_frames, const double* d_phis,
                          int num_frames, double* d_sum_out, double* d_count_out, double* d_last_mean_out,
                          void* stream);
int msgpu_mean_from_sums_device(msgpu_context* ctx, int level, const double* d_sum, const double* d_count,
                                const double* d_fill, double* d_mean_out, void* stream);

/* One stage of series matching in one call: msgpu_register_batch followed by
 * msgpu_warp_mean of the raw templates with their displacements (the stage
 * loop of matchSeries<>(), matchSeries.h:1284-1316, with averageSeries).
 * One upload of the images, one download of the results.                  */
int msgpu_match_series_stage(msgpu_context* ctx, const msgpu_params* p, const double* reference,
                             const double* templates, int num_templates, double* phis_out,
                             double* energies_out, int* steps_out, double* mean_out, double* count_out);
int msgpu_match_series_stage_device(msgpu_context* ctx, const msgpu_params* p, const double* d_reference,
                                    const double* d_templates, int num_templates, double* d_phis_out,
                                    double* d_energies_out, int* d_steps_out, double* d_mean_out,
                                    double* d_count_out, void* stream);

/* --- ragged batches -------------------------------------------------------
 * Many series of different sizes in one batch (no counterpart in the
 * reference, which registers one frame at a time): every template is
 * registered to the reference of its series as msgpu_register_batch does,
 * and one level-kernel launch per level serves every series that has that
 * level (the largest series run alone on their finest levels).  Each series
 * brings its own level (precision = input = stop level); of msgpu_params the
 * batch uses start_level (common to all series), lambda, lambda_factor
 * (weights count from each series' own stop level), max_gd_iterations,
 * stop_epsilon, the normalisation keys, resample_deformation, use_fp64 and
 * data_term.  A frame's result does not depend on the batch it is in.    */
typedef struct {
  int level;                 /* (2^level+1)^2 images                          */
  int num_templates;
  const double* reference;   /* one image                                     */
  const double* templates;   /* num_templates images                          */
  double* phis_out;          /* num_templates * 2 * (2^level+1)^2 doubles     */
  double* energies_out;      /* nullable: num_templates doubles               */
} msgpu_series_desc;
/* host buffers; synchronous */
int msgpu_register_ragged(msgpu_context* ctx, const msgpu_params* p, const msgpu_series_desc* series,
                          int num_series);
/* device buffers, enqueued on `stream` */
int msgpu_register_ragged_device(msgpu_context* ctx, const msgpu_params* p, const msgpu_series_desc* series,
                                 int num_series, void* stream);

/* --- the seismic line-shift model (matchSeismicSeries): its energy --------
 * Images are nx x ny doubles, x fastest; displacements shift along x in the
 * units of a line (h = 1/(nx-1)), as findXShift passes them
 * (matchSeries.h:860-864).                                                   */
/* FELineShiftRegisEnergy (registration.h:2137-2193): the mean over the lines
 * of the 1-D normalized cross-correlation of each reference line and its
 * template line shifted by phix (lines whose first reference or template
 * value is NaN are skipped); de_out (nullable): its derivative.            */
int msgpu_lineshift_energy(msgpu_context* ctx, int nx, int ny, const double* R, const double* T, const double* phix,
                           double* energy_out, double* de_out);
/* num_images images back to back, one energy each; device pointers.      */
int msgpu_lineshift_energy_device(msgpu_context* ctx, int nx, int ny, int num_images, const double* d_R,
                                  const double* d_T, const double* d_phix, double* d_energy_out, double* d_de_out,
                                  void* stream);
/* findXShift's regulariser (matchSeries.h:819-845) on the nx x ny grid
 * (h = 1/(max(nx,ny)-1)): K = stiffX + yreg * stiffY for laplace_weight <= 0,
 * K = laplace_weight * L M^-1 L + stiffX + yreg * stiffY for laplace_weight
 * > 0 (qc::assembleLaplaceSquareRegMatrix, hyperelastic.h:234-251; grids of
 * at least 5 x 5 nodes); energy 1/2 phix.K phix and K phix.                */
int msgpu_xshift_reg(msgpu_context* ctx, int nx, int ny, double yreg, double laplace_weight, const double* phix,
                     double* energy_out, double* kphi_out);
int msgpu_xshift_reg_device(msgpu_context* ctx, int nx, int ny, int num_images, double yreg, double laplace_weight,
                            const double* d_phix, double* d_energy_out, double* d_kphi_out, void* stream);

/* findXShift (matchSeries.h:805-865), laplaceWeight as in msgpu_xshift_reg: the gradient
 * flow with automatic filter width, Fletcher-Reeves NCG and Armijo steps on
 * E = line-shift data term + lambda * 1/2 phix.K phix, in the metric of
 * (M + sigma^2/2 L)^{-1} (CholeskyBasedInverseH1Metric, linearSmoothOp.h:
 * 345-378, here applied exactly through the spectral basis of the grid).
 *   phix: nx*ny doubles, the x-displacement in/out in the units of the 2-D
 *   grid (h = 1/(max(nx,ny)-1); scaled to line units inside, as findXShift
 *   does).  max_iter: maxGDIterations (the reference's default is 500).
 *   energy_out, steps_out (nullable): host values.                         */
int msgpu_find_xshift(msgpu_context* ctx, int nx, int ny, const double* R, const double* T, double lambda,
                      double yreg, double laplace_weight, int max_iter, double* phix, double* energy_out,
                      int* steps_out);
int msgpu_find_xshift_device(msgpu_context* ctx, int nx, int ny, const double* d_R, const double* d_T, double lambda,
                             double yreg, double laplace_weight, int max_iter, double* d_phix, double* energy_out,
                             int* steps_out, void* stream);

/* replaceEmptyLinesWithNaN (matchSeismicSeries.h:141-157), which
 * XShiftNonDyadicRegistrationMultilevelDescent applies to its reference and
 * template before the non-dyadic solve (matchSeismicSeries.h:179-185,
 * 211-228): every line of the num_images images (nx*ny each, back to back)
 * whose squared norm is 0 is overwritten in place by quiet NaNs, so that the
 * line-shift data term skips it (registration.h:2150-2151).  replaced_out
 * (nullable, host): the number of lines replaced.                          */
int msgpu_empty_lines_to_nan(msgpu_context* ctx, int nx, int ny, int num_images, double* img, int* replaced_out);
int msgpu_empty_lines_to_nan_device(msgpu_context* ctx, int nx, int ny, int num_images, double* d_img,
                                    int* replaced_out, void* stream);

/* removeEmptyLinesFromImage (matchSeismicSeries.h:101-136), the input of the
 * dyadic pre-stage (initMLADroppingEmptyLines, matchSeismicSeries.h:
 * 187-192): out (capacity nx*ny; not the input) receives the lines of img
 * whose squared norm is not 0 and which are not all NaN, in order; with
 * keep_top_bottom (keepEmptyTopBottomBlocks) preceded and followed by zero
 * lines for the empty blocks at the top and bottom, counted in units of the
 * non-empty lines' mean distance.  *out_ny: the lines written.  Only empty
 * lines: MSGPU_ERR_INVALID_ARG "Input contains only empty lines"; the same
 * code for keep_top_bottom with a single non-empty line, where the reference
 * divides by zero.                                                         */
int msgpu_remove_empty_lines(msgpu_context* ctx, int nx, int ny, const double* img, int keep_top_bottom, double* out,
                             int* out_ny);
int msgpu_remove_empty_lines_device(msgpu_context* ctx, int nx, int ny, const double* d_img, int keep_top_bottom,
                                    double* d_out, int* out_ny, void* stream);

/* findXShiftYConst (matchSeries.h:873-920), the non-dyadic solve of
 * XShiftNonDyadicRegistrationMultilevelDescent under
 * forceNonDyadicXShiftYConst (matchSeismicSeries.h:197-201): one shift per
 * line, started from the line means of phix, by four gradient descents
 * (GridlessGradientDescent, Fletcher-Reeves NCG, Armijo steps; no metric)
 * against the template smoothed along x by boxes of 13, 9 and 5 samples and
 * then unsmoothed, on the line-shift data term alone.  phix (nx*ny) in/out,
 * returned constant along each line; energy_out, steps_out (nullable, host):
 * the last descent's energy and steps.                                     */
int msgpu_find_xshift_yconst(msgpu_context* ctx, int nx, int ny, const double* R, const double* T, int max_iter,
                             double* phix, double* energy_out, int* steps_out);
int msgpu_find_xshift_yconst_device(msgpu_context* ctx, int nx, int ny, const double* d_R, const double* d_T,
                                    int max_iter, double* d_phix, double* energy_out, int* steps_out, void* stream);

/* findXShift for num_images images (host buffers, back to back): R is one
 * reference for all (r_per_image = 0, e.g. the mean stack) or one per image;
 * phix in/out; energies_out, steps_out (nullable) per image.  The images are
 * spread over `workers` host threads (< 1: 4), each with its own stream and
 * buffers, so that their descents overlap on the GPU (no counterpart in the
 * reference, which registers one image at a time).  Kernel-launch counts of
 * all workers are summed in msgpu_get_stats.                               */
int msgpu_find_xshift_batch(msgpu_context* ctx, int nx, int ny, int num_images, const double* R, int r_per_image,
                            const double* T, double lambda, double yreg, double laplace_weight, int max_iter,
                            double* phix, double* energies_out, int* steps_out, int workers);

/* --- series pipeline ------------------------------------------------------ */
/* Options of matchSeries<>() beyond the registration keys (parameter-file
 * names of the reference).                                                  */
typedef struct {
  int refine_start_level;            /* refineStartLevel (required by the reference) */
  int refine_stop_level;             /* refineStopLevel (default precisionLevel)     */
  int num_extra_stages;              /* numExtraStages                               */
  double extra_stages_lambda_factor; /* extraStagesLambdaFactor                      */
  int use_median_as_new_target;      /* useMedianAsNewTarget                         */
  int dont_accumulate_deformation;   /* dontAccumulateDeformation                    */
} msgpu_series_params;
/* refine levels = the registration's start_level .. precision_level, no extra
 * stages, factor 1, average as the new target, accumulation on.             */
void msgpu_series_params_default(const msgpu_params* p, msgpu_series_params* s);

/* matchSeries<>() (matchSeries.h:1250-1320) with SeriesMatching::matchSeries
 * (matchSeries.h:87-265) and averageSeries (matchSeries.h:353-445) per stage:
 *   stage 1: frame 0 is the reference, frames 1..F-1 the templates; every
 *   extra stage registers frames 0..F-1 to the previous stage's average (or
 *   median) with lambda = the "%f" print of lambda * extra_stages_lambda_factor.
 *   With accumulation each template is registered to the previous template
 *   (all of a stage in one batch), composed with the accumulated displacement
 *   (ConcatAndSmoothlyExtendDeformations) and, from the second template on,
 *   refined against the stage's reference on refine_start..refine_stop, one
 *   template after the other; without accumulation every template is
 *   registered to the stage's reference.
 *   frames      : num_frames images of (2^precision_level+1)^2 doubles
 *                 (input_level must equal precision_level; stop_level too)
 *   phis_out    : the last stage's displacements, m x 2 x N doubles, m =
 *                 num_frames-1 without extra stages, num_frames with them
 *   energies_out (nullable): per stage and template the energy of its last
 *                 solve (energies.txt): (num_frames-1) + extra*num_frames
 *   average_out + count_out, median_out (nullable): the last stage's average
 *                 with its sample count, and median, of the warped raw frames */
int msgpu_match_series(msgpu_context* ctx, const msgpu_params* p, const msgpu_series_params* s,
                       const double* frames, int num_frames, double* phis_out, double* energies_out,
                       double* average_out, double* median_out, double* count_out);
int msgpu_match_series_device(msgpu_context* ctx, const msgpu_params* p, const msgpu_series_params* s,
                              const double* d_frames, int num_frames, double* d_phis_out, double* d_energies_out,
                              double* d_average_out, double* d_median_out, double* d_count_out, void* stream);

/* ConcatAndSmoothlyExtendDeformations (deformations.h:498-520) as called by
 * composeDeformations(d1, d2, inout) (registration.h:584-586): the
 * displacement of (id + d1) o (id + d2); where x + d2(x) leaves the domain the
 * result is the discrete harmonic extension of SmoothlyExtendImage
 * (deformations.h:364-410, PCG to g.g < 1e-16, at most 1000 steps).
 *   d1, d2, inout: 2*N doubles [x | y]; inout holds the solver's initial
 *   guess on entry (the destination's previous content in the reference).
 *   iterations_out (nullable): PCG steps of the two components.            */
int msgpu_compose(msgpu_context* ctx, int level, const double* d1, const double* d2, double* inout,
                  int* iterations_out);
int msgpu_compose_device(msgpu_context* ctx, int level, const double* d_d1, const double* d_d2, double* d_inout,
                         void* stream);

/* Median of the warped frames over the finite samples (averageSeries,
 * matchSeries.h:442, MultiVector::getMedianVecOverComponents,
 * multiVector.cpp:99-117); pixels without samples take the last frame's mean. */
int msgpu_warp_median(msgpu_context* ctx, int level, const double* frames, const double* phis, int num_frames,
                      double* median_out);
int msgpu_warp_median_device(msgpu_context* ctx, int level, const double* d_frames, const double* d_phis,
                             int num_frames, double* d_median_out, void* stream);

/* --- on-disk arrays (host only, no context) --------------------------------
 * The reference's 2-D array files (qc::ScalarArray<QC_2D>::save / load,
 * scalarArray.cpp:330-420, 481-569; header auxiliary.h:10-45): magic P2, P5,
 * P7, P8, P9, Pa, Pb, '#' comments, "numX numY", "max", raw values x fastest;
 * compressed by file-name suffix like aol::Bzipifstream (.bz2, .q2bz, .q3bz
 * bzip2; .gz, .svgz, .zz zlib/gzip); and ".dm3" / ".dm4" Gatan
 * DigitalMicrograph images (qc::DM3Reader, dm3Import.h: the last image of the
 * ImageList).  Values are returned as doubles.
 * Errors: status code plus msgpu_io_last_error() (per host thread).          */
const char* msgpu_io_last_error(void);
/* out == NULL: only *nx, *ny are returned.  capacity: doubles at out.       */
int msgpu_read_array(const char* path, double* out, long long capacity, int* nx, int* ny);
/* type 9 (double binary, the reference's PGM_DOUBLE_BINARY) or 8 (float).  */
int msgpu_write_array(const char* path, const double* data, int nx, int ny, int type);
/* count files of nx x ny values each into out (count*nx*ny doubles), decoded
 * by `threads` host threads (< 1: one per hardware thread); every file must
 * have the given size (the frames of a series).                            */
int msgpu_read_arrays(const char* const* paths, int count, int nx, int ny, double* out, int threads);
/* The same in the background: returns at once with a task (NULL on invalid
 * arguments), whose msgpu_io_wait returns the status and frees it; out must
 * stay valid until then.  Lets the decoding of the next series overlap the
 * GPU work on the current one (no counterpart in the reference, which loads
 * each frame when its registration starts, matchSeries.h:141).            */
typedef struct msgpu_io_task msgpu_io_task;
msgpu_io_task* msgpu_read_arrays_start(const char* const* paths, int count, int nx, int ny, double* out,
                                       int threads);
int msgpu_io_wait(msgpu_io_task* task);
/* A displacement as one file per component, named by a printf mask with one
 * %d (qc::MultiArray::load / save, multiArray.h:272-306, e.g. the
 * reference's "deformation_09_%d.dat.bz2"); phi: [x | y], 2*nx*ny doubles. */
int msgpu_read_displacement(const char* mask, int nx, int ny, double* phi);
int msgpu_write_displacement(const char* mask, const double* phi, int nx, int ny);

/* Per-call statistics (no counterpart in the reference; used for the roofline).
 * With profiling on, every batch call records CUDA events around each level
 * launch on its stream and waits for them at the end of the call.          */
typedef struct {
  int kernel_launches;          /* kernels launched by the last batch call  */
  int num_levels;               /* start..stop of the last batch call       */
  int first_level;
  float level_ms[16];           /* device time of each level launch         */
  long long level_steps[16];    /* gradient steps summed over the frames    */
  long long level_evals[16];    /* energy evaluations summed over the frames */
  int level_cluster[16];        /* CTAs of the level launch (persistent grid) */
  /* clock cycles per CTA (average over the grid) spent in each pass kind of
   * the level kernel: initial energy, gradient, V-cycle down, coarse
   * V-cycle, V-cycle up, NCG + first trial, further line-search trials,
   * waiting for work and completing passes                                 */
  long long level_pass_cycles[16][8];
  int graph_replayed;           /* 1: the last device batch call replayed a
                                   captured CUDA graph (one launch)          */
  /* exact sums (sum order 0) per level: term buffers whose sums were added
   * in order, clock cycles of the binade predictions, control steps settled
   * by bounded sums (certified steps), clock cycles of the ordered walks
   * (summed over the buffers), chunks walked, chunks added term by term,
   * cycles of those term-by-term additions and cycles of the walk (both
   * summed over the walking warps)                                          */
  long long level_xs[16][8];
} msgpu_stats;
int msgpu_set_profiling(msgpu_context* ctx, int on);
/* Pass timeline of one level's launch, recorded by profiled calls
 * (msgpu_set_profiling on) that solve their levels with the level kernel:
 * msgpu_register_batch{,_device}, the stage and series entry points built
 * on it (a call with several batches keeps the last one's events) and the
 * ragged entry points. msgpu_set_trace(ctx, level, capacity)
 * records up to `capacity` events (at most 2^26) of the level kernel at
 * `level` (-1: none, the default); msgpu_get_trace copies the last profiled
 * call's events, at most `capacity`, to out (two words each) and returns
 * how many there were (-1 on invalid arguments). Word 0 is the GPU's global
 * timer in ns; word 1 packs the event in bits 56-63, the CTA in bits 32-55
 * and a value in bits 0-31: event 1 a pass published and 2 a pass completed
 * (value instance << 8 | pass kind: 0 initial energy, 1 gradient, 2 V-cycle
 * down, 3 coarse V-cycle, 4 V-cycle up, 5 NCG + first trial, 6 trial, 7
 * flush, 8-11 NCC sub-passes, 12 summaries of exact sums, 13 instance
 * finished), 3 a wait for work of 500 ns or more (value its length in ns,
 * word 0 its start), 4 an ordered walk of exact sums (value its length), 5
 * an open control step that has a term buffer's sums added in order (value
 * instance << 16 | buffer << 12 | reason << 8 | kind of the pass whose step
 * is open; reason 11: a buffer the open decision was evaluated from, else
 * 0: the pass's own sums, 1-10: a bounded value of the state, in the order
 * energy at the new position, energy, f, Df, the two line-search energies,
 * E_reg at the position, the last E_reg, the two line-search E_reg).
 * Profiling aid; no counterpart in the reference (whose only tracing is a
 * stopwatch and gprof). */
int msgpu_set_trace(msgpu_context* ctx, int level, unsigned int capacity);
long long msgpu_get_trace(const msgpu_context* ctx, unsigned long long* out, long long capacity);
/* CUDA graphs for msgpu_register_batch_device (and the stage entry points
 * built on it), default on: the second call with the same parameters and
 * buffers captures the batch's launches (per level: the level kernel, the
 * collection of the results, the prolongation; before them the image
 * preparation) into one graph, later such calls replay it as a single
 * launch.  The first call after a change of parameters or buffers runs
 * directly.  No counterpart in the reference.                             */
int msgpu_set_graphs(msgpu_context* ctx, int on);

/* The scheduling table of a context, per precision (use_fp64 0 or 1) and
 * level, and its autotuner: msgpu_autotune_device runs the batch of
 * msgpu_register_batch_device (same arguments; d_phis_scratch receives
 * num_templates * 2 * N doubles) once per candidate setting (chunk_div in
 * {12, 24, 48}, chunk_max in {8, 16, 32}, 1 or 2 CTAs per SM), times every
 * level's launch with CUDA events, and keeps for each level startLevel ..
 * stopLevel the fastest setting.  Synchronous.                            */
/* The reference-order sum of the level solve on its own (no counterpart in
 * the reference; exposed so that it can be checked on any data): *d_out =
 * the sequentially rounded 0 + t_0 + t_1 + ... of the (2^level+1)^2 doubles
 * at d_terms, in their order.  Device pointers, enqueued on `stream`.     */
int msgpu_exact_sum_device(msgpu_context* ctx, int level, const double* d_terms, double* d_out, void* stream);

int msgpu_get_tuning(const msgpu_context* ctx, int use_fp64, int level, msgpu_level_tuning* out);
int msgpu_set_tuning(msgpu_context* ctx, int use_fp64, int level, const msgpu_level_tuning* t);
int msgpu_autotune_device(msgpu_context* ctx, const msgpu_params* p, const double* d_reference,
                          const double* d_templates, int num_templates, double* d_phis_scratch, void* stream);
int msgpu_get_stats(const msgpu_context* ctx, msgpu_stats* out);

/* --- single operators of the path (parity entry points) ----------------- */
/* E = SSDEnergy + lambda * DisplacementLengthEnergy and DE = SSDForce +
 * lambda * L phi (registration.h:971-982, 1584-1667); with the NCC data term
 * (msgpu_set_data_term) NormalizedCrossCorrelationEnergy and its variation
 * (registration.h:1909-1983) instead of the SSD parts.  de_out: 2*N doubles. */
int msgpu_energy(msgpu_context* ctx, int level, const double* R, const double* T, const double* phix,
                 const double* phiy, double lambda, int use_fp64, double* energy_out, double* de_out);
/* LinearSmoothOp::apply with sigma (linearSmoothOp.cpp:591-612).          */
int msgpu_smooth(msgpu_context* ctx, int level, double sigma, int use_fp64, const double* in, double* out);
/* RestrictOp<STD_QUOC_RESTRICT>::apply, fine level -> fine level - 1.      */
int msgpu_restrict(msgpu_context* ctx, int fine_level, const double* in, double* out);
/* ProlongOp::apply, coarse level -> coarse level + 1.                      */
int msgpu_prolong(msgpu_context* ctx, int coarse_level, const double* in, double* out);
/* Image preparation (normalisation only, registration.h:335-346).         */
int msgpu_normalize(msgpu_context* ctx, const double* in, int count, double saturation_percent,
                    int normalize_min_to_zero, double* out);
/* One level solve, StandardRegistration::findTransformation
 * (registration.h:967-1021): phix/phiy are updated in place.  trace
 * (nullable) receives up to max_trace rows of (energy, tau, sigma, evals).  */
int msgpu_gd_level(msgpu_context* ctx, int level, const double* R, const double* T, double* phix,
                   double* phiy, double lambda, int max_iter, double stop_eps, int use_fp64,
                   double* energy_out, int* steps_out, double* trace, int max_trace);

/* msgpu_gd_level with the reference's per-level energy log instead of the
 * trace: energy_log receives min(steps, max_rows - 1) + 1 rows of
 * (iteration - 1, lambda * E_reg at the new position, energy at the new
 * position), the first row (-1) for the initial position -- the
 * columns the reference writes to energy_%02d.txt (gradientDescent.h:
 * 254-272, through findTransformation, registration.h:967-1000).           */
int msgpu_gd_level_log(msgpu_context* ctx, int level, const double* R, const double* T, double* phix,
                       double* phiy, double lambda, int max_iter, double stop_eps, int use_fp64, double* energy_out,
                       int* steps_out, double* energy_log, int max_rows);

/* --- allocation-free level solve ----------------------------------------
 * No counterpart in the reference.  The same level solve as msgpu_gd_level
 * with its global sums in the fixed parallel order (sum order 1; the term
 * blocks of the reference order would not fit the static array), for
 * callers that cannot allocate device memory: applications whose device
 * memory belongs to their own pool allocator (cudaMalloc/cudaFree from other
 * code would synchronise the device and fragment the pool), or hosts that
 * admit only a fixed, known device footprint.  It needs no context and
 * allocates nothing: its scratch (pitched image copies, the gradient-flow
 * arena and the multigrid pyramid) lives in one static device array of
 * 12 MiB that every GPU loading this library holds until the process exits.
 *   Limit: levels up to 8 (257^2 nodes) in FP64 or FP32; larger levels
 *   return MSGPU_ERR_SIZE without touching the device.
 *   d_R, d_T   : device, (2^level+1)^2 doubles each (prepared images)
 *   d_phi      : device, 2*(2^level+1)^2 doubles [phi_x, phi_y], updated in place
 *   d_energy_out / d_steps_out : device, one double / one int (nullable)
 *   stream     : cudaStream_t (NULL = legacy default stream); the call
 *                returns after enqueueing.
 * The first call on a device (with that device current) does a one-time
 * set-up: it looks up the device address of the scratch array and uploads
 * the finite-element tables; make that first call before any stream capture.
 * Every call on a device shares the one scratch array and leaves its
 * contents behind (each call clears what must start at zero); calls whose
 * work overlaps on the GPU (other streams, other host threads) race on it,
 * so serialise them.  The set-up is cached per device for the life of the
 * process: cudaDeviceReset on that device after the first call is not
 * supported (the cached address and the uploaded tables would be stale).
 * Errors are status codes only (no context holds a message):
 * MSGPU_ERR_INVALID_ARG, MSGPU_ERR_SIZE, MSGPU_ERR_CUDA.  Because the call
 * returns before the GPU runs, a solve whose scheduler gave up waiting (see
 * msgpu_set_wait_limits) is reported in its outputs: *d_steps_out = -1 and
 * *d_energy_out = NaN, with d_phi holding an unfinished displacement.        */
int msgpu_gd_level_noalloc(int level, const double* d_R, const double* d_T, double* d_phi, double lambda,
                           int max_iter, double stop_eps, int use_fp64, double* d_energy_out, int* d_steps_out,
                           void* stream);

/* --- learned warm start (no counterpart in the reference) -----------------
 * A U-Net on 2^l+1 node grids maps the prepared reference and template of a
 * frame pair at the network's input level l0 to a displacement at level
 * l0-1, which starts the gradient flow there instead of the coarse levels
 * startLevel..l0-1 of the plain method.  Encoder 16-32-64-128 channels
 * (3x3 convolutions, stride-2 convolutions between the node grids), decoder
 * by bilinear prolongation and [skip | upsampled] concatenation down to
 * level l0-1, ReLU, a 2-channel head; bf16 weights and activations, fp32
 * accumulation (tensor pipe), fp32 master parameters trained with Adam on
 * the mean squared difference to the plain method's displacements.
 * Parameter layout (msgpu_net_get_params): layer after layer (e0a e0b e1a
 * e1b e2a e2b e3a e3b d2a d2b d1a d1b head), W[cout][3][3][cin] then b[cout]. */
typedef struct msgpu_net msgpu_net;
long long msgpu_net_num_params(void);
/* input_level l0 in 4..11; parameters He-initialised from seed.            */
int msgpu_net_create(msgpu_context* ctx, int input_level, unsigned long long seed, msgpu_net** out);
int msgpu_net_destroy(msgpu_net* net);
int msgpu_net_input_level(const msgpu_net* net);
/* Forward convolutions on the fifth-generation tensor cores (tcgen05.mma,
 * TMEM accumulators; default 1) or on mma.sync (0).  The data-gradient and
 * weight-gradient convolutions of training use mma.sync either way; the two
 * forward paths differ only in the order of the fp32 accumulation.         */
int msgpu_net_set_tensor_cores(msgpu_net* net, int tcgen05);
int msgpu_net_get_params(msgpu_net* net, float* out);
int msgpu_net_set_params(msgpu_net* net, const float* in);   /* resets Adam */
int msgpu_net_save(msgpu_net* net, const char* path);
int msgpu_net_load(msgpu_net* net, const char* path);
/* Prediction for `batch` pairs of prepared images at level l0 (device):
 * reference image i at d_R + i * r_stride (r_stride 0: one shared
 * reference), template i at d_T + i * N0; d_phi_out: batch x 2 x N1
 * doubles ([x | y] per frame, domain units, level l0-1).                    */
int msgpu_net_predict_device(msgpu_net* net, const double* d_R, long long r_stride, const double* d_T, int batch,
                             double* d_phi_out, void* stream);
/* One Adam step on a batch against target displacements (batch x 2 x N1,
 * domain units); loss_out (host, nullable): the batch's mean squared
 * difference in pixels of level l0-1, before the step.                      */
int msgpu_net_train_step_device(msgpu_net* net, const double* d_R, long long r_stride, const double* d_T,
                                const double* d_phi_target, int batch, float lr, float* loss_out, void* stream);
/* Loss, prediction and the flat parameter gradient without an update (host
 * arrays; R and T: batch images each).                                      */
int msgpu_net_loss_grad(msgpu_net* net, const double* R, const double* T, const double* phi_target, int batch,
                        float* loss_out, double* phi_out, float* grad_out);
/* The images of the registration path prepared (prepareMultilevelArray,
 * registration.h:331-367) and restricted to `level`: count images of
 * input_level in, count images of `level` out (device).                     */
int msgpu_prepare_images_device(msgpu_context* ctx, const msgpu_params* p, const double* d_images, int count,
                                int level, double* d_out, void* stream);
/* msgpu_register_batch started from the network's prediction at level
 * l0-1 (which must lie in startLevel..stopLevel; inputLevel >= l0).  With
 * plain_energies (the plain method's final energies, nullable) the frames
 * are registered to that stated energy tolerance: the warm-started solve of
 * the stop level ends as soon as a frame's energy is within
 * rel_tol * |plain energy| of (or below) its plain energy (running up to
 * twice maxGDIterations steps to get there), and a frame that ends above
 * that is registered again from the plain start;
 * warm_used_out[f] (host, nullable) = 1 where the warm start was kept.
 * steps_out has the plain layout (stop-start+1 levels per frame; levels
 * below l0-1 count 0 for warm-started frames).                             */
int msgpu_register_batch_warm(msgpu_context* ctx, const msgpu_params* p, msgpu_net* net, const double* reference,
                              const double* templates, int num_templates, const double* plain_energies,
                              double rel_tol, double* phis_out, double* energies_out, int* steps_out,
                              int* warm_used_out);
int msgpu_register_batch_warm_device(msgpu_context* ctx, const msgpu_params* p, msgpu_net* net,
                                     const double* d_reference, const double* d_templates, int num_templates,
                                     const double* d_plain_energies, double rel_tol, double* d_phis_out,
                                     double* d_energies_out, int* d_steps_out, int* warm_used_out, void* stream);

#ifdef __cplusplus
}
#endif
#endif
