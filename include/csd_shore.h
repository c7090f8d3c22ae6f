/*
 * csd_shore.h - C ABI of the B200 3D-SHORE volume fit (libcsdshore.so).
 *
 * This is the drop-in boundary for cs_dmri's masked-voxel SHORE fit.  The
 * reference binds the same operation three ways:
 *
 *   Rust library : fit_shore(&DwiData, &ShoreFitSpec, on_voxel)
 *                  -> Result<ShoreFitOutput>            (src/fit.rs:687)
 *   PyO3         : _cs_dmri.shore_fit(data, bvals, bvecs, mask, **kw)
 *                                                       (python/src/models.rs:70-198)
 *   per voxel    : trait Solver { fn fit(&Problem) }    (src/solver/mod.rs:49-51)
 *
 * A per-voxel call is far too fine for a GPU, so the boundary sits at the
 * volume level (fit_shore / fit_volume_*), and every entry point below
 * replaces one of the reference's volume-level interfaces.  All buffers are
 * owned by the caller; the handle owns device memory, streams and the
 * per-gradient-table setup cache.  Nothing here takes or returns a torch type.
 *
 * Layouts follow the reference exactly (src/io/dwi.rs:22-40, src/fit.rs:89):
 *   data          float32 (X, Y, Z, N), C order: a voxel's N samples contiguous
 *   mask          uint8   (X, Y, Z), non-zero = fit this voxel
 *   coefficients  float32 (X, Y, Z, K), C order, zeros outside the mask
 *   diagnostic maps (X, Y, Z) float32 / uint32 / uint8
 * Coefficient order is the BrainSuite SHORE order (n, l even <= n, m)
 * (src/basis/shore.rs:29-44): K = 72 at radial order 6, 145 at order 8.
 *
 * Status codes mirror CsDmriError (src/lib.rs:62-81):
 *   0 ok, 1 invalid argument / dimension mismatch (CsDmriError::Dimension,
 *   ::Other), 2 fit refused (CsDmriError::Fit, shell guard src/fit.rs:691-717),
 *   3 numerical (a normal matrix that is not positive definite; the reference
 *   panics at src/solver/tikhonov.rs:44), 4 CUDA error, 5 timeout (a bounded
 *   device wait gave up).  A message is written to `err` (NUL-terminated,
 *   truncated to err_len).  Per-voxel non-convergence is not an error: it is
 *   reported through the iterations map and the converged flags.
 */
#ifndef CSD_SHORE_H
#define CSD_SHORE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CSD_ABI_VERSION 1

enum csd_status {
  CSD_OK = 0,
  CSD_ERR_INVALID = 1,
  CSD_ERR_FIT_REFUSED = 2,
  CSD_ERR_NUMERICAL = 3,
  CSD_ERR_CUDA = 4,
  CSD_ERR_TIMEOUT = 5
};

/* ShoreRegularization (src/fit.rs:595-610); values match the reference's
 * regularization_kind map (1 = L1, 2 = L2, 3 = amplitude ICLS). */
enum csd_regularization {
  CSD_REG_L1 = 1,
  CSD_REG_L2 = 2,
  CSD_REG_NONNEG = 3
};

/* AlphaMode (src/fit.rs:545-550). */
enum csd_alpha_mode {
  CSD_ALPHA_FIXED = 0,
  CSD_ALPHA_RATIO = 1,
  CSD_ALPHA_PATH_BIC = 2,
  CSD_ALPHA_L2_ANCHORED = 3
};

/* Arithmetic of the FISTA iterations.  FP64 is the reference-faithful path:
 * the same iteration, step 1/L and stopping rule as src/solver/fista.rs:70-143
 * evaluated in IEEE double.  MIXED (radial order 6 only; L2 and nonneg fits
 * ignore it) keeps the iterates, the stopping rule and the gradient
 * accumulator in FP64 and forms the per-iteration Gram product G (x_k -
 * x_{k-1}) exactly from int8 digit slices on the tensor cores, accurate to
 * about 2^-32 relative; voxels whose stopping decision falls within 1 % of
 * tol are re-fitted in FP64. */
enum csd_precision {
  CSD_PRECISION_FP64 = 0,
  CSD_PRECISION_MIXED = 1,
  /* The two converged-optimum modes (fixed alpha or alpha ratio, radial
   * order <= 6) return the LASSO minimiser of (1/(2n)) ||M c - s||^2 +
   * alpha ||c||_1 itself, certified per voxel by its KKT conditions (the
   * witness of the reference's tests/common/mod.rs:127-153), instead of the
   * iterate the reference's stopping rule leaves (fista.rs:120-127), which
   * sits a relative 1e-5 .. 1e-2 from it.  A fixed number of FISTA
   * iterations (chosen per table by a timed autotuning batch among 16, 24, 32 and 48,
   * or fixed with csd_set_option CSD_OPT_KKT_ITERATIONS) finds
   * the support; an FP64 active-set polish (Lawson-Hanson style, with signs
   * in place of non-negativity) solves G_SS c_S = b_S - n alpha sign(c_S) on
   * it, moving coefficients in and out until no sign disagrees and every
   * off-support |M_j^T (M c - s)| / n <= alpha (1 + 1e-9); voxels it has not
   * certified within its round limit are fitted by the FP64 FISTA path with
   * the reference stopping rule and polished again.  The iterations map counts the FISTA
   * iterations plus the polish rounds, and the converged flag is the
   * certificate.  MIXED_KKT runs the iterations in TF32 on the tensor cores
   * (FP32 accumulation); FP64_KKT runs them in FP64, as a reference for it. */
  CSD_PRECISION_MIXED_KKT = 2,
  CSD_PRECISION_FP64_KKT = 3
};

/* Gradient table (src/qspace.rs:90-130).  big_delta / small_delta in seconds;
 * pass NaN for either to use the TORTOISE estimate at gmax 0.08 T/m
 * (src/qspace.rs:213-227), as the Python binding does (python/src/lib.rs:89). */
typedef struct csd_gtab {
  const double* bvals;      /* N */
  const double* bvecs;      /* N x 3, row-major */
  int32_t n;
  double big_delta;
  double small_delta;
  double b0_threshold;      /* default 50 s/mm^2 */
} csd_gtab;

/* ShoreFitSpec (src/fit.rs:634-669) flattened, with the kwargs of
 * _cs_dmri.shore_fit (python/src/models.rs:70-76).  csd_default_spec() fills
 * the reference defaults. */
typedef struct csd_shore_spec {
  int32_t radial_order;     /* positive, even (models.rs:142-144); default 6 */
  double zeta;              /* default 700 */
  int32_t regularization;   /* csd_regularization; default L1 */
  int32_t alpha_mode;       /* csd_alpha_mode; default L2_ANCHORED */
  double alpha;             /* Fixed alpha and FISTA seed alpha; default 1.0 */
  double alpha_ratio;       /* default 1e-3 */
  int32_t path_n_alphas;    /* default 20 */
  double path_eps;          /* <= 0: mode default (1e-3 path-bic, 1e-4 l2-anchored) */
  double slack;             /* default 0.05 */
  int32_t max_iter;         /* FISTA, default 1000 */
  double tol;               /* FISTA, default 1e-6 */
  int32_t non_negative;     /* FISTA coefficient projection, default 0 */
  double lambda_n;          /* Tikhonov radial weight, default 1e-8 */
  double lambda_l;          /* Tikhonov angular weight, default 1e-8 */
  int32_t nonneg_max_iter;  /* ICLS, default 200 */
  double nonneg_tol;        /* ICLS, default 1e-9 */
  double nonneg_epsilon;    /* ICLS, default 1e-10 */
  int32_t diagnostics;      /* fill the diagnostic maps; default 0 */
  int32_t allow_single_shell; /* default 0 */
  int32_t precision;        /* csd_precision; default FP64 */
} csd_shore_spec;

/* Outputs of one volume fit: ShoreFitOutput (src/fit.rs:672-683) plus the
 * diagnostics maps of VolumeDiagnostics (src/fit.rs:31-43).  Pointers are
 * caller-owned; the optional ones may be NULL.  The maps are written only when
 * spec.diagnostics is set; alpha/bic are written for L1 and rss_l2 for the
 * L2-anchored strategy, exactly where the reference returns Some(..). */
typedef struct csd_fit_result {
  /* required */
  float* coefficients;          /* X*Y*Z*K */
  /* optional maps (X*Y*Z) */
  float* r2;
  float* residual_l2;
  uint32_t* iterations;
  uint8_t* regularization_kind;
  float* alpha;
  float* bic;
  float* rss_l2;
  /* optional: FP64 coefficients of the masked voxels, V x K, in the
   * canonical x-y-z mask order (src/voxel_loop.rs:28-42), for parity checks */
  double* coef64;
  /* optional: per masked voxel 1 = converged (V entries, mask order) */
  uint8_t* converged;

  /* scalar results, written by the call */
  int32_t n_coeffs;
  int64_t n_voxels;
  int32_t has_alpha_distribution;
  double alpha_distribution[3]; /* median, p10, p90 (src/fit.rs:334-352) */
  double representative_alpha;
  double big_delta_seconds;
  double small_delta_seconds;
  double tau_seconds;
  int32_t delta_source;         /* 0 user supplied, 1 TORTOISE estimate */
  int32_t n_shells;
  double dwi_shells[32];        /* mean b of the non-zero shells, ascending */
  int32_t lmax;                 /* amplitude-ICLS constraint order */
  int32_t n_constraint_dirs;    /* amplitude-ICLS sphere size */
  uint64_t total_iterations;    /* sum of solver iterations over the mask */
  char warnings[2048];          /* '\n'-separated, as ShoreFitOutput::warnings */
} csd_fit_result;

/* Opaque handle: device memory, streams, cached per-table setup. */
typedef struct csd_handle csd_handle;

/* Library / ABI identification. */
const char* csd_version(void);
int csd_abi_version(void);

/* Fill `spec` with ShoreFitSpec::default() and the PyO3 kwarg defaults
 * (src/fit.rs:647-669, python/src/models.rs:70-76). */
void csd_default_spec(csd_shore_spec* spec);

/* Number of SHORE coefficients at `radial_order` (ShoreBasis::new,
 * src/basis/shore.rs:29-44). */
int csd_shore_n_coeffs(int32_t radial_order);

/* Create / destroy a handle bound to CUDA device `device`. */
int csd_create(csd_handle** out, int32_t device, char* err, size_t err_len);
void csd_destroy(csd_handle* h);

/* Whole-volume fit from HOST buffers (replaces fit_shore, src/fit.rs:687, and
 * _cs_dmri.shore_fit, python/src/models.rs:77).  Host-to-device copies of the
 * data and the device-to-host copies of every output happen inside the call.
 * Blocking. */
int csd_shore_fit_volume(csd_handle* h, const float* data, const uint8_t* mask,
                         int64_t X, int64_t Y, int64_t Z, const csd_gtab* gtab,
                         const csd_shore_spec* spec, csd_fit_result* out,
                         char* err, size_t err_len);

/* Same fit, with `data`, `mask` and every output pointer of `out` in DEVICE
 * memory of the handle's device (e.g. torch tensors' data_ptr()).  Work is
 * queued on `stream` (a cudaStream_t; NULL = the handle's stream); the call
 * returns after the stream has finished, so outputs are ready on return.
 * Replaces the same interface as csd_shore_fit_volume. */
int csd_shore_fit_volume_device(csd_handle* h, const float* d_data, const uint8_t* d_mask,
                                int64_t X, int64_t Y, int64_t Z, const csd_gtab* gtab,
                                const csd_shore_spec* spec, csd_fit_result* out,
                                void* stream, char* err, size_t err_len);

/* Design matrix M (N x K, row-major, FP64) of the SHORE basis for `gtab`,
 * built on the device (replaces ShoreBasis::design_matrix,
 * src/basis/shore.rs:122-178).  `out` is a host buffer of N*K doubles. */
int csd_shore_design_matrix(csd_handle* h, const csd_gtab* gtab, int32_t radial_order,
                            double zeta, double* out, char* err, size_t err_len);

/* Per-handle counters of the last fit, for measurement: kernel-only device
 * time of each stage in milliseconds (CUDA events on the fit stream) and the
 * number of kernel launches the fit issued. */
typedef struct csd_fit_timing {
  float ms_setup;       /* design, Gram, factorizations, Lipschitz */
  float ms_rhs;         /* A^T s over the mask */
  float ms_solve;       /* FISTA / Tikhonov / ICLS iterations */
  float ms_epilogue;    /* residual, R^2, scatter */
  float ms_total;       /* device time from first to last kernel */
  int32_t launches;     /* kernels launched by the fit */
  float ms_solve_kernel;/* duration of the dominant solve kernel alone */
  double tensor_flops;  /* FP64 tensor-core FLOPs the FISTA launches executed */
  float ms_mixed_kernel;/* the mixed-precision FISTA kernel alone (0 in FP64) */
  double int8_tensor_ops;      /* int8 tensor-core ops it issued (2 per MAC) */
  uint64_t fp64_rerun_voxels;  /* voxels the stop-decision guard re-ran in FP64 */
  int32_t fista_warps;         /* FISTA kernel warps per CTA the autotuner chose for the table (0: none) */
  float fista_tune_ms12;       /* the autotuning batch's time with 12 warps per CTA */
  float fista_tune_ms16;       /* ... and with 16 */
  int64_t fista_parked;        /* voxels the two-pass FISTA schedule stopped at the cap and resumed,
                                  slowest-first, in its second pass (0: single pass) */
  /* converged-optimum modes (zero otherwise) */
  float ms_kkt_iterate;        /* support identification: the TF32 tensor-core (or FP64) FISTA iterations */
  float ms_kkt_polish;         /* first FP64 polish and certificate */
  float ms_kkt_fallback;       /* FP64 FISTA of the voxels it left uncertified and their last polish */
  int64_t kkt_fallback_voxels; /* voxels the first polish did not certify (fitted again in FP64) */
  int64_t kkt_uncertified;     /* voxels left without a certificate */
  uint64_t kkt_rounds;         /* polish rounds, summed over voxels and passes */
  double tf32_tensor_flops;    /* TF32 tensor-core FLOPs issued (2 per multiply-add) */
  double kkt_max;              /* largest KKT residual of a certified voxel */
  /* host buffers of csd_shore_fit_volume (host clock; zero when unused) */
  float ms_host_gather;        /* pageable input: masked rows gathered into page-locked staging (the
                                  pipelined fit gathers chunk by chunk, overlapped with the device) */
  float ms_host_copy_out;      /* pageable output: the page-locked output volume copied out */
  int32_t kkt_iterations;      /* converged-optimum modes: support-identification iterations used */
  float kkt_tune_ms[4];        /* the autotuner's batch times with 16, 24, 32 and 48 of them */
  int64_t kkt_overflow;        /* voxels whose support outgrew the first polish pass (32 coefficients) */
} csd_fit_timing;

int csd_last_timing(const csd_handle* h, csd_fit_timing* out);

/* Tuning options of a handle (they never change a result's meaning):
 *   CSD_OPT_FISTA_SHAPE     FP64 FISTA kernel: 0 = the per-table autotuned
 *                           choice (default), 12 or 16 warps per CTA of the
 *                           DMMA kernel, 1 = the register kernel; every
 *                           shape computes the same iterates
 *   CSD_OPT_FISTA_SCHEDULE  0 = single-pass FISTA; 1 = the two-pass
 *                           schedule where it applies (default); a value
 *                           >= 2 also sets its cap (iteration of the first
 *                           pass' end, default 80)
 *   CSD_OPT_KKT_ITERATIONS  FISTA iterations of the converged-optimum
 *                           modes' support identification (1 .. 100000;
 *                           0, the default, = the autotuner's choice per
 *                           gradient table among 16, 24, 32 and 48)
 *   CSD_OPT_KKT_ROUNDS      solves the first polish of the converged-optimum
 *                           modes may take per voxel before the voxel goes
 *                           to the FP64 FISTA fallback (1 .. 4096, default 48)
 *   CSD_OPT_TENSOR_WAIT_NS  how long a tensor-core kernel (MIXED, MIXED_KKT)
 *                           waits for one batch of its products before it
 *                           gives up, lets the products in flight land (a
 *                           separate 2 s bound), frees its tensor memory and
 *                           makes the call return CSD_ERR_TIMEOUT
 *                           (1 .. 2e9 ns, default 2e9); a tiny value makes
 *                           that failure path testable
 *   CSD_OPT_ICLS            amplitude-positivity QP kernel: 0 = the Gram
 *                           form (constraint values carried through
 *                           Gamma = W^T W; radial orders <= 6, the default),
 *                           1 = the orthogonal-basis form (any order); both
 *                           follow the reference's iteration path
 * Returns CSD_ERR_INVALID for an unknown option or value. */
enum csd_option {
  CSD_OPT_FISTA_SHAPE = 1,
  CSD_OPT_FISTA_SCHEDULE = 2,
  CSD_OPT_KKT_ITERATIONS = 3,
  CSD_OPT_TENSOR_WAIT_NS = 4,
  CSD_OPT_KKT_ROUNDS = 5,
  CSD_OPT_ICLS = 6
};
int csd_set_option(csd_handle* h, int32_t option, int64_t value);

/* ---- post-fit maps over a coefficient volume (X, Y, Z, K) f32, C order;
 * host buffers in and out; the radial order fixes K. */

/* Signal predicted by the coefficients on a new gradient table,
 * (X, Y, Z, target->n) f32; voxels whose coefficients are all zero are
 * written as zeros.  Replaces synthesize_volume (src/synth.rs:15-84) and
 * _cs_dmri.shore_predict (python/src/models.rs:252-278). */
int csd_shore_predict(csd_handle* h, const float* coefficients, int64_t X, int64_t Y, int64_t Z,
                      int32_t radial_order, double zeta, const csd_gtab* target, float* signal_out,
                      char* err, size_t err_len);

/* Tournier-ordered ODF SH coefficients, (X, Y, Z, (lmax+1)(lmax+2)/2) f32,
 * zeros outside `mask` (NULL = every voxel); lmax even and <= radial_order.
 * Replaces _cs_dmri.shore_odf_sh (python/src/models.rs:201-250) with the
 * projection of src/odf.rs:79-102. */
int csd_shore_odf_sh(csd_handle* h, const float* coefficients, int64_t X, int64_t Y, int64_t Z,
                     int32_t radial_order, double zeta, int32_t lmax, const uint8_t* mask,
                     float* sh_out, char* err, size_t err_len);

/* RTOP, RTAP, RTPP, MSD, QIV and NG maps, each (X, Y, Z) f32, zero outside
 * `mask`.  `directions` (X, Y, Z, 3) f32 may be NULL (RTAP / RTPP NaN);
 * units 0 = micrometre (the reference default), 1 = millimetre; with
 * `reject_outliers` a scalar above outlier_factor x its p99 is NaN.
 * Replaces _cs_dmri.shore_microstructure (python/src/models.rs:283-341) and
 * compute_microstructure (src/io/microstructure.rs:155-298). */
int csd_shore_microstructure(csd_handle* h, const float* coefficients, int64_t X, int64_t Y, int64_t Z,
                             int32_t radial_order, double zeta, const uint8_t* mask,
                             const float* directions, int32_t units, int32_t reject_outliers,
                             float outlier_factor, float* rtop, float* rtap, float* rtpp, float* msd,
                             float* qiv, float* ng, char* err, size_t err_len);

/* GFA and ODF peaks of every masked voxel (NULL mask = every voxel): the
 * quantities the reference's SHORE ODX export computes
 * (src/io/odx_out.rs:1008-1090; defaults there: npeaks 5, relative
 * threshold 0.5, separation 25 degrees).  The ODF is sampled on the
 * hemisphere of the class I geodesic sphere of `sphere_frequency` (1..10;
 * 181 directions at 6) - the reference samples DSI Studio's ODF8
 * hemisphere, not available here - with amplitudes clipped at 0.  GFA per
 * odx_out.rs:1036-1050; peaks are mesh local maxima in decreasing amplitude,
 * stopping below relative_peak_threshold x the largest, skipping any within
 * min_separation_angle_deg of a kept one, up to npeaks (1..8).  Outputs
 * (host, f32): gfa (X, Y, Z); peak_dirs (X, Y, Z, npeaks, 3) unit vectors in
 * the fit frame; peak_values / peak_qa (X, Y, Z, npeaks), the amplitude and
 * the amplitude above the voxel's smallest sampled one; zeros past the peaks
 * found and outside the mask. */
int csd_shore_odf_peaks(csd_handle* h, const float* coefficients, int64_t X, int64_t Y, int64_t Z,
                        int32_t radial_order, double zeta, const uint8_t* mask, int32_t sphere_frequency,
                        int32_t npeaks, double relative_peak_threshold, double min_separation_angle_deg,
                        float* gfa, float* peak_dirs, float* peak_values, float* peak_qa, char* err,
                        size_t err_len);

/* ---- differentiable fit.  No counterpart in the reference, which computes
 * no derivatives: these entry points differentiate the solution maps of its
 * solvers (LASSO, src/solver/fista.rs:70-143; Tikhonov,
 * src/solver/tikhonov.rs:26-76) and of the maps taken on coefficients.  All
 * arrays are DEVICE memory of the handle's device, row-major.  Work is
 * queued on `stream` (NULL = the legacy default stream) and the calls return
 * once it is queued, without waiting for it (a call that builds a new
 * gradient table's setup waits for that setup): results are ready when the
 * stream reaches them.  Calls on one handle share its scratch buffers, so they must
 * be ordered on one stream. */

/* Fit of a batch of voxel signals, float32 (n_voxels, N): regularization L1
 * with alpha_mode FIXED (spec->alpha, or one alpha per voxel in `d_alpha`,
 * nullable) and an optional warm start `d_warm` (n_voxels, K), or L2.
 * FP64 coefficients (n_voxels, K) out; `d_iterations` (n_voxels) nullable.
 * `d_order` (nullable) is a permutation of 0 .. n_voxels-1: the order in which
 * the persistent FISTA kernel takes the voxels up.  Putting the voxels that
 * need the most iterations first (known, for instance, from the previous fit
 * of the same batch) keeps them from starting late and finishing alone; the
 * results do not depend on the order.  The per-voxel arithmetic is that of
 * csd_shore_fit_volume. */
int csd_shore_fit_batch_device(csd_handle* h, const float* d_signals, int64_t n_voxels,
                               const csd_gtab* gtab, const csd_shore_spec* spec,
                               const double* d_alpha, const double* d_warm, const int64_t* d_order,
                               double* d_coef, uint32_t* d_iterations, void* stream, char* err,
                               size_t err_len);

/* Adjoint of that fit at the coefficients `d_coef` (n_voxels, K) for the
 * upstream gradient `d_grad_coef` (n_voxels, K).  L1: implicit derivative on
 * the support of each voxel's coefficients, w_S = G_SS^-1 g_S with
 * G = M^T M; L2: w = H^-1 g with H the normal matrix.  Outputs (each
 * nullable): the gradient on the signals M w as float32 and / or float64
 * (n_voxels, N), and per voxel (n_voxels, 2) the gradient on the
 * hyper-parameters: L1 (d/dalpha, 0) with d/dalpha = -N sign(c_S) . w_S, L2
 * (d/dlambda_n, d/dlambda_l).  A voxel whose support matrix is not positive
 * definite gets NaN gradients and is added to the device counter
 * `d_n_singular` (nullable). */
int csd_shore_fit_adjoint_device(csd_handle* h, const csd_gtab* gtab, const csd_shore_spec* spec,
                                 const double* d_coef, const double* d_grad_coef, int64_t n_voxels,
                                 float* d_grad_signal, double* d_grad_signal64, double* d_grad_hyper,
                                 uint64_t* d_n_singular, void* stream, char* err, size_t err_len);

/* out[v][r] = sum_k A[r][k] in[v][k] for a fixed matrix A given TRANSPOSED,
 * `d_At` (cols, rows): in (n_voxels, cols), out (n_voxels, rows), FP64.
 * With A an ODF matrix (below) this samples ODFs; with the design matrix of
 * a target table it predicts signals (src/synth.rs:15-84); with A^T (pass A
 * itself as d_At) it is the adjoint of either. */
int csd_apply_rows_device(csd_handle* h, const double* d_At, int32_t rows, int32_t cols,
                          const double* d_in, int64_t n_voxels, double* d_out, void* stream,
                          char* err, size_t err_len);

/* ODF amplitudes on `n_dirs` directions (n_dirs x 3, host) per SHORE
 * coefficient: (n_dirs, K) host FP64 = sh2amp(dirs, radial_order) x the
 * SHORE-to-Tournier projection (src/odf.rs:79-102), the SH values rounded to
 * float32 as the reference's sh2amp table is. */
int csd_shore_odf_matrix(csd_handle* h, int32_t radial_order, double zeta, const double* dirs,
                         int32_t n_dirs, double* out, char* err, size_t err_len);

/* RTOP (src/scalars/microstructure.rs:98-118) of FP64 coefficients
 * (n_voxels, K) -> (n_voxels), and its adjoint: the gradient on the
 * coefficients (n_voxels, K) for an upstream gradient (n_voxels). */
int csd_shore_rtop_device(csd_handle* h, int32_t radial_order, double zeta, const double* d_coef,
                          int64_t n_voxels, double* d_rtop, void* stream, char* err, size_t err_len);
int csd_shore_rtop_adjoint_device(csd_handle* h, int32_t radial_order, double zeta,
                                  const double* d_coef, int64_t n_voxels, const double* d_grad_rtop,
                                  double* d_grad_coef, void* stream, char* err, size_t err_len);

/* L1 fit (alpha_mode FIXED; one alpha per voxel in `d_alpha`, nullable) of
 * a batch of voxel signals, float32 (n_voxels, N), each on its OWN design:
 * the effective table of its gradient-deviation tensor (`d_graddev`,
 * (n_voxels, 9) row-major T, nullable = identity; src/graddev.rs:160-185:
 * q = T^T g, b_eff = b |q|^2, dir = q / |q|) restricted to the samples it
 * keeps (`d_keep`, (n_voxels, N) non-zero = keep, nullable = all).  The
 * reference computes that table but fits SHORE with one shared design.  Per
 * voxel: G_v = M_v^T M_v, L_v = sigma_max(M_v)^2 / n_v and the FISTA of
 * src/solver/fista.rs:70-143.  Radial orders 6 and 8.  Outputs (device):
 * coefficients (n_voxels, K) FP64, iterations, converged, and (nullable) L_v
 * and the kept sample count.  Asynchronous like the entry points above.
 * With precision FP64_KKT or MIXED_KKT each voxel's fit is its certified
 * LASSO optimum (as for csd_shore_fit_volume; support-identification
 * iterations on the voxel's own Gram matrix, then one warp polishes and
 * certifies): converged = certified, and the call waits for its work and
 * reports the uncertified count and the polish rounds through
 * csd_last_timing.  That mode's support iterations step by 1 / (1.12 L)
 * from a 10-step Lanczos estimate of L_v (the value reported in
 * d_lipschitz); a voxel left uncertified runs the full 40-step estimate and
 * the reference FISTA.  FP64_KKT runs everything in FP64.  MIXED_KKT keeps
 * G_v as two FP32 parts hi = fl32(G), lo = fl32(G - hi) (48 bits of G in
 * the space of the FP64 matrix) and runs the Lanczos estimate and the
 * support iterations in FP32 on hi; the polish, the certificate and any
 * uncertified voxel's FISTA run in FP64 on hi + lo. */
int csd_shore_fit_graddev_device(csd_handle* h, const float* d_signals, int64_t n_voxels,
                                 const csd_gtab* gtab, const csd_shore_spec* spec,
                                 const double* d_graddev, const uint8_t* d_keep,
                                 const double* d_alpha, double* d_coef, uint32_t* d_iterations,
                                 uint8_t* d_converged, double* d_lipschitz, int32_t* d_n_rows,
                                 void* stream, char* err, size_t err_len);

/* Class I geodesic sphere of `frequency` (10 f^2 + 2 vertices; 362 at f = 6),
 * or one vertex per antipodal pair with `hemisphere`.  Writes the unit
 * vectors (count x 3) to `out` when `capacity` >= count; returns the count,
 * -1 for a frequency outside 1..64. */
int csd_geodesic_sphere(int32_t frequency, int32_t hemisphere, double* out, int32_t capacity);

/* Allocation-free fixed-alpha FISTA fit of a batch of voxels.
 *
 * No counterpart in the reference: it exists for callers that cannot let a
 * library call cudaMalloc - applications whose device memory is owned by
 * their own pool allocator (a framework's caching allocator, a server with a
 * fixed memory budget) and latency-critical pipelines that cannot afford the
 * device-wide synchronisation of cudaFree or an allocation failure mid-run.
 * It allocates nothing: all scratch lives in one static device array of about
 * 10.3 MB that the library reserves on every GPU that loads it, until exit.
 *
 * Inputs and outputs are caller-owned DEVICE memory on the current device:
 * `d_signals` float32 (n_voxels, N) row-major, `d_coeffs` float32
 * (n_voxels, K), `d_iterations` uint32 (n_voxels) or NULL.  `spec` must ask
 * for L1 with a fixed alpha and precision FP64 (anything else returns
 * CSD_ERR_INVALID); the result is the same as csd_shore_fit_volume's FP64
 * fit for those voxels.  Limits: n_voxels <= 8192, N <= 1024, radial order
 * <= 6; larger requests return CSD_ERR_INVALID with a message.  The first
 * call on a device looks up the array's device address
 * (cudaGetSymbolAddress) with that device current and keeps it for the life
 * of the process; make that first call before any stream capture, and do not
 * call this entry point after the process has reset the device
 * (cudaDeviceReset unloads the array).  All calls share the one array and it
 * keeps the last call's contents (each call rebuilds what it reads and
 * zeroes its work counter): calls that overlap on the GPU race.  Work is
 * queued on `stream` (a cudaStream_t, NULL = the legacy default stream); the
 * call copies the Lipschitz constant of the table to the host and waits for
 * `stream` to finish before it returns. */
int csd_shore_fista_batch_noalloc(const csd_gtab* gtab, const csd_shore_spec* spec,
                                  const float* d_signals, int64_t n_voxels, float* d_coeffs,
                                  uint32_t* d_iterations, void* stream, char* err,
                                  size_t err_len);

#ifdef __cplusplus
}
#endif

#endif /* CSD_SHORE_H */
