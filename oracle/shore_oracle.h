/*
 * shore_oracle.h - CPU FP64 oracle for the SHORE fit.  TEST INFRASTRUCTURE.
 *
 * A plain C++17 restatement of cs_dmri's SHORE fit path (basis, gradient
 * table, FISTA, Tikhonov, Goldfarb-Idnani ICLS, alpha strategies, volume
 * driver), used only as the checker in tests/, by __graft_entry__.smoke() and
 * as the timed CPU baseline of bench.py.  The product (libcsdshore.so) never
 * links, loads or calls it.
 *
 * The volume entry point takes the same csd_gtab / csd_shore_spec /
 * csd_fit_result structs as the product (include/csd_shore.h) so that tests
 * drive both with identical arguments.
 */
#ifndef SHORE_ORACLE_H
#define SHORE_ORACLE_H

#include "../include/csd_shore.h"

#ifdef __cplusplus
extern "C" {
#endif

/* math.rs */
double oracle_factorial(uint32_t n);
double oracle_gamma(double x);
double oracle_assoc_legendre(uint32_t l, uint32_t m, double x);
double oracle_gen_laguerre(uint32_t n, double alpha, double x);
double oracle_hyp2f1(double a, double b, double c, double z);

/* qspace.rs */
int oracle_qvals(const csd_gtab* g, double* q_out, double* big_delta, double* small_delta,
                 int32_t* delta_source);
/* shells: writes b of every shell (b0 shell first as 0.0 when present) and a
 * shell id per gradient; returns the number of shells. */
int oracle_shells(const double* bvals, int32_t n, double b0_threshold, double tolerance,
                  double* shell_b, int32_t* shell_of);
void oracle_tortoise_deltas(const double* bvals, int32_t n, double gmax, double* big_delta,
                            double* small_delta);

/* basis/shore.rs */
int oracle_n_coeffs(int32_t radial_order);
void oracle_shore_indices(int32_t radial_order, int32_t* n_out, int32_t* l_out, int32_t* m_out);
double oracle_kappa(double zeta, uint32_t n, uint32_t l);
double oracle_shore_radial(uint32_t n, uint32_t l, double q, double zeta);
void oracle_brainsuite_sh_block(uint32_t l, double theta, double phi, double* out);
int oracle_design_matrix(const csd_gtab* g, int32_t radial_order, double zeta, double* out);
void oracle_regularization(int32_t radial_order, double* n_diag, double* l_diag);

/* odf.rs */
double oracle_radial_factor(uint32_t n, uint32_t l, double zeta);
void oracle_brainsuite_to_tournier(uint32_t l, int32_t k, int32_t* idx, double* sign);
int oracle_shore_to_tournier(int32_t radial_order, double zeta, int32_t lmax, double* out);
/* Constraint sphere: 321 hemisphere directions of a 642-vertex geodesic
 * icosphere (unit vectors, row-major 3 per direction). */
int oracle_odf8_hemisphere(double* dirs_out);
void oracle_sh2amp_cart(const double* dirs, int32_t n_dirs, int32_t lmax, double* out);

/* solver/fista.rs */
double oracle_sigma_max(const double* design, int32_t m, int32_t n);
int oracle_fista_fit(const double* design, int32_t m, int32_t n, const double* signal,
                     double alpha, int32_t max_iter, double tol, int32_t non_negative,
                     const double* warm, double* coef, int32_t* iterations,
                     int32_t* converged, double* residual_l2);

/* solver/tikhonov.rs */
int oracle_tikhonov_fit(const double* design, int32_t m, int32_t n, const double* n_diag,
                        const double* l_diag, double lambda_n, double lambda_l,
                        const double* signal, double* coef, double* residual_l2);

/* solver/icls.rs */
int oracle_icls_solve(const double* h, int32_t m, int32_t n, const double* c, int32_t mc,
                      const double* b, int32_t max_iter, double tol, double epsilon,
                      double* x, int32_t* iterations, int32_t* final_active,
                      int32_t* converged, int32_t* infeasible);

/* solver/alpha.rs */
double oracle_alpha_max(const double* design, int32_t m, int32_t n, const double* signal);
int oracle_log_path(double alpha_max, int32_t n, double eps, double* out);
double oracle_bic(int32_t n_grads, double rss, int32_t k_nonzero);

/* fit.rs: whole-volume fit with `n_threads` worker threads (0 = all cores). */
int oracle_shore_fit_volume(const float* data, const uint8_t* mask, int64_t X, int64_t Y,
                            int64_t Z, const csd_gtab* gtab, const csd_shore_spec* spec,
                            csd_fit_result* out, int32_t n_threads, char* err, size_t err_len);

void oracle_default_spec(csd_shore_spec* spec);

/* synth.rs:15-84 / python/src/models.rs:252-278: signal of a coefficient
 * volume (X, Y, Z, K) f32 on a new gradient table -> (X, Y, Z, N) f32. */
int oracle_shore_predict(const float* coeffs, int64_t X, int64_t Y, int64_t Z, int32_t radial_order,
                         double zeta, const csd_gtab* target, float* out, char* err, size_t err_len);

/* python/src/models.rs:201-250 with odf.rs:79-102: Tournier-ordered ODF SH
 * coefficients (X, Y, Z, (lmax+1)(lmax+2)/2) f32; mask may be NULL. */
int oracle_shore_odf_sh(const float* coeffs, int64_t X, int64_t Y, int64_t Z, int32_t radial_order,
                        double zeta, int32_t lmax, const uint8_t* mask, float* out, char* err,
                        size_t err_len);

/* scalars/microstructure.rs + io/microstructure.rs:155-298 as exposed by
 * python/src/models.rs:283-341: six (X, Y, Z) f32 maps, zero outside the
 * mask.  units 0 = um, 1 = mm; reject != 0 applies the p99 outlier rule with
 * factor `outlier_factor`.  directions (X, Y, Z, 3) f32 may be NULL. */
int oracle_shore_microstructure(const float* coeffs, int64_t X, int64_t Y, int64_t Z,
                                int32_t radial_order, double zeta, const uint8_t* mask,
                                const float* directions, int32_t units, int32_t reject,
                                float outlier_factor, float* rtop, float* rtap, float* rtpp,
                                float* msd, float* qiv, float* ng, char* err, size_t err_len);

/* Per-voxel scalars of one FP64 coefficient vector (scalars/microstructure.rs):
 * out = {rtop, msd, qiv, ng, rtap, rtpp}; dir may be NULL (RTAP/RTPP NaN). */
void oracle_microstructure_voxel(const double* coefs, int32_t radial_order, double zeta,
                                 const double* dir, double* out);
double oracle_micro_alpha_factor(uint32_t n, uint32_t l, double zeta);

#ifdef __cplusplus
}
#endif

#endif
