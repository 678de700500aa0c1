/* cavity_oracle.h -- TEST INFRASTRUCTURE ONLY (the oracle).
 *
 * C ABI of the CPU FP64 restatement of the reference solver
 * (bbrangeo/cfd_cavity src/uniform/solver.rs, post.rs, rng.rs).  Loaded by
 * the tests and by bench.py's CPU baseline through ctypes; never by the
 * product library.  See cavity_oracle.hpp for the parity status.
 */
#ifndef CAVITY_ORACLE_H
#define CAVITY_ORACLE_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_params {
    int32_t nx, ny;
    double ra, pr, cs, pr_t, utarget;
    uint64_t seed;
    int32_t jobs;
    double alpha_mult, nu_start_mult;
    int32_t has_nu_override;
    double nu_override;
    int32_t init_mode;   /* 0 linear theta + noise (reference), 1 theta = 0 + noise */
    double noise_amp;    /* reference: 1e-3 */
    int32_t geq_order;   /* 2 quadratic (default), 1 linear */
    const double* t_hot_profile; /* [ny] or NULL */
    double t_cold;
} orc_params;

/* Scalars of the solver: nu, alpha, alpha_phys, beta_eff, lz, lx, tau, tau_t,
 * time_step, spin_up_steps (10 doubles). */
#define ORC_INFO_LEN 10
/* Diagnostics: nusselt_hot, nusselt_cold, nusselt_hot_wall_link, total_mass,
 * total_f_mass, max_u, max_uy, nu_t_max, finite (1/0), y_plus_hot,
 * nusselt_volume (11 doubles). */
#define ORC_DIAG_LEN 11

void* orc_create(const orc_params* p, int32_t* err);
void orc_destroy(void* h);
void orc_step(void* h, int64_t n);
void orc_collide(void* h, int64_t step);
void orc_stream(void* h);
void orc_bounce_back(void* h);
void orc_thermal_bc(void* h);
void orc_macro(void* h);
void orc_noslip(void* h);
void orc_init_from_fields(void* h, const double* rho, const double* ux, const double* uy, const double* t);
void orc_get_fields(void* h, double* rho, double* ux, double* uy, double* t, double* nu_t, double* fy);
void orc_set_fields(void* h, const double* rho, const double* ux, const double* uy, const double* t,
                    const double* fy);
void orc_get_pops(void* h, double* f, double* g);
void orc_set_pops(void* h, const double* f, const double* g);
void orc_info(void* h, double* out);
void orc_diag(void* h, double* out);
void orc_set_time_step(void* h, int64_t t);

/* Dynamic mixed-scale SGS model (src/uniform/solver.rs:215-220, 562-828,
 * 1195-1261): switch, one evaluation on the current state, its statistics
 * and per-node nu_t / alpha_t (NULL to skip), the Lilly coefficient and the
 * mixed factor. */
void orc_set_dynamic_sgs(void* h, int32_t on, double smag_alpha, double nu_sm_min, double eta_test);
void orc_compute_dynamic_sgs(void* h);
void orc_dynamic_stats(void* h, double* out4, double* nu_t_pre, double* alpha_t_pre);
double orc_lilly_coefficient(double num, double den);
/* interpolate_field, src/uniform/snapshot.rs:102-131 (dst [nx1*ny1]). */
void orc_interpolate_field(const double* src, int64_t nx0, int64_t ny0, int64_t nx1, int64_t ny1, double* dst);
double orc_mixed_factor(double a, double b, double alpha);

/* Equilibria and lattice weights (crate oxiphysics_lbm, pinned by
 * src/uniform/tests.rs:116-133). */
double orc_feq(int32_t i, double rho, double ux, double uy);
double orc_geq(int32_t i, double t, double ux, double uy, int32_t order);
double orc_weight(int32_t i);
void orc_velocity(int32_t i, int32_t* cx, int32_t* cy);
/* nusselt_hot, nusselt_cold of the current state (post.rs:68-111). */
void orc_nusselt(void* h, double* hot, double* cold);

/* TimeAverager (src/uniform/post.rs:11-57). */
void* orc_avg_create(int64_t n);
void orc_avg_destroy(void* a);
void orc_avg_accumulate(void* a, void* h);
/* means: ux, uy, t, nu_t, uu; returns the sample count. */
int64_t orc_avg_means(void* a, double* ux, double* uy, double* t, double* nu_t, double* uu);
/* nusselt_from_mean, src/main.rs:740-753. */
double orc_nusselt_from_mean(void* h, const double* t_mean, int32_t hot);

/* FP64 tangent-linear oracle: J = mean of nusselt_hot over the states after
 * s steps, s in [ws, n_steps], and dJ . v for v = (dtheta[ny], dcs) in the
 * (hot-wall profile, Cs) parameters.  Returns 0 or the orc_create error. */
int orc_tl_nusselt(const orc_params* p, int64_t n_steps, int64_t ws, const double* dtheta, double dcs,
                   double* J, double* dJ);

/* Block-refined (octree) cavity, src/octree/solver.rs (molecular, or the
 * dynamic mixed-scale SGS model of src/octree/smag.rs).  levels 2 or 3; odd_exact selects the tau- ratio for the odd
 * rescaling.  *err = 1 on invalid arguments (CavitySolver::new asserts). */
void* orc_oct_create(int32_t nx0, int32_t ny0, int32_t bl_width, double ra, double pr, double utarget,
                     uint64_t seed, int32_t odd_exact, int32_t levels, double nu_start_mult, int32_t has_nu,
                     double nu, int32_t* err);
void orc_oct_destroy(void* h);
void orc_oct_step(void* h, int64_t n);
/* level 0 coarse, 1/2 hot/cold L1 blocks, 3/4 hot/cold L2 strips. */
int32_t orc_oct_level_dims(void* h, int32_t level, int32_t* nx, int32_t* ny);
int32_t orc_oct_get_level(void* h, int32_t level, double* rho, double* ux, double* uy, double* t, double* f,
                          double* g);
void orc_oct_info(void* h, double* out13);
int32_t orc_oct_restart_level(void* h, int32_t level, const double* rho, const double* ux, const double* uy,
                              const double* t);
void orc_oct_set_time_step(void* h, int64_t t);
void orc_oct_diag(void* h, double* out9);
void orc_oct_set_dynamic_sgs(void* h, int32_t on, double smag_alpha, double nu_sm_min, double eta_test);
void orc_oct_dynamic_stats(void* h, double* out14);
int32_t orc_oct_get_nut(void* h, int32_t level, double* nut, double* at);

#ifdef __cplusplus
}
#endif
#endif
