/* oracle/sed_oracle.h -- TEST INFRASTRUCTURE.
 *
 * CPU restatement of the reference's transport step (the oracle).  It mirrors
 * the C ABI of include/sedona_gpu.h one for one, with an `oracle_` prefix, so
 * a test can drive the oracle and the CUDA library with identical inputs.
 * Only tests, the smoke check and bench.py's cpu_baseline leg may load it; the
 * product never calls it.
 */
#ifndef SED_ORACLE_H
#define SED_ORACLE_H
#include "../include/sedona_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_ctx oracle_ctx;

int oracle_ctx_create(const sed_transport_params* params, oracle_ctx** out);
int oracle_set_grid(oracle_ctx* o, const sed_grid* grid);
int oracle_set_atomic_data(oracle_ctx* o, const sed_atomic_data* atoms);
int oracle_set_opacity_params(oracle_ctx* o, const sed_opacity_params* op);
int oracle_set_opacity(oracle_ctx* o, double dt);
int oracle_load_opacity(oracle_ctx* o, const double* abs, const double* scat,
                        const double* emis_cdf, const double* eps_imc);
/* packets [first, first+count) of the step's emission are propagated; the
 * tallies are normalised only when `finish` is set (lets tests sample) */
int oracle_transport(oracle_ctx* o, double dt, sed_step_stats* stats);
int oracle_transport_range(oracle_ctx* o, double dt, int64_t first, int64_t count, int finish,
                           sed_step_stats* stats);
int oracle_get_spectrum(oracle_ctx* o, double* flux, double* click);
int oracle_get_zone_tallies(oracle_ctx* o, double* J_nu, double* e_abs, double* e_rad,
                            double* fx, double* fy, double* fz, double* fr);
int oracle_get_opacity(oracle_ctx* o, double* abs, double* scat, double* emis_cdf,
                       double* n_elec, double* eps_imc, double* planck_mean,
                       double* rosseland_mean, double* L_thermal);
int oracle_record_packets(oracle_ctx* o, int32_t enable);
int oracle_get_packet_records(oracle_ctx* o, int64_t n, int32_t* fate, int32_t* ind,
                              int32_t* draws, double* state9);
/* line bins computed at set_atomic_data (locate_within_bounds of each line) */
int oracle_get_fuzz_bins(oracle_ctx* o, int32_t* bins);
/* locate_array::locate / locate_within_bounds on an arbitrary grid (for tests) */
int oracle_locate(const sed_locate_grid* g, double x);
/* common random numbers and the differentiable transport (weighted forward,
 * its exact Jacobian accumulated forward-mode per packet, and the VJP) */
int oracle_set_rng_step(oracle_ctx* o, uint32_t step);
int oracle_diff_forward(oracle_ctx* o, double dt, const double* abs_scale, int32_t n_bands, sed_step_stats* stats);
int oracle_diff_vjp(oracle_ctx* o, const double* grad_flux, double* grad_scale, sed_step_stats* stats);
int oracle_diff_vjp_density(oracle_ctx* o, const double* grad_flux, double* grad_rho, sed_step_stats* st);
int oracle_diff_jacobian(oracle_ctx* o, double* jac, sed_step_stats* stats);
int oracle_diff_scale_extinction(oracle_ctx* o, const double* rho_scale);
/* packets carried between time-dependent steps, the transport clock, and
 * the initial radiation field's packets */
int64_t oracle_n_particles(oracle_ctx* o);
int oracle_wipe_spectra(oracle_ctx* o);
int oracle_set_core_source(oracle_ctx* o, double luminosity, const double* weights);
int oracle_get_particles(oracle_ctx* o, int64_t n, int32_t* ind, int32_t* type, double* state9);
int oracle_set_time(oracle_ctx* o, double t_now);
double oracle_get_time(oracle_ctx* o);
int oracle_initialize_particles(oracle_ctx* o, int64_t n, const double* e_rad);
/* packet counts of the next steps */
int oracle_set_emission(oracle_ctx* o, double core_n_emit, int64_t n_emit_radioactive);
/* radioactive source results of the last step */
int oracle_get_gamma_spectrum(oracle_ctx* o, double* flux, double* click);
int oracle_get_radioactive_tallies(oracle_ctx* o, double* L_radio_emit, double* L_radio_dep);
/* radiative-equilibrium temperature solve after a transport step */
int oracle_solve_temperature(oracle_ctx* o, int32_t set_Tgas_to_Trad, double* T_gas, int32_t* n_unsolved);
const char* oracle_last_error(oracle_ctx* o);
/* Philox4x32-10 block and the packet-stream uniform (oracle/philox.h) */
void oracle_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
double oracle_uniform(uint32_t seed, uint64_t pid, uint32_t step, uint32_t n);
void oracle_ctx_destroy(oracle_ctx* o);

#ifdef __cplusplus
}
#endif
#endif
