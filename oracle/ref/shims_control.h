// oracle/ref/shims_control.h -- TEST INFRASTRUCTURE (oracle harness only).
// Harness-side control of the Philox stand-in for the GSL generator.
#ifndef ORACLE_SHIMS_CONTROL_H
#define ORACLE_SHIMS_CONTROL_H
#include <stdint.h>

// every gsl_rng_uniform call draws from the generator's own seeded stream
void oracle_rng_free_running();
// calls on this thread draw (seed, pid, step, n0), (seed, pid, step, n0+1), ...
void oracle_rng_packet(uint32_t seed, uint64_t pid, uint32_t step, uint32_t n0);
uint32_t oracle_rng_packet_draws();
// calls on this thread walk packets pid_base, pid_base+1, ... taking
// `draws_per_packet` draws (counter 0 .. k-1) from each
void oracle_rng_emission(uint32_t seed, uint64_t pid_base, uint32_t step, uint32_t draws_per_packet);
uint64_t oracle_rng_emission_draws();

#endif
