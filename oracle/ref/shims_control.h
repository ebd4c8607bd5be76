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
// calls on this thread first serve `n_prefix` draws from a stream no packet
// uses, then walk packets pid_base, pid_base+1, ...; after each draw `fn`
// gets the packet (relative to pid_base) and its draws so far and returns
// the packet's number of draws once it is known (0 while it is not)
typedef uint32_t (*oracle_rng_count_fn)(void* user, uint64_t packet, const double* u, uint32_t n_drawn);
void oracle_rng_walk(uint32_t seed, uint64_t pid_base, uint32_t step, uint32_t n_prefix, oracle_rng_count_fn fn,
                     void* user);

#endif
