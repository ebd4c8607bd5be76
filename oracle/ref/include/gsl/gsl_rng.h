/* Stand-in for the GSL random-number API used by the reference transport
 * (thread_RNG). Test infrastructure for the oracle harness: the generator is
 * Philox4x32-10, either replaying per-packet streams chosen by the harness or
 * free-running per generator seed. */
#ifndef ORACLE_SHIM_GSL_RNG_H
#define ORACLE_SHIM_GSL_RNG_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct { const char* name; } gsl_rng_type;

typedef struct gsl_rng {
  const gsl_rng_type* type;
  unsigned long seed;     /* key of the free-running stream */
  unsigned long long n;   /* draws taken from the free-running stream */
  void* state;            /* points at seed, for gsl_rng_state */
} gsl_rng;

extern const gsl_rng_type* gsl_rng_default;
extern unsigned long gsl_rng_default_seed;

const gsl_rng_type* gsl_rng_env_setup(void);
gsl_rng* gsl_rng_alloc(const gsl_rng_type* T);
void gsl_rng_free(gsl_rng* r);
void gsl_rng_set(const gsl_rng* r, unsigned long seed);
unsigned long gsl_rng_get(const gsl_rng* r);
double gsl_rng_uniform(const gsl_rng* r);
size_t gsl_rng_size(const gsl_rng* r);
void* gsl_rng_state(const gsl_rng* r);

#ifdef __cplusplus
}
#endif
#endif
