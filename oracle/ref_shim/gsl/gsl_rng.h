/* Stand-in for the GSL generator API that SAMoS's RNG class calls
 * (src/utils/rng.cpp:34-69).  A generator is (seed, counter): draw number c
 * of stream `seed` is the project's counter-based noise (Philox-4x32-10 +
 * Box-Muller, defined in oracle/samos_oracle.c and on the GPU), so the
 * reference's own integrators consume exactly the stream the oracle and the
 * CUDA path consume, one counter value per gsl_rng_uniform /
 * gsl_ran_gaussian call.  Test infrastructure for the reference-source
 * oracle build. */
#ifndef SHIM_GSL_RNG_H
#define SHIM_GSL_RNG_H
#include <stdint.h>
#include <stdlib.h>

#ifdef __cplusplus
extern "C" {
#endif

double or_noise_gauss(uint32_t seed, uint64_t counter);
double or_noise_uniform(uint32_t seed, uint64_t counter);

typedef struct { const char* name; } gsl_rng_type;
typedef struct { uint32_t seed; uint64_t counter; } gsl_rng;

static const gsl_rng_type shim_counter_stream = { "counter-philox" };
static const gsl_rng_type* gsl_rng_default = &shim_counter_stream;

static inline const gsl_rng_type* gsl_rng_env_setup(void) { return gsl_rng_default; }
static inline gsl_rng* gsl_rng_alloc(const gsl_rng_type* t)
{
  (void)t;
  gsl_rng* r = (gsl_rng*)calloc(1, sizeof(gsl_rng));
  return r;
}
static inline void gsl_rng_set(gsl_rng* r, unsigned long seed)
{
  r->seed = (uint32_t)seed;
  r->counter = 0;
}
static inline void gsl_rng_free(gsl_rng* r) { free(r); }
static inline double gsl_rng_uniform(gsl_rng* r) { return or_noise_uniform(r->seed, r->counter++); }

#ifdef __cplusplus
}
#endif
#endif
