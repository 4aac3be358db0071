/* Stand-in for gsl_ran_gaussian (see gsl_rng.h): sigma times the standard
 * normal draw at the generator's counter.  Test infrastructure for the
 * reference-source oracle build. */
#ifndef SHIM_GSL_RANDIST_H
#define SHIM_GSL_RANDIST_H
#include "gsl_rng.h"
#ifdef __cplusplus
extern "C" {
#endif
static inline double gsl_ran_gaussian(gsl_rng* r, double sigma) { return sigma * or_noise_gauss(r->seed, r->counter++); }
#ifdef __cplusplus
}
#endif
#endif
