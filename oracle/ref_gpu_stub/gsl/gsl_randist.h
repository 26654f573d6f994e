/* TEST INFRASTRUCTURE ONLY. Stand-in for GSL's Gaussian draw (see gsl_rng.h here): zeros. */
#ifndef GPL_REF_GSL_RANDIST_STUB
#define GPL_REF_GSL_RANDIST_STUB
#include "gsl_rng.h"
static inline double gsl_ran_gaussian(const gsl_rng* r, double sigma) { (void)r; (void)sigma; return 0.0; }
#endif
