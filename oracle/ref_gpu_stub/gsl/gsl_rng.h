/* TEST INFRASTRUCTURE ONLY. Stand-in for GSL's random-number interface, which the reference uses
 * only to draw its initial inducing points (util.c:42-87). The reference's own CUDA build here
 * always receives T through --init-params, which overwrites those draws, so this stand-in
 * returns zeros. */
#ifndef GPL_REF_GSL_RNG_STUB
#define GPL_REF_GSL_RNG_STUB
typedef struct { int unused; } gsl_rng_type;
typedef struct { unsigned long seed; } gsl_rng;
static const gsl_rng_type gpl_stub_mt19937 = {0};
static const gsl_rng_type* gsl_rng_mt19937 = &gpl_stub_mt19937;
static inline void gsl_rng_env_setup(void) {}
static inline gsl_rng* gsl_rng_alloc(const gsl_rng_type* t) { (void)t; static gsl_rng r; return &r; }
static inline void gsl_rng_set(gsl_rng* r, unsigned long s) { r->seed = s; }
static inline void gsl_rng_free(gsl_rng* r) { (void)r; }
#endif
