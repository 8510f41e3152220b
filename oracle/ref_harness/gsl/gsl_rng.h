/* Stand-in for GSL's random-number interface (GSL is not installed here).
 * The reference allocates a generator unconditionally (FOF.c:41-42) but only
 * draws from it when subsampling is on (FOF.c:209,251).  The harness never
 * enables subsampling; drawing aborts so a silent wrong answer is impossible. */
#ifndef CMH_REF_HARNESS_GSL_RNG_H
#define CMH_REF_HARNESS_GSL_RNG_H
#ifdef __cplusplus
extern "C" {
#endif
typedef struct { int unused; } gsl_rng_type;
typedef struct { unsigned long state; } gsl_rng;
extern const gsl_rng_type *gsl_rng_ranlxd1;
gsl_rng *gsl_rng_alloc(const gsl_rng_type *t);
void gsl_rng_set(gsl_rng *r, unsigned long seed);
double gsl_rng_uniform(gsl_rng *r);
void gsl_rng_free(gsl_rng *r);
#ifdef __cplusplus
}
#endif
#endif
