/* Empty stand-in for GSL's <gsl/gsl_integration.h>: the reference includes it from
 * vars.h:8-12 but only uses it in the variable-linking-length build, which
 * does not compile (main.c:39 names an undeclared Nlink) and is not built. */
#ifndef CMH_REF_HARNESS_GSL_INTEGRATION_H
#define CMH_REF_HARNESS_GSL_INTEGRATION_H
#endif
