/* oracle/shim/gsl/gsl_histogram.h -- opaque GSL type stand-ins so the reference's
 * data_types.h compiles (its stats path is off; test infrastructure only). */
#ifndef NS2D_SHIM_GSL_GSL_HISTOGRAM_H
#define NS2D_SHIM_GSL_GSL_HISTOGRAM_H
typedef struct gsl_histogram gsl_histogram;
typedef struct gsl_rstat_workspace gsl_rstat_workspace;
#endif
