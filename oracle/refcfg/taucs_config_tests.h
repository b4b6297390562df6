/* BLAS symbol convention of the OpenBLAS the oracle links (Fortran names with
 * a trailing underscore). */
#define TAUCS_BLAS_UNDERSCORE
